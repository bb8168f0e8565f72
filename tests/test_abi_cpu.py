"""C ABI and host-side checks that need no GPU."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "rcwa_b200.h")


def _lib():
    from openrcwa_b200 import build
    if not os.path.exists(build.LIB):
        build.build()
    import openrcwa_b200 as o
    return o, o.load()


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rcwa_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    o, lib = _lib()
    decl = declared_functions()
    assert len(decl) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", o.abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if " T " in l)
    missing = [d for d in decl if d not in exported]
    assert not missing, missing
    assert set(decl) <= set(o.EXPORTS)
    for d in decl:
        getattr(lib, d)


def test_status_strings_and_argument_checks():
    o, lib = _lib()
    for code in range(10):
        assert lib.rcwa_status_string(code)
    h = ctypes.c_void_p()
    rc = lib.rcwa_engine_create(0, ctypes.byref(h))
    if rc == 0:
        lib.rcwa_engine_destroy(h)
        pytest.skip("a GPU is present")
    assert rc == o.abi.RCWA_ERR_NODEVICE
    assert lib.rcwa_engine_create(0, None) == o.abi.RCWA_ERR_INVALID
    assert lib.rcwa_plan_execute(None, None) == o.abi.RCWA_ERR_INVALID
    assert lib.rcwa_plan_rescatter(None, None) == o.abi.RCWA_ERR_INVALID
    assert lib.rcwa_zgeev_batched_noalloc(0, 1, None, None, None, None, None) == o.abi.RCWA_ERR_INVALID
    # the z-integrators reject a missing engine or missing samples before any device work
    null12 = [None] * 12
    assert lib.rcwa_rcwa_integrate(None, 4, 2, 1.0, 0.0, 1.0, *null12) == o.abi.RCWA_ERR_INVALID
    assert lib.rcwa_differential_integrate(None, 4, 2, 1.0, 0.0, 1.0, *null12) == o.abi.RCWA_ERR_INVALID
    assert lib.rcwa_redheffer_integrate(None, 4, 1.0, 0.0, 1.0, 1e-3, 100, o.abi.RCWA_SAMPLER(),
                                        None, *([None] * 10), None, None) == o.abi.RCWA_ERR_INVALID


def test_product_fails_loudly_without_its_library(monkeypatch):
    import openrcwa_b200.abi as abi
    monkeypatch.setattr(abi, "_lib", None)
    monkeypatch.setattr(abi, "LIB_PATH", "/nonexistent/librcwa_b200.so")
    with pytest.raises(RuntimeError):
        abi.load()


def test_c_header_is_plain_c():
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-fsyntax-only", "-x", "c", HEADER], check=True)


def test_cpp_adapters_compile_without_eigen():
    src = os.path.join(ROOT, "tests", "cpp", "adapter_grating.cpp")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-DRCWA_B200_NO_EIGEN", "-fsyntax-only",
                    "-I", os.path.join(ROOT, "include", "openrcwa_b200"), src], check=True)


def test_integrator_adapters_build_and_fail_softly_without_a_device(tmp_path):
    # the core/ integrator adapters with a LayerSampler-shaped sampler: they
    # compile without Eigen, link against the library, and with no device
    # report and leave their outputs empty, as the other adapters do
    o, lib = _lib()
    h = ctypes.c_void_p()
    if lib.rcwa_engine_create(0, ctypes.byref(h)) == 0:
        lib.rcwa_engine_destroy(h)
        pytest.skip("a GPU is present")
    src = os.path.join(ROOT, "tests", "cpp", "adapter_integrators.cpp")
    libdir = os.path.dirname(o.abi.LIB_PATH)
    exe = os.path.join(tmp_path, "adapter_integrators")
    inc = os.path.join(ROOT, "include", "openrcwa_b200")
    subprocess.run(["g++", "-std=c++17", "-Wall", "-DRCWA_B200_NO_EIGEN", "-I", inc, src, "-L", libdir, "-lrcwa_b200",
                    "-Wl,-rpath," + libdir, "-o", exe], check=True)
    out = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0
    assert out.stdout.split() == ["0", "0", "0", "0"]
    assert "engine unavailable" in out.stderr


# where the reference sources are mounted: the drop-in recipe knows (REF env var)
REF = subprocess.run(["sh", os.path.join(ROOT, "oracle", "build_ref.sh"), "--print-ref"], capture_output=True,
                     text=True).stdout.strip()


@pytest.mark.skipif(not os.path.exists(os.path.join(REF, "sol", "rcwa_bridge.cpp")),
                    reason="reference sources not mounted")
def test_reference_bridge_compiles_unmodified_against_adapters(tmp_path):
    subprocess.run(["g++", "-std=c++17", "-DRCWA_B200_NO_EIGEN", "-c", os.path.join(REF, "sol", "rcwa_bridge.cpp"),
                    "-I", os.path.join(ROOT, "include", "openrcwa_b200"), "-I", os.path.join(REF, "include"),
                    "-o", str(tmp_path / "b.o")], check=True)


def test_product_code_never_touches_the_oracle():
    for base in ("openrcwa_b200", "include"):
        for dirpath, _, files in os.walk(os.path.join(ROOT, base)):
            for f in files:
                if f.endswith((".py", ".cu", ".cuh", ".h", ".hpp", ".cpp")):
                    text = open(os.path.join(dirpath, f), errors="ignore").read()
                    assert "oracle" not in text.lower(), os.path.join(dirpath, f)


def test_workload_shapes():
    from openrcwa_b200 import workloads
    st, pts, pxy = workloads.pillars_2d(seed=0)
    assert st[0].N == 441 and pts.shape == (2048, 4) and pxy.shape == (2048, 2, 2)
    assert st[0].eps.shape[0] == 7 and np.all(st[0].thickness[1:-1] > 0)
    st, pts, pxy = workloads.grating_1d()
    assert st[0].N == 11 and pts.shape == (16, 4)
    starts = {workloads.shard_start(r, 4, 32, k) for r in range(4) for k in range(3)}
    assert len(starts) == 12


def test_uneven_workload_distribution():
    # the uneven batch: orders, layer counts and materials span their ranges
    from openrcwa_b200 import workloads
    st, pts, pxy = workloads.uneven_batch(seed=0, n_instances=400)
    assert len(st) == 400 and pts.shape == (400, 4) and pxy.shape == (400, 2, 2)
    nh = np.array([s.nHx for s in st])
    assert nh.min() == 3 and nh.max() == 15 and np.all(np.array([s.nHy for s in st]) == nh)
    layers = np.array([s.eps.shape[0] - 2 for s in st])
    assert layers.min() == 1 and layers.max() == 10
    lam = pts[:, 1]
    assert lam.min() >= 400e-9 and lam.max() <= 1000e-9
    theta = np.degrees(np.arcsin(pts[:, 2] / (2 * np.pi / lam)))
    assert theta.min() >= 0 and theta.max() <= 70 and np.all(pts[:, 3] == 0)
    eps_in = np.concatenate([s.eps[1:-1].reshape(s.eps.shape[0] - 2, -1)[:, 0] for s in st])
    # half the layers are drawn as lossy metal, the rest from the Lorentz pole
    # (which is also negative above its resonance); all are passive
    box = (eps_in.real >= -30) & (eps_in.real <= -5) & (eps_in.imag >= 0.5) & (eps_in.imag <= 3)
    assert 0.3 < box.mean() < 0.7
    assert np.all(np.isfinite(eps_in)) and np.all(eps_in.imag >= 0)
    thick = np.concatenate([s.thickness[1:-1] for s in st])
    assert thick.min() >= 20e-9 and thick.max() <= 500e-9


def test_surrogate_sampler_ranges():
    from openrcwa_b200 import surrogate
    P = surrogate.sample(5000, np.random.default_rng(0))
    assert P.shape == (5000, len(surrogate.PARAMS))
    lo, hi = surrogate.RANGES[:, 0], surrogate.RANGES[:, 1]
    assert np.all(P >= lo) and np.all(P <= hi)


def test_circular_pillar_tables_match_the_oracle_closed_form():
    import oracle.rcwa_oracle as ro
    from openrcwa_b200 import workloads
    L, R = 4e-7, 1.3e-7
    F = workloads.disk_laurent_table(L, L, R, (0.5 * L, 0.5 * L), complex(2.1, 0.01), 1.0, 6)
    Fo = ro.circle_fourier2d(L, L, R, (0.5 * L, 0.5 * L), complex(2.1, 0.01), 1.0, 13, 13)
    assert F.shape == (25, 25) and np.max(np.abs(F - Fo)) < 1e-14
    st, pts, pxy = workloads.circular_pillars(seed=0, nH=3, n_lambda=4, n_layers=5)
    assert st[0].f2d.shape == (5, 13, 13) and pts.shape == (4, 4) and st[0].N == 49
