"""Drop-in checks on the GPU.

* The reference's own sol/rcwa_bridge.cpp, unmodified, compiled against this
  engine's RCWASolver/Layer headers (oracle/_ref/rcwa_bridge_dropin, built by
  oracle/build_ref.sh), writes rcwa_efficiency.csv / rcwa_orders.csv that must
  agree with the oracle's rcwa_run.
* The header-only C++ API (tests/cpp/adapter_grating.cpp) reproduces the
  grating known answer.
"""
import csv
import os
import subprocess

import numpy as np
import pytest

from oracle.rcwa_oracle import OfdSetup, RcwaLayerSpec as L, rcwa_run
from tests import magnetic_cases

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DROPIN = os.path.join(ROOT, "oracle", "_ref", "rcwa_bridge_dropin")

OFD = """OpenRCWA 4 2
title = drop-in check
rcwa = 5 3.0e-7 2 3.0e-7
rcwalayer = 1.0 1.0 0.5 0
rcwalayer = 4.0 1.0 0.5 2.0e-7 0.1 0 0.7
rcwalayer = 2.25 2.25 0.5 0
rcwaincidence = 20 30
frequency1 = 4.3e14 7.5e14 4
end
"""


@pytest.mark.skipif(not os.path.exists(DROPIN), reason="oracle/_ref not built (oracle/build_ref.sh)")
def test_reference_bridge_unmodified_on_engine(tmp_path):
    (tmp_path / "in.ofd").write_text(OFD)
    out = subprocess.run([DROPIN, "in.ofd"], cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    rows = list(csv.DictReader(open(tmp_path / "rcwa_efficiency.csv")))
    setup = OfdSetup(nHx=5, period_x=3e-7, nHy=2, period_y=3e-7,
                     layers=[L(1, 1, .5, 0), L(4, 1, .5, 2e-7, 0.1, 0, 0.7), L(2.25, 2.25, .5, 0)],
                     freqs=[4.3e14 + k * 0.8e14 for k in range(5)], theta=20.0, phi=30.0)
    ref = rcwa_run(setup)
    assert len(rows) == len(ref)
    for row, r in zip(rows, ref):
        got = np.array([float(row["R_TE"]), float(row["T_TE"]), float(row["R_TM"]), float(row["T_TM"])])
        want = np.array([r["R"][0], r["T"][0], r["R"][1], r["T"][1]])
        assert np.max(np.abs(got - want)) < 2e-8, (got, want)
    orders = list(csv.DictReader(open(tmp_path / "rcwa_orders.csv")))
    assert len(orders) > 0
    for o in orders:
        f = [i for i, r in enumerate(ref) if abs(r["freq"] - float(o["frequency[Hz]"])) < 1e3][0]
        pol = 0 if o["pol"] == "TE" else 1
        k = (int(o["m"]) + 5) * 5 + (int(o["n"]) + 2)
        assert abs(float(o["R"]) - ref[f]["ordR"][pol][k]) < 2e-8
        assert abs(float(o["T"]) - ref[f]["ordT"][pol][k]) < 2e-8


def test_cpp_api_adapter(tmp_path):
    exe = tmp_path / "adapter_grating"
    lib = os.path.join(ROOT, "openrcwa_b200", "lib")
    subprocess.run(["g++", "-std=c++17", "-O1", "-DRCWA_B200_NO_EIGEN", "-I",
                    os.path.join(ROOT, "include", "openrcwa_b200"),
                    os.path.join(ROOT, "tests", "cpp", "adapter_grating.cpp"), "-L", lib, "-lrcwa_b200",
                    f"-Wl,-rpath,{lib}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    lines = out.stdout.strip().splitlines()
    vals = [list(map(float, ln.split())) for ln in lines[:2]]
    ref = rcwa_run(OfdSetup(nHx=5, period_x=3e-7, layers=[L(1, 1, .5, 0), L(4, 1, .5, 2e-7), L(2.25, 2.25, .5, 0)],
                            freqs=[6.5e14]))[0]
    # Rud() / Tdd(): against the oracle's cascade matrices in field space
    # (W_top Rud W_top^-1, W_bottom Tdd W_top^-1), which does not depend on
    # the basis LAPACK picks inside the half-spaces' degenerate eigenspaces
    rows, cols = map(int, lines[2].split())
    assert rows == cols == 22
    m = np.array([list(map(float, ln.split())) for ln in lines[3:3 + rows * cols]]).reshape(rows, cols, 4)
    Rud, Tdd = m[..., 0] + 1j * m[..., 1], m[..., 2] + 1j * m[..., 3]
    from oracle.rcwa_oracle import OracleLayer, RCWASolver
    sol = RCWASolver(5, 0)
    cx, cy = np.array([0, 1.5e-7, 3e-7]), np.array([0, 3e-7])
    for e in ([1, 1], [4, 1], [2.25, 2.25]):
        sol.addLayer(OracleLayer(cx, cy, np.array([e], dtype=complex)))
    sol.solve(2.99792458e8 / 6.5e14, [0, 1, 2], [0, 2e-7, 0])
    Wt, Wb = sol.sol[0].W, sol.sol[2].W
    Rf = Wt @ sol.Rud @ np.linalg.inv(Wt)
    Tf = Wb @ sol.Tdd @ np.linalg.inv(Wt)
    assert np.max(np.abs(Rud - Rf)) < 1e-9 * max(1.0, np.abs(Rf).max())
    assert np.max(np.abs(Tdd - Tf)) < 1e-9 * max(1.0, np.abs(Tf).max())
    assert abs(vals[0][0] - ref["R"][0]) < 1e-9 and abs(vals[1][0] - ref["R"][1]) < 1e-9
    assert abs(vals[0][1] - ref["T"][0]) < 1e-9 and abs(vals[1][1] - ref["T"][1]) < 1e-9
    assert abs(vals[0][0] - 0.138130) < 1e-6 and abs(vals[1][0] - 0.204841) < 1e-6


DRIVER = os.path.join(ROOT, "oracle", "_ref", "rcwa_driver_dropin")

# .orcwa inputs for the reference's orcwa_rcwa (rcwa/RCWAInput.cpp keys):
# a square lattice of dielectric pillars (z cylinders) on a glass substrate at
# normal incidence, a lossy, dispersive sphere above a slab at oblique
# incidence with circular polarisation, magnetic pillars with magnetic loss
# on a magnetic substrate, and the reference's magnetically lossy slab
# (material_mu)
ORCWA = {
    "magnetic_pillars": magnetic_cases.PILLARS,
    "magnetic_slab": magnetic_cases.slab("material = 1 4.0 0 1.0 0\nmaterial_mu = 2 4.0 0.5\n"),
    # pillars that run through the substrate slab to the bottom of the
    # domain: the transmission half-space is patterned
    "patterned_substrate": """OpenRCWA 4 2
title = drop-in check: pillars through the substrate
xmesh = -2.0e-07 20 2.0e-07
ymesh = -2.0e-07 20 2.0e-07
zmesh = -5e-07 10 -1.5e-07 10 0.0 10 4e-07
material = 1 2.25 0 1 0
material = 1 6.0 0 1 0
geometry = 2 1 -2.0e-07 2.0e-07 -2.0e-07 2.0e-07 -5e-07 -1.5e-07
geometry = 3 1 -1.2e-07 1.2e-07 -1.0e-07 1.0e-07 -5e-07 0
planewave = 15 20 2
rcwaorder = 2 2
frequency1 = 4.0e14 5.0e14 1
end
""",
    "pillars": """OpenRCWA 4 2
title = drop-in check: pillar metasurface
xmesh = -2.0e-07 20 2.0e-07
ymesh = -2.0e-07 20 2.0e-07
zmesh = -5e-07 10 -1.5e-07 10 0.0 10 4e-07
material = 1 2.25 0 1 0
material = 1 6.0 0 1 0
geometry = 2 1 -2.0e-07 2.0e-07 -2.0e-07 2.0e-07 -5e-07 -1.5e-07
geometry = 3 11 -1.2e-07 1.2e-07 -1.0e-07 1.0e-07 -1.5e-07 0
planewave = 0 0 1
rcwaorder = 3 3
frequency1 = 3.6e14 5.6e14 4
end
""",
    "sphere": """OpenRCWA 4 2
title = drop-in check: sphere, oblique circular incidence
xmesh = -2.5e-07 20 2.5e-07
ymesh = -2.0e-07 20 2.0e-07
zmesh = -4e-07 10 -1.2e-07 10 2.0e-07 10 5e-07
material = 1 2.1 0 1 0
material = 1 3.0 0 1 0
material_dispersion = 3 2.0 3.0e15 5.0e13 4.5e15
geometry = 2 1 -2.5e-07 2.5e-07 -2.0e-07 2.0e-07 -4e-07 -1.2e-07
geometry = 3 2 -1.5e-07 1.5e-07 -1.2e-07 1.2e-07 -1.2e-07 1.8e-07
planewave = 25 30 4
rcwaorder = 2 2
frequency1 = 4.0e14 5.0e14 2
end
""",
}


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("case", sorted(ORCWA))
def test_reference_driver_unmodified_on_engine(tmp_path, case):
    # the reference's rcwa/RCWADriver.cpp, rcwa/RCWAInput.cpp and
    # src/rcwa_Main.cpp, unmodified, on the engine's adapters: the verbose CSV
    # (8 significant digits) against the oracle's restatement of the driver
    from oracle import driver_oracle
    (tmp_path / "in.orcwa").write_text(ORCWA[case])
    out = subprocess.run([DRIVER, "-v", "-o", "out.csv", "in.orcwa"], cwd=tmp_path, capture_output=True, text=True,
                         timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    rows = [list(map(float, ln.split(","))) for ln in open(tmp_path / "out.csv") if not ln.startswith("#")]
    ref = driver_oracle.run(ORCWA[case])
    assert len(rows) == len(ref)
    for row, r in zip(rows, ref):
        nord = r["REF"].size
        assert abs(row[0] - r["lambda"]) < 1e-7 * r["lambda"]
        # the CSV holds 8 significant digits: compare to that precision
        got = np.array(row[1:5])
        want = np.array([r["R"], r["T"], r["A"], r["R"] + r["T"]])
        assert np.all(np.abs(got - want) < 2e-8 * np.maximum(1.0, 5 * np.abs(want))), (got, want)
        for col, ref_v in ((row[5:5 + nord], r["REF"]), (row[5 + nord:5 + 2 * nord], r["TRN"])):
            assert np.all(np.abs(np.array(col) - ref_v) < 2e-8 * np.maximum(1.0, 5 * np.abs(ref_v)))
