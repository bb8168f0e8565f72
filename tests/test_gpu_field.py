"""Fields inside a solved stack (rcwa_plan_field): the mode amplitudes of
RCWASolver::evaluateIntermediateField (rcwa/RCWASolver.cpp:1505-1644) and the
slices of saveFieldImage (:707-1012) against the oracle's restatement, the
continuity of the tangential fields across an interior interface at a size the
oracle does not reach, and the unmodified driver's field CSV."""
import math
import os
import subprocess

import numpy as np
import pytest

import oracle.rcwa_oracle as orc
import openrcwa_b200 as o

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "oracle", "_ref", "rcwa_driver_dropin")


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _grating_1d():
    cx, cy = np.array([0.0, 0.15, 0.5]), np.array([0.0, 0.5])
    eps = np.array([[[1.0, 1.0]], [[4.0 + 0.1j, 1.5]], [[2.0, 3.0]], [[2.25, 2.25]]], dtype=complex)
    return cx, cy, eps, np.array([0.0, 0.2, 0.3, 0.0])


def _pillars_2d(top_patterned=False):
    g = np.linspace(-0.2, 0.2, 9)
    c = 0.5 * (g[1:] + g[:-1])
    ins = (np.abs(c[:, None] - 0.02) < 0.09) & (np.abs(c[None, :] + 0.01) < 0.13)
    sup = np.where(ins, 1.8, 1.0) if top_patterned else np.full((8, 8), 1.0)
    eps = np.array([sup, np.where(ins, 6.0 + 0.1j, 1.5), np.where(ins, 2.0, 3.5 + 0.05j), np.full((8, 8), 2.25)],
                   dtype=complex)
    return g, g, eps, np.array([0.0, 0.15, 0.1, 0.0])


def _oracle_solver(cx, cy, eps, nHx, nHy, thick, lam, kx0, ky0):
    s = orc.RCWASolver(nHx, nHy)
    for e in eps:
        s.addLayer(orc.OracleLayer(cx, cy, e))
    s.setBlochWavevector(kx0, ky0)
    s.solve(lam, list(range(len(eps))), list(thick))
    return s


def _case(eng, cx, cy, eps, nHx, nHy, thick, lam, th, ph, px, py):
    k0 = 2 * math.pi / lam
    kx0 = k0 * math.sin(math.radians(th)) * math.cos(math.radians(ph))
    ky0 = k0 * math.sin(math.radians(th)) * math.sin(math.radians(ph))
    st = o.Stack(nHx, nHy, cx, cy, eps, thick)
    plan = eng.plan([st], np.array([[0, lam, kx0, ky0]]), np.array([[[px, py]]], dtype=complex))
    plan.execute()
    s = _oracle_solver(cx, cy, eps, nHx, nHy, thick, lam, kx0, ky0)
    c = s.generateHorizontalPlaneWave(px, py, 0)
    inp = [(i, v) for i, v in enumerate(c) if abs(v) > 1e-14]
    return plan, s, inp


@pytest.mark.parametrize("component", range(6))
def test_grating_xz_slices_against_oracle(eng, component):
    cx, cy, eps, thick = _grating_1d()
    plan, s, inp = _case(eng, cx, cy, eps, 5, 0, thick, 0.6, 17.0, 0.0, math.cos(math.radians(17.0)), 0.4j)
    f = plan.field(0, math.cos(math.radians(17.0)), 0.4j, 1, 0.1, component, nres1=64)
    plan.close()
    fo = s.fieldSlice(1, 0.1, component, inp, [0, 1, 2, 3], list(thick), nRes1=64)
    assert f.shape == fo.shape
    assert np.max(np.abs(f - fo)) <= 1e-9 * max(1.0, np.max(np.abs(fo)))


@pytest.mark.parametrize("slice_,coord,component", [(0, 0.2, 0), (0, 0.05, 2), (0, 0.2, 5), (2, -0.03, 4),
                                                    (1, 0.07, 3)])
@pytest.mark.parametrize("top_patterned", [False, True])
def test_pillar_slices_against_oracle(eng, slice_, coord, component, top_patterned):
    cx, cy, eps, thick = _pillars_2d(top_patterned)
    px, py = 0.8 * math.cos(math.radians(25)), 0.6j
    plan, s, inp = _case(eng, cx, cy, eps, 3, 3, thick, 0.55, 25.0, 35.0, px, py)
    f = plan.field(0, px, py, slice_, coord, component, nres1=40)
    plan.close()
    fo = s.fieldSlice(slice_, coord, component, inp, [0, 1, 2, 3], list(thick), nRes1=40)
    assert f.shape == fo.shape
    assert np.max(np.abs(f - fo)) <= 1e-9 * max(1.0, np.max(np.abs(fo)))


def test_tangential_fields_are_continuous_at_a_large_order(eng):
    # Nx = Ny = 9 (n = 722): Ex, Ey, Hx, Hy just above and below the interface
    # between the two interior layers (depth 0.15) agree
    cx, cy, eps, thick = _pillars_2d()
    lam, th, ph = 0.6, 20.0, 10.0
    k0 = 2 * math.pi / lam
    pts = np.array([[0, lam, k0 * math.sin(math.radians(th)) * math.cos(math.radians(ph)),
                     k0 * math.sin(math.radians(th)) * math.sin(math.radians(ph))]])
    plan = eng.plan([o.Stack(9, 9, cx, cy, eps, thick)], pts, np.array([[[0.7, 0.5]]], dtype=complex))
    plan.execute()
    for comp in (0, 1, 3, 4):
        above = plan.field(0, 0.7, 0.5, 0, 0.15 - 1e-9, comp, nres1=32)
        below = plan.field(0, 0.7, 0.5, 0, 0.15 + 1e-9, comp, nres1=32)
        assert np.max(np.abs(above - below)) < 1e-6 * np.max(np.abs(above)), comp
    plan.close()


ORCWA_FIELD = """OpenRCWA 4 2
title = drop-in check: field slice
xmesh = -2.0e-07 20 2.0e-07
ymesh = -2.0e-07 20 2.0e-07
zmesh = -5e-07 10 -1.5e-07 10 0.0 10 4e-07
material = 1 2.25 0 1 0
material = 1 6.0 0 1 0
geometry = 2 1 -2.0e-07 2.0e-07 -2.0e-07 2.0e-07 -5e-07 -1.5e-07
geometry = 3 1 -1.2e-07 1.2e-07 -1.0e-07 1.0e-07 -1.5e-07 0
planewave = 20 30 1
rcwaorder = 2 2
frequency1 = 4.0e14 5.0e14 1
end
"""


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("component,slice_,coord,opt", [("Ex", "xz", "0.05", "re"), ("Hz", "yz", "-0.02", "mod"),
                                                        ("Ez", "xz", "0.0", "im")])
def test_driver_field_csv(tmp_path, component, slice_, coord, opt):
    from oracle import driver_oracle
    (tmp_path / "in.orcwa").write_text(ORCWA_FIELD)
    out = subprocess.run([DRIVER, "-o", "out.csv", "-field", component, "-slice", slice_, "-scoord", coord,
                          "-sopt", opt, "-fieldout", "f.csv", "in.orcwa"], cwd=tmp_path, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    got = np.array([[float(v) for v in ln.split(",")] for ln in open(tmp_path / "f.csv") if ln.strip()])
    comp = ["Ex", "Ey", "Ez", "Hx", "Hy", "Hz"].index(component)
    sl = {"xy": 0, "xz": 1, "yz": 2}[slice_]
    want = driver_oracle.run(ORCWA_FIELD, field=(comp, sl, float(coord), {"mod": 0, "re": 1, "im": 2}[opt]))[0]["field"]
    assert got.shape == want.shape
    # 8 significant digits in the CSV
    assert np.max(np.abs(got - want)) <= 2e-8 * max(1.0, 5 * np.max(np.abs(want)))


@pytest.mark.skipif(not os.path.exists(DRIVER), reason="oracle/_ref not built (oracle/build_ref.sh)")
@pytest.mark.parametrize("slice_,coord", [("xz", "0.05"), ("xy", "0.07")])
def test_driver_device_csv(tmp_path, slice_, coord):
    # saveDeviceImage through the adapter: the permittivity of the interior
    # layers on the slice, against the driver oracle's restatement
    from oracle import driver_oracle
    (tmp_path / "in.orcwa").write_text(ORCWA_FIELD)
    out = subprocess.run([DRIVER, "-o", "out.csv", "-device", "-slice", slice_, "-scoord", coord, "-deviceout",
                          "d.csv", "in.orcwa"], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stdout + out.stderr
    got = np.array([[float(v) for v in ln.split(",")] for ln in open(tmp_path / "d.csv") if ln.strip()])
    sl = {"xy": 0, "xz": 1, "yz": 2}[slice_]
    want = driver_oracle.run(ORCWA_FIELD, device=(sl, float(coord)))[0]["device"]
    assert got.shape == want.shape
    assert np.max(np.abs(got - want)) <= 1e-7 * np.max(np.abs(want))
