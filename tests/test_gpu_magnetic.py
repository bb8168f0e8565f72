"""Magnetic layers on the engine (the permeability of rcwa_stack.mu): the
dense P and Q of the magnetic branch (rcwa/Layer.cpp:128-164,205-213), the
magnetic half-spaces and the mu terms of the efficiencies
(rcwa/RCWASolver.cpp:1826-1907), against the oracle at 1e-9, the reference's
magnetic Fresnel known answers, and duality at a size the oracle does not
reach."""
import math

import numpy as np
import pytest

import oracle.rcwa_oracle as orc
import openrcwa_b200 as o
from tests import magnetic_cases as mc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _oracle(cx, cy, eps, mu, nHx, nHy, thick, pts, pxy):
    out = []
    for p in range(len(pts)):
        s = orc.RCWASolver(nHx, nHy)
        for e, m in zip(eps, mu):
            s.addLayer(orc.OracleLayer(cx, cy, e, mu=m))
        s.setBlochWavevector(pts[p, 2], pts[p, 3])
        s.solve(pts[p, 1], list(range(len(eps))), list(thick))
        k0 = 2 * math.pi / pts[p, 1]
        rows = [s.scatterPlaneWave(s.generateHorizontalPlaneWave(pxy[p, x, 0], pxy[p, x, 1], 0), 0, len(eps) - 1, k0)
                for x in range(pxy.shape[1])]
        out.append((np.array([a.sum() for a, _ in rows]), np.array([b.sum() for _, b in rows]),
                    np.array([a for a, _ in rows]), np.array([b for _, b in rows])))
    return out


def _points(lams, thetas, phis):
    pts, pxy = [], []
    for lam, th, ph in zip(lams, thetas, phis):
        k0 = 2 * math.pi / lam
        st = math.sin(math.radians(th))
        pts.append((0, lam, k0 * st * math.cos(math.radians(ph)), k0 * st * math.sin(math.radians(ph))))
        c = math.cos(math.radians(th))
        tm = (c * math.cos(math.radians(ph)), c * math.sin(math.radians(ph)))
        te = (-math.sin(math.radians(ph)), math.cos(math.radians(ph)))
        pxy.append([tm, te])
    return np.array(pts), np.array(pxy, dtype=complex)


def _pillar_stack(nh):
    # 2D: a magnetic, magnetically lossy pillar in a magnetic film on a
    # magnetic substrate; air above
    g = np.linspace(0.0, 0.4, 9)
    ins = (np.abs(g[:-1, None] + 0.025 - 0.2) < 0.06) & (np.abs(g[None, :-1] + 0.025 - 0.2) < 0.11)
    e_pat = np.where(ins, 5.0 + 0.05j, 1.8)
    m_pat = np.where(ins, 2.0 + 0.1j, 1.2)
    eps = [np.full((8, 8), 1.0 + 0j), e_pat, np.full((8, 8), 3.0 + 0j), np.full((8, 8), 2.25 + 0j)]
    mu = [np.ones((8, 8), dtype=complex), m_pat, np.full((8, 8), 1.0 + 0j), np.full((8, 8), 1.5 + 0j)]
    thick = np.array([0.0, 0.15, 0.1, 0.0])
    st = o.Stack(nh, nh, g, g, np.array(eps), thick, mu=np.array(mu))
    return st, g, eps, mu, thick


@pytest.mark.parametrize("nh", [2, 4])
def test_magnetic_pillars_against_oracle(eng, nh):
    st, g, eps, mu, thick = _pillar_stack(nh)
    pts, pxy = _points([0.55, 0.7], [0.0, 25.0], [0.0, 30.0])
    R, T, REF, TRN, status = eng.solve_batch([st], pts, pxy)
    assert not np.any(status)
    for p, (Ro, To, REFo, TRNo) in enumerate(_oracle(g, g, eps, mu, nh, nh, thick, pts, pxy)):
        assert np.max(np.abs(R[p] - Ro)) < 1e-9 and np.max(np.abs(T[p] - To)) < 1e-9
        assert np.max(np.abs(REF[p] - REFo)) < 1e-9 and np.max(np.abs(TRN[p] - TRNo)) < 1e-9
    Rm, Tm, _, _, sm = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
    assert not np.any(sm)
    assert np.max(np.abs(Rm - R)) < 1e-4 and np.max(np.abs(Tm - T)) < 1e-4


def _interface(eps2, mu2, nh=4):
    cx, cy = np.array([0.0, 0.5]), np.array([0.0, 0.5])
    e = np.array([[[1.0]], [[eps2]]], dtype=complex)
    m = np.array([[[1.0]], [[mu2]]], dtype=complex)
    return o.Stack(nh, 0, cx, cy, e, np.zeros(2), mu=m)


def test_magnetic_fresnel_known_answers(eng):
    # tests/test_rcwa_input.cpp:2037-2089 of the reference: eps = mu = 4 is
    # impedance matched; the angle sweep and eps != mu follow the analytic
    # Fresnel reflectance; swapping eps and mu swaps TM and TE
    for (e2, m2) in ((4.0, 4.0), (2.25, 3.0), (3.0, 2.25)):
        thetas = [0.0, 30.0, 45.0, 60.0]
        pts, pxy = _points([0.6] * 4, thetas, [0.0] * 4)
        R, T, _, _, status = eng.solve_batch([_interface(e2, m2)], pts, pxy, orders=False)
        assert not np.any(status)
        assert np.max(np.abs(R + T - 1.0)) < 1e-12
        for k, th in enumerate(thetas):
            assert abs(R[k, 0] - mc.fresnel_r(th, e2, m2, 1)) < 1e-9
            assert abs(R[k, 1] - mc.fresnel_r(th, e2, m2, 2)) < 1e-9
        if e2 == m2:
            assert R[0, 0] < 1e-9


def test_duality_at_a_large_order(eng):
    # eps <-> mu everywhere exchanges TM and TE (n = 2 * 17^2 = 578)
    nh = 8
    st, g, eps, mu, thick = _pillar_stack(nh)
    dual = o.Stack(nh, nh, g, g, np.array(mu), thick, mu=np.array(eps))
    pts, pxy = _points([0.6], [20.0], [35.0])
    R1, T1, _, _, s1 = eng.solve_batch([st], pts, pxy, orders=False)
    R2, T2, _, _, s2 = eng.solve_batch([dual], pts, pxy, orders=False)
    assert not np.any(s1) and not np.any(s2)
    assert abs(R1[0, 0] - R2[0, 1]) < 1e-9 and abs(R1[0, 1] - R2[0, 0]) < 1e-9
    assert abs(T1[0, 0] - T2[0, 1]) < 1e-9 and abs(T1[0, 1] - T2[0, 0]) < 1e-9


def test_unit_mu_matches_no_mu(eng):
    st, g, eps, mu, thick = _pillar_stack(3)
    a = o.Stack(3, 3, g, g, np.array(eps), thick)
    b = o.Stack(3, 3, g, g, np.array(eps), thick, mu=np.ones_like(np.array(eps)))
    pts, pxy = _points([0.6], [10.0], [0.0])
    Ra, Ta, _, _, _ = eng.solve_batch([a], pts, pxy, orders=False)
    Rb, Tb, _, _, _ = eng.solve_batch([b], pts, pxy, orders=False)
    assert np.array_equal(Ra, Rb) and np.array_equal(Ta, Tb)


def test_bad_permeability_is_rejected(eng):
    st, g, eps, mu, thick = _pillar_stack(2)
    pts, pxy = _points([0.6], [0.0], [0.0])
    m = np.array(mu)
    m[1, 0, 0] = complex(float("nan"), 0.0)
    with pytest.raises(o.RcwaError) as ex:
        eng.solve_batch([o.Stack(2, 2, g, g, np.array(eps), thick, mu=m)], pts, pxy)
    assert ex.value.code == o.abi.RCWA_ERR_NONFINITE
    m = np.array(mu)
    m[1, 0, 0] = 0.0
    with pytest.raises(o.RcwaError) as ex:
        eng.solve_batch([o.Stack(2, 2, g, g, np.array(eps), thick, mu=m)], pts, pxy)
    assert ex.value.code == o.abi.RCWA_ERR_INVALID
