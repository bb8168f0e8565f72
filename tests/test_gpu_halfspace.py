"""Patterned half-spaces: a superstrate or substrate whose cells differ takes
its modes from the eigensolver, as the reference solves every layer type
(rcwa/RCWASolver.cpp:194-210); the first interface then takes the dense LU
route, generateHorizontalPlaneWave's vector is W_ref^-1 [px delta; py delta]
(rcwa/Layer.cpp:453-480) and the efficiencies take the half-spaces' values at
(0, 0) (rcwa/RCWASolver.cpp:1823-1830).  Against the oracle, which follows
the reference there, at 1e-9."""
import math

import numpy as np
import pytest

import oracle.rcwa_oracle as orc
import openrcwa_b200 as o

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _stack(nh, top, bottom, mu_bottom=None):
    # 2D: a rectangular pillar layer between half-spaces; `top` / `bottom`
    # pattern the superstrate / substrate with the same pillar
    g = np.linspace(-0.2, 0.2, 9)
    c = 0.5 * (g[1:] + g[:-1])
    ins = (np.abs(c[:, None] - 0.02) < 0.09) & (np.abs(c[None, :] + 0.01) < 0.13)
    sup = np.where(ins, 2.0, 1.0) if top else np.full((8, 8), 1.0)
    sub = np.where(ins, 4.0 + 0.2j, 2.25) if bottom else np.full((8, 8), 2.25)
    eps = np.array([sup, np.where(ins, 6.0 + 0.1j, 1.5), sub], dtype=complex)
    mu = None
    if mu_bottom is not None:
        mu = np.ones_like(eps)
        mu[2] = np.where(ins, mu_bottom, 1.0)
    thick = np.array([0.0, 0.2, 0.0])
    return o.Stack(nh, nh, g, g, eps, thick, mu=mu), g, eps, mu, thick


def _points(lams, thetas, phis, n_inc=1.0):
    pts, pxy = [], []
    for lam, th, ph in zip(lams, thetas, phis):
        k0 = 2 * math.pi / lam
        st = n_inc * math.sin(math.radians(th))
        pts.append((0, lam, k0 * st * math.cos(math.radians(ph)), k0 * st * math.sin(math.radians(ph))))
        c = math.cos(math.radians(th))
        pxy.append([(c * math.cos(math.radians(ph)), c * math.sin(math.radians(ph))),
                    (-math.sin(math.radians(ph)), math.cos(math.radians(ph)))])
    return np.array(pts), np.array(pxy, dtype=complex)


def _oracle(g, eps, mu, nh, thick, pts, pxy):
    out = []
    for p in range(len(pts)):
        s = orc.RCWASolver(nh, nh)
        for l in range(eps.shape[0]):
            s.addLayer(orc.OracleLayer(g, g, eps[l], mu=None if mu is None else mu[l]))
        s.setBlochWavevector(pts[p, 2], pts[p, 3])
        s.solve(pts[p, 1], list(range(eps.shape[0])), list(thick))
        k0 = 2 * math.pi / pts[p, 1]
        rows = [s.scatterPlaneWave(s.generateHorizontalPlaneWave(pxy[p, x, 0], pxy[p, x, 1], 0), 0,
                                   eps.shape[0] - 1, k0) for x in range(pxy.shape[1])]
        out.append((np.array([a.sum() for a, _ in rows]), np.array([b.sum() for _, b in rows]),
                    np.array([a for a, _ in rows]), np.array([b for _, b in rows])))
    return out


@pytest.mark.parametrize("top,bottom", [(False, True), (True, False), (True, True)])
def test_patterned_half_spaces_against_oracle(eng, top, bottom):
    nh = 3
    st, g, eps, mu, thick = _stack(nh, top, bottom)
    pts, pxy = _points([0.55, 0.7], [0.0, 30.0], [0.0, 20.0])
    R, T, REF, TRN, status = eng.solve_batch([st], pts, pxy)
    assert not np.any(status)
    for p, (Ro, To, REFo, TRNo) in enumerate(_oracle(g, eps, mu, nh, thick, pts, pxy)):
        assert np.max(np.abs(R[p] - Ro)) < 1e-9 and np.max(np.abs(T[p] - To)) < 1e-9
        assert np.max(np.abs(REF[p] - REFo)) < 1e-9 and np.max(np.abs(TRN[p] - TRNo)) < 1e-9
    Rm, Tm, _, _, sm = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
    assert not np.any(sm)
    assert np.max(np.abs(Rm - R)) < 1e-4 and np.max(np.abs(Tm - T)) < 1e-4


def test_patterned_magnetic_substrate_and_rescatter(eng):
    nh = 2
    st, g, eps, mu, thick = _stack(nh, False, True, mu_bottom=1.7 + 0.05j)
    pts, pxy = _points([0.6], [25.0], [40.0])
    plan = eng.plan([st], pts, pxy)
    plan.execute()
    R, T, REF, TRN, status = plan.results(orders=True)
    assert not np.any(status)
    Ro, To, _, _ = _oracle(g, eps, mu, nh, thick, pts, pxy)[0]
    assert np.max(np.abs(R[0] - Ro)) < 1e-9 and np.max(np.abs(T[0] - To)) < 1e-9
    # a new incident polarisation on the solved plan (rcwa_plan_rescatter)
    q = np.array([[[0.6, 0.3j], [0.2, -0.5]]], dtype=complex)
    plan.rescatter(q)
    R2, T2, _, _, s2 = plan.results()
    plan.close()
    Rq, Tq, _, _ = _oracle(g, eps, mu, nh, thick, pts, q)[0]
    assert not np.any(s2)
    assert np.max(np.abs(R2[0] - Rq)) < 1e-9 and np.max(np.abs(T2[0] - Tq)) < 1e-9
