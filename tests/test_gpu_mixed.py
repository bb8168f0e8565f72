"""The mixed-precision solve (cascade GEMMs, modal V products and the updates
between the 128-wide blocks of the interface and tau factorisations and
solves in 3xTF32 on tcgen05; eigensolve, LU panels and triangles in FP64):
every efficiency within 1e-4 of the FP64 oracle (the mixed-precision
accuracy bound), and the FP64 plan on the same inputs within 1e-9."""
import numpy as np
import pytest

import oracle.rcwa_oracle as orc
from oracle.rcwa_oracle import OfdSetup, RcwaLayerSpec as L

import openrcwa_b200 as o

pytestmark = pytest.mark.gpu

TOL_MIXED = 1e-4


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _setup(seed, nh):
    rng = np.random.default_rng(seed)
    layers = [L(1, 1, .5, 0)]
    for _ in range(3):
        layers.append(L(rng.uniform(2, 12), 1.0, rng.uniform(.2, .8), rng.uniform(50e-9, 300e-9),
                        rng.uniform(0, .5), 0.0, rng.uniform(.2, .8)))
    layers.append(L(2.25, 2.25, .5, 0))
    return OfdSetup(nHx=nh, period_x=4e-7, nHy=nh, period_y=4e-7, layers=layers,
                    freqs=orc.C0 / rng.uniform(400e-9, 800e-9, 2), theta=rng.uniform(0, 60), phi=rng.uniform(0, 90))


def _stack_points(s):
    xe = orc.common_edges(s.period_x, [l.fill for l in s.layers])
    ye = orc.common_edges(s.py(), [l.fill_y for l in s.layers])
    eps = np.array([orc.make_layer_eps(l, complex(l.eps1, l.eps1i), complex(l.eps2, l.eps2i), xe, ye)
                    for l in s.layers])
    st = o.Stack(s.nHx, s.nHy, xe, ye, eps, [0] + [l.thickness for l in s.layers[1:-1]] + [0])
    ref = orc.rcwa_run(s)
    pts = [(0, r["lam"], r["kx0"], r["ky0"]) for r in ref]
    te, tm = orc.polarisation_vectors(s.theta, s.phi)
    pxy = np.array([[te, tm]] * len(pts), dtype=complex)
    return st, np.array(pts), pxy, ref


@pytest.mark.parametrize("seed,nh", [(0, 3), (1, 5), (2, 7)])
def test_mixed_within_1e4_of_oracle(eng, seed, nh):
    s = _setup(seed, nh)
    st, pts, pxy, ref = _stack_points(s)
    Rm, Tm, REFm, TRNm, stm = eng.solve_batch([st], pts, pxy, precision=o.RCWA_PREC_MIXED)
    R6, T6, _, _, st6 = eng.solve_batch([st], pts, pxy, precision=o.RCWA_PREC_FP64)
    assert not np.any(stm) and not np.any(st6)
    for p, r in enumerate(ref):
        assert np.max(np.abs(R6[p] - r["R"])) < 1e-9 and np.max(np.abs(T6[p] - r["T"])) < 1e-9
        assert np.max(np.abs(Rm[p] - r["R"])) < TOL_MIXED, (Rm[p], r["R"])
        assert np.max(np.abs(Tm[p] - r["T"])) < TOL_MIXED, (Tm[p], r["T"])
        assert np.max(np.abs(REFm[p] - r["REF"])) < TOL_MIXED
        assert np.max(np.abs(TRNm[p] - r["TRN"])) < TOL_MIXED


def test_mixed_lossless_energy(eng):
    # lossless layers: R + T = 1 to the mixed bound
    s = _setup(4, 5)
    for l in s.layers:
        l.eps1i = 0.0
        l.eps2i = 0.0
    st, pts, pxy, _ = _stack_points(s)
    R, T, _, _, status = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
    assert not np.any(status)
    assert np.max(np.abs(R + T - 1.0)) < TOL_MIXED


def test_mixed_keeps_fp64_products_for_metal(eng):
    # a stack with a metal layer: the mixed plan routes it to FP64 products,
    # so its results equal the FP64 plan's bit for bit
    from openrcwa_b200 import workloads
    st = workloads.rect_stack(4, 4, 4e-7, 4e-7, [(complex(-20.0, 1.5), 1.0, 0.5, 0.4, 2e-7),
                                                 (complex(4.0, 0.1), 1.0, 0.3, 0.7, 1e-7)])
    lam = 6e-7
    k0 = 2 * np.pi / lam
    pts = np.array([(0, lam, k0 * 0.3, 0.1 * k0)])
    pxy = np.array([[(0.0, 1.0), (1.0, 0.0)]], dtype=complex)
    Rm, Tm, _, _, sm = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
    R6, T6, _, _, s6 = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_FP64)
    assert not np.any(sm) and not np.any(s6)
    assert np.array_equal(Rm, R6) and np.array_equal(Tm, T6)
