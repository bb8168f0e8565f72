"""Parity of the CUDA engine (through the C ABI) with the CPU oracle.

Tolerances: 1e-9 absolute on every efficiency (the plain FP64 contract), 1e-12
relative on convolution matrices, eigen-residuals below 1e-10.
"""
import math

import numpy as np
import pytest

import oracle.rcwa_oracle as orc
from oracle.rcwa_oracle import OfdSetup, RcwaLayerSpec as L, RcwaPole

pytestmark = pytest.mark.gpu

TOL_RT = 1e-9


@pytest.fixture(scope="module")
def eng():
    import openrcwa_b200 as o
    e = o.Engine(0)
    yield e
    e.close()


def rand_grid(rng, n_x, n_y, period_x=1.0, period_y=1.0):
    cx = np.concatenate([[0.0], np.sort(rng.uniform(0, period_x, n_x - 1)), [period_x]])
    cy = np.concatenate([[0.0], np.sort(rng.uniform(0, period_y, n_y - 1)), [period_y]])
    eps = rng.uniform(1, 6, (n_y, n_x)) + 1j * rng.uniform(0, 0.5, (n_y, n_x))
    return cx, cy, eps


def test_fourier1d(eng):
    rng = np.random.default_rng(1)
    x = np.concatenate([[0.0], np.sort(rng.uniform(0, 2.0, 4)), [2.0]])
    f = rng.normal(size=5) + 1j * rng.normal(size=5)
    for M in (1, 5, 21):
        got = eng.fourier1d(x, 2.0, f, M)
        ref = orc.fourier1d(x, 2.0, f, M)
        assert np.max(np.abs(got - ref)) < 1e-13 * max(1, np.max(np.abs(ref)))


@pytest.mark.parametrize("nx,ny,cells", [(3, 3, (2, 2)), (11, 1, (2, 1)), (5, 7, (3, 4)), (9, 9, (4, 3))])
def test_fourier2d_all_rules(eng, nx, ny, cells):
    rng = np.random.default_rng(nx * 100 + ny)
    cx, cy, eps = rand_grid(rng, cells[0], cells[1], 1.3, 0.7)
    for opt in (orc.ContinuousXY, orc.DiscontinuousX, orc.DiscontinuousY):
        got = eng.fourier2d(cx, cy, eps, nx, ny, opt)
        ref = orc.fourier2d(cx, cy, eps, nx, ny, opt)
        assert np.max(np.abs(got - ref)) < 1e-12 * np.max(np.abs(ref)), opt


def _match_eigs(a, b):
    """max distance after greedy nearest matching of two eigenvalue sets."""
    b = list(b)
    worst = 0.0
    for z in sorted(a, key=lambda t: -abs(t)):
        d = [abs(z - w) for w in b]
        k = int(np.argmin(d))
        worst = max(worst, d[k] / max(1.0, abs(z)))
        b.pop(k)
    return worst


@pytest.mark.parametrize("n", [1, 2, 3, 7, 22, 33, 63, 64, 65, 100, 130, 257])
def test_zgeev_random(eng, n):
    rng = np.random.default_rng(n)
    A = rng.normal(size=(3, n, n)) + 1j * rng.normal(size=(3, n, n))
    w, VR, info = eng.zgeev(A)
    assert np.all(info == 0)
    for b in range(3):
        nA = np.abs(A[b]).max()
        res = np.abs(A[b] @ VR[b] - VR[b] * w[b][None, :]).max() / nA
        assert res < 1e-12 * n, res
        assert np.allclose(np.linalg.norm(VR[b], axis=0), 1.0, atol=1e-13)
        assert _match_eigs(w[b], np.linalg.eigvals(A[b])) < 1e-10


def test_zgeev_degenerate(eng):
    # exactly repeated eigenvalues with a full eigenbasis (the +-m structure)
    rng = np.random.default_rng(7)
    n = 24
    S = rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))
    d = np.repeat(rng.normal(size=n // 2) + 1j * rng.normal(size=n // 2), 2)
    A = S @ np.diag(d) @ np.linalg.inv(S)
    w, VR, info = eng.zgeev(A)
    assert info[0] == 0
    res = np.abs(A @ VR[0] - VR[0] * w[0][None, :]).max() / np.abs(A).max()
    assert res < 1e-9
    assert np.linalg.cond(VR[0]) < 1e8


def test_layer_solve_vs_oracle(eng):
    rng = np.random.default_rng(3)
    nx, ny = 5, 3
    cx, cy, eps = rand_grid(rng, 3, 2, 0.5, 0.4)
    lam = 0.6
    k0 = 2 * math.pi / lam
    alpha, beta = orc.alpha_beta(nx, ny, 0.5, 0.4, 0.3 * k0, 0.1 * k0)
    W, V, g, ev = eng.layer_solve(cx, cy, eps, nx, ny, alpha, beta, lam)
    sol = orc.layer_solve(cx, cy, eps, alpha, beta, lam, nx, ny, keep=True)
    PQ = sol.P @ sol.Q
    assert _match_eigs(ev, sol.eigenvalues) < 1e-11
    res = np.abs(PQ @ W - W * ev[None, :]).max() / np.abs(PQ).max()
    assert res < 1e-11
    keff = orc.gamma_sqrt(ev)
    assert np.allclose(g, keff / k0, rtol=1e-12, atol=0)
    Vref = (sol.Q @ W) / keff[None, :]
    assert np.abs(V - Vref).max() < 1e-11 * np.abs(Vref).max()


def _cmp_ofd(eng, setup, tol=TOL_RT):
    R, T, oR, oT, st = eng.ofd_solve(setup)
    assert np.all(st == 0), st
    ref = orc.rcwa_run(setup)
    for f, r in enumerate(ref):
        assert np.max(np.abs(R[f] - r["R"])) < tol, (f, R[f], r["R"])
        assert np.max(np.abs(T[f] - r["T"])) < tol, (f, T[f], r["T"])
        assert np.max(np.abs(oR[:, f, :] - r["ordR"])) < tol
        assert np.max(np.abs(oT[:, f, :] - r["ordT"])) < tol
    return R, T


GRATING = [L(1, 1, .5, 0), L(4, 1, .5, 2e-7), L(2.25, 2.25, .5, 0)]


def test_grating_cfg1_16_and_17_points(eng):
    # the metric's 16-point grid and the reference's 17-point frequency1 grid
    _cmp_ofd(eng, OfdSetup(nHx=5, period_x=3e-7, layers=GRATING, freqs=np.linspace(4.3e14, 7.5e14, 16)))
    R, T = _cmp_ofd(eng, OfdSetup(nHx=5, period_x=3e-7, layers=GRATING,
                                  freqs=[4.3e14 + k * 0.2e14 for k in range(17)]))
    assert abs(R[11, 0] - 0.138130) < 1e-6 and abs(R[11, 1] - 0.204841) < 1e-6
    assert np.all(np.abs(R + T - 1) < 1e-10)


@pytest.mark.parametrize("N,rte,rtm", [(12, 0.138187, 0.206747), (20, 0.138193, 0.206805)])
def test_grating_convergence_kat(eng, N, rte, rtm):
    R, T, _, _, st = eng.ofd_solve(OfdSetup(nHx=N, period_x=3e-7, layers=GRATING, freqs=[6.5e14]))
    assert abs(R[0, 0] - rte) < 1e-6 and abs(R[0, 1] - rtm) < 1e-6


def test_oblique_metal_drude_kats(eng):
    R, T = _cmp_ofd(eng, OfdSetup(nHx=3, period_x=3e-7, layers=[L(1, 1, .5, 0), L(2.25, 2.25, .5, 0)],
                                  freqs=[5e14], theta=56.30993247))
    assert abs(R[0, 0] - 0.147929) < 1e-6 and R[0, 1] < 1e-8
    R, T = _cmp_ofd(eng, OfdSetup(nHx=3, period_x=3e-7, freqs=[4.9966e14],
                                  layers=[L(1, 1, .5, 0), L(-17.74, -17.74, .5, 3e-8, .18, .18),
                                          L(2.25, 2.25, .5, 0)]))
    assert abs(R[0, 0] - 0.909420) < 1e-6 and abs(T[0, 0] - 0.084430) < 1e-6
    poles = [RcwaPole(1, 1, 1.0, 1.36e16, 3.0e13, 0.0), RcwaPole(1, 2, 1.0, 1.36e16, 3.0e13, 0.0)]
    _cmp_ofd(eng, OfdSetup(nHx=2, period_x=5e-7, layers=[L(1, 1, .5, 0), L(1, 1, .5, 3e-8), L(2.25, 2.25, .5, 0)],
                           freqs=[4e14 + k * 0.5e14 for k in range(7)], poles=poles))


def test_rect2d_symmetry(eng):
    R, T = _cmp_ofd(eng, OfdSetup(nHx=4, period_x=5e-7, nHy=4, period_y=5e-7,
                                  layers=[L(1, 1, .5, 0), L(2.25, 1, .6, 2e-7, 0, 0, .6), L(2.25, 2.25, .5, 0)],
                                  freqs=np.linspace(3.331e14, 4.835e14, 9)))
    assert np.all((R[:, 0] - R[:, 1]) ** 2 < 1e-12)
    assert np.all(((R + T) - 1) ** 2 < 1e-12)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_random_2d_conical_stacks(eng, seed):
    rng = np.random.default_rng(seed)
    nl = int(rng.integers(1, 4))
    layers = [L(1, 1, .5, 0)]
    for _ in range(nl):
        layers.append(L(rng.uniform(2, 12), 1.0, rng.uniform(.2, .8), rng.uniform(50e-9, 300e-9),
                        rng.uniform(0, .5), 0.0, rng.uniform(.2, .8)))
    layers.append(L(2.25, 2.25, .5, 0))
    setup = OfdSetup(nHx=3, period_x=4e-7, nHy=2, period_y=4e-7, layers=layers,
                     freqs=orc.C0 / rng.uniform(400e-9, 800e-9, 3), theta=rng.uniform(0, 60), phi=rng.uniform(0, 90))
    _cmp_ofd(eng, setup)


def test_batch_mixed_sizes_and_layer_counts(eng):
    import openrcwa_b200 as o
    rng = np.random.default_rng(11)
    stacks, setups = [], []
    for (nHx, nHy, nl) in [(2, 2, 1), (3, 1, 3), (2, 2, 2), (4, 0, 0)]:
        layers = [L(1, 1, .5, 0)] + [L(rng.uniform(2, 8), 1.0, rng.uniform(.2, .8), rng.uniform(5e-8, 3e-7),
                                       rng.uniform(0, .3), 0.0, rng.uniform(.3, .9)) for _ in range(nl)] + \
                 [L(2.25, 2.25, .5, 0)]
        s = OfdSetup(nHx=nHx, period_x=5e-7, nHy=nHy, period_y=4e-7, layers=layers, freqs=[5.5e14],
                     theta=25.0, phi=30.0)
        setups.append(s)
        xe = orc.common_edges(s.period_x, [l.fill for l in layers])
        ye = orc.common_edges(s.py(), [l.fill_y for l in layers])
        eps = np.array([orc.make_layer_eps(l, complex(l.eps1, l.eps1i), complex(l.eps2, l.eps2i), xe, ye)
                        for l in layers])
        stacks.append(o.Stack(nHx, nHy, xe, ye, eps, [0] + [l.thickness for l in layers[1:-1]] + [0]))
    pts, pxy = [], []
    for i, s in enumerate(setups):
        r = orc.rcwa_run(s)[0]
        pts.append((i, r["lam"], r["kx0"], r["ky0"]))
        te, tm = orc.polarisation_vectors(s.theta, s.phi)
        pxy.append([te, tm])
    R, T, REF, TRN, st = eng.solve_batch(stacks, pts, np.array(pxy, dtype=complex))
    assert np.all(st == 0)
    for i, s in enumerate(setups):
        r = orc.rcwa_run(s)[0]
        assert np.max(np.abs(R[i] - r["R"])) < TOL_RT and np.max(np.abs(T[i] - r["T"])) < TOL_RT
        assert np.max(np.abs(REF[i] - r["REF"])) < TOL_RT and np.max(np.abs(TRN[i] - r["TRN"])) < TOL_RT


def test_grazing_incidence_reports_status(eng):
    R, T, _, _, st = eng.ofd_solve(OfdSetup(nHx=1, period_x=3e-7, layers=[L(1, 1, .5, 0), L(2.25, 2.25, .5, 0)],
                                            freqs=[5e14], theta=90.0))
    assert st[0] == 6  # RCWA_ERR_GRAZING


def test_invalid_setup_rejected(eng):
    import openrcwa_b200 as o
    with pytest.raises(o.RcwaError):
        eng.ofd_solve(OfdSetup(nHx=1, period_x=3e-7, layers=[L(1, 1, .5, 0)], freqs=[5e14]))


def test_large_orders_panel_lu_path(eng):
    # n = 162 and a small batch: the interface and tau factorisations take the
    # multi-launch panel LU instead of one CTA per matrix
    rng = np.random.default_rng(5)
    layers = [L(1, 1, .5, 0)]
    for _ in range(2):
        layers.append(L(rng.uniform(2, 12), 1.0, rng.uniform(.2, .8), rng.uniform(50e-9, 300e-9),
                        rng.uniform(0, .5), 0.0, rng.uniform(.2, .8)))
    layers.append(L(2.25, 2.25, .5, 0))
    setup = OfdSetup(nHx=4, period_x=4e-7, nHy=4, period_y=4e-7, layers=layers,
                     freqs=orc.C0 / np.array([450e-9, 700e-9]), theta=35.0, phi=20.0)
    _cmp_ofd(eng, setup)


def test_plan_graph_replay_and_rescatter(eng):
    # first execution launches directly, later ones replay a captured CUDA
    # graph (recaptured when stage profiling is switched); all bit-identical
    import openrcwa_b200 as o
    from openrcwa_b200 import workloads
    stacks, pts, pxy = workloads.pillars_2d(seed=3, nH=3)
    bp, bx = workloads.batch_slice(pts, pxy, 0, 6)
    plan = eng.plan(stacks, bp, bx)
    outs = []
    for prof in (True, True, True, False, False, True, False):
        plan.set_profiling(prof)
        plan.execute()
        outs.append(plan.results(orders=True))
    for r in outs[1:]:
        for a, b in zip(outs[0], r):
            assert np.array_equal(a, b)
    assert plan.launch_count() > 0
    # rescatter: swap TE/TM and compare with a fresh solve
    bx2 = np.ascontiguousarray(bx[:, ::-1, :])
    plan.rescatter(bx2)
    R, T, _, _, st = plan.results()
    R2, T2, _, _, st2 = eng.solve_batch(stacks, bp, bx2, orders=False)
    assert not np.any(st) and not np.any(st2)
    assert np.max(np.abs(R - R2)) < 1e-12 and np.max(np.abs(T - T2)) < 1e-12
    plan.close()


def test_uneven_batch_sizes_and_materials(eng):
    # cfg3's instance mix (Lorentz and metal layers, 1-3 layers, nH 3..5)
    # in one call, every point against the oracle
    import openrcwa_b200 as o
    from openrcwa_b200 import workloads
    stacks, pts, pxy = workloads.uneven_batch(seed=2, n_instances=6, nh_range=(3, 5), max_layers=3)
    R, T, REF, TRN, st = eng.solve_batch(stacks, pts, pxy)
    assert np.all(st == 0)
    for i, s in enumerate(stacks):
        sol = orc.RCWASolver(s.nHx, s.nHy)
        for l in range(s.eps.shape[0]):
            sol.addLayer(orc.OracleLayer(s.cx, s.cy, s.eps[l]))
        sol.setBlochWavevector(pts[i, 2], pts[i, 3])
        sol.solve(pts[i, 1], list(range(s.eps.shape[0])), list(s.thickness))
        k0 = 2 * math.pi / pts[i, 1]
        for x in range(2):
            c = sol.generateHorizontalPlaneWave(pxy[i, x, 0], pxy[i, x, 1], 0)
            ref, trn = sol.scatterPlaneWave(c, 0, s.eps.shape[0] - 1, k0)
            assert abs(R[i, x] - ref.sum()) < TOL_RT and abs(T[i, x] - trn.sum()) < TOL_RT


def test_largest_order_count(eng):
    # nH = 15 (961 orders, 1922 x 1922 layer matrices), one patterned layer
    import openrcwa_b200 as o
    from openrcwa_b200 import workloads
    st = workloads.rect_stack(15, 15, 4e-7, 4e-7, [(complex(6.0, 0.2), 1.0, 0.4, 0.6, 1.5e-7)])
    lam = 7e-7
    k0 = 2 * math.pi / lam
    pts = np.array([(0, lam, k0 * math.sin(0.3), 0.0)])
    te, tm = workloads.pol_vectors(math.degrees(0.3), 0.0)
    pxy = np.array([[te, tm]], dtype=complex)
    R, T, _, _, status = eng.solve_batch([st], pts, pxy, orders=False)
    assert not np.any(status)
    sol = orc.RCWASolver(15, 15)
    for l in range(st.eps.shape[0]):
        sol.addLayer(orc.OracleLayer(st.cx, st.cy, st.eps[l]))
    sol.setBlochWavevector(pts[0, 2], pts[0, 3])
    sol.solve(lam, list(range(st.eps.shape[0])), list(st.thickness))
    for x in range(2):
        c = sol.generateHorizontalPlaneWave(pxy[0, x, 0], pxy[0, x, 1], 0)
        ref, trn = sol.scatterPlaneWave(c, 0, st.eps.shape[0] - 1, k0)
        assert abs(R[0, x] - ref.sum()) < TOL_RT and abs(T[0, x] - trn.sum()) < TOL_RT
