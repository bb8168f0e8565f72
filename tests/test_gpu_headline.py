"""Parity at the benchmark sizes against oracle fixtures (tests/golden/make_large.py).

* The 2D pillar sweep at Nx=Ny=10 (441 orders, 882 x 882 layer matrices, five
  lossy layers, conical incidence): the exact 148-point batch the benchmark
  times, through the FP64 plan (every R, T and per-order efficiency within
  1e-9 of the oracle) and the mixed plan (within 1e-4 of the oracle), and a
  lossless copy of the stack on which R + T = 1 within 1e-10.
* Instances of the uneven workload at their real sizes (nH up to 15, up to six
  layers) in one call: the all-dielectric ones within 1e-9 (FP64) and 1e-4
  (mixed) of the oracle; the metallic ones within 1e-9 where the oracle's own
  answer is trustworthy (its LU and SVD solves agree to 1e-10 and R + T <= 1).
  On thick metal stacks the reference's interface solves W_a^-1 W_b
  (rcwa/RCWASolver.cpp:495-614) lose their accuracy, the oracle's answers then
  depend on the LAPACK path, and only the status and finiteness are checked.
"""
import os

import numpy as np
import pytest

import openrcwa_b200 as o
from openrcwa_b200 import workloads

pytestmark = pytest.mark.gpu

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_FP64 = 1e-9
TOL_MIXED = 1e-4
BATCH = 148


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _plan_results(eng, stacks, pts, pxy, precision):
    plan = eng.plan(stacks, pts, pxy, precision=precision)
    plan.execute()
    R, T, ref, trn, status = plan.results(orders=True)
    plan.close()
    return R, T, ref, trn, status


def _orders(flat, n_pts, n_exc, N, p):
    return flat.reshape(n_pts, n_exc, N)[p]


@pytest.mark.parametrize("precision,tol", [(o.RCWA_PREC_FP64, TOL_FP64), (o.RCWA_PREC_MIXED, TOL_MIXED)])
def test_pillar_benchmark_batch_against_oracle(eng, precision, tol):
    g = np.load(os.path.join(HERE, "pillars_nh10_points.npz"))
    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=10)
    bp, bx = workloads.batch_slice(pts, pxy, workloads.shard_start(0, 1, BATCH, 0), BATCH)
    R, T, ref, trn, status = _plan_results(eng, stacks, bp, bx, precision)
    assert not np.any(status)
    N = stacks[0].N
    for k, p in enumerate(g["points"]):
        assert np.max(np.abs(R[p] - g["R"][k])) < tol, (p, R[p], g["R"][k])
        assert np.max(np.abs(T[p] - g["T"][k])) < tol, (p, T[p], g["T"][k])
        assert np.max(np.abs(_orders(ref, BATCH, 2, N, p) - g["REF"][k])) < tol
        assert np.max(np.abs(_orders(trn, BATCH, 2, N, p) - g["TRN"][k])) < tol
    # every point of the batch: efficiencies in range (lossy stack: R + T < 1)
    assert np.all(R >= -1e-12) and np.all(T >= -1e-12) and np.all(R + T <= 1 + tol)


def test_pillar_lossless_energy(eng):
    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=10)
    st = stacks[0]
    lossless = o.Stack(st.nHx, st.nHy, st.cx, st.cy, st.eps.real.astype(complex), st.thickness)
    bp, bx = workloads.batch_slice(pts, pxy, 0, 16)
    R, T, _, _, status = eng.solve_batch([lossless], bp, bx, orders=False)
    assert not np.any(status)
    assert np.max(np.abs(R + T - 1.0)) < 1e-10
    Rm, Tm, _, _, status = eng.solve_batch([lossless], bp, bx, orders=False, precision=o.RCWA_PREC_MIXED)
    assert not np.any(status)
    assert np.max(np.abs(Rm + Tm - 1.0)) < TOL_MIXED
    assert np.max(np.abs(Rm - R)) < TOL_MIXED and np.max(np.abs(Tm - T)) < TOL_MIXED


def test_uneven_instances_at_real_sizes(eng):
    g = np.load(os.path.join(HERE, "uneven_sample.npz"))
    ids = [int(i) for i in g["ids"]]
    all_st, all_pts, all_pxy = workloads.uneven_batch(seed=0, n_instances=max(ids) + 1)
    stacks = [all_st[i] for i in ids]
    pts = np.array([(k, all_pts[i][1], all_pts[i][2], all_pts[i][3]) for k, i in enumerate(ids)])
    pxy = all_pxy[ids]
    res = {}
    for prec in (o.RCWA_PREC_FP64, o.RCWA_PREC_MIXED):
        R, T, REF, TRN, status = eng.solve_batch(stacks, pts, pxy, precision=prec)
        assert not np.any(status), status
        res[prec] = (R, T, REF, TRN)
    checked = 0
    for k, i in enumerate(ids):
        R, T, REF, TRN = res[o.RCWA_PREC_FP64]
        assert np.all(np.isfinite(R[k])) and np.all(np.isfinite(T[k]))
        if g["metal"][k] and not g["sane"][k]:
            continue
        assert np.max(np.abs(R[k] - g["R"][k])) < TOL_FP64, (i, R[k], g["R"][k])
        assert np.max(np.abs(T[k] - g["T"][k])) < TOL_FP64, (i, T[k], g["T"][k])
        assert np.max(np.abs(REF[k] - g["REF_%d" % i])) < TOL_FP64
        assert np.max(np.abs(TRN[k] - g["TRN_%d" % i])) < TOL_FP64
        checked += 1
        if not g["metal"][k]:
            Rm, Tm, REFm, TRNm = res[o.RCWA_PREC_MIXED]
            assert np.max(np.abs(Rm[k] - g["R"][k])) < TOL_MIXED and np.max(np.abs(Tm[k] - g["T"][k])) < TOL_MIXED
            assert np.max(np.abs(REFm[k] - g["REF_%d" % i])) < TOL_MIXED
    assert checked >= 8
