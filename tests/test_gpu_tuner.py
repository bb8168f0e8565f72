"""Schedule autotuner on the GPU: measurements return a candidate with a time
for each, every forced schedule gives the oracle's efficiencies (1e-9), a
mixed plan whose products the tuner sends to the FP64 path equals the FP64
plan bit for bit, automatic mode records its choices, and a saved table
drives a second engine."""
import os

import numpy as np
import pytest

import openrcwa_b200 as o
from tests.test_gpu_mixed import _setup, _stack_points

pytestmark = pytest.mark.gpu

TOL = 1e-9


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


@pytest.fixture(scope="module")
def case():
    return _stack_points(_setup(11, 5))   # n = 242, 2 points, 3 patterned layers


def _check_oracle(R, T, REF, TRN, ref):
    for p, r in enumerate(ref):
        assert np.max(np.abs(R[p] - r["R"])) < TOL and np.max(np.abs(T[p] - r["T"])) < TOL
        assert np.max(np.abs(REF[p] - r["REF"])) < TOL and np.max(np.abs(TRN[p] - r["TRN"])) < TOL


@pytest.mark.parametrize("op,n,batch", [("lu", 162, 8), ("lu", 242, 300), ("schur", 130, 4), ("product", 200, 4)])
def test_measure_returns_a_timed_candidate(eng, op, n, batch):
    t = o.Tuner()
    choice, ms = t.measure(eng, op, n, batch)
    assert choice in t.candidates(op, n)
    assert set(ms) == set(t.candidates(op, n)) and all(v > 0 for v in ms.values())
    assert ms[choice] == min(ms.values())
    assert t.get(op, n, batch) == choice
    t.close()


@pytest.mark.parametrize("lu", [0, 1])
@pytest.mark.parametrize("cross", [64, 96, 128, 192])
def test_every_schedule_matches_oracle(eng, case, lu, cross):
    st, pts, pxy, ref = case
    n = 2 * st.N
    t = o.Tuner()
    for b in (1, 2 * len(pts)):
        t.set("lu", n, b, lu)
    t.set("schur", n, 3 * len(pts), cross)
    eng.set_tuner(t, o.RCWA_TUNING_TABLE)
    try:
        plan = eng.plan([st], pts, pxy)
        sched = plan.schedule()
        assert sched == [{"n": n, "points": len(pts), "lu_interface": lu, "lu_tau": lu, "schur_crossover": cross,
                          "product": 1}]   # an FP64 plan: FP64 products
        plan.execute()
        R, T, ref_o, trn_o, status = plan.results(orders=True)
        plan.close()
        REF = ref_o.reshape(len(pts), pxy.shape[1], st.N)
        TRN = trn_o.reshape(len(pts), pxy.shape[1], st.N)
    finally:
        eng.set_tuner(None, o.RCWA_TUNING_OFF)
    assert not np.any(status)
    _check_oracle(R, T, REF, TRN, ref)


def test_blocked_lu_schedule_matches_oracle(eng):
    # LU choice 2 (128-column blocks, K = 128 trailing updates) at n = 338:
    # three blocks, the last one ragged
    st, pts, pxy, ref = _stack_points(_setup(12, 6))
    n = 2 * st.N
    t = o.Tuner()
    for b in (len(pts), 2 * len(pts)):
        t.set("lu", n, b, 2)
    eng.set_tuner(t, o.RCWA_TUNING_TABLE)
    try:
        plan = eng.plan([st], pts, pxy)
        sched = plan.schedule()[0]
        assert sched["lu_interface"] == 2 and sched["lu_tau"] == 2
        plan.execute()
        R, T, ref_o, trn_o, status = plan.results(orders=True)
        plan.close()
    finally:
        eng.set_tuner(None, o.RCWA_TUNING_OFF)
    assert not np.any(status)
    _check_oracle(R, T, ref_o.reshape(len(pts), pxy.shape[1], st.N), trn_o.reshape(len(pts), pxy.shape[1], st.N), ref)


def test_mixed_plan_with_fp64_products_equals_fp64_plan(eng, case):
    st, pts, pxy, _ = case
    n = 2 * st.N
    t = o.Tuner()
    t.set("product", n, len(pts), 1)
    eng.set_tuner(t, o.RCWA_TUNING_TABLE)
    try:
        Rm, Tm, _, _, sm = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
        R6, T6, _, _, s6 = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_FP64)
    finally:
        eng.set_tuner(None, o.RCWA_TUNING_OFF)
    assert not np.any(sm) and not np.any(s6)
    assert np.array_equal(Rm, R6) and np.array_equal(Tm, T6)


def test_wide_tensor_core_tiles_match_the_oracle(eng, case):
    # product choice 2: 3xTF32 on 128 x 256 output tiles (one CTA per SM)
    st, pts, pxy, ref = case
    n = 2 * st.N
    t = o.Tuner()
    t.set("product", n, len(pts), 2)
    eng.set_tuner(t, o.RCWA_TUNING_TABLE)
    try:
        plan = eng.plan([st], pts, pxy, o.RCWA_PREC_MIXED)
        assert plan.schedule()[0]["product"] == 2
        plan.execute()
        R, T, ref_o, trn_o, status = plan.results(orders=True)
        plan.close()
        R0, T0, _, _, s0 = eng.solve_batch([st], pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
    finally:
        eng.set_tuner(None, o.RCWA_TUNING_OFF)
    assert not np.any(status) and not np.any(s0)
    for p, r in enumerate(ref):
        assert np.max(np.abs(R[p] - r["R"])) < 1e-4 and np.max(np.abs(T[p] - r["T"])) < 1e-4
    assert np.max(np.abs(R - R0)) < 1e-5 and np.max(np.abs(T - T0)) < 1e-5


def test_auto_mode_records_and_stays_exact(eng, case, tmp_path):
    st, pts, pxy, ref = case
    n = 2 * st.N
    t = o.Tuner()
    eng.set_tuner(t, o.RCWA_TUNING_AUTO)
    try:
        R, T, REF, TRN, status = eng.solve_batch([st], pts, pxy, precision=o.RCWA_PREC_MIXED)
        R6, T6, REF6, TRN6, status6 = eng.solve_batch([st], pts, pxy)
    finally:
        eng.set_tuner(None, o.RCWA_TUNING_OFF)
    assert not np.any(status) and not np.any(status6)
    _check_oracle(R6, T6, REF6, TRN6, ref)
    assert np.max(np.abs(R - R6)) < 1e-4 and np.max(np.abs(T - T6)) < 1e-4
    ops = sorted({e["op"] for e in t.entries() if e["n"] == n})
    assert ops == ["lu", "product", "schur"]
    for e in t.entries():
        assert e["choice"] in t.candidates(e["op"], e["n"])
        assert all(v > 0 for v in e["ms"].values())
    # the saved table drives a second engine without measuring
    path = os.path.join(tmp_path, "sched.txt")
    t.save(path)
    u = o.Tuner()
    u.load(path)
    e2 = o.Engine(0)
    e2.set_tuner(u, o.RCWA_TUNING_TABLE)
    plan = e2.plan([st], pts, pxy, o.RCWA_PREC_MIXED)
    sched = plan.schedule()[0]
    plan.close()
    e2.close()
    assert sched["schur_crossover"] == t.get("schur", n, 3 * len(pts))
    assert sched["lu_tau"] == t.get("lu", n, len(pts))
    assert sched["lu_interface"] == t.get("lu", n, 2 * len(pts))
    assert sched["product"] == t.get("product", n, len(pts))
    assert len(u.entries()) == len(t.entries())


@pytest.mark.parametrize("cross", [64, 128])
def test_small_matrix_schur_paths(eng, cross):
    # n = 98: multishift kernel (64) or the single-shift kernel for the whole
    # matrix (128, the built-in rule below 128 rows)
    st, pts, pxy, ref = _stack_points(_setup(12, 3))
    n = 2 * st.N
    t = o.Tuner()
    t.set("schur", n, 3 * len(pts), cross)
    eng.set_tuner(t, o.RCWA_TUNING_TABLE)
    try:
        R, T, REF, TRN, status = eng.solve_batch([st], pts, pxy)
    finally:
        eng.set_tuner(None, o.RCWA_TUNING_OFF)
    assert n == 98 and not np.any(status)
    _check_oracle(R, T, REF, TRN, ref)
