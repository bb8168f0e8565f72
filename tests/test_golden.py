"""Oracle and engine against the committed golden fixtures (tests/golden)."""
import os

import numpy as np
import pytest

from oracle.rcwa_oracle import rcwa_run
from tests.golden.make_golden import CASES

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_fixture(name):
    g = np.load(os.path.join(HERE, name + ".npz"))
    out = rcwa_run(CASES[name])
    assert np.max(np.abs(np.array([r["R"] for r in out]) - g["R"])) < 1e-12
    assert np.max(np.abs(np.array([r["T"] for r in out]) - g["T"])) < 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(CASES))
def test_engine_matches_fixture(name):
    import openrcwa_b200 as o
    g = np.load(os.path.join(HERE, name + ".npz"))
    eng = o.Engine(0)
    R, T, oR, oT, st = eng.ofd_solve(CASES[name])
    eng.close()
    assert np.all(st == 0)
    assert np.max(np.abs(R - g["R"])) < 1e-9 and np.max(np.abs(T - g["T"])) < 1e-9
    assert np.max(np.abs(np.transpose(oR, (1, 0, 2)) - g["ordR"])) < 1e-9
    assert np.max(np.abs(np.transpose(oT, (1, 0, 2)) - g["ordT"])) < 1e-9


def test_oracle_reproduces_large_fixtures_on_small_members():
    """The benchmark-size fixtures (tests/golden/make_large.py) against a fresh
    oracle run of their cheapest members, and their shapes and ranges."""
    from openrcwa_b200 import workloads
    from tests.golden.make_large import oracle_point
    g = np.load(os.path.join(HERE, "uneven_sample.npz"))
    ids = [int(i) for i in g["ids"]]
    stacks, pts, pxy = workloads.uneven_batch(seed=0, n_instances=max(ids) + 1)
    for i in (57, 361, 11):
        k = ids.index(i)
        R, T, REF, TRN = oracle_point(stacks[i], pts[i], pxy[i])
        assert np.max(np.abs(R - g["R"][k])) < 1e-12 and np.max(np.abs(T - g["T"][k])) < 1e-12
        assert np.max(np.abs(REF - g["REF_%d" % i])) < 1e-12 and np.max(np.abs(TRN - g["TRN_%d" % i])) < 1e-12
    assert np.sum(~g["metal"]) == 8 and np.all(g["sane"][~g["metal"]])
    p = np.load(os.path.join(HERE, "pillars_nh10_points.npz"))
    assert p["REF"].shape == (3, 2, 441) and p["TRN"].shape == (3, 2, 441)
    assert np.allclose(p["REF"].sum(axis=2), p["R"], atol=1e-12) and np.allclose(p["TRN"].sum(axis=2), p["T"],
                                                                                   atol=1e-12)
    assert np.all(p["R"] + p["T"] < 1.0) and np.all(p["R"] > 0) and np.all(p["T"] > 0)
