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
