"""Stacks given by Laurent coefficient tables (rcwa_engine_solve_tables): the
large-order circular-pillar structure at reduced order against the oracle
(the same tables, all three convolution matrices from the Laurent rule), and
energy conservation on lossless pillars."""
import math

import numpy as np
import pytest

import oracle.rcwa_oracle as orc
import openrcwa_b200 as o
from openrcwa_b200 import workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _oracle(st, pts, pxy):
    """R, T, REF, TRN of every point through the oracle with table layers."""
    L = st.thickness.size
    cx, cy = np.array([0.0, st.Lx]), np.array([0.0, st.Ly])
    out = []
    for p in range(len(pts)):
        sol = orc.RCWASolver(st.nHx, st.nHy)
        for l in range(L):
            if l == 0 or l == L - 1:
                sol.addLayer(orc.OracleLayer(cx, cy, np.array([[st.eps_half[0 if l == 0 else 1]]])))
            else:
                F = st.f2d[l - 1]
                mean = F[F.shape[0] // 2, F.shape[1] // 2]
                sol.addLayer(orc.OracleLayer(cx, cy, np.array([[mean]]), f2d=F))
        sol.setBlochWavevector(pts[p, 2], pts[p, 3])
        sol.solve(pts[p, 1], list(range(L)), list(st.thickness))
        k0 = 2 * math.pi / pts[p, 1]
        r = []
        for e in range(pxy.shape[1]):
            c = sol.generateHorizontalPlaneWave(pxy[p, e, 0], pxy[p, e, 1], 0)
            r.append(sol.scatterPlaneWave(c, 0, L - 1, k0))
        out.append((np.array([a.sum() for a, _ in r]), np.array([b.sum() for _, b in r]),
                    np.array([a for a, _ in r]), np.array([b for _, b in r])))
    return out


@pytest.mark.parametrize("nh,layers", [(3, 4), (6, 3)])
def test_circular_pillars_against_oracle(eng, nh, layers):
    stacks, pts, pxy = workloads.circular_pillars(seed=nh, nH=nh, n_lambda=3, n_layers=layers)
    R, T, REF, TRN, status = eng.solve_batch(stacks, pts, pxy)
    assert not np.any(status)
    for p, (Ro, To, REFo, TRNo) in enumerate(_oracle(stacks[0], pts, pxy)):
        assert np.max(np.abs(R[p] - Ro)) < 1e-9 and np.max(np.abs(T[p] - To)) < 1e-9
        assert np.max(np.abs(REF[p] - REFo)) < 1e-9 and np.max(np.abs(TRN[p] - TRNo)) < 1e-9
    Rm, Tm, _, _, sm = eng.solve_batch(stacks, pts, pxy, orders=False, precision=o.RCWA_PREC_MIXED)
    assert not np.any(sm)
    assert np.max(np.abs(Rm - R)) < 1e-4 and np.max(np.abs(Tm - T)) < 1e-4


def test_lossless_circular_pillars_conserve_energy(eng):
    stacks, pts, pxy = workloads.circular_pillars(seed=5, nH=8, n_lambda=4, n_layers=6)
    st = stacks[0]
    lossless = o.TableStack(st.nHx, st.nHy, st.Lx, st.Ly, st.eps_half,
                            np.array([workloads.disk_laurent_table(st.Lx, st.Ly, 0.3 * st.Lx, (0.5 * st.Lx,) * 2,
                                                                   4.0 if k % 2 == 0 else 2.1, 1.0, st.nHx)
                                      for k in range(st.f2d.shape[0])]), st.thickness)
    R, T, _, _, status = eng.solve_batch([lossless], pts, pxy, orders=False)
    assert not np.any(status)
    assert np.max(np.abs(R + T - 1.0)) < 1e-10
    # normal incidence on a C4-symmetric pillar: TE and TM are degenerate
    assert np.max(np.abs(R[:, 0] - R[:, 1])) < 1e-9


def test_table_stack_rejects_bad_input(eng):
    stacks, pts, pxy = workloads.circular_pillars(seed=1, nH=2, n_lambda=1, n_layers=2)
    st = stacks[0]
    st.f2d[0, 0, 0] = complex(float("nan"), 0.0)
    with pytest.raises(o.RcwaError) as ex:
        eng.solve_batch(stacks, pts, pxy)
    assert ex.value.code == o.abi.RCWA_ERR_NONFINITE
