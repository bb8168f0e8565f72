"""The eigensolver with a team (thread-block cluster) of CTAs per matrix
(rcwa_set_eig_cluster): the team splits the rows of the Hessenberg panel
products, the tiles of its GEMMs and the off-window lines of the Schur sweeps,
and every element is computed by the same operations as with one CTA, so the
eigenvalues and eigenvectors are identical bit for bit for every team size."""
import numpy as np
import pytest

import openrcwa_b200 as o

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    o.set_eig_cluster(0)
    e.close()


def _matrices(n, b, seed):
    rng = np.random.default_rng(seed)
    return rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n))


@pytest.mark.parametrize("n,b", [(200, 3), (450, 2)])
def test_team_sizes_give_identical_results(eng, n, b):
    A = _matrices(n, b, n)
    o.set_eig_cluster(1)
    w1, V1, i1 = eng.zgeev(A)
    assert not np.any(i1)
    for team in (2, 3, 8):
        o.set_eig_cluster(team)
        assert o.eig_cluster_size(n, b) == team
        w, V, info = eng.zgeev(A)
        assert not np.any(info)
        assert np.array_equal(w, w1) and np.array_equal(V, V1), team
    o.set_eig_cluster(0)
    for k in range(b):
        res = np.abs(A[k] @ V1[k] - V1[k] * w1[k][None, :]).max() / np.abs(A[k]).max()
        assert res < 1e-11


def test_automatic_team_for_few_large_matrices(eng):
    o.set_eig_cluster(0)
    assert o.eig_cluster_size(882, 4) == 1        # below the order threshold
    assert o.eig_cluster_size(1200, 148) == 1     # the batch fills the GPU
    team = o.eig_cluster_size(1200, 4)
    assert 2 <= team <= 8
    A = _matrices(1200, 4, 7)
    w, V, _ = eng.zgeev(A)
    o.set_eig_cluster(1)
    w1, V1, _ = eng.zgeev(A)
    o.set_eig_cluster(0)
    assert np.array_equal(w, w1) and np.array_equal(V, V1)


def test_solve_with_teams_matches_single_cta(eng):
    # one point of a 2D pillar grating at Nx = Ny = 11 (n = 1058): three layer
    # eigensolves and LU batches of one and two matrices, so the automatic
    # rule gives the eigensolver and the LU panels clusters of CTAs; R, T and
    # every order must equal the one-CTA solve bit for bit
    from openrcwa_b200 import workloads
    stacks, pts, pxy = workloads.pillars_2d(seed=3, nH=11, n_lambda=1, n_angle=1, n_layers=3)
    o.set_eig_cluster(0)
    o.set_lu_cluster(0)
    assert o.eig_cluster_size(1058, 3) > 1 and o.lu_cluster_size(1058, 1) > 1
    R, T, REF, TRN, st = eng.solve_batch(stacks, pts[:1], pxy[:1])
    o.set_eig_cluster(1)
    o.set_lu_cluster(1)
    try:
        R1, T1, REF1, TRN1, st1 = eng.solve_batch(stacks, pts[:1], pxy[:1])
    finally:
        o.set_eig_cluster(0)
        o.set_lu_cluster(0)
    assert not np.any(st) and not np.any(st1)
    assert np.array_equal(R, R1) and np.array_equal(T, T1)
    assert np.array_equal(REF[0], REF1[0]) and np.array_equal(TRN[0], TRN1[0])
    assert np.all(R + T <= 1.0 + 1e-9)  # lossy layers
