"""Parity of the slab S-matrix and Redheffer star product (CUDA, through the C
ABI) with the CPU oracle, plus the exact relations of the z-integrators.

Tolerance: 1e-10 relative to the largest entry of each compared block (FP64
throughout; the reference computes the same quantities with Eigen LU solves).
"""
import math

import numpy as np
import pytest

from oracle import smatrix_oracle as so
from tests.test_smatrix_oracle import pillar_modes, sym, uniform_modes

pytestmark = pytest.mark.gpu

TOL = 1e-10


@pytest.fixture(scope="module")
def eng():
    import openrcwa_b200 as o
    e = o.Engine(0)
    yield e
    e.close()


def rel(a, b):
    return np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300)


@pytest.mark.parametrize("nx,ny", [(3, 3), (11, 1), (7, 7)])
def test_slab_smatrix_parity(eng, nx, ny):
    lams = [0.9, 1.0, 1.3]
    wzs = [0.05, 0.21, 0.4]
    Ws, Vs, gs, W0s, V0s = [], [], [], [], []
    for k, lam in enumerate(lams):
        W, V, g = pillar_modes(nx, ny, lam, 5.0 + 0.3j * k)
        W0, V0, _ = uniform_modes(nx, ny, lam, 1.0 + 1.25 * k)
        Ws.append(W); Vs.append(V); gs.append(g); W0s.append(W0); V0s.append(V0)
    R, T, st = eng.slab_smatrix(np.stack(Ws), np.stack(Vs), np.stack(gs), np.stack(W0s), np.stack(V0s),
                                np.array(lams), np.array(wzs))
    assert not np.any(st)
    for k in range(len(lams)):
        Rr, Tr = so.slab_smatrix(Ws[k], Vs[k], gs[k], W0s[k], V0s[k], lams[k], wzs[k])
        assert rel(R[k], Rr) < TOL
        assert rel(T[k], Tr) < TOL


def test_uniform_section_own_basis(eng):
    lam, wz = 1.0, 0.37
    W, V, g = pillar_modes(5, 5, lam, 8.0 + 0.1j)
    R, T, st = eng.slab_smatrix(W, V, g, W, V, lam, wz)
    X = np.exp(1j * g * lam / (2 * math.pi) * wz)
    assert not np.any(st)
    assert np.max(np.abs(R[0])) < 1e-12
    assert np.max(np.abs(T[0] - np.diag(X))) < 1e-12


def test_star_product_chain_parity(eng):
    nx = ny = 5
    lam = 1.0
    W0, V0, _ = uniform_modes(nx, ny, lam, 2.25)
    S_gpu = so.identity_smatrix(2 * nx * ny)
    S_ref = so.identity_smatrix(2 * nx * ny)
    for k, (e1, wz) in enumerate([(4.0, 0.1), (2.1 + 0.01j, 0.07), (9.0 + 0.4j, 0.15), (3.0, 0.05)]):
        W, V, g = pillar_modes(nx, ny, lam, e1, fill=(0.3 + 0.1 * k, 0.5))
        R, T, st = eng.slab_smatrix(W, V, g, W0, V0, lam, wz)
        assert not np.any(st)
        S_gpu, st = eng.star_product(S_gpu, sym(R[0], T[0]))
        assert not np.any(st)
        S_ref = so.star_product(S_ref, sym(*so.slab_smatrix(W, V, g, W0, V0, lam, wz)))
    for key in ("Rud", "Rdu", "Tdd", "Tuu"):
        assert rel(S_gpu[key][0], S_ref[key]) < TOL, key


def test_composition_law_large(eng):
    nx = ny = 9  # n = 162
    lam = 1.0
    W, V, g = pillar_modes(nx, ny, lam, 6.0 + 0.2j)
    W0, V0, _ = uniform_modes(nx, ny, lam, 1.0)
    R, T, _ = eng.slab_smatrix(np.stack([W, W, W]), np.stack([V, V, V]), np.stack([g, g, g]),
                               np.stack([W0] * 3), np.stack([V0] * 3), lam, np.array([0.11, 0.17, 0.28]))
    n = W.shape[0]
    S, st = eng.star_product(so.identity_smatrix(n), sym(R[0], T[0]))
    S, st2 = eng.star_product(S, sym(R[1], T[1]))
    assert not np.any(st) and not np.any(st2)
    for key, ref in (("Rud", R[2]), ("Rdu", R[2]), ("Tdd", T[2]), ("Tuu", T[2])):
        assert rel(S[key][0], ref) < 1e-9, key


def test_singular_slab_reports_status(eng):
    n = 8
    Z = np.zeros((n, n), dtype=complex)
    I = np.eye(n, dtype=complex)
    g = np.ones(n, dtype=complex)
    _, _, st = eng.slab_smatrix(np.stack([Z, I]), np.stack([I, I]), np.stack([g, g]), np.stack([I, I]),
                                np.stack([I * 2, I * 2]), 1.0, 0.1)
    assert st[0] != 0 and st[1] == 0
