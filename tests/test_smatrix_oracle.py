"""Slab S-matrix / Redheffer star-product oracle pinned by exact relations.

tests/test_core_integrators.cpp:[1] of the reference: a z-uniform section
seen from its own eigenbasis has Rud = Rdu = 0 and Tuu = Tdd =
diag(exp(i gamma L/k0)).  The composition law (two slabs of one layer, star
multiplied, equal the single slab of the summed thickness, in any reference
basis) pins the star product and the slab formulas against each other.
"""
import math

import numpy as np
import pytest

from oracle import rcwa_oracle as ro
from oracle import smatrix_oracle as so


def pillar_modes(nx, ny, lam, eps1, fill=(0.45, 0.6), period=(0.8, 0.7), kx0=0.3, ky0=0.2):
    """W, V, keff (unscaled propagation constants) of one rectangle layer."""
    Lx, Ly = period
    cx = np.array([0.0, fill[0] * Lx, Lx])
    cy = np.array([0.0, fill[1] * Ly, Ly])
    eps = np.array([[eps1, 1.0], [1.0, 1.0]], dtype=complex)
    a, b = ro.alpha_beta(nx, ny, Lx, Ly, kx0, ky0)
    sol = ro.layer_solve(cx, cy, eps, a, b, lam, nx, ny)
    k0 = 2 * math.pi / lam
    return sol.W, sol.V, sol.gamma * k0


def uniform_modes(nx, ny, lam, eps, period=(0.8, 0.7), kx0=0.3, ky0=0.2):
    Lx, Ly = period
    cx = np.array([0.0, Lx])
    cy = np.array([0.0, Ly])
    a, b = ro.alpha_beta(nx, ny, Lx, Ly, kx0, ky0)
    sol = ro.layer_solve(cx, cy, np.array([[eps]], dtype=complex), a, b, lam, nx, ny)
    return sol.W, sol.V, sol.gamma * 2 * math.pi / lam


def sym(R, T):
    return {"rud": R, "rdu": R, "tdd": T, "tuu": T}


@pytest.mark.parametrize("nx,ny", [(3, 3), (5, 1)])
def test_uniform_section_in_own_basis(nx, ny):
    lam, wz = 1.0, 0.37
    W, V, g = pillar_modes(nx, ny, lam, 6.0 + 0.2j)
    R, T = so.slab_smatrix(W, V, g, W, V, lam, wz)
    X = np.exp(1j * g * lam / (2 * math.pi) * wz)
    assert np.max(np.abs(R)) < 1e-12
    assert np.max(np.abs(T - np.diag(X))) < 1e-12


@pytest.mark.parametrize("nx,ny", [(3, 3), (5, 1)])
def test_slab_composition_law(nx, ny):
    lam = 1.0
    W, V, g = pillar_modes(nx, ny, lam, 6.0 + 0.2j)
    W0, V0, _ = uniform_modes(nx, ny, lam, 1.0)
    d1, d2 = 0.13, 0.21
    S = so.identity_smatrix(W.shape[0])
    S = so.star_product(S, sym(*so.slab_smatrix(W, V, g, W0, V0, lam, d1)))
    S = so.star_product(S, sym(*so.slab_smatrix(W, V, g, W0, V0, lam, d2)))
    R, T = so.slab_smatrix(W, V, g, W0, V0, lam, d1 + d2)
    scale = max(np.max(np.abs(T)), 1.0)
    for key, ref in (("Rud", R), ("Rdu", R), ("Tdd", T), ("Tuu", T)):
        assert np.max(np.abs(S[key] - ref)) < 1e-10 * scale, key


def test_star_product_identity_is_neutral():
    rng = np.random.default_rng(3)
    n = 12
    s = {k: rng.standard_normal((n, n)) * 0.3 + 1j * rng.standard_normal((n, n)) * 0.3
         for k in ("rud", "rdu", "tdd", "tuu")}
    S = so.star_product(so.identity_smatrix(n), s)
    assert np.allclose(S["Rud"], s["rud"]) and np.allclose(S["Rdu"], s["rdu"])
    assert np.allclose(S["Tdd"], s["tdd"]) and np.allclose(S["Tuu"], s["tuu"])
