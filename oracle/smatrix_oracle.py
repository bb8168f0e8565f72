"""CPU oracle for the slab scattering matrix and the Redheffer star product.

TEST INFRASTRUCTURE ONLY: imported by ``tests/`` as the checker for the
engine's ``rcwa_slab_smatrix_batched`` / ``rcwa_star_product_batched``; the
product never calls it.

Restates, in NumPy:

* ``dtmm::RCWAScatterMatrix::compute_v2`` (rcwa/RCWAScatterMatrix.cpp:90-146):
  the symmetric S-matrix of one z-uniform slab (modes W, V, gamma) seen from a
  reference medium (W0, V0).  ``Rdu() == Rud()`` and ``Tdd() == Tuu()``
  (rcwa/RCWAScatterMatrix.h:40-47).
* the Redheffer star product of the z-integrators
  (core/RCWAIntegrator.cpp:57-67, core/RedhefferIntegrator.cpp:136-146).

Eigen's ``PartialPivLU::solve`` / ``inverse`` map to ``numpy.linalg.solve`` /
``numpy.linalg.inv`` (LAPACK getrf/getrs/getri).
"""
from __future__ import annotations

import math

import numpy as np


def slab_smatrix(W, V, gamma, W0, V0, lam, wz):
    """(Rud, Tuu) of a slab of thickness ``wz`` at wavelength ``lam``.

    rcwa/RCWAScatterMatrix.cpp:113-146: X = exp(i gamma wz/k0) with
    wz/k0 = lam/(2 pi) * wz (:114-117); F0 = W^-1 W0, G0 = V^-1 V0 (:119-126);
    A = F0 + G0, B = F0 - G0 (:128-129); invAB, invAXA, invAXB (:131-136);
    Rud = (I - invAXB^2)^-1 (invAXB invAXA - invAB) (:139-144);
    Tuu = (I - invAXB^2)^-1 (invAXA - invAXB invAB) (:145-146).
    """
    n = W.shape[0]
    ss = lam / (2.0 * math.pi) * wz
    X = np.exp(1j * np.asarray(gamma) * ss)
    F0 = np.linalg.solve(W, W0)
    G0 = np.linalg.solve(V, V0)
    A = F0 + G0
    B = F0 - G0
    invAB = np.linalg.solve(A, B)
    invAXA = np.linalg.solve(A, X[:, None] * A)
    invAXB = np.linalg.solve(A, X[:, None] * B)
    M = np.eye(n) - invAXB @ invAXB
    Rud = np.linalg.solve(M, invAXB @ invAXA - invAB)
    Tuu = np.linalg.solve(M, invAXA - invAXB @ invAB)
    return Rud, Tuu


def star_product(S, s):
    """Accumulate slab ``s`` below the running S-matrix ``S``.

    ``S`` and ``s`` are dicts with keys Rud, Rdu, Tdd, Tuu.  Follows
    core/RCWAIntegrator.cpp:57-67: C1 = (I - rdu Rud)^-1 (explicit inverse),
    C2 = I + Rud C1 rdu, then Rdu += Tdd rdu C2 Tuu, Tdd = Tdd C1 tdd,
    Rud = rud + tuu Rud C1 tdd, Tuu = tuu C2 Tuu (all with the old values).
    """
    n = S["Rud"].shape[0]
    I = np.eye(n)
    C1 = np.linalg.inv(I - s["rdu"] @ S["Rud"])
    C2 = I + S["Rud"] @ C1 @ s["rdu"]
    return {
        "Rdu": S["Rdu"] + S["Tdd"] @ s["rdu"] @ C2 @ S["Tuu"],
        "Tdd": S["Tdd"] @ C1 @ s["tdd"],
        "Rud": s["rud"] + s["tuu"] @ S["Rud"] @ C1 @ s["tdd"],
        "Tuu": s["tuu"] @ C2 @ S["Tuu"],
    }


def identity_smatrix(n):
    """Start of the cascade (core/RCWAIntegrator.cpp:36-39)."""
    I = np.eye(n, dtype=complex)
    Z = np.zeros((n, n), dtype=complex)
    return {"Tdd": I.copy(), "Tuu": I.copy(), "Rud": Z.copy(), "Rdu": Z.copy()}
