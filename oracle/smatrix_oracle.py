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
* RCWAIntegrator::compute (core/RCWAIntegrator.cpp:21-86) over sampled P, Q.
* DifferentialIntegrator::compute (core/DifferentialIntegrator.cpp:21-133).
* RedhefferIntegrator::compute (core/RedhefferIntegrator.cpp:190-328), the
  adaptive triple division, with the sampler called back for new depths.

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


def wave_equation_modes(P, Q):
    """WaveEquationSolver::solve (rcwa/WaveEquationSolver.cpp:24-37) with
    LAPACK's zgeev: W = eigenvectors of P Q, keff = GammaSqrtOp(eigenvalues),
    V = Q W keff^-1."""
    from oracle.rcwa_oracle import gamma_sqrt
    lam, W = np.linalg.eig(P @ Q)
    keff = gamma_sqrt(lam)
    V = (Q @ W) / keff[None, :]
    return W, V, keff


def rcwa_integrate(P, Q, lam, z0, z1):
    """RCWAIntegrator::compute (core/RCWAIntegrator.cpp:21-86) over given samples.

    ``P[k], Q[k]`` are the sampler's matrices (LayerSampler::sample) at the
    depths z0 (k = 0), the midpoints z0 + (i + 1/2) dz of the N = len(P) - 2
    slabs (k = 1 .. N, dz = (z1 - z0) / N) and z1 (k = N + 1).  Every slab's
    S-matrix is taken against the modes at z1 (:28-34, :49-50), the slabs are
    cascaded from the top down with the star product (:36-68), and the last
    step brings the top side into the modes at z0 (:70-85).  Returns a dict
    with Tdd, Tuu, Rud, Rdu, W0, V0, gam0, W1, V1, gam1.
    """
    N = len(P) - 2
    W1, V1, g1 = wave_equation_modes(P[N + 1], Q[N + 1])
    n = W1.shape[0]
    S = identity_smatrix(n)
    dz = (z1 - z0) / N if N > 0 else 0.0
    for i in range(N):
        W, V, g = wave_equation_modes(P[1 + i], Q[1 + i])
        rud, tuu = slab_smatrix(W, V, g, W1, V1, lam, dz)
        S = star_product(S, {"rud": rud, "rdu": rud, "tdd": tuu, "tuu": tuu})
    W0, V0, g0 = wave_equation_modes(P[0], Q[0])
    F = np.linalg.solve(W1, W0)
    G = np.linalg.solve(V1, V0)
    A = 0.5 * (F + G)
    B = 0.5 * (F - G)
    M = A - S["Rdu"] @ B
    Rdu = np.linalg.solve(M, S["Rdu"] @ A - B)
    Tdd = np.linalg.solve(M, S["Tdd"])
    Rud = S["Tuu"] @ B @ Tdd + S["Rud"]
    Tuu = S["Tuu"] @ (B @ Rdu + A)
    return {"Tdd": Tdd, "Tuu": Tuu, "Rud": Rud, "Rdu": Rdu, "W0": W0, "V0": V0, "gam0": g0,
            "W1": W1, "V1": V1, "gam1": g1}


def field_space(out):
    """The integrator's S-blocks as operators on tangential fields, free of the
    eigenvectors' order, scale and phase: W0 Tdd W1^-1, W1 Tuu W0^-1,
    W1 Rud W1^-1, W0 Rdu W0^-1 (Tdd and Rdu act on the z0 side on the left,
    Tuu and Rud on the z1 side)."""
    W0, W1 = out["W0"], out["W1"]
    i0, i1 = np.linalg.inv(W0), np.linalg.inv(W1)
    return {"Tdd": W0 @ out["Tdd"] @ i1, "Tuu": W1 @ out["Tuu"] @ i0,
            "Rud": W1 @ out["Rud"] @ i1, "Rdu": W0 @ out["Rdu"] @ i0}


def _top_projection(S, W1, V1, W0, V0):
    """The last step of RCWAIntegrator / DifferentialIntegrator::compute
    (core/RCWAIntegrator.cpp:73-85, core/DifferentialIntegrator.cpp:116-133):
    the cascade, built in the modes at z1, brought into the modes at z0."""
    F = np.linalg.solve(W1, W0)
    G = np.linalg.solve(V1, V0)
    A = 0.5 * (F + G)
    B = 0.5 * (F - G)
    M = A - S["Rdu"] @ B
    Rdu = np.linalg.solve(M, S["Rdu"] @ A - B)
    Tdd = np.linalg.solve(M, S["Tdd"])
    Rud = S["Tuu"] @ B @ Tdd + S["Rud"]
    Tuu = S["Tuu"] @ (B @ Rdu + A)
    return {"Tdd": Tdd, "Tuu": Tuu, "Rud": Rud, "Rdu": Rdu}


def differential_integrate(P, Q, lam, z0, z1):
    """DifferentialIntegrator::compute (core/DifferentialIntegrator.cpp:21-133).

    ``P[k], Q[k]`` are the sampler's matrices at z0 + k dz/2, k = 0 .. 2N
    (dz = (z1 - z0) / N): every slab i takes its left end (2i), midpoint
    (2i + 1) and right end (2i + 2).  The modes at z0 and z1 are those of
    samples 0 and 2N.  Per slab the fourth-order transfer blocks L11, L12,
    L21, L22 (:55-66) are taken into the modes at z1 (:73-86), turned into an
    S-matrix (:93-97) and cascaded with the star product (:104-114).
    """
    N = (len(P) - 1) // 2
    W1, V1, g1 = wave_equation_modes(P[2 * N], Q[2 * N])
    W0, V0, g0 = wave_equation_modes(P[0], Q[0])
    n = W1.shape[0]
    k0 = 2 * math.pi / lam
    dz = (z1 - z0) / N
    I = np.eye(n)
    S = identity_smatrix(n)
    c = dz * dz / (k0 * k0)
    for i in range(N):
        P0, P1, P2 = P[2 * i], P[2 * i + 1], P[2 * i + 2]
        Q0, Q1, Q2 = Q[2 * i], Q[2 * i + 1], Q[2 * i + 2]
        L11 = I - c / 6 * (P1 @ Q0 + P1 @ Q1 + P2 @ Q1 - c / 4 * P2 @ Q1 @ P1 @ Q0)
        L12 = 1j * dz / (6 * k0) * (P0 + 4 * P1 + P2 - c / 2 * (P1 @ Q1 @ P0 + P2 @ Q1 @ P1))
        L21 = 1j * dz / (6 * k0) * (Q0 + 4 * Q1 + Q2 - c / 2 * (Q1 @ P1 @ Q0 + Q2 @ P1 @ Q1))
        L22 = I - c / 6 * (Q1 @ P0 + Q1 @ P1 + Q2 @ P1 - c / 4 * Q2 @ P1 @ Q1 @ P0)
        wl11, wl12 = np.linalg.solve(W1, L11), np.linalg.solve(W1, L12)
        vl21, vl22 = np.linalg.solve(V1, L21), np.linalg.solve(V1, L22)
        A11, A12 = 0.5 * (wl11 + vl21), 0.5 * (wl12 + vl22)
        A21, A22 = 0.5 * (wl11 - vl21), 0.5 * (wl12 - vl22)
        T11 = A11 @ W1 + A12 @ V1
        T12 = A11 @ W1 - A12 @ V1
        T21 = A21 @ W1 + A22 @ V1
        T22 = A21 @ W1 - A22 @ V1
        tdd = np.linalg.inv(T22)
        rud = T12 @ tdd
        rdu = -np.linalg.solve(T22, T21)
        tuu = T11 + T12 @ rdu
        S = star_product(S, {"rud": rud, "rdu": rdu, "tdd": tdd, "tuu": tuu})
    out = _top_projection(S, W1, V1, W0, V0)
    out.update({"W0": W0, "V0": V0, "gam0": g0, "W1": W1, "V1": V1, "gam1": g1})
    return out


def _perturbation(sample, z0, z1, lam, P0, Q0, P1, Q1, Pr, Qr, W, V, gam):
    """RedhefferIntegrator::evaluatePerturbationAndDifference
    (core/RedhefferIntegrator.cpp:330-398): first-order S-matrix of [z0, z1]
    around the reference modes (W, V, gam) of the interval's midpoint, by
    Simpson's rule; the midpoint term vanishes (the midpoint sample is the
    reference).  Returns (tdd, tuu, rud, rdu, diffError)."""
    k0 = 2 * math.pi / lam
    L = z1 - z0
    dA, dB = [], []
    for Pk, Qk in ((P0, Q0), (P1, Q1)):
        x = np.linalg.solve(W, (Pk - Pr) @ V)
        y = np.linalg.solve(V, (Qk - Qr) @ W)
        dA.append(x + y)
        dB.append(x - y)
    pf = np.exp(1j * L / k0 * gam)
    c = 1j * L / (6 * 2 * k0)
    tuu = c * (pf[:, None] * dA[0] + dA[1] * pf[None, :])
    rud = -c * (pf[:, None] * dB[0] * pf[None, :] + dB[1])
    rdu = -c * (dB[0] + pf[:, None] * dB[1] * pf[None, :])
    tdd = c * (dA[0] * pf[None, :] + pf[:, None] * dA[1])
    err = max(np.abs(m).max() for m in (tuu, rud, rdu, tdd))
    return tdd + np.diag(pf), tuu + np.diag(pf), rud, rdu, err


def redheffer_integrate(sample, lam, z0, z1, pe, max_intervals=100000):
    """RedhefferIntegrator::compute (core/RedhefferIntegrator.cpp:190-328,
    the triple-division branch): an interval whose perturbation S-matrix
    (around its midpoint's modes) has an entry above ``pe`` is split into
    thirds, the middle third keeping the parent's reference; accepted
    intervals are projected from the previous interval's modes and cascaded
    from the top down; the bottom is brought into the modes at z1.
    ``sample(z)`` returns (P, Q).  Returns the dict of rcwa_integrate plus
    N (accepted intervals) and nEigVal (eigen-solves)."""
    cache = {}

    def smp(z):
        if z not in cache:
            cache[z] = sample(z)
        return cache[z]

    P0, Q0 = smp(z0)
    P1, Q1 = smp(z1)
    W0, V0, g0 = wave_equation_modes(P0, Q0)
    W1, V1, g1 = wave_equation_modes(P1, Q1)
    zm = 0.5 * (z0 + z1)
    Pm, Qm = smp(zm)
    Wm, Vm, gm = wave_equation_modes(Pm, Qm)
    n = W0.shape[0]
    state = {"S": identity_smatrix(n), "leftW": W0, "leftV": V0, "N": 0, "nEig": 3}

    def accept(s, W, V):
        tdd, tuu, rud, rdu = s
        F = np.linalg.solve(W, state["leftW"])
        G = np.linalg.solve(V, state["leftV"])
        A, B = 0.5 * (F + G), 0.5 * (F - G)
        M = A - rdu @ B
        rdu = np.linalg.solve(M, rdu @ A - B)
        tdd = np.linalg.solve(M, tdd)
        rud = tuu @ B @ tdd + rud
        tuu = tuu @ A + tuu @ B @ rdu
        state["leftW"], state["leftV"] = W, V
        state["S"] = star_product(state["S"], {"rud": rud, "rdu": rdu, "tdd": tdd, "tuu": tuu})
        state["N"] += 1

    def rec(Pr, Qr, W, V, g, za, zb, Pa, Qa, Pb, Qb):
        tdd, tuu, rud, rdu, err = _perturbation(None, za, zb, lam, Pa, Qa, Pb, Qb, Pr, Qr, W, V, g)
        if err <= pe:
            if state["N"] >= max_intervals:
                raise RuntimeError("interval limit")
            accept((tdd, tuu, rud, rdu), W, V)
            return
        zm0 = 2.0 / 3.0 * za + 1.0 / 3.0 * zb
        zm1 = 1.0 / 3.0 * za + 2.0 / 3.0 * zb
        Pt, Qt = smp(0.5 * (za + zm0))
        Pk, Qk = smp(zm0)
        Wt, Vt, gt = wave_equation_modes(Pt, Qt)
        state["nEig"] += 1
        rec(Pt, Qt, Wt, Vt, gt, za, zm0, Pa, Qa, Pk, Qk)
        Pt2, Qt2 = smp(zm1)
        rec(Pr, Qr, W, V, g, zm0, zm1, Pk, Qk, Pt2, Qt2)
        Pk2, Qk2 = smp(0.5 * (zm1 + zb))
        Wk, Vk, gk = wave_equation_modes(Pk2, Qk2)
        state["nEig"] += 1
        rec(Pk2, Qk2, Wk, Vk, gk, zm1, zb, Pt2, Qt2, Pb, Qb)

    rec(Pm, Qm, Wm, Vm, gm, z0, z1, P0, Q0, P1, Q1)
    # the bottom into the modes at z1 (:235-245)
    S = state["S"]
    F = np.linalg.solve(state["leftW"], W1)
    G = np.linalg.solve(state["leftV"], V1)
    A, B = 0.5 * (F + G), 0.5 * (F - G)
    M = A - S["Rud"] @ B
    Tuu = np.linalg.solve(M, S["Tuu"])
    Rud = np.linalg.solve(M, S["Rud"] @ A - B)
    Rdu = S["Rdu"] + S["Tdd"] @ B @ Tuu
    Tdd = S["Tdd"] @ (B @ Rud + A)
    return {"Tdd": Tdd, "Tuu": Tuu, "Rud": Rud, "Rdu": Rdu, "W0": W0, "V0": V0, "gam0": g0,
            "W1": W1, "V1": V1, "gam1": g1, "N": state["N"], "nEigVal": state["nEig"]}
