"""Sampled z-varying structures for the z-integrator tests: a small
dielectric waveguide cross-section (a core in cladding, 7 x 5 harmonics,
periodic boundaries) whose core's right edge moves with depth, sampled like
VarLayerSampler::sample (core/VarLayerSampler.cpp:52-68: the edges at depth z,
then Layer::waveEqnCoeff with LayerSampler's Kx, Ky, core/LayerSampler.cpp:9-31)
through the oracle's restatement of waveEqnCoeff."""
import math

import numpy as np

import oracle.rcwa_oracle as orc

Z0, Z1 = -0.1, 1.1
NX, NY = 7, 5
LAM = 1.55
XE = np.array([0.0, 0.5, 1.5, 2.6, 3.7, 3.9, 5.0, 5.5])
YE = np.array([0.0, 0.5, 1.5, 1.58, 1.8, 2.8, 3.3])


def _eps():
    cl, co = 1.445 ** 2, 3.48 ** 2
    eps = np.full((len(YE) - 1, len(XE) - 1), cl, dtype=complex)
    eps[3, 2] = co
    return eps


def sample(z, moving):
    """(P, Q) at depth z; with `moving` the edge x[3] goes 2.6 -> 3.7 over z in [0, 1]."""
    x = XE.copy()
    if moving:
        x[3] = 2.6 if z < 0 else (3.7 if z > 1 else (1 - z) * 2.6 + z * 3.7)
    Lx, Ly = XE[-1] - XE[0], YE[-1] - YE[0]
    # LayerSampler::evaluateAlphaBeta: mode ny*i + j, no Bloch offset
    alpha, beta = orc.alpha_beta(NX, NY, Lx, Ly, 0.0, 0.0)
    P, Q, _, _, _ = orc.wave_eqn_coeff(x, YE, _eps(), alpha, beta, LAM, NX, NY)
    return P, Q


def samples(nslab, moving, z0=Z0, z1=Z1):
    """P, Q stacked as [nslab + 2, n, n]: z0, the slab midpoints, z1."""
    dz = (z1 - z0) / nslab if nslab > 0 else 0.0
    zs = [z0] + [z0 + (i + 0.5) * dz for i in range(nslab)] + [z1]
    PQ = [sample(z, moving) for z in zs]
    return np.array([p for p, _ in PQ]), np.array([q for _, q in PQ])


def half_step_samples(nslab, moving, z0=Z0, z1=Z1):
    """P, Q stacked as [2 nslab + 1, n, n] at z0 + k dz/2 (the differential
    integrator's left ends, midpoints and right ends)."""
    dz = (z1 - z0) / nslab
    PQ = [sample(z0 + k * dz / 2, moving) for k in range(2 * nslab + 1)]
    return np.array([p for p, _ in PQ]), np.array([q for _, q in PQ])
