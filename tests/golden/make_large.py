"""Golden fixtures at the benchmark sizes, generated with the CPU oracle.

pillars_nh10_points.npz: three points (0, 77, 147) of the first 148-point batch
  of the 2D pillar sweep workloads.pillars_2d(seed=0, nH=10) -- Nx=Ny=10, 441
  orders, 882 x 882 layer matrices, five lossy patterned layers, conical
  incidence -- with R, T and the per-order REF/TRN of TE and TM.
uneven_sample.npz: instances of workloads.uneven_batch(seed=0) at their real
  sizes (nH up to 15, up to 6 layers): eight all-dielectric instances, and
  four with metal or above-resonance Lorentz layers solved twice by the
  oracle (LU solves, then SVD least-squares solves); `sane` marks those whose
  two oracle answers agree to 1e-10 and keep R + T <= 1, the ones on which the
  reference's own arithmetic is trustworthy.

Takes several minutes (LAPACK zgeev on 882..1922-row matrices).
Run: python tests/golden/make_large.py
"""
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle.rcwa_oracle import OracleLayer, RCWASolver  # noqa: E402
from openrcwa_b200 import workloads  # noqa: E402

PILLAR_POINTS = [0, 77, 147]
UNEVEN_DIELECTRIC = [1, 37, 57, 280, 361, 556, 572, 603]
UNEVEN_METAL = [5, 6, 7, 11]


def oracle_point(st, pt, pxy, lstsq=False):
    """R, T [n_exc] and REF, TRN [n_exc, N] of one point through the oracle's
    RCWASolver (rcwa/RCWASolver.cpp:139-148, 1778-1908)."""
    s = RCWASolver(st.nHx, st.nHy, lstsq=lstsq)
    L = st.eps.shape[0]
    for l in range(L):
        s.addLayer(OracleLayer(st.cx, st.cy, st.eps[l]))
    s.setBlochWavevector(pt[2], pt[3])
    s.solve(pt[1], list(range(L)), list(st.thickness))
    k0 = 2 * math.pi / pt[1]
    R, T, REF, TRN = [], [], [], []
    for e in range(pxy.shape[0]):
        c = s.generateHorizontalPlaneWave(pxy[e, 0], pxy[e, 1], 0)
        ref, trn = s.scatterPlaneWave(c, 0, L - 1, k0)
        R.append(ref.sum())
        T.append(trn.sum())
        REF.append(ref)
        TRN.append(trn)
    return np.array(R), np.array(T), np.array(REF), np.array(TRN)


def pillars():
    stacks, pts, pxy = workloads.pillars_2d(seed=0, nH=10)
    out = [oracle_point(stacks[0], pts[p], pxy[p]) for p in PILLAR_POINTS]
    np.savez_compressed(os.path.join(HERE, "pillars_nh10_points.npz"), points=np.array(PILLAR_POINTS),
                        R=np.array([o[0] for o in out]), T=np.array([o[1] for o in out]),
                        REF=np.array([o[2] for o in out]), TRN=np.array([o[3] for o in out]))
    print("pillars_nh10_points")


def uneven():
    ids = UNEVEN_DIELECTRIC + UNEVEN_METAL
    stacks, pts, pxy = workloads.uneven_batch(seed=0, n_instances=max(ids) + 1)
    R, T, R2, T2, sane = [], [], [], [], []
    REF, TRN = {}, {}
    for i in ids:
        r, t, ref, trn = oracle_point(stacks[i], pts[i], pxy[i])
        R.append(r)
        T.append(t)
        REF["REF_%d" % i] = ref
        TRN["TRN_%d" % i] = trn
        if i in UNEVEN_METAL:
            r2, t2, _, _ = oracle_point(stacks[i], pts[i], pxy[i], lstsq=True)
        else:
            r2, t2 = r, t
        R2.append(r2)
        T2.append(t2)
        ok = (np.max(np.abs(r - r2)) < 1e-10 and np.max(np.abs(t - t2)) < 1e-10 and np.all(r + t <= 1 + 1e-9)
              and np.all(r >= -1e-12) and np.all(t >= -1e-12))
        sane.append(ok)
        print(i, stacks[i].nHx, stacks[i].eps.shape[0] - 2, r + t, ok, flush=True)
    np.savez_compressed(os.path.join(HERE, "uneven_sample.npz"), ids=np.array(ids),
                        metal=np.array([i in UNEVEN_METAL for i in ids]), R=np.array(R), T=np.array(T),
                        R_lstsq=np.array(R2), T_lstsq=np.array(T2), sane=np.array(sane), **REF, **TRN)
    print("uneven_sample")


if __name__ == "__main__":
    which = sys.argv[1:] or ["pillars", "uneven"]
    if "pillars" in which:
        pillars()
    if "uneven" in which:
        uneven()
