"""Learned surrogate of the RCWA efficiencies, with the engine's solve as its
fallback and the reference for its error.

The network (rcwa_mlp_*: GPU training and tensor-core inference) maps eleven
grating parameters -- fill_x, fill_y, thickness, Re/Im eps1, eps2, lambda,
theta, phi, period_x, period_y -- of a one-rectangle 2D grating (superstrate
eps 1, substrate eps 2.25) to the TE reflection and transmission efficiencies
of the 25 lowest orders (m, n in [-2, 2]^2) and the total R and T (52 outputs).
Training data come from this engine's FP64 solve.  A query goes to the
engine instead of the network when

* it lies outside the training data (the hull check): a parameter outside the
  training set's range, or a squared feature-space distance to the nearest
  training row above the ``hull_quantile`` of the training rows' own
  leave-one-out nearest-neighbour distances (a GPU brute-force search),
* the stack is lossless (Im eps1 = 0, eps2 real) and the predicted total
  R + T misses 1 by more than ``energy_tol`` (1e-3),
* it is drawn for the random audit (``audit`` fraction, 2% by default); the
  audited rows report the network's error against the solve.

Fallbacks and audits run through the mixed-precision engine by default
(``fallback_precision``): within 1e-4 of the FP64 solve and faster, which is
what lets a surrogate with a 2% audit approach a 100x speed-up at all.
"""
from __future__ import annotations

import math
from typing import Dict, Optional

import numpy as np

from .abi import Engine, Mlp, RCWA_PREC_FP64, RCWA_PREC_MIXED
from .workloads import pol_vectors, rect_stack

PARAMS = ("fill_x", "fill_y", "thickness", "eps_re", "eps_im", "eps2", "lambda", "theta", "phi", "period_x",
          "period_y")
RANGES = np.array([(0.2, 0.8), (0.2, 0.8), (50e-9, 300e-9), (2.0, 12.0), (0.0, 0.5), (1.0, 2.0),
                   (400e-9, 800e-9), (0.0, 60.0), (0.0, 90.0), (350e-9, 450e-9), (350e-9, 450e-9)])
N_LOW = 2  # orders m, n in [-N_LOW, N_LOW]
N_OUT = 2 * (2 * N_LOW + 1) ** 2 + 2
SOURCE_NET, SOURCE_HULL, SOURCE_ENERGY, SOURCE_AUDIT = 0, 1, 2, 3


def sample(n: int, rng: np.random.Generator, ranges: np.ndarray = RANGES) -> np.ndarray:
    """Uniform parameter rows (n x 11) over ``ranges``."""
    lo, hi = ranges[:, 0], ranges[:, 1]
    return lo + (hi - lo) * rng.random((n, len(PARAMS)))


def _order_index(nh: int) -> np.ndarray:
    """Positions of the orders (m, n), m, n in [-N_LOW, N_LOW], in the engine's
    order layout k = (2 nh + 1)(m + nh) + (n + nh)."""
    w = 2 * nh + 1
    return np.array([w * (m + nh) + (k + nh) for m in range(-N_LOW, N_LOW + 1) for k in range(-N_LOW, N_LOW + 1)])


def solve(eng: Engine, P: np.ndarray, nh: int, chunk: int = 512, precision: int = RCWA_PREC_FP64) -> np.ndarray:
    """The 52 targets of every parameter row by the engine's solve (TE)."""
    if nh < N_LOW:
        raise ValueError(f"nh must be at least {N_LOW}")
    sel = _order_index(nh)
    out = np.zeros((P.shape[0], N_OUT))
    for c0 in range(0, P.shape[0], chunk):
        rows = P[c0:c0 + chunk]
        stacks, pts, pxy = [], [], []
        for i, p in enumerate(rows):
            fx, fy, d, er, ei, e2, lam, th, ph, px, py = p
            stacks.append(rect_stack(nh, nh, px, py, [(complex(er, ei), complex(e2, 0.0), fx, fy, d)]))
            k0 = 2 * math.pi / lam
            st = math.sin(math.radians(th))
            pts.append((i, lam, k0 * st * math.cos(math.radians(ph)), k0 * st * math.sin(math.radians(ph))))
            te, _ = pol_vectors(th, ph)
            pxy.append([te])
        R, T, REF, TRN, status = eng.solve_batch(stacks, np.array(pts), np.array(pxy, dtype=complex),
                                                  orders=True, precision=precision)
        if np.any(status):
            raise RuntimeError(f"solve status {status[status != 0][:4]}")
        for i in range(len(rows)):
            out[c0 + i, :25] = REF[i][0][sel]
            out[c0 + i, 25:50] = TRN[i][0][sel]
            out[c0 + i, 50] = R[i, 0]
            out[c0 + i, 51] = T[i, 0]
    return out


class Surrogate:
    def __init__(self, eng: Engine, nh: int, hidden: int = 256, layers: int = 4, seed: int = 0,
                 fallback_precision: int = RCWA_PREC_MIXED):
        self.eng, self.nh = eng, nh
        self.net = Mlp(eng, len(PARAMS), hidden, layers, N_OUT, seed=seed)
        self.lo: Optional[np.ndarray] = None
        self.hi: Optional[np.ndarray] = None
        self.fallback_precision = fallback_precision
        self.hull_d2: Optional[float] = None

    def features(self, P: np.ndarray) -> np.ndarray:
        """Parameters scaled to [-1, 1] over the training range."""
        span = np.where(self.hi > self.lo, self.hi - self.lo, 1.0)
        return (2.0 * (P - self.lo) / span - 1.0).astype(np.float32)

    def fit(self, P: np.ndarray, Y: np.ndarray, epochs: int = 60, batch: int = 256, lr: float = 2e-3,
            seed: int = 0, hull_quantile: float = 0.999, hull_sample: int = 8192) -> np.ndarray:
        """Train on parameter rows P and their solved targets Y; returns the
        per-epoch loss.  The hull threshold is the ``hull_quantile`` of the
        leave-one-out nearest-neighbour distances of ``hull_sample`` training
        rows."""
        self.lo, self.hi = P.min(axis=0), P.max(axis=0)
        F = self.features(P)
        self.net.set_data(F, Y.astype(np.float32))
        rng = np.random.default_rng(seed)
        pick = rng.choice(len(F), size=min(hull_sample, len(F)), replace=False)
        self.hull_d2 = float(np.quantile(self.net.nn_distance(F[pick], skip_self=True), hull_quantile))
        return self.net.train(epochs, batch, lr, seed)

    def predict(self, P: np.ndarray) -> np.ndarray:
        """The network alone (BF16 on the tensor cores)."""
        return self.net.predict(self.features(P), tensor_cores=True).astype(np.float64)

    def query(self, P: np.ndarray, audit: float = 0.02, energy_tol: float = 1e-3,
              seed: int = 0) -> Dict[str, np.ndarray]:
        """Network answers with the solve as fallback.  Returns the targets, the
        source of every row (SOURCE_*) and, for the audited rows, the largest
        absolute difference between network and solve."""
        Y = self.predict(P)
        src = np.full(P.shape[0], SOURCE_NET)
        outside = np.any((P < self.lo) | (P > self.hi), axis=1)
        if self.hull_d2 is not None:
            outside |= self.net.nn_distance(self.features(P)) > self.hull_d2
        src[outside] = SOURCE_HULL
        lossless = (P[:, 4] == 0.0)
        bad_energy = lossless & (np.abs(Y[:, 50] + Y[:, 51] - 1.0) > energy_tol) & (src == SOURCE_NET)
        src[bad_energy] = SOURCE_ENERGY
        rng = np.random.default_rng(seed)
        audited = (rng.random(P.shape[0]) < audit) & (src == SOURCE_NET)
        src[audited] = SOURCE_AUDIT
        fall = src != SOURCE_NET
        audit_err = np.zeros(0)
        if np.any(fall):
            Ys = solve(self.eng, P[fall], self.nh, chunk=4096, precision=self.fallback_precision)
            idx = np.nonzero(fall)[0]
            aud = src[idx] == SOURCE_AUDIT
            audit_err = np.max(np.abs(Y[idx[aud]] - Ys[aud]), axis=1) if np.any(aud) else np.zeros(0)
            Y[idx] = Ys
        return {"Y": Y, "source": src, "audit_err": audit_err}

    def close(self):
        self.net.close()
