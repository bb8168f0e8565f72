"""CPU oracle for the RCWA diffraction-efficiency hot path.

TEST INFRASTRUCTURE ONLY.  This module is the checker that the CUDA engine is
compared against; only ``tests/``, ``__graft_entry__.smoke()`` and the CPU
baseline legs of ``bench.py`` may import it.  The product path (the C-ABI
library under ``openrcwa_b200/``) never calls it and has no CPU fallback.

It restates, in NumPy, the plain (non-PML, non-magnetic) RCWA solve of
Sirokujira/OpenRCWA on the LAPACKE eigen-solver branch.  Every function names
the reference lines it follows.  Eigen decompositions used by the reference map
to LAPACK equivalents:

* ``BDCSVD::solve`` / ``CompleteOrthogonalDecomposition::solve`` (minimum-norm
  least squares) -> ``numpy.linalg.solve`` for the full-rank square systems met
  on this path (identical up to rounding); ``lstsq=True`` switches to the
  SVD-based minimum-norm solve for cross-checks.
* ``PartialPivLU::inverse`` -> ``numpy.linalg.inv`` (LAPACK getrf/getri).
* ``LAPACKE_zgeev('N','V')`` -> ``numpy.linalg.eig`` (LAPACK zgeev).

Units follow the reference: lengths in metres (``.ofd`` path), wavenumbers in
rad/m, permittivities relative, time convention exp(-i w t).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

C0 = 2.99792458e8  # sol/rcwa_bridge.cpp:44
PI = 3.1415926535897932  # rcwa/defns.h:25 (the reference's own constant)

ContinuousXY, DiscontinuousX, DiscontinuousY = 0, 1, 2  # rcwa/FourierSolver2D.h:8-13


# --------------------------------------------------------------------------
# Fourier coefficients (rcwa/FourierSolver1D.cpp:11-41, rcwa/MathFunction.h:6-9)
# --------------------------------------------------------------------------
def sinc(x: np.ndarray) -> np.ndarray:
    """sin(pi x)/(pi x) with sinc(0)=1 (rcwa/MathFunction.h:6-9)."""
    x = np.asarray(x, dtype=np.float64)
    out = np.ones_like(x)
    nz = x != 0.0
    out[nz] = np.sin(PI * x[nz]) / (PI * x[nz])
    return out


def fourier1d(x: Sequence[float], d: float, f: Sequence[complex], M: int) -> np.ndarray:
    """FourierSolver1D::solve (rcwa/FourierSolver1D.cpp:11-41).

    F_m = sum_cells f_c/d * (x1-x0) * exp(-i pi m (x1+x0)/d) * sinc(m (x1-x0)/d),
    m = i - (M-1)/2 for i in [0, M).  The m = 0 term is f_c/d*(x1-x0).
    """
    x = np.asarray(x, dtype=np.float64)
    f = np.asarray(f, dtype=np.complex128)
    assert f.size == x.size - 1, "function configuration does not match coordinates"
    m = (np.arange(M) - (M - 1) // 2).astype(np.float64)[:, None]
    x0 = x[:-1][None, :]
    x1 = x[1:][None, :]
    w = x1 - x0
    ph = np.exp(-1j * (m * PI * (x1 + x0) / d))
    term = f[None, :] / d * ph * sinc(m * w / d) * w
    m0 = (m[:, 0] == 0)
    term[m0, :] = (f[None, :] / d * w)[0]
    return term.sum(axis=1)


def toeplitz_dense(vec: np.ndarray) -> np.ndarray:
    """ToeplitzMatrixXcs(vec).toDense(): T(r,c) = vec[n-1+r-c]
    (rcwa/ToeplitzMatrixXcs.cpp:8-44)."""
    n = (vec.size + 1) // 2
    r = np.arange(n)[:, None]
    c = np.arange(n)[None, :]
    return vec[n - 1 + r - c]


def block_toeplitz_dense(F2D: np.ndarray) -> np.ndarray:
    """BlockToeplitzMatrixXcs(F2D).toDense() (rcwa/BlockToeplitzMatrixXcs.cpp:5-53):
    A(row,col) = F2D[(m-j)+nx-1, (n-l)+ny-1], m=row/ny, n=row%ny, j=col/ny, l=col%ny."""
    nx = (F2D.shape[0] + 1) // 2
    ny = (F2D.shape[1] + 1) // 2
    row = np.arange(nx * ny)
    m, n = row // ny, row % ny
    dm = m[:, None] - m[None, :] + nx - 1
    dn = n[:, None] - n[None, :] + ny - 1
    return F2D[dm, dn]


def _check_sorted(c: np.ndarray) -> None:
    # FourierSolver1D::reorder/refill (rcwa/FourierSolver1D.cpp:145-193) only
    # change anything for non-ascending coordinates, which the callers on this
    # path never produce (commonEdges sorts, rcwa_bridge.cpp:52-67).
    if np.any(np.diff(c) < 0):
        raise ValueError("cell coordinates must be ascending on this path")


def fourier2d(cx, cy, f: np.ndarray, nx: int, ny: int, opt: int) -> np.ndarray:
    """FourierSolver2D::solve (rcwa/FourierSolver2D.cpp:12-351).

    f has shape (len(cy)-1, len(cx)-1): row = y strip, column = x strip.
    DiscontinuousX (:43-144): per y strip, inverse of the Toeplitz matrix of the
    x-coefficients of 1/eps (Li inverse rule), Kronecker-combined with the y
    strip indicator coefficients.  DiscontinuousY (:145-249) is the transpose
    analogue.  ContinuousXY (:250-349): Laurent rule, block Toeplitz.
    """
    cx = np.asarray(cx, dtype=np.float64)
    cy = np.asarray(cy, dtype=np.float64)
    _check_sorted(cx)
    _check_sorted(cy)
    f = np.asarray(f, dtype=np.complex128)
    dx = cx[-1] - cx[0]
    dy = cy[-1] - cy[0]
    N = nx * ny
    Ff = np.zeros((N, N), dtype=np.complex128)
    if opt == DiscontinuousX:
        for i in range(cy.size - 1):
            fInv = fourier1d(cx, dx, 1.0 / f[i, :], 2 * nx - 1)
            Tinv = np.linalg.inv(toeplitz_dense(fInv))
            fY1 = fourier1d([cy[i], cy[i + 1]], dy, [1.0], 2 * ny - 1)
            # Ff(ii*ny+jj, kk*ny+ll) += fY1(jj-ll+ny-1) * Tinv(ii,kk)  (:111-142)
            Ff += np.kron(Tinv, toeplitz_dense(fY1))
    elif opt == DiscontinuousY:
        for i in range(cx.size - 1):
            fInv = fourier1d(cy, dy, 1.0 / f[:, i], 2 * ny - 1)
            Sinv = np.linalg.inv(toeplitz_dense(fInv))
            fX1 = fourier1d([cx[i], cx[i + 1]], dx, [1.0], 2 * nx - 1)
            # Ff(ii*ny+jj, kk*ny+ll) += fX1(ii-kk+nx-1) * Sinv(jj,ll)  (:221-247)
            Ff += np.kron(toeplitz_dense(fX1), Sinv)
    elif opt == ContinuousXY:
        F2D = np.zeros((2 * nx - 1, 2 * ny - 1), dtype=np.complex128)
        for i in range(cy.size - 1):
            fFi = fourier1d(cx, dx, f[i, :], 2 * nx - 1)
            fY1 = fourier1d([cy[i], cy[i + 1]], dy, [1.0], 2 * ny - 1)
            F2D += np.outer(fFi, fY1)  # :323
        Ff = block_toeplitz_dense(F2D)  # :340
    else:
        raise ValueError("unknown FourierSolverOption")
    return Ff


def circle_fourier2d(Lx: float, Ly: float, radius: float, center, eps1: complex, eps2: complex,
                     nx: int, ny: int) -> np.ndarray:
    """2D Fourier coefficients of a circular pillar (eps1 inside a disk of the
    given radius and center, eps2 elsewhere) in the unit cell [0,Lx]x[0,Ly],
    in the layout of the F2D table of FourierSolver2D's ContinuousXY branch
    (rcwa/FourierSolver2D.cpp:250-349): F2D[m+nx-1, n+ny-1] =
    (1/(Lx Ly)) * integral of eps(x,y) exp(-i 2pi (m x/Lx + n y/Ly)).

    The reference has no analytic circle: its .orcwa driver staircases curved
    shapes into rectangles, subdividing their bounding boxes into
    N_CURVED_CELLS = 8 strips per curved axis (rcwa/RCWADriver.cpp:19-37).  This is the closed form of
    the disk transform, integral over the disk of exp(-i G.r) =
    exp(-i G.c) 2 pi R^2 J1(|G| R) / (|G| R) (pi R^2 at G = 0), the Laurent
    rule for all three tensors of the circular-pillar layers."""
    from scipy.special import j1
    m = np.arange(-(nx - 1), nx)[:, None]
    n = np.arange(-(ny - 1), ny)[None, :]
    gx = 2 * PI * m / Lx
    gy = 2 * PI * n / Ly
    g = np.hypot(gx, gy)
    gr = g * radius
    with np.errstate(invalid="ignore", divide="ignore"):
        airy = np.where(gr > 0, 2 * j1(gr) / np.where(gr > 0, gr, 1.0), 1.0)
    disk = PI * radius * radius * airy * np.exp(-1j * (gx * center[0] + gy * center[1]))
    F2D = (eps1 - eps2) * disk / (Lx * Ly)
    F2D[nx - 1, ny - 1] += eps2
    return F2D.astype(np.complex128)


def circle_staircase(Lx: float, Ly: float, radius: float, center, eps1: complex, eps2: complex, cells: int):
    """A staircase of a circular pillar on a uniform cells x cells grid (a cell
    takes eps1 when its center lies in the disk), for convergence checks of
    circle_fourier2d (the reference's .orcwa driver staircases circles on a
    coarser, shape-aligned grid, rcwa/RCWADriver.cpp:19-37): returns the cell
    edges cx, cy and the (cells x cells) permittivity grid, row = y."""
    cx = np.linspace(0.0, Lx, cells + 1)
    cy = np.linspace(0.0, Ly, cells + 1)
    xm = 0.5 * (cx[1:] + cx[:-1])
    ym = 0.5 * (cy[1:] + cy[:-1])
    inside = (xm[None, :] - center[0]) ** 2 + (ym[:, None] - center[1]) ** 2 < radius * radius
    return cx, cy, np.where(inside, eps1, eps2).astype(np.complex128)


# --------------------------------------------------------------------------
# Layer eigenproblem (rcwa/Layer.cpp:75-273, rcwa/WaveEquationSolver.cpp:8-37)
# --------------------------------------------------------------------------
def gamma_sqrt(g: np.ndarray) -> np.ndarray:
    """GammaSqrtOp (rcwa/WaveEquationSolver.cpp:8-22): principal sqrt, negated if
    Im<0, then negated again if |Im|<|Re| and Re<0."""
    gv = np.sqrt(np.asarray(g, dtype=np.complex128))
    gv = np.where(gv.imag < 0, -gv, gv)
    flip = (np.abs(gv.imag) < np.abs(gv.real)) & (gv.real < 0)
    return np.where(flip, -gv, gv)


def _solve(A, B, lstsq=False):
    if lstsq:
        return np.linalg.lstsq(A, B, rcond=None)[0]
    return np.linalg.solve(A, B)


def wave_eqn_coeff(cx, cy, eps, alpha, beta, lam, nx, ny, lstsq=False, f2d=None, mu=None):
    """Layer::waveEqnCoeff (rcwa/Layer.cpp:75-253).

    Kx, Ky are the dense diagonal matrices of RCWASolver::evaluateKMatrices
    (rcwa/RCWASolver.cpp:150-185, PML disabled).  Returns (P, Q, fe11, fe22, fe33).
    With f2d (a (2nx-1) x (2ny-1) Laurent table, e.g. circle_fourier2d), the
    three convolution matrices are its block-Toeplitz matrix (the Laurent rule
    for every tensor; the reference has no such layer, it staircases curved
    shapes, rcwa/RCWADriver.cpp:19-37).
    With mu (a cell matrix like eps) that differs from 1 anywhere by more than
    1e-12 (Layer::Layer, rcwa/Layer.cpp:64-71) the magnetic branch applies:
    the permeability's three convolution matrices replace the identity in P,
    and mu_zz^-1 Kx, mu_zz^-1 Ky replace Kx, Ky in Q (:128-164, :205-213).
    """
    magnetic = mu is not None and bool(np.any(np.abs(np.asarray(mu, dtype=np.complex128) - 1.0) > 1e-12))
    if f2d is not None:
        fe11 = fe22 = fe33 = block_toeplitz_dense(np.asarray(f2d, dtype=np.complex128))
    else:
        fe11 = fourier2d(cx, cy, eps, nx, ny, DiscontinuousX)  # :102-105
        fe22 = fourier2d(cx, cy, eps, nx, ny, DiscontinuousY)  # :109-112
        fe33 = fourier2d(cx, cy, eps, nx, ny, ContinuousXY)    # :116-119
    N = nx * ny
    Kx = np.diag(np.asarray(alpha, dtype=np.complex128))
    Ky = np.diag(np.asarray(beta, dtype=np.complex128))
    F1h = _solve(fe33, Kx, lstsq)  # BDCSVD(fe33).solve(Kx)  :122-123
    F2h = _solve(fe33, Ky, lstsq)  # :124
    k0 = 2 * PI / lam
    k02 = k0 * k0
    I = np.eye(N)
    if magnetic:
        mu = np.asarray(mu, dtype=np.complex128)
        fmu11 = fourier2d(cx, cy, mu, nx, ny, DiscontinuousX)  # :132-133
        fmu22 = fourier2d(cx, cy, mu, nx, ny, DiscontinuousY)  # :135-136
        fmu33 = fourier2d(cx, cy, mu, nx, ny, ContinuousXY)    # :138-140
        G1h = _solve(fmu33, Kx, lstsq)  # :143
        G2h = _solve(fmu33, Ky, lstsq)  # :144
    else:
        fmu11 = fmu22 = I
        G1h, G2h = Kx, Ky
    P = np.empty((2 * N, 2 * N), dtype=np.complex128)
    P[:N, :N] = Kx @ F2h                   # :156
    P[:N, N:] = -Kx @ F1h + k02 * fmu22    # :157,162,167
    P[N:, :N] = Ky @ F2h - k02 * fmu11     # :158,163,168
    P[N:, N:] = -Ky @ F1h                  # :159
    Q = np.empty_like(P)
    Q[:N, :N] = -Kx @ G2h                  # :209,216
    Q[:N, N:] = Kx @ G1h - k02 * fe22      # :210,217
    Q[N:, :N] = -Ky @ G2h + k02 * fe11     # :211,218
    Q[N:, N:] = Ky @ G1h                   # :212,219
    return P, Q, fe11, fe22, fe33


def eig_residual(A, W, d):
    """Relative residual used by MKLEigenSolver (rcwa/MKLEigenSolver.hpp:66-79)."""
    nA = np.abs(A).max()
    if not nA > 0:
        return 0.0
    return float(np.abs(A @ W - W * d[None, :]).max() / nA)


def wave_equation_solve(P, Q):
    """WaveEquationSolver::solve (rcwa/WaveEquationSolver.cpp:24-37) with the
    LAPACKE zgeev branch of MKLEigenSolver (rcwa/MKLEigenSolver.hpp:102-179).

    Returns (PQ, W, V, keff, eigenvalues).  The reference switches to the
    perturbed Eigen solver when the residual exceeds 1e-8; the oracle raises
    instead so that such a case is never silently compared.
    """
    PQ = P @ Q
    lam, W = np.linalg.eig(PQ)
    if eig_residual(PQ, W, lam) > 1e-8:
        raise FloatingPointError("zgeev residual above 1e-8 (reference would fall back)")
    keff = gamma_sqrt(lam)
    V = (Q @ W) / keff[None, :]
    return PQ, W, V, keff, lam


@dataclass
class LayerSolution:
    W: np.ndarray
    V: np.ndarray
    gamma: np.ndarray  # keff / k0 (rcwa/Layer.cpp:269)
    eigenvalues: np.ndarray
    fe11: np.ndarray = None
    fe22: np.ndarray = None
    fe33: np.ndarray = None
    P: np.ndarray = None
    Q: np.ndarray = None


def layer_solve(cx, cy, eps, alpha, beta, lam, nx, ny, keep=False, lstsq=False, f2d=None, mu=None):
    """Layer::solve (rcwa/Layer.cpp:255-273)."""
    P, Q, fe11, fe22, fe33 = wave_eqn_coeff(cx, cy, eps, alpha, beta, lam, nx, ny, lstsq, f2d, mu)
    PQ, W, V, keff, ev = wave_equation_solve(P, Q)
    k0 = 2 * PI / lam
    sol = LayerSolution(W=W, V=V, gamma=keff / k0, eigenvalues=ev)
    if keep:
        sol.fe11, sol.fe22, sol.fe33, sol.P, sol.Q = fe11, fe22, fe33, P, Q
    return sol


def alpha_beta(nx, ny, Lx, Ly, kx0, ky0):
    """RCWASolver::evaluateAlphaBeta (rcwa/RCWASolver.cpp:242-266): mode k = ny*i+j."""
    Nx, Ny = (nx - 1) // 2, (ny - 1) // 2
    i = np.repeat(np.arange(nx), ny)
    j = np.tile(np.arange(ny), nx)
    alpha = (2 * PI / Lx) * (i - Nx) + kx0
    beta = (2 * PI / Ly) * (j - Ny) + ky0
    return alpha.astype(np.float64), beta.astype(np.float64)


def layer_eps_at(cx, cy, eps, x, y):
    """Layer::eps(x, y) cell lookup (rcwa/Layer.cpp:383-429)."""
    Lx = cx[-1] - cx[0]
    while x < cx[0]:
        x += Lx
    while x > cx[-1]:
        x -= Lx
    ix = next(i for i in range(len(cx) - 1) if x <= cx[i + 1])
    iy = next(j for j in range(len(cy) - 1) if y <= cy[j + 1])
    return complex(eps[iy, ix])


# --------------------------------------------------------------------------
# The solver (rcwa/RCWASolver.cpp)
# --------------------------------------------------------------------------
@dataclass
class OracleLayer:
    cx: np.ndarray
    cy: np.ndarray
    eps: np.ndarray  # (len(cy)-1, len(cx)-1)
    f2d: np.ndarray = None  # optional Laurent table replacing the cells' three rules
    mu: np.ndarray = None   # optional relative permeability per cell (None: 1)


class RCWASolver:
    """Restatement of RCWASolver with PML disabled (the path used by
    sol/rcwa_bridge.cpp:273-283 and rcwa/RCWADriver.cpp:284-333)."""

    def __init__(self, nX: int, nY: int, lstsq: bool = False):
        self.nx = 2 * nX + 1  # rcwa/RCWASolver.h:67-78
        self.ny = 2 * nY + 1
        self.layers: List[OracleLayer] = []
        self.kx0 = 0.0
        self.ky0 = 0.0
        self.lstsq = lstsq
        self.sol: List[LayerSolution] = []
        self.keep = False

    def addLayer(self, layer: OracleLayer):
        # rcwa/RCWASolver.cpp:108-137 (edge consistency; mismatches are dropped)
        if self.layers:
            a, b = self.layers[0], layer
            same = (a.cx[-1] - a.cx[0] == b.cx[-1] - b.cx[0] and a.cy[-1] - a.cy[0] == b.cy[-1] - b.cy[0]
                    and a.cx[0] == b.cx[0] and a.cx[1] == b.cx[1] and a.cx[-2] == b.cx[-2]
                    and a.cx[-1] == b.cx[-1] and a.cy[0] == b.cy[0] and a.cy[1] == b.cy[1]
                    and a.cy[-2] == b.cy[-2] and a.cy[-1] == b.cy[-1])
            if not same:
                return False
        self.layers.append(layer)
        return True

    def setBlochWavevector(self, kx0, ky0):
        self.kx0, self.ky0 = float(kx0), float(ky0)

    @property
    def Lx(self):
        return self.layers[0].cx[-1] - self.layers[0].cx[0]

    @property
    def Ly(self):
        return self.layers[0].cy[-1] - self.layers[0].cy[0]

    def solve(self, lam: float, stack: Sequence[int], thickness: Sequence[float]):
        """RCWASolver::solve (rcwa/RCWASolver.cpp:139-148)."""
        self.lam = lam
        self.alpha, self.beta = alpha_beta(self.nx, self.ny, self.Lx, self.Ly, self.kx0, self.ky0)
        # solveLayers (:194-210): every layer type, half-spaces included
        self.sol = [layer_solve(L.cx, L.cy, L.eps, self.alpha, self.beta, lam, self.nx, self.ny,
                                keep=self.keep, lstsq=self.lstsq, f2d=L.f2d, mu=L.mu) for L in self.layers]
        self._interfaces(stack)
        self._scatter_matrix(stack, thickness)

    def _interfaces(self, stack):
        """evaluateInterfaces without translation (rcwa/RCWASolver.cpp:495-571)."""
        pairs = sorted(set((stack[i], stack[i + 1]) for i in range(len(stack) - 1)))
        n = 2 * self.nx * self.ny
        self.iE, self.iH = [], []
        for (a, b) in pairs:
            if a == b:
                self.iE.append(np.eye(n, dtype=np.complex128))
                self.iH.append(np.eye(n, dtype=np.complex128))
            else:
                self.iE.append(_solve(self.sol[a].W, self.sol[b].W, self.lstsq))
                self.iH.append(_solve(self.sol[a].V, self.sol[b].V, self.lstsq))
        self.imap = [pairs.index((stack[i], stack[i + 1])) for i in range(len(stack) - 1)]

    def _scatter_matrix(self, stack, thickness):
        """evaluateScatterMatrix, RTCM cascade bottom->top (rcwa/RCWASolver.cpp:378-492)."""
        n = 2 * self.nx * self.ny
        nL = len(stack)
        Tdd = np.eye(n, dtype=np.complex128)
        Rud = np.zeros((n, n), dtype=np.complex128)
        self.taus = []  # taus_ (rcwa/RCWASolver.cpp:454), kept for the intermediate fields
        for i in range(nL - 1):
            index = nL - i - 1
            li = stack[index]
            if i == 0:
                phi = np.ones(n, dtype=np.complex128)
            else:
                phi = np.exp(1j * self.sol[li].gamma * thickness[index])  # :423
            wRud = phi[:, None] * Rud * phi[None, :]  # :433
            wTdd = Tdd * phi[None, :]                 # :434
            k = self.imap[index - 1]
            F = self.iE[k] + self.iE[k] @ wRud        # :440-441
            G = self.iH[k] - self.iH[k] @ wRud        # :442-443
            tau = np.linalg.inv(F + G)                # PartialPivLU inverse :451-453
            self.taus.append(tau)
            Rud = -2.0 * G @ tau + np.eye(n)          # :457-458
            Tdd = 2.0 * wTdd @ tau                    # :460
        self.Rud, self.Tdd = Rud, Tdd

    def evaluateIntermediateField(self, inputCoeffs, stack, thickness):
        """evaluateIntermediateField, input given as (index, value) pairs
        (rcwa/RCWASolver.cpp:1505-1644): the mode amplitudes c_m (backward)
        and c_p (forward) of every interior layer, top to bottom
        (c_m[k], c_p[k] belong to stack[k + 1]).  Eigen's PartialPivLU and
        CompleteOrthogonalDecomposition solves are LU solves here."""
        n = 2 * self.nx * self.ny
        nL = len(stack)
        if nL < 3:
            return [], []
        I = np.eye(n, dtype=np.complex128)
        S11, S12, S21, S22, phases = [], [], [], [], []
        Rud = np.zeros((n, n), dtype=np.complex128)
        REF = [Rud]
        for i in range(nL - 1):
            index = nL - i - 1
            li = stack[index]
            phase = np.ones(n, dtype=np.complex128) if i == 0 else np.exp(1j * self.sol[li].gamma * thickness[index])
            phases.append(phase)
            k = self.imap[index - 1]
            IE, IH = self.iE[k], self.iH[k]
            t11 = 0.5 * (IE + IH)
            t12 = 0.5 * (IE - IH)
            inv_t22 = np.linalg.inv(t11)
            inv_t22_t12 = np.linalg.solve(t11, t12)
            S11.append(t11 - t12 @ inv_t22_t12)
            S12.append(t12 @ inv_t22)
            S21.append(-inv_t22_t12)
            S22.append(inv_t22)
            if i == 0:
                for_inv_s22 = t11
            wRud = phase[:, None] * Rud * phase[None, :]
            G = IH - IH @ wRud
            Rud = -2.0 * G @ self.taus[i] + I
            REF.append(Rud)
        inp = np.zeros(n, dtype=np.complex128)
        for idx, v in inputCoeffs:
            inp[idx] = v
        R = self.Rud @ inp
        T = self.Tdd @ inp
        nI = nL - 2
        c_m, c_p, d = [None] * nI, [None] * nI, [None] * nI
        c_m[nI - 1] = S12[0] @ (for_inv_s22 @ T)
        temp = np.linalg.solve(S11[nL - 2], R - S12[nL - 2] @ inp)
        c_p[0] = S21[nL - 2] @ temp + S22[nL - 2] @ inp
        d[nI - 1] = phases[nL - 2] * c_p[0]
        for i in range(nI - 2, -1, -1):
            c_m[nI - i - 2] = REF[i + 2] @ d[i + 1]
            tempi = np.linalg.solve(S11[i + 1], c_m[nI - i - 2] - S12[i + 1] @ d[i + 1])
            c_p[nI - i - 1] = S21[i + 1] @ tempi + S22[i + 1] @ d[i + 1]
            d[i] = phases[i + 1] * c_p[nI - i - 1]
        return c_m, c_p

    def fieldSlice(self, sliceType, sliceCoord, component, inputCoeffs, stack, thickness, nRes1=500):
        """The field that saveFieldImage writes, before the CSV formatting
        (rcwa/RCWASolver.cpp:707-1012, no layer translation): sliceType 0 = XY
        at depth sliceCoord, 1 = XZ at y = sliceCoord, 2 = YZ at x =
        sliceCoord (z from the top of the first interior layer); component
        0..5 = Ex, Ey, Ez, Hx, Hy, Hz.  Returns the (nRes2 x nRes1) complex
        field."""
        c_m, c_p = self.evaluateIntermediateField(inputCoeffs, stack, thickness)
        if not c_m:
            return None
        L0 = self.layers[0]
        nx, ny = self.nx, self.ny
        Lx = L0.cx[-1] - L0.cx[0]
        Ly = L0.cy[-1] - L0.cy[0]
        if sliceType == 1:
            s1, L1, s2, L2 = L0.cx[0], Lx, 0.0, float(sum(thickness[1:len(stack) - 1]))
        elif sliceType == 2:
            s1, L1, s2, L2 = L0.cy[0], Ly, 0.0, float(sum(thickness[1:len(stack) - 1]))
        else:
            s1, L1, s2, L2 = L0.cx[0], Lx, L0.cy[0], Ly
        nRes2 = max(int(nRes1 * L2 / L1), 1)
        x1 = s1 + (L1 / nRes1) * (np.arange(nRes1) + 0.5)
        x2 = s2 + (L2 / nRes2) * (np.arange(nRes2) + 0.5)
        N = nx * ny
        k0 = 2 * PI / self.lam
        a = self.alpha.astype(np.complex128)
        b = self.beta.astype(np.complex128)

        def harmonics(z):
            z0, layer0 = 0.0, -1
            for j in range(1, len(stack) - 1):
                z1 = z0 + thickness[j]
                if z0 <= z <= z1:
                    layer0 = j - 1
                    break
                z0 = z1
            lt = stack[layer0 + 1]
            g = self.sol[lt].gamma
            u_p = c_p[layer0] * np.exp(1j * (z - z0) * g)
            d_m = c_m[layer0] * np.exp(-1j * (z - z1) * g)
            W, V = self.sol[lt].W, self.sol[lt].V
            if component in (0, 1):
                h = (W @ (u_p + d_m))[N * component:N * (component + 1)]
            elif component in (3, 4):
                h = (V @ (u_p - d_m))[N * (component - 3):N * (component - 2)]
            elif component == 5:
                E = W @ (u_p + d_m)
                h = 1j / (k0 * k0) * (a * E[N:] - b * E[:N])
            else:
                H = V @ (u_p - d_m)
                Ly_ = self.layers[lt]
                fe33 = fourier2d(Ly_.cx, Ly_.cy, Ly_.eps, nx, ny, ContinuousXY) if Ly_.f2d is None else \
                    block_toeplitz_dense(np.asarray(Ly_.f2d, dtype=np.complex128))
                h = 1j * np.linalg.solve(fe33, a * H[N:] - b * H[:N])
            return h.reshape(nx, ny)  # harmonics2d(i, j) = h[j + i * ny]

        mx, my = (nx - 1) // 2, (ny - 1) // 2
        m = np.arange(-mx, mx + 1)
        q = np.arange(-my, my + 1)
        field = np.zeros((nRes2, nRes1), dtype=np.complex128)
        if sliceType in (1, 2):
            for i, z in enumerate(x2):
                H2 = harmonics(z)
                if sliceType == 1:
                    one = H2 @ np.exp(1j * (2 * PI * q / Ly + self.ky0) * sliceCoord)
                    wav = np.exp(1j * np.outer(x1, 2 * PI * m / Lx + self.kx0))
                else:
                    one = H2.T @ np.exp(1j * (2 * PI * m / Lx + self.kx0) * sliceCoord)
                    wav = np.exp(1j * np.outer(x1, 2 * PI * q / Ly + self.ky0))
                field[i] = wav @ one
        else:
            H2 = harmonics(sliceCoord)
            wx = np.exp(1j * np.outer(x1, 2 * PI * m / L1 + self.kx0))   # (nRes1, nx)
            wy = np.exp(1j * np.outer(x2, 2 * PI * q / L2 + self.ky0))   # (nRes2, ny)
            field = wy @ H2.T @ wx.T
        return field

    def generateHorizontalPlaneWave(self, px, py, layerType):
        """generateHorizontalPlaneWave + Layer::generatePlaneWave
        (rcwa/RCWASolver.cpp:1778-1789, rcwa/Layer.cpp:453-480)."""
        N = self.nx * self.ny
        delta = np.zeros(N, dtype=np.complex128)
        delta[self.ny * (self.nx - 1) // 2 + (self.ny - 1) // 2] = 1.0
        s = np.concatenate([px * delta, py * delta])
        return _solve(self.sol[layerType].W, s, self.lstsq)  # BDCSVD solve

    def scatterPlaneWave(self, cInc, ref, trn, k0):
        """scatterPlaneWave (rcwa/RCWASolver.cpp:1792-1908).  Returns (REF, TRN)
        or (None, None) where the reference returns early with empty vectors."""
        N = self.nx * self.ny
        cref = self.Rud @ cInc
        ctrn = self.Tdd @ cInc
        rxy = self.sol[ref].W @ cref
        txy = self.sol[trn].W @ ctrn
        rx, ry, tx, ty = rxy[:N], rxy[N:], txy[:N], txy[N:]
        Lr, Lt = self.layers[ref], self.layers[trn]
        eps_ref = layer_eps_at(Lr.cx, Lr.cy, Lr.eps, 0.0, 0.0)
        eps_trn = layer_eps_at(Lt.cx, Lt.cy, Lt.eps, 0.0, 0.0)
        # Layer::mu(x, y), the same cell lookup (rcwa/Layer.cpp:431-450); k^2 = k0^2 eps mu (:1826-1830)
        mu_ref = 1.0 + 0j if Lr.mu is None else layer_eps_at(Lr.cx, Lr.cy, Lr.mu, 0.0, 0.0)
        mu_trn = 1.0 + 0j if Lt.mu is None else layer_eps_at(Lt.cx, Lt.cy, Lt.mu, 0.0, 0.0)
        a = self.alpha.astype(np.complex128)
        b = self.beta.astype(np.complex128)
        kref2 = k0 * k0 * eps_ref * mu_ref
        ktrn2 = k0 * k0 * eps_trn * mu_trn
        Kzref = -np.sqrt(kref2 - a * a - b * b)  # :1835
        Kztrn = np.sqrt(ktrn2 - a * a - b * b)   # :1836
        if np.any(Kzref == 0) or np.any(Kztrn == 0):
            return None, None  # :1843-1847
        rz = (a * rx + b * ry) / Kzref
        tz = (a * tx + b * ty) / Kztrn
        r = np.abs(rx) ** 2 + np.abs(ry) ** 2 + np.abs(rz) ** 2
        t = np.abs(tx) ** 2 + np.abs(ty) ** 2 + np.abs(tz) ** 2
        inc = self.ny * (self.nx - 1) // 2 + (self.ny - 1) // 2
        Kzinc = abs(Kzref[inc].real)
        if Kzinc < 1e-12 * k0:
            return None, None  # :1898-1901
        # the transmitted flux carries mu_ref / mu_trn (S_z ~ kz / mu, :1902-1907)
        return np.abs(Kzref.real) * r / Kzinc, abs(mu_ref / mu_trn) * np.abs(Kztrn.real) * t / Kzinc


# --------------------------------------------------------------------------
# The .ofd bridge (sol/rcwa_bridge.cpp)
# --------------------------------------------------------------------------
@dataclass
class RcwaLayerSpec:
    """rcwalayer_t (include/orcwa_rcwa.h:26-35)."""
    eps1: float
    eps2: float
    fill: float
    thickness: float
    eps1i: float = 0.0
    eps2i: float = 0.0
    fill_y: float = 1.0


@dataclass
class RcwaPole:
    """rcwapole_t (include/orcwa_rcwa.h:44-51); layer is 0-based."""
    layer: int
    side: int
    einf: float
    ae: float
    be: float
    ce: float


@dataclass
class OfdSetup:
    """The globals rcwa_run reads (include/orcwa_rcwa.h:53-70, rcwa_bridge.cpp:35-40)."""
    nHx: int
    period_x: float
    layers: List[RcwaLayerSpec]
    freqs: Sequence[float]
    nHy: int = 0
    period_y: Optional[float] = None
    theta: float = 0.0
    phi: float = 0.0
    poles: List[RcwaPole] = field(default_factory=list)

    def py(self):
        return self.period_x if self.period_y is None else self.period_y


def common_edges(period, fills):
    """commonEdges (sol/rcwa_bridge.cpp:52-67)."""
    e = [0.0] + [f * period for f in fills if f < 1.0] + [period]
    e.sort()
    u = []
    for v in e:
        if not u or (v - u[-1]) > 1e-12 * period:
            u.append(v)
    return np.array(u, dtype=np.float64)


def make_layer_eps(l: RcwaLayerSpec, e1, e2, xe, ye):
    """makeLayer (sol/rcwa_bridge.cpp:72-89): eps1 inside [0,fill*px]x[0,fill_y*py]."""
    px, py = xe[-1], ye[-1]
    eps = np.empty((ye.size - 1, xe.size - 1), dtype=np.complex128)
    for j in range(ye.size - 1):
        yc = 0.5 * (ye[j] + ye[j + 1])
        for i in range(xe.size - 1):
            xc = 0.5 * (xe[i] + xe[i + 1])
            eps[j, i] = e1 if (xc < l.fill * px) and (yc < l.fill_y * py) else e2
    return eps


def layer_eps(setup: OfdSetup, n: int, side: int, omega: float) -> complex:
    """layerEps, Lorentz poles (sol/rcwa_bridge.cpp:91-123)."""
    l = setup.layers[n]
    disp = [p for p in setup.poles if p.layer == n and p.side == side]
    if not any(p.ae != 0.0 for p in disp):
        return complex(l.eps1, l.eps1i) if side == 1 else complex(l.eps2, l.eps2i)
    einf = 0.0
    for p in disp:
        einf = p.einf
    e = complex(einf, 0.0)
    for p in disp:
        if p.ae == 0.0:
            continue
        e += complex(p.ae * p.ae, 0.0) / complex(p.ce * p.ce - omega * omega, -p.be * omega)
    return e


def polarisation_vectors(theta_deg, phi_deg):
    """TE/TM transverse unit vectors (sol/rcwa_bridge.cpp:179-196)."""
    th = theta_deg * PI / 180.0
    ph = phi_deg * PI / 180.0
    if abs(math.sin(th)) < 1e-9:
        return (0.0, 1.0), (1.0, 0.0)  # TE, TM
    return (-math.sin(ph), math.cos(ph)), (math.cos(th) * math.cos(ph), math.cos(th) * math.sin(ph))


def rcwa_run(setup: OfdSetup, lstsq=False, keep=False):
    """rcwa_run (sol/rcwa_bridge.cpp:145-366) without file output.

    Returns a list of dicts per frequency: freq, lam, R[2], T[2] (TE, TM),
    REF/TRN per order (unmasked, [2][N]) and the masked per-order arrays
    ordR/ordT ([2][N]) that the bridge writes.
    """
    L = len(setup.layers)
    if L < 2 or setup.period_x <= 0 or len(setup.freqs) < 1:
        raise ValueError("invalid rcwa setup")
    te, tm = polarisation_vectors(setup.theta, setup.phi)
    th = setup.theta * PI / 180.0
    ph = setup.phi * PI / 180.0
    xe = common_edges(setup.period_x, [l.fill for l in setup.layers])
    ye = common_edges(setup.py(), [l.fill_y for l in setup.layers])
    stack = list(range(L))
    thick = [0.0 if n in (0, L - 1) else setup.layers[n].thickness for n in range(L)]
    nOrdX, nOrdY = 2 * setup.nHx + 1, 2 * setup.nHy + 1
    out = []
    for freq in setup.freqs:
        if freq <= 0:
            raise ValueError("invalid frequency1 data")
        lam = C0 / freq
        k0 = 2.0 * PI / lam
        omega = 2.0 * PI * freq
        eps_inc = layer_eps(setup, 0, 1, omega)
        n_inc = max(np.sqrt(complex(eps_inc)).real, 1e-6)
        solver = RCWASolver(setup.nHx, setup.nHy, lstsq=lstsq)
        solver.keep = keep
        for n in range(L):
            eps = make_layer_eps(setup.layers[n], layer_eps(setup, n, 1, omega),
                                 layer_eps(setup, n, 2, omega), xe, ye)
            solver.addLayer(OracleLayer(xe, ye, eps))
        kx0 = k0 * n_inc * math.sin(th) * math.cos(ph)
        ky0 = k0 * n_inc * math.sin(th) * math.sin(ph)
        solver.setBlochWavevector(kx0, ky0)
        solver.solve(lam, stack, thick)
        # propagating-order masks (rcwa_bridge.cpp:289-300)
        kr2 = k0 * k0 * eps_inc.real
        kt2 = k0 * k0 * layer_eps(setup, L - 1, 1, omega).real
        k = np.arange(nOrdX * nOrdY)
        m = k // nOrdY - setup.nHx
        nn = k % nOrdY - setup.nHy
        kx = kx0 + 2.0 * PI * m / setup.period_x
        ky = ky0 + 2.0 * PI * nn / setup.py()
        kt = kx * kx + ky * ky
        propR, propT = kt < kr2, kt < kt2
        R, T, REF, TRN, ordR, ordT = [], [], [], [], [], []
        for (px, py) in (te, tm):
            c = solver.generateHorizontalPlaneWave(px, py, 0)
            rf, tr = solver.scatterPlaneWave(c, 0, L - 1, k0)
            if rf is None:
                raise FloatingPointError("scatterPlaneWave returned early (grazing / kz == 0)")
            R.append(rf.sum())
            T.append(tr.sum())
            REF.append(rf)
            TRN.append(tr)
            ordR.append(np.where(propR, rf, 0.0))
            ordT.append(np.where(propT, tr, 0.0))
        rec = dict(freq=freq, lam=lam, R=np.array(R), T=np.array(T), REF=np.array(REF),
                   TRN=np.array(TRN), ordR=np.array(ordR), ordT=np.array(ordT),
                   kx0=kx0, ky0=ky0)
        if keep:
            rec["solver"] = solver
        out.append(rec)
    return out
