"""Seeded synthetic workloads with the shapes of the engine's benchmark configurations.

Each builder returns (stacks, points, pxy) for Engine.solve_batch / Engine.plan:
points rows are (stack index, wavelength, kx0, ky0) and pxy holds the TE and TM
transverse polarisation vectors of each point (as sol/rcwa_bridge.cpp:187-196
defines them).  Lengths are in metres.
"""
from __future__ import annotations

import math

import numpy as np

from .abi import Stack, TableStack

PI = 3.1415926535897932


def pol_vectors(theta_deg, phi_deg):
    th, ph = math.radians(theta_deg), math.radians(phi_deg)
    if abs(math.sin(th)) < 1e-9:
        return (0.0, 1.0), (1.0, 0.0)
    return (-math.sin(ph), math.cos(ph)), (math.cos(th) * math.cos(ph), math.cos(th) * math.sin(ph))


def _edges(period, fills):
    e = sorted([0.0] + [f * period for f in fills if f < 1.0] + [period])
    u = []
    for v in e:
        if not u or v - u[-1] > 1e-12 * period:
            u.append(v)
    return np.array(u)


def rect_stack(nHx, nHy, px, py, layers, eps_sup=1.0, eps_sub=2.25):
    """layers: list of (eps1, eps2, fill_x, fill_y, thickness); one eps1
    rectangle [0, fx*px] x [0, fy*py] per layer on the merged edge grid."""
    xe = _edges(px, [l[2] for l in layers])
    ye = _edges(py, [l[3] for l in layers])
    xc = 0.5 * (xe[1:] + xe[:-1])
    yc = 0.5 * (ye[1:] + ye[:-1])
    eps = [np.full((ye.size - 1, xe.size - 1), eps_sup, dtype=complex)]
    for (e1, e2, fx, fy, _) in layers:
        inside = (yc[:, None] < fy * py) & (xc[None, :] < fx * px)
        eps.append(np.where(inside, e1, e2).astype(complex))
    eps.append(np.full((ye.size - 1, xe.size - 1), eps_sub, dtype=complex))
    thick = [0.0] + [l[4] for l in layers] + [0.0]
    return Stack(nHx, nHy, xe, ye, np.array(eps), thick)


def grating_1d(n_freq=16, nH=5):
    """The 1D lamellar grating: period 300 nm, eps 4/1 fill 0.5, 200 nm, on
    glass, normal incidence, n_freq frequencies 4.3e14-7.5e14 Hz."""
    st = rect_stack(nH, 0, 3e-7, 3e-7, [(4.0, 1.0, 0.5, 1.0, 2e-7)])
    freqs = np.linspace(4.3e14, 7.5e14, n_freq)
    lam = 2.99792458e8 / freqs
    pts = np.array([(0, l, 0.0, 0.0) for l in lam])
    te, tm = pol_vectors(0.0, 0.0)
    pxy = np.array([[te, tm]] * len(lam), dtype=complex)
    return [st], pts, pxy


def pillars_2d(seed=0, nH=10, n_lambda=256, n_angle=8, n_layers=5):
    """2D rectangular-pillar grating: Nx=Ny=nH, period 400 x 400 nm, n_layers
    patterned layers with fills ~U(0.2, 0.8), thickness ~U(50, 300) nm,
    eps1 = U(2, 12) + i U(0, 0.5), eps2 = 1, superstrate 1, substrate 2.25;
    n_lambda wavelengths 400-800 nm x n_angle (theta ~ U(0, 60), phi ~ U(0, 90))
    conical incidences.  Points are ordered angle-major within each wavelength."""
    rng = np.random.default_rng(seed)
    layers = []
    for _ in range(n_layers):
        fx, fy = rng.uniform(0.2, 0.8, 2)
        d = rng.uniform(50e-9, 300e-9)
        e1 = complex(rng.uniform(2, 12), rng.uniform(0, 0.5))
        layers.append((e1, 1.0, fx, fy, d))
    st = rect_stack(nH, nH, 4e-7, 4e-7, layers)
    th = rng.uniform(0, 60, n_angle)
    ph = rng.uniform(0, 90, n_angle)
    lam = np.linspace(400e-9, 800e-9, n_lambda)
    pts, pxy = [], []
    for l in lam:
        k0 = 2 * PI / l
        for a in range(n_angle):
            t, p = math.radians(th[a]), math.radians(ph[a])
            pts.append((0, l, k0 * math.sin(t) * math.cos(p), k0 * math.sin(t) * math.sin(p)))
            pxy.append(pol_vectors(th[a], ph[a]))
    return [st], np.array(pts), np.array(pxy, dtype=complex)


def lorentz_eps(einf, ae, be, ce, omega):
    """Single-pole Lorentz permittivity einf + ae^2 / (ce^2 - w^2 - i be w)
    (the pole model of sol/rcwa_bridge.cpp:116-121, angular frequencies)."""
    return einf + ae * ae / (ce * ce - omega * omega - 1j * be * omega)


def uneven_batch(seed=0, n_instances=4096, nh_range=(3, 15), max_layers=10, period=4e-7):
    """Independent 2D-grating instances of uneven size: nH = Nx = Ny ~ U{3..15}
    (49-961 orders), 1..max_layers patterned layers, each one rectangle with
    fills ~U(0.1, 0.9) and thickness ~U(20, 500) nm, eps1 from a one-pole
    Lorentz model (einf ~U(1, 4), ae ~U(1e15, 5e15), be ~U(1e13, 1e14),
    ce ~U(2e15, 6e15) rad/s) or a lossy metal -U(5, 30) + iU(0.5, 3), eps2 = 1;
    one point per instance at lambda ~U(400, 1000) nm, theta ~U(0, 70) deg,
    phi = 0.  Returns (stacks, points, pxy) with TE and TM per point."""
    rng = np.random.default_rng(seed)
    stacks, pts, pxy = [], [], []
    for i in range(n_instances):
        nh = int(rng.integers(nh_range[0], nh_range[1] + 1))
        nl = int(rng.integers(1, max_layers + 1))
        lam = rng.uniform(400e-9, 1000e-9)
        omega = 2 * PI * 2.99792458e8 / lam
        layers = []
        for _ in range(nl):
            fx, fy = rng.uniform(0.1, 0.9, 2)
            d = rng.uniform(20e-9, 500e-9)
            if rng.random() < 0.5:
                e1 = lorentz_eps(rng.uniform(1, 4), rng.uniform(1e15, 5e15), rng.uniform(1e13, 1e14),
                                 rng.uniform(2e15, 6e15), omega)
            else:
                e1 = complex(-rng.uniform(5, 30), rng.uniform(0.5, 3))
            layers.append((e1, 1.0, fx, fy, d))
        stacks.append(rect_stack(nh, nh, period, period, layers))
        th = rng.uniform(0, 70)
        k0 = 2 * PI / lam
        pts.append((i, lam, k0 * math.sin(math.radians(th)), 0.0))
        pxy.append(pol_vectors(th, 0.0))
    return stacks, np.array(pts), np.array(pxy, dtype=complex)


def disk_laurent_table(Lx, Ly, radius, center, eps1, eps2, nH):
    """Laurent coefficients of a circular pillar (eps1 in a disk of the given
    radius and center, eps2 elsewhere) for 2nH+1 orders per axis:
    F[m + 2nH, n + 2nH] = (1/(Lx Ly)) integral eps exp(-i (gx x + gy y)) =
    eps2 delta_mn + (eps1 - eps2) pi R^2 (2 J1(g R)/(g R)) exp(-i g.c)/(Lx Ly),
    g = 2 pi (m/Lx, n/Ly) (the Fourier transform of a disk, an Airy pattern)."""
    from scipy.special import j1
    m = np.arange(-2 * nH, 2 * nH + 1)[:, None]
    n = np.arange(-2 * nH, 2 * nH + 1)[None, :]
    gx, gy = 2 * PI * m / Lx, 2 * PI * n / Ly
    gr = np.hypot(gx, gy) * radius
    safe = np.where(gr > 0, gr, 1.0)
    airy = np.where(gr > 0, 2.0 * j1(safe) / safe, 1.0)
    F = (eps1 - eps2) * PI * radius * radius * airy * np.exp(-1j * (gx * center[0] + gy * center[1])) / (Lx * Ly)
    F[2 * nH, 2 * nH] += eps2
    return F.astype(np.complex128)


def circular_pillars(seed=0, nH=25, n_lambda=32, n_layers=20, period=4e-7, lossless=False):
    """Large-order single structure: n_layers circular-pillar layers (one disk
    per layer centred in the cell, radius/period ~U(0.2, 0.45), thickness
    ~U(20, 100) nm, eps1 alternating 4.0 and 2.1+0.01i (2.1 when lossless),
    eps2 = 1) between a superstrate of eps 1 and a substrate of 2.25, period x
    period cells (400 nm), 2nH+1 orders per axis; n_lambda wavelengths
    500-900 nm at normal incidence, TE and TM.  The layers' Laurent tables are
    the closed-form disk transform.  Returns ([TableStack], points, pxy)."""
    rng = np.random.default_rng(seed)
    f2d, thick = [], [0.0]
    for k in range(n_layers):
        r = rng.uniform(0.2, 0.45) * period
        d = rng.uniform(20e-9, 100e-9)
        e1 = 4.0 if k % 2 == 0 else complex(2.1, 0.0 if lossless else 0.01)
        f2d.append(disk_laurent_table(period, period, r, (0.5 * period, 0.5 * period), e1, 1.0, nH))
        thick.append(d)
    thick.append(0.0)
    st = TableStack(nH, nH, period, period, np.array([1.0, 2.25], dtype=complex), np.array(f2d), thick)
    lam = np.linspace(500e-9, 900e-9, n_lambda)
    te, tm = pol_vectors(0.0, 0.0)
    pts = np.array([(0, l, 0.0, 0.0) for l in lam])
    pxy = np.array([[te, tm]] * len(lam), dtype=complex)
    return [st], pts, pxy


def batch_slice(points, pxy, start, count):
    idx = (np.arange(count) + start) % len(points)
    return points[idx], pxy[idx]


def shard_start(rank: int, world: int, batch: int, step: int) -> int:
    """First sweep index of the batch a rank solves at a step: ranks take
    disjoint consecutive batches (weak scaling, no data exchange)."""
    return (step * world + rank) * batch
