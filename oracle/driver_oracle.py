"""CPU restatement of the reference's orcwa_rcwa path (TEST INFRASTRUCTURE
ONLY): the .orcwa parser (rcwa/RCWAInput.cpp), the geometry-to-layers driver
(rcwa/RCWADriver.cpp) and the solve loop, on top of the RCWASolver oracle in
rcwa_oracle.py.  It serves as the reference answer for the drop-in test of the
unmodified driver compiled against the engine's C++ adapters.

Covered: xmesh/ymesh/zmesh (end points), material, material_eps,
material_index, material_mu, material_dispersion, geometry (box, sphere,
cylinders along z/x/y), planewave (pol 1-5), rcwaorder, frequency1/2 and
wavelength, background; lengths in micrometres as the parser stores them.
Magnetic materials (relative permeability and magnetic conductivity) follow
muAt / hasMagneticMaterial (rcwa/RCWADriver.cpp:126-157) into the oracle's
magnetic branch of the wave equation.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List

import numpy as np

from .rcwa_oracle import OracleLayer, RCWASolver

C0 = 2.99792458e8
C0_UM = 2.99792458e14   # rcwa/RCWADriver.cpp:15
EPS0 = 8.854187817e-12  # :16
MU0 = 1.25663706212e-6  # :17
M_TO_UM = 1e6
N_CURVED = 8            # N_CURVED_CELLS / N_CURVED_SLICES (RCWADriver.cpp:21, RCWAInput.cpp:435)
BOX, SPHERE, CYL_Z, CYL_X, CYL_Y = 1, 2, 11, 12, 13


@dataclass
class Box:
    material: int
    shape: int
    x0: float
    x1: float
    y0: float
    y1: float
    z0: float
    z1: float

    def contains_xyz(self, xc, yc, zc):
        """RCWABox::containsXYZ (rcwa/RCWAInput.cpp:46-90)."""
        if zc < self.z0 or zc > self.z1:
            return False
        cx, cy, cz = 0.5 * (self.x0 + self.x1), 0.5 * (self.y0 + self.y1), 0.5 * (self.z0 + self.z1)
        rx, ry, rz = 0.5 * (self.x1 - self.x0), 0.5 * (self.y1 - self.y0), 0.5 * (self.z1 - self.z0)
        if self.shape == BOX:
            return self.x0 <= xc <= self.x1 and self.y0 <= yc <= self.y1
        if self.shape == SPHERE:
            if rx <= 0 or ry <= 0 or rz <= 0:
                return False
            return ((xc - cx) / rx) ** 2 + ((yc - cy) / ry) ** 2 + ((zc - cz) / rz) ** 2 <= 1.0
        if self.shape == CYL_Z:
            if rx <= 0 or ry <= 0:
                return False
            return ((xc - cx) / rx) ** 2 + ((yc - cy) / ry) ** 2 <= 1.0
        if self.shape == CYL_X:
            if ry <= 0 or rz <= 0 or xc < self.x0 or xc > self.x1:
                return False
            return ((yc - cy) / ry) ** 2 + ((zc - cz) / rz) ** 2 <= 1.0
        if self.shape == CYL_Y:
            if rx <= 0 or rz <= 0 or yc < self.y0 or yc > self.y1:
                return False
            return ((xc - cx) / rx) ** 2 + ((zc - cz) / rz) ** 2 <= 1.0
        return False


@dataclass
class Problem:
    xmin: float = 0.0
    xmax: float = 0.0
    ymin: float = 0.0
    ymax: float = 0.0
    zmin: float = 0.0
    zmax: float = 0.0
    nHx: int = 10
    nHy: int = 0
    eps: List[complex] = field(default_factory=lambda: [1.0 + 0j, 1.0 + 1e8j])  # 0 air, 1 PEC (:141-145)
    mu: List[complex] = field(default_factory=lambda: [1.0 + 0j, 1.0 + 0j])
    sigma: List[float] = field(default_factory=lambda: [0.0, 0.0])
    msigma: List[float] = field(default_factory=lambda: [0.0, 0.0])
    disp: List[tuple] = field(default_factory=lambda: [(0.0, []), (0.0, [])])
    boxes: List[Box] = field(default_factory=list)
    theta: float = 0.0
    phi: float = 0.0
    pol: int = 1
    psi: float = 0.0
    background: complex = 1.0 + 0j
    lambdas: List[float] = field(default_factory=list)


def parse(text: str) -> Problem:
    """parseRCWAInput (rcwa/RCWAInput.cpp:134-428) for the keys above."""
    p = Problem()
    have = {"1": False, "2": False}
    lines = [ln for ln in text.splitlines() if ln.strip()]
    for k, line in enumerate(lines):
        tok = line.replace(",", " ").split()
        if k == 0:
            if tok[0] not in ("OpenRCWA", "OpenTHFD"):
                raise ValueError("not an OpenRCWA file")
            continue
        if tok[0] == "end":
            break
        if len(tok) < 3 or tok[1] != "=" or tok[0].startswith("#"):
            continue
        key, v = tok[0], tok[2:]
        f = [float(x) for x in v] if key not in ("title",) else []
        if key == "xmesh":
            p.xmin, p.xmax = f[0] * M_TO_UM, f[-1] * M_TO_UM
        elif key == "ymesh":
            p.ymin, p.ymax = f[0] * M_TO_UM, f[-1] * M_TO_UM
        elif key == "zmesh":
            p.zmin, p.zmax = f[0] * M_TO_UM, f[-1] * M_TO_UM
        elif key == "material" and len(f) >= 2:
            p.eps.append(complex(f[1], 0.0))
            p.sigma.append(f[2] if len(f) >= 3 else 0.0)
            p.mu.append(complex(f[3] if len(f) >= 4 else 1.0, 0.0))
            p.msigma.append(f[4] if len(f) >= 5 else 0.0)
            p.disp.append((0.0, []))
        elif key in ("material_eps", "material_index") and len(f) >= 2:
            m = int(f[0])
            a, b = f[1], (f[2] if len(f) >= 3 else 0.0)
            p.eps[m] = complex(a, b) ** 2 if key == "material_index" else complex(a, b)
        elif key == "material_mu" and len(f) >= 2:
            # rcwa/RCWAInput.cpp:254-268
            m = int(f[0])
            if 0 <= m < len(p.mu):
                p.mu[m] = complex(f[1], f[2] if len(f) >= 3 else 0.0)
        elif key == "material_dispersion" and len(f) >= 5:
            m = int(f[0])
            einf, poles = p.disp[m]
            if f[2] != 0.0:
                poles = poles + [(f[2], f[3], f[4])]
            p.disp[m] = (f[1], poles)
        elif key == "geometry" and len(f) >= 8:
            if int(f[1]) in (BOX, SPHERE, CYL_Z, CYL_X, CYL_Y):
                p.boxes.append(Box(int(f[0]), int(f[1]), *[x * M_TO_UM for x in f[2:8]]))
        elif key == "planewave" and len(f) >= 3:
            p.theta, p.phi, p.pol = f[0], f[1], int(f[2])
            if len(f) >= 4:
                p.psi = f[3]
            if p.pol < 1 or p.pol > 5:
                p.pol = 1
        elif key == "rcwaorder":
            p.nHx = int(f[0])
            if len(f) >= 2:
                p.nHy = int(f[1])
        elif key in ("frequency1", "frequency2", "frequency") and len(f) >= 3:
            which = "2" if key == "frequency2" else "1"
            if not have[which]:
                f0, f1, nd = f[0], f[1], max(int(f[2]), 0)
                for i in range(nd + 1):
                    fr = f0 if nd == 0 else f0 + (f1 - f0) * i / nd
                    if fr > 0:
                        p.lambdas.append(C0 / fr * M_TO_UM)
                have[which] = True
        elif key in ("wavelength", "lambda"):
            if len(f) >= 3:
                l0, l1, nd = f[0], f[1], max(int(f[2]), 0)
                p.lambdas += [l0 if nd == 0 else l0 + (l1 - l0) * i / nd for i in range(nd + 1)]
            elif f:
                p.lambdas.append(f[0])
        elif key == "background":
            p.background = complex(f[0], f[1] if len(f) >= 2 else 0.0)
    p.lambdas = sorted(set(lam for lam in p.lambdas if lam > 0))
    return p


def z_edges(p: Problem):
    """deriveZEdges (rcwa/RCWAInput.cpp:430-453)."""
    e = {p.zmin, p.zmax}
    for b in p.boxes:
        if p.zmin <= b.z0 <= p.zmax:
            e.add(b.z0)
        if p.zmin <= b.z1 <= p.zmax:
            e.add(b.z1)
        if b.shape in (SPHERE, CYL_X, CYL_Y):
            for i in range(1, N_CURVED):
                z = b.z0 + (b.z1 - b.z0) * i / N_CURVED
                if p.zmin <= z <= p.zmax:
                    e.add(z)
    return sorted(e)


def grid(p: Problem, axis: str):
    """buildCommonXGrid / buildCommonYGrid (rcwa/RCWADriver.cpp:50-82): box
    edges plus N_CURVED subdivisions of curved shapes' extents."""
    lo, hi = (p.xmin, p.xmax) if axis == "x" else (p.ymin, p.ymax)
    s = {lo, hi}
    for b in p.boxes:
        a0, a1 = (b.x0, b.x1) if axis == "x" else (b.y0, b.y1)
        a0, a1 = max(a0, lo), min(a1, hi)
        if lo < a0 < hi:
            s.add(a0)
        if lo < a1 < hi:
            s.add(a1)
        curved = b.shape in ((SPHERE, CYL_Z, CYL_Y) if axis == "x" else (SPHERE, CYL_Z, CYL_X))
        if curved and a0 < a1:
            for i in range(1, N_CURVED):
                v = a0 + (a1 - a0) * i / N_CURVED
                if lo < v < hi:
                    s.add(v)
    return np.array(sorted(s))


def eps_at(p: Problem, x, y, z, lam):
    """epsAt (rcwa/RCWADriver.cpp:88-125): the last containing box wins; a
    Lorentz model replaces the static value; conductivity adds i sigma/(w eps0)."""
    e = p.background
    for b in p.boxes:
        if not b.contains_xyz(x, y, z):
            continue
        m = b.material
        if m < 0 or m >= len(p.eps):
            continue
        e = p.eps[m]
        w = 2 * math.pi * C0_UM / lam
        einf, poles = p.disp[m]
        if poles:
            e = complex(einf, 0.0)
            for ae, be, ce in poles:
                e += (ae * ae) / complex(ce * ce - w * w, -be * w)
        if p.sigma[m] != 0.0:
            e += complex(0.0, p.sigma[m] / (w * EPS0))
    return complex(e)


def mu_at(p: Problem, x, y, z, lam):
    """muAt (rcwa/RCWADriver.cpp:126-147): the last containing box wins; a
    magnetic conductivity adds i msigma/(w mu0)."""
    m = 1.0 + 0j
    for b in p.boxes:
        if not b.contains_xyz(x, y, z):
            continue
        mi = b.material
        if mi < 0 or mi >= len(p.mu):
            continue
        m = p.mu[mi]
        if mi < len(p.msigma) and p.msigma[mi] != 0.0:
            w = 2 * math.pi * C0_UM / lam
            m += complex(0.0, p.msigma[mi] / (w * MU0))
    return complex(m)


def has_magnetic(p: Problem) -> bool:
    """hasMagneticMaterial (rcwa/RCWADriver.cpp:150-157)."""
    return any(abs(m - 1.0) > 1e-12 for m in p.mu) or any(s != 0.0 for s in p.msigma)


def device_image(sol, slice_, coord, stack, thickness, n1=2000):
    """saveDeviceImage (rcwa/RCWASolver.cpp:1322-1487) without translations:
    the real part of the interior layers' permittivity on the slice, a depth
    z belonging to the layer with z0 <= z < z1."""
    L0 = sol.layers[0]
    Lx, Ly = L0.cx[-1] - L0.cx[0], L0.cy[-1] - L0.cy[0]
    if slice_ == 1:
        s1, L1, s2, L2 = L0.cx[0], Lx, 0.0, float(sum(thickness[1:len(stack) - 1]))
    elif slice_ == 2:
        s1, L1, s2, L2 = L0.cy[0], Ly, 0.0, float(sum(thickness[1:len(stack) - 1]))
    else:
        s1, L1, s2, L2 = L0.cx[0], Lx, L0.cy[0], Ly
    n2 = max(int(n1 * L2 / L1), 1)

    def layer_at(z):
        z0 = 0.0
        for j in range(1, len(stack) - 1):
            z1 = z0 + thickness[j]
            if z0 <= z < z1:
                return j
            z0 = z1
        raise ValueError("depth outside the interior layers")

    def cells(edges, v):
        # the first cell whose upper edge is >= v (Layer::eps, rcwa/Layer.cpp:383-429)
        return np.searchsorted(np.asarray(edges)[1:], v, side="left")

    out = np.zeros((n2, n1))
    c1 = s1 + (L1 / n1) * (np.arange(n1) + 0.5)
    for i in range(n2):
        c2 = s2 + (L2 / n2) * (i + 0.5)
        lay = sol.layers[stack[layer_at(coord if slice_ == 0 else c2)]]
        x, y = (c1, np.full(n1, coord)) if slice_ == 1 else \
            ((np.full(n1, coord), c1) if slice_ == 2 else (c1, np.full(n1, c2)))
        per = lay.cx[-1] - lay.cx[0]
        x = np.where(x < lay.cx[0], x + per, np.where(x > lay.cx[-1], x - per, x))
        out[i] = np.asarray(lay.eps)[cells(lay.cy, y), cells(lay.cx, x)].real
    return out


def run(text: str, field=None, device=None):
    """runRCWA (rcwa/RCWADriver.cpp:196-378): per wavelength (micrometres) R,
    T, A and the per-order REF/TRN vectors.  field = (component, slice,
    coord, opt) adds, for the first wavelength, the values saveFieldImage
    writes (:336-356; opt 0 modulus, 1 real, 2 imaginary part) as "field"."""
    p = parse(text)
    magnetic = has_magnetic(p)
    ze = z_edges(p)
    xg, yg = grid(p, "x"), grid(p, "y")
    centers = [0.5 * (ze[i] + ze[i - 1]) for i in range(len(ze) - 1, 0, -1)]
    thick = [ze[i] - ze[i - 1] for i in range(len(ze) - 1, 0, -1)]
    th, ph = math.radians(p.theta), math.radians(p.phi)
    if abs(math.sin(th)) < 1e-9:
        tm, te = (1.0, 0.0), (0.0, 1.0)
    else:
        tm = (math.cos(th) * math.cos(ph), math.cos(th) * math.sin(ph))
        te = (-math.sin(ph), math.cos(ph))
    r2 = 1.0 / math.sqrt(2.0)
    a_tm, a_te = {2: (0.0, 1.0), 3: (math.cos(math.radians(p.psi)), math.sin(math.radians(p.psi))),
                  4: (r2, 1j * r2), 5: (r2, -1j * r2)}.get(p.pol, (1.0, 0.0))
    px = a_tm * tm[0] + a_te * te[0]
    py = a_tm * tm[1] + a_te * te[1]
    xc = 0.5 * (xg[1:] + xg[:-1])
    yc = 0.5 * (yg[1:] + yg[:-1])
    out = []
    for lam in p.lambdas:
        sol = RCWASolver(p.nHx, p.nHy)
        for zc in centers:
            eps = np.array([[eps_at(p, x, y, zc, lam) for x in xc] for y in yc])
            mu = np.array([[mu_at(p, x, y, zc, lam) for x in xc] for y in yc]) if magnetic else None
            sol.addLayer(OracleLayer(xg, yg, eps, mu=mu))
        k0 = 2 * math.pi / lam
        e_inc = eps_at(p, 0.5 * (p.xmin + p.xmax), 0.5 * (p.ymin + p.ymax), centers[0], lam)
        mu_inc = mu_at(p, 0.5 * (p.xmin + p.xmax), 0.5 * (p.ymin + p.ymax), centers[0], lam) if magnetic else 1.0
        n_inc = max(np.sqrt(complex(e_inc) * complex(mu_inc)).real, 1e-6)  # :305-312
        sol.setBlochWavevector(k0 * n_inc * math.sin(th) * math.cos(ph), k0 * n_inc * math.sin(th) * math.sin(ph))
        stack = list(range(len(centers)))
        sol.solve(lam, stack, thick)
        c = sol.generateHorizontalPlaneWave(px, py, 0)
        ref, trn = sol.scatterPlaneWave(c, 0, len(centers) - 1, k0)
        fval = dval = None
        if device is not None and not out:
            dval = device_image(sol, device[0], device[1], stack, thick)
        if field is not None and not out:
            comp, sl, coord, opt = field
            inp = [(i, v) for i, v in enumerate(c) if abs(v) > 1e-14]
            f = sol.fieldSlice(sl, coord, comp, inp, stack, thick)
            fval = np.abs(f) if opt == 0 else (f.real if opt == 1 else f.imag)
        out.append({"lambda": lam, "R": ref.sum(), "T": trn.sum(), "A": 1 - ref.sum() - trn.sum(), "REF": ref,
                    "TRN": trn, "field": fval, "device": dval})
    return out
