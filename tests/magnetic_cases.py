"""Magnetic-material inputs shared by the oracle tests and the engine tests.

The .orcwa texts follow the reference's own magnetic known-answer cases
(tests/test_rcwa_input.cpp:1990-2175 of the reference): a half-space of
(eps, mu) below air, a magnetic slab between air half-spaces, and the
analytic Fresnel reflectance of a magnetic interface (:1998-2009).
"""
import math

import numpy as np


def interface(eps, mu, theta, pol, extra=""):
    """Air above a half-space of (eps, mu), one material line (:2011-2035)."""
    return (f"OpenRCWA 4 2\ntitle = magnetic interface\n"
            f"xmesh = -2.5e-07 10 2.5e-07\nymesh = -2.5e-07 10 2.5e-07\n"
            f"zmesh = -5e-07 10 0.0 10 1e-06\n"
            f"material = 1 {eps!r} 0 {mu!r} 0\n{extra}"
            f"geometry = 2 1 -2.5e-07 2.5e-07 -2.5e-07 2.5e-07 -5e-07 0\n"
            f"planewave = {theta!r} 0 {pol}\npbc = 1 1 0\nrcwaorder = 4 0\nwavelength = 0.6\nend\n")


def slab(material_lines):
    """A 0.3 um slab of material 2 between air half-spaces (:2132-2146)."""
    return ("OpenRCWA 4 2\ntitle = magnetic loss slab\n"
            "xmesh = -2.5e-07 10 2.5e-07\nymesh = -2.5e-07 10 2.5e-07\n"
            "zmesh = -1e-06 10 0.0 10 3e-07 10 7e-07\n" + material_lines +
            "geometry = 2 1 -2.5e-07 2.5e-07 -2.5e-07 2.5e-07 0 3e-07\n"
            "planewave = 0 0 1\npbc = 1 1 0\nrcwaorder = 4 0\nwavelength = 0.6\nend\n")


def fresnel_r(theta_deg, e2, m2, pol):
    """|r|^2 of air -> (e2, m2); pol 2 = TE, otherwise TM (:1998-2009)."""
    t = math.radians(theta_deg)
    n2 = math.sqrt(e2 * m2)
    k1z, s = math.cos(t), math.sin(t)
    k2z = math.sqrt(n2 * n2 - s * s)
    r = (m2 * k1z - k2z) / (m2 * k1z + k2z) if pol == 2 else (e2 * k1z - k2z) / (e2 * k1z + k2z)
    return r * r


# a patterned magnetic metasurface: pillars with eps, mu and magnetic loss on a
# magnetic substrate, oblique incidence with circular polarisation
PILLARS = """OpenRCWA 4 2
title = magnetic pillars
xmesh = -2.0e-07 20 2.0e-07
ymesh = -2.0e-07 20 2.0e-07
zmesh = -5e-07 10 -1.5e-07 10 0.0 10 4e-07
material = 1 2.25 0 1.5 0
material = 1 5.0 0 2.0 4.0e8
geometry = 2 1 -2.0e-07 2.0e-07 -2.0e-07 2.0e-07 -5e-07 -1.5e-07
geometry = 3 11 -1.2e-07 1.2e-07 -1.0e-07 1.0e-07 -1.5e-07 0
planewave = 20 30 4
rcwaorder = 2 2
frequency1 = 4.0e14 5.0e14 1
end
"""


def grating_layers(eps_pat, mu_pat, eps_sub, mu_sub):
    """A 1D two-cell grating (period 0.5, cell edge at 0.2) on a uniform
    substrate, air above: (cx, cy, [eps per layer], [mu per layer])."""
    cx, cy = np.array([0.0, 0.2, 0.5]), np.array([0.0, 0.5])
    eps = [np.array([[1.0, 1.0]], dtype=complex), np.array([eps_pat], dtype=complex),
           np.array([[eps_sub, eps_sub]], dtype=complex)]
    mu = [np.array([[1.0, 1.0]], dtype=complex), np.array([mu_pat], dtype=complex),
          np.array([[mu_sub, mu_sub]], dtype=complex)]
    return cx, cy, eps, mu
