"""The oracle's magnetic branch (rcwa/Layer.cpp:128-164,205-213 and the
permeability terms of rcwa/RCWASolver.cpp:1826-1907) pinned against the
reference's magnetic known answers (tests/test_rcwa_input.cpp:1990-2175): the
analytic Fresnel reflectance of a magnetic interface, the impedance-matched
interface, electromagnetic duality, the material_mu keyword and magnetic
loss.  The reference asserts 2e-3 against the analytic values; the oracle
holds them to 1e-9."""
import math

import numpy as np
import pytest

import oracle.rcwa_oracle as orc
from oracle import driver_oracle
from tests import magnetic_cases as mc


def test_impedance_matched_interface():
    r = driver_oracle.run(mc.interface(4.0, 4.0, 0.0, 1))[0]
    assert r["R"] < 1e-9 and abs(r["R"] + r["T"] - 1.0) < 1e-12


@pytest.mark.parametrize("theta", [30.0, 45.0, 60.0])
@pytest.mark.parametrize("pol", [1, 2])
def test_magnetic_fresnel(theta, pol):
    r = driver_oracle.run(mc.interface(4.0, 4.0, theta, pol))[0]
    assert abs(r["R"] - mc.fresnel_r(theta, 4.0, 4.0, pol)) < 1e-9
    assert abs(r["R"] + r["T"] - 1.0) < 1e-12


def test_asymmetric_eps_mu_and_duality():
    tm = driver_oracle.run(mc.interface(2.25, 3.0, 45.0, 1))[0]["R"]
    te = driver_oracle.run(mc.interface(2.25, 3.0, 45.0, 2))[0]["R"]
    assert abs(tm - mc.fresnel_r(45, 2.25, 3.0, 1)) < 1e-9
    assert abs(te - mc.fresnel_r(45, 2.25, 3.0, 2)) < 1e-9
    assert abs(tm - te) > 1e-2
    swap_tm = driver_oracle.run(mc.interface(3.0, 2.25, 45.0, 1))[0]["R"]
    assert abs(swap_tm - te) < 1e-9


def test_material_mu_keyword_and_magnetic_loss():
    a = driver_oracle.run(mc.interface(4.0, 1.0, 0.0, 1, extra="material_mu = 2 4.0 0.0\n"))[0]["R"]
    b = driver_oracle.run(mc.interface(4.0, 4.0, 0.0, 1))[0]["R"]
    assert abs(a - b) < 1e-12 and a < 1e-9
    lossless = driver_oracle.run(mc.slab("material = 1 4.0 0 4.0 0\n"))[0]
    lossy = driver_oracle.run(mc.slab("material = 1 4.0 0 1.0 0\nmaterial_mu = 2 4.0 0.5\n"))[0]
    assert abs(lossless["A"]) < 1e-10
    assert lossy["A"] > 0.05 and lossy["R"] + lossy["T"] < 1.0 - 1e-3
    # an omitted permeability is 1: the non-magnetic path
    c = driver_oracle.run(mc.interface(2.25, 1.0, 0.0, 1))[0]["R"]
    d = driver_oracle.run(mc.interface(2.25, 1.0, 0.0, 1).replace(" 0 1.0 0\n", " 0\n", 1))[0]["R"]
    assert abs(c - d) < 1e-12


def _grating(eps_pat, mu_pat, eps_sub, mu_sub, px, py, theta, nh=6, lam=0.7):
    cx, cy, eps, mu = mc.grating_layers(eps_pat, mu_pat, eps_sub, mu_sub)
    s = orc.RCWASolver(nh, 0)
    for e, m in zip(eps, mu):
        s.addLayer(orc.OracleLayer(cx, cy, e, mu=m))
    k0 = 2 * math.pi / lam
    s.setBlochWavevector(k0 * math.sin(math.radians(theta)), 0.0)
    s.solve(lam, [0, 1, 2], [0.0, 0.3, 0.0])
    R, T = s.scatterPlaneWave(s.generateHorizontalPlaneWave(px, py, 0), 0, 2, k0)
    return R.sum(), T.sum()


@pytest.mark.parametrize("theta", [0.0, 20.0])
def test_duality_on_a_patterned_magnetic_grating(theta):
    # exchanging eps and mu in every cell exchanges TM and TE: this holds for
    # the discretised equations too, since P's permittivity rules mirror Q's
    # permeability rules; it exercises all three permeability matrices
    e, m = [4.0 + 0.1j, 1.5], [2.0 + 0.05j, 1.0]
    c = math.cos(math.radians(theta))
    for (pe, pm), (qe, qm) in (((c, 0.0), (0.0, 1.0)), ((0.0, 1.0), (c, 0.0))):
        R1, T1 = _grating(e, m, 2.25, 1.5, pe, pm, theta)
        R2, T2 = _grating(m, e, 1.5, 2.25, qe, qm, theta)
        assert abs(R1 - R2) < 1e-12 and abs(T1 - T2) < 1e-12


def test_unit_mu_is_the_non_magnetic_path():
    cx, cy, eps, _ = mc.grating_layers([4.0, 1.5], [1.0, 1.0], 2.25, 1.0)
    a, b = orc.alpha_beta(13, 1, 0.5, 0.5, 1.0, 0.0)
    P0, Q0, *_ = orc.wave_eqn_coeff(cx, cy, eps[1], a, b, 0.7, 13, 1)
    P1, Q1, *_ = orc.wave_eqn_coeff(cx, cy, eps[1], a, b, 0.7, 13, 1, mu=np.ones((1, 2), dtype=complex))
    assert np.array_equal(P0, P1) and np.array_equal(Q0, Q1)
