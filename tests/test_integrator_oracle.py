"""The oracle's restatement of RCWAIntegrator::compute (core/RCWAIntegrator.cpp:
21-86) pinned by the properties the reference's own integrator test checks
(tests/test_core_integrators.cpp:81-146): a z-uniform region gives
Tuu = Tdd = diag(exp(i gamma L/k0)) and no reflection whatever the slab
count (:83-99), and with a moving core edge the slab cascade converges with
the slab count at second order (:119-139).  Also: the S-blocks as
field-space operators do not depend on the order, scale or phase of the
sampled modes (the form the GPU parity tests compare)."""
import numpy as np
import pytest

import oracle.smatrix_oracle as so
from tests import integrator_cases as ic


@pytest.mark.parametrize("nslab", [1, 8])
def test_uniform_region_is_a_phase(nslab):
    P, Q = ic.samples(nslab, moving=False)
    out = so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
    L = (ic.Z1 - ic.Z0) * ic.LAM / (2 * np.pi)   # L / k0
    want = np.diag(np.exp(1j * out["gam0"] * L))
    assert np.abs(out["Tuu"] - want).max() < 1e-8 and np.abs(out["Tdd"] - want).max() < 1e-8
    assert np.abs(out["Rud"]).max() < 1e-8 and np.abs(out["Rdu"]).max() < 1e-8


def test_moving_edge_converges_at_second_order():
    P, Q = ic.samples(256, moving=True)
    Tref = so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)["Tuu"]
    scale = np.abs(Tref).max()
    errs = []
    for N in (8, 16, 32, 64):
        P, Q = ic.samples(N, moving=True)
        errs.append(np.abs(so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)["Tuu"] - Tref).max() / scale)
    ratios = [a / b for a, b in zip(errs, errs[1:])]
    assert all(r > 3.0 for r in ratios), errs
    assert errs[-1] < 1e-4


def test_field_space_blocks_ignore_the_mode_gauge(monkeypatch):
    P, Q = ic.samples(6, moving=True)
    base = so.field_space(so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))
    rng = np.random.default_rng(3)
    orig = so.wave_equation_modes

    def gauged(Pm, Qm):
        W, V, k = orig(Pm, Qm)
        perm = rng.permutation(W.shape[0])
        ph = np.exp(1j * rng.uniform(0, 2 * np.pi, W.shape[0])) * rng.uniform(0.5, 2.0, W.shape[0])
        return W[:, perm] * ph, V[:, perm] * ph, k[perm]

    monkeypatch.setattr(so, "wave_equation_modes", gauged)
    other = so.field_space(so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))
    for k in base:
        assert np.abs(base[k] - other[k]).max() < 1e-12 * max(1.0, np.abs(base[k]).max()), k


def test_differential_converges_to_the_uniform_phase():
    # tests/test_core_integrators.cpp:100-116: the numerical integration
    # approaches the analytic phase as the slab count grows
    L = (ic.Z1 - ic.Z0) * ic.LAM / (2 * np.pi)
    errs = []
    for N in (64, 128, 256):
        P, Q = ic.half_step_samples(N, moving=False)
        out = so.differential_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
        errs.append(np.abs(out["Tuu"] - np.diag(np.exp(1j * out["gam0"] * L))).max())
    assert errs[0] > errs[1] > errs[2] and errs[2] < 1e-5, errs


def test_differential_agrees_with_rcwa():
    # tests/test_core_integrators.cpp:141-146 (at 256 slabs each)
    P, Q = ic.samples(256, moving=True)
    Tr = so.field_space(so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))["Tuu"]
    P, Q = ic.half_step_samples(256, moving=True)
    Td = so.field_space(so.differential_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))["Tuu"]
    assert np.abs(Td - Tr).max() / np.abs(Tr).max() < 1e-5


def test_redheffer_agrees_with_rcwa():
    # tests/test_core_integrators.cpp:141-151: pe = 1e-3 against the RCWA
    # integrator with 256 slabs (the reference takes 512), relative 1e-3
    P, Q = ic.samples(256, moving=True)
    Tr = so.field_space(so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))["Tuu"]
    out = so.redheffer_integrate(lambda z: ic.sample(z, True), ic.LAM, ic.Z0, ic.Z1, 1e-3)
    Th = so.field_space(out)["Tuu"]
    assert out["N"] > 1
    assert np.abs(Th - Tr).max() / np.abs(Tr).max() < 1e-3


def test_redheffer_uniform_region_is_one_interval():
    out = so.redheffer_integrate(lambda z: ic.sample(z, False), ic.LAM, ic.Z0, ic.Z1, 1e-3)
    L = (ic.Z1 - ic.Z0) * ic.LAM / (2 * np.pi)
    assert out["N"] == 1
    assert np.abs(out["Tuu"] - np.diag(np.exp(1j * out["gam0"] * L))).max() < 1e-8
    assert np.abs(out["Rud"]).max() < 1e-8
