"""rcwa_rcwa_integrate (RCWAIntegrator::compute, core/RCWAIntegrator.cpp:21-86)
against the oracle's restatement: the four S-blocks as field-space operators
(free of the eigenvectors' order and phase, which the GPU eigensolver need
not share with LAPACK) within 1e-9, for even and odd slab counts (the
pairwise cascade carries a slab over), one slab and none; the reference
test's uniform-region phase (tests/test_core_integrators.cpp:83-99) and
second-order convergence (:119-139) on the device's own output."""
import numpy as np
import pytest

import oracle.smatrix_oracle as so
import openrcwa_b200 as o
from tests import integrator_cases as ic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


@pytest.mark.parametrize("nslab", [0, 1, 8, 13])
def test_matches_oracle_in_field_space(eng, nslab):
    P, Q = ic.samples(nslab, moving=True)
    got = eng.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
    want = so.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
    # the modes themselves: eigenpairs of P Q at both ends
    for W, V, g, k in ((got["W0"], got["V0"], got["gam0"], 0), (got["W1"], got["V1"], got["gam1"], -1)):
        PQ = P[k] @ Q[k]
        assert np.abs(PQ @ W - W * (g * g)[None, :]).max() < 1e-9 * np.abs(PQ).max()
        assert np.abs(Q[k] @ W - V * g[None, :]).max() < 1e-9 * np.abs(Q[k]).max()
    fg, fw = so.field_space(got), so.field_space(want)
    for key in fg:
        assert np.abs(fg[key] - fw[key]).max() < 1e-9 * max(1.0, np.abs(fw[key]).max()), key


@pytest.mark.parametrize("nslab", [1, 8])
def test_uniform_region_is_a_phase(eng, nslab):
    P, Q = ic.samples(nslab, moving=False)
    out = eng.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
    L = (ic.Z1 - ic.Z0) * ic.LAM / (2 * np.pi)
    want = np.diag(np.exp(1j * out["gam0"] * L))
    assert np.abs(out["Tuu"] - want).max() < 1e-8 and np.abs(out["Tdd"] - want).max() < 1e-8
    assert np.abs(out["Rud"]).max() < 1e-8 and np.abs(out["Rdu"]).max() < 1e-8


def test_moving_edge_converges_at_second_order(eng):
    # the modes at z0 and z1 are the same samples for every slab count, so
    # the modal Tuu of different counts compare directly
    P, Q = ic.samples(512, moving=True)
    Tref = eng.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)["Tuu"]
    scale = np.abs(Tref).max()
    errs = []
    for N in (16, 32, 64, 128):
        P, Q = ic.samples(N, moving=True)
        errs.append(np.abs(eng.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)["Tuu"] - Tref).max() / scale)
    assert all(a / b > 3.0 for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-4


@pytest.mark.parametrize("nslab", [1, 7, 16])
def test_differential_matches_oracle_in_field_space(eng, nslab):
    P, Q = ic.half_step_samples(nslab, moving=True)
    got = eng.differential_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
    want = so.differential_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1)
    fg, fw = so.field_space(got), so.field_space(want)
    for key in fg:
        assert np.abs(fg[key] - fw[key]).max() < 1e-9 * max(1.0, np.abs(fw[key]).max()), key


def test_differential_agrees_with_rcwa_on_the_device(eng):
    # in field space: the two integrators' end modes need not be ordered alike
    P, Q = ic.samples(512, moving=True)
    Tr = so.field_space(eng.rcwa_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))["Tuu"]
    P, Q = ic.half_step_samples(512, moving=True)
    Td = so.field_space(eng.differential_integrate(P, Q, ic.LAM, ic.Z0, ic.Z1))["Tuu"]
    assert np.abs(Td - Tr).max() / np.abs(Tr).max() < 1e-5


@pytest.mark.parametrize("pe", [1e-2, 1e-3])
def test_redheffer_matches_oracle(eng, pe):
    sampler = lambda z: ic.sample(z, True)
    n = 2 * ic.NX * ic.NY
    got = eng.redheffer_integrate(sampler, n, ic.LAM, ic.Z0, ic.Z1, pe)
    want = so.redheffer_integrate(sampler, ic.LAM, ic.Z0, ic.Z1, pe)
    # the same subdivision, and the same S-matrix in field space
    assert got["N"] == want["N"] and got["n_eig"] == want["nEigVal"]
    fg, fw = so.field_space(got), so.field_space(want)
    for key in fg:
        assert np.abs(fg[key] - fw[key]).max() < 1e-9 * max(1.0, np.abs(fw[key]).max()), key


def test_redheffer_uniform_and_sampler_failure(eng):
    n = 2 * ic.NX * ic.NY
    out = eng.redheffer_integrate(lambda z: ic.sample(z, False), n, ic.LAM, ic.Z0, ic.Z1, 1e-3)
    L = (ic.Z1 - ic.Z0) * ic.LAM / (2 * np.pi)
    assert out["N"] == 1
    assert np.abs(out["Tuu"] - np.diag(np.exp(1j * out["gam0"] * L))).max() < 1e-8

    def bad(z):
        raise KeyError("no sample at %g" % z)

    with pytest.raises(KeyError):
        eng.redheffer_integrate(bad, n, ic.LAM, ic.Z0, ic.Z1, 1e-3)
