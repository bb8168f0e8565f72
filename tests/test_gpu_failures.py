"""Failure paths of the engine, each injected on the host so that no GPU
faults or hangs: a NaN permittivity, a NaN matrix handed to the eigensolver,
exactly singular systems in the S-matrix kernels, and a QR sweep cap of one
sweep.  Every case must come back as its RCWA_* status code, and the engine
must stay usable afterwards.

The reference reports such cases on std::cerr or not at all (LAPACK's zgeev
info, rcwa/MKLEigenSolver.hpp:131-160; Eigen's PartialPivLU returns inf/NaN,
rcwa/RCWASolver.cpp:451-453); here they are per-point status codes.
"""
import math

import numpy as np
import pytest

import openrcwa_b200 as o
from openrcwa_b200 import abi, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def eng():
    e = o.Engine(0)
    yield e
    e.close()


def _small_2d():
    st = workloads.rect_stack(3, 3, 4e-7, 4e-7, [(complex(6.0, 0.2), 1.0, 0.4, 0.6, 1.5e-7),
                                                 (complex(3.0, 0.0), 1.0, 0.7, 0.3, 0.8e-7)])
    lam = 6e-7
    k0 = 2 * math.pi / lam
    pts = np.array([(0, lam, 0.2 * k0, 0.1 * k0), (0, 5e-7, 0.0, 0.0)])
    pxy = np.array([[(0.0, 1.0), (1.0, 0.0)]] * 2, dtype=complex)
    return st, pts, pxy


def test_nan_permittivity_is_rejected_before_any_launch(eng):
    st, pts, pxy = _small_2d()
    st.eps[1, 0, 0] = complex(float("nan"), 0.0)
    with pytest.raises(o.RcwaError) as ex:
        eng.solve_batch([st], pts, pxy)
    assert ex.value.code == abi.RCWA_ERR_NONFINITE
    assert "non-finite" in eng.last_error()


def test_nan_matrix_reports_nonfinite_from_the_eigensolver(eng):
    rng = np.random.default_rng(3)
    for n in (30, 100):   # single-shift and multishift Schur kernels
        A = rng.normal(size=(3, n, n)) + 1j * rng.normal(size=(3, n, n))
        A[1, n // 2, n // 3] = complex(float("nan"), 1.0)
        w, VR, info = eng.zgeev(A)
        assert info[1] == abi.RCWA_ERR_NONFINITE, info
        assert info[0] == 0 and info[2] == 0
        res = np.abs(A[0] @ VR[0] - VR[0] * w[0][None, :]).max() / np.abs(A[0]).max()
        assert res < 1e-12 * n


def test_singular_star_product_and_slab(eng):
    n, b = 6, 3
    rng = np.random.default_rng(4)
    eye = np.broadcast_to(np.eye(n, dtype=complex), (b, n, n)).copy()
    # item 1: rdu Rud = I, so I - rdu Rud is exactly zero
    Rud = 0.1 * (rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n)))
    Rud[1] = np.eye(n)
    S = {"Rud": Rud, "Rdu": np.zeros((b, n, n), complex), "Tdd": eye, "Tuu": eye}
    rdu = 0.1 * (rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n)))
    rdu[1] = np.eye(n)
    s = {"rud": rdu, "rdu": rdu, "tdd": eye, "tuu": eye}
    _, st = eng.star_product(S, s)
    assert list(st) == [0, abi.RCWA_ERR_SINGULAR, 0]
    # slab seen from W0 = W, V0 = -V: A = W^-1 W0 + V^-1 V0 = 0
    W = eye + 0.1 * (rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n)))
    V = eye + 0.1 * (rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n)))
    V0 = V.copy()
    V0[2] = -V[2]
    gamma = rng.uniform(0.5, 2.0, (b, n)) + 0.1j
    _, _, st = eng.slab_smatrix(W, V, gamma, W.copy(), V0, 6e-7, 1e-7)
    assert st[2] == abi.RCWA_ERR_SINGULAR and st[0] == 0 and st[1] == 0


def test_qr_sweep_cap_reports_noconv_and_resets(eng):
    rng = np.random.default_rng(6)
    st, pts, pxy = _small_2d()
    try:
        o.set_qr_sweep_limit(1)
        for n in (30, 100):
            A = rng.normal(size=(2, n, n)) + 1j * rng.normal(size=(2, n, n))
            _, _, info = eng.zgeev(A)
            assert np.all(info == abi.RCWA_ERR_NOCONV), info
        R, T, _, _, status = eng.solve_batch([st], pts, pxy, orders=False)
        assert np.all(status == abi.RCWA_ERR_NOCONV), status
    finally:
        o.set_qr_sweep_limit(0)
    with pytest.raises(o.RcwaError):
        o.set_qr_sweep_limit(-1)
    # the engine is still usable and back to the built-in budget
    R, T, _, _, status = eng.solve_batch([st], pts, pxy, orders=False)
    assert not np.any(status)
    assert np.all(np.abs(R + T - 1.0) < 0.2)
