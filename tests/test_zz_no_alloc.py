"""The allocation-free eigensolver entry point (rcwa_zgeev_batched_noalloc).

It exists for callers that cannot call cudaMalloc themselves (code running
inside another framework's memory pool, real-time loops, fixed device
footprints): they hand in their own device buffers and the solver's scratch
comes from a static device array.  This test acts as such a caller: the device
buffers come from torch, the entry point is called through the C ABI twice in a
row on different inputs, and each result must match the allocating entry
point (rcwa_zgeev_batched) within the eigen tolerance the other GPU tests use.
Kept in its own file so that pytest collects it last.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _run_noalloc(lib, torch, A):
    b, n, _ = A.shape
    dA = torch.from_numpy(np.ascontiguousarray(A).view(np.float64)).cuda()
    dw = torch.zeros((b, n, 2), dtype=torch.float64, device="cuda")
    dV = torch.zeros((b, n, n, 2), dtype=torch.float64, device="cuda")
    dinfo = torch.full((b,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    rc = lib.rcwa_zgeev_batched_noalloc(n, b, ctypes.c_void_p(dA.data_ptr()), ctypes.c_void_p(dw.data_ptr()),
                                        ctypes.c_void_p(dV.data_ptr()), ctypes.c_void_p(dinfo.data_ptr()), None)
    torch.cuda.synchronize()
    assert rc == 0
    w = dw.cpu().numpy().view(np.complex128).reshape(b, n)
    V = dV.cpu().numpy().view(np.complex128).reshape(b, n, n)
    return w, V, dinfo.cpu().numpy()


def test_noalloc_matches_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    import openrcwa_b200 as o
    eng = o.Engine(0)
    lib = o.load()
    rng = np.random.default_rng(5)
    cases = [(22, 16), (64, 64)]
    # one untimed call per size first: it is where lazy module loading reserves
    # the static scratch, and it leaves torch's caching pool holding blocks of
    # every size the checked calls use, so that the free device memory can
    # only move afterwards if the entry point itself allocates
    inputs = [rng.normal(size=(b, n, n)) + 1j * rng.normal(size=(b, n, n)) for (n, b) in cases]
    refs = [eng.zgeev(A.copy()) for A in inputs]
    for A in inputs:
        _run_noalloc(lib, torch, A)
    free0 = torch.cuda.mem_get_info()[0]
    for A, (w_ref, V_ref, info_ref) in zip(inputs, refs):
        b, n, _ = A.shape
        w, V, info = _run_noalloc(lib, torch, A)
        assert np.all(info == 0) and np.all(info_ref == 0)
        assert np.max(np.abs(w - w_ref)) < 1e-12 * np.max(np.abs(w_ref))
        assert np.max(np.abs(V - V_ref)) < 1e-12
        for k in range(b):
            res = np.abs(A[k] @ V[k] - V[k] * w[k][None, :]).max() / np.abs(A[k]).max()
            assert res < 1e-12 * n
    # the two calls after the warm-up left the device's free memory unchanged
    # (torch's own buffers of the calls come from its caching pool, whose
    # blocks were reserved by the warm-up calls of the same sizes)
    assert torch.cuda.mem_get_info()[0] == free0
    eng.close()


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import openrcwa_b200 as o
    lib = o.load()
    dummy = ctypes.c_void_p(16)
    assert lib.rcwa_zgeev_batched_noalloc(65, 1, dummy, dummy, dummy, dummy, None) == o.abi.RCWA_ERR_UNSUPPORTED
    assert lib.rcwa_zgeev_batched_noalloc(8, 65, dummy, dummy, dummy, dummy, None) == o.abi.RCWA_ERR_UNSUPPORTED
