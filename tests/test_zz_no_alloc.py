"""The allocation-free Ozaki entry point, called through the C ABI.

Callers that cannot allocate device memory when they call (inside a stream capture that must
not gain allocation nodes, under an allocator that owns all device memory, after a
no-allocation start-up) use mgx_gemm_ozaki_noalloc, whose workspace is a fixed device array.
Its results must equal the allocating entry point's (bit for bit, as every Ozaki result here is
compared) on consecutive calls, since the calls share that array.  This file runs last.
"""
import ctypes

import numpy as np
import pytest

from conftest import rng_matrix

pytestmark = pytest.mark.gpu


def _vp(t):
    return ctypes.c_void_p(t.data_ptr())


def test_noalloc_matches_allocating_entry_point_on_consecutive_calls(mgx):
    import torch
    L = mgx.lib()
    rng = np.random.default_rng(2024)
    results = []
    for (m, n, k, s) in [(300, 257, 1000, 8), (512, 384, 700, 9)]:   # two calls in a row, different shapes
        A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
        dA = torch.from_numpy(A).cuda()
        dB = torch.from_numpy(B).cuda()
        c_free = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
        rc = L.mgx_gemm_ozaki_noalloc(_vp(dA), _vp(dB), _vp(c_free), m, n, k, k, n, n, 0, s, None)
        assert rc == 0, L.mgx_last_error_message()
        ws = torch.empty(L.mgx_ozaki_workspace_size(m, n, k, s), dtype=torch.uint8, device="cuda")
        c_ref = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
        rc = L.mgx_gemm_ozaki(_vp(dA), _vp(dB), _vp(c_ref), m, n, k, k, n, n, 0, s, _vp(ws), ws.numel(), None)
        assert rc == 0, L.mgx_last_error_message()
        torch.cuda.synchronize()
        assert torch.equal(c_free.view(torch.int64), c_ref.view(torch.int64))
        results.append(c_free.cpu().numpy())
    assert results[0].shape != results[1].shape
    code = ctypes.c_int()
    assert L.mgx_device_status(ctypes.byref(code)) == 0 and code.value == 0


def test_noalloc_call_leaves_device_memory_unchanged(mgx):
    """After the first call on the device (which may load the library's kernels), a call takes
    no device memory: the device's free bytes are the same before and after it."""
    import torch
    L = mgx.lib()
    rng = np.random.default_rng(7)
    m, n, k, s = 256, 320, 512, 8
    dA = torch.from_numpy(rng_matrix(rng, (m, k), "wide")).cuda()
    dB = torch.from_numpy(rng_matrix(rng, (k, n), "wide")).cuda()
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    first = torch.empty_like(dC)
    assert L.mgx_gemm_ozaki_noalloc(_vp(dA), _vp(dB), _vp(first), m, n, k, k, n, n, 0, s, None) == 0
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    rc = L.mgx_gemm_ozaki_noalloc(_vp(dA), _vp(dB), _vp(dC), m, n, k, k, n, n, 0, s, None)
    torch.cuda.synchronize()
    free_after = torch.cuda.mem_get_info()[0]
    assert rc == 0, L.mgx_last_error_message()
    assert free_after == free_before
    assert torch.equal(dC.view(torch.int64), first.view(torch.int64))


def test_noalloc_rejects_products_beyond_its_array(mgx):
    L = mgx.lib()
    m = n = k = 4096
    assert L.mgx_ozaki_workspace_size(m, n, k, 8) > (32 << 20)
    rc = L.mgx_gemm_ozaki_noalloc(None, None, None, m, n, k, k, n, n, 0, 8, None)
    assert rc == -5
    assert b"workspace" in L.mgx_last_error_message()
