"""MGXBench's own GPU kernel (sharedABMultiply via ABMultiply, built unmodified from its sources
into oracle/_ref) timed beside this library's FP64 and Ozaki kernels on the same inputs, at the
square sizes of the 1D configurations (N = 1024; N = 8192 as 4 row panels; N = 16384).  The
reference kernel is the checker here: it gives the 'reference GPU kernel' time and its result
bounds ours.  Run with -s to see the JSON lines."""
import json

import numpy as np
import pytest

from gpu_util import ref_kernels, vp

pytestmark = pytest.mark.gpu


def _events_ms(fn, reps):
    import torch
    fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


@pytest.mark.parametrize("n,panels,reps", [(1024, 1, 10), (8192, 4, 2), (16384, 1, 1)])
def test_reference_kernel_vs_ours(mgx, oracle, n, panels, reps):
    import torch
    R = ref_kernels(oracle)
    if R is None:
        pytest.skip("oracle/_ref/libref_mulmat.so not built")
    A = torch.empty((n, n), dtype=torch.float64, device="cuda")
    B = torch.empty((n, n), dtype=torch.float64, device="cuda")
    mgx.fill_matrix(A, 1, seed=n + 1)
    mgx.fill_matrix(B, 1, seed=n + 2)
    C_ref = torch.empty_like(A)
    C_ours = torch.empty_like(A)
    mi = n // panels

    def ref():
        for r in range(panels):
            assert R.ref_ab_multiply(vp(A[r * mi:]), vp(B), vp(C_ref[r * mi:]), mi, n, n, n, n, n) == 0

    def ours():
        for r in range(panels):
            mgx.gemm_fp64(A[r * mi:(r + 1) * mi], B, C_ours[r * mi:(r + 1) * mi])

    t_ref = _events_ms(ref, reps)
    t_ours = _events_ms(ours, max(reps, 3))
    ws = mgx.OzakiWorkspace()
    t_oz = _events_ms(lambda: mgx.gemm_ozaki(A, B, C_ours, splits=8, workspace=ws), max(reps, 3))
    ours()
    torch.cuda.synchronize()
    flop = 2.0 * n ** 3
    rows = (n // 2 - 64, 128)
    e_ref = mgx.error_vs_dd(A, B, C_ref, *rows)["normwise"]
    e_ours = mgx.error_vs_dd(A, B, C_ours, *rows)["normwise"]
    print(json.dumps({"n": n, "row_panels": panels, "reference_kernel_tflops": flop / t_ref / 1e9,
                      "fp64_tflops": flop / t_ours / 1e9, "ozaki8_effective_tflops": flop / t_oz / 1e9,
                      "speedup_fp64_vs_reference_kernel": t_ref / t_ours,
                      "reference_normwise_err": e_ref, "fp64_normwise_err": e_ours}))
    assert t_ours < t_ref
    assert e_ours <= max(4 * e_ref, 1e-15)
