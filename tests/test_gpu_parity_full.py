"""Parity at the workload sizes, not only on small cases.

A row of every product form here depends only on that row of A and on all of B (its scale, its
digits or residues, and the column scales of B), so the oracle computes chosen rows of the full
product exactly as the GPU computes them.  The rows are taken from different raster groups of
each kernel's work order (groups of 16 tile rows of 256 for the CRT form, 8 of 128 for the slice
form and the native FP64 kernel), including the first and last rows of groups, so the work-item
mapping of full-size launches is checked element for element:

  * N = 16384, A and B u 2^e with e uniform in [-20, 20] (the headline workload): the CRT form
    with 15 moduli and the slice form with 8 slices bit-identical to the oracle's restatements;
    the native FP64 kernel inside the summation-order bound of the reference's FMA chain;
  * 1D emulation of 4 ranks at N = 8192 (row panels of 2048 x 8192, one launch per rank), native
    FP64 within the same bound;
  * the 3 x 5 SUMMA grid M = 12288, N = 20480, K = 16384 with 512-wide panels: the CRT and slice
    plans bit-identical to the oracle, the FP64 plan within the bound of the oracle's SUMMA;
  * always-on small cases whose tile rows cross one raster group and end in a partial one.

Reference arithmetic: 1D-row-block/mulmat_kernel.cu:39-80 (the FMA chain the oracle restates
and tests/golden pins bit for bit), 2D-block-matrix/mmb.cu:239-361 (the panel loop).
"""
import numpy as np
import pytest

from conftest import gamma, rng_matrix
from gpu_util import bits, dev, host

pytestmark = pytest.mark.gpu

CRT_GROUP_ROWS = 16 * 256
SLICE_GROUP_ROWS = 8 * 128


def _rows(m, group_rows, extra, seed):
    """Rows at the edges of raster groups and tiles, plus a few random ones."""
    picks = {0, m - 1}
    for g in range(group_rows, m, group_rows):
        picks |= {g - 1, g}
    picks |= {min(m - 1, 255), min(m - 1, 256), min(m - 1, 1023), min(m - 1, 1024)}
    rng = np.random.default_rng(seed)
    picks |= set(int(r) for r in rng.integers(0, m, extra))
    return np.array(sorted(picks))


def _device_inputs(mgx, m, n, k, kind, seeds):
    import torch
    A = torch.empty((m, k), dtype=torch.float64, device="cuda")
    B = torch.empty((k, n), dtype=torch.float64, device="cuda")
    mgx.fill_matrix(A, kind, e_range=20 if kind == 2 else 0, seed=seeds[0])
    mgx.fill_matrix(B, kind, e_range=20 if kind == 2 else 0, seed=seeds[1])
    return A, B


def _fp64_bound(A_rows, B):
    return 2 * gamma(A_rows.shape[1]) * (np.abs(A_rows) @ np.abs(B))


@pytest.fixture(scope="module")
def headline(mgx):
    """N = 16384 wide-exponent inputs, generated on the GPU, with host copies of the sampled
    rows of A and of all of B."""
    import torch
    N = 16384
    A, B = _device_inputs(mgx, N, N, N, 2, (1000, 1001))
    rows = _rows(N, CRT_GROUP_ROWS, 4, 16384)
    idx = torch.from_numpy(rows).cuda()
    out = {"N": N, "A": A, "B": B, "rows": rows, "A_rows": host(A.index_select(0, idx)), "B_h": host(B)}
    yield out
    out.clear()
    torch.cuda.empty_cache()


def test_crt_full_size_rows_bit_exact(mgx, oracle, headline):
    import torch
    N, A, B, rows = headline["N"], headline["A"], headline["B"], headline["rows"]
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(A, B, C, moduli=15)
    got = host(C.index_select(0, torch.from_numpy(rows).cuda()))
    del C
    ref = oracle.crt_gemm(headline["A_rows"], headline["B_h"], 15)
    assert np.array_equal(bits(got), bits(ref)), f"rows differ: {rows[np.any(bits(got) != bits(ref), axis=1)]}"
    assert mgx.device_status() == 0


def test_slices_full_size_rows_bit_exact(mgx, oracle, headline):
    import torch
    N, A, B = headline["N"], headline["A"], headline["B"]
    rows = headline["rows"]
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(A, B, C, splits=8)
    got = host(C.index_select(0, torch.from_numpy(rows).cuda()))
    del C
    ref = oracle.ozaki_gemm(headline["A_rows"], headline["B_h"], 8)
    assert np.array_equal(bits(got), bits(ref)), f"rows differ: {rows[np.any(bits(got) != bits(ref), axis=1)]}"
    assert mgx.device_status() == 0


def test_fp64_full_size_rows_within_bound(mgx, oracle, headline):
    import torch
    N, A, B, rows = headline["N"], headline["A"], headline["B"], headline["rows"]
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mgx.ab_multiply(A, B, C)
    got = host(C.index_select(0, torch.from_numpy(rows).cuda()))
    del C
    Ar, Bh = headline["A_rows"], headline["B_h"]
    assert np.all(np.abs(got - oracle.ab_multiply(Ar, Bh)) <= _fp64_bound(Ar, Bh))


def test_fp64_four_rank_panels_rows_within_bound(mgx, oracle):
    """1D emulation of 4 ranks at N = 8192: each rank's 2048 x 8192 row panel times B as its own
    launch (the reference's per-rank ABMultiply, 1D-row-block/mmb.cu:627-925)."""
    import torch
    N, P = 8192, 4
    A, B = _device_inputs(mgx, N, N, N, 1, (77, 78))
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mi = N // P
    for r in range(P):
        mgx.ab_multiply(A[r * mi:(r + 1) * mi], B, C[r * mi:(r + 1) * mi])
    rows = np.array(sorted({r * mi + o for r in range(P) for o in (0, 1023, 1024, mi - 1)}))
    idx = torch.from_numpy(rows).cuda()
    got, Ar, Bh = host(C.index_select(0, idx)), host(A.index_select(0, idx)), host(B)
    assert np.all(np.abs(got - oracle.ab_multiply(Ar, Bh)) <= _fp64_bound(Ar, Bh))


def test_summa_grid_full_size_rows(mgx, oracle):
    """The 3 x 5 grid M = 12288, N = 20480, K = 16384, 512-wide panels: the CRT and slice plans
    (one product of all of C) bit-identical to the oracle, the FP64 plan (every block and panel in
    one persistent kernel) within the bound of the oracle's panel loop."""
    import torch
    M, N, K, pr, pc, bk = 12288, 20480, 16384, 3, 5, 512
    A, B = _device_inputs(mgx, M, N, K, 1, (41, 42))
    C = torch.empty((M, N), dtype=torch.float64, device="cuda")
    rows = _rows(M, CRT_GROUP_ROWS, 3, 12288)
    idx = torch.from_numpy(rows).cuda()
    Ar, Bh = host(A.index_select(0, idx)), host(B)
    for form, s, ref in ((mgx.FORM_CRT, 15, lambda: oracle.crt_gemm(Ar, Bh, 15)),
                         (mgx.FORM_OZAKI, 8, lambda: oracle.ozaki_gemm(Ar, Bh, 8))):
        plan = mgx.SummaPlan(M, N, K, pr, pc, bk, form=form, splits=s)
        plan.run(A, B, C)
        got = host(C.index_select(0, idx))
        plan.close()
        assert np.array_equal(bits(got), bits(ref())), f"form {form}"
    plan = mgx.SummaPlan(M, N, K, pr, pc, bk, form=mgx.FORM_FP64)
    plan.run(A, B, C)
    got = host(C.index_select(0, idx))
    plan.close()
    ref = oracle.summa2d(Ar, Bh, bk)
    # both sum the K products of an element in some order whose depth is at most K plus the
    # panel additions: each lies within gamma_(K + panels) |A||B| of the exact value
    panels = (K + bk - 1) // bk
    bound = 2 * gamma(K + panels) * (np.abs(Ar) @ np.abs(Bh))
    assert np.all(np.abs(got - ref) <= bound)
    assert mgx.device_status() == 0


@pytest.mark.parametrize("m,n,k", [(4400, 300, 200), (4097, 257, 96)])
def test_crt_partial_raster_group_bit_exact(mgx, oracle, m, n, k):
    """More than 16 tile rows of 256: the work order crosses a raster group and ends in a
    partial one."""
    import torch
    rng = np.random.default_rng(m + n + k)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=15)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, 15)))


@pytest.mark.parametrize("m,n,k", [(1100, 300, 200), (2200, 130, 64)])
def test_slices_and_fp64_partial_raster_group(mgx, oracle, m, n, k):
    """More than 8 tile rows of 128 (the slice form's and the FP64 kernel's raster group)."""
    import torch
    rng = np.random.default_rng(m * 3 + n + k)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dA, dB, dC, splits=8)
    assert np.array_equal(bits(host(dC)), bits(oracle.ozaki_gemm(A, B, 8)))
    mgx.ab_multiply(dA, dB, dC)
    assert np.all(np.abs(host(dC) - oracle.ab_multiply(A, B)) <= _fp64_bound(A, B))
