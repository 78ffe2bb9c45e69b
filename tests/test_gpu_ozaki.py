"""Ozaki INT8 tensor-core form on the GPU: bit-identical to the oracle's restatement (the digit
slices and int32 sums are integer work; the FP64 recombination follows the same operations in the
same order), and accurate against the double-double product."""
import numpy as np
import pytest

from conftest import rng_matrix
from gpu_util import bits, dev, host, vp

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k,s", [(128, 128, 32, 3), (128, 128, 256, 8), (1, 1, 1, 4), (77, 200, 333, 5),
                                     (300, 129, 1000, 7), (256, 256, 512, 9), (130, 260, 96, 2), (64, 64, 64, 12)])
def test_ozaki_bit_exact_vs_oracle(mgx, oracle, m, n, k, s):
    import torch
    rng = np.random.default_rng(m * 31 + n * 7 + k + s)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dev(A), dev(B), dC, splits=s)
    C = host(dC)
    assert np.array_equal(bits(C), bits(oracle.ozaki_gemm(A, B, s)))
    assert mgx.device_status() == 0


def test_ozaki_beta_one_and_uniform(mgx, oracle):
    rng = np.random.default_rng(3)
    A, B, C0 = rng_matrix(rng, (200, 300)), rng_matrix(rng, (300, 170)), rng_matrix(rng, (200, 170))
    dC = dev(C0)
    mgx.gemm_ozaki(dev(A), dev(B), dC, splits=8, beta_one=True)
    assert np.array_equal(bits(host(dC)), bits(oracle.ozaki_gemm(A, B, 8, C=C0.copy(), beta_one=True)))


def test_ozaki_split_multiply_phases(mgx, oracle):
    import torch
    rng = np.random.default_rng(4)
    A, B = rng_matrix(rng, (256, 512), "wide"), rng_matrix(rng, (512, 384), "wide")
    ws = torch.empty(mgx.ozaki_workspace_size(256, 384, 512, 8), dtype=torch.uint8, device="cuda")
    mgx.ozaki_split(dev(A), dev(B), 8, ws)
    dC = torch.empty((256, 384), dtype=torch.float64, device="cuda")
    mgx.ozaki_multiply(dC, 512, 8, ws)
    first = host(dC).copy()
    mgx.ozaki_multiply(dC, 512, 8, ws)      # slices reused
    assert np.array_equal(bits(first), bits(host(dC)))
    assert np.array_equal(bits(first), bits(oracle.ozaki_gemm(A, B, 8)))


@pytest.mark.parametrize("s,target", [(8, 1e-15), (9, 1e-16)])
def test_ozaki_accuracy_wide_exponents(mgx, oracle, s, target):
    import torch
    rng = np.random.default_rng(5)
    A, B = rng_matrix(rng, (512, 2048), "wide"), rng_matrix(rng, (2048, 512), "wide")
    dA, dB = dev(A), dev(B)
    dC = torch.empty((512, 512), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dA, dB, dC, splits=s)
    e = mgx.error_vs_dd(dA, dB, dC)
    assert e["normwise"] <= target


def test_ozaki_integer_known_answer(mgx):
    import torch
    N = 1024
    A = torch.ones((N, N), dtype=torch.float64, device="cuda")
    B = torch.full((N, N), 2.0, dtype=torch.float64, device="cuda")
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(A, B, C, splits=3)
    assert torch.all(C == 2.0 * N)


def test_ozaki_nonfinite_marks_rows_and_columns(mgx):
    import torch
    rng = np.random.default_rng(6)
    A, B = rng_matrix(rng, (140, 64)), rng_matrix(rng, (64, 150))
    A[5, 7] = np.inf
    B[3, 9] = np.nan
    dC = torch.empty((140, 150), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dev(A), dev(B), dC, splits=4)
    C = host(dC)
    assert mgx.device_status() == 4          # non-finite input recorded on the device
    assert np.all(np.isnan(C[5])) and np.all(np.isnan(C[:, 9]))
    mask = np.ones_like(C, dtype=bool)
    mask[5] = False
    mask[:, 9] = False
    assert np.all(np.isfinite(C[mask]))


def test_ozaki_k_beyond_int32_headroom(mgx, oracle):
    """K larger than one int32 accumulation allows is split into ordered chunks."""
    import torch
    s = 12
    kmax = mgx.ozaki_kmax(s)
    k = kmax + 200
    rng = np.random.default_rng(7)
    A, B = rng_matrix(rng, (8, k)), rng_matrix(rng, (k, 8))
    dC = torch.empty((8, 8), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dev(A), dev(B), dC, splits=s)
    assert np.array_equal(bits(host(dC)), bits(oracle.ozaki_gemm(A, B, s)))


@pytest.mark.parametrize("form,panels,m,n,k", [(1, 1, 333, 270, 515), (1, 3, 333, 270, 515), (0, 4, 333, 270, 515),
                                               (1, 4, 700, 201, 300), (0, 4, 700, 201, 300), (1, 10, 129, 1000, 64),
                                               (0, 2, 1, 1, 1)])
def test_host_buffer_entry_point_matches_device_path(mgx, oracle, form, panels, m, n, k):
    """mgx_gemm_host (PCIe copies overlapped with the product in a 2D block schedule: row panels
    of A x column panels of B, uneven panels, odd n) gives the same bits as the device-buffer
    entry points, and writes every element of C."""
    import torch
    rng = np.random.default_rng(11 + m + n)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    hA = torch.from_numpy(A).pin_memory()
    hB = torch.from_numpy(B).pin_memory()
    hC = torch.full((m, n), np.nan, dtype=torch.float64).pin_memory()
    mgx.gemm_host(hA, hB, hC, form=form, splits=8, panels=panels)
    torch.cuda.synchronize()
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    if form == 1:
        mgx.gemm_ozaki(dev(A), dev(B), dC, splits=8)
    else:
        mgx.gemm_fp64(dev(A), dev(B), dC)
    assert np.array_equal(bits(hC.numpy()), bits(host(dC)))
    # the pool's cached scratch can be handed back, and the path allocates again afterwards
    mgx.scratch_trim()
    hC2 = torch.full((m, n), np.nan, dtype=torch.float64).pin_memory()
    mgx.gemm_host(hA, hB, hC2, form=form, splits=8, panels=panels)
    torch.cuda.synchronize()
    assert np.array_equal(bits(hC2.numpy()), bits(hC.numpy()))


@pytest.mark.parametrize("m,n,k,s,ks", [(200, 150, 2000, 8, 4), (129, 257, 300, 7, 2), (7, 9, 13, 8, 8),
                                         (333, 127, 1000, 8, 16), (256, 256, 4096, 9, 64), (64, 66, 64, 3, 3)])
def test_splitk_bit_identical_to_oracle(mgx, oracle, m, n, k, s, ks):
    """Ozaki split-K: per-slice recombination, slices added in order -- integer work and the same
    FP64 operations as the oracle's restatement, so bit-identical; normwise error as unsplit."""
    import torch
    rng = np.random.default_rng(m + n + k + s + ks)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dA, dB, dC, splits=s, ksplit=ks)
    ref = oracle.ozaki_gemm_splitk(A, B, s, ks)
    assert np.array_equal(bits(host(dC)), bits(ref))
    # deterministic, and beta_one adds into C
    C0 = rng_matrix(rng, (m, n))
    dC2 = dev(C0)
    mgx.gemm_ozaki(dA, dB, dC2, splits=s, ksplit=ks, beta_one=True)
    assert np.array_equal(bits(host(dC2)), bits(oracle.ozaki_gemm_splitk(A, B, s, ks, C=C0.copy(), beta_one=True)))
    assert mgx.device_status() == 0


def test_splitk_limits(mgx, oracle):
    import torch
    rng = np.random.default_rng(3)
    m, n, k = 100, 90, 700
    A, B = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n))
    dA, dB = dev(A), dev(B)
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    # one slice is the plain Ozaki product
    mgx.gemm_ozaki(dA, dB, dC, splits=8, ksplit=1)
    assert np.array_equal(bits(host(dC)), bits(oracle.ozaki_gemm(A, B, 8)))
    need = mgx.ozaki_splitk_workspace_size(m, n, k, 8, 4)
    assert need >= mgx.ozaki_workspace_size(m, n, k, 8) + 4 * m * n * 8
    small = torch.empty(need - 512, dtype=torch.uint8, device="cuda")
    L = mgx.lib()
    rc = L.mgx_gemm_ozaki_splitk(vp(dA), vp(dB), vp(dC), m, n, k, k, n, n, 0, 8, 4, vp(small), small.numel(), None)
    assert rc == -5  # MGX_E_WORKSPACE
    kk = mgx.ozaki_kmax(12) + 32
    assert mgx.ozaki_splitk_workspace_size(8, 8, kk, 12, 4) == 0
    big = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    Ak = torch.zeros((8, kk), dtype=torch.float64, device="cuda")
    Bk = torch.zeros((kk, 8), dtype=torch.float64, device="cuda")
    Ck = torch.empty((8, 8), dtype=torch.float64, device="cuda")
    rc = L.mgx_gemm_ozaki_splitk(vp(Ak), vp(Bk), vp(Ck), 8, 8, kk, kk, 8, 8, 0, 12, 4, vp(big), big.numel(), None)
    assert rc == -6  # MGX_E_UNSUPPORTED: k above one int32 accumulation
