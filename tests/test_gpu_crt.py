"""CRT form (Ozaki scheme II) on the GPU: bit-identical to the oracle's restatement (the scales,
residues and residue products are integer work; the CRT recombination follows the same FP64
operations in the same order), and accurate against the double-double product."""
import numpy as np
import pytest

from conftest import rng_matrix
from gpu_util import bits, dev, host

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("m,n,k,q,kind", [
    (256, 256, 256, 15, "wide"), (1, 1, 1, 8, "uniform"), (77, 200, 333, 14, "wide"),
    (300, 129, 1000, 15, "uniform"), (513, 257, 96, 16, "wide"), (256, 512, 64, 12, "wide"),
    (130, 260, 2048, 9, "wide"), (64, 600, 31, 13, "uniform"), (520, 40, 700, 10, "wide"),
    (257, 255, 4100, 11, "uniform")])
def test_crt_bit_exact_vs_oracle(mgx, oracle, m, n, k, q, kind):
    import torch
    rng = np.random.default_rng(m * 31 + n * 7 + k + q)
    A, B = rng_matrix(rng, (m, k), kind), rng_matrix(rng, (k, n), kind)
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=q)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, q)))
    assert mgx.device_status() == 0


def test_crt_zero_rows_columns_and_extreme_scales(mgx, oracle):
    """Zero rows/columns (scale 0), rows of subnormals (scale > 1023, two-step) and rows near the
    top of the range all go through the same integer scaling."""
    import torch
    rng = np.random.default_rng(11)
    A, B = rng_matrix(rng, (300, 500), "wide"), rng_matrix(rng, (500, 270), "wide")
    A[3] = 0.0
    B[:, 8] = 0.0
    A[7] *= 2.0 ** -1060
    A[9] *= 2.0 ** 900
    B[:, 11] *= 2.0 ** -700
    dC = torch.empty((300, 270), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=15)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, 15)))
    assert mgx.device_status() == 0


def test_crt_beta_one(mgx, oracle):
    rng = np.random.default_rng(3)
    A, B, C0 = rng_matrix(rng, (200, 300)), rng_matrix(rng, (300, 170)), rng_matrix(rng, (200, 170))
    dC = dev(C0)
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=14, beta_one=True)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, 14, C=C0.copy(), beta_one=True)))


def test_crt_k_beyond_one_int32_accumulation(mgx, oracle):
    """K longer than one exact int32 residue accumulation runs in chunks added in order."""
    import torch
    rng = np.random.default_rng(12)
    k = mgx.crt_kmax() + 1000
    assert k - 1000 == oracle.crt_kmax()
    A, B = rng_matrix(rng, (9, k), "wide"), rng_matrix(rng, (k, 7), "wide")
    dC = torch.empty((9, 7), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=16)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, 16)))


def test_crt_integer_known_answer(mgx):
    import torch
    N = 1024
    A = torch.ones((N, N), dtype=torch.float64, device="cuda")
    B = torch.full((N, N), 2.0, dtype=torch.float64, device="cuda")
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(A, B, C, moduli=8)
    assert torch.all(C == 2.0 * N)


@pytest.mark.parametrize("kind", ["wide", "uniform"])
def test_crt_accuracy_chosen_moduli(mgx, kind):
    """The a-priori modulus count meets 1e-15 normwise against the double-double product."""
    import torch
    rng = np.random.default_rng(5)
    k = 4096
    q = mgx.crt_choose_moduli(k, 1e-15)
    A, B = rng_matrix(rng, (512, k), kind), rng_matrix(rng, (k, 512), kind)
    dA, dB = dev(A), dev(B)
    dC = torch.empty((512, 512), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dA, dB, dC, moduli=q)
    assert mgx.error_vs_dd(dA, dB, dC)["normwise"] <= 1e-15


def test_crt_nonfinite_marks_rows_and_columns(mgx):
    import torch
    rng = np.random.default_rng(6)
    A, B = rng_matrix(rng, (140, 64)), rng_matrix(rng, (64, 150))
    A[5, 7] = np.inf
    B[3, 9] = np.nan
    dC = torch.empty((140, 150), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=15)
    C = host(dC)
    assert mgx.device_status() == 4
    assert np.all(np.isnan(C[5])) and np.all(np.isnan(C[:, 9]))
    keep = np.ones(140, bool)
    keep[5] = False
    assert np.all(np.isfinite(np.delete(C[keep], 9, axis=1)))


def test_crt_argument_errors(mgx):
    import torch
    A = torch.ones((4, 4), dtype=torch.float64, device="cuda")
    for q in (7, 17):
        with pytest.raises(mgx.MgxError):
            mgx.gemm_ozaki_crt(A, A, A.clone(), moduli=q)
    assert mgx.crt_workspace_size(4, 4, 4, 7) == 0


def test_crt_phases_reuse_residues(mgx, oracle):
    """split once, then products + combine twice: same result, equal to the oracle."""
    import torch
    rng = np.random.default_rng(21)
    m, n, k, q = 300, 520, 777, 15
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    ws = torch.empty(mgx.crt_workspace_size(m, n, k, q), dtype=torch.uint8, device="cuda")
    mgx.crt_split(dev(A), dev(B), q, ws)
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.crt_products(m, n, k, q, ws)
    mgx.crt_combine(dC, k, q, ws)
    first = host(dC).copy()
    mgx.crt_products(m, n, k, q, ws)
    mgx.crt_combine(dC, k, q, ws)
    assert np.array_equal(bits(first), bits(host(dC)))
    assert np.array_equal(bits(first), bits(oracle.crt_gemm(A, B, q)))


@pytest.mark.parametrize("m,n,k,panels", [(1000, 700, 900, 3), (512, 512, 256, 1), (300, 1100, 64, 8), (257, 255, 300, 2),
                                          (2000, 1500, 300, 32), (1800, 2600, 100, 64)])
def test_crt_host_buffer_path_matches_device_path(mgx, m, n, k, panels):
    """mgx_gemm_host with the CRT form (panels of 256 rows/columns prepared as they arrive; at
    each step the new row strip and column strip computed from them, with unequal numbers of
    row and column panels) gives the device path's result bit for bit."""
    import torch
    rng = np.random.default_rng(m + n + k)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    hA, hB = torch.from_numpy(A).pin_memory(), torch.from_numpy(B).pin_memory()
    hC = torch.empty((m, n), dtype=torch.float64).pin_memory()
    mgx.gemm_host(hA, hB, hC, form=mgx.FORM_CRT, splits=15, panels=panels)
    torch.cuda.synchronize()
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=15)
    assert np.array_equal(bits(hC.numpy()), bits(host(dC)))
    assert mgx.device_status() == 0


@pytest.mark.parametrize("m,n,k,q,ksplit", [
    (256, 256, 4096, 15, 4), (100, 300, 2000, 14, 3), (513, 130, 1000, 16, 16), (64, 64, 96, 12, 7),
    (257, 255, 4100, 11, 5), (40, 520, 700, 10, 64)])
def test_crt_splitk_bit_exact_vs_oracle(mgx, oracle, m, n, k, q, ksplit):
    """Split-K CRT form: the K slices' residue products are added modulo each p before the CRT
    rebuild, so the result equals the whole-K form's and the oracle's bit for bit (ksplit is
    clamped to the K blocks; uneven last slices included)."""
    import torch
    rng = np.random.default_rng(m + 3 * n + 5 * k + ksplit)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dA, dB, dC, moduli=q, ksplit=ksplit)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, q)))
    whole = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dA, dB, whole, moduli=q)
    assert torch.equal(whole.view(torch.int64), dC.view(torch.int64))
    assert mgx.device_status() == 0


def test_crt_splitk_beta_one_and_limits(mgx, oracle):
    import torch
    rng = np.random.default_rng(8)
    A, B, C0 = rng_matrix(rng, (130, 3000)), rng_matrix(rng, (3000, 90)), rng_matrix(rng, (130, 90))
    dC = dev(C0)
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=13, beta_one=True, ksplit=6)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, 13, C=C0.copy(), beta_one=True)))
    kmax = mgx.crt_kmax()
    assert mgx.crt_splitk_workspace_size(8, 8, kmax + 1, 15, 4) == 0
    assert mgx.crt_splitk_workspace_size(8, 8, kmax, 15, 4) > mgx.crt_workspace_size(8, 8, kmax, 15)
    X = torch.ones((4, kmax + 32), dtype=torch.float64, device="cuda")
    with pytest.raises(mgx.MgxError):
        mgx.gemm_ozaki_crt(X, X.t().contiguous(), torch.empty((4, 4), dtype=torch.float64, device="cuda"),
                           moduli=15, ksplit=4)
    assert mgx.device_status() == 0
