"""Native FP64 path on the GPU against the oracle (reference-kernel arithmetic) and MGXBench's own
kernels.  Tolerance: the two compute the same sums in different orders, so for every element
|C - C_ref| <= 2 gamma_K (|A||B|)_ij, gamma_K = K u / (1 - K u) (any-order summation bound);
integer-valued products are exact."""
import numpy as np
import pytest

from conftest import gamma, rng_matrix
from gpu_util import bits, dev, host, ref_kernels, vp

pytestmark = pytest.mark.gpu

SHAPES = [(1, 1, 1), (7, 9, 13), (128, 128, 32), (129, 257, 300), (256, 384, 512), (333, 127, 1000),
          (64, 64, 2), (1024, 1024, 1024)]


def check_close(C, A, B, oracle, k):
    hi, lo, ab = oracle.gemm_dd(A, B)
    ref = oracle.ab_multiply(A, B)
    bound = 2 * gamma(max(k, 1)) * ab + 1e-300
    assert np.all(np.abs(C - ref) <= bound)
    e_ours = oracle.error_metrics(C, (hi, lo, ab))["normwise"]
    e_ref = oracle.error_metrics(ref, (hi, lo, ab))["normwise"]
    assert e_ours <= max(4 * e_ref, 1e-15)


@pytest.mark.parametrize("m,n,k", SHAPES)
def test_ab_multiply_matches_oracle(mgx, oracle, m, n, k):
    import torch
    rng = np.random.default_rng(m + 7 * n + 13 * k)
    A, B = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n))
    dA, dB = dev(A), dev(B)
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.ab_multiply(dA, dB, dC)
    check_close(host(dC), A, B, oracle, k)
    assert mgx.device_status() == 0


@pytest.mark.parametrize("N", [32, 200, 1024])
def test_constant_known_answer_exact(mgx, N):
    import torch
    A = torch.ones((N, N), dtype=torch.float64, device="cuda")
    B = torch.full((N, N), 2.0, dtype=torch.float64, device="cuda")
    C = torch.empty((N, N), dtype=torch.float64, device="cuda")
    mgx.ab_multiply(A, B, C)
    ok, v = mgx.validate_matrix_c(C, N, N, 2.0 * N)
    assert ok and v.invalid == 0 and v.max_abs_error == 0.0
    assert torch.all(C == 2.0 * N)


def test_integer_products_exact(mgx):
    rng = np.random.default_rng(1)
    A = rng.integers(-2000, 2000, (300, 500)).astype(np.float64)
    B = rng.integers(-2000, 2000, (500, 260)).astype(np.float64)
    import torch
    dC = torch.empty((300, 260), dtype=torch.float64, device="cuda")
    mgx.ab_multiply(dev(A), dev(B), dC)
    assert np.array_equal(host(dC), (A.astype(np.int64) @ B.astype(np.int64)).astype(np.float64))


@pytest.mark.parametrize("k_total,k_offset,k_chunk", [(512, 0, 512), (512, 128, 256), (1000, 992, 8),
                                                      (300, 37, 100), (100, 64, 64), (96, 96, 32)])
def test_accumulate_matches_oracle(mgx, oracle, k_total, k_offset, k_chunk):
    import torch
    rng = np.random.default_rng(k_total + k_offset)
    m, n = 130, 70
    A = rng_matrix(rng, (m, k_total))
    Bc = rng_matrix(rng, (k_chunk, n))
    C0 = rng_matrix(rng, (m, n))
    dC = dev(C0)
    mgx.ab_multiply_accumulate_async(dev(A), dev(Bc), dC, m, n, k_total, k_offset, k_chunk, k_total, n, n)
    C = host(dC)
    Cref = C0.copy()
    oracle.ab_multiply_accumulate(A, Bc, Cref, k_offset, k_chunk)
    live = max(0, min(k_chunk, k_total - k_offset))
    Aw = np.zeros((m, k_chunk))
    Aw[:, :live] = A[:, k_offset:k_offset + live]
    _, _, ab = oracle.gemm_dd(Aw, Bc)
    assert np.all(np.abs(C - Cref) <= 2 * gamma(k_chunk) * ab + 2.0 ** -52 * np.abs(Cref) + 1e-300)


def test_generic_loader_odd_leading_dimension(mgx, oracle):
    """lda = 301 (odd) cannot be described to TMA; the plain-load producer handles it."""
    import torch
    rng = np.random.default_rng(2)
    m, n, k = 190, 150, 300
    Afull = rng_matrix(rng, (m, 301))
    B = rng_matrix(rng, (k, n))
    dA = dev(Afull)
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.ab_multiply(dA, dev(B), dC, m=m, n=n, k=k, lda=301, ldb=n, ldc=n)
    check_close(host(dC), Afull[:, :k], B, oracle, k)


def test_beta_one_and_streams(mgx, oracle):
    import torch
    rng = np.random.default_rng(4)
    A, B, C0 = rng_matrix(rng, (256, 128)), rng_matrix(rng, (128, 192)), rng_matrix(rng, (256, 192))
    s = torch.cuda.Stream()
    dC = dev(C0)
    with torch.cuda.stream(s):
        mgx.gemm_fp64(dev(A), dev(B), dC, beta_one=True, stream=s)
    s.synchronize()
    C = host(dC)
    P = oracle.ab_multiply(A, B)
    _, _, ab = oracle.gemm_dd(A, B)
    assert np.all(np.abs(C - (C0 + P)) <= 2 * gamma(128) * ab + 2.0 ** -52 * np.abs(C0 + P))


def test_reference_kernels_pin_the_oracle(mgx, oracle):
    """MGXBench's own sharedABMultiply / sharedABMultiplyAccumulate (built from its sources) give
    bit-identical results to the oracle's restatement; ours agree within the stated bound."""
    import torch
    R = ref_kernels(oracle)
    if R is None:
        pytest.skip("oracle/_ref/libref_mulmat.so not built")
    rng = np.random.default_rng(6)
    for (m, n, k) in [(33, 47, 65), (128, 96, 257), (100, 200, 300)]:
        A, B = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n))
        dA, dB = dev(A), dev(B)
        dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
        assert R.ref_ab_multiply(vp(dA), vp(dB), vp(dC), m, n, k, k, n, n) == 0
        Cref_gpu = host(dC)
        assert np.array_equal(bits(Cref_gpu), bits(oracle.ab_multiply(A, B)))
        dC2 = torch.empty((m, n), dtype=torch.float64, device="cuda")
        mgx.ab_multiply(dA, dB, dC2)
        check_close(host(dC2), A, B, oracle, k)
        # accumulate form with a K chunk (the 1D pipeline's call, 1D-row-block/mmb.cu:791)
        C0 = rng_matrix(rng, (m, n))
        kc = k // 2
        dC3 = dev(C0)
        assert R.ref_ab_multiply_accumulate(vp(dA), vp(dB[kc:]), vp(dC3), m, n, k, kc, k - kc, k, n, n, None) == 0
        Cacc = C0.copy()
        oracle.ab_multiply_accumulate(A, B[kc:], Cacc, kc, k - kc)
        assert np.array_equal(bits(host(dC3)), bits(Cacc))


@pytest.mark.parametrize("m,n,k,ks", [(200, 150, 2000, 4), (129, 257, 300, 2), (7, 9, 13, 8), (333, 127, 1000, 16),
                                      (256, 256, 4096, 64), (64, 64, 64, 3)])
def test_splitk_matches_oracle(mgx, oracle, m, n, k, ks):
    """Split-K: each slice is an FP64 sum, slices summed in order; the any-order bound still holds."""
    import torch
    rng = np.random.default_rng(m * 3 + n + k + ks)
    A, B = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n))
    dA, dB = dev(A), dev(B)
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dA, dB, dC, ksplit=ks)
    check_close(host(dC), A, B, oracle, k)
    # deterministic: slices are reduced in a fixed order
    dC2 = torch.empty_like(dC)
    mgx.gemm_fp64(dA, dB, dC2, ksplit=ks)
    assert np.array_equal(bits(host(dC)), bits(host(dC2)))
    assert mgx.device_status() == 0


def test_splitk_accumulates_and_checks_workspace(mgx, oracle):
    import ctypes
    import torch
    rng = np.random.default_rng(5)
    m, n, k = 150, 98, 1500
    A, B, C0 = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n)), rng_matrix(rng, (m, n))
    dC = dev(C0)
    mgx.gemm_fp64(dev(A), dev(B), dC, beta_one=True, ksplit=6)
    ref = C0 + oracle.ab_multiply(A, B)
    _, _, ab = oracle.gemm_dd(A, B)
    assert np.all(np.abs(host(dC) - ref) <= 2 * gamma(k + 1) * (ab + np.abs(C0)) + 1e-300)
    need = mgx.fp64_splitk_workspace_size(m, n, k, 6)
    assert need >= 6 * m * n * 8
    assert mgx.fp64_splitk_workspace_size(m, n, 31, 6) == 0  # one K block: one slice
    small = torch.empty(need // 2, dtype=torch.uint8, device="cuda")
    rc = mgx.lib().mgx_gemm_fp64_splitk(vp(dev(A)), vp(dev(B)), vp(dC), m, n, k, k, n, n, 0, 6, vp(small),
                                        small.numel(), None)
    assert rc == -5  # MGX_E_WORKSPACE


@pytest.mark.parametrize("m,n,k,ksplit", [(1, 1, 1, 1), (65, 129, 300, 1), (64, 128, 32, 1), (333, 127, 1000, 4),
                                          (1024, 1024, 1024, 1), (1024, 1024, 1024, 2), (2200, 300, 200, 1),
                                          (130, 260, 4096, 8)])
def test_small_tile_is_bit_identical_to_the_default_tile(mgx, oracle, m, n, k, ksplit):
    """64 x 128 output tiles (mgx_gemm_fp64_tiled, tile_m = 64) reduce every element over K in the
    same order as the 128 x 128 tiles: the results are identical, whole-K and split-K, and inside
    the oracle's bound."""
    import torch
    rng = np.random.default_rng(m + n + k + ksplit)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    c64 = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    c128 = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dA, dB, c64, ksplit=ksplit, tile_m=64)
    mgx.gemm_fp64(dA, dB, c128, ksplit=ksplit)
    assert torch.equal(c64.view(torch.int64), c128.view(torch.int64))
    check_close(host(c64), A, B, oracle, k)
    assert mgx.device_status() == 0


def test_small_tile_beta_one_and_odd_pitch(mgx, oracle):
    """beta = 1 and operands that need the even-pitch copy (odd leading dimensions) through the
    64-row tile."""
    import torch
    rng = np.random.default_rng(5)
    m, n, k = 150, 100, 300          # leading dimensions 301 and 101
    Ab, Bb = rng_matrix(rng, (m, k + 1)), rng_matrix(rng, (k, n + 1))
    A, B = Ab[:, :k], Bb[:, :n]
    C0 = rng_matrix(rng, (m, n))
    dAb, dBb = dev(Ab), dev(Bb)
    dA, dB = dAb[:, :k], dBb[:, :n]
    c64, c128 = dev(C0), dev(C0)
    mgx.gemm_fp64(dA, dB, c64, beta_one=True, tile_m=64)
    mgx.gemm_fp64(dA, dB, c128, beta_one=True)
    assert torch.equal(c64.view(torch.int64), c128.view(torch.int64))
    ref = C0 + oracle.ab_multiply(np.ascontiguousarray(A), np.ascontiguousarray(B))
    assert np.all(np.abs(host(c64) - ref) <= 2 * gamma(k + 1) * (np.abs(A) @ np.abs(B) + np.abs(C0)))


@pytest.mark.parametrize("m,n,k,ksplit", [(1, 1, 1, 1), (65, 129, 300, 1), (64, 128, 32, 1), (333, 127, 1000, 4),
                                          (1024, 1024, 1024, 1), (1024, 1024, 1024, 2), (2200, 300, 200, 1),
                                          (130, 260, 4096, 8)])
def test_small_tile_is_bit_identical_to_the_default_tile(mgx, oracle, m, n, k, ksplit):
    """64 x 128 output tiles (mgx_gemm_fp64_tiled, tile_m = 64) reduce every element over K in the
    same order as the 128 x 128 tiles: the results are identical, whole-K and split-K, and inside
    the oracle's bound."""
    import torch
    rng = np.random.default_rng(m + n + k + ksplit)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    c64 = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    c128 = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dA, dB, c64, ksplit=ksplit, tile_m=64)
    mgx.gemm_fp64(dA, dB, c128, ksplit=ksplit)
    assert torch.equal(c64.view(torch.int64), c128.view(torch.int64))
    check_close(host(c64), A, B, oracle, k)
    assert mgx.device_status() == 0


def test_small_tile_beta_one_and_odd_pitch(mgx, oracle):
    """beta = 1 and operands that need the even-pitch copy (odd leading dimensions) through the
    64-row tile."""
    import torch
    rng = np.random.default_rng(5)
    m, n, k = 150, 100, 300          # leading dimensions 301 and 101
    Ab, Bb = rng_matrix(rng, (m, k + 1)), rng_matrix(rng, (k, n + 1))
    A, B = Ab[:, :k], Bb[:, :n]
    C0 = rng_matrix(rng, (m, n))
    dAb, dBb = dev(Ab), dev(Bb)
    dA, dB = dAb[:, :k], dBb[:, :n]
    c64, c128 = dev(C0), dev(C0)
    mgx.gemm_fp64(dA, dB, c64, beta_one=True, tile_m=64)
    mgx.gemm_fp64(dA, dB, c128, beta_one=True)
    assert torch.equal(c64.view(torch.int64), c128.view(torch.int64))
    ref = C0 + oracle.ab_multiply(np.ascontiguousarray(A), np.ascontiguousarray(B))
    assert np.all(np.abs(host(c64) - ref) <= 2 * gamma(k + 1) * (np.abs(A) @ np.abs(B) + np.abs(C0)))


@pytest.mark.parametrize("m,n,k", [(1024, 1024, 1024), (64, 128, 32), (64, 128, 4096), (333, 127, 1000),
                                   (2200, 300, 200), (100, 700, 5000), (1, 1, 1), (4096, 2048, 512)])
def test_streamk_within_bound_and_deterministic(mgx, oracle, m, n, k):
    """Stream-K over 64 x 128 tiles (mgx_gemm_fp64_streamk): every CTA takes an equal share of all
    tiles' K blocks, and a tile split between CTAs is finished by the last to arrive, adding the
    pieces in K order.  Shapes with one unit per CTA, a single tile split into 128 pieces, and
    tiles split at uneven places; the result is inside the oracle's bound and identical on a
    second run."""
    import torch
    rng = np.random.default_rng(m * 5 + n + k)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    c1 = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    c2 = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dA, dB, c1, ksplit=0)
    mgx.gemm_fp64(dA, dB, c2, ksplit=0)
    assert torch.equal(c1.view(torch.int64), c2.view(torch.int64))
    check_close(host(c1), A, B, oracle, k)
    assert mgx.device_status() == 0


def test_streamk_tickets_need_no_reset(mgx, oracle):
    """The stream-K tickets are tagged per launch instead of being cleared before it: a workspace
    full of arbitrary bytes, and one left by a product of another tiling (tickets of other tiles
    at other counts), give the same bits as a fresh zeroed workspace."""
    import torch
    rng = np.random.default_rng(77)
    m, n, k = 1024, 1024, 1024
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    need = mgx.lib().mgx_fp64_streamk_workspace_size(m, n, k)
    fresh = mgx.OzakiWorkspace()
    fresh.get(need).zero_()
    ref = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dA, dB, ref, ksplit=0, workspace=fresh)
    junk = mgx.OzakiWorkspace()
    buf = junk.get(need)
    buf.copy_(torch.from_numpy(rng.integers(0, 256, buf.numel(), dtype=np.uint8)).cuda())
    c = torch.empty_like(ref)
    mgx.gemm_fp64(dA, dB, c, ksplit=0, workspace=junk)
    assert torch.equal(c.view(torch.int64), ref.view(torch.int64))
    # another tiling on the same workspace first, then this product again, twice in a row
    A2, B2 = rng_matrix(rng, (333, 5000), "wide"), rng_matrix(rng, (5000, 700), "wide")
    c2 = torch.empty((333, 700), dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dev(A2), dev(B2), c2, ksplit=0, workspace=junk)
    for _ in range(2):
        c.fill_(np.nan)
        mgx.gemm_fp64(dA, dB, c, ksplit=0, workspace=junk)
        assert torch.equal(c.view(torch.int64), ref.view(torch.int64))
    check_close(host(ref), A, B, oracle, k)
    assert mgx.device_status() == 0


def test_streamk_beta_one_and_odd_pitch(mgx, oracle):
    import torch
    rng = np.random.default_rng(8)
    m, n, k = 150, 100, 1300
    Ab, Bb = rng_matrix(rng, (m, k + 1)), rng_matrix(rng, (k, n + 1))
    A, B = Ab[:, :k], Bb[:, :n]
    C0 = rng_matrix(rng, (m, n))
    dAb, dBb = dev(Ab), dev(Bb)
    dC = dev(C0)
    mgx.gemm_fp64(dAb[:, :k], dBb[:, :n], dC, beta_one=True, ksplit=0)
    ref = C0 + oracle.ab_multiply(np.ascontiguousarray(A), np.ascontiguousarray(B))
    assert np.all(np.abs(host(dC) - ref) <= 2 * gamma(k + 1) * (np.abs(A) @ np.abs(B) + np.abs(C0)))
    assert mgx.device_status() == 0


@pytest.mark.parametrize("ksplit,tile_m", [(1, 128), (1, 64), (0, 64), (4, 128)])
def test_dependent_launches_keep_stream_order(mgx, ksplit, tile_m):
    """The FP64 kernels are programmatic dependent launches: each one's set-up overlaps the end of
    the previous kernel in the stream, and it touches memory only after that kernel has finished.
    Chained products (each reads the previous one's output) and repeated C += A B on one C,
    issued back to back, give the same bits as the same calls with a full synchronisation
    between them."""
    import torch
    rng = np.random.default_rng(31 + ksplit + tile_m)
    n = 512
    A = dev(rng_matrix(rng, (n, n))) / n
    B = dev(rng_matrix(rng, (n, n))) / n

    def chain(sync):
        xs = [A]
        for _ in range(4):
            y = torch.empty_like(A)
            mgx.gemm_fp64(xs[-1], B, y, ksplit=ksplit, tile_m=tile_m)
            if sync:
                torch.cuda.synchronize()
            xs.append(y)
        c = torch.zeros_like(A)
        for _ in range(4):
            mgx.gemm_fp64(A, B, c, beta_one=True, ksplit=ksplit, tile_m=tile_m)
            if sync:
                torch.cuda.synchronize()
        torch.cuda.synchronize()
        return xs[1:], c

    ys1, c1 = chain(False)
    ys2, c2 = chain(True)
    for a, b in zip(ys1, ys2):
        assert torch.equal(a.view(torch.int64), b.view(torch.int64))
    assert torch.equal(c1.view(torch.int64), c2.view(torch.int64))
    assert mgx.device_status() == 0
