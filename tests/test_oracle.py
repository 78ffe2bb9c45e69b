"""CPU oracle against MGXBench's own rules and known answers (no GPU)."""
from fractions import Fraction

import numpy as np
import pytest

from conftest import rng_matrix


def bits(x):
    return np.ascontiguousarray(x).view(np.uint64)


@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (3, 5, 7), (31, 33, 65), (129, 257, 300), (64, 1030, 513), (7, 9, 0)])
def test_blocked_chain_equals_reference_loop(oracle, m, n, k):
    """The blocked oracle keeps one sequential FMA chain per output (mulmat_kernel.cu:72-73)."""
    rng = np.random.default_rng(m * 1000 + n + k)
    A, B = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n))
    assert np.array_equal(bits(oracle.ab_multiply(A, B)), bits(oracle.ab_multiply(A, B, naive=True)))


def test_constant_known_answer(oracle):
    """A = 1, B = 2 gives C = 2K exactly (1D-row-block/mmb.cu:944-958)."""
    for N in (32, 100, 257):
        C = oracle.ab_multiply(np.ones((N, N)), np.full((N, N), 2.0))
        assert np.all(C == 2.0 * N)
        assert oracle.validate_constant(C, 2.0 * N) == (0, 0.0, 0.0)
        assert oracle.validate_2d(C, 2.0 * N) == -1


def test_integer_products_exact(oracle):
    rng = np.random.default_rng(3)
    A = rng.integers(-1000, 1000, (40, 70)).astype(np.float64)
    B = rng.integers(-1000, 1000, (70, 30)).astype(np.float64)
    exact = (A.astype(np.int64) @ B.astype(np.int64)).astype(np.float64)
    assert np.array_equal(oracle.ab_multiply(A, B), exact)
    assert np.array_equal(oracle.summa2d(A, B, 16), exact)


@pytest.mark.parametrize("k,req,want", [(16384, 0, 2048), (1000, 0, 992), (20, 0, 20), (16384, 100, 96),
                                        (16384, 31, 31), (64, 5000, 64), (8, -3, 8)])
def test_pipeline_k_chunk_rule(oracle, k, req, want):
    """pipeline_k_chunk_from_env (1D-row-block/mmb.cu:109-128)."""
    assert oracle.pipeline_k_chunk(k, req) == want


def test_accumulate_is_partial_then_add(oracle):
    """C += (chunk partial), one rounding (mulmat_kernel.cu:113-141); A beyond k_total reads 0."""
    rng = np.random.default_rng(5)
    m, n, kt = 9, 11, 40
    A, B = rng_matrix(rng, (m, kt)), rng_matrix(rng, (kt, n))
    C0 = rng_matrix(rng, (m, n))
    C = C0.copy()
    oracle.ab_multiply_accumulate(A, B[16:40], C, 16, 24)
    P = oracle.ab_multiply(A[:, 16:40], B[16:40])
    assert np.array_equal(bits(C), bits(C0 + P))
    # chunk running past k_total: those A columns are zero
    C2 = C0.copy()
    Bc = rng_matrix(rng, (16, n))
    oracle.ab_multiply_accumulate(A, Bc, C2, 32, 16)
    P2 = oracle.ab_multiply(np.hstack([A[:, 32:40], np.zeros((m, 8))]), Bc)
    assert np.array_equal(bits(C2), bits(C0 + P2))


def test_mm1d_structures(oracle):
    rng = np.random.default_rng(9)
    N = 96
    A, B = rng_matrix(rng, (N, N)), rng_matrix(rng, (N, N))
    sync = oracle.mm1d(A, B, ranks=4, chunked=False, k_chunk=32)
    assert np.array_equal(bits(sync), bits(oracle.ab_multiply(A, B)))
    ch = oracle.mm1d(A, B, ranks=4, chunked=True, k_chunk=32)
    ref = np.zeros((N, N))
    for c in range(3):
        ref += oracle.ab_multiply(A[:, 32 * c:32 * c + 32], B[32 * c:32 * c + 32])
    assert np.array_equal(bits(ch), bits(ref))


def test_validation_rules(oracle):
    C = np.full(10, 64.0)
    C[3] = 64.0 + 1e-8      # abs > 1e-9 and rel > 1e-12: invalid
    C[4] = 64.0 + 1e-13     # within both
    C[5] = np.nan           # the reference's comparisons are false for NaN
    n, ma, mr = oracle.validate_constant(C, 64.0)
    assert n == 1 and ma == pytest.approx(1e-8, rel=1e-6) and mr == pytest.approx(1e-8 / 64, rel=1e-6)
    n2, _, _ = oracle.validate_constant(C, 64.0, count_nonfinite=True)
    assert n2 == 2
    assert oracle.validate_2d(C, 64.0) == 3


def test_double_double_against_exact_rationals(oracle):
    rng = np.random.default_rng(11)
    A, B = rng_matrix(rng, (5, 200), "wide"), rng_matrix(rng, (200, 4), "wide")
    hi, lo, ab = oracle.gemm_dd(A, B)
    for i in range(5):
        for j in range(4):
            exact = sum(Fraction(A[i, k]) * Fraction(B[k, j]) for k in range(200))
            err = abs(Fraction(hi[i, j]) + Fraction(lo[i, j]) - exact)
            assert err <= Fraction(ab[i, j]) * Fraction(2.0 ** -100)


def test_error_metrics(oracle):
    rng = np.random.default_rng(12)
    A, B = rng_matrix(rng, (30, 50)), rng_matrix(rng, (50, 20))
    ref = oracle.gemm_dd(A, B)
    e = oracle.error_metrics(ref[0], ref)
    assert e["normwise"] < 1e-16 and e["max_componentwise"] < 2.0 ** -52


# ---------------------------------------------------------------- Ozaki form (this project's algorithm)
def test_ozaki_digits_reconstruct(oracle):
    rng = np.random.default_rng(13)
    A, B = rng_matrix(rng, (17, 40), "wide"), rng_matrix(rng, (40, 23), "wide")
    s = 9
    da, db, ea, eb = oracle.ozaki_split(A, B, s)
    assert da.min() >= -64 and da.max() <= 64 and db.min() >= -64 and db.max() <= 64
    assert np.all(da[:, :, 40:] == 0) and np.all(db[:, :, 40:] == 0)
    w = np.exp2(-7.0 * np.arange(s))
    recA = np.einsum("t,tik->ik", w, da[:, :, :40].astype(np.float64)) * np.exp2(ea - 6.0)[:, None]
    assert np.max(np.abs(recA - A) / np.exp2(ea)[:, None]) < 2.0 ** (-7 * s + 1)
    recB = np.einsum("t,tjk->jk", w, db[:, :, :40].astype(np.float64)) * np.exp2(eb - 6.0)[:, None]
    assert np.max(np.abs(recB - B.T) / np.exp2(eb)[:, None]) < 2.0 ** (-7 * s + 1)


def test_ozaki_exact_on_short_integers(oracle):
    rng = np.random.default_rng(14)
    A = rng.integers(-100, 100, (20, 33)).astype(np.float64)
    B = rng.integers(-100, 100, (33, 21)).astype(np.float64)
    exact = (A.astype(np.int64) @ B.astype(np.int64)).astype(np.float64)
    assert np.array_equal(oracle.ozaki_gemm(A, B, 3), exact)
    assert np.array_equal(oracle.ozaki_gemm(np.ones((8, 64)), np.full((64, 8), 2.0), 2), np.full((8, 8), 128.0))


def test_ozaki_error_falls_with_splits(oracle):
    rng = np.random.default_rng(15)
    A, B = rng_matrix(rng, (48, 300), "wide"), rng_matrix(rng, (300, 40), "wide")
    ref = oracle.gemm_dd(A, B)
    errs = [oracle.error_metrics(oracle.ozaki_gemm(A, B, s), ref)["normwise"] for s in range(3, 10)]
    assert all(b < a for a, b in zip(errs, errs[1:-1]))
    assert errs[5] <= 1e-15   # s = 8 meets the 1e-15 target on wide-exponent inputs
    assert errs[6] <= 1e-16


def test_ozaki_rejects_nonfinite(oracle):
    A = np.ones((4, 4))
    A[1, 2] = np.inf
    with pytest.raises(ValueError):
        oracle.ozaki_gemm(A, np.ones((4, 4)), 4)


def test_ozaki_kmax_bounds_int32(oracle):
    for s in range(2, 13):
        km = oracle.ozaki_kmax(s)
        assert s * 64 * 64 * km < 2 ** 31 <= s * 64 * 64 * (km + 1)


def test_ozaki_splitk_restatement(oracle):
    """The split-K restatement: one slice is the plain form bit for bit; more slices change only
    the final additions (same exponents and digits), so the error stays at the unsplit level."""
    rng = np.random.default_rng(21)
    A = rng.uniform(-1, 1, (40, 700)) * np.exp2(rng.integers(-20, 21, (40, 700)))
    B = rng.uniform(-1, 1, (700, 33)) * np.exp2(rng.integers(-20, 21, (700, 33)))
    one = oracle.ozaki_gemm_splitk(A, B, 8, 1)
    assert np.array_equal(one.view(np.uint64), oracle.ozaki_gemm(A, B, 8).view(np.uint64))
    ref = oracle.gemm_dd(A, B)
    e1 = oracle.error_metrics(one, ref)["normwise"]
    for ks in (2, 5, 22, 100):
        e = oracle.error_metrics(oracle.ozaki_gemm_splitk(A, B, 8, ks), ref)["normwise"]
        assert e <= 2 * e1 + 1e-16
    with pytest.raises(ValueError):
        oracle.ozaki_gemm_splitk(np.zeros((2, 70000)), np.zeros((70000, 2)), 8, 2)


# ------------------------------------------------------------------ CRT form (Ozaki scheme II)
# The reference has no INT8 form, so nothing of its own pins this restatement; exact integer
# arithmetic does: every step before the final FP64 rounding is integer work.
CRT_MODULI = (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193)


def _crt_exact(A, B, q, sg, tu):
    """Scaled integers A' = rint(A 2^sigma), B' = rint(B 2^tau) (ties to even, exact rationals)
    and the exact integer product C' = A' B'."""
    Ai = [[round(Fraction(float(a)) * Fraction(2) ** int(s)) for a in row] for row, s in zip(A, sg)]
    Bi = [[round(Fraction(float(B[kk, j])) * Fraction(2) ** int(tu[j])) for j in range(B.shape[1])]
          for kk in range(B.shape[0])]
    C = [[sum(Ai[i][kk] * Bi[kk][j] for kk in range(len(Bi))) for j in range(B.shape[1])] for i in range(len(Ai))]
    return Ai, Bi, C


@pytest.mark.parametrize("q,kind,er", [(15, "wide", 20), (12, "uniform", 0), (16, "wide", 35), (9, "wide", 5)])
def test_crt_oracle_against_exact_integers(oracle, q, kind, er):
    import math
    rng = np.random.default_rng(q * 7 + er)
    m, n, k = 7, 6, 150
    A, B = rng_matrix(rng, (m, k), kind, er), rng_matrix(rng, (k, n), kind, er)
    A[2] = 0.0
    sg, tu, rc = oracle.crt_scales(A, B, q)
    assert rc == 0
    P = math.prod(CRT_MODULI[:q])
    L = P.bit_length()
    alpha, beta = (L - 3) // 2, L - 3 - (L - 3) // 2
    # the scale puts every row / column 2-norm at or below 2^alpha / 2^beta
    for i in range(m):
        if np.any(A[i]):
            assert sum((Fraction(float(a)) * Fraction(2) ** int(sg[i])) ** 2 for a in A[i]) <= Fraction(4) ** alpha
    for j in range(n):
        assert sum((Fraction(float(b)) * Fraction(2) ** int(tu[j])) ** 2 for b in B[:, j]) <= Fraction(4) ** beta
    Ai, Bi, Cx = _crt_exact(A, B, q, sg, tu)
    # residues: the symmetric residue of the exact scaled integer, modulus by modulus
    ra, rb, _, _ = oracle.crt_residues(A, B, q)
    for l, p in enumerate(CRT_MODULI[:q]):
        sym = (lambda x: ((x + 128) % 256) - 128) if p == 256 else (lambda x: ((x + p // 2) % p) - p // 2)
        assert all(int(ra[l, i, kk]) == sym(Ai[i][kk]) for i in range(m) for kk in range(k))
        assert all(int(rb[l, j, kk]) == sym(Bi[kk][j]) for j in range(n) for kk in range(k))
    # every exact product lies within a quarter of P (unique CRT reconstruction), and the FP64
    # result is that integer scaled back, within the two roundings of the recombination
    C = oracle.crt_gemm(A, B, q)
    for i in range(m):
        for j in range(n):
            assert 4 * abs(Cx[i][j]) < P
            exact = Fraction(Cx[i][j]) * Fraction(2) ** (-int(sg[i]) - int(tu[j]))
            if exact == 0:
                assert C[i, j] == 0.0
            else:
                assert abs(Fraction(float(C[i, j])) - exact) <= 2 * abs(exact) * Fraction(2) ** -53

