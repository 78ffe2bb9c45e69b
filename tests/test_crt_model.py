"""The CRT form's a-priori modulus count (mgx_crt_choose_moduli, a host function of the library)
checked on the CPU against the oracle's restatement: the chosen count meets the target against
the double-double product, and one modulus fewer does not always, so the rule is not wasteful."""
import numpy as np
import pytest

from conftest import rng_matrix


@pytest.mark.parametrize("k,kind", [(256, "wide"), (1024, "uniform"), (4096, "wide")])
def test_chosen_moduli_meet_the_target(mgx, oracle, k, kind):
    rng = np.random.default_rng(k)
    A, B = rng_matrix(rng, (48, k), kind), rng_matrix(rng, (k, 40), kind)
    ref = oracle.gemm_dd(A, B)
    q = mgx.crt_choose_moduli(k, 1e-15)
    assert 8 <= q <= 16
    assert oracle.error_metrics(oracle.crt_gemm(A, B, q), ref)["normwise"] <= 1e-15
    # two moduli fewer misses it by a wide margin: the rule sits near the edge
    assert oracle.error_metrics(oracle.crt_gemm(A, B, q - 2), ref)["normwise"] > 1e-15


def test_choice_grows_with_k_and_tightens_with_target(mgx):
    qs = [mgx.crt_choose_moduli(k, 1e-15) for k in (64, 1024, 16384, 130816)]
    assert qs == sorted(qs) and qs[-1] == 16
    assert mgx.crt_choose_moduli(4096, 1e-9) < mgx.crt_choose_moduli(4096, 1e-15)
    assert mgx.crt_kmax() == 130816


def test_biased_barrett_reduction_of_the_epilogue():
    """The epilogue's g mod p for an int32 accumulator of K <= KMAX int8 products
    (|g| <= 2^14 K): a = g + p floor(2^31 / p) wraps into (0, 2^32), q = umulhi(a, ceil(2^32 / p))
    is floor(a / p) or one more, and the unsigned min of r = a - q p and r + p is the residue.
    Restated in 32-bit wrap-around arithmetic over the range's edges and 2^22 random values per
    modulus (all 2 x 2^14 x 130816 + 1 values were checked once on the CPU, with no mismatch)."""
    rng = np.random.default_rng(1)
    G = 2 ** 14 * 130816
    edges = np.array([-G, -G + 1, -1, 0, 1, G - 1, G], np.int64)
    g = np.concatenate([edges, rng.integers(-G, G + 1, 2 ** 22, dtype=np.int64)])
    mask = np.uint64(2 ** 32 - 1)
    for p in (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193):
        M = np.uint64((2 ** 32 - 1) // p + 1)
        bias = np.uint64(p * (2 ** 31 // p))
        a = ((g.astype(np.uint64) & mask) + bias) & mask
        assert np.all(a > 0)
        r = (a - ((a * M) >> np.uint64(32)) * np.uint64(p)) & mask
        R = np.minimum(r, (r + np.uint64(p)) & mask)
        assert np.array_equal(R.astype(np.int64), np.mod(g, p)), p


def test_barrett_reduction_of_the_epilogue():
    """The split-K recombination's g mod p (any int32 g, every modulus): q = umulhi(|g|,
    ceil(2^32 / p)) is floor(|g| / p) or one more, corrected by one add, then the sign.  Restated
    here in uint64 arithmetic over every edge value and 2^22 random ones per modulus (the
    exhaustive check of all 2^32 inputs was run once on the CPU when it was written)."""
    rng = np.random.default_rng(0)
    edges = np.array([-2 ** 31, -2 ** 31 + 1, -1, 0, 1, 2 ** 31 - 1, 2 ** 31 - 2], np.int64)
    g = np.concatenate([edges, rng.integers(-2 ** 31, 2 ** 31, 2 ** 22, dtype=np.int64)])
    for p in (256, 255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197, 193):
        M = np.uint64((2 ** 32 - 1) // p + 1)
        a = np.abs(g).astype(np.uint64)
        q = (a * M) >> np.uint64(32)
        r = a.astype(np.int64) - (q * np.uint64(p)).astype(np.int64)
        r = np.where(r < 0, r + p, r)
        R = np.where((g >= 0) | (r == 0), r, p - r)
        assert np.array_equal(R, np.mod(g, p)), p

