"""Randomised shapes (seeded): the Ozaki form (whole-K and split-K, every split count) is
bit-identical to the oracle's restatement, and the native FP64 form (whole-K and split-K) stays
within the any-order summation bound, on ragged m, n, k including odd leading dimensions.  The
CRT form (every modulus count) is bit-identical to its restatement on ragged shapes."""
import numpy as np
import pytest

from conftest import gamma, rng_matrix
from gpu_util import bits, dev, host

pytestmark = pytest.mark.gpu

CASES = []
_rng = np.random.default_rng(2026)
for _ in range(24):
    CASES.append((int(_rng.integers(1, 300)), int(_rng.integers(1, 300)), int(_rng.integers(1, 700)),
                  int(_rng.integers(2, 13)), int(_rng.choice([1, 1, 2, 3, 5, 16]))))


@pytest.mark.parametrize("m,n,k,s,ks", CASES)
def test_random_shape(mgx, oracle, m, n, k, s, ks):
    import torch
    rng = np.random.default_rng(m * 1000003 + n * 1009 + k * 7 + s + ks)
    A, B = rng_matrix(rng, (m, k), "wide"), rng_matrix(rng, (k, n), "wide")
    dA, dB = dev(A), dev(B)
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dA, dB, dC, splits=s, ksplit=ks)
    ref = oracle.ozaki_gemm_splitk(A, B, s, ks) if ks > 1 else oracle.ozaki_gemm(A, B, s)
    assert np.array_equal(bits(host(dC)), bits(ref))
    dF = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_fp64(dA, dB, dF, ksplit=ks)
    _, _, ab = oracle.gemm_dd(A, B)
    assert np.all(np.abs(host(dF) - oracle.ab_multiply(A, B)) <= 2 * gamma(max(k, 1)) * ab + 1e-300)
    assert mgx.device_status() == 0


CRT_CASES = []
_rng2 = np.random.default_rng(2027)
for _ in range(16):
    CRT_CASES.append((int(_rng2.integers(1, 600)), int(_rng2.integers(1, 600)), int(_rng2.integers(1, 1500)),
                      int(_rng2.integers(8, 17)), int(_rng2.choice([0, 5, 20, 40]))))


@pytest.mark.parametrize("m,n,k,q,er", CRT_CASES)
def test_random_shape_crt(mgx, oracle, m, n, k, q, er):
    """The CRT form on ragged shapes (tiles of 256 partly filled, K not a multiple of 32) and
    exponent spreads from none to 2^+-40: bit-identical to the oracle's restatement."""
    import torch
    rng = np.random.default_rng(m * 7919 + n * 104729 + k * 13 + q + er)
    kind = "wide" if er else "uniform"
    A, B = rng_matrix(rng, (m, k), kind, max(er, 1)), rng_matrix(rng, (k, n), kind, max(er, 1))
    dC = torch.full((m, n), np.nan, dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki_crt(dev(A), dev(B), dC, moduli=q)
    assert np.array_equal(bits(host(dC)), bits(oracle.crt_gemm(A, B, q)))
    assert mgx.device_status() == 0
