"""validate_matrix_C replacement and the double-double error check on the GPU."""
import numpy as np
import pytest

from conftest import rng_matrix
from gpu_util import dev, host, ref_kernels, vp

pytestmark = pytest.mark.gpu


def test_validation_counts_like_the_reference(mgx, oracle):
    rng = np.random.default_rng(1)
    C = np.full((300, 257), 128.0)
    idx = rng.choice(C.size, 40, replace=False)
    C.flat[idx[:20]] += rng.uniform(1e-8, 1e-3, 20)   # invalid
    C.flat[idx[20:]] += 1e-14                          # inside the tolerances
    ok, v = mgx.validate_matrix_c(dev(C), 300, 257, 128.0)
    n, ma, mr = oracle.validate_constant(C, 128.0)
    assert not ok and v.invalid == n == 20
    assert v.max_abs_error == ma and v.max_rel_error == mr


def test_validation_counts_nonfinite(mgx, oracle):
    C = np.full((64, 64), 128.0)
    C[3, 4] = np.nan
    C[5, 6] = np.inf
    ok, v = mgx.validate_matrix_c(dev(C), 64, 64, 128.0)
    assert not ok and v.invalid == oracle.validate_constant(C, 128.0, count_nonfinite=True)[0] == 2


def test_validation_block_matches_reference_text(mgx, oracle, capfd):
    R = ref_kernels(oracle)
    C = np.full((40, 50), 100.0)
    C[1, 1] = 100.5
    dC = dev(C)
    mgx.validate_matrix_c(dC, 40, 50, 100.0, print_block=True)
    ours = capfd.readouterr().out
    assert "NUMERICAL VALIDATION" in ours and "Invalid elements   : 1" in ours and "Result             : FAIL" in ours
    if R is not None:
        R.ref_validate_matrix_C(vp(dC), 40, 50, 100.0, 1e-9, 1e-12)
        import ctypes
        ctypes.CDLL(None).fflush(None)
        theirs = capfd.readouterr().out
        assert theirs.strip() == ours.strip()


def test_dd_error_matches_cpu(mgx, oracle):
    import torch
    rng = np.random.default_rng(2)
    A, B = rng_matrix(rng, (150, 400), "wide"), rng_matrix(rng, (400, 130), "wide")
    C = oracle.ab_multiply(A, B)
    e_gpu = mgx.error_vs_dd(dev(A), dev(B), dev(C), floor_rel=2.0 ** -40)
    e_cpu = oracle.error_metrics(C, oracle.gemm_dd(A, B), floor_rel=2.0 ** -40)
    assert e_gpu["rows_checked"] == 150
    for key in ("normwise", "max_componentwise", "max_abs"):
        assert e_gpu[key] == pytest.approx(e_cpu[key], rel=1e-6, abs=1e-300)
    part = mgx.error_vs_dd(dev(A), dev(B), dev(C), row_start=50, row_count=20)
    assert part["rows_checked"] == 20


def test_fill_is_counter_based(mgx):
    import torch
    X = torch.empty((100, 64), dtype=torch.float64, device="cuda")
    Y = torch.empty((100, 64), dtype=torch.float64, device="cuda")
    mgx.fill_matrix(X, 2, e_range=20, seed=5)
    mgx.fill_matrix(Y, 2, e_range=20, seed=5)
    x = host(X)
    assert np.array_equal(x, host(Y)) and np.all(np.abs(x) < 2.0 ** 20)
    mgx.fill_matrix(X, 1, seed=6)
    x = host(X)
    assert x.min() >= -1.0 and x.max() < 1.0 and abs(x.mean()) < 0.05
