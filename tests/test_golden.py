"""The oracle reproduces MGXBench's own kernels bit for bit (fixtures made by
tests/golden/make_golden.py from the reference's unmodified mulmat_kernel.cu on a GPU)."""
import numpy as np
import pytest

from conftest import ROOT

GOLDEN = ROOT / "tests" / "golden" / "ref_kernels.npz"
pytestmark = pytest.mark.skipif(not GOLDEN.exists(), reason="golden fixtures not generated yet")


def bits(x):
    return np.ascontiguousarray(x).view(np.uint64)


def test_multiply_fixtures(oracle):
    g = np.load(GOLDEN)
    cases = sorted({k.split("_")[0] for k in g.files if k.startswith("mul")})
    assert cases
    for c in cases:
        assert np.array_equal(bits(oracle.ab_multiply(g[c + "_A"], g[c + "_B"])), bits(g[c + "_C"])), c


def test_accumulate_fixtures(oracle):
    g = np.load(GOLDEN)
    cases = sorted({k.split("_")[0] for k in g.files if k.startswith("acc")})
    assert cases
    for c in cases:
        m, n, kt, ko, kc = (int(x) for x in g[c + "_args"])
        C = g[c + "_C0"].copy()
        oracle.ab_multiply_accumulate(g[c + "_A"], g[c + "_B"], C, ko, kc)
        assert np.array_equal(bits(C), bits(g[c + "_C"])), c


def test_validation_text_format():
    g = np.load(GOLDEN)
    text = str(g["validation_text"])
    assert text.count("NUMERICAL VALIDATION") == 2
    assert "Invalid elements   : 1" in text and "Result             : FAIL" in text
    assert "Result             : PASS" in text
