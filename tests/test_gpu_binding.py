"""The reference-side binding (mgxbench_b200/binding/mulmat_kernel_mgx.cpp) on the GPU.

build/mgx_binding_check declares MGXBench's three per-rank functions exactly as its drivers do
(1D-row-block/mmb.cu:162-164, 2D-block-matrix/mmb.cu:20-22) and calls them through the binding:
ABMultiply and the chunked ABMultiplyAccumulateAsync sequence of the 1D driver
(1D-row-block/mmb.cu:738-858) must give the library's own results bit for bit, inside the oracle's
summation-order bound, and validate_matrix_C must pass the reference's known-answer check."""
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gamma, rng_matrix
from gpu_util import bits, dev, host

pytestmark = pytest.mark.gpu

CHECK = ROOT / "build" / "mgx_binding_check"


@pytest.mark.parametrize("m,n,k,kc", [(200, 300, 1000, 256), (513, 129, 777, 100)])
def test_binding_forwards_to_the_library(mgx, oracle, tmp_path, m, n, k, kc):
    import torch
    assert CHECK.exists(), "build/mgx_binding_check not built (python -c 'import __graft_entry__ as g; g.build()')"
    rng = np.random.default_rng(m + n + k)
    A, B = rng_matrix(rng, (m, k)), rng_matrix(rng, (k, n))
    A.tofile(tmp_path / "A.bin")
    B.tofile(tmp_path / "B.bin")
    out = subprocess.run([str(CHECK), str(m), str(n), str(k), str(kc), str(tmp_path)], capture_output=True,
                         text=True, timeout=300)
    assert out.returncode == 0, out.stdout + out.stderr
    assert "binding_check validate=1" in out.stdout
    assert "NUMERICAL VALIDATION" in out.stdout
    c_sync = np.fromfile(tmp_path / "C_sync.bin", dtype=np.float64).reshape(m, n)
    c_chunk = np.fromfile(tmp_path / "C_chunk.bin", dtype=np.float64).reshape(m, n)

    # the same calls made directly on the library
    dA, dB = dev(A), dev(B)
    dC = torch.empty((m, n), dtype=torch.float64, device="cuda")
    mgx.ab_multiply(dA, dB, dC)
    assert np.array_equal(bits(c_sync), bits(host(dC)))
    dC.zero_()
    for off in range(0, k, kc):
        ln = min(kc, k - off)
        mgx.ab_multiply_accumulate_async(dA, dB[off:off + ln], dC, m, n, k, off, ln, k, n, n)
    assert np.array_equal(bits(c_chunk), bits(host(dC)))

    # and the oracle's reference arithmetic, within the summation-order bound
    ab = np.abs(A) @ np.abs(B)
    assert np.all(np.abs(c_sync - oracle.ab_multiply(A, B)) <= 2 * gamma(k) * ab)
    ref = np.zeros((m, n))
    for off in range(0, k, kc):
        ln = min(kc, k - off)
        ref = oracle.ab_multiply_accumulate(A, B[off:off + ln], ref, off, ln)
    assert np.all(np.abs(c_chunk - ref) <= 2 * gamma(k) * ab + 2 * gamma(k) * np.abs(ref))
