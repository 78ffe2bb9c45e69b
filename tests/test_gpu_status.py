"""Failure detection without a GPU fault: every device-side wait in the library is bounded, and
a wait that runs out records a code in the device status word instead of hanging.  Here a
kernel waits on a barrier that nothing completes (mgx_wait_probe); the status word reports the
timeout, reading it clears it, and the context keeps working."""
import time

import numpy as np
import pytest

from conftest import rng_matrix
from gpu_util import dev, host

pytestmark = pytest.mark.gpu


def test_bounded_wait_reports_timeout_and_context_survives(mgx, oracle):
    import torch
    assert mgx.device_status() == 0
    t0 = time.perf_counter()
    assert mgx.lib().mgx_wait_probe(50000) == 0          # gives up after 50 ms
    dt = time.perf_counter() - t0
    assert 0.04 <= dt < 5.0
    assert mgx.device_status() == 1                        # full-stage wait ran out
    assert mgx.device_status() == 0                        # reading clears it
    assert mgx.lib().mgx_wait_probe(0) == -1               # limits outside 1 us .. 2 s are refused
    rng = np.random.default_rng(4)
    A, B = rng_matrix(rng, (64, 96), "wide"), rng_matrix(rng, (96, 80), "wide")
    dC = torch.empty((64, 80), dtype=torch.float64, device="cuda")
    mgx.gemm_ozaki(dev(A), dev(B), dC, splits=8)
    assert np.array_equal(host(dC).view(np.uint64), oracle.ozaki_gemm(A, B, 8).view(np.uint64))
    assert mgx.device_status() == 0
