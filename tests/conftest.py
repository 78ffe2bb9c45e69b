"""pytest configuration: the `gpu` marker, repository paths and shared helpers."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

# MGXBench's own sources, for the tests that run its unmodified scripts or kernels.  They are not
# part of this repository; tests that need them skip, saying so, where the directory is absent.
REFERENCE = Path(os.environ.get("MGXBENCH_REFERENCE", "/root/reference"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    # Keep the no-allocation entry point's test last so an early stop has already run the rest.
    items.sort(key=lambda it: 1 if "test_zz_" in it.nodeid else 0)


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.lib()
    return O


@pytest.fixture(scope="session")
def mgx():
    import mgxbench_b200 as m
    m.lib()
    return m


def gamma(k: int) -> float:
    """gamma_k = k u / (1 - k u): componentwise bound of any FP64 summation order of k products."""
    u = 2.0 ** -53
    return k * u / (1 - k * u)


def rng_matrix(rng, shape, kind="uniform", e_range=20):
    x = rng.uniform(-1.0, 1.0, shape)
    if kind == "wide":
        x = x * np.exp2(rng.integers(-e_range, e_range + 1, shape))
    return x
