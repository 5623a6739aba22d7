import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libindexgen_cuda.so")
    config.addinivalue_line("markers", "slow: takes more than ~20 s on the CPU")


def load_golden(name):
    return np.load(os.path.join(GOLDEN, name))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def igctx():
    """A library context on cuda:0 (GPU tests only)."""
    from indexgen_b200 import Context

    ctx = Context(0)
    yield ctx
    ctx.close()
