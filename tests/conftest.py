"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
if GOLDEN not in sys.path:
    sys.path.insert(0, GOLDEN)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the sm_100a kernels")


@pytest.fixture(scope="session")
def oracle():
    from oracle import build as OB
    OB.build_oracle()
    from oracle import oracle as O
    return O


@pytest.fixture(scope="session")
def dmf():
    import dyn_maxflow_b200 as D
    return D


@pytest.fixture(scope="session")
def golden_dir():
    return GOLDEN
