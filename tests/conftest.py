import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200)")


@pytest.fixture(scope="session")
def port():
    from oracle.oracle import Port

    return Port()


@pytest.fixture(scope="session")
def ref():
    from oracle.oracle import Ref

    if not Ref.available():
        pytest.skip("reference oracle library oracle/_ref not built")
    return Ref()


@pytest.fixture(scope="session")
def rng():
    return np.random.default_rng(12345)
