import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle.oracle import Oracle
    return Oracle("port")


@pytest.fixture(scope="session")
def ref_oracle():
    from oracle.oracle import Oracle, ref_available
    if not ref_available():
        pytest.skip("reference kernels (oracle/_ref) not built")
    return Oracle("ref")


@pytest.fixture(scope="session")
def gpu():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    import matops_b200
    return matops_b200


@pytest.fixture
def rng():
    return np.random.default_rng(12345)
