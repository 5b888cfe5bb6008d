import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def yq():
    """libyq_ops.so, built in-tree if missing."""
    from yallasql_b200 import _abi, build
    if not os.path.exists(_abi.LIB_PATH):
        build.build_ops()
    return _abi.load()


@pytest.fixture(scope="session")
def cuda(yq):
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU tests need CUDA; run them on a B200 (pytest -m gpu)")
    torch.cuda.init()
    return torch.device("cuda")


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle
