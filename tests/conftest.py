import os
import sys

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
for p in (HERE, REPO):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a); runs the product library")


@pytest.fixture(scope="session")
def cuda():
    """torch with a CUDA device; a gpu-marked test fails (does not skip) without one."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test needs a CUDA device")
    torch.cuda.init()
    return torch


@pytest.fixture(scope="session")
def qla(cuda):
    import qla_b200
    qla_b200.lib()
    qla_b200.clear_error()
    return qla_b200
