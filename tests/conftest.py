import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def O():
    from tests.oracle import oracle
    return oracle()


@pytest.fixture(scope="session")
def R():
    from tests.oracle import reference
    r = reference()
    if r is None:
        pytest.skip("reference engine not built (oracle/_ref needs the reference sources)")
    return r


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    from pentago_b200 import capi
    capi.check(capi.lib().pg_init())
    return torch.device("cuda:0")
