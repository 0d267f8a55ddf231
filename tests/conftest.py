import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "dspsr-kanyixia_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def b2():
    import dspsr_b200
    dspsr_b200._capi.lib()
    return dspsr_b200


@pytest.fixture(scope="session")
def ctx(b2):
    import torch
    assert torch.cuda.is_available(), "the gpu tests need a CUDA device"
    torch.cuda.init()
    c = b2.Context(0, None)
    yield c
    c.close()
