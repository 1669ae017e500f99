import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libpcgpu.so")


@pytest.fixture(scope="session")
def golden():
    from tests.oracle_lib import load_golden
    return load_golden()


@pytest.fixture(scope="session")
def oracle():
    from tests.oracle_lib import Oracle
    return Oracle()


@pytest.fixture(scope="session")
def gpu_ctx():
    import potreeconverter_b200 as pc
    ctx = pc.Context()
    yield ctx
    ctx.close()
