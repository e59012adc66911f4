import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU")


@pytest.fixture(scope="session")
def port():
    from oracle import oracle as orc
    if not orc.available("port"):
        orc.build()
    return orc.Oracle("port")


@pytest.fixture(scope="session")
def ref():
    from oracle import oracle as orc
    if not orc.available("reference"):
        pytest.skip("oracle/_ref not built (needs the reference tree)")
    return orc.Oracle("reference")


@pytest.fixture(scope="session")
def lib_path():
    from gpupdal_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def nbg(lib_path):
    from gpupdal_b200.native import Context
    return Context(0)
