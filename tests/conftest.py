import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libmufflon_core.so")


@pytest.fixture(scope="session")
def oracle():
    from oracle import pyoracle
    pyoracle.lib()
    return pyoracle


@pytest.fixture(scope="session")
def core_lib_path():
    from mufflon_b200 import build
    return build.build()


@pytest.fixture(scope="session")
def dll(core_lib_path):
    from mufflon_b200 import bindings
    d = bindings.DllInterface(core_lib_path)
    yield d
    d.close()
