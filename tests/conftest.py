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


def build_c_example(core_lib_path, out_dir):
    """Compiles tests/cpp/load_and_render.c with gcc -std=c99 against include/
    and the in-tree libraries; returns the executable's path."""
    import subprocess
    lib_dir = os.path.dirname(core_lib_path)
    exe = os.path.join(out_dir, "load_and_render")
    subprocess.run(["gcc", "-std=c99", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "load_and_render.c"), "-o", exe, "-L", lib_dir,
                    "-lmufflon_loader", "-lmufflon_core", f"-Wl,-rpath,{lib_dir}"], check=True, capture_output=True)
    return exe
