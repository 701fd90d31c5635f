import os
import shutil
import sys
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def gpu_lib():
    """The product library on a machine with a GPU; fails (not skips) if the
    library is missing, because the GPU tests must exercise the native path."""
    from germaine_b200 import _lib
    lib = _lib.load()
    return lib


@pytest.fixture
def short_tmp():
    """A temporary directory with a short path: the reference formats file
    names into 74-byte buffers, which pytest's tmp_path can overflow."""
    d = tempfile.mkdtemp(prefix="gm", dir="/tmp")
    try:
        yield d
    finally:
        shutil.rmtree(d, ignore_errors=True)
