"""The C-ABI library loads without a GPU and exports every function that
include/*.h declares; the engine refuses to run without a device."""
import ctypes
import glob
import os
import re

import pytest

from germaine_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_header_declares_something():
    names = declared_functions()
    assert "gm_factor" in names and "gm_solve" in names


@pytest.mark.parametrize("name", declared_functions())
def test_symbol_exported(name):
    lib = _lib.load()
    assert hasattr(lib, name), f"{name} declared in include/ but not exported by {_lib.LIB_PATH}"


def test_python_binding_lists_every_symbol():
    missing = set(declared_functions()) - set(_lib.EXPORTS)
    assert not missing, f"declared but not bound in germaine_b200/_lib.py: {sorted(missing)}" 


def test_no_device_no_cpu_path():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    cfg = _lib.GmConfig(20, 20, 10.0, 2, 0, 90.0, 0.0, 1, 0, 0, 16, 1e-10, 5)
    h = ctypes.c_void_p()
    rc = lib.gm_engine_create(0, ctypes.byref(cfg), ctypes.byref(h))
    assert rc == _lib.GM_ERROR_CUDA
    assert b"no CUDA device" in lib.gm_last_error()
