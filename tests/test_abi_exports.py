"""The C-ABI libraries load without a GPU and export every function that
include/*.h declares (germaine_gpu.h: libgermaine_gpu.so, germaine_umfpack.h:
libgermaine_umfpack.so); the engine refuses to run without a device."""
import ctypes
import glob
import os
import re

import pytest

from germaine_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


HEADER_LIB = {"germaine_gpu.h": (_lib.load, _lib.LIB_PATH, _lib.EXPORTS),
              "germaine_umfpack.h": (_lib.load_umfpack, _lib.UMFPACK_LIB_PATH, _lib.UMFPACK_EXPORTS)}


def declared_functions(header=None):
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        if header is not None and os.path.basename(h) != header:
            continue
        text = re.sub(r"/\*.*?\*/", "", open(h).read(), flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(\w+)\s*\(", text, flags=re.M):
            name = m.group(1)
            if name not in ("if", "while", "for", "return", "sizeof"):
                names.add(name)
    return sorted(names)


def test_header_declares_something():
    names = declared_functions()
    assert "gm_factor" in names and "gm_solve" in names and "umfpack_zi_numeric" in names


def test_every_header_has_a_library():
    headers = {os.path.basename(h) for h in glob.glob(os.path.join(ROOT, "include", "*.h"))}
    assert headers == set(HEADER_LIB)


@pytest.mark.parametrize("header,name", [(h, n) for h in sorted(HEADER_LIB) for n in declared_functions(h)])
def test_symbol_exported(header, name):
    load, path, _ = HEADER_LIB[header]
    lib = load()
    assert hasattr(lib, name), f"{name} declared in include/{header} but not exported by {path}"


@pytest.mark.parametrize("header", sorted(HEADER_LIB))
def test_python_binding_lists_every_symbol(header):
    missing = set(declared_functions(header)) - set(HEADER_LIB[header][2])
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
