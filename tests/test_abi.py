"""The C-ABI library loads and exports every entry point include/*.h declares
(no compute: these run without a GPU)."""
import ctypes
import glob
import os
import re

import pytest

from conftest import ROOT


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(dmst_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_builds_and_loads():
    from dummest_b200 import build, _ffi
    build.build()
    lib = _ffi.load()
    assert lib is not None


def test_every_declared_symbol_is_exported():
    from dummest_b200 import _ffi
    lib = ctypes.CDLL(_ffi.LIB_PATH)
    decl = declared_functions()
    assert len(decl) >= 20
    missing = [n for n in decl if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers them all
    assert sorted(decl) == sorted(_ffi.exported_symbols())


def test_status_strings():
    from dummest_b200 import _ffi
    lib = _ffi.load()
    for st in (0, -1, -2, -3, -4, -5, -6):
        assert lib.dmst_strerror(st)


def test_ctx_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from dummest_b200 import _ffi
    lib = _ffi.load()
    h = ctypes.c_void_p()
    st = lib.dmst_ctx_create(None, ctypes.byref(h))
    assert st == _ffi.DMST_EDEVICE and not h.value
