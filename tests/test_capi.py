"""The C-ABI library loads and exports every entry point include/litho_gpu.h
declares; calls that need no device behave (no compute calls here)."""
import ctypes as C
import os
import re

import pytest

from lithoinv3d_b200 import _native, library_path

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(lf_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_builds_and_loads():
    lib = _native.load()
    assert os.path.exists(library_path())
    assert lib is not None


def test_every_declared_symbol_is_exported():
    lib = C.CDLL(library_path())
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(_native.SIGNATURES) <= declared_symbols()


def test_no_device_create_fails_cleanly():
    lib = _native.load()
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a device is present")
    except ImportError:
        pass
    h = C.c_void_p()
    st = lib.lf_create(C.byref(h), 0)
    assert st == 2  # LF_ECUDA: there is no CPU fallback
    assert not h.value


def test_null_arguments_rejected():
    lib = _native.load()
    assert lib.lf_create(None, 0) == 1
    assert lib.lf_model_create(None) == 1
    assert lib.lf_forward(None, None, None, None) == 1
    assert lib.lf_objective_grad(None, None, None, None) == 1
    assert lib.lf_set_precision(None, 0) == 1
