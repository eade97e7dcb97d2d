"""The C-ABI library loads and exports every entry point include/spring_gpu.h declares (CPU only)."""
import ctypes as ct
import os
import re

import pytest

from spring_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "spring_gpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(spring_[a-z0-9_]+)\s*\(", src)))


def test_header_and_binding_agree():
    assert sorted(L.exported_symbols()) == _declared()


def test_library_exports_every_symbol():
    lib = L.load()
    for name in _declared():
        assert hasattr(lib, name), name


def test_library_is_sm100a_build():
    # the fatbin of an sm_100a build names the architecture
    data = open(L.LIB_PATH, "rb").read()
    assert b"sm_100a" in data


def test_create_without_gpu_fails_cleanly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = L.load()
    d = L.spring_dims()
    d.nbasis = 2
    for k in range(3):
        d.mesh[k] = 4
    d.n_temps = 1
    d.device = -1
    h = ct.c_void_p()
    rc = lib.spring_ctx_create(ct.byref(h), ct.byref(d))
    assert rc != 0 and not h.value
    assert lib.spring_ctx_destroy(None) == L.SPRING_ERR_ARG
