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


def test_build_targets_sm100a():
    # the build compiles every kernel for sm_100a only (no other architecture, no PTX for JIT)
    from spring_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


@pytest.mark.gpu
def test_kernels_are_sm100_binaries():
    # the runtime reports the binary architecture of the library's kernels (cudaFuncGetAttributes)
    lib = L.load()
    v = ct.c_int(0)
    assert lib.spring_binary_version(0, ct.byref(v)) == 0
    assert v.value == 100


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
