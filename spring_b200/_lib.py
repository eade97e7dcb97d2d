"""ctypes binding of libspring_b200.so (the C ABI declared in include/spring_gpu.h).

There is no fallback: if the library is missing or cannot be loaded, importing
the bindings raises.  Build it with ``python -m spring_b200.build``.
"""
from __future__ import annotations

import ctypes as ct
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libspring_b200.so")

SPRING_OK = 0
SPRING_ERR_ARG = 1
SPRING_ERR_STATE = 2
SPRING_ERR_CUDA = 3
SPRING_ERR_ALLOC = 4
SPRING_ERR_UNSUPPORTED = 5
SPRING_ERR_INJECTED = 6
SPRING_ERR_TIMEOUT = 7
SPRING_OPT_GENERIC_V3 = 1
SPRING_OPT_WAIT_POLLS = 2
SPRING_OPT_FP64_PRESCREEN = 3
SPRING_DELTA_GAUSS = 0
SPRING_DELTA_TETRA = 1
SPRING_FP64 = 0
SPRING_BF16 = 1
SPRING_BF16X3 = 2
SPRING_MLP_INPUTS = 5
SPRING_MLP_PARAMS = 33921


class spring_dims(ct.Structure):
    _fields_ = [("nbasis", ct.c_int), ("mesh", ct.c_int * 3), ("n_temps", ct.c_int), ("device", ct.c_int)]


P = ct.c_void_p
I = ct.c_int
D = ct.c_double

# name -> argtypes (every function returns int unless listed in _RESTYPE)
SIGNATURES = {
    "spring_ctx_create": [ct.POINTER(P), ct.POINTER(spring_dims)],
    "spring_ctx_destroy": [P],
    "spring_last_error": [P],
    "spring_set_stream": [P, P],
    "spring_synchronize": [P],
    "spring_kernel_launches": [P, P],
    "spring_set_crystal": [P, P, P],
    "spring_set_fc2": [P, I, P, P, P],
    "spring_set_fc3": [P, I, P, P, P],
    "spring_set_fc4": [P, I, P, P, P],
    "spring_make_mesh": [P, P, I, P, P, P],
    "spring_find_irr_q": [P, I, P, I, P, P, P, P],
    "spring_compute_phonons": [P, P, D],
    "spring_set_phonons": [P, I, P, P, P, P, P, P],
    "spring_get_phonons": [P, I, P, P, P, P, P],
    "spring_enumerate3": [P, I, P, P, P],
    "spring_prepare3": [P],
    "spring_set_profiling": [P, I],
    "spring_set_option": [P, I, I],
    "spring_set_precision": [P, I],
    "spring_mlp_init": [P, ct.c_ulonglong],
    "spring_mlp_set_params": [P, P],
    "spring_mlp_get_params": [P, P],
    "spring_mlp_loss_grad": [P, I, P, P, P, P],
    "spring_mlp_train": [P, I, P, P, I, I, ct.c_float, ct.c_ulonglong, P],
    "spring_mlp_predict": [P, I, P, P, I],
    "spring_kappa_iter": [P, D, I, P, P, P],
    "spring_kappa_iter_gauss": [P, D, D, I, P, P, P, P],
    "spring_set_dipole": [P, P, P, P, I, D, D, P, P, P],
    "spring_get_dipole": [P, P, P, P, P, P],
    "spring_set_point_defect": [P, P, I, P, P, P, P, D, I, I],
    "spring_linewidth_pd": [P, I, I, P, I],
    "spring_kernel_time": [P, ct.c_char_p, P, P],
    "spring_tc_stats": [P, P, P],
    "spring_binary_version": [I, P],
    "spring_scatter_w3": [P, I, P],
    "spring_linewidth3": [P, I, I, I, D, P, P, P],
    "spring_linewidth_iso": [P, I, I, I, D, P, P],
    "spring_linewidth3_tetra_noalloc": [P, I, P, P, P],
    "spring_enumerate4": [P, I, P, P, ct.c_longlong, P],
    "spring_linewidth4": [P, I, I, I, D, P, P],
    "spring_linewidth4_modes": [P, I, I, D, P, P],
    "spring_path_qpoints": [P, I, P, P, P, P, P],
    "spring_linewidth_path": [P, I, P, P, I, D, P, P],
    "spring_reset_linewidths": [P],
    "spring_get_linewidths": [P, P],
    "spring_set_linewidths": [P, P],
    "spring_kappa_rta": [P, I, I, P, P, P, P],
    "spring_debug_inject_fault": [P, I, I],
    "spring_batch_create": [ct.POINTER(P)],
    "spring_batch_destroy": [P],
    "spring_batch_last_error": [P],
    "spring_batch_add_linewidth3": [P, P, I, I, D, P, P],
    "spring_batch_set_config": [P, P],
    "spring_batch_get_config": [P, P],
    "spring_batch_tune": [P, P, P, P],
    "spring_batch_run": [P],
    "spring_batch_result": [P, I, P, P, P],
    "spring_batch_add_path": [P, P, I, P, P, D, P],
    "spring_batch_path_result": [P, I, P, P],
}
_RESTYPE = {"spring_last_error": ct.c_char_p, "spring_batch_last_error": ct.c_char_p}

_lib = None


def load():
    """Load the library once; raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m spring_b200.build` "
                          "(there is no CPU fallback)")
    lib = ct.CDLL(LIB_PATH)
    for name, args in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = _RESTYPE.get(name, ct.c_int)
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return list(SIGNATURES)
