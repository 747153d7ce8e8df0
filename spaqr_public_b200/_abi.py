"""ctypes binding of the spaQR-B200 C ABI (include/spaqr_b200.h).

The shared library is built in-tree (``spaqr_public_b200/_build/libspaqr_b200.so``)
by ``spaqr_public_b200.build.build()``. Loading fails loudly when it is missing:
there is no CPU fallback for the numerical path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libspaqr_b200.so")

SPQ_OK = 0
SPQ_FP64 = 0
SPQ_FP32 = 1
STATUS = {
    0: "SPQ_OK", 1: "SPQ_ERR_ARG", 2: "SPQ_ERR_STATE", 3: "SPQ_ERR_CUDA", 4: "SPQ_ERR_NUMERIC",
    5: "SPQ_ERR_ALLOC", 6: "SPQ_ERR_UNSUPPORTED", 7: "SPQ_ERR_NOCONV",
}

# Every symbol include/spaqr_b200.h declares, with its ctypes signature.
_i = C.c_int
_d = C.c_double
_p = C.c_void_p
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)
_llp = C.POINTER(C.c_longlong)
SIGNATURES = {
    "spq_last_error": (C.c_char_p, []),
    "spq_version": (_i, []),
    "spq_device_count": (_i, [_ip]),
    "spq_create": (_i, [C.POINTER(_p), _i, _i]),
    "spq_destroy": (_i, [_p]),
    "spq_set_tol": (_i, [_p, _d]),
    "spq_set_scale": (_i, [_p, _i]),
    "spq_set_order": (_i, [_p, C.c_float]),
    "spq_set_hsl": (_i, [_p, _i]),
    "spq_set_square": (_i, [_p, _i]),
    "spq_set_coords": (_i, [_p, _i, _i, _dp]),
    "spq_set_coords_grid": (_i, [_p, _i, _i]),
    "spq_set_parts": (_i, [_p, _i, _ip]),
    "spq_set_fill_rule": (_i, [_p, _i]),
    "spq_graph_parts": (_i, [_i, _i, _ip, _ip, _i, _ip]),
    "spq_set_precision": (_i, [_p, _i]),
    "spq_set_device": (_i, [_p, _i]),
    "spq_set_verbose": (_i, [_p, _i]),
    "spq_partition": (_i, [_p, _i, _i, _ip, _ip, _dp]),
    "spq_assemble": (_i, [_p, _i, _i, _ip, _ip, _dp]),
    "spq_factorize": (_i, [_p]),
    "spq_factorize_batch": (_i, [C.POINTER(_p), _i, _i]),
    "spq_solve": (_i, [_p, _dp, _dp]),
    "spq_solve_nrml": (_i, [_p, _dp, _dp]),
    "spq_solve_dev": (_i, [_p, _p, _p]),
    "spq_solve_nrml_dev": (_i, [_p, _p, _p]),
    "spq_gmres": (_i, [_p, _i, _i, _ip, _ip, _dp, _dp, _dp, _i, _i, _d, _ip, _dp]),
    "spq_cgls": (_i, [_p, _i, _i, _ip, _ip, _dp, _dp, _dp, _i, _d, _ip, _dp]),
    "spq_cgls_dev": (_i, [_p, _i, _i, _p, _p, _p, _p, _p, _p, _p, _p, _i, _d, _ip, _dp]),
    "spq_get_perm": (_i, [_p, _ip, _ip]),
    "spq_log_size": (_i, [_p, _llp]),
    "spq_get_log": (_i, [_p, _llp]),
    "spq_num_bottom": (_i, [_p, _ip]),
    "spq_get_bottom": (_i, [_p, _ip]),
    "spq_get_stats": (_i, [_p, _dp, _llp]),
    "spq_get_level_times": (_i, [_p, _dp]),
    "spq_get_host_times": (_i, [_p, _dp]),
    "spq_trim_memory": (_i, []),
    "spq_pool_memory": (_i, [_i, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
    "spq_autotune_set_mode": (_i, [_i]),
    "spq_autotune_get": (_i, [_ip, _ip, _ip]),
    "spq_autotune_reset": (_i, []),
    "spq_autotune_save": (_i, [C.c_char_p]),
    "spq_autotune_load": (_i, [C.c_char_p]),
    "spq_column_normalize": (_i, [_i, _i, _ip, _ip, _dp]),
    "spq_solve_to_residual": (_i, [_p, _i, _i, _ip, _ip, _dp, _dp, _dp, _d, _d, _i, _i, _ip, _dp]),
    "spq_solve_to_residual_dev": (_i, [_p, _i, _p, _p, _p, _p, _p, _d, _d, _i, _i, _ip, _dp]),
    "spq_gmres_dev": (_i, [_p, _i, _p, _p, _p, _p, _p, _i, _i, _d, _ip, _dp]),
    "spq_gmres_dev_noalloc": (_i, [_p, _i, _p, _p, _p, _p, _p, _i, _i, _d, _ip, _dp]),
    "spq_solve_adjoint": (_i, [_p, _dp, _dp]),
    "spq_solve_adjoint_dev": (_i, [_p, _p, _p]),
    "spq_gmres_adjoint": (_i, [_p, _i, _i, _ip, _ip, _dp, _dp, _dp, _i, _i, _d, _ip, _dp]),
    "spq_gmres_adjoint_dev": (_i, [_p, _i, _p, _p, _p, _p, _p, _i, _i, _d, _ip, _dp]),
    "spq_solve_to_residual_adjoint_dev": (_i, [_p, _i, _p, _p, _p, _p, _p, _d, _d, _i, _i, _ip, _dp]),
    "spq_get_launches": (_i, [_p, _llp, _llp, _llp, _llp]),
    "spq_set_profile": (_i, [_p, _i]),
    "spq_get_kernel_stats": (_i, [_p, _i, _dp]),
    "spq_reset_kernel_stats": (_i, [_p]),
    "spq_get_stream": (_i, [_p, C.POINTER(_p)]),
    "spq_profile_solve_waves": (_i, [_p, _dp, _i, _ip]),
}

KERNEL_FAMILIES = ["copy", "panel_qr", "trailing_update", "trsm", "rrqr", "spars_writeback", "assemble_scatter",
                   "precond_apply"]
KERNEL_NAMES = {  # device function names as they appear in ncu launch lists
    "copy": "k_copy", "panel_qr": "k_panel", "trailing_update": "k_trailing", "trsm": "k_trsm", "rrqr": "k_rrqr",
    "spars_writeback": "k_spars_wb", "assemble_scatter": "k_scatter_values", "precond_apply": "k_solve_step",
}

_lib = None


class SpqError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads the in-tree shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"spaQR-B200 library not built ({LIB_PATH}); run spaqr_public_b200.build.build()")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc):
    if rc != SPQ_OK:
        raise SpqError(rc, lib().spq_last_error().decode())


def iptr(a):
    return a.ctypes.data_as(_ip)


def dptr(a):
    return a.ctypes.data_as(_dp)
