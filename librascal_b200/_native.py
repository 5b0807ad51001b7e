"""ctypes binding of the C ABI in include/rascal_b200.h.

The shared library is built in-tree (``python -m librascal_b200.build``) and
loaded from ``librascal_b200/_lib``. There is no fallback: every call of the
package goes through this library, and a missing or unloadable library is an
error.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "librascal_b200.so")

RGPU_OK = 0
PRECISION_FP64 = 0
PRECISION_FP32 = 1
ERR_INVALID_ARGUMENT = 1  # RGPU_ERR_INVALID_ARGUMENT
ERR_CAPACITY = 3  # RGPU_ERR_CAPACITY
ERR_TIMEOUT = 4  # RGPU_ERR_TIMEOUT
ERR_NOT_COMPUTED = 7  # RGPU_ERR_NOT_COMPUTED

_EXC_OVERFLOW = 3

c_int_p = ctypes.POINTER(ctypes.c_int32)
c_i64_p = ctypes.POINTER(ctypes.c_int64)
c_dbl_p = ctypes.POINTER(ctypes.c_double)
c_u8_p = ctypes.POINTER(ctypes.c_uint8)
c_void_pp = ctypes.POINTER(ctypes.c_void_p)

# name -> (restype, argtypes)
SIGNATURES = {
    "rgpu_last_error": (ctypes.c_char_p, []),
    "rgpu_error_kind": (ctypes.c_int, []),
    "rgpu_version": (ctypes.c_int, []),
    "rgpu_calculator_create": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_char_p, c_void_pp]),
    "rgpu_calculator_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rgpu_calculator_name": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "rgpu_calculator_spline_shape": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    "rgpu_calculator_spline_table": (ctypes.c_int, [ctypes.c_void_p, c_dbl_p, c_dbl_p, c_dbl_p]),
    "rgpu_structures_create": (ctypes.c_int, [c_void_pp]),
    "rgpu_structures_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rgpu_structures_set": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_i64_p, c_dbl_p, c_int_p,
                                           c_dbl_p, c_int_p, c_u8_p]),
    "rgpu_structures_update_positions": (ctypes.c_int, [ctypes.c_void_p, c_dbl_p]),
    "rgpu_structures_invalidate": (ctypes.c_int, [ctypes.c_void_p]),
    "rgpu_structures_stream": (ctypes.c_int, [ctypes.c_void_p, c_void_pp]),
    "rgpu_neighbour_list_build": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double]),
    "rgpu_neighbour_list_size": (ctypes.c_int, [ctypes.c_void_p, c_i64_p, c_i64_p]),
    "rgpu_neighbour_list_get": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_i64_p, c_int_p, c_int_p,
                                               c_dbl_p, c_dbl_p]),
    "rgpu_compute": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    "rgpu_get_species": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_int_p]),
    "rgpu_get_feature_keys": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_int_p, c_int_p]),
    "rgpu_get_features": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, c_int_p,
                                         c_dbl_p]),
    "rgpu_get_features_gradient": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                                  c_int_p, c_dbl_p]),
    "rgpu_gap_model_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_int_p, ctypes.c_int32,
                                             c_int_p, c_dbl_p, c_dbl_p, ctypes.c_int32, c_dbl_p,
                                             c_void_pp]),
    "rgpu_gap_model_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "rgpu_gap_predict": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, c_dbl_p,
                                        c_dbl_p]),
    "rgpu_gap_predict_stress": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, c_dbl_p,
                                               c_dbl_p, c_dbl_p]),
    "rgpu_gap_forward_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rgpu_gap_backward_dev": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rgpu_md_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, c_dbl_p, c_dbl_p, c_dbl_p, c_dbl_p]),
    "rgpu_md_step_info": (ctypes.c_int, [ctypes.c_void_p, c_int_p, c_i64_p]),
    "rgpu_sparse_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, c_dbl_p]),
    "rgpu_sparse_kernel_derivative": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, c_dbl_p]),
    "rgpu_sparse_kernel_mm": (ctypes.c_int, [ctypes.c_void_p, c_dbl_p]),
    "rgpu_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "rgpu_kernel_launches": (ctypes.c_int64, [ctypes.c_int]),
    "rgpu_stage_times": (ctypes.c_int, [ctypes.c_void_p, c_dbl_p, ctypes.c_int32]),
    "rgpu_measure_fma_peak": (ctypes.c_int, [ctypes.c_int, c_dbl_p]),
    "rgpu_set_tile_config": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int_p,
                                            ctypes.c_int32]),
    "rgpu_get_tile_config": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int_p]),
    "rgpu_structures_use_graphs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "rgpu_structures_graph_info": (ctypes.c_int, [ctypes.c_void_p, c_i64_p]),
    "rgpu_debug_gemm_bf16x3": (ctypes.c_int, [ctypes.c_int, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                              ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "rgpu_debug_set_gemm_wait_limit": (ctypes.c_int, [ctypes.c_int64]),
    "rgpu_debug_packed_layout": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_i64_p, c_i64_p,
                                                c_dbl_p, c_dbl_p, c_dbl_p]),
    "rgpu_gap_energies_noalloc": (ctypes.c_int, [ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                                 ctypes.c_void_p, ctypes.c_void_p]),
}

_lib = None


def lib():
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                "librascal_b200 native library not found at %s; build it with "
                "`python -m librascal_b200.build`" % LIB_PATH)
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        # launch shapes chosen by the autotuner (tuned_tiles.json)
        from . import tune
        tune.install_table(L)
        _lib = L
    return _lib


def check(status):
    """Raise the Python exception the reference's bindings would raise."""
    if status == RGPU_OK:
        return
    L = lib()
    msg = L.rgpu_last_error().decode(errors="replace")
    if L.rgpu_error_kind() == _EXC_OVERFLOW:
        raise OverflowError(msg)
    raise RuntimeError(msg)


def ptr(a, t):
    if a is None:
        return None
    return a.ctypes.data_as(t)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def i64(a):
    return np.ascontiguousarray(a, dtype=np.int64)
