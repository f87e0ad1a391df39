"""ctypes declarations of the C ABI in include/spmv_b200.h (libspmv_b200.so)."""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char, c_char_p, c_double, c_float, c_int, c_int32, c_int64, c_uint32, c_void_p

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "lib", "libspmv_b200.so")

NOALLOC_MAX_ELEMS = 262144   # SPMV_NOALLOC_MAX_ELEMS

# status codes
SPMV_OK = 0
SPMV_ERR_ARG = 1
SPMV_ERR_CSR = 2
SPMV_ERR_CUDA = 3
SPMV_ERR_NOMEM = 4
SPMV_ERR_UNSUPPORTED = 5
SPMV_ERR_TIMEOUT = 6
SPMV_ERR_BOUNDS = 7
SPMV_ERR_NO_DEVICE = 8
SPMV_ERR_OVERFLOW = 9

# formats (one per reference executable)
FORMATS = {
    "csr_naive": 0,
    "csr_vec": 1,
    "sell": 2,
    "sell_sorted": 3,
    "sell_c_s": 4,
    "div_rf": 5,
}

VALUES_F64 = 0
VALUES_F32 = 1

# exportable arrays: name -> (id, numpy dtype)
ARRAYS = {
    "row_ptr": (0, "int32"), "col_ind": (1, "int32"), "values": (2, "float64"),
    "row_cluster_ptr": (10, "int32"), "ja": (11, "int32"), "a": (12, "float64"),
    "permutation": (13, "int32"), "rev_permutation": (14, "int32"), "ranges": (15, "int64"),
    "row_order": (20, "int32"), "slice_widths": (21, "int32"), "slice_pointers": (22, "int64"),
    "column_indices": (23, "int32"), "sellcs_values": (24, "float64"),
    "div_data": (30, "uint8"), "div_packets": (31, "int64"), "div_groups": (32, "int64"),
    "div_thread_bytes": (33, "int64"), "div_thread_groups": (34, "int64"),
}


class FormatDesc(ctypes.Structure):
    _fields_ = [
        ("format", c_int32), ("num_threads", c_int32), ("vec_len", c_int32), ("sellcs_c", c_int32),
        ("sellcs_sigma", c_int32), ("div_packet_vals", c_int32), ("div_tolerance", c_double),
        ("exact", c_int32), ("values", c_int32), ("block_nnz", c_int32), ("block_rows", c_int32),
        ("stages", c_int32), ("ctas_per_sm", c_int32), ("kernel", c_int32), ("threads", c_int32),
        ("wait_limit_us", c_int32), ("debug_flags", c_int32), ("div_packet_reordering", c_int32),
        ("pack_cols", c_int32), ("row_assign", c_int32), ("reserved", c_int32),
    ]


class Info(ctypes.Structure):
    _fields_ = [
        ("m", c_int64), ("n", c_int64), ("nnz", c_int64), ("mem_footprint", c_double),
        ("csr_mem_footprint", c_double), ("stored_elems", c_int64), ("device_bytes", c_int64),
        ("convert_ms", c_double), ("kernels_per_run", c_int32), ("format", c_int32),
        ("format_name", c_char * 64), ("alloc_ms", c_double), ("copy_in_ms", c_double),
        ("x_lo", c_int64), ("x_hi", c_int64), ("x_col0", c_int64),
    ]


# every exported entry point of include/spmv_b200.h: name -> (restype, argtypes)
SIGNATURES = {
    "spmv_format_desc_init": (None, [POINTER(FormatDesc), c_int32]),
    "spmv_create": (c_void_p, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_int64, c_int64,
                               POINTER(FormatDesc), POINTER(c_int)]),
    "spmv_create_device": (c_void_p, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64,
                                      POINTER(FormatDesc), c_void_p, POINTER(c_int)]),
    "spmv_run": (c_int, [c_void_p, c_void_p, c_void_p]),
    "spmv_run_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_run_device_f32": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_run_f32": (c_int, [c_void_p, c_void_p, c_void_p]),
    "spmv_run_device_mixed_noalloc": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_features": (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_int64, c_void_p]),
    "spmv_features_device": (c_int, [c_void_p, c_void_p, c_int64, c_int64, c_int64, c_void_p, c_void_p]),
    "spmv_mlp_create": (c_void_p, [c_int32, c_int32, c_int32, c_int32, c_void_p, POINTER(c_int)]),
    "spmv_mlp_num_params": (c_int32, [c_void_p]),
    "spmv_mlp_get": (c_int, [c_void_p, c_int32, c_void_p]),
    "spmv_mlp_set": (c_int, [c_void_p, c_void_p]),
    "spmv_mlp_forward": (c_int, [c_void_p, c_void_p, c_int32, c_void_p, c_void_p]),
    "spmv_mlp_forward_host": (c_int, [c_void_p, c_void_p, c_int32, c_void_p]),
    "spmv_mlp_loss_grad": (c_int, [c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p]),
    "spmv_mlp_adam_step": (c_int, [c_void_p, c_float, c_float, c_float, c_float, c_float, c_void_p]),
    "spmv_mlp_destroy": (None, [c_void_p]),
    "spmv_sync": (c_int, [c_void_p]),
    "spmv_get_info": (c_int, [c_void_p, POINTER(Info)]),
    "spmv_export": (c_int, [c_void_p, c_int32, c_void_p, POINTER(c_int64)]),
    "spmv_destroy": (None, [c_void_p]),
    "spmv_last_error": (c_char_p, []),
    "spmv_statistics_print_labels": (c_int, [c_char_p, c_int64]),
    "spmv_statistics_print_data": (c_int, [c_void_p, c_char_p, c_int64]),
    "spmv_artgen_create": (c_void_p, [c_int64, c_int64, c_double, c_double, c_char_p, c_char_p, c_double, c_double,
                                      c_double, c_double, c_uint32, c_int, POINTER(c_int)]),
    "spmv_artgen_nnz": (c_int64, [c_void_p]),
    "spmv_artgen_get": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_artgen_destroy": (None, [c_void_p]),
    "spmv_version": (c_char_p, []),
    "spmv_format_desc_size": (ctypes.c_size_t, []),
    "spmv_info_size": (ctypes.c_size_t, []),
    "spmv_batch_create": (c_void_p, [c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     POINTER(c_int)]),
    "spmv_batch_run_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_batch_run_graph": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_batch_sync": (c_int, [c_void_p]),
    "spmv_batch_info": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_batch_destroy": (None, [c_void_p]),
    "spmv_mtx_read": (c_void_p, [c_char_p, c_int32, POINTER(c_int)]),
    "spmv_mtx_info": (c_int, [c_void_p] + [c_void_p] * 7),
    "spmv_mtx_get": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_mtx_destroy": (None, [c_void_p]),
    "spmv_coo_to_csr_device": (c_int, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_void_p, c_void_p,
                                       c_void_p, c_void_p]),
    "spmv_expand_symmetric": (c_void_p, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, POINTER(c_int)]),
    "spmv_drop_upper": (c_void_p, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, POINTER(c_int)]),
    "spmv_rcm": (c_void_p, [c_void_p, c_void_p, c_void_p, c_int64, c_int64, c_int64, c_int32, POINTER(c_int)]),
    "spmv_csr_out_info": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_csr_out_get": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_csr_out_destroy": (None, [c_void_p]),
    "spmv_gen_create_device": (c_void_p, [c_int64, c_int64, c_double, c_double, c_char_p, c_char_p, c_double, c_double,
                                          c_double, c_double, c_uint32, c_void_p, POINTER(c_int)]),
    "spmv_gen_info": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_gen_copy_device": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "spmv_gen_destroy": (None, [c_void_p]),
    "spmv_gen_host_check": (c_int64, [c_int64, c_int64, c_double, c_double, c_char_p, c_char_p, c_double, c_double,
                                      c_double, c_double, c_uint32, c_void_p, c_void_p, c_void_p, c_int64]),
}

_lib = None


def load():
    """Load libspmv_b200.so (raises if it has not been built: there is no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"libspmv_b200.so is not built ({LIB_PATH}); run `python spmv-dare_b200/build.py`")
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        # the structs declared here must be the library's: a stale build would otherwise read
        # or write past them
        for name, st in (("spmv_format_desc_size", FormatDesc), ("spmv_info_size", Info)):
            if getattr(lib, name)() != ctypes.sizeof(st):
                raise RuntimeError(f"{LIB_PATH}: {name}() = {getattr(lib, name)()} but the binding's struct has "
                                   f"{ctypes.sizeof(st)} bytes: rebuild the library")
        _lib = lib
    return _lib
