"""ctypes binding of libsparseb.so (the C ABI declared in include/sparseb.h).

The shared library is built in-tree by ``sparsebackends_b200.build``.  There is
no fallback: if the library cannot be loaded, every call raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsparseb.so")

i64 = C.c_int64
u64 = C.c_uint64
vp = C.c_void_p
P_i64 = C.POINTER(i64)
P_u64 = C.POINTER(u64)
P_f64 = C.POINTER(C.c_double)
P_int = C.POINTER(C.c_int)

# name: (restype, argtypes) — mirrors include/sparseb.h
SIGNATURES = {
    "sb_ctx_create": (C.c_int, [C.c_int, C.c_uint, C.POINTER(vp)]),
    "sb_ctx_destroy": (C.c_int, [vp]),
    "sb_last_error": (C.c_char_p, [vp]),
    "sb_ctx_set_stream": (C.c_int, [vp, vp]),
    "sb_ctx_get_stream": (vp, [vp]),
    "sb_ctx_synchronize": (C.c_int, [vp]),
    "sb_ctx_launch_count": (i64, [vp]),
    "sb_ctx_set_precision": (C.c_int, [vp, C.c_int]),
    "sb_ctx_get_precision": (C.c_int, [vp]),
    "sb_ctx_set_profiling": (C.c_int, [vp, C.c_int]),
    "sb_ctx_profile_summary": (C.c_int, [vp, C.c_int, P_i64, P_f64, P_f64, P_f64]),
    "sb_tensor_create_dense": (C.c_int, [vp, C.c_int, P_i64, P_f64, C.POINTER(vp)]),
    "sb_tensor_create_dense_device": (C.c_int, [vp, C.c_int, P_i64, vp, C.POINTER(vp)]),
    "sb_tensor_create_bs": (C.c_int, [vp, C.c_int, P_i64, C.c_int, i64, P_i64, P_i64, P_f64, C.POINTER(vp)]),
    "sb_tensor_create_bs_ragged": (C.c_int, [vp, C.c_int, P_i64, C.c_int, i64, P_i64, P_i64, P_f64,
                                             C.POINTER(vp)]),
    "sb_tensor_block_dims": (C.c_int, [vp, P_int, P_i64, P_i64]),
    "sb_tensor_create_bs_f32": (C.c_int, [vp, C.c_int, P_i64, C.c_int, C.POINTER(vp)]),
    "sb_tensor_storage_f32": (C.c_int, [vp, P_int]),
    "sb_tensor_is_dense": (C.c_int, [vp, P_int]),
    "sb_tensor_to_uniform": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "sb_tensor_to_ragged": (C.c_int, [vp, vp, P_i64, C.c_int, C.POINTER(vp)]),
    "sb_tensor_crop_padding": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "sb_tensor_create_coo": (C.c_int, [vp, C.c_int, P_i64, i64, P_i64, P_f64, C.c_int, C.POINTER(vp)]),
    "sb_tensor_create_aliased": (C.c_int, [vp, C.c_int, P_i64, C.c_int, i64, P_f64, i64, P_i64, P_i64, P_f64,
                                           C.POINTER(vp)]),
    "sb_tensor_free": (C.c_int, [vp]),
    "sb_tensor_info": (C.c_int, [vp, P_int, P_int, P_i64, P_int, P_i64, P_i64, P_i64, P_int]),
    "sb_tensor_export_bs": (C.c_int, [vp, vp, P_i64, P_i64, P_f64]),
    "sb_tensor_export_bs_async": (C.c_int, [vp, vp, P_i64, P_i64, P_f64]),
    "sb_tensor_export_coo": (C.c_int, [vp, vp, P_i64, P_f64]),
    "sb_tensor_export_aliased": (C.c_int, [vp, vp, P_f64, P_i64, P_i64, P_f64]),
    "sb_tensor_export_dense": (C.c_int, [vp, vp, P_f64]),
    "sb_tensor_device_data": (C.c_int, [vp, C.POINTER(vp), P_i64]),
    "sb_contract": (C.c_int, [vp, vp, P_u64, C.c_int, vp, P_u64, C.c_int, vp, P_u64, C.c_int]),
    "sb_permutedims": (C.c_int, [vp, vp, P_int, C.POINTER(vp)]),
    "sb_coo_sort": (C.c_int, [vp, vp]),
    "sb_blocksparse_from_dense": (C.c_int, [vp, vp, C.c_int, C.c_double, C.c_double, C.c_int, C.POINTER(vp)]),
    "sb_coo_from_dense": (C.c_int, [vp, vp, C.c_double, C.c_double, C.POINTER(vp)]),
    "sb_to_dense": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "sb_aliased_to_blocksparse": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "sb_ctx_capture_begin": (C.c_int, [vp]),
    "sb_ctx_capture_end": (C.c_int, [vp, C.POINTER(vp)]),
    "sb_graph_launch": (C.c_int, [vp, vp]),
    "sb_graph_free": (C.c_int, [vp]),
    "sb_tensor_norm": (C.c_int, [vp, vp, P_f64]),
    "sb_tensor_dot": (C.c_int, [vp, vp, vp, P_f64]),
    "sb_tensor_copy": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "sb_tensor_similar": (C.c_int, [vp, vp, C.POINTER(vp)]),
    "sb_tensor_scale": (C.c_int, [vp, vp, C.c_double]),
    "sb_tensor_fill": (C.c_int, [vp, vp, C.c_double]),
    "sb_tensor_map": (C.c_int, [vp, vp, vp, C.c_int, C.c_double, C.c_double]),
    "sb_tensor_add": (C.c_int, [vp, vp, vp, C.POINTER(vp)]),
    "sb_fuse_axes": (C.c_int, [vp, vp, C.c_int, C.c_int, C.POINTER(vp)]),
    "sb_blocksparse_left_qr": (C.c_int, [vp, vp, C.POINTER(vp), C.POINTER(vp), P_i64, P_i64, P_i64, P_i64]),
    "sb_blocksparse_svd": (C.c_int, [vp, vp, C.c_int, i64, i64, C.c_double, C.POINTER(vp), C.POINTER(vp), P_f64,
                                     i64, P_i64, P_f64]),
    "sb_block_gemm_f64_noalloc": (C.c_int, [vp, vp, vp, vp, C.c_int32, P_i64, C.POINTER(C.c_int32),
                                            C.POINTER(C.c_int32), C.POINTER(C.c_int32), P_i64, P_i64,
                                            C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                                            C.c_int, C.c_int, C.c_char_p, C.c_int32]),
}

STATUS = {
    0: "SB_OK", 1: "SB_ERR_INVALID_ARG", 2: "SB_ERR_DIM_MISMATCH", 3: "SB_ERR_LABEL",
    4: "SB_ERR_UNSUPPORTED_LAYOUT", 5: "SB_ERR_UNSUPPORTED_TYPES", 6: "SB_ERR_OOM", 7: "SB_ERR_TIMEOUT",
    8: "SB_ERR_CUDA", 9: "SB_ERR_ASSERTION",
}

_lock = threading.Lock()
_lib = None


def load(path: str = LIB_PATH) -> C.CDLL:
    """Load and type the library (no GPU needed to load it)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise ImportError(
                f"libsparseb.so not found at {path}; build it with `python -m sparsebackends_b200.build`")
        lib = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib
