"""goav1_b200 - the AV1 post-reconstruction filter chain of goav1 on NVIDIA B200.

The product is libgoav1pf.so (hand-written sm_100a CUDA behind the C ABI in
include/goav1pf.h).  This package loads it and mirrors goav1's post-filter
runner interface for Python callers (postfilter.PostFilterRunner).  There is
no CPU fallback: without the built library or a CUDA device every entry point
raises.
"""

import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libgoav1pf.so")
_lib = None


def lib():
    """The loaded C-ABI library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("goav1_b200: %s is missing; build it with `python -m goav1_b200.build`" % LIB_PATH)
    L = C.CDLL(LIB_PATH)
    L.pf_abi_version.restype = C.c_int
    L.pf_status_string.argtypes = [C.c_int]
    L.pf_status_string.restype = C.c_char_p
    L.pf_status_detail.restype = C.c_char_p
    L.pf_create.argtypes = [C.POINTER(abi.pf_config), C.POINTER(C.c_int)]
    L.pf_create.restype = C.c_void_p
    L.pf_destroy.argtypes = [C.c_void_p]
    L.pf_destroy.restype = None
    L.pf_frame_apply.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame_side),
                                 C.POINTER(abi.pf_frame), C.POINTER(abi.pf_stats)]
    L.pf_frame_validate.argtypes = [C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame_side), C.POINTER(abi.pf_frame)]
    L.pf_sync.argtypes = [C.c_void_p]
    L.pf_stream.argtypes = [C.c_void_p]
    L.pf_stream.restype = C.c_void_p
    L.pf_batch_apply.argtypes = [C.c_void_p, C.POINTER(abi.pf_batch_item), C.c_int32, C.POINTER(abi.pf_stats)]
    L.pf_cdef_search.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame), C.c_void_p,
                                 C.POINTER(abi.pf_cdef_search_params), C.c_void_p, C.c_void_p,
                                 C.POINTER(abi.pf_cdef_search_result)]
    L.pf_film_grain_static.argtypes = [C.POINTER(abi.pf_frame), C.POINTER(abi.pf_film_grain),
                                       C.POINTER(abi.pf_frame), C.c_void_p]
    L.pf_cdef_features.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.c_void_p, C.c_int32, C.c_int32,
                                   C.c_void_p]
    L.pf_cdef_mlp_forward.argtypes = [C.c_void_p, C.POINTER(abi.pf_cdef_mlp), C.c_void_p, C.c_int32, C.c_void_p]
    L.pf_cdef_mlp_gradients.argtypes = [C.c_void_p, C.POINTER(abi.pf_cdef_mlp), C.c_void_p, C.c_void_p, C.c_int32,
                                        C.POINTER(C.c_float), C.POINTER(abi.pf_cdef_mlp_grads)]
    L.pf_cdef_mlp_train.argtypes = [C.c_void_p, C.POINTER(abi.pf_cdef_mlp), C.c_void_p, C.c_void_p, C.c_int32,
                                    C.POINTER(abi.pf_cdef_mlp_train_params), C.c_void_p]
    L.pf_cdef_search_learned.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame), C.c_void_p,
                                         C.POINTER(abi.pf_cdef_search_params), C.POINTER(abi.pf_cdef_mlp), C.c_float,
                                         C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                         C.POINTER(abi.pf_cdef_search_result),
                                         C.POINTER(abi.pf_cdef_learned_stats)]
    L.pf_batch_graphs.argtypes = [C.c_void_p, C.c_int32]
    L.pf_set_persistent.argtypes = [C.c_void_p, C.c_int32, C.c_int32]
    L.pf_set_schedule.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.pf_schedule)]
    L.pf_get_schedule.argtypes = [C.c_void_p, C.c_int32, C.POINTER(abi.pf_schedule)]
    L.pf_set_frame_groups.argtypes = [C.c_void_p, C.c_int32]
    L.pf_autotune.argtypes = [C.c_void_p, C.POINTER(abi.pf_batch_item), C.c_int32, C.c_int32,
                              C.POINTER(abi.pf_tune_result)]
    L.pf_cdef_apply.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.c_void_p, C.POINTER(abi.pf_cdef_search_params),
                                C.POINTER(abi.pf_cdef_search_result), C.c_void_p]
    L.pf_frame_apply_superres.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame_side),
                                          C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame), C.POINTER(abi.pf_stats)]
    L.pf_superres_upscale.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame)]
    L.pf_batch_apply_superres.argtypes = [C.c_void_p, C.POINTER(abi.pf_superres_item), C.c_int32,
                                          C.POINTER(abi.pf_stats)]
    L.pf_lf_build.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_uint32,
                              C.POINTER(abi.pf_lf_levels), C.c_int32, C.c_int32, C.c_int32, C.c_void_p,
                              C.c_void_p, C.c_uint32]
    L.pf_lr_search.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame),
                               C.POINTER(abi.pf_frame), C.c_void_p, C.c_int32]
    L.pf_diag_issue_rate.argtypes = [C.c_int32, C.POINTER(C.c_double), C.POINTER(C.c_double)]
    L.pf_cdef_search_level_rtc.argtypes = [C.c_int32, C.c_int32]
    L.pf_cdef_plan_picture.argtypes = [C.c_int32] * 4 + [C.POINTER(abi.pf_cdef_ref_strengths), C.c_int32,
                                                         C.POINTER(abi.pf_cdef_plan)]
    L.pf_cdef_search_ex.argtypes = [C.c_void_p, C.POINTER(abi.pf_frame), C.POINTER(abi.pf_frame), C.c_void_p,
                                    C.POINTER(abi.pf_cdef_search_params), C.POINTER(abi.pf_cdef_search_ctrls),
                                    C.c_void_p, C.c_void_p, C.POINTER(abi.pf_cdef_search_result)]
    if L.pf_abi_version() != 3:
        raise RuntimeError("goav1_b200: ABI version mismatch")
    _lib = L
    return L
