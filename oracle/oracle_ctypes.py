"""ctypes loader for the CPU oracle library (test infrastructure only).

Used by tests/ and by bench.py's cpu_baseline leg; the product never imports
it.  Builds oracle/_build/liboracle.so with make when it is missing.
"""

import ctypes as C
import os
import subprocess

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        _lib.oracle_frame_apply.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_loop_filter.argtypes = [C.c_void_p, C.c_void_p]
        _lib.oracle_cdef.argtypes = [C.c_void_p, C.c_void_p]
        _lib.oracle_cdef_find_dir.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int32)]
        _lib.oracle_cdef_filter_block.argtypes = [C.c_void_p, C.c_void_p] + [C.c_int] * 9
        _lib.oracle_cdef_filter_block.restype = None
        _lib.oracle_lpf_line.argtypes = [C.c_void_p] + [C.c_int] * 4
        _lib.oracle_lpf_line.restype = None
        _lib.oracle_lfsr_next.argtypes = [C.POINTER(C.c_uint16), C.c_int]
        _lib.oracle_lfsr_next.restype = C.c_uint16
        _lib.oracle_stripe_seed.argtypes = [C.c_uint16, C.c_int]
        _lib.oracle_stripe_seed.restype = C.c_uint16
        _lib.oracle_scaling_lut.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        _lib.oracle_scale_lut.argtypes = [C.c_void_p, C.c_int, C.c_int]
        _lib.oracle_luma_grain.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
        _lib.oracle_chroma_grain.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_int] * 4
        _lib.oracle_gaussian.argtypes = [C.c_int]
        _lib.oracle_gaussian.restype = C.c_int16
        _lib.oracle_sgr_decode_xq.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.oracle_sgr_decode_xq.restype = None
        _lib.oracle_wiener.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_int]
        _lib.oracle_wiener.restype = None
        _lib.oracle_sgr.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int,
                                    C.c_void_p, C.c_int]
        _lib.oracle_sgr.restype = None
        _lib.oracle_cdef_adjust_strength.argtypes = [C.c_int, C.c_int32]
        _lib.oracle_cdef_search.argtypes = [C.c_void_p] * 7
        _lib.oracle_cdef_select.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.oracle_cdef_select_ex.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p,
                                               C.c_void_p]
        _lib.oracle_cdef_features.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p]
        _lib.oracle_mlp_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
        _lib.oracle_mlp_forward.restype = None
        _lib.oracle_mlp_gradients.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_mlp_gradients.restype = None
        _lib.oracle_mlp_loss_grad_f64.argtypes = [C.c_void_p] * 5 + [C.c_int, C.c_void_p, C.c_void_p]
        _lib.oracle_mlp_loss_grad_f64.restype = None
        _lib.oracle_lr_search.argtypes = [C.c_void_p] * 4 + [C.c_int]
        _lib.oracle_superres_row.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int]
        _lib.oracle_superres_row.restype = None
        _lib.oracle_superres_upscale.argtypes = [C.c_void_p, C.c_void_p]
        _lib.oracle_frame_apply_superres.argtypes = [C.c_void_p] * 4
        _lib.oracle_lf_build.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                         C.c_void_p, C.c_void_p]
        _lib.oracle_lf_build_ordered.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p] + [C.c_int] * 5 + [
            C.c_void_p]
        _lib.oracle_lf_mask_block.argtypes = [C.c_int, C.c_void_p] + [C.c_int] * 6 + [C.c_void_p] * 3 + [C.c_int] * 2
        _lib.oracle_lf_mask_block.restype = None
        _lib.oracle_lf_block_levels.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    return _lib


def frame_apply(frame_pf, side, display_pf=None):
    """Runs the whole chain on a host pf_frame (in place)."""
    return lib().oracle_frame_apply(C.byref(frame_pf), C.byref(side),
                                    C.byref(display_pf) if display_pf is not None else None)
