"""ctypes mirror of include/goav1pf.h (the C ABI of the post-filter chain).

These Structure classes are the Python view of the boundary structs; field
order and types follow the header exactly.  They carry plain pointers and
sizes only, so the same layout is what a cgo binding passes from goav1's
FrameWorkPostFilterContext.
"""

import ctypes as C

PF_OK = 0
PF_ERR_INVALID_CDEF = -1
PF_ERR_INVALID_FILTER = -2
PF_ERR_INVALID_PLAN = -3
PF_ERR_UNSUPPORTED = -4
PF_ERR_SHORT_BUFFER = -5
PF_ERR_INVALID_FORMAT = -6
PF_ERR_INVALID_ARG = -7
PF_ERR_DEVICE = -8
PF_ERR_TIMEOUT = -9
PF_ERR_NO_DEVICE = -10
PF_ERR_INVALID_BATCH = -11

PF_STAGE_LOOP_FILTER = 1 << 0
PF_STAGE_CDEF = 1 << 1
PF_STAGE_LOOP_RESTORATION = 1 << 2
PF_STAGE_FILM_GRAIN = 1 << 3
PF_STAGE_EXTEND_BORDERS = 1 << 4
PF_STAGES_ALL = 0x1F

PF_MEM_HOST = 0
PF_MEM_DEVICE = 1

PF_LR_NONE = 0
PF_LR_SWITCHABLE = 1
PF_LR_WIENER = 2
PF_LR_SGRPROJ = 3

PF_LF_MASK_WORDS = 640


class pf_plane(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("stride", C.c_int64),
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("alloc_width", C.c_int32),
        ("alloc_height", C.c_int32),
    ]


class pf_frame(C.Structure):
    _fields_ = [
        ("width", C.c_int32),
        ("height", C.c_int32),
        ("bit_depth", C.c_uint8),
        ("ss_x", C.c_uint8),
        ("ss_y", C.c_uint8),
        ("mono", C.c_uint8),
        ("memory", C.c_uint8),
        ("reserved", C.c_uint8 * 3),
        ("plane", pf_plane * 3),
    ]


class pf_loop_filter(C.Structure):
    _fields_ = [
        ("level_y", C.c_uint8 * 2),
        ("level_u", C.c_uint8),
        ("level_v", C.c_uint8),
        ("sharpness", C.c_uint8),
        ("reserved", C.c_uint8 * 3),
        ("masks", C.c_void_p),
        ("sb128_w", C.c_int32),
        ("sb128_h", C.c_int32),
        ("level_cache", C.c_void_p),
        ("mi_cols", C.c_int32),
        ("mi_rows", C.c_int32),
    ]


class pf_cdef(C.Structure):
    _fields_ = [
        ("damping", C.c_uint8),
        ("bits", C.c_uint8),
        ("strength_count", C.c_uint8),
        ("reserved", C.c_uint8),
        ("y_strength", C.c_uint8 * 8),
        ("uv_strength", C.c_uint8 * 8),
        ("index", C.c_void_p),
        ("read", C.c_void_p),
        ("index_stride", C.c_int32),
        ("index_rows", C.c_int32),
        ("noskip", C.c_void_p),
    ]


class pf_lr_unit(C.Structure):
    _fields_ = [
        ("type", C.c_uint8),
        ("sgr_set", C.c_uint8),
        ("sgr_xqd", C.c_int8 * 2),
        ("wiener_v", C.c_int8 * 3),
        ("wiener_h", C.c_int8 * 3),
    ]


class pf_restoration(C.Structure):
    _fields_ = [
        ("type", C.c_uint8 * 3),
        ("reserved", C.c_uint8),
        ("unit_size_y", C.c_uint16),
        ("unit_size_uv", C.c_uint16),
        ("units", C.c_void_p * 3),
        ("unit_count", C.c_int32 * 3),
    ]


class pf_film_grain(C.Structure):
    _fields_ = [
        ("apply", C.c_uint8),
        ("chroma_scaling_from_luma", C.c_uint8),
        ("seed", C.c_uint16),
        ("num_y_points", C.c_uint8),
        ("y_points", (C.c_uint8 * 2) * 14),
        ("num_cb_points", C.c_uint8),
        ("cb_points", (C.c_uint8 * 2) * 10),
        ("num_cr_points", C.c_uint8),
        ("cr_points", (C.c_uint8 * 2) * 10),
        ("scaling_shift", C.c_uint8),
        ("ar_coeff_lag", C.c_uint8),
        ("ar_coeffs_y", C.c_int8 * 24),
        ("ar_coeffs_cb", C.c_int8 * 25),
        ("ar_coeffs_cr", C.c_int8 * 25),
        ("ar_coeff_shift", C.c_uint8),
        ("grain_scale_shift", C.c_uint8),
        ("cb_mult", C.c_uint8),
        ("cb_luma_mult", C.c_uint8),
        ("cb_offset", C.c_uint16),
        ("cr_mult", C.c_uint8),
        ("cr_luma_mult", C.c_uint8),
        ("cr_offset", C.c_uint16),
        ("overlap", C.c_uint8),
        ("clip_to_restricted_range", C.c_uint8),
        ("matrix_identity", C.c_uint8),
        ("reserved", C.c_uint8),
    ]


class pf_frame_side(C.Structure):
    _fields_ = [
        ("stages", C.c_uint32),
        ("side_memory", C.c_uint32),
        ("lf", pf_loop_filter),
        ("cdef", pf_cdef),
        ("lr", pf_restoration),
        ("fg", pf_film_grain),
    ]


class pf_stats(C.Structure):
    _fields_ = [
        ("completed", C.c_uint32),
        ("cdef_units", C.c_uint32),
        ("lr_units", C.c_uint32),
        ("fg_rows", C.c_uint32),
        ("stage_ms", C.c_float * 5),
    ]


class pf_config(C.Structure):
    _fields_ = [
        ("device", C.c_int32),
        ("timing", C.c_int32),
        ("max_width", C.c_int64),
        ("max_height", C.c_int64),
        ("wait_timeout_us", C.c_int64),
    ]


class pf_batch_item(C.Structure):
    _fields_ = [
        ("frame", C.POINTER(pf_frame)),
        ("side", C.POINTER(pf_frame_side)),
        ("display", C.POINTER(pf_frame)),
    ]


class pf_superres_item(C.Structure):
    _fields_ = [
        ("coded", C.POINTER(pf_frame)),
        ("side", C.POINTER(pf_frame_side)),
        ("up", C.POINTER(pf_frame)),
        ("display", C.POINTER(pf_frame)),
    ]


class pf_cdef_search_params(C.Structure):
    _fields_ = [
        ("qindex", C.c_int32),
        ("damping", C.c_int32),
        ("max_presets", C.c_int32),
        ("lam", C.c_double),
    ]


class pf_cdef_search_result(C.Structure):
    _fields_ = [
        ("bits", C.c_uint8),
        ("strength_count", C.c_uint8),
        ("y_strength", C.c_uint8 * 8),
        ("uv_strength", C.c_uint8 * 8),
        ("reserved", C.c_uint8 * 2),
        ("cost", C.c_double),
    ]


PF_CDEF_MAX_TRIALS = 64
PF_CDEF_NOT_A_TRIAL = 0x7FFFFFFF


class pf_cdef_search_ctrls(C.Structure):
    _fields_ = [
        ("count", C.c_int32),
        ("y", C.c_int8 * PF_CDEF_MAX_TRIALS),
        ("uv", C.c_int8 * PF_CDEF_MAX_TRIALS),
        ("subsampling", C.c_int32),
        ("uv_from_y", C.c_int32),
    ]


class pf_cdef_ref_strengths(C.Structure):
    _fields_ = [
        ("count", C.c_uint8),
        ("y", C.c_uint8 * 8),
        ("uv", C.c_uint8 * 8),
    ]


class pf_cdef_plan(C.Structure):
    _fields_ = [
        ("on", C.c_int32),
        ("search", C.c_int32),
        ("y_strength", C.c_uint8),
        ("uv_strength", C.c_uint8),
        ("reserved", C.c_uint8 * 2),
        ("ctrls", pf_cdef_search_ctrls),
    ]


PF_LEARNED_REFINE = 1
PF_TUNE_DEBLOCK, PF_TUNE_CDEF, PF_TUNE_RESTORATION, PF_TUNE_FILM_GRAIN, PF_TUNE_GROUPS = 0, 1, 2, 3, 4


class pf_schedule(C.Structure):
    _fields_ = [
        ("ctas", C.c_int32),
        ("units_per_cta", C.c_int32),
        ("staging", C.c_int32),
        ("tile", C.c_int32),
    ]

    def as_dict(self):
        return {"ctas": self.ctas, "units_per_cta": self.units_per_cta, "staging": self.staging,
                "tile": self.tile}


class pf_tune_result(C.Structure):
    _fields_ = [
        ("chosen", pf_schedule * PF_TUNE_GROUPS),
        ("ms", C.c_float * PF_TUNE_GROUPS),
        ("ms_default", C.c_float * PF_TUNE_GROUPS),
        ("frame_groups", C.c_int32),
        ("ms_groups", C.c_float * 2),
    ]

PF_MLP_FEATURES = 40
PF_MLP_HIDDEN = 64
PF_MLP_CLASSES = 64
PF_MLP_OUTPUTS = 2 * PF_MLP_CLASSES
PF_MLP_PARAMS = (PF_MLP_HIDDEN * PF_MLP_FEATURES + PF_MLP_HIDDEN * PF_MLP_HIDDEN + PF_MLP_OUTPUTS * PF_MLP_HIDDEN
                 + 2 * PF_MLP_HIDDEN + PF_MLP_OUTPUTS)


class pf_cdef_mlp(C.Structure):
    _fields_ = [
        ("w1", C.c_uint16 * (PF_MLP_HIDDEN * PF_MLP_FEATURES)),
        ("w2", C.c_uint16 * (PF_MLP_HIDDEN * PF_MLP_HIDDEN)),
        ("w3", C.c_uint16 * (PF_MLP_OUTPUTS * PF_MLP_HIDDEN)),
        ("b1", C.c_float * PF_MLP_HIDDEN),
        ("b2", C.c_float * PF_MLP_HIDDEN),
        ("b3", C.c_float * PF_MLP_OUTPUTS),
        ("feat_shift", C.c_float * PF_MLP_FEATURES),
        ("feat_scale", C.c_float * PF_MLP_FEATURES),
    ]


class pf_cdef_mlp_grads(C.Structure):
    _fields_ = [
        ("w1", C.c_float * (PF_MLP_HIDDEN * PF_MLP_FEATURES)),
        ("w2", C.c_float * (PF_MLP_HIDDEN * PF_MLP_HIDDEN)),
        ("w3", C.c_float * (PF_MLP_OUTPUTS * PF_MLP_HIDDEN)),
        ("b1", C.c_float * PF_MLP_HIDDEN),
        ("b2", C.c_float * PF_MLP_HIDDEN),
        ("b3", C.c_float * PF_MLP_OUTPUTS),
    ]


class pf_cdef_mlp_train_params(C.Structure):
    _fields_ = [
        ("epochs", C.c_int32),
        ("batch", C.c_int32),
        ("lr", C.c_float),
        ("beta1", C.c_float),
        ("beta2", C.c_float),
        ("eps", C.c_float),
        ("weight_decay", C.c_float),
        ("seed", C.c_uint32),
    ]


class pf_cdef_learned_stats(C.Structure):
    _fields_ = [
        ("blocks", C.c_int32),
        ("fallback_luma", C.c_int32),
        ("fallback_chroma", C.c_int32),
        ("trials_luma", C.c_int32),
        ("trials_chroma", C.c_int32),
        ("stage_ms", C.c_float * 4),
    ]


PF_LR_WIENER_CANDIDATES = 6
PF_LR_SGR_PRESETS = 4


class pf_lr_search_unit(C.Structure):
    _fields_ = [
        ("x0", C.c_int32),
        ("y0", C.c_int32),
        ("x1", C.c_int32),
        ("y1", C.c_int32),
        ("base_sse", C.c_uint64),
        ("sse", C.c_uint64),
        ("wiener_sse", C.c_uint64),
        ("sgr_sse", C.c_uint64),
        ("wiener_candidate", C.c_int8),
        ("sgr_preset", C.c_int8),
        ("reserved", C.c_uint8 * 2),
        ("unit", pf_lr_unit),
    ]


def lr_unit_grid(width, height):
    """(horz, vert) luma restoration units of 64 samples
    (tile/restoration_schedule.go:400-409)."""
    return max((width + 32) // 64, 1), max((height + 32) // 64, 1)


class pf_lf_record(C.Structure):
    """threading.FrameWorkLoopFilterBlockRecord, one per MI cell (32 bytes)."""
    _fields_ = [
        ("mi_col", C.c_uint16),
        ("mi_row", C.c_uint16),
        ("mi_col_end", C.c_uint16),
        ("mi_row_end", C.c_uint16),
        ("block_size", C.c_uint8),
        ("valid", C.c_uint8),
        ("intra", C.c_uint8),
        ("skip", C.c_uint8),
        ("tx_y", C.c_uint8),
        ("tx_uv", C.c_uint8),
        ("has_uv", C.c_uint8),
        ("segment_id", C.c_uint8),
        ("ref_frame", C.c_uint8),
        ("mode", C.c_uint8),
        ("delta_lf_from_base", C.c_int8),
        ("delta_lf", C.c_int8 * 4),
        ("reserved0", C.c_uint8),
        ("tx_split", C.c_uint16 * 2),
        ("reserved1", C.c_uint32),
    ]


# The same record as a numpy dtype (record maps are built as arrays).
LF_RECORD_DTYPE = None


def lf_record_dtype():
    import numpy as np

    global LF_RECORD_DTYPE
    if LF_RECORD_DTYPE is None:
        LF_RECORD_DTYPE = np.dtype([
            ("mi_col", "<u2"), ("mi_row", "<u2"), ("mi_col_end", "<u2"), ("mi_row_end", "<u2"),
            ("block_size", "u1"), ("valid", "u1"), ("intra", "u1"), ("skip", "u1"), ("tx_y", "u1"),
            ("tx_uv", "u1"), ("has_uv", "u1"), ("segment_id", "u1"), ("ref_frame", "u1"), ("mode", "u1"),
            ("delta_lf_from_base", "i1"), ("delta_lf", "i1", (4,)), ("reserved0", "u1"),
            ("tx_split", "<u2", (2,)), ("reserved1", "<u4")])
        assert LF_RECORD_DTYPE.itemsize == C.sizeof(pf_lf_record) == 32
    return LF_RECORD_DTYPE


class pf_lf_levels(C.Structure):
    """loopfilter.PrepareLevelResolver inputs."""
    _fields_ = [
        ("level_y", C.c_uint8 * 2),
        ("level_u", C.c_uint8),
        ("level_v", C.c_uint8),
        ("delta_lf_present", C.c_uint8),
        ("delta_lf_multi", C.c_uint8),
        ("segmentation_enabled", C.c_uint8),
        ("mode_ref_delta_enabled", C.c_uint8),
        ("ref_delta", C.c_int8 * 8),
        ("mode_delta", C.c_int8 * 2),
        ("reserved", C.c_uint8 * 2),
        ("segment_delta", (C.c_int16 * 4) * 8),
    ]


# Every symbol include/goav1pf.h declares (checked by tests/test_abi.py).
EXPORTED_SYMBOLS = (
    "pf_abi_version",
    "pf_status_string",
    "pf_status_detail",
    "pf_create",
    "pf_destroy",
    "pf_frame_apply",
    "pf_frame_validate",
    "pf_sync",
    "pf_stream",
    "pf_batch_apply",
    "pf_cdef_search",
    "pf_film_grain_static",
    "pf_cdef_features",
    "pf_cdef_mlp_forward",
    "pf_cdef_mlp_gradients",
    "pf_cdef_mlp_train",
    "pf_cdef_search_learned",
    "pf_batch_graphs",
    "pf_set_persistent",
    "pf_set_schedule",
    "pf_get_schedule",
    "pf_set_frame_groups",
    "pf_autotune",
    "pf_lr_search",
    "pf_cdef_apply",
    "pf_superres_upscale",
    "pf_frame_apply_superres",
    "pf_batch_apply_superres",
    "pf_lf_build",
    "pf_diag_issue_rate",
    "pf_cdef_search_level_rtc",
    "pf_cdef_plan_picture",
    "pf_cdef_search_ex",
)
