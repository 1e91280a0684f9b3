"""The CPU oracle against goav1's own known-answer vectors (tests/golden/kats.json,
extracted from the reference test files by tests/golden/extract_kats.py)."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi


def test_lfsr_values_and_registers(oracle, kats):
    k = kats["lfsr8"]
    reg = C.c_uint16(k["seed"])
    for v, r in zip(k["values"], k["registers"]):
        assert oracle.oracle_lfsr_next(C.byref(reg), 8) == v
        assert reg.value == r
    k = kats["lfsr11"]
    reg = C.c_uint16(k["seed"])
    for v in k["values"]:
        assert oracle.oracle_lfsr_next(C.byref(reg), 11) == v


def test_fg_plane_and_stripe_seeds(oracle, kats):
    k = kats["fg_seeds"]
    assert k["seed"] ^ 0xB524 == k["cb"]
    assert k["seed"] ^ 0x49D8 == k["cr"]
    assert oracle.oracle_stripe_seed(k["seed"], k["stripe_line"]) == k["stripe"]


def test_gaussian_table(oracle, kats):
    k = kats["gaussian"]
    vals = np.array([oracle.oracle_gaussian(i) for i in range(2048)], np.int64)
    assert vals.sum() == k["sum"]
    assert np.abs(vals).sum() == k["abs"]
    assert ((np.arange(2048) + 1) * vals).sum() == k["weighted"]
    assert list(vals[:8]) == k["first"]
    assert list(vals[k["mid_start"]:k["mid_start"] + 8]) == k["mid"]
    assert list(vals[-8:]) == k["last"]
    assert oracle.oracle_gaussian(2048) == oracle.oracle_gaussian(0)


def test_scaling_lut(oracle, kats):
    for case in kats["scaling_lut"]["cases"]:
        pts = np.array(case["points"], np.uint8).reshape(-1, 2)
        lut = np.zeros(256, np.uint8)
        oracle.oracle_scaling_lut(lut.ctypes.data, pts.ctypes.data if len(pts) else None, len(pts))
        for x, want in case["samples"].items():
            assert lut[int(x)] == want, (case["name"], x)


def test_cdef_direction_patterns(oracle, kats):
    fills = {
        "constant": lambda r, c: 128,
        "horizontal": lambda r, c: r * 32,
        "vertical": lambda r, c: c * 32,
    }
    for case in kats["cdef_dir"]["cases"]:
        img = np.array([[fills[case["name"]](r, c) for c in range(8)] for r in range(8)], np.uint16)
        var = C.c_int32()
        d = oracle.oracle_cdef_find_dir(img.ctypes.data, 8, 0, C.byref(var))
        assert (d, var.value) == (case["dir"], case["var"])


def test_filter14_q32_row7_unchanged(oracle, kats):
    k = kats["filter14_q32_row7"]
    rows = np.array(k["rows"], np.uint16)
    x = k["edge_x"]
    for y in range(rows.shape[0]):
        line = rows[y, x - 8:x + 8].copy()
        oracle.oracle_lpf_line(line.ctypes.data, k["bit_depth"], k["level"], k["sharpness"], 16)
        if y == 7:
            assert line[8] == rows[7, x]


def test_sgr_decode_xq(oracle, kats):
    for case in kats["sgr_xq"]["cases"]:
        xqd = np.array(case["xqd"], np.int8)
        xq = np.zeros(2, np.int16)
        oracle.oracle_sgr_decode_xq(xqd.ctypes.data, case["set"], xq.ctypes.data)
        assert list(xq) == case["want"]


def test_sgr_constant_blocks_stay_constant(oracle):
    # restoration_test.go TestSelfguidedRestorationConstantBlocksStayInRange.
    for bd in (8, 10, 12):
        mx = (1 << bd) - 1
        for (w, h) in ((4, 4), (17, 19), (64, 64)):
            for s in range(16):
                stride = w + 6
                src = np.full((h + 6) * stride, mx // 3, np.uint16)
                dst = np.zeros(w * h, np.uint16)
                xqd = np.array([13, -9], np.int8)
                oracle.oracle_sgr(src.ctypes.data + 2 * (3 * stride + 3), stride, dst.ctypes.data, w, w, h, s,
                                  xqd.ctypes.data, bd)
                assert dst.max() <= mx and (dst == dst[0]).all()


def test_wiener_default_identity_on_flat(oracle, kats):
    # A flat window is a fixed point of any normalised Wiener filter.
    taps = kats["wiener"]["default"][:7]
    assert sum(taps) == 0 and taps[3] == -22
    f = np.array(taps, np.int16)
    for bd in (8, 10, 12):
        w, h, stride = 16, 8, 22
        src = np.full((h + 6) * stride, 100 << (bd - 8), np.uint16)
        dst = np.zeros(w * h, np.uint16)
        oracle.oracle_wiener(src.ctypes.data + 2 * (3 * stride + 3), stride, dst.ctypes.data, w, w, h,
                             f.ctypes.data, f.ctypes.data, bd)
        assert (dst == 100 << (bd - 8)).all()


def test_superres_rows(oracle, kats):
    """superres_test.go:10-47: the normative rows, 8- and 10-bit."""
    for case in kats["superres_rows"]["cases"]:
        src = np.array(case["src"], np.uint16)
        dst = np.zeros(case["dst_width"], np.uint16)
        oracle.oracle_superres_row(src.ctypes.data, len(src), len(src), dst.ctypes.data, len(dst), case["bit_depth"])
        assert list(dst) == case["want"], case["name"]


def test_superres_libaom_aligned_row(oracle, kats):
    """superres_aligned_libaom_test.go:17-51: libaom's row for a coded width of
    107 read over the 112-column MI-aligned span, upscaled to 160."""
    r = kats["superres_libaom_row"]
    src = np.array(r["src_row"], np.uint16)
    dst = np.zeros(r["upscaled_width"], np.uint16)
    oracle.oracle_superres_row(src.ctypes.data, r["aligned_width"], r["coded_width"], dst.ctypes.data, len(dst), 8)
    assert list(dst) == r["want"]


def test_superres_constant_rows_stay_constant(oracle):
    """superres_test.go:49-70: unity-gain phases keep a flat row flat."""
    for value, bd in ((100, 8), (200, 8), (700, 10), (4095, 12)):
        src = np.full(16, value, np.uint16)
        for dw in (17, 20, 32):
            dst = np.zeros(dw, np.uint16)
            oracle.oracle_superres_row(src.ctypes.data, 16, 16, dst.ctypes.data, dw, bd)
            assert (dst == value).all()
