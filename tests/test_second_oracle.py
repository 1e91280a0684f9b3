"""The filter arithmetic pinned twice: goav1's literal known-answer vectors
asserted against both CPU oracles, and the two oracles driven against each
other over random inputs (CPU only; integer work, tolerance zero).

oracle/pf_oracle.cpp restates goav1's production Go paths and is what the
CUDA kernels are compared with; oracle/second_oracle.c restates the same
arithmetic from goav1's in-test libaom restatements and from the AV1
specification's own formulation of each process.  Agreement of the two on
the reference's test corpora (regenerated here with the tests' own seeded
generator) and on random inputs across bit depths, strengths, dampings,
directions, Wiener taps, all 16 self-guided parameter sets and the
film-grain options pins the first oracle's filter outputs beyond the
primitives; goav1's literal vectors pin both."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi

# ---------------------------------------------------------------------------
# Bindings of the kernel-level entry points of both oracles.


@pytest.fixture(scope="module")
def L(oracle):
    o = oracle
    o.oracle_lpf_line_thr.argtypes = [C.c_void_p] + [C.c_int] * 5
    o.oracle_lpf_line_thr.restype = None
    o.oracle_lf_thresholds.argtypes = [C.c_int, C.c_int] + [C.POINTER(C.c_int)] * 3
    o.oracle_lf_thresholds.restype = None
    o.oracle_cdef_chroma_dir.argtypes = [C.c_int] * 3
    o.oracle_fg_apply_plane.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                        C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_int] * 4
    o.so_lf_filter.argtypes = [C.c_int, C.c_void_p] + [C.c_int] * 4
    o.so_cdef_filter_block.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p] + [C.c_int] * 9
    o.so_cdef_filter_block.restype = None
    o.so_cdef_find_dir.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_int32)]
    o.so_cdef_adjust_strength.argtypes = [C.c_int, C.c_int32]
    o.so_cdef_chroma_dir.argtypes = [C.c_int] * 3
    o.so_wiener.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_void_p,
                            C.c_void_p, C.c_int]
    o.so_wiener.restype = None
    o.so_sgr_params.argtypes = [C.c_int] + [C.POINTER(C.c_int)] * 4
    o.so_sgr_params.restype = None
    o.so_sgr_decode_xq.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
    o.so_sgr_decode_xq.restype = None
    o.so_sgr_x_by_xplus1.argtypes = [C.c_int]
    o.so_sgr_one_by_n.argtypes = [C.c_int]
    o.so_sgr.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, C.c_void_p,
                         C.c_int]
    o.so_sgr.restype = None
    o.so_grain_templates.argtypes = [C.c_void_p] * 4 + [C.c_int] * 3
    o.so_grain_templates.restype = None
    o.so_scaling_lut.argtypes = [C.c_void_p, C.c_void_p, C.c_int]
    o.so_scaling_lut.restype = None
    o.so_grain_apply_plane.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_int, C.c_int,
                                       C.c_void_p, C.c_void_p, C.c_void_p] + [C.c_int] * 4
    o.so_grain_apply_plane.restype = None
    return o


def ptr(a):
    return a.ctypes.data


class LCG:
    """The seeded generator goav1's CDEF and restoration tests build their
    corpora with (cdef/cdef_test.go:730-745, restoration_test.go:793-804)."""

    def __init__(self, seed):
        self.state = seed

    def generate(self, rng):
        self.state = (1103515245 * self.state + 12345) & 0x7FFFFFFF
        return self.state % rng


# ---------------------------------------------------------------------------
# Deblocking

WD = {4: 4, 6: 6, 8: 8, 14: 16}


def primary_line(L, width, line, q0, bd, limit, blimit, hev):
    """The first oracle on one line (q0 at index q0 of `line`)."""
    buf = np.zeros(16, np.uint16)
    for i in range(16):
        buf[i] = line[min(max(q0 + i - 8, 0), len(line) - 1)]
    L.oracle_lpf_line_thr(ptr(buf), bd, blimit, limit, hev, WD[width])
    return [int(buf[8 + k - q0]) for k in range(len(line))]


def second_line(L, width, line, q0, bd, limit, blimit, hev):
    half = width // 2
    s = np.array([line[q0 - half + i] for i in range(width)], np.int32)
    assert L.so_lf_filter(width, ptr(s), bd, limit, blimit, hev) == 0
    out = list(line)
    for i in range(width):
        out[q0 - half + i] = int(s[i])
    return out


def test_lf_edge_kats_both_oracles(L, kats):
    """Every literal Filter4/6/8/14Edge vector of loopfilter_test.go."""
    assert len(kats["lf_edge_kats"]) >= 12
    for k in kats["lf_edge_kats"]:
        for bd in k["bit_depths"]:
            for name, fn in (("first", primary_line), ("second", second_line)):
                got = fn(L, k["width"], k["line"], k["q0"], bd, k["limit"], k["blimit"], k["hev"])
                for pos, want in k["want"].items():
                    assert got[int(pos)] == want, (name, k["name"], bd, pos, got)


def test_lf_thresholds_kat(L, kats):
    for c in kats["lf_thresholds"]["cases"]:
        E, I, H = C.c_int(), C.c_int(), C.c_int()
        L.oracle_lf_thresholds(c["level"], c["sharpness"], C.byref(E), C.byref(I), C.byref(H))
        assert (I.value, E.value, H.value) == (c["limit"], c["blimit"], c["hev"]), c


def test_lf_cref_corpus_agrees(L, kats):
    """The sample lists goav1's MatchesCReference tests use (their libaom
    restatement is the second oracle here)."""
    n = 0
    for c in kats["lf_cref_samples"]:
        for s in c["samples"]:
            q0 = c["width"] // 2
            a = primary_line(L, c["width"], s, q0, c["bit_depth"], c["limit"], c["blimit"], c["hev"])
            b = second_line(L, c["width"], s, q0, c["bit_depth"], c["limit"], c["blimit"], c["hev"])
            assert a == b, (c["width"], c["bit_depth"], s, a, b)
            n += 1
    assert n >= 40


@pytest.mark.parametrize("width", [4, 6, 8, 14])
@pytest.mark.parametrize("bd", [8, 10, 12])
def test_lf_random_lines_agree(L, width, bd):
    """Random lines (flat, near-flat, stepped and noisy) under thresholds
    from every level and sharpness and under random explicit ones."""
    rng = np.random.default_rng(1000 * width + bd)
    maxv = (1 << bd) - 1
    scale = 1 << (bd - 8)
    filtered = 0
    for i in range(3000):
        kind = i % 4
        base = int(rng.integers(0, maxv + 1))
        if kind == 0:
            line = [base] * width
        elif kind == 1:
            line = [base + int(v) for v in rng.integers(-2 * scale, 2 * scale + 1, width)]
        elif kind == 2:
            step = int(rng.integers(-40, 41)) * scale
            line = [base + (step if j >= width // 2 else 0) + int(v)
                    for j, v in enumerate(rng.integers(-scale, scale + 1, width))]
        else:
            line = [int(v) for v in rng.integers(0, maxv + 1, width)]
        line = [min(max(v, 0), maxv) for v in line]
        if i % 2:
            E, I, H = C.c_int(), C.c_int(), C.c_int()
            L.oracle_lf_thresholds(int(rng.integers(0, 64)), int(rng.integers(0, 8)), C.byref(E), C.byref(I),
                                   C.byref(H))
            limit, blimit, hev = I.value, E.value, H.value
        else:
            limit, blimit, hev = int(rng.integers(0, 64)), int(rng.integers(0, 200)), int(rng.integers(0, 16))
        q0 = width // 2
        a = primary_line(L, width, line, q0, bd, limit, blimit, hev)
        b = second_line(L, width, line, q0, bd, limit, blimit, hev)
        assert a == b, (width, bd, line, limit, blimit, hev, a, b)
        filtered += a != line
    assert filtered > 300  # the corpus exercises the filters, not only the masks


# ---------------------------------------------------------------------------
# CDEF

BSTRIDE, VB, HB, VERY_LARGE = 144, 2, 8, 0x4000
ORIGIN = VB * BSTRIDE + HB


def cdef_block_input(rnd, depth, boundary, it):
    """makeCDEFBlockInput + applyCDEFBoundary (cdef/cdef_test.go:316-353)."""
    rows = 8 + 2 * VB
    mask = (1 << depth) - 1
    level = it << (depth - 8)
    a = np.array([min((rnd.generate(1 << 16) & mask) + level, mask) for _ in range(rows * BSTRIDE)], np.uint16)
    a = a.reshape(rows, BSTRIDE)
    if boundary & 1:
        a[:, :HB] = VERY_LARGE
    if boundary & 2:
        a[:, HB + 8:] = VERY_LARGE
    if boundary & 4:
        a[:VB, :] = VERY_LARGE
    if boundary & 8:
        a[VB + 8:, :] = VERY_LARGE
    return np.ascontiguousarray(a.reshape(-1))


def test_cdef_filter_block_reference_corpus(L):
    """TestFilterBlockMatchesLibaomCorpus (cdef/cdef_test.go:39-83), its
    inputs regenerated with the test's own generator and seed: every size,
    boundary, depth, direction and strength pair, both oracles equal."""
    rnd = LCG(0xBABA)
    n = 0
    for w, h in ((4, 4), (4, 8), (8, 4), (8, 8)):
        for boundary in range(16):
            for depth in (8, 10, 12):
                shift = depth - 8
                for it in range(2):
                    inp = cdef_block_input(rnd, depth, boundary, it)
                    for d in range(8):
                        for pri in [0, 1 << shift, 4 << shift, 8 << shift, 15 << shift]:
                            for sec in [0, 1 << shift, 2 << shift, 4 << shift]:
                                pd, sd = 3 + shift + boundary % 3, 4 + shift + (boundary >> 2) % 3
                                a = np.zeros(64, np.uint16)
                                b = np.zeros(64, np.uint16)
                                L.oracle_cdef_filter_block(ptr(a), ptr(inp), ORIGIN, pri, sec, d, pd, sd, shift, w, h)
                                L.so_cdef_filter_block(ptr(b), w, 0, ptr(inp), ORIGIN, pri, sec, d, pd, sd, shift, w,
                                                       h)
                                assert np.array_equal(a[:w * h], b[:w * h]), (w, h, boundary, depth, d, pri, sec)
                                n += 1
    assert n == 4 * 16 * 3 * 2 * 8 * 5 * 4


def test_cdef_filter_block_random_strengths(L):
    """Every primary strength 0-15 and secondary {0,1,2,4} at every damping
    the chain uses (3-6, plus the bit-depth shift, minus one for chroma)."""
    rng = np.random.default_rng(7)
    for depth in (8, 10, 12):
        shift = depth - 8
        for _ in range(300):
            inp = rng.integers(0, 1 << depth, 12 * BSTRIDE).astype(np.uint16)
            if rng.random() < 0.3:
                inp[rng.random(inp.size) < 0.2] = VERY_LARGE
            pri = int(rng.integers(0, 16)) << shift
            sec = int(rng.choice([0, 1, 2, 4])) << shift
            damp = int(rng.integers(3, 7)) + shift - int(rng.integers(0, 2))
            d = int(rng.integers(0, 8))
            a = np.zeros(64, np.uint16)
            b = np.zeros(64, np.uint16)
            L.oracle_cdef_filter_block(ptr(a), ptr(inp), ORIGIN, pri, sec, d, damp, damp, shift, 8, 8)
            L.so_cdef_filter_block(ptr(b), 8, 0, ptr(inp), ORIGIN, pri, sec, d, damp, damp, shift, 8, 8)
            assert np.array_equal(a, b), (depth, pri, sec, damp, d)


def test_cdef_direction_and_strength_agree(L, kats):
    rng = np.random.default_rng(11)
    for shift in range(5):
        for i in range(2000):
            if i % 3 == 0:
                img = rng.integers(0, 256 << shift, 64).astype(np.uint16)
            else:  # directional texture
                yy, xx = np.mgrid[0:8, 0:8]
                ang = rng.random() * np.pi
                v = 128 + 100 * np.sin((xx * np.cos(ang) + yy * np.sin(ang)) * rng.uniform(0.3, 1.5))
                img = (np.clip(v + rng.normal(0, 3, (8, 8)), 0, 255).astype(np.int64) << shift).astype(np.uint16)
                img = img.reshape(-1)
            va, vb = C.c_int32(), C.c_int32()
            da = L.oracle_cdef_find_dir(ptr(img), 8, shift, C.byref(va))
            db = L.so_cdef_find_dir(ptr(img), 8, shift, C.byref(vb))
            assert (da, va.value) == (db, vb.value), (shift, img)
    for strength in range(0, 64):
        for var in [0, 1, 63, 64, 127, 128, 1000, 4095, 4096, 65535, 1 << 18, 1 << 20, (1 << 30) - 1]:
            assert L.oracle_cdef_adjust_strength(strength, var) == L.so_cdef_adjust_strength(strength, var)
    # The chroma direction conversion: goav1's 4:2:2 case, and every direction
    # of 4:2:2 and 4:4:0 in both oracles.
    k = kats["cdef_chroma_dir"]
    for d, want in zip(k["luma_dirs"], k["want"]):
        assert L.oracle_cdef_chroma_dir(d, k["xdec"], k["ydec"]) == want
        assert L.so_cdef_chroma_dir(d, k["xdec"], k["ydec"]) == want
    for xdec, ydec in ((1, 0), (0, 1), (0, 0), (1, 1)):
        for d in range(8):
            assert L.oracle_cdef_chroma_dir(d, xdec, ydec) == L.so_cdef_chroma_dir(d, xdec, ydec)


# ---------------------------------------------------------------------------
# Wiener


def wiener_taps(t0, t1, t2):
    """NewWienerFilter (restoration/wiener.go:44-47)."""
    return np.array([t0, t1, t2, -2 * (t0 + t1 + t2), t2, t1, t0], np.int16)


def run_wiener(L, src, stride, origin, w, h, vf, hf, bd):
    a = np.zeros(w * h, np.uint16)
    b = np.zeros(w * h, np.uint16)
    L.oracle_wiener(src.ctypes.data + 2 * origin, stride, ptr(a), w, w, h, ptr(vf), ptr(hf), bd)
    L.so_wiener(ptr(src), stride, origin, ptr(b), w, w, h, ptr(vf), ptr(hf), bd)
    return a, b


def test_wiener_reference_corpus(L):
    """TestApplyWienerRestorationMatchesReferenceCorpus
    (restoration_test.go:1651-1707) with its seeded inputs: the first oracle
    against referenceWienerPixel's restatement."""
    rnd = LCG(0xBABA ^ 0x57)
    cases = [(8, 8, 8, wiener_taps(3, -7, 15), wiener_taps(3, -7, 15)),
             (10, 13, 9, wiener_taps(-4, -13, 29), wiener_taps(7, -5, 13)),
             (12, 64, 31, wiener_taps(10, -23, 21), wiener_taps(-5, 8, 46))]
    for bd, w, h, vf, hf in cases:
        stride = w + 6 + 4
        origin = 3 * stride + 3 + 2
        src = np.array([rnd.generate((1 << bd)) for _ in range(stride * (h + 6))], np.uint16)
        a, b = run_wiener(L, src, stride, origin, w, h, vf, hf, bd)
        assert np.array_equal(a, b), (bd, w, h)


def test_wiener_random_taps_agree(L):
    """Taps over the whole coded ranges t0 [-5,10], t1 [-23,8], t2 [-17,46]
    (restoration/wiener.go:11-30), random sizes, every bit depth."""
    rng = np.random.default_rng(3)
    for i in range(240):
        bd = (8, 10, 12)[i % 3]
        w, h = int(rng.integers(1, 65)), int(rng.integers(1, 65))
        vf = wiener_taps(int(rng.integers(-5, 11)), int(rng.integers(-23, 9)), int(rng.integers(-17, 47)))
        hf = wiener_taps(int(rng.integers(-5, 11)), int(rng.integers(-23, 9)), int(rng.integers(-17, 47)))
        if i % 5 == 0:
            vf[0] = vf[6] = 0  # chroma's 5-tap filter
            vf[3] = -2 * (vf[1] + vf[2])
        stride = w + 6
        src = rng.integers(0, 1 << bd, stride * (h + 6)).astype(np.uint16)
        if i % 4 == 0:  # smooth content, where the clamps bind less often
            src = np.clip(rng.integers(0, 1 << bd) + rng.integers(-8, 9, src.size), 0, (1 << bd) - 1).astype(np.uint16)
        a, b = run_wiener(L, src, stride, 3 * stride + 3, w, h, vf, hf, bd)
        assert np.array_equal(a, b), (bd, w, h, vf, hf)


# ---------------------------------------------------------------------------
# Self-guided restoration


def test_sgr_tables_from_the_spec_match_goav1(L, kats):
    """The second oracle derives s, x/(x+1) and 1/n by formula; they equal
    goav1's tables as its tests state them."""
    for set_, e in enumerate(kats["sgr_params"]["sets"]):
        r0, s0, r1, s1 = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        L.so_sgr_params(set_, C.byref(r0), C.byref(s0), C.byref(r1), C.byref(s1))
        assert [r0.value, r1.value] == e["radius"], set_
        for r, s, want in ((r0.value, s0.value, e["s"][0]), (r1.value, s1.value, e["s"][1])):
            assert s == (want if r else 0) and (r or want == -1), (set_, s, want)
    for z, want in kats["sgr_x_by_xplus1"]["checks"].items():
        assert L.so_sgr_x_by_xplus1(int(z)) == want
    for z in range(256):  # the formula against every entry of goav1's table
        assert L.so_sgr_x_by_xplus1(z) == L.oracle_sgr_x_by_xplus1(z), z
    k = kats["sgr_one_by_x"]
    assert L.so_sgr_one_by_n(1) == k["n1"] and L.so_sgr_one_by_n(25) == k["n25"]
    for c in kats["sgr_xq"]["cases"]:
        xqd = np.array(c["xqd"], np.int8)
        a, b = C.c_int(), C.c_int()
        L.so_sgr_decode_xq(ptr(xqd), c["set"], C.byref(a), C.byref(b))
        assert [a.value, b.value] == c["want"], c


def run_sgr(L, src, stride, origin, w, h, set_, xqd, bd):
    a = np.zeros(w * h, np.uint16)
    b = np.zeros(w * h, np.uint16)
    L.oracle_sgr(src.ctypes.data + 2 * origin, stride, ptr(a), w, w, h, set_, ptr(xqd), bd)
    L.so_sgr(ptr(src), stride, origin, ptr(b), w, w, h, set_, ptr(xqd), bd)
    return a, b


def test_sgr_reference_corpus(L):
    """TestSGRApplySeparableMatchesReference (restoration_test.go:283-330)
    with its seeded inputs: every bit depth, size and all 16 parameter sets."""
    rnd = LCG(0xBABA ^ 0x0B0C)
    sizes = [(1, 1), (4, 4), (5, 5), (8, 8), (13, 11), (31, 64), (64, 16), (64, 64), (2, 3), (7, 7)]
    for bd in (8, 10, 12):
        for w, h in sizes:
            for set_ in range(16):
                stride = w + 6 + 5
                origin = 3 * stride + 3
                src = np.array([rnd.generate(1 << bd) for _ in range(stride * (h + 6))], np.uint16)
                xqd = np.array([rnd.generate(96) - 48, rnd.generate(96) - 48], np.int8)
                a, b = run_sgr(L, src, stride, origin, w, h, set_, xqd, bd)
                assert np.array_equal(a, b), (bd, w, h, set_, xqd)


def test_sgr_coded_xqd_ranges_agree(L):
    """xqd over the coded ranges [-96,31] and [-32,95]
    (restoration/selfguided.go:26-29), smooth and noisy units."""
    rng = np.random.default_rng(5)
    for i in range(160):
        bd = (8, 10, 12)[i % 3]
        set_ = i % 16
        w, h = int(rng.integers(1, 40)), int(rng.integers(1, 40))
        stride = w + 6
        if i % 2:
            src = rng.integers(0, 1 << bd, stride * (h + 6))
        else:
            src = np.clip(rng.integers(0, 1 << bd) + rng.integers(-20, 21, stride * (h + 6)), 0, (1 << bd) - 1)
        src = src.astype(np.uint16)
        xqd = np.array([rng.integers(-96, 32), rng.integers(-32, 96)], np.int8)
        a, b = run_sgr(L, src, stride, 3 * stride + 3, w, h, set_, xqd, bd)
        assert np.array_equal(a, b), (bd, w, h, set_, xqd)


# ---------------------------------------------------------------------------
# Film grain


def random_grain_params(rng, bd, ss):
    fg = abi.pf_film_grain()
    fg.apply = 1
    fg.seed = int(rng.integers(0, 1 << 16))
    fg.num_y_points = int(rng.choice([0, 2, 8, 14]))
    xs = np.sort(rng.choice(256, 14, replace=False))
    for i in range(14):
        fg.y_points[i][0], fg.y_points[i][1] = int(xs[i]), int(rng.integers(0, 256))
    fg.chroma_scaling_from_luma = int(rng.random() < 0.25)
    for pts, name in ((fg.cb_points, "num_cb_points"), (fg.cr_points, "num_cr_points")):
        n = 0 if fg.chroma_scaling_from_luma else int(rng.choice([0, 1, 5, 10]))
        setattr(fg, name, n)
        xs = np.sort(rng.choice(256, 10, replace=False))
        for i in range(10):
            pts[i][0], pts[i][1] = int(xs[i]), int(rng.integers(0, 256))
    fg.scaling_shift = int(rng.integers(8, 12))
    fg.ar_coeff_lag = int(rng.integers(0, 4))
    for arr, n in ((fg.ar_coeffs_y, 24), (fg.ar_coeffs_cb, 25), (fg.ar_coeffs_cr, 25)):
        for i in range(n):
            arr[i] = int(rng.integers(-128, 128))
    fg.ar_coeff_shift = int(rng.integers(6, 10))
    fg.grain_scale_shift = int(rng.integers(0, 4))
    fg.cb_mult, fg.cb_luma_mult, fg.cb_offset = int(rng.integers(0, 256)), int(rng.integers(0, 256)), int(
        rng.integers(0, 512))
    fg.cr_mult, fg.cr_luma_mult, fg.cr_offset = int(rng.integers(0, 256)), int(rng.integers(0, 256)), int(
        rng.integers(0, 512))
    fg.overlap = int(rng.random() < 0.7)
    fg.clip_to_restricted_range = int(rng.random() < 0.3)
    fg.matrix_identity = int(rng.random() < 0.3)
    return fg


def test_grain_templates_agree(L):
    """Luma and chroma templates for every AR lag, coefficient and shift
    range, bit depth and chroma layout."""
    rng = np.random.default_rng(9)
    for i in range(96):
        bd = (8, 10, 12)[i % 3]
        ssx, ssy = ((1, 1), (1, 0), (0, 0))[(i // 3) % 3]
        fg = random_grain_params(rng, bd, (ssx, ssy))
        lg = np.zeros(73 * 82, np.int16)
        L.oracle_luma_grain(ptr(lg), C.byref(fg), bd)
        so = [np.zeros(73 * 82, np.int16) for _ in range(3)]
        L.so_grain_templates(ptr(so[0]), ptr(so[1]), ptr(so[2]), C.byref(fg), bd, ssx, ssy)
        assert np.array_equal(lg, so[0]), (i, "luma")
        for p in (1, 2):
            active = fg.chroma_scaling_from_luma or (fg.num_cb_points if p == 1 else fg.num_cr_points)
            if not active:
                continue  # an inactive plane's template is never read
            cg = np.zeros(73 * 82, np.int16)
            L.oracle_chroma_grain(ptr(cg), ptr(lg), C.byref(fg), p, bd, ssx, ssy)
            assert np.array_equal(cg, so[p]), (i, p)


def test_scaling_lut_kats_second_oracle(L, kats):
    for c in kats["scaling_lut"]["cases"]:
        pts = np.array(c["points"], np.uint8).reshape(-1, 2)
        lut = np.zeros(256, np.uint8)
        L.so_scaling_lut(ptr(lut), ptr(pts), len(pts))
        for x, v in c["samples"].items():
            assert lut[int(x)] == v, (c["name"], x)


def apply_plane_both(L, src, luma, fw, fh, grain, lut, fg, plane, bd, ssx, ssy):
    stride = src.shape[1]
    a = np.zeros_like(src)
    b = np.zeros_like(src)
    lp = ptr(luma) if luma is not None else None
    ls = luma.shape[1] if luma is not None else 0
    L.oracle_fg_apply_plane(ptr(src), ptr(a), stride, lp, ls, fw, fh, ptr(grain), ptr(lut), C.byref(fg), plane, bd,
                            ssx, ssy)
    L.so_grain_apply_plane(ptr(src), ptr(b), stride, lp, ls, fw, fh, ptr(grain), ptr(lut), C.byref(fg), plane, bd,
                           ssx, ssy)
    return a, b


def test_grain_row_kats_both_oracles(L, kats):
    """goav1's literal ApplyLumaRow / ApplyChromaRow vectors
    (filmgrain/filmgrain_test.go): templates set at the positions the
    stripe's LFSR offsets select, scaled, blended and clipped."""
    assert len(kats["fg_rows"]) == 10
    for k in kats["fg_rows"]:
        p = k["params"]
        luma_kind = k["plane"] == "luma"
        ssx, ssy = (0, 0) if luma_kind else (p.get("SubsamplingX", 0), p.get("SubsamplingY", 0))
        plane = 0 if luma_kind else 1
        row = p.get("Row", 0)
        bh = 32 >> ssy
        width, height, stride = p["Width"], p["Height"], p["Stride"]
        ph = row * bh + height
        fw = (width << ssx) - (1 if p.get("OddLumaWidth") else 0)
        fh = ph << ssy
        src = np.zeros((ph, stride), np.uint16)
        src[row * bh:, :width] = k["src_value"]
        luma = None
        if not luma_kind:
            luma = np.full((fh, max(fw, 1) + 2), k["luma_value"], np.uint16)
        lut = np.full(256, k["lut"]["fill"], np.uint8)
        for idx, v in k["lut"]["set"].items():
            lut[int(idx)] = v
        grain = np.zeros(73 * 82, np.int16)
        for g in k["grain"]:
            if luma_kind:
                col = 9 + 2 * (g["offset"] >> 4) + g["x"] + 32 * g["block_col"]
                r = 9 + 2 * (g["offset"] & 15) + g["y"] + 32 * g["block_row"]
            else:
                col = (6 + (g["offset"] >> 4) if ssx else 9 + 2 * (g["offset"] >> 4)) + g["x"] + (32 >> ssx) * g["block_col"]
                r = (6 + (g["offset"] & 15) if ssy else 9 + 2 * (g["offset"] & 15)) + g["y"] + (32 >> ssy) * g["block_row"]
            grain[r * 82 + col] = g["value"]
        fg = abi.pf_film_grain()
        fg.apply, fg.seed, fg.scaling_shift = 1, p.get("Seed", 0), p["ScalingShift"]
        fg.overlap = p.get("Overlap", 0)
        fg.clip_to_restricted_range = p.get("ClipToRestrictedRange", 0)
        fg.matrix_identity = p.get("MatrixIdentity", 0)
        fg.chroma_scaling_from_luma = p.get("ChromaScalingFromLuma", 0)
        fg.cb_mult, fg.cb_luma_mult, fg.cb_offset = p.get("ChromaMult", 0), p.get("ChromaLumaMult", 0), p.get(
            "ChromaOffset", 0)
        a, b = apply_plane_both(L, src, luma, fw, fh, grain, lut, fg, plane, p["BitDepth"], ssx, ssy)
        for name, out in (("first", a), ("second", b)):
            band = out[row * bh:]
            for c in k["checks"]:
                y, x = divmod(c["index"], stride)
                assert band[y, x] == c["want"], (name, k["name"], c, band[y, x])


def test_grain_apply_random_planes_agree(L):
    """Whole planes, odd and even sizes, every chroma layout and bit depth,
    overlap on and off, restricted-range clipping, identity matrices, chroma
    scaling from luma and the chroma mult/offset formula."""
    rng = np.random.default_rng(21)
    for i in range(120):
        bd = (8, 10, 12)[i % 3]
        ssx, ssy = ((1, 1), (1, 0), (0, 0))[(i // 3) % 3]
        fg = random_grain_params(rng, bd, (ssx, ssy))
        fw, fh = int(rng.integers(1, 200)), int(rng.integers(1, 140))
        luma = rng.integers(0, 1 << bd, (fh, fw + 3)).astype(np.uint16)
        templates = [np.zeros(73 * 82, np.int16) for _ in range(3)]
        L.so_grain_templates(ptr(templates[0]), ptr(templates[1]), ptr(templates[2]), C.byref(fg), bd, ssx, ssy)
        for plane in (0, 1, 2):
            sx, sy = (ssx, ssy) if plane else (0, 0)
            pw, ph = (fw + sx) >> sx, (fh + sy) >> sy
            src = luma if plane == 0 else rng.integers(0, 1 << bd, (ph, pw + 3)).astype(np.uint16)
            lut = rng.integers(0, 256, 256).astype(np.uint8)
            a, b = apply_plane_both(L, src, luma if plane else None, fw, fh, templates[plane], lut, fg, plane, bd,
                                    ssx, ssy)
            assert np.array_equal(a[:, :pw], b[:, :pw]), (i, plane, bd, ssx, ssy, fw, fh)
