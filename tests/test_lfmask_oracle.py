"""CPU oracle for the deblocking-mask build from the block record map
(oracle/lfmask_oracle.cpp), pinned three ways:

  * the reference's own known-answer tests of the mask functions
    (internal/av1/lfmask/mask_test.go:205-357): the same blocks, contexts and
    expected mask words;
  * its level resolver against dav1d's per-frame level table, the
    equivalence goav1's TestCalcLFValuesMatchesResolver
    (lfmask/values_test.go:16-105) asserts, over random headers;
  * the neighbour-derived map build against the decode-order build with
    carried contexts on single-tile frames, which goav1 documents as equal
    bit for bit (threading/loop_filter_masks.go:330-345, :425-447)."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi, synth

TX = {"4x4": 0, "8x8": 1, "16x16": 2, "4x16": 13}
INIT_Y, INIT_UV = 2, 1


@pytest.fixture(scope="module")
def lib():
    import oracle_ctypes

    return oracle_ctypes.lib()


def y_word(m, d, pos, s, half):
    return int(m[((d * 32 + pos) * 3 + s) * 2 + half])


def uv_word(m, d, pos, s, half):
    return int(m[384 + ((d * 32 + pos) * 2 + s) * 2 + half])


def mask_block(lib, kind, by4, bx4, w4, h4, skip, tx, split=(0, 0), a=None, l=None, ss=(0, 0), init=INIT_Y):
    m = np.zeros(abi.PF_LF_MASK_WORDS, np.uint16)
    a = np.full(32, init, np.uint8) if a is None else a
    l = np.full(32, init, np.uint8) if l is None else l
    sp = np.array(split, np.uint16)
    lib.oracle_lf_mask_block(kind, m.ctypes.data, by4, bx4, w4, h4, skip, tx, sp.ctypes.data, a.ctypes.data,
                             l.ctypes.data, ss[0], ss[1])
    return m, a, l


def test_kat_intra_4x4(lib):
    # mask_test.go:205-227
    m, a, l = mask_block(lib, 0, 0, 0, 1, 1, 0, TX["4x4"])
    assert y_word(m, 0, 0, 0, 0) == 1 and y_word(m, 1, 0, 0, 0) == 1
    assert all(y_word(m, 0, 0, s, 0) == 0 for s in (1, 2))
    assert a[0] == 0 and l[0] == 0


def test_kat_inter_8x8(lib):
    # mask_test.go:229-259
    m, a, l = mask_block(lib, 1, 0, 0, 2, 2, 0, TX["8x8"])
    assert y_word(m, 0, 0, 1, 0) == 0b11 and y_word(m, 1, 0, 1, 0) == 0b11
    assert y_word(m, 0, 1, 0, 0) == 0 and y_word(m, 0, 1, 1, 0) == 0
    assert list(a[:2]) == [1, 1] and list(l[:2]) == [1, 1]


def test_kat_inter_16x16_split_inner(lib):
    # mask_test.go:261-284: the depth-0 split of a 16x16 into four 8x8.
    m, _, _ = mask_block(lib, 1, 0, 0, 4, 4, 0, TX["16x16"], split=(1, 0))
    assert y_word(m, 0, 2, 1, 0) == 0b1111
    assert y_word(m, 1, 2, 1, 0) == 0b1111
    assert y_word(m, 0, 0, 1, 0) == 0b1111


def test_kat_chroma_420(lib):
    # mask_test.go:286-304
    m, a, l = mask_block(lib, 2, 0, 0, 1, 1, 0, TX["4x4"], ss=(1, 1), init=INIT_UV)
    assert uv_word(m, 0, 0, 0, 0) == 1 and uv_word(m, 1, 0, 0, 0) == 1
    assert a[0] == 0 and l[0] == 0


def test_kat_inter_high_column(lib):
    # mask_test.go:306-327: rows 20..23 land in the high 16-bit lane.
    m, _, _ = mask_block(lib, 1, 20, 0, 1, 4, 0, TX["4x16"])
    assert y_word(m, 0, 0, 0, 1) == 0b11110000
    assert y_word(m, 0, 0, 0, 0) == 0


def test_kat_create_intra_level_cache(lib):
    # mask_test.go:329-357: an 8x8 intra block at the origin of an 8x8 MI
    # grid, 4:2:0, levels (10, 11, 12, 13): its 2x2 luma cells and its one
    # chroma cell.  The rest of the grid is 8x8 intra blocks as well.
    rec = np.zeros((8, 8), abi.lf_record_dtype())
    for y in range(0, 8, 2):
        for x in range(0, 8, 2):
            r = rec[y:y + 2, x:x + 2]
            r["mi_col"], r["mi_row"], r["mi_col_end"], r["mi_row_end"] = x, y, x + 2, y + 2
            r["block_size"], r["valid"], r["intra"] = 17, 1, 1
            r["tx_y"], r["tx_uv"], r["has_uv"] = TX["8x8"], TX["4x4"], 1
    lv = abi.pf_lf_levels()
    lv.level_y[0], lv.level_y[1], lv.level_u, lv.level_v = 10, 11, 12, 13
    masks = np.zeros((1, abi.PF_LF_MASK_WORDS), np.uint16)
    lc = np.zeros((8, 8, 4), np.uint8)
    assert lib.oracle_lf_build(rec.ctypes.data, 8, 8, C.byref(lv), 1, 1, 0, masks.ctypes.data, lc.ctypes.data) == 0
    assert (lc[:2, :2, :2] == [10, 11]).all()
    assert list(lc[0, 0, 2:]) == [12, 13]
    # Every 8x8 block: a class-1 luma left edge at each even column, the
    # frame's left edge included (its context is the reset value 2).
    assert y_word(masks[0], 0, 0, 1, 0) == 0xFF and y_word(masks[0], 0, 2, 1, 0) == 0xFF


def _clip(v, lo=0, hi=63):
    return max(lo, min(hi, v))


def _calc_lf_value(base_lvl, lf_delta, seg_delta, mode_ref, ref_delta, mode_delta):
    # dav1d calc_lf_value as goav1 restates it (lfmask/values.go:59-81):
    # out[ref][mode] for the per-frame table.
    base = _clip(_clip(base_lvl + lf_delta) + seg_delta)
    if not mode_ref:
        return [[base, base] for _ in range(8)]
    sh = 1 if base >= 32 else 0
    out = [[_clip(base + ref_delta[0] * (1 << sh))] * 2]
    for r in range(1, 8):
        out.append([_clip(base + (mode_delta[m] + ref_delta[r]) * (1 << sh)) for m in range(2)])
    return out


def _calc_lf_values(lv, lf_delta):
    # CalcLFValues (lfmask/values.go:87-119): values[seg][dir][ref][mode].
    nseg = 8 if lv.segmentation_enabled else 1
    zero = [[[0, 0] for _ in range(8)] for _ in range(4)]
    if lv.level_y[0] == 0 and lv.level_y[1] == 0:
        return [zero] * nseg
    d0 = lf_delta[0]
    d1, d2, d3 = (lf_delta[1], lf_delta[2], lf_delta[3]) if lv.delta_lf_multi else (d0, d0, d0)
    out = []
    for s in range(nseg):
        sd = list(lv.segment_delta[s]) if lv.segmentation_enabled else [0, 0, 0, 0]
        args = (bool(lv.mode_ref_delta_enabled), list(lv.ref_delta), list(lv.mode_delta))
        t = [_calc_lf_value(lv.level_y[0], d0, sd[0], *args), _calc_lf_value(lv.level_y[1], d1, sd[1], *args)]
        for base, d, sdd in ((lv.level_u, d2, sd[2]), (lv.level_v, d3, sd[3])):
            t.append([[0, 0]] * 8 if base == 0 else _calc_lf_value(base, d, sdd, *args))
        out.append(t)
    return out


def test_level_resolver_matches_per_frame_table(lib):
    """ResolveBlockLevels (oracle) == dav1d's per-frame table lookup
    lflvl[seg][dir][ref][mode] over random headers, as values_test.go:16-105
    asserts in the reference."""
    rng = np.random.default_rng(1)

    def level():
        k = rng.integers(0, 4)
        return 0 if k == 0 else (int(rng.integers(28, 36)) if k == 1 else int(rng.integers(0, 64)))

    for _ in range(1500):
        lv = abi.pf_lf_levels()
        lv.level_y[0], lv.level_y[1] = (0, 0) if rng.integers(0, 8) == 0 else (level(), level())
        lv.level_u, lv.level_v = level(), level()
        lv.mode_ref_delta_enabled = int(rng.integers(0, 2))
        for i in range(8):
            lv.ref_delta[i] = int(rng.integers(-63, 64))
        lv.mode_delta[0], lv.mode_delta[1] = int(rng.integers(-63, 64)), int(rng.integers(-63, 64))
        lv.segmentation_enabled = int(rng.integers(0, 2))
        for s in range(8):
            if rng.integers(0, 3):
                for k in range(4):
                    lv.segment_delta[s][k] = int(rng.integers(-63, 64))
        lv.delta_lf_present = int(rng.integers(0, 2))
        lv.delta_lf_multi = int(rng.integers(0, 2))
        r = np.zeros(1, abi.lf_record_dtype())
        from_base, multi = 0, [0, 0, 0, 0]
        if lv.delta_lf_present:
            from_base = int(rng.integers(-63, 64))
            multi = [int(v) for v in rng.integers(-63, 64, size=4)]
        r["delta_lf_from_base"], r["delta_lf"] = from_base, multi
        lf_delta = [0, 0, 0, 0]
        if lv.delta_lf_present:
            lf_delta = multi if lv.delta_lf_multi else [from_base, 0, 0, 0]
        table = _calc_lf_values(lv, lf_delta)
        out = np.zeros(4, np.uint8)
        for seg in range(8):
            for ref in range(8):
                for mode in range(2):
                    r["segment_id"], r["ref_frame"], r["mode"] = seg, ref, mode
                    assert lib.oracle_lf_block_levels(C.byref(lv), 0, r.ctypes.data, out.ctypes.data) == 0
                    t = table[seg if lv.segmentation_enabled else 0]
                    m = mode if ref else 0
                    want = [t[0][ref][m], t[1][ref][m], t[2][ref][m], t[3][ref][m]]
                    assert list(out) == want, (seg, ref, mode)


def oracle_build(lib, rec, lv, ss=(1, 1), mono=False):
    rows, cols = rec.shape
    sbw, sbh = (cols + 31) // 32, (rows + 31) // 32
    masks = np.zeros((sbw * sbh, abi.PF_LF_MASK_WORDS), np.uint16)
    lc = np.zeros((rows, cols, 4), np.uint8)
    st = lib.oracle_lf_build(rec.ctypes.data, cols, rows, C.byref(lv), ss[0], ss[1], int(mono), masks.ctypes.data,
                             lc.ctypes.data)
    return st, masks, lc


@pytest.mark.parametrize("cols,rows,ss,sb128,mono", [
    (480, 270, (1, 1), True, False),
    (480, 270, (1, 1), False, False),
    (160, 90, (1, 0), True, False),
    (160, 90, (0, 0), False, False),
    (100, 66, (1, 1), False, True),
    (38, 24, (1, 1), True, False),
])
def test_map_build_equals_decode_order_build(lib, cols, rows, ss, sb128, mono):
    for seed in range(3):
        rec, order = synth.make_lf_map(seed, cols, rows, ss=ss, mono=mono, sb128=sb128)
        st, masks, _ = oracle_build(lib, rec, synth.make_lf_levels(seed), ss, mono)
        assert st == 0
        ordered = np.zeros_like(masks)
        assert lib.oracle_lf_build_ordered(rec.ctypes.data, cols, rows, order.ctypes.data, len(order),
                                           5 if sb128 else 4, ss[0], ss[1], int(mono), ordered.ctypes.data) == 0
        assert np.array_equal(masks, ordered), "differ in %d words" % int((masks != ordered).sum())
        assert masks.any()


def test_errors_in_walk_order(lib):
    rec, _ = synth.make_lf_map(7, 64, 32)
    lv = synth.make_lf_levels(7, "deltas")
    assert oracle_build(lib, rec, lv)[0] == 0
    r0 = rec[0, 0]
    bad = rec.copy()
    # A block start whose MIColEnd is not past its cell: threading.ErrInvalidBatch.
    bad[r0["mi_row"]:r0["mi_row_end"], r0["mi_col"]:r0["mi_col_end"]]["mi_col_end"] = 0
    assert oracle_build(lib, bad, lv)[0] == abi.PF_ERR_INVALID_BATCH
    # The walk jumps over the inside of a block: a bad cell there is never read.
    wide = np.argwhere((rec["mi_col_end"] - rec["mi_col"] >= 2) & (rec["mi_col"] == np.arange(64)[None, :]))
    y, x = wide[0]
    bad = rec.copy()
    bad[y, x + 1]["mi_col_end"] = 0
    assert bad[y, x + 1]["mi_col_end"] == 0
    assert oracle_build(lib, bad, lv)[0] == 0
    bad = rec.copy()
    bad[r0["mi_row"]:r0["mi_row_end"], r0["mi_col"]:r0["mi_col_end"]]["ref_frame"] = 8
    assert oracle_build(lib, bad, lv)[0] == abi.PF_ERR_INVALID_FILTER
    bad = rec.copy()
    bad[r0["mi_row"]:r0["mi_row_end"], r0["mi_col"]:r0["mi_col_end"]]["segment_id"] = 9
    assert oracle_build(lib, bad, lv)[0] == abi.PF_ERR_INVALID_FILTER
    lv0 = synth.make_lf_levels(7)  # segmentation off: the segment id is not consulted
    assert oracle_build(lib, bad, lv0)[0] == 0


@pytest.mark.parametrize("cols,rows,sb128", [(480, 270, True), (480, 270, False), (38, 24, True), (2, 66, False)])
def test_synthetic_maps_partition_the_grid(cols, rows, sb128):
    """The generated record maps are what the decoder writes: every cell
    holds the record of the one block covering it (its visible rectangle
    clamped to the grid), blocks are AV1 sizes aligned to their own size
    inside one superblock, and the decode order lists each origin once."""
    bdims, txd, _ = synth.av1_tables()
    rec, order = synth.make_lf_map(5, cols, rows, sb128=sb128)
    assert rec["valid"].all()
    seen = np.zeros((rows, cols), np.int32)
    sb = 32 if sb128 else 16
    origins = set()
    for o in order:
        x, y = int(o) % cols, int(o) // cols
        r = rec[y, x]
        assert (r["mi_col"], r["mi_row"]) == (x, y) and o not in origins
        origins.add(o)
        w4, h4 = bdims[r["block_size"]]
        assert x % w4 == 0 and y % h4 == 0  # AV1 blocks sit on their own size
        assert x // sb == (x + w4 - 1) // sb and y // sb == (y + h4 - 1) // sb
        x1, y1 = min(x + w4, cols), min(y + h4, rows)
        assert (r["mi_col_end"], r["mi_row_end"]) == (x1, y1)
        cells = rec[y:y1, x:x1]
        assert (cells == r).all()
        seen[y:y1, x:x1] += 1
        assert r["tx_y"] < 19 and r["tx_uv"] < 19
        tw, th = txd[r["tx_y"]][:2]
        assert tw <= w4 and th <= h4  # a transform never exceeds its block
    assert (seen == 1).all()
