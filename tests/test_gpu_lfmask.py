"""GPU build of the deblocking masks and level cache from the block record map
(pf_lf_build) vs the CPU oracle (oracle/lfmask_oracle.cpp: BuildFromMap and
populateLoopFilterLevelCacheFromMap restated block by block, pinned by the
reference's known-answer tests).  Every mask word and level byte identical
(integer path, tolerance zero), for 64/128 superblocks, every chroma layout,
every level-resolver mode, frame sizes that cut blocks at the edges, host
and device records, the reference's error statuses, and the deblocking
chain driven by the GPU-built masks."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def runner():
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    yield r
    r.close()


def oracle(rec, lv, ss=(1, 1), mono=False):
    import oracle_ctypes

    rows, cols = rec.shape
    sbw, sbh = (cols + 31) // 32, (rows + 31) // 32
    masks = np.zeros((sbw * sbh, abi.PF_LF_MASK_WORDS), np.uint16)
    lc = np.zeros((rows, cols, 4), np.uint8)
    st = oracle_ctypes.lib().oracle_lf_build(rec.ctypes.data, cols, rows, C.byref(lv), ss[0], ss[1], int(mono),
                                             masks.ctypes.data, lc.ctypes.data)
    return st, masks, lc


def check(runner, rec, lv, ss=(1, 1), mono=False):
    st, want_m, want_l = oracle(rec, lv, ss, mono)
    assert st == 0
    got_m, got_l = runner.lf_build(rec, lv, ss[0], ss[1], mono)
    assert np.array_equal(want_m, got_m), "masks differ in %d words" % int((want_m != got_m).sum())
    assert np.array_equal(want_l, got_l), "level cache differs in %d bytes" % int((want_l != got_l).sum())
    return got_m, got_l


@pytest.mark.parametrize("ss,sb128,levels", [
    ((1, 1), True, "plain"),
    ((1, 1), False, "deltas"),
    ((1, 0), True, "single"),
    ((0, 0), False, "deltas"),
    ((0, 1), True, "plain"),
])
def test_1080p(runner, ss, sb128, levels):
    for seed in range(2):
        rec, _ = synth.make_lf_map(seed, 480, 270, ss=ss, sb128=sb128)
        m, lc = check(runner, rec, synth.make_lf_levels(seed, levels), ss)
        assert m.any() and lc.any()


@pytest.mark.parametrize("cols,rows,ss,mono,levels", [
    (50, 34, (1, 1), False, "deltas"),
    (2, 2, (1, 1), False, "plain"),
    (34, 2, (1, 0), False, "single"),
    (2, 66, (0, 0), False, "deltas"),
    (100, 66, (1, 1), True, "deltas"),
    (480, 270, (1, 1), False, "zero"),
    (960, 540, (1, 1), False, "deltas"),
])
def test_sizes_layouts_levels(runner, cols, rows, ss, mono, levels):
    rec, _ = synth.make_lf_map(cols + rows, cols, rows, ss=ss, mono=mono, sb128=cols % 4 == 0)
    m, lc = check(runner, rec, synth.make_lf_levels(cols, levels), ss, mono)
    if mono:
        assert not m[:, 384:].any() and not lc[:, :, 2:].any()


def test_dense_small_blocks_and_var_tx(runner):
    # Mostly 4x4/8x8 blocks and split transform trees: the densest masks.
    rec, _ = synth.make_lf_map(3, 480, 270, p_split=0.9, p_intra=0.2, p_skip=0.1, p_vartx=1.0)
    check(runner, rec, synth.make_lf_levels(3, "deltas"))


def test_invalid_cells(runner):
    # Cells with no valid record (the reference's reset contexts apply).
    rec, _ = synth.make_lf_map(9, 128, 64)
    rng = np.random.default_rng(9)
    for _ in range(40):
        r = rec[rng.integers(0, 64), rng.integers(0, 128)]
        rec[r["mi_row"]:r["mi_row_end"], r["mi_col"]:r["mi_col_end"]]["valid"] = 0
    check(runner, rec, synth.make_lf_levels(9, "deltas"))


def test_device_records(runner):
    import torch

    rec, _ = synth.make_lf_map(4, 480, 270)
    lv = synth.make_lf_levels(4, "deltas")
    _, want_m, want_l = oracle(rec, lv)
    drec = torch.from_numpy(rec.view(np.uint8).reshape(270, 480, 32).copy()).cuda()
    m, lc = runner.lf_build(drec, lv)
    torch.cuda.synchronize()
    assert np.array_equal(m.cpu().numpy().view(np.uint16), want_m)
    assert np.array_equal(lc.cpu().numpy(), want_l)


def test_errors(runner):
    from goav1_b200.postfilter import ErrInvalidArgument, ErrInvalidBatch, ErrInvalidFilter

    rec, _ = synth.make_lf_map(7, 64, 32)
    lv = synth.make_lf_levels(7, "deltas")
    check(runner, rec, lv)
    r0 = rec[0, 0]
    blk = (slice(int(r0["mi_row"]), int(r0["mi_row_end"])), slice(int(r0["mi_col"]), int(r0["mi_col_end"])))
    cases = [("mi_col_end", 0, ErrInvalidBatch), ("ref_frame", 8, ErrInvalidFilter), ("mode", 2, ErrInvalidFilter),
             ("segment_id", 8, ErrInvalidFilter), ("block_size", 22, ErrInvalidBatch), ("tx_y", 19, ErrInvalidBatch),
             ("tx_uv", 40, ErrInvalidBatch)]
    for field, value, err in cases:
        bad = rec.copy()
        bad[blk][field] = value
        assert oracle(bad, lv)[0] == err.code, field
        with pytest.raises(err):
            runner.lf_build(bad, lv)
    # The first error in the walk's raster order wins: a filter error on row 0
    # before a batch error further down.
    bad = rec.copy()
    bad[blk]["ref_frame"] = 9
    bad[20:, :]["mi_col_end"] = 0
    assert oracle(bad, lv)[0] == abi.PF_ERR_INVALID_FILTER
    with pytest.raises(ErrInvalidFilter):
        runner.lf_build(bad, lv)
    with pytest.raises(ErrInvalidArgument):
        runner.lf_build(rec[:, :63], lv)  # odd MI width
    # After an error the context still works.
    check(runner, rec, lv)


def test_masks_drive_the_deblocking(runner):
    """The chain's deblocking stage on GPU-built masks and levels equals the
    oracle's chain on the oracle-built ones."""
    import oracle_ctypes

    frame, si = synth.make_frame(1, 21, width=1920, height=1080, stages=abi.PF_STAGE_LOOP_FILTER)
    rec, _ = synth.make_lf_map(21, 480, 270)
    lv = synth.make_lf_levels(21, "deltas")
    masks, lc = check(runner, rec, lv)
    lf = si.side.lf
    lf.level_y[0], lf.level_y[1], lf.level_u, lf.level_v = lv.level_y[0], lv.level_y[1], lv.level_u, lv.level_v
    lf.masks, lf.level_cache = masks.ctypes.data, lc.ctypes.data
    lf.sb128_w, lf.sb128_h, lf.mi_cols, lf.mi_rows = 15, 9, 480, 270
    want = frame.copy()
    assert oracle_ctypes.frame_apply(want.pf(), si.side) == 0
    got = frame.copy()
    runner.apply(got.pf(), si.side)
    for p, (a, b) in enumerate(zip(want.planes, got.planes)):
        assert np.array_equal(a, b), "plane %d differs in %d samples" % (p, int((a != b).sum()))
    assert not np.array_equal(want.planes[0], frame.planes[0])


def test_rows_longer_than_one_walk_chunk(runner):
    """MI rows of more than 1024 cells (the row walk goes 1024 cells at a time):
    parity, and errors found in the second and third chunks."""
    from goav1_b200.postfilter import ErrInvalidBatch, ErrInvalidFilter

    rec, _ = synth.make_lf_map(11, 2200, 40)
    lv = synth.make_lf_levels(11, "deltas")
    check(runner, rec, lv)
    for col, field, value, err in ((1500, "mi_col_end", 0, ErrInvalidBatch), (2100, "ref_frame", 8, ErrInvalidFilter)):
        r = rec[5, col]
        blk = (slice(int(r["mi_row"]), int(r["mi_row_end"])), slice(int(r["mi_col"]), int(r["mi_col_end"])))
        bad = rec.copy()
        bad[blk][field] = value
        assert oracle(bad, lv)[0] == err.code
        with pytest.raises(err):
            runner.lf_build(bad, lv)
