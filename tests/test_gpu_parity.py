"""Bit-exact parity of the CUDA post-filter chain against the CPU oracle.

Every case runs the same seeded frame + side information through the oracle
(oracle/pf_oracle.cpp) and through libgoav1pf.so via the C ABI, then compares
every allocated sample of the reference frame and of the film-grain display
frame.  The tolerance is zero: all arithmetic on the path is integer.
"""

import numpy as np
import pytest

from goav1_b200 import abi, synth

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def runner():
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner(timing=True)
    yield r
    r.close()


def _oracle(fr, si):
    import oracle_ctypes

    ref = fr.copy()
    disp = fr.like()
    st = oracle_ctypes.frame_apply(ref.pf(), si.side, disp.pf())
    assert st == 0
    return ref, disp


def _gpu(runner, fr, si):
    out = fr.copy()
    disp = fr.like()
    runner.apply(out.pf(), si.side, disp.pf())
    return out, disp


def _assert_same(a, b, what):
    for i, (pa, pb) in enumerate(zip(a.planes, b.planes)):
        if not np.array_equal(pa, pb):
            ys, xs = np.nonzero(pa != pb)
            raise AssertionError("%s plane %d: %d samples differ, first at (x=%d, y=%d): oracle %d gpu %d"
                                 % (what, i, len(ys), xs[0], ys[0], pa[ys[0], xs[0]], pb[ys[0], xs[0]]))


def _check(runner, fr, si, display=True):
    ref, rdisp = _oracle(fr, si)
    out, gdisp = _gpu(runner, fr, si)
    _assert_same(ref, out, "reference frame")
    if display and (si.side.stages & abi.PF_STAGE_FILM_GRAIN):
        _assert_same(rdisp, gdisp, "display frame")


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_config0_deblock_cdef(runner, seed):
    fr, si = synth.make_frame(0, seed)
    _check(runner, fr, si)


@pytest.mark.parametrize("stages", [
    abi.PF_STAGE_LOOP_FILTER,
    abi.PF_STAGE_CDEF,
    abi.PF_STAGE_LOOP_RESTORATION,
    abi.PF_STAGE_FILM_GRAIN,
    abi.PF_STAGE_EXTEND_BORDERS,
    abi.PF_STAGE_CDEF | abi.PF_STAGE_LOOP_RESTORATION,
])
def test_single_stages(runner, stages):
    fr, si = synth.make_frame(1, 5, width=320, height=240, stages=stages)
    _check(runner, fr, si)


def test_config1_full_chain_1080p(runner):
    fr, si = synth.make_frame(1, 2, frame_index=0)
    _check(runner, fr, si)


def test_config2_full_chain_4k_10bit(runner):
    fr, si = synth.make_frame(2, 3, frame_index=0)
    _check(runner, fr, si)


@pytest.mark.parametrize("w,h", [(66, 66), (130, 98), (200, 130), (33, 17), (1, 1), (72, 520)])
@pytest.mark.parametrize("bd", [8, 10, 12])
def test_odd_sizes_full_chain(runner, w, h, bd):
    fr, si = synth.make_frame(1, 11 + w + h, width=w, height=h, bit_depth=bd)
    _check(runner, fr, si)


@pytest.mark.parametrize("ss", [(0, 0), (1, 0)])
@pytest.mark.parametrize("bd", [8, 10])
def test_chroma_formats(runner, ss, bd):
    fr, si = synth.make_frame(1, 21, width=208, height=144, bit_depth=bd, ss=ss)
    _check(runner, fr, si)


def test_device_resident_matches_host_path(runner):
    import torch
    from goav1_b200.postfilter import DeviceFrame, device_side

    fr, si = synth.make_frame(1, 7, width=640, height=360)
    ref, rdisp = _oracle(fr, si)
    dfr = DeviceFrame(fr)
    ddisp = DeviceFrame(fr.like())
    dsi = device_side(si, fr)
    runner.apply(dfr.pf(), dsi.side, ddisp.pf())
    runner.sync()
    torch.cuda.synchronize()
    _assert_same(ref, dfr.download(), "device reference")
    _assert_same(rdisp, ddisp.download(), "device display")


def test_error_leaves_frame_untouched(runner):
    from goav1_b200 import postfilter

    fr, si = synth.make_frame(1, 9, width=128, height=128)
    si.side.cdef.damping = 2
    out = fr.copy()
    with pytest.raises(postfilter.ErrInvalidCDEF):
        runner.apply(out.pf(), si.side, fr.like().pf())
    _assert_same(fr, out, "untouched")


def test_repeated_calls_are_deterministic(runner):
    fr, si = synth.make_frame(1, 4, width=512, height=256)
    a, da = _gpu(runner, fr, si)
    b, db = _gpu(runner, fr, si)
    _assert_same(a, b, "repeat")
    _assert_same(da, db, "repeat display")


def test_batch_mixed_sizes_depths_formats(runner):
    """One pf_batch_apply over frames of different size, bit depth and chroma
    format equals per-frame oracle runs."""
    from goav1_b200.postfilter import DeviceFrame, device_side

    specs = [dict(width=320, height=180), dict(width=320, height=180), dict(width=640, height=360, bit_depth=10),
             dict(width=256, height=144, ss=(0, 0)), dict(width=200, height=130, bit_depth=12, ss=(1, 0)),
             dict(width=66, height=66)]
    frames = [synth.make_frame(1, 100 + i, **kw) for i, kw in enumerate(specs)]
    items, keep = [], []
    for fr, si in frames:
        d, dd, ds = DeviceFrame(fr), DeviceFrame(fr.like()), device_side(si, fr)
        keep.append((d, dd, ds))
        items.append((d.pf(), ds.side, dd.pf()))
    runner.apply_batch(items)
    runner.sync()
    for (fr, si), (d, dd, _) in zip(frames, keep):
        ref, rdisp = _oracle(fr, si)
        _assert_same(ref, d.download(), "batch reference")
        _assert_same(rdisp, dd.download(), "batch display")


@pytest.mark.parametrize("lag", [0, 1, 2, 3])
@pytest.mark.parametrize("variant", ["all", "no_luma_points", "cfl", "422_10bit", "444"])
def test_film_grain_ar_lags(runner, lag, variant):
    """The grain templates' AR recursion for every lag (compiled per lag),
    with and without luma scaling points (the chroma luma term), chroma
    scaling from luma, and each chroma layout."""
    kw = dict(width=160, height=96, stages=abi.PF_STAGE_FILM_GRAIN)
    if variant == "422_10bit":
        kw.update(ss=(1, 0), bit_depth=10)
    if variant == "444":
        kw.update(ss=(0, 0))
    fr, si = synth.make_frame(1, 40 + lag, **kw)
    fg = si.side.fg
    fg.ar_coeff_lag = lag
    if variant == "no_luma_points":
        fg.num_y_points = 0
    if variant == "cfl":
        fg.chroma_scaling_from_luma = 1
    _check(runner, fr, si)


def test_frame_apply_graphs_match_oracle():
    """Single-frame calls with the context's graphs on (pf_batch_graphs): a
    call of a new signature captures the chain, with the event the
    reference frame's download waits on as an external node, and the next
    call of that signature replays it with new frames.  Pageable host frames,
    page-locked host frames and device frames, each call against the oracle."""
    from goav1_b200.postfilter import DeviceFrame, PostFilterRunner, device_side

    r = PostFilterRunner()
    try:
        r.batch_graphs(True)
        frames = [synth.make_frame(1, 7 + i, width=320, height=240) for i in range(2)]
        for fr, si in frames:
            ref, rdisp = _oracle(fr, si)
            for call in range(2):  # capture, then replay
                out, gdisp = _gpu(r, fr, si)
                _assert_same(ref, out, "pageable reference frame, call %d" % call)
                _assert_same(rdisp, gdisp, "pageable display frame, call %d" % call)
                out, gdisp = fr.back_to_back(pinned=True), fr.back_to_back(pinned=True, like=True)
                r.apply(out.pf(), si.side, gdisp.pf())
                _assert_same(ref, out, "page-locked reference frame, call %d" % call)
                _assert_same(rdisp, gdisp, "page-locked display frame, call %d" % call)
                d, dd, ds = DeviceFrame(fr), DeviceFrame(fr.like()), device_side(si, fr)
                r.apply(d.pf(), ds.side, dd.pf())
                r.sync()
                _assert_same(ref, d.download(), "device reference frame, call %d" % call)
                _assert_same(rdisp, dd.download(), "device display frame, call %d" % call)
    finally:
        r.close()
