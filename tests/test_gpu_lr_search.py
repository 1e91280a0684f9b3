"""GPU encoder loop-restoration search (pf_lr_search) vs the CPU oracle
(oracle/lr_search_oracle.cpp): every unit record (rectangle, the four SSEs,
the Wiener and SGR picks, the decision) and the restored luma plane must be
identical (integer path, tolerance zero)."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi, synth

pytestmark = pytest.mark.gpu

SIZES = [(1920, 1080, 2000), (1280, 720, 2001), (640, 360, 2002), (200, 136, 1), (128, 128, 2), (96, 80, 3),
         (16, 16, 4), (72, 40, 5), (1000, 600, 6)]


@pytest.fixture(scope="module")
def runner():
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    yield r
    r.close()


def _oracle(src, rec):
    import oracle_ctypes

    horz, vert = abi.lr_unit_grid(rec.width, rec.height)
    units = (abi.pf_lr_search_unit * (horz * vert))()
    out = rec.copy()
    assert oracle_ctypes.lib().oracle_lr_search(C.byref(src.pf()), C.byref(rec.pf()), C.byref(out.pf()), units,
                                                horz * vert) == 0
    return units, out


def _assert_units(want, got):
    assert len(want) == len(got)
    bad = [i for i, (a, b) in enumerate(zip(want, got)) if bytes(a) != bytes(b)]
    assert not bad, "unit records differ at %s (of %d)" % (bad[:8], len(want))


@pytest.mark.parametrize("w,h,seed", SIZES)
def test_device_frames_match_oracle(runner, w, h, seed):
    from goav1_b200.postfilter import DeviceFrame

    src, rec, _ = synth.make_lr_search_pair(seed, w, h)
    want, out = _oracle(src, rec)
    ds, dr = DeviceFrame(src), DeviceFrame(rec)
    dout = DeviceFrame(rec.like())
    got = runner.lr_search(ds.pf(), dr.pf(), dout.pf())
    _assert_units(want, got)
    res = dout.download()
    assert np.array_equal(res.planes[0][:h, :w], out.planes[0][:h, :w]), \
        "restored luma differs in %d samples" % int((res.planes[0][:h, :w] != out.planes[0][:h, :w]).sum())
    # Only the cropped luma plane is written.
    assert not res.planes[0][h:].any() and not res.planes[0][:, w:].any()
    assert not res.planes[1].any() and not res.planes[2].any()
    # The inputs are left as they were.
    assert np.array_equal(dr.download().planes[0], rec.planes[0])


@pytest.mark.parametrize("w,h,seed", [(640, 360, 7), (200, 136, 8)])
def test_host_frames_and_search_only(runner, w, h, seed):
    src, rec, _ = synth.make_lr_search_pair(seed, w, h)
    want, out = _oracle(src, rec)
    res = rec.copy()
    _assert_units(want, runner.lr_search(src.pf(), rec.pf(), res.pf()))
    assert np.array_equal(res.planes[0], out.planes[0])
    _assert_units(want, runner.lr_search(src.pf(), rec.pf()))


def test_in_place_on_device(runner):
    from goav1_b200.postfilter import DeviceFrame

    src, rec, _ = synth.make_lr_search_pair(9, 1280, 720)
    want, out = _oracle(src, rec)
    ds, dr = DeviceFrame(src), DeviceFrame(rec)
    _assert_units(want, runner.lr_search(ds.pf(), dr.pf(), dr.pf()))
    assert np.array_equal(dr.download().planes[0], out.planes[0])


def test_full_size_records_agree_with_applied_output(runner):
    """At 1080p, independent of the oracle: each unit's reported SSE is the
    SSE of the restored output over its rectangle, never above the
    unfiltered SSE, and the units tile the frame exactly."""
    from goav1_b200.postfilter import DeviceFrame

    src, rec, _ = synth.make_lr_search_pair(2010, 1920, 1080)
    ds, dr = DeviceFrame(src), DeviceFrame(rec)
    dout = DeviceFrame(rec.like())
    units = runner.lr_search(ds.pf(), dr.pf(), dout.pf())
    res = dout.download().planes[0].astype(np.int64)
    s = src.planes[0].astype(np.int64)
    cover = np.zeros((1080, 1920), np.int32)
    for u in units:
        d = s[u.y0:u.y1, u.x0:u.x1] - res[u.y0:u.y1, u.x0:u.x1]
        assert int((d * d).sum()) == u.sse
        assert u.sse <= u.base_sse
        cover[u.y0:u.y1, u.x0:u.x1] += 1
    assert (cover == 1).all()
    kinds = [u.unit.type for u in units]
    assert kinds.count(abi.PF_LR_SGRPROJ) and kinds.count(abi.PF_LR_NONE)


def test_arguments_are_checked(runner):
    from goav1_b200.postfilter import ErrInvalidArgument, ErrShortBuffer, ErrUnsupportedPostFilter
    from goav1_b200 import lib

    src, rec, _ = synth.make_lr_search_pair(1, 128, 128)
    ten = synth.HostFrame.alloc(128, 128, 10)
    with pytest.raises(ErrUnsupportedPostFilter):
        runner.lr_search(ten.pf(), ten.pf())
    other = synth.HostFrame.alloc(136, 128, 8)
    with pytest.raises(ErrUnsupportedPostFilter):
        runner.lr_search(src.pf(), other.pf())
    units = (abi.pf_lr_search_unit * 3)()
    st = lib().pf_lr_search(runner._h, C.byref(src.pf()), C.byref(rec.pf()), None, units, 3)
    assert st == abi.PF_ERR_SHORT_BUFFER
    dev = rec.pf(memory=abi.PF_MEM_DEVICE)
    st = lib().pf_lr_search(runner._h, C.byref(src.pf()), C.byref(dev), None, None, 0)
    assert st == abi.PF_ERR_INVALID_ARG
    with pytest.raises(ErrInvalidArgument):
        from goav1_b200.postfilter import check

        check(lib().pf_lr_search(None, C.byref(src.pf()), C.byref(rec.pf()), None, None, 0))
