"""The encoder's CDEF application on the GPU (pf_cdef_apply) vs the CPU
oracle: the searched parameters and per-block indices, with the units coded
as the decoder rebuilds them from the noskip words, must filter the
reconstruction exactly as the oracle's decoder CDEF does (integer path,
tolerance zero).  The unit marking is restated here from
internal/av1/encoder/cdef_apply.go:202-235 (markFromLoopFilterMap)."""

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


def mark_units(noskip, fb_index, w, h):
    ucols, urows = (w + 63) // 64, (h + 63) // 64
    cols8, rows8 = (w + 7) >> 3, (h + 7) >> 3
    read = np.ones(ucols * urows, np.uint8)
    index = np.zeros(ucols * urows, np.uint8)
    for uy in range(urows):
        for ux in range(ucols):
            u = uy * ucols + ux
            if noskip is not None:
                in_frame = 0
                for by in range(min(8, rows8 - uy * 8)):
                    for bx in range(min(8, cols8 - ux * 8)):
                        in_frame |= 1 << (by * 8 + bx)
                word = int.from_bytes(bytes(noskip[u * 8:u * 8 + 8]), "little")
                read[u] = 1 if word & in_frame else 0
            if read[u] and fb_index is not None:
                index[u] = fb_index[u]
    return read, index


def oracle_apply(frame, noskip, qindex, res, fb_index, damping=0):
    import oracle_ctypes

    w, h = frame.width, frame.height
    read, index = mark_units(noskip, fb_index, w, h)
    side = abi.pf_frame_side()
    side.stages = abi.PF_STAGE_CDEF
    side.side_memory = abi.PF_MEM_HOST
    c = side.cdef
    c.damping = damping or 3 + (qindex >> 6)
    c.bits = res.bits
    c.strength_count = 1 << res.bits
    for i in range(8):
        c.y_strength[i], c.uv_strength[i] = res.y_strength[i], res.uv_strength[i]
    keep = [read, index, noskip]
    c.index = index.ctypes.data
    c.read = read.ctypes.data
    c.index_stride, c.index_rows = (w + 63) // 64, (h + 63) // 64
    if noskip is not None:
        c.noskip = noskip.ctypes.data
    assert oracle_ctypes.lib().oracle_cdef(C.byref(frame.pf()), C.byref(side)) == 0
    del keep


def _searched(runner, seed, w, h, qindex=120, lam=4000.0):
    src, rec, side, _ = synth.make_search_pair(seed, w, h)
    runner.apply(rec.pf(), side.side)  # deblock
    ucols, urows = (w + 63) // 64, (h + 63) // 64
    ns = np.ctypeslib.as_array((C.c_uint8 * (ucols * urows * 8)).from_address(side.side.cdef.noskip)).copy()
    res, _, idx = runner.cdef_search(src.pf(), rec.pf(), ns, qindex, lam, want_mse=False)
    return rec, ns, res, idx


def _assert_frames(a, b):
    for p, (pa, pb) in enumerate(zip(a.planes, b.planes)):
        assert np.array_equal(pa, pb), "plane %d differs in %d samples" % (p, int((pa != pb).sum()))


@pytest.mark.parametrize("w,h,seed", [(1920, 1080, 2000), (640, 360, 11), (200, 130, 12)])
def test_apply_matches_oracle(runner, w, h, seed):
    from goav1_b200.postfilter import DeviceFrame

    rec, ns, res, idx = _searched(runner, seed, w, h)
    assert res.bits > 0
    want = rec.copy()
    oracle_apply(want, ns, 120, res, idx)
    got = rec.copy()
    runner.cdef_apply(got.pf(), ns, 120, res, idx)
    _assert_frames(want, got)
    dev = DeviceFrame(rec)
    runner.cdef_apply(dev.pf(), ns, 120, res, idx)
    _assert_frames(want, dev.download())
    assert not np.array_equal(want.planes[0], rec.planes[0])


def test_apply_without_noskip_or_index(runner):
    rec, ns, res, idx = _searched(runner, 13, 320, 200)
    # Sparse words: every third unit without residual, and bottom-row units
    # (25 rows of 8x8 blocks: only block row 0 of unit row 3 is in the frame)
    # whose only set bits lie below the frame, which leaves them uncoded.
    sparse = ns.copy().reshape(-1, 8)
    sparse[::3] = 0
    sparse[15:17] = np.frombuffer((0xFFFFFFFFFFFFFF00).to_bytes(8, "little"), np.uint8)
    sparse = sparse.reshape(-1)
    read, _ = mark_units(sparse, idx, 320, 200)
    assert read[15] == 0 and read[16] == 0 and read[0] == 0 and read[1] == 1
    for noskip, fb in ((None, idx), (ns, None), (None, None), (sparse, idx)):
        want = rec.copy()
        oracle_apply(want, noskip, 120, res, fb)
        got = rec.copy()
        runner.cdef_apply(got.pf(), noskip, 120, res, fb)
        _assert_frames(want, got)


def test_zero_strengths_leave_recon_untouched(runner):
    rec, ns, res, idx = _searched(runner, 14, 256, 128)
    zero = abi.pf_cdef_search_result()
    zero.bits = 1
    got = rec.copy()
    runner.cdef_apply(got.pf(), ns, 120, zero, idx)
    _assert_frames(rec, got)


def test_apply_arguments_are_checked(runner):
    from goav1_b200.postfilter import ErrInvalidCDEF, ErrUnsupportedPostFilter

    rec, ns, res, idx = _searched(runner, 15, 128, 128)
    ten = synth.HostFrame.alloc(128, 128, 10)
    with pytest.raises(ErrUnsupportedPostFilter):
        runner.cdef_apply(ten.pf(), ns, 120, res, idx)
    bad = abi.pf_cdef_search_result()
    C.memmove(C.byref(bad), C.byref(res), C.sizeof(bad))
    bad.bits = 4
    with pytest.raises(ErrInvalidCDEF):
        runner.cdef_apply(rec.pf(), ns, 120, bad, idx)
    bad.bits = res.bits
    with pytest.raises(ErrInvalidCDEF):
        runner.cdef_apply(rec.pf(), ns, 400, res, idx)  # damping 3 + (400 >> 6) = 9
