"""pf_film_grain_static: film grain for callers that cannot allocate device memory.

A caller adding grain on a presentation thread, or one whose device memory is
owned by another allocator, cannot make the cudaMalloc calls a pf_ctx makes.
pf_film_grain_static keeps its scratch in a fixed file-scope device array
instead.  This checks, through the C ABI, that two calls in a row produce the
display frames the CPU oracle's chain produces with only the film-grain stage
(and, on the same frames, that pf_frame_apply agrees; integer path: the
tolerance is zero), that a first call on a non-blocking stream sees the grain
tables, and that frames beyond the array's stated maximum are rejected before
anything runs.
"""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi, synth

pytestmark = pytest.mark.gpu


def _same(a, b, what):
    for i, (pa, pb) in enumerate(zip(a.planes, b.planes)):
        assert np.array_equal(pa, pb), "%s plane %d differs in %d samples" % (what, i, int((pa != pb).sum()))


def _oracle_display(fr, si):
    import oracle_ctypes

    ref, disp = fr.copy(), fr.like()
    assert oracle_ctypes.frame_apply(ref.pf(), si.side, disp.pf()) == abi.PF_OK
    return disp


def test_static_grain_matches_oracle_and_frame_apply_twice():
    import torch

    import goav1_b200
    from goav1_b200.postfilter import DeviceFrame, PostFilterRunner, device_side

    L = goav1_b200.lib()
    runner = PostFilterRunner()
    # A non-blocking stream: the first call's table upload must be complete
    # before its kernels run, whatever stream the caller uses.
    side_stream = torch.cuda.Stream()
    cases = [dict(width=640, height=360), dict(width=200, height=130, bit_depth=10)]
    for call, kw in enumerate(cases):
        fr, si = synth.make_frame(1, 400 + call, stages=abi.PF_STAGE_FILM_GRAIN, **kw)
        want = _oracle_display(fr, si)
        ref = DeviceFrame(fr)
        expected = DeviceFrame(fr.like())
        runner.apply(ref.pf(), device_side(si, fr).side, expected.pf())
        runner.sync()
        got = DeviceFrame(fr.like())
        st = L.pf_film_grain_static(C.byref(ref.pf()), C.byref(si.side.fg), C.byref(got.pf()),
                                    C.c_void_p(side_stream.cuda_stream))
        assert st == abi.PF_OK, L.pf_status_string(st)
        side_stream.synchronize()
        out = got.download()
        _same(want, out, "call %d against the oracle" % call)
        _same(expected.download(), out, "call %d against pf_frame_apply" % call)
    runner.close()


def test_static_grain_rejects_frames_beyond_the_scratch_limit():
    import goav1_b200
    from goav1_b200.postfilter import DeviceFrame

    L = goav1_b200.lib()
    # ceil(8224/32) * ceil(8192/32) = 257 * 256 > 65536 blocks.
    fr = synth.HostFrame.alloc(8224, 8192, 8)
    si_fg = synth.make_frame(1, 7, width=64, height=64)[1].side.fg
    d, out = DeviceFrame(fr), DeviceFrame(fr)
    assert L.pf_film_grain_static(C.byref(d.pf()), C.byref(si_fg), C.byref(out.pf()), None) == abi.PF_ERR_SHORT_BUFFER
