"""The chain on super-resolved frames (pf_frame_apply_superres) vs the CPU
oracle (oracle_frame_apply_superres): deblocking and CDEF on the coded frame,
the stripe-boundary rows saved from the deblocked coded rows and upscaled,
the upscale, then restoration, border extension and grain on the upscaled
frame.  Every allocated sample of the coded, upscaled and display frames is
compared (integer path, tolerance zero)."""

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


class SuperResCase:
    """A coded frame with its side information; the restoration units are
    those of a frame of the upscaled width (the restoration grid is the
    upscaled one), the rest is the coded frame's."""

    def __init__(self, upscaled_w, h, denom, seed, bd=8, ss=(1, 1), stages=abi.PF_STAGES_ALL):
        cw = (8 * upscaled_w + denom // 2) // denom
        self.coded, self.csi = synth.make_frame(1, seed, width=cw, height=h, bit_depth=bd, ss=ss, stages=stages)
        upf, self.usi = synth.make_frame(1, seed + 1, width=upscaled_w, height=h, bit_depth=bd, ss=ss,
                                         stages=stages)
        self.side = abi.pf_frame_side()
        C.memmove(C.byref(self.side), C.byref(self.csi.side), C.sizeof(self.side))
        self.side.lr = self.usi.side.lr
        self.up = upf.like()
        # Non-zero padding, to see that only what should be written is.
        for p in self.up.planes:
            p[:] = 3


def run_oracle(case):
    import oracle_ctypes

    coded, up, disp = case.coded.copy(), case.up.copy(), case.up.like()
    st = oracle_ctypes.lib().oracle_frame_apply_superres(C.byref(coded.pf()), C.byref(case.side), C.byref(up.pf()),
                                                          C.byref(disp.pf()))
    assert st == 0
    return coded, up, disp


def assert_same(want, got, what):
    for p, (a, b) in enumerate(zip(want.planes, got.planes)):
        assert np.array_equal(a, b), "%s plane %d differs in %d samples" % (what, p, int((a != b).sum()))


def check(runner, case, device=False):
    want = run_oracle(case)
    coded, up, disp = case.coded.copy(), case.up.copy(), case.up.like()
    if device:
        from goav1_b200.postfilter import DeviceFrame

        dc, du, dd = DeviceFrame(coded), DeviceFrame(up), DeviceFrame(disp)
        runner.apply_superres(dc.pf(), case.side, du.pf(), dd.pf())
        coded, up, disp = dc.download(), du.download(), dd.download()
    else:
        runner.apply_superres(coded.pf(), case.side, up.pf(), disp.pf())
    for name, a, b in zip(("coded", "upscaled", "display"), want, (coded, up, disp)):
        assert_same(a, b, name)


@pytest.mark.parametrize("denom", [9, 12, 16])
def test_full_chain_1080p(runner, denom):
    check(runner, SuperResCase(1920, 1080, denom, seed=300 + denom))


@pytest.mark.parametrize("w,h,denom,bd,ss", [
    (640, 360, 13, 10, (1, 1)),
    (416, 240, 10, 12, (1, 1)),
    (320, 200, 11, 8, (0, 0)),
    (352, 144, 15, 10, (1, 0)),
    (200, 130, 14, 8, (1, 1)),
])
def test_sizes_depths_layouts(runner, w, h, denom, bd, ss):
    check(runner, SuperResCase(w, h, denom, seed=w + h, bd=bd, ss=ss))


def test_device_frames(runner):
    check(runner, SuperResCase(1280, 720, 12, seed=11), device=True)


@pytest.mark.parametrize("stages", [
    abi.PF_STAGE_LOOP_FILTER | abi.PF_STAGE_CDEF,
    abi.PF_STAGE_LOOP_RESTORATION,
    abi.PF_STAGE_CDEF | abi.PF_STAGE_LOOP_RESTORATION,
    abi.PF_STAGE_LOOP_FILTER | abi.PF_STAGE_LOOP_RESTORATION | abi.PF_STAGE_FILM_GRAIN,
])
def test_stage_subsets(runner, stages):
    check(runner, SuperResCase(480, 272, 12, seed=stages, stages=stages))


def test_arguments_are_checked(runner):
    from goav1_b200.postfilter import ErrInvalidFormat

    case = SuperResCase(320, 128, 12, seed=5)
    with pytest.raises(ErrInvalidFormat):
        runner.apply_superres(case.coded.pf(), case.side, case.coded.pf())
    before = case.coded.copy()
    narrow = synth.HostFrame.alloc(case.coded.width, 128, 8)
    with pytest.raises(ErrInvalidFormat):
        runner.apply_superres(case.coded.pf(), case.side, narrow.pf())
    assert_same(before, case.coded, "coded after a rejected call")
