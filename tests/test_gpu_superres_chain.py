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


# A batch of super-resolved frames of mixed size, depth, layout, denominator
# and stage set through one pf_batch_apply_superres: every frame must equal
# the oracle's per-frame chain.
BATCH = [
    dict(w=1920, h=1080, denom=12, seed=700),
    dict(w=640, h=360, denom=13, seed=701, bd=10),
    dict(w=416, h=240, denom=10, seed=702, bd=12),
    dict(w=320, h=200, denom=11, seed=703, ss=(0, 0)),
    dict(w=352, h=144, denom=15, seed=704, bd=10, ss=(1, 0)),
    dict(w=480, h=272, denom=9, seed=705, stages=abi.PF_STAGE_LOOP_FILTER | abi.PF_STAGE_CDEF),
    dict(w=480, h=272, denom=16, seed=706, stages=abi.PF_STAGE_LOOP_RESTORATION | abi.PF_STAGE_FILM_GRAIN),
    dict(w=1280, h=720, denom=12, seed=707),
]


def _cases():
    out = []
    for kw in BATCH:
        kw = dict(kw)
        out.append(SuperResCase(kw.pop("w"), kw.pop("h"), kw.pop("denom"), kw.pop("seed"), **kw))
    return out


def test_batch_device_frames_match_oracle(runner):
    from goav1_b200.postfilter import DeviceFrame

    cases = _cases()
    wants = [run_oracle(c) for c in cases]
    dev = [(DeviceFrame(c.coded.copy()), DeviceFrame(c.up.copy()), DeviceFrame(c.up.like())) for c in cases]
    st = runner.apply_batch_superres([(dc.pf(), c.side, du.pf(), dd.pf()) for c, (dc, du, dd) in zip(cases, dev)])
    runner.sync()
    assert st.completed & abi.PF_STAGE_LOOP_RESTORATION
    for i, (want, (dc, du, dd)) in enumerate(zip(wants, dev)):
        for name, a, b in zip(("coded", "upscaled", "display"), want, (dc.download(), du.download(), dd.download())):
            assert_same(a, b, "frame %d %s" % (i, name))


def test_batch_host_frames_match_oracle(runner):
    cases = _cases()[1:4]
    wants = [run_oracle(c) for c in cases]
    got = [(c.coded.copy(), c.up.copy(), c.up.like()) for c in cases]
    runner.apply_batch_superres([(gc.pf(), c.side, gu.pf(), gd.pf()) for c, (gc, gu, gd) in zip(cases, got)])
    for i, (want, g) in enumerate(zip(wants, got)):
        for name, a, b in zip(("coded", "upscaled", "display"), want, g):
            assert_same(a, b, "frame %d %s" % (i, name))


def test_batch_rejects_mixed_memory_and_bad_items(runner):
    from goav1_b200.postfilter import DeviceFrame, ErrInvalidArgument, ErrInvalidFormat

    cases = _cases()[2:4]
    dc = DeviceFrame(cases[0].coded.copy())
    du = DeviceFrame(cases[0].up.copy())
    with pytest.raises(ErrInvalidArgument):
        runner.apply_batch_superres([(dc.pf(), cases[0].side, du.pf(), None),
                                     (cases[1].coded.pf(), cases[1].side, cases[1].up.pf(), None)])
    before = cases[0].coded.copy()
    disp = cases[0].up.like()
    with pytest.raises(ErrInvalidFormat):
        runner.apply_batch_superres([(cases[0].coded.pf(), cases[0].side, cases[0].up.pf(), disp.pf()),
                                     (cases[1].coded.pf(), cases[1].side, cases[1].coded.pf(), None)])
    assert_same(before, cases[0].coded, "coded after a rejected batch")
