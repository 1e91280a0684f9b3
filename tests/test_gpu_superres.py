"""GPU super-resolution upscale (pf_superres_upscale) vs the CPU oracle
(oracle/superres_oracle.cpp, pinned by the reference's known-answer rows):
every written sample identical (integer path, tolerance zero), for every
denominator the bitstream allows (9..16, coded width = (8 * upscaled + d / 2)
/ d), 8/10/12-bit, 4:2:0, 4:2:2, 4:4:4 and monochrome, host and device
frames, odd and MI-unaligned coded widths."""

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


def coded_width(upscaled, denom):
    return (8 * upscaled + denom // 2) // denom


def make_pair(upscaled_w, h, denom, bd=8, ss=(1, 1), mono=False, seed=0):
    """A coded frame with random samples everywhere in its allocation (so the
    columns past the crop, which the upscaler reads, are not zero) and a zeroed
    upscaled frame."""
    cw = coded_width(upscaled_w, denom)
    rng = np.random.default_rng([seed, cw, h, bd])
    coded = synth.HostFrame.alloc(cw, h, bd, ss_x=ss[0], ss_y=ss[1])
    for p in coded.planes:
        p[:] = rng.integers(0, 1 << bd, size=p.shape)
    up = synth.HostFrame.alloc(upscaled_w, h, bd, ss_x=ss[0], ss_y=ss[1])
    if mono:
        coded.mono = up.mono = 1
    return coded, up


def oracle(coded, up):
    import oracle_ctypes

    want = up.copy()
    assert oracle_ctypes.lib().oracle_superres_upscale(C.byref(coded.pf()), C.byref(want.pf())) == 0
    return want


def assert_planes(want, got, nplanes=3):
    for p in range(nplanes):
        a, b = want.planes[p], got.planes[p]
        assert np.array_equal(a, b), "plane %d differs in %d samples" % (p, int((a != b).sum()))


@pytest.mark.parametrize("denom", list(range(9, 17)))
def test_every_denominator_1080p(runner, denom):
    coded, up = make_pair(1920, 1080, denom, seed=denom)
    want = oracle(coded, up)
    runner.superres_upscale(coded.pf(), up.pf())
    assert_planes(want, up)


@pytest.mark.parametrize("w,h,denom,bd,ss", [
    (160, 128, 12, 8, (1, 1)),   # the reference's libaom case: coded width 107, aligned span 112
    (333, 77, 9, 10, (1, 1)),
    (258, 65, 16, 12, (1, 1)),
    (200, 48, 13, 8, (1, 0)),
    (130, 40, 11, 10, (0, 0)),
    (17, 9, 10, 8, (1, 1)),
    (3840, 64, 14, 10, (1, 1)),
])
def test_sizes_depths_layouts(runner, w, h, denom, bd, ss):
    coded, up = make_pair(w, h, denom, bd=bd, ss=ss, seed=w + h)
    want = oracle(coded, up)
    runner.superres_upscale(coded.pf(), up.pf())
    assert_planes(want, up)


def test_device_frames_and_monochrome(runner):
    from goav1_b200.postfilter import DeviceFrame

    coded, up = make_pair(1280, 720, 15, bd=10, seed=3)
    want = oracle(coded, up)
    dc, du = DeviceFrame(coded), DeviceFrame(up)
    runner.superres_upscale(dc.pf(), du.pf())
    assert_planes(want, du.download())
    mc, mu = make_pair(640, 96, 12, mono=True, seed=4)
    want = oracle(mc, mu)
    runner.superres_upscale(mc.pf(), mu.pf())
    assert_planes(want, mu, nplanes=1)
    assert not mu.planes[1].any() and not mu.planes[2].any()


def test_only_the_crop_is_written(runner):
    coded, up = make_pair(200, 50, 12, seed=5)
    for p in up.planes:
        p[:] = 77
    want = oracle(coded, up)
    runner.superres_upscale(coded.pf(), up.pf())
    assert_planes(want, up)
    assert (up.planes[0][50:] == 77).all() and (up.planes[0][:, 200:] == 77).all()


def test_arguments_are_checked(runner):
    from goav1_b200.postfilter import ErrInvalidArgument, ErrInvalidFormat, ErrShortBuffer

    coded, up = make_pair(160, 64, 12)
    with pytest.raises(ErrInvalidFormat):
        runner.superres_upscale(coded.pf(), coded.pf())  # not wider
    other = synth.HostFrame.alloc(160, 64, 10)
    with pytest.raises(ErrInvalidFormat):
        runner.superres_upscale(coded.pf(), other.pf())  # bit depth differs
    short = up.pf()
    short.plane[0].alloc_width = 100
    with pytest.raises(ErrShortBuffer):
        runner.superres_upscale(coded.pf(), short)
    dev = up.pf(memory=abi.PF_MEM_DEVICE)
    with pytest.raises(ErrInvalidArgument):
        runner.superres_upscale(coded.pf(), dev)
