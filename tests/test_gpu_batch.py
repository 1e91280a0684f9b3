"""Batch scheduling on the GPU: CUDA-graph capture and replay, the stage
schedules (persistent CTAs, work items per CTA, staging depth, deblocking
tile shape) and the autotuner must not change a single sample.

The batch is a reduced form of the mixed workload (640x360 and 1280x720
8-bit 4:2:0, 1920x1080 10-bit 4:2:0, 1280x720 8-bit 4:4:4, each with its own
seed and full-chain side information); every frame is compared bit-exactly
with the oracle (tolerance zero, integer arithmetic)."""

import numpy as np
import pytest

from goav1_b200 import abi, synth

pytestmark = pytest.mark.gpu

SPECS = [dict(width=640, height=360)] * 3 + [dict(width=1280, height=720)] * 2 + \
        [dict(width=1920, height=1080, bit_depth=10)] + [dict(width=1280, height=720, ss=(0, 0))] * 2


def mixed_frames(seed0=100):
    return [synth.make_frame(1, seed0 + i, **kw) for i, kw in enumerate(SPECS)]


@pytest.fixture(scope="module")
def frames():
    return mixed_frames()


@pytest.fixture(scope="module")
def expected(frames):
    import oracle_ctypes

    out = []
    for fr, si in frames:
        ref, disp = fr.copy(), fr.like()
        assert oracle_ctypes.frame_apply(ref.pf(), si.side, disp.pf()) == 0
        out.append((ref, disp))
    return out


class Batch:
    """Device copies of the frames, displays and side information."""

    def __init__(self, frames):
        from goav1_b200.postfilter import DeviceFrame, device_side

        self.frames = frames
        self.dev = [(DeviceFrame(fr), DeviceFrame(fr.like()), device_side(si, fr)) for fr, si in frames]
        self.items = [(d.pf(), s.side, dd.pf()) for d, dd, s in self.dev]

    def reset(self):
        for (fr, _), (d, _, _) in zip(self.frames, self.dev):
            d.upload(fr)


def assert_batch(batch, expected, what):
    for i, ((ref, disp), (d, dd, _)) in enumerate(zip(expected, batch.dev)):
        for name, a, b in (("reference", ref, d.download()), ("display", disp, dd.download())):
            for p, (pa, pb) in enumerate(zip(a.planes, b.planes)):
                assert np.array_equal(pa, pb), "%s: frame %d %s plane %d differs in %d samples" % (
                    what, i, name, p, int((pa != pb).sum()))


def test_graph_capture_and_replays_match_oracle(frames, expected):
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    r.batch_graphs(True)
    b = Batch(frames)
    # Run 1 captures slot A, run 2 slot B, runs 3 and 4 replay them.
    for run in range(4):
        b.reset()
        r.apply_batch(b.items)
        r.sync()
        assert_batch(b, expected, "graph run %d" % run)
    r.close()


def test_persistent_ctas_match_oracle(frames, expected):
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    for g in range(abi.PF_TUNE_GROUPS):
        r.set_persistent(g, 296)
    b = Batch(frames)
    r.apply_batch(b.items)
    r.sync()
    assert_batch(b, expected, "persistent")
    r.close()


# Every value of every schedule dimension (tile shape, work items per CTA,
# staging depth), alone and with persistent CTAs, on every stage group.
SCHEDULES = [dict(tile=t) for t in range(1, 4)] + \
    [dict(units_per_cta=u) for u in (2, 3, 4, 8, 16)] + \
    [dict(units_per_cta=u, staging=d) for u, d in ((1, 1), (1, 3), (2, 1), (4, 2), (4, 3), (16, 3))] + \
    [dict(units_per_cta=4, staging=2, ctas=148), dict(units_per_cta=2, staging=1, ctas=7, tile=2)]


@pytest.mark.parametrize("sched", SCHEDULES, ids=lambda d: "-".join("%s%d" % kv for kv in sorted(d.items())))
def test_schedules_match_oracle(frames, expected, sched):
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    for g in range(abi.PF_TUNE_GROUPS):
        kw = dict(sched)
        if g not in (abi.PF_TUNE_DEBLOCK, abi.PF_TUNE_FILM_GRAIN):
            kw.pop("tile", None)
        r.set_schedule(g, **kw)
        got = r.get_schedule(g).as_dict()
        assert all(got[k] == v for k, v in kw.items())
    b = Batch(frames)
    r.apply_batch(b.items)
    r.sync()
    assert_batch(b, expected, "schedule %r" % sched)
    r.close()


@pytest.mark.parametrize("graphs", [False, True])
def test_frame_groups_match_oracle(frames, expected, graphs):
    """Two frame groups on two streams, with persistent CTAs and chunks on
    some stages, plain and captured as a graph (two runs: capture, replay)."""
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    r.set_frame_groups(2)
    r.set_schedule(abi.PF_TUNE_CDEF, ctas=148, units_per_cta=2)
    r.set_schedule(abi.PF_TUNE_RESTORATION, units_per_cta=4, staging=1)
    r.batch_graphs(graphs)
    b = Batch(frames)
    for run in range(2 if graphs else 1):
        b.reset()
        r.apply_batch(b.items)
        r.sync()
        assert_batch(b, expected, "frame groups run %d" % run)
    r.close()


def test_autotune_then_graphs_match_oracle(frames, expected):
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    scratch = Batch(frames)  # the tuner filters these in place
    res = r.autotune(scratch.items, reps=1)
    for g in range(abi.PF_TUNE_GROUPS):
        c = res.chosen[g]
        assert c.ctas >= 0 and 1 <= c.units_per_cta <= 16 and 0 <= c.staging <= 3
        assert c.tile == 0 or g in (abi.PF_TUNE_DEBLOCK, abi.PF_TUNE_FILM_GRAIN)
        assert r.get_schedule(g).as_dict() == c.as_dict()
    assert all(m > 0 for m in res.ms)
    assert all(m <= d for m, d in zip(res.ms, res.ms_default))
    assert res.frame_groups in (1, 2) and all(m > 0 for m in res.ms_groups)
    r.batch_graphs(True)
    b = Batch(frames)
    for run in range(2):
        b.reset()
        r.apply_batch(b.items)
        r.sync()
        assert_batch(b, expected, "tuned run %d" % run)
    r.close()


def test_scheduling_arguments_are_checked():
    from goav1_b200.postfilter import ErrInvalidArgument, PostFilterRunner

    r = PostFilterRunner()
    with pytest.raises(ErrInvalidArgument):
        r.set_persistent(abi.PF_TUNE_GROUPS, 10)
    with pytest.raises(ErrInvalidArgument):
        r.set_persistent(0, -1)
    with pytest.raises(ErrInvalidArgument):
        r.batch_graphs(2)
    for bad in (0, 3, -1):
        with pytest.raises(ErrInvalidArgument):
            r.set_frame_groups(bad)
    for g, kw in ((abi.PF_TUNE_CDEF, dict(tile=1)), (abi.PF_TUNE_FILM_GRAIN, dict(tile=4)), (0, dict(tile=4)),
                  (0, dict(units_per_cta=0)),
                  (0, dict(units_per_cta=17)), (0, dict(staging=4)), (0, dict(units_per_cta=2, staging=2)),
                  (0, dict(units_per_cta=8, staging=4)), (0, dict(ctas=-1)), (abi.PF_TUNE_GROUPS, {})):
        with pytest.raises(ErrInvalidArgument):
            r.set_schedule(g, **kw)
    r.close()


def _host_copy(fr, pinned, like=False):
    """A host copy of a frame (or a zeroed frame of its geometry), in
    page-locked memory when `pinned`."""
    out = fr.like() if like else fr.copy()
    if pinned:
        import torch

        keep = []
        for k, p in enumerate(out.planes):
            t = torch.empty(p.shape, dtype=torch.uint8 if p.dtype == np.uint8 else torch.int16, pin_memory=True)
            a = t.numpy().view(p.dtype)
            a[:] = p
            out.planes[k] = a
            keep.append(t)
        out._pin = keep
    return out


@pytest.mark.parametrize("pinned,b2b", [(True, False), (False, False), (True, True), (False, True)])
def test_host_frame_batches_match_oracle(frames, expected, pinned, b2b):
    """Host frames through pf_batch_apply's chunked copy/compute pipeline:
    13 frames (four chunks, so the three staging slots wrap) in two calls;
    planes in separate buffers, or back to back in one buffer as goav1
    allocates a frame (each frame then moves as one copy each way)."""
    from goav1_b200.postfilter import PostFilterRunner

    def host(fr, like=False):
        return fr.back_to_back(pinned, like=like) if b2b else _host_copy(fr, pinned, like=like)

    order = list(range(len(frames))) + list(range(5))
    r = PostFilterRunner()
    for call in range(2):
        hosts = [(host(frames[i][0]), host(frames[i][0], like=True)) for i in order]
        items = [(h.pf(), frames[i][1].side, d.pf()) for (h, d), i in zip(hosts, order)]
        stats = r.apply_batch(items)
        assert stats.completed == abi.PF_STAGES_ALL
        for k, ((h, d), i) in enumerate(zip(hosts, order)):
            ref, disp = expected[i]
            for name, a, b in (("reference", ref, h), ("display", disp, d)):
                for p, (pa, pb) in enumerate(zip(a.planes, b.planes)):
                    assert np.array_equal(pa, pb), "call %d item %d %s plane %d differs in %d samples" % (
                        call, k, name, p, int((pa != pb).sum()))
    r.close()


def test_mixed_host_and_device_batch_is_rejected(frames):
    from goav1_b200.postfilter import DeviceFrame, ErrInvalidArgument, PostFilterRunner

    r = PostFilterRunner()
    (f0, s0), (f1, s1) = frames[0], frames[1]
    d1 = DeviceFrame(f1)
    dd1 = DeviceFrame(f1.like())
    h0, hd0 = f0.copy(), f0.like()
    with pytest.raises(ErrInvalidArgument):
        r.apply_batch([(h0.pf(), s0.side, hd0.pf()), (d1.pf(), s1.side, dd1.pf())])
    assert np.array_equal(h0.planes[0], f0.planes[0])
    r.close()


@pytest.mark.parametrize("pinned", [True, False])
def test_single_back_to_back_host_frames(frames, expected, pinned):
    """pf_frame_apply on host frames whose planes lie back to back."""
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    for i, (fr, si) in enumerate(frames):
        h, d = fr.back_to_back(pinned), fr.back_to_back(pinned, like=True)
        r.apply(h.pf(), si.side, d.pf())
        ref, disp = expected[i]
        for name, a, b in (("reference", ref, h), ("display", disp, d)):
            for p, (pa, pb) in enumerate(zip(a.planes, b.planes)):
                assert np.array_equal(pa, pb), "frame %d %s plane %d differs" % (i, name, p)
    r.close()

