"""Parity on exactly the configurations the benchmark times and evaluates.

* the 1080p 8-bit 4:2:0 chain workload (seed 2, per-frame global motion):
  frames 0, 29 and 59 of the 60-frame batch, one batched call;
* the 4K 10-bit 4:2:0 workload (seed 3): frames 0 and 15 of its 16;
* the full 48-frame mixed queue (seeds 100-147: 16x640x360 and 16x1280x720
  8-bit 4:2:0, 8x1920x1080 10-bit 4:2:0, 8x1280x720 8-bit 4:4:4) through the
  autotuned, graph-captured path, capture and replay;
* the exhaustive CDEF search at 1080p on the learned-selection evaluation
  frames (seeds 2000 and 2001), against the search oracle.

Every sample, table entry and decision is compared with the oracle at
tolerance zero (integer arithmetic throughout)."""

import ctypes as C
import multiprocessing as mp
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from goav1_b200 import abi, learned, synth

pytestmark = pytest.mark.gpu

MIXED_SPECS = ([dict(width=640, height=360)] * 16 + [dict(width=1280, height=720)] * 16 +
               [dict(width=1920, height=1080, bit_depth=10)] * 8 + [dict(width=1280, height=720, ss=(0, 0))] * 8)


def _chain_frame(i):
    return synth.make_frame(1, 2, frame_index=i)


def _uhd_frame(i):
    return synth.make_frame(2, 3, frame_index=i, width=3840, height=2160, bit_depth=10)


def _mixed_frame(i):
    return synth.make_frame(1, 100 + i, **MIXED_SPECS[i])


def _gen(fn, idx):
    with mp.get_context("spawn").Pool(min(8, len(idx))) as pool:
        return pool.map(fn, idx)


def _oracle_outputs(frames):
    import oracle_ctypes

    lib = oracle_ctypes.lib()

    def one(item):
        fr, si = item
        ref, disp = fr.copy(), fr.like()
        assert lib.oracle_frame_apply(C.byref(ref.pf()), C.byref(si.side), C.byref(disp.pf())) == 0
        return ref, disp

    with ThreadPoolExecutor(16) as ex:
        return list(ex.map(one, frames))


def _device(frames):
    from goav1_b200.postfilter import DeviceFrame, device_side

    dev = [(DeviceFrame(fr), DeviceFrame(fr.like()), device_side(si, fr)) for fr, si in frames]
    return dev, [(d.pf(), s.side, dd.pf()) for d, dd, s in dev]


def _assert_equal(expected, dev, what, labels):
    for lab, (ref, disp), (d, dd, _) in zip(labels, expected, dev):
        for name, a, b in (("reference", ref, d.download()), ("display", disp, dd.download())):
            for p, (pa, pb) in enumerate(zip(a.planes, b.planes)):
                assert np.array_equal(pa, pb), "%s: frame %s %s plane %d differs in %d samples" % (
                    what, lab, name, p, int((pa != pb).sum()))


@pytest.mark.parametrize("fn,idx,what", [(_chain_frame, [0, 29, 59], "1080p 8-bit workload"),
                                         (_uhd_frame, [0, 15], "4K 10-bit workload")])
def test_benchmark_workload_frames_match_oracle(fn, idx, what):
    from goav1_b200.postfilter import PostFilterRunner

    frames = _gen(fn, idx)
    expected = _oracle_outputs(frames)
    dev, items = _device(frames)
    r = PostFilterRunner()
    r.apply_batch(items)
    r.sync()
    _assert_equal(expected, dev, what, idx)
    r.close()


def test_mixed_48_frame_queue_matches_oracle():
    from goav1_b200.postfilter import PostFilterRunner

    idx = list(range(len(MIXED_SPECS)))
    frames = _gen(_mixed_frame, idx)
    expected = _oracle_outputs(frames)
    r = PostFilterRunner()
    scratch, scratch_items = _device(frames)
    r.autotune(scratch_items, reps=1)
    del scratch, scratch_items
    r.batch_graphs(True)
    dev, items = _device(frames)
    arr = r.batch_items(items)
    # Run 0 captures the graph of this batch signature's first slot, run 1
    # the second slot, run 2 replays the first.
    for run in range(3):
        for (fr, _), (d, _, _) in zip(frames, dev):
            d.upload(fr)
        r.apply_batch(arr)
        r.sync()
        _assert_equal(expected, dev, "mixed queue run %d" % run, idx)
    r.close()


def _search_oracle(src, rec, noskip, qindex, lam):
    import oracle_ctypes

    w, h = rec.width, rec.height
    mi_cols, mi_rows = ((w + 7) >> 3) << 1, ((h + 7) >> 3) << 1
    nfb = ((mi_cols + 15) // 16) * ((mi_rows + 15) // 16)
    mse = np.zeros((2, nfb, 64), np.uint64)
    idx = np.zeros(nfb, np.uint8)
    res = abi.pf_cdef_search_result()
    prm = abi.pf_cdef_search_params(qindex=qindex, damping=0, max_presets=8, lam=lam)
    assert oracle_ctypes.lib().oracle_cdef_search(C.byref(src.pf()), C.byref(rec.pf()), noskip.ctypes.data,
                                                  C.byref(prm), mse.ctypes.data, idx.ctypes.data, C.byref(res)) == 0
    return res, mse, idx


def test_exhaustive_search_1080p_matches_oracle():
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    for seed, src, rec, side, _ in learned.search_frames([2000, 2001], 1920, 1080, workers=2):
        r.apply(rec.pf(), side.side)  # deblock, as the benchmark's search leg does
        ns = learned.noskip_of(side, rec)
        q = learned.frame_qindex(seed)
        r0, m0, i0 = _search_oracle(src, rec, ns, q, learned.LAMBDA)
        r1, m1, i1 = r.cdef_search(src.pf(), rec.pf(), ns, q, learned.LAMBDA)
        assert np.array_equal(m0, m1), "seed %d: SSE tables differ in %d entries" % (seed, int((m0 != m1).sum()))
        assert np.array_equal(i0, i1), seed
        assert (r0.bits, r0.strength_count, list(r0.y_strength), list(r0.uv_strength), r0.cost) == \
            (r1.bits, r1.strength_count, list(r1.y_strength), list(r1.uv_strength), r1.cost), seed
    r.close()
