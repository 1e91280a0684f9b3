"""PF_ERR_TIMEOUT on the GPU without a fault: a context with a 1 us wait
deadline queues a 30-frame 1080p batch (a few milliseconds of real work),
pf_sync gives up with PF_ERR_TIMEOUT while it runs, the context stays usable,
later pf_sync calls return once the work is done, and the frames then equal
the oracle's (tolerance zero)."""

import time

import numpy as np
import pytest

from goav1_b200 import synth

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_then_completes():
    import oracle_ctypes

    from goav1_b200.postfilter import DeviceFrame, ErrTimeout, PostFilterRunner, device_side

    frames = [synth.make_frame(1, 2, frame_index=i) for i in range(30)]
    dev = [(DeviceFrame(fr), DeviceFrame(fr.like()), device_side(si, fr)) for fr, si in frames]
    r = PostFilterRunner(wait_timeout_us=1)
    items = r.batch_items([(d.pf(), s.side, dd.pf()) for d, dd, s in dev])
    r.apply_batch(items)  # device frames and side information: queued, no wait
    with pytest.raises(ErrTimeout):
        r.sync()
    for _ in range(20000):  # bounded: the batch needs a few milliseconds
        try:
            r.sync()
            break
        except ErrTimeout:
            time.sleep(0.0005)
    else:
        pytest.fail("the batch did not finish")
    for k in (0, 29):
        fr, si = frames[k]
        ref, disp = fr.copy(), fr.like()
        assert oracle_ctypes.frame_apply(ref.pf(), si.side, disp.pf()) == 0
        d, dd, _ = dev[k]
        for a, b in zip(ref.planes + disp.planes, d.download().planes + dd.download().planes):
            assert np.array_equal(a, b), k
    r.close()
