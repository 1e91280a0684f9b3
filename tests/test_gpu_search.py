"""GPU encoder CDEF search vs the CPU oracle (oracle/cdef_search_oracle.cpp):
the per-block SSE table, the chosen presets and the per-block preset index
must be identical (integer path, tolerance zero)."""

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


def _oracle(src, rec, noskip, qindex, lam, max_presets):
    import oracle_ctypes

    w, h = rec.width, rec.height
    mi_cols, mi_rows = ((w + 7) >> 3) << 1, ((h + 7) >> 3) << 1
    nfb = ((mi_cols + 15) // 16) * ((mi_rows + 15) // 16)
    mse = np.zeros((2, nfb, 64), np.uint64)
    idx = np.zeros(nfb, np.uint8)
    res = abi.pf_cdef_search_result()
    prm = abi.pf_cdef_search_params(qindex=qindex, damping=0, max_presets=max_presets, lam=lam)
    st = oracle_ctypes.lib().oracle_cdef_search(C.byref(src.pf()), C.byref(rec.pf()),
                                                noskip.ctypes.data if noskip is not None else None, C.byref(prm),
                                                mse.ctypes.data, idx.ctypes.data, C.byref(res))
    assert st == 0
    return res, mse, idx


def _noskip(side, fr):
    ucols, urows = (fr.width + 63) // 64, (fr.height + 63) // 64
    return np.ctypeslib.as_array((C.c_uint8 * (ucols * urows * 8)).from_address(side.side.cdef.noskip)).copy()


@pytest.mark.parametrize("w,h,qindex,lam", [(256, 192, 100, 2000.0), (640, 360, 180, 9000.0), (200, 130, 40, 300.0)])
def test_search_matches_oracle(runner, w, h, qindex, lam):
    src, rec, side, _ = synth.make_search_pair(7 + w, w, h)
    ns = _noskip(side, rec)
    r0, m0, i0 = _oracle(src, rec, ns, qindex, lam, 8)
    r1, m1, i1 = runner.cdef_search(src.pf(), rec.pf(), ns, qindex, lam)
    assert np.array_equal(m0, m1), "SSE tables differ in %d entries" % int((m0 != m1).sum())
    assert np.array_equal(i0, i1)
    assert (r0.bits, r0.strength_count) == (r1.bits, r1.strength_count)
    assert list(r0.y_strength) == list(r1.y_strength) and list(r0.uv_strength) == list(r1.uv_strength)
    assert r0.cost == r1.cost


def test_search_all_blocks_without_noskip(runner):
    src, rec, _, _ = synth.make_search_pair(3, 192, 128)
    r0, m0, i0 = _oracle(src, rec, None, 128, 4000.0, 4)
    r1, m1, i1 = runner.cdef_search(src.pf(), rec.pf(), None, 128, 4000.0, max_presets=4)
    assert np.array_equal(m0, m1) and np.array_equal(i0, i1)
    assert list(r0.y_strength) == list(r1.y_strength) and r0.bits == r1.bits


def test_search_rejects_unsupported_formats(runner):
    from goav1_b200.postfilter import ErrUnsupportedPostFilter

    fr = synth.HostFrame.alloc(64, 64, 10)
    with pytest.raises(ErrUnsupportedPostFilter):
        runner.cdef_search(fr.pf(), fr.pf(), None, 100, 1000.0)
