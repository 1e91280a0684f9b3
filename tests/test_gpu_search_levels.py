"""GPU encoder CDEF search at every search level (pf_cdef_search_ex over the
picture plan of pf_cdef_plan_picture) against the search oracle: the SSE
table (untested chroma trials, the subsampled luma rows of levels 6-8 scaled
back, the entries past the trial list), the presets and the per-block index
must be identical (integer path, tolerance zero)."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi, learned, synth
from goav1_b200.postfilter import cdef_plan_picture

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def runner():
    from goav1_b200.postfilter import PostFilterRunner

    r = PostFilterRunner()
    yield r
    r.close()


def _oracle(src, rec, noskip, qindex, lam, ctrls):
    import oracle_ctypes

    o = oracle_ctypes.lib()
    o.oracle_cdef_search_ex.argtypes = [C.c_void_p] * 8
    w, h = rec.width, rec.height
    mi_cols, mi_rows = ((w + 7) >> 3) << 1, ((h + 7) >> 3) << 1
    nfb = ((mi_cols + 15) // 16) * ((mi_rows + 15) // 16)
    mse = np.zeros((2, nfb, 64), np.uint64)
    idx = np.zeros(nfb, np.uint8)
    res = abi.pf_cdef_search_result()
    prm = abi.pf_cdef_search_params(qindex=qindex, damping=0, max_presets=8, lam=lam)
    assert o.oracle_cdef_search_ex(C.byref(src.pf()), C.byref(rec.pf()),
                                   noskip.ctypes.data if noskip is not None else None, C.byref(prm),
                                   C.byref(ctrls), mse.ctypes.data, idx.ctypes.data, C.byref(res)) == 0
    return res, mse, idx


def _noskip(side, fr):
    ucols, urows = (fr.width + 63) // 64, (fr.height + 63) // 64
    return np.ctypeslib.as_array((C.c_uint8 * (ucols * urows * 8)).from_address(side.side.cdef.noskip)).copy()


def _ref(y, uv, count=1):
    r = abi.pf_cdef_ref_strengths()
    r.count = count
    for i in range(count):
        r.y[i], r.uv[i] = y[i], uv[i]
    return r


def _plans():
    """(name, plan): every level's intra plan, and the inter plans that
    search with the reference's strength (levels 5-8)."""
    out = []
    for level in range(1, 9):
        out.append(("L%d intra" % level, cdef_plan_picture(level, True, is_base=True, not_highest_layer=True)))
    for level, base, nhl in ((5, True, False), (6, True, False), (7, False, True), (8, False, False)):
        p = cdef_plan_picture(level, False, is_base=base, not_highest_layer=nhl, ref=_ref([37], [5]))
        if p.search:
            out.append(("L%d inter" % level, p))
    return out


def _same(r0, m0, i0, r1, m1, i1, what):
    assert np.array_equal(m0, m1), "%s: SSE tables differ in %d entries" % (what, int((m0 != m1).sum()))
    assert np.array_equal(i0, i1), what
    assert (r0.bits, r0.strength_count, list(r0.y_strength), list(r0.uv_strength), r0.cost) == \
        (r1.bits, r1.strength_count, list(r1.y_strength), list(r1.uv_strength), r1.cost), what


@pytest.mark.parametrize("w,h,qindex,lam", [(256, 192, 100, 2000.0), (640, 360, 180, 9000.0), (200, 130, 40, 300.0)])
def test_every_level_matches_oracle(runner, w, h, qindex, lam):
    src, rec, side, _ = synth.make_search_pair(11 + w, w, h)
    ns = _noskip(side, rec)
    plans = _plans()
    assert len(plans) >= 10
    for name, plan in plans:
        r0, m0, i0 = _oracle(src, rec, ns, qindex, lam, plan.ctrls)
        r1, m1, i1 = runner.cdef_search_ex(src.pf(), rec.pf(), ns, qindex, lam, plan.ctrls)
        _same(r0, m0, i0, r1, m1, i1, "%s %dx%d" % (name, w, h))
        assert (m1[:, :, plan.ctrls.count:] == abi.PF_CDEF_NOT_A_TRIAL).all()


def test_level1_ex_is_pf_cdef_search(runner):
    src, rec, side, _ = synth.make_search_pair(5, 320, 240)
    ns = _noskip(side, rec)
    plan = cdef_plan_picture(1, True)
    a = runner.cdef_search(src.pf(), rec.pf(), ns, 120, 3000.0)
    b = runner.cdef_search_ex(src.pf(), rec.pf(), ns, 120, 3000.0, plan.ctrls)
    _same(*a, *b, "level 1")


def test_rtc_levels_at_1080p(runner):
    """The levels goav1's real-time encoder runs (5 on intra pictures, 8 on
    camera-content inter pictures, 7 on screen content) on a 1080p frame of
    the learned-selection evaluation set."""
    seed = 2002
    for s, src, rec, side, _ in learned.search_frames([seed], 1920, 1080, workers=1):
        runner.apply(rec.pf(), side.side)
        ns = learned.noskip_of(side, rec)
        q = learned.frame_qindex(s)
        for name, plan in (("L5 intra", cdef_plan_picture(5, True)),
                           ("L8 inter base", cdef_plan_picture(8, False, is_base=True)),
                           ("L7 inter", cdef_plan_picture(7, False, is_base=True, not_highest_layer=True))):
            assert plan.search, name
            r0, m0, i0 = _oracle(src, rec, ns, q, learned.LAMBDA, plan.ctrls)
            r1, m1, i1 = runner.cdef_search_ex(src.pf(), rec.pf(), ns, q, learned.LAMBDA, plan.ctrls)
            _same(r0, m0, i0, r1, m1, i1, name + " 1080p")
