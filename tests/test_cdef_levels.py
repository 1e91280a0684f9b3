"""CDEF search levels 1-8 on the host: the picture plan the library derives
(pf_cdef_plan_picture: setSVTCDEFSearchControls, the skip detector and
updateOnRefInfo, as planSVTCDEF runs them in goav1's encoder,
internal/av1/encoder/cdef_frame.go:34-54 and cdef_search.go:72-272) equals
the oracle's independent restatement for every level, picture kind, layer
flag, reference and skip share.  Host logic only (no device call)."""

import ctypes as C
import itertools

import numpy as np
import pytest

from goav1_b200 import abi


@pytest.fixture(scope="module")
def L():
    import goav1_b200

    return goav1_b200.lib()


@pytest.fixture(scope="module")
def O(oracle):
    oracle.oracle_cdef_plan_picture.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_int, C.c_void_p]
    return oracle


def refs(rng):
    out = []
    for count in (1, 2, 4, 8):
        for _ in range(6):
            r = abi.pf_cdef_ref_strengths()
            r.count = count
            for i in range(8):
                r.y[i] = int(rng.integers(0, 64))
                r.uv[i] = int(rng.integers(0, 64))
            out.append(r)
    # References equal to the level's first strengths (searchBestRefFS drops
    # or keeps trials on equality) and all-zero ones (predYF == 0 turns CDEF off).
    for y0, uv0 in ((0, 0), (0, 60), (60, 0), (28, 28)):
        r = abi.pf_cdef_ref_strengths()
        r.count = 1
        r.y[0], r.uv[0] = y0, uv0
        out.append(r)
    return out


def test_rtc_levels(L):
    # svtRTCCDEFSearchLevel: 5 on I slices, 7 screen / 8 camera otherwise.
    assert [L.pf_cdef_search_level_rtc(i, s) for i, s in ((1, 0), (1, 1), (0, 1), (0, 0))] == [5, 5, 7, 8]


def test_plan_matches_oracle_every_level(L, O):
    rng = np.random.default_rng(4)
    rs = refs(rng)
    n = 0
    for level, islice, base, nhl in itertools.product(range(0, 9), (0, 1), (0, 1), (0, 1)):
        for ref in rs:
            for skip in (0, 75, 76, 100):
                a, b = abi.pf_cdef_plan(), abi.pf_cdef_plan()
                assert L.pf_cdef_plan_picture(level, islice, base, nhl, C.byref(ref), skip, C.byref(a)) == 0
                assert O.oracle_cdef_plan_picture(level, islice, base, nhl, C.byref(ref), skip, C.byref(b)) == 0
                assert bytes(a) == bytes(b), (level, islice, base, nhl, list(ref.y), list(ref.uv), skip)
                n += 1
    assert n == 9 * 8 * 28 * 4


def test_plan_level_shapes(L):
    """The level tables as goav1 sets them: trial counts, chroma lists and
    subsampling on intra base-layer pictures of a lower layer (no reference
    strength involved)."""
    want = {1: (64, 64, 1), 2: (48, 12, 1), 3: (20, 5, 1), 4: (12, 3, 1), 5: (6, 3, 1), 6: (4, 2, 4), 7: (4, 2, 4),
            8: (4, 0, 4)}
    for level, (count, chroma, ss) in want.items():
        p = abi.pf_cdef_plan()
        assert L.pf_cdef_plan_picture(level, 1, 1, 1, None, 0, C.byref(p)) == 0
        t = p.ctrls
        assert p.on and p.search
        assert (t.count, sum(1 for g in range(t.count) if t.uv[g] >= 0), t.subsampling) == (count, chroma, ss), level
        assert t.uv_from_y == (level == 8)
    p = abi.pf_cdef_plan()
    assert L.pf_cdef_plan_picture(9, 1, 1, 0, None, 0, C.byref(p)) == abi.PF_ERR_UNSUPPORTED


def test_reference_strength_plans(L):
    # Level 8, inter, not base: use_reference_cdef_fs -> the midpoint of the
    # reference's luma strengths, no search.
    r = abi.pf_cdef_ref_strengths()
    r.count = 2
    r.y[0], r.y[1] = 10, 40
    p = abi.pf_cdef_plan()
    assert L.pf_cdef_plan_picture(8, 0, 0, 0, C.byref(r), 0, C.byref(p)) == 0
    assert p.on and not p.search and p.y_strength == 25 and p.uv_strength == 0
    # Level 7 non-base picture whose reference was mostly skip: CDEF off.
    assert L.pf_cdef_plan_picture(7, 0, 0, 1, C.byref(r), 80, C.byref(p)) == 0
    assert not p.on
    # Level 5 inter, highest layer: search_best_ref_fs -> the first strength
    # and the reference's.
    assert L.pf_cdef_plan_picture(5, 0, 1, 0, C.byref(r), 0, C.byref(p)) == 0
    assert p.on and p.search and p.ctrls.count == 2 and list(p.ctrls.y[:2]) == [0, 10]
