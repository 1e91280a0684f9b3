"""The loop-restoration search oracle (oracle/lr_search_oracle.cpp) against a
direct numpy restatement of the reference's search logic.

The reference tests this path only by an encode/decode round trip
(encoder_public_test.go:1867-1893, frames of 128x128 and 96x80), which needs
its Go encoder.  Here the unit grid, SearchWienerUnitU8's horizontal-only
scoring and acceptance rule, SearchSGRProjUnitU8's acceptance rule and the
Wiener / SGRProj / none decision are restated independently in numpy
(internal/av1/encoder/restoration.go:149-263, encoder/keyframe_lossy.go:
2310-2383, :2422-2453); the exact filters come from the oracle's Wiener and
SGR restatements, which tests/test_oracle_kat.py pins."""

import ctypes as C

import numpy as np
import pytest

from goav1_b200 import abi, synth

WIENER_SETS = [(0, -3, 12), (0, -5, 18), (0, -2, 8), (0, 2, 10), (1, 4, 14), (0, -1, 4)]
SGR_PRESETS = [(0, 8, 24), (2, 16, 40), (10, 0, 48), (14, 24, 72)]
U64_MAX = (1 << 64) - 1


@pytest.fixture(scope="module")
def oracle():
    import oracle_ctypes

    return oracle_ctypes.lib()


def _filter(oracle, bord, x0, y0, w, h, kind, p):
    """Exact Wiener (kind 'w', set p) or SGR (kind 's', preset p) of one unit
    of the 3-sample bordered recon."""
    out = np.zeros((h, w), np.uint16)
    bs = bord.shape[1]
    origin = bord.ctypes.data + 2 * ((y0 + 3) * bs + x0 + 3)
    if kind == "w":
        t0, t1, t2 = WIENER_SETS[p]
        f = np.array([t0, t1, t2, -2 * (t0 + t1 + t2), t2, t1, t0], np.int16)
        oracle.oracle_wiener(origin, bs, out.ctypes.data, w, w, h, f.ctypes.data, f.ctypes.data, 8)
    else:
        s, a, b = SGR_PRESETS[p]
        xqd = np.array([a, b], np.int8)
        oracle.oracle_sgr(origin, bs, out.ctypes.data, w, w, h, s, xqd.ctypes.data, 8)
    return out.astype(np.int64)


def py_lr_search(oracle, src, rec):
    H, W = rec.shape
    horz, vert = abi.lr_unit_grid(W, H)
    bord = np.ascontiguousarray(np.pad(rec, 3, mode="edge").astype(np.uint16))
    cols = np.pad(rec.astype(np.int64), ((0, 0), (3, 3)), mode="edge")
    out = rec.copy()
    recs = []
    for row in range(vert):
        for col in range(horz):
            x0, x1 = col * 64, (W if col + 1 == horz else col * 64 + 64)
            y0, y1 = row * 64, (H if row + 1 == vert else row * 64 + 64)
            y0 -= 8 if y0 > 0 else 0
            y1 -= 8 if y1 < H else 0
            w, h = x1 - x0, y1 - y0
            fits = w <= 64 and h <= 64
            s = src[y0:y1, x0:x1].astype(np.int64)
            base = int(((s - rec[y0:y1, x0:x1].astype(np.int64)) ** 2).sum())
            wpick, best = -1, base
            if base:
                for c, (t0, t1, t2) in enumerate(WIENER_SETS):
                    f = [t0, t1, t2, -2 * (t0 + t1 + t2), t2, t1, t0]
                    hs = sum(f[k] * cols[y0:y1, x0 + k:x0 + k + w] for k in range(7))
                    sse = int(((s - np.clip((hs + 64) >> 7, 0, 255)) ** 2).sum())
                    if sse + w * h < best:
                        best, wpick = sse, c
            kind, dec, wsse = "n", U64_MAX, U64_MAX
            if wpick >= 0 and fits:
                wsse = int(((s - _filter(oracle, bord, x0, y0, w, h, "w", wpick)) ** 2).sum())
                kind, dec = "w", wsse
            spick, ssse = -1, U64_MAX
            if fits:
                ssse = base
                if base:
                    for p in range(4):
                        sse = int(((s - _filter(oracle, bord, x0, y0, w, h, "s", p)) ** 2).sum())
                        if sse + w * h < ssse:
                            ssse, spick = sse, p
                if spick >= 0 and ssse < dec:
                    kind, dec = "s", ssse
            if kind != "n":
                out[y0:y1, x0:x1] = _filter(oracle, bord, x0, y0, w, h, kind, wpick if kind == "w" else spick)
            recs.append(dict(rect=(x0, y0, x1, y1), base=base, sse=base if kind == "n" else dec, wiener_sse=wsse,
                             sgr_sse=ssse, wc=wpick, sp=spick, kind=kind))
    return recs, out


def run_oracle(oracle, src, rec, restored):
    horz, vert = abi.lr_unit_grid(rec.width, rec.height)
    units = (abi.pf_lr_search_unit * (horz * vert))()
    st = oracle.oracle_lr_search(C.byref(src.pf()), C.byref(rec.pf()),
                                 C.byref(restored.pf()) if restored is not None else None, units, horz * vert)
    return st, units


@pytest.mark.parametrize("w,h,seed", [(128, 128, 1), (96, 80, 2), (200, 136, 1), (256, 200, 3), (16, 16, 4),
                                      (72, 40, 5), (320, 184, 6)])
def test_oracle_matches_numpy_restatement(oracle, w, h, seed):
    src, rec, _ = synth.make_lr_search_pair(seed, w, h)
    restored = rec.copy()
    st, units = run_oracle(oracle, src, rec, restored)
    assert st == 0
    want, out = py_lr_search(oracle, src.planes[0][:h, :w], rec.planes[0][:h, :w])
    assert len(units) == len(want)
    for u, r in zip(units, want):
        assert (u.x0, u.y0, u.x1, u.y1) == r["rect"]
        assert (u.base_sse, u.sse, u.wiener_sse, u.sgr_sse) == (r["base"], r["sse"], r["wiener_sse"], r["sgr_sse"])
        assert (u.wiener_candidate, u.sgr_preset) == (r["wc"], r["sp"])
        t = {"n": abi.PF_LR_NONE, "w": abi.PF_LR_WIENER, "s": abi.PF_LR_SGRPROJ}[r["kind"]]
        assert u.unit.type == t
        if t == abi.PF_LR_WIENER:
            assert tuple(u.unit.wiener_h) == tuple(u.unit.wiener_v) == WIENER_SETS[r["wc"]]
        if t == abi.PF_LR_SGRPROJ:
            s, a, b = SGR_PRESETS[r["sp"]]
            assert (u.unit.sgr_set, u.unit.sgr_xqd[0], u.unit.sgr_xqd[1]) == (s, a, b)
    assert np.array_equal(restored.planes[0][:h, :w], out)
    # Only the cropped luma is written.
    assert np.array_equal(restored.planes[0][h:], rec.planes[0][h:])
    assert np.array_equal(restored.planes[0][:, w:], rec.planes[0][:, w:])
    assert all(np.array_equal(a, b) for a, b in zip(restored.planes[1:], rec.planes[1:]))


def test_oracle_covers_every_branch(oracle):
    """The workload exercises Wiener, SGRProj and none decisions, zero
    unfiltered SSE, Wiener picks that lose to SGR, and units over 64."""
    src, rec, _ = synth.make_lr_search_pair(3, 1280, 720)
    st, units = run_oracle(oracle, src, rec, None)
    assert st == 0
    kinds = [u.unit.type for u in units]
    assert kinds.count(abi.PF_LR_WIENER) and kinds.count(abi.PF_LR_SGRPROJ) and kinds.count(abi.PF_LR_NONE)
    assert any(u.base_sse == 0 for u in units)
    assert any(u.wiener_candidate >= 0 and u.unit.type == abi.PF_LR_SGRPROJ for u in units)
    assert any(u.y1 - u.y0 > 64 and u.unit.type == abi.PF_LR_NONE for u in units)


def test_oracle_in_place_equals_separate_output(oracle):
    src, rec, _ = synth.make_lr_search_pair(8, 200, 136)
    sep = rec.copy()
    _, u0 = run_oracle(oracle, src, rec, sep)
    inplace = rec.copy()
    _, u1 = run_oracle(oracle, src, inplace, inplace)
    assert bytes(u0) == bytes(u1)
    assert np.array_equal(sep.planes[0], inplace.planes[0])


def test_search_unit_record_layout():
    assert C.sizeof(abi.pf_lr_search_unit) == 64
    assert abi.pf_lr_search_unit.unit.offset == 52
    assert abi.lr_unit_grid(1920, 1080) == (30, 17)
    assert abi.lr_unit_grid(16, 16) == (1, 1)
    assert abi.lr_unit_grid(96, 80) == (2, 1)
