"""The film-grain template kernel's wavefront schedule, restated on the CPU.

`ar_warp` in goav1_b200/csrc/pf_fg.cu runs a template's AR recursion
(filmgrain/luma.go:83-158, chroma.go:92-199) as one warp: AR row v on lane
v mod 32 at column t - 4v, the rows above arriving by shuffles out of
register rings (for lag 3 as a packed int16 pair for `__dp2a_lo`), in a
padded lane-major shared layout where pass-through samples carry a +16384
mark.  This test models those 32 lanes step by step with numpy (the
shuffles, the rings, the pair packing with `__byte_perm`, the dot products,
the marks and the running addresses exactly as the kernel forms them) and
checks the result against the direct recursion, and every address against
the plane buffer.  It needs no GPU; the GPU parity tests check the kernel
itself against the oracle.
"""

import numpy as np
import pytest

ROW, PLANE, COL0, NONAR = 128, 32 * 4 * 128, 4, 16384


def _direct(g, lt, co, lag, cs, bd, w, h):
    """The recursion in raster order (luma.go:83-158 / chroma.go:92-199)."""
    g = g.copy()
    ro, gmin, gmax = 1 << (cs - 1), -(1 << (bd - 1)), (1 << (bd - 1)) - 1
    for y in range(3, h):
        for x in range(3, w - 3):
            s, pos = 0, 0
            for dy in range(-lag, 1):
                for dx in range(-lag, lag + 1):
                    if dy == 0 and dx == 0:
                        break
                    s += co[pos] * int(g[y + dy, x + dx])
                    pos += 1
            if lt is not None:
                s += co[pos] * int(lt[y, x])
            g[y, x] = min(max(int(g[y, x]) + ((s + ro) >> cs), gmin), gmax)
    return g


def _tpl_at(y, x):
    v = y - 3
    return (4 * (v & 31) + (v >> 5) + 1) * ROW + x + COL0


def _s16(a):
    a = np.asarray(a, np.int64) & 0xFFFF
    return np.where(a >= 0x8000, a - 0x10000, a)


def _s8(a):
    a = np.asarray(a, np.int64) & 0xFF
    return np.where(a >= 0x80, a - 0x100, a)


def _dp2a_lo(a, b, c):
    """__dp2a_lo: the two int16 halves of a times the low two int8 bytes of b."""
    a, b = np.asarray(a, np.int64), np.asarray(b, np.int64)
    return _s16(a) * _s8(b) + _s16(a >> 16) * _s8(b >> 8) + c


def _byte_perm(a, b, sel):
    src = [(np.asarray(a, np.int64) >> (8 * i)) & 0xFF for i in range(4)] + \
          [(np.asarray(b, np.int64) >> (8 * i)) & 0xFF for i in range(4)]
    r = sum(src[(sel >> (4 * i)) & 7] << (8 * i) for i in range(4))
    return np.where(r >= 2 ** 31, r - 2 ** 32, r)


def _kernel(g, lt, co, lag, cs, bd, w, h):
    """ar_warp's 32 lanes, step by step; returns the template and the
    lowest and highest address touched."""
    mem = np.full(PLANE, NONAR, np.int64)
    for y in range(h):
        for x in range(w):
            mem[_tpl_at(y, x)] = int(g[y, x]) + (0 if (y >= 3 and 3 <= x < w - 3) else NONAR)
    lmem = None
    if lt is not None:
        lmem = np.full(PLANE, 12345, np.int64)  # only AR positions are read
        for y in range(3, h):
            for x in range(3, w - 3):
                lmem[_tpl_at(y, x)] = lt[y, x]
    W = 2 * lag + 1
    U = 2 * W
    ro, gmin, gmax = 1 << (cs - 1), -(1 << (bd - 1)), (1 << (bd - 1)) - 1
    cp, c1 = [0] * W, [0] * W
    for j in range(W):
        if lag >= 2:
            cp[j] = (co[2 * lag - j] & 0xFF) | ((co[W + 2 * lag - j] & 0xFF) << 8)
        if lag == 3:
            c1[j] = co[2 * W + 2 * lag - j]
        if lag == 1:
            c1[j] = co[2 * lag - j]
    cin = [0] + [co[lag * W + lag - m] for m in range(1, lag + 1)]
    coL = co[2 * lag * (lag + 1)] if lt is not None else 0
    lane = np.arange(32)
    src = (lane + 31) & 31
    acc = np.full((W, 32), ro, np.int64)
    ring = np.zeros((U, 32), np.int64)
    ring2 = np.zeros((U, 32), np.int64)
    pos0 = 508 * lane + 132
    tend = 4 * (h - 4) + w - 3
    lo, hi = PLANE, -1
    t0 = -4 * lag
    while t0 < tend:
        for k in range(U):
            if lag == 3:
                q = ring2[(k + U - 4) % U][src]
                v1 = ring[(k + U - 1) % U][src]
                for j in range(W - 1, -1, -1):
                    acc[(j + k) % W] = _dp2a_lo(q, cp[j], acc[(j + k) % W])
                for j in range(W - 1, -1, -1):
                    acc[(j + k) % W] += c1[j] * v1
                ring2[k] = _byte_perm(q, v1, 0x5432)
            elif lag == 2:
                v1 = ring[(k + U - 2) % U][src]
                v2 = ring2[(k + U - 4) % U][src]
                pr = _byte_perm(v2, v1, 0x5410)
                ring2[k] = v1
                for j in range(W - 1, -1, -1):
                    acc[(j + k) % W] = _dp2a_lo(pr, cp[j], acc[(j + k) % W])
            else:
                v1 = ring[(k + U - 3) % U][src]
                for j in range(W - 1, -1, -1):
                    acc[(j + k) % W] += c1[j] * v1
            a = pos0 + t0 + k
            lo, hi = min(lo, int(a.min())), max(hi, int(a.max()))
            g0 = _s16(mem[a])
            s = acc[k % W].copy()
            if lmem is not None:
                s = s + _s16(lmem[a]) * coL
            o = np.clip(g0 + (s >> cs), gmin, gmax)
            out = np.where(g0 >= NONAR // 2, g0 - NONAR, o)
            mem[a] = out
            ring[k] = out
            acc[k % W] = ro
            for m in range(1, lag + 1):
                acc[(m + k) % W] += cin[m] * out
        t0 += U
    res = np.zeros_like(g)
    for y in range(73):
        for x in range(82):
            v = int(_s16(mem[_tpl_at(y, x)]))
            res[y, x] = v - NONAR if v >= NONAR // 2 else v
    return res, lo, hi


@pytest.mark.parametrize("lag", [1, 2, 3])
@pytest.mark.parametrize("shape,luma_term,bd", [((82, 73), False, 8), ((44, 38), True, 10), ((44, 73), True, 12)])
def test_wavefront_schedule_matches_recursion(lag, shape, luma_term, bd):
    w, h = shape
    rng = np.random.default_rng(100 * lag + w + bd)
    co = [int(c) for c in rng.integers(-128, 128, 2 * lag * (lag + 1) + (1 if luma_term else 0))]
    cs = int(rng.integers(6, 10))
    lim = 1 << (bd - 1)
    g = np.zeros((73, 82), np.int64)
    g[:h, :w] = rng.integers(-lim, lim, (h, w))
    lt = None
    if luma_term:
        lt = np.zeros((73, 82), np.int64)
        lt[:h, :w] = rng.integers(-lim, lim, (h, w))
    got, lo, hi = _kernel(g, lt, co, lag, cs, bd, w, h)
    assert np.array_equal(got, _direct(g, lt, co, lag, cs, bd, w, h))
    assert 0 <= lo and hi < PLANE, (lo, hi)
