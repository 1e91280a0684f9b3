"""Seeded synthetic frames and side information for the post-filter workloads.

The reference measures on no public corpus for this path, so every workload
is generated from a seed: a reconstruction built from 2-D cosine gradients,
per-8x8 DC offsets and Gaussian noise, plus the decode-time side information
goav1's decoder would hand its post-filter runner (deblocking edge masks and
level cache, CDEF index map and noskip words, restoration units, film-grain
parameters).  Layouts are exactly the reference's (see include/goav1pf.h).

Frames are allocated like goav1's frame.RequiredSize (frame/buffer.go:141-186):
planes are padded to the 64-pixel superblock grid and reconstruction data
fills the whole allocation, so the 8-aligned padding that CDEF and the
deblocking taps may touch holds real samples.
"""

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi

# ---------------------------------------------------------------------------
# Frame container


@dataclass
class HostFrame:
    """Planes of one frame in host memory (numpy), with a pf_frame view."""

    width: int
    height: int
    bit_depth: int
    ss_x: int
    ss_y: int
    planes: list  # numpy arrays [alloc_h, alloc_w], uint8 or uint16
    crop: list  # (w, h) per plane
    mono: int = 0

    @staticmethod
    def alloc(width, height, bit_depth, ss_x=1, ss_y=1, sb=64):
        dtype = np.uint8 if bit_depth == 8 else np.uint16
        aw = (width + sb - 1) // sb * sb
        ah = (height + sb - 1) // sb * sb
        planes = [np.zeros((ah, aw), dtype)]
        crop = [(width, height)]
        cw, ch = (width + ss_x) >> ss_x, (height + ss_y) >> ss_y
        planes.append(np.zeros((ah >> ss_y, aw >> ss_x), dtype))
        planes.append(np.zeros((ah >> ss_y, aw >> ss_x), dtype))
        crop += [(cw, ch), (cw, ch)]
        return HostFrame(width, height, bit_depth, ss_x, ss_y, planes, crop)

    def copy(self):
        return HostFrame(self.width, self.height, self.bit_depth, self.ss_x, self.ss_y,
                         [p.copy() for p in self.planes], list(self.crop), self.mono)

    def like(self):
        return HostFrame(self.width, self.height, self.bit_depth, self.ss_x, self.ss_y,
                         [np.zeros_like(p) for p in self.planes], list(self.crop), self.mono)

    def back_to_back(self, pinned=False, like=False):
        """A copy (or, with `like`, a zeroed frame of the same geometry) whose
        planes lie back to back in one buffer, Y then U then V, as goav1's
        frame.Bind lays a frame out (frame/buffer.go:141-236); page-locked
        when `pinned`."""
        sizes = [p.nbytes for p in self.planes]
        if pinned:
            import torch

            buf_t = torch.zeros(sum(sizes), dtype=torch.uint8, pin_memory=True)
            buf = buf_t.numpy()
        else:
            buf_t, buf = None, np.zeros(sum(sizes), np.uint8)
        planes, at = [], 0
        for p, n in zip(self.planes, sizes):
            a = buf[at:at + n].view(p.dtype).reshape(p.shape)
            if not like:
                a[:] = p
            planes.append(a)
            at += n
        out = HostFrame(self.width, self.height, self.bit_depth, self.ss_x, self.ss_y, planes, list(self.crop),
                        self.mono)
        out._buf = (buf_t, buf)
        return out

    def pf(self, memory=abi.PF_MEM_HOST, ptrs=None):
        f = abi.pf_frame()
        f.width, f.height = self.width, self.height
        f.bit_depth, f.ss_x, f.ss_y, f.mono = self.bit_depth, self.ss_x, self.ss_y, self.mono
        f.memory = memory
        for i, p in enumerate(self.planes):
            f.plane[i].data = ptrs[i] if ptrs is not None else p.ctypes.data
            f.plane[i].stride = p.strides[0]
            f.plane[i].width, f.plane[i].height = self.crop[i]
            f.plane[i].alloc_height, f.plane[i].alloc_width = p.shape
        return f

    @property
    def luma_pixels(self):
        return self.width * self.height

    def nbytes(self):
        return sum(p.nbytes for p in self.planes)


@dataclass
class SideInfo:
    """Side information arrays plus the pf_frame_side struct pointing at them.

    Picklable (for process pools): the struct travels as bytes with each
    pointer recorded as an index into `keep`, and is re-pointed on arrival."""

    side: abi.pf_frame_side
    keep: list = field(default_factory=list)  # arrays the struct points into
    blocks: dict = field(default_factory=dict)  # generator bookkeeping

    _PTRS = (("lf", "masks"), ("lf", "level_cache"), ("cdef", "index"), ("cdef", "read"), ("cdef", "noskip"))

    def __getstate__(self):
        addrs = [k.ctypes.data if isinstance(k, np.ndarray) else C.addressof(k) for k in self.keep]

        def find(a):
            if not a:
                return None
            if a not in addrs:
                raise ValueError("pf_frame_side points outside its kept arrays")
            return addrs.index(a)

        ptrs = {"%s.%s" % sf: find(getattr(getattr(self.side, sf[0]), sf[1])) for sf in self._PTRS}
        for p in range(3):
            ptrs["lr.units.%d" % p] = find(self.side.lr.units[p])
        keep = [k if isinstance(k, np.ndarray) else (type(k)._type_, type(k)._length_, bytes(k)) for k in self.keep]
        return {"side": bytes(self.side), "ptrs": ptrs, "keep": keep, "blocks": self.blocks}

    def __setstate__(self, st):
        self.keep = [k if isinstance(k, np.ndarray) else (k[0] * k[1]).from_buffer_copy(k[2]) for k in st["keep"]]
        self.blocks = st["blocks"]
        self.side = abi.pf_frame_side.from_buffer_copy(st["side"])

        def addr(i):
            if i is None:
                return None
            k = self.keep[i]
            return k.ctypes.data if isinstance(k, np.ndarray) else C.addressof(k)

        for s, f in self._PTRS:
            setattr(getattr(self.side, s), f, addr(st["ptrs"]["%s.%s" % (s, f)]))
        for p in range(3):
            self.side.lr.units[p] = addr(st["ptrs"]["lr.units.%d" % p])


# ---------------------------------------------------------------------------
# Content


def gen_content(rng, frame, noise_sigma, dc_range, mv=(0, 0), params=None):
    """Cosine-gradient texture + per-8x8 DC offsets + Gaussian noise, clipped.

    params (periods/phases/amplitudes) can be passed so a sequence shares one
    texture translated by a per-frame motion vector."""
    maxv = (1 << frame.bit_depth) - 1
    scale = 1 << (frame.bit_depth - 8)
    if params is None:
        params = []
        for _ in range(3):
            params.append(dict(
                px=rng.uniform(8, 64), py=rng.uniform(8, 64),
                qx=rng.uniform(8, 64), qy=rng.uniform(8, 64),
                fx=rng.uniform(0, 2 * np.pi), fy=rng.uniform(0, 2 * np.pi),
                a=rng.uniform(20, 60), b=rng.uniform(10, 40), c=rng.uniform(10, 30)))
    for i, p in enumerate(frame.planes):
        h, w = p.shape
        sx = frame.ss_x if i else 0
        sy = frame.ss_y if i else 0
        pr = params[i]
        ys = (np.arange(h, dtype=np.float64) + (mv[1] >> sy))[:, None]
        xs = (np.arange(w, dtype=np.float64) + (mv[0] >> sx))[None, :]
        tex = (128 + pr["a"] * np.cos(2 * np.pi * xs / pr["px"] + pr["fx"])
               + pr["b"] * np.cos(2 * np.pi * ys / pr["py"] + pr["fy"])
               + pr["c"] * np.cos(2 * np.pi * xs / pr["qx"]) * np.cos(2 * np.pi * ys / pr["qy"]))
        tex = tex * scale
        dc = rng.integers(-dc_range, dc_range + 1, size=((h + 7) // 8, (w + 7) // 8))
        tex = tex + np.repeat(np.repeat(dc, 8, 0), 8, 1)[:h, :w]
        if noise_sigma:
            tex = tex + rng.normal(0.0, noise_sigma, size=(h, w))
        p[:] = np.clip(np.rint(tex), 0, maxv).astype(p.dtype)
    return params


# ---------------------------------------------------------------------------
# Block / transform layout


def aligned_blocks(rng, mi_cols, mi_rows, sizes=(1, 2, 4, 8)):
    """Config-0 layout: per aligned 32x32 region one square size from
    {4,8,16,32} px; transform = block.  Returns a list of (x4, y4, s4)."""
    blocks = []
    for y4 in range(0, mi_rows, 8):
        for x4 in range(0, mi_cols, 8):
            s4 = int(rng.choice(sizes))
            for yy in range(y4, min(y4 + 8, mi_rows), s4):
                for xx in range(x4, min(x4 + 8, mi_cols), s4):
                    blocks.append((xx, yy, s4, s4))
    return blocks


def quadtree_blocks(rng, mi_cols, mi_rows, split_p=0.55):
    """Config-1 layout: a random quadtree over 64x64 superblocks down to 4x4.
    Returns (x4, y4, block s4, tx s4) with tx <= block (and <= 32 px)."""
    blocks = []

    def rec(x4, y4, s4):
        if x4 >= mi_cols or y4 >= mi_rows:
            return
        if s4 > 1 and rng.random() < split_p:
            h = s4 // 2
            for dy in (0, h):
                for dx in (0, h):
                    rec(x4 + dx, y4 + dy, h)
            return
        tmax = min(s4, 8)
        choices = [t for t in (1, 2, 4, 8) if t <= tmax]
        blocks.append((x4, y4, s4, int(rng.choice(choices))))

    for y4 in range(0, mi_rows, 16):
        for x4 in range(0, mi_cols, 16):
            rec(x4, y4, 16)
    return blocks


def _class_luma(t4):
    return np.minimum(np.log2(t4).astype(np.int32), 2)


def build_lf_masks(frame, blocks, mi_cols, mi_rows):
    """Deblocking edge masks in lfmask.FilterMask layout (lfmask/mask.go:25-41).

    An edge sits on every transform boundary (every block is coded intra, so
    inner transform edges are filtered); its width class is the smaller of
    the transform classes on its two sides (the rule dav1d's
    mask_edges_intra/chroma carries through its a[]/l[] context arrays,
    lfmask/mask.go:334-430)."""
    sb128_w = (mi_cols + 31) // 32
    sb128_h = (mi_rows + 31) // 32
    masks = np.zeros((sb128_h * sb128_w, abi.PF_LF_MASK_WORDS), np.uint16)
    # Luma transform grid: tx size (4-px units) and tx origin per cell.
    owner = _owner_grid(blocks, mi_cols, mi_rows)
    barr = np.asarray(blocks, np.int32).reshape(-1, 4)
    b0x, b0y, bsz, txs = (barr[owner, k] for k in range(4))
    gy, gx = np.mgrid[0:mi_rows, 0:mi_cols]
    tx0x = b0x + ((gx - b0x) // txs) * txs
    tx0y = b0y + ((gy - b0y) // txs) * txs

    def put(region_idx, word_idx, bit):
        np.bitwise_or.at(masks, (region_idx, word_idx), (1 << bit).astype(np.uint16))

    cls = _class_luma(txs)
    # vertical edges (dir 0): left side of a tx, x4 > 0
    sel = (tx0x == gx) & (gx > 0)
    y, x = gy[sel], gx[sel]
    k = np.minimum(cls[y, x], cls[y, x - 1])
    reg = (y // 32) * sb128_w + (x // 32)
    pos, b = x & 31, y & 31
    put(reg, ((0 * 32 + pos) * 3 + k) * 2 + (b >> 4), b & 15)
    sel = (tx0y == gy) & (gy > 0)
    y, x = gy[sel], gx[sel]
    k = np.minimum(cls[y, x], cls[y - 1, x])
    reg = (y // 32) * sb128_w + (x // 32)
    pos, b = y & 31, x & 31
    put(reg, ((1 * 32 + pos) * 3 + k) * 2 + (b >> 4), b & 15)

    # Chroma: a block of s4 luma cells owns a chroma transform of
    # max(1, s4 >> ss) chroma cells (at most 8), aligned to its own size.
    ssx, ssy = frame.ss_x, frame.ss_y
    cc, cr = (mi_cols + ssx) >> ssx, (mi_rows + ssy) >> ssy
    cgy, cgx = np.mgrid[0:cr, 0:cc]
    ly = np.minimum(cgy << ssy, mi_rows - 1)
    lx = np.minimum(cgx << ssx, mi_cols - 1)
    cts = np.clip(np.minimum(bsz[ly, lx] >> ssx, bsz[ly, lx] >> ssy), 1, 8)
    ct0x = (cgx // cts) * cts
    ct0y = (cgy // cts) * cts
    ccls = (cts >= 2).astype(np.int32)
    rw, rh = 32 >> ssx, 32 >> ssy
    lane_v, lane_h = 16 >> ssy, 16 >> ssx
    sel = (ct0x == cgx) & (cgx > 0)
    y, x = cgy[sel], cgx[sel]
    k = np.minimum(ccls[y, x], ccls[y, x - 1])
    reg = (y // rh) * sb128_w + (x // rw)
    pos, b = x % rw, y % rh
    put(reg, 384 + ((0 * 32 + pos) * 2 + k) * 2 + b // lane_v, b % lane_v)
    sel = (ct0y == cgy) & (cgy > 0)
    y, x = cgy[sel], cgx[sel]
    k = np.minimum(ccls[y, x], ccls[y - 1, x])
    reg = (y // rh) * sb128_w + (x // rw)
    pos, b = y % rh, x % rw
    put(reg, 384 + ((1 * 32 + pos) * 2 + k) * 2 + b // lane_h, b % lane_h)
    return masks, sb128_w, sb128_h, (b0x, b0y)


def calc_lf_values(level_y, level_u, level_v, seg_deltas):
    """dav1d_calc_lf_values without delta_lf / mode-ref deltas
    (lfmask/values.go:59-119): levels[seg] = (YV, YH, U, V)."""
    out = []
    for sd in seg_deltas:
        lv = []
        for base, d in zip((level_y[0], level_y[1], level_u, level_v), sd):
            if level_y[0] == 0 and level_y[1] == 0:
                lv.append(0)
                continue
            if base == 0 and len(lv) >= 2:  # chroma with zero base
                lv.append(0)
                continue
            lv.append(int(np.clip(np.clip(base, 0, 63) + d, 0, 63)))
        out.append(lv)
    return out


def _owner_grid(blocks, mi_cols, mi_rows):
    owner = np.zeros((mi_rows, mi_cols), np.int32)
    for bi, (x4, y4, s4, _t4) in enumerate(blocks):
        owner[y4:y4 + s4, x4:x4 + s4] = bi
    return owner


def build_level_cache(frame, blocks, mi_cols, mi_rows, seg_of_block, seg_levels):
    """Level cache: 4 bytes per MI cell [YV, YH, U, V]; chroma cells at chroma
    coordinates with the luma stride (postfilter_loopfilter_masks.go:135-228)."""
    lc = np.zeros((mi_rows, mi_cols, 4), np.uint8)
    ssx, ssy = frame.ss_x, frame.ss_y
    owner = _owner_grid(blocks, mi_cols, mi_rows)
    lv = np.asarray(seg_levels, np.uint8)[np.asarray(seg_of_block)]  # [nblocks, 4]
    lc[:, :, 0] = lv[owner, 0]
    lc[:, :, 1] = lv[owner, 1]
    cc, cr = (mi_cols + ssx) >> ssx, (mi_rows + ssy) >> ssy
    cy = np.minimum(np.arange(cr) << ssy, mi_rows - 1)
    cx = np.minimum(np.arange(cc) << ssx, mi_cols - 1)
    co = owner[np.ix_(cy, cx)]
    lc[:cr, :cc, 2] = lv[co, 2]
    lc[:cr, :cc, 3] = lv[co, 3]
    return lc


def build_noskip(blocks, skip, mi_cols, mi_rows):
    """CDEF noskip words (threading/loop_filter_noskip.go:27-71): 8 bytes per
    64x64 unit, bit by*8+bx set when the 8x8 block carries residual; bits of
    blocks outside the frame are preset."""
    ucols, urows = (mi_cols + 15) >> 4, (mi_rows + 15) >> 4
    owner = _owner_grid(blocks, mi_cols, mi_rows)
    coded = ~np.asarray(skip, bool)[owner]  # per 4x4 cell
    c8 = np.zeros((urows * 8, ucols * 8), bool)
    r8, k8 = (mi_rows + 1) >> 1, (mi_cols + 1) >> 1
    pad = np.zeros((r8 * 2, k8 * 2), bool)
    pad[:mi_rows, :mi_cols] = coded
    c8[:r8, :k8] = pad.reshape(r8, 2, k8, 2).any(axis=(1, 3))
    valid_c, valid_r = mi_cols >> 1, mi_rows >> 1
    c8[:, valid_c:] = True
    c8[valid_r:, :] = True
    bits = c8.reshape(urows, 8, ucols, 8).transpose(0, 2, 1, 3)  # [ur, uc, by, bx]
    ns = np.packbits(bits, axis=-1, bitorder="little")[..., 0]
    return np.ascontiguousarray(ns.astype(np.uint8))


# ---------------------------------------------------------------------------
# Workload builders


def _pack_cdef(pri, sec):
    code = {0: 0, 1: 1, 2: 2, 4: 3}[sec]
    return (pri << 2) | code


def make_frame(config, seed, frame_index=0, texture=None, width=None, height=None,
               bit_depth=None, ss=None, stages=abi.PF_STAGES_ALL):
    """Builds (HostFrame, SideInfo) for a workload configuration.

    config 0: 352x288 8-bit 4:2:0, deblock + CDEF (aligned square blocks).
    config 1: 1920x1080 8-bit 4:2:0 full chain (quadtree, segments, LR, FG).
    config 2: 3840x2160 10-bit 4:2:0 full chain.
    Sizes / depth / subsampling can be overridden (the batched mix)."""
    rng = np.random.default_rng([seed, frame_index])
    if config == 0:
        W, H, bd, (ssx, ssy) = 352, 288, 8, (1, 1)
    elif config == 1:
        W, H, bd, (ssx, ssy) = 1920, 1080, 8, (1, 1)
    elif config == 2:
        W, H, bd, (ssx, ssy) = 3840, 2160, 10, (1, 1)
    else:
        raise ValueError(config)
    W = width or W
    H = height or H
    bd = bit_depth or bd
    if ss is not None:
        ssx, ssy = ss
    fr = HostFrame.alloc(W, H, bd, ssx, ssy)
    mi_cols, mi_rows = ((W + 7) >> 3) << 1, ((H + 7) >> 3) << 1
    if config == 0:
        gen_content(rng, fr, 4.0, 12)
        blocks = aligned_blocks(rng, mi_cols, mi_rows)
        nseg = 1
    else:
        scale = 1 << (bd - 8)
        mv = (int(rng.integers(-8, 9)) * (frame_index + 1), int(rng.integers(-8, 9)) * (frame_index + 1))
        tex_rng = np.random.default_rng([seed, 0xC0DE])
        params = texture or None
        if params is None:
            params = gen_content(tex_rng, fr.like(), 0, 0)
        gen_content(rng, fr, 4.0 * scale if bd == 8 else 16.0, 12 * scale if bd == 8 else 48, mv=mv, params=params)
        blocks = quadtree_blocks(rng, mi_cols, mi_rows)
        nseg = 8
    nb = len(blocks)
    skip = rng.random(nb) < 0.3
    seg_of_block = rng.integers(0, nseg, size=nb)

    side = abi.pf_frame_side()
    side.stages = stages
    keep = []

    # Deblocking.
    lvl = [int(v) for v in rng.integers(0, 64, size=4)]
    lf = side.lf
    lf.level_y[0], lf.level_y[1], lf.level_u, lf.level_v = lvl
    lf.sharpness = 0
    seg_deltas = [[0, 0, 0, 0]] if nseg == 1 else [list(rng.integers(-15, 16, size=4)) for _ in range(nseg)]
    seg_levels = calc_lf_values(lvl[0:2], lvl[2], lvl[3], seg_deltas)
    masks, sw, sh, _ = build_lf_masks(fr, blocks, mi_cols, mi_rows)
    lc = build_level_cache(fr, blocks, mi_cols, mi_rows, seg_of_block, seg_levels)
    keep += [masks, lc]
    lf.masks, lf.sb128_w, lf.sb128_h = masks.ctypes.data, sw, sh
    lf.level_cache, lf.mi_cols, lf.mi_rows = lc.ctypes.data, mi_cols, mi_rows

    # CDEF.
    cd = side.cdef
    ucols, urows = (W + 63) // 64, (H + 63) // 64
    if config == 0:
        cd.bits, cd.damping = 2, 3
    else:
        cd.bits, cd.damping = 3, int(rng.integers(3, 7))
    cd.strength_count = 1 << cd.bits
    for i in range(cd.strength_count):
        cd.y_strength[i] = _pack_cdef(int(rng.integers(0, 16)), int(rng.choice([0, 1, 2, 4])))
        cd.uv_strength[i] = _pack_cdef(int(rng.integers(0, 16)), int(rng.choice([0, 1, 2, 4])))
    noskip = build_noskip(blocks, skip, mi_cols, mi_rows)
    index = rng.integers(0, cd.strength_count, size=(urows, ucols)).astype(np.uint8)
    # Read=false for units whose in-frame 8x8 blocks are all skip.
    bits = np.unpackbits(noskip, axis=-1, bitorder="little").astype(bool).reshape(urows, ucols, 8, 8)
    gy = np.arange(urows)[:, None, None, None] * 8 + np.arange(8)[None, None, :, None]
    gx = np.arange(ucols)[None, :, None, None] * 8 + np.arange(8)[None, None, None, :]
    inside = (gy < (mi_rows >> 1)) & (gx < (mi_cols >> 1))
    read = (bits & inside).any(axis=(2, 3)).astype(np.uint8)
    keep += [noskip, index, read]
    cd.index, cd.read = index.ctypes.data, read.ctypes.data
    cd.index_stride, cd.index_rows = ucols, urows
    cd.noskip = noskip.ctypes.data

    # Loop restoration.
    lr = side.lr
    if config == 0:
        lr.type[0] = lr.type[1] = lr.type[2] = abi.PF_LR_NONE
        side.stages &= ~abi.PF_STAGE_LOOP_RESTORATION
    else:
        lr.unit_size_y = 128 if config == 1 else 256
        lr.unit_size_uv = 64 if config == 1 else 128
        for p in range(3):
            lr.type[p] = abi.PF_LR_SWITCHABLE
            us = lr.unit_size_y if p == 0 else lr.unit_size_uv
            pw, ph = fr.crop[p]
            hz = max(1, (pw + us // 2) // us)
            vt = max(1, (ph + us // 2) // us)
            units = (abi.pf_lr_unit * (hz * vt))()
            for i in range(hz * vt):
                u = units[i]
                u.type = [abi.PF_LR_NONE, abi.PF_LR_WIENER, abi.PF_LR_SGRPROJ][int(rng.integers(0, 3))]
                t0 = 0 if p else int(rng.integers(-5, 11))
                u.wiener_v[0], u.wiener_v[1], u.wiener_v[2] = t0, int(rng.integers(-23, 9)), int(rng.integers(-17, 47))
                t0 = 0 if p else int(rng.integers(-5, 11))
                u.wiener_h[0], u.wiener_h[1], u.wiener_h[2] = t0, int(rng.integers(-23, 9)), int(rng.integers(-17, 47))
                u.sgr_set = int(rng.integers(0, 16))
                u.sgr_xqd[0], u.sgr_xqd[1] = int(rng.integers(-96, 32)), int(rng.integers(-32, 96))
            keep.append(units)
            lr.units[p] = C.addressof(units)
            lr.unit_count[p] = hz * vt

    # Film grain.
    fg = side.fg
    if config == 0:
        side.stages &= ~abi.PF_STAGE_FILM_GRAIN
    else:
        fg.apply = 1
        fg.seed = int(rng.integers(0, 65536))
        fg.num_y_points = 14
        xs = np.sort(rng.choice(256, size=14, replace=False))
        for i in range(14):
            fg.y_points[i][0], fg.y_points[i][1] = int(xs[i]), int(rng.integers(0, 256))
        fg.chroma_scaling_from_luma = 0
        for pts, name in ((fg.cb_points, "num_cb_points"), (fg.cr_points, "num_cr_points")):
            xs = np.sort(rng.choice(256, size=10, replace=False))
            for i in range(10):
                pts[i][0], pts[i][1] = int(xs[i]), int(rng.integers(0, 256))
            setattr(fg, name, 10)
        fg.scaling_shift = 11 if config == 2 else int(rng.integers(8, 12))
        fg.ar_coeff_lag = 3
        for i in range(24):
            fg.ar_coeffs_y[i] = int(rng.integers(-128, 128))
        for i in range(25):
            fg.ar_coeffs_cb[i] = int(rng.integers(-128, 128))
            fg.ar_coeffs_cr[i] = int(rng.integers(-128, 128))
        fg.ar_coeff_shift = int(rng.integers(6, 10))
        fg.grain_scale_shift = 0
        fg.cb_mult, fg.cb_luma_mult, fg.cb_offset = int(rng.integers(0, 256)), int(rng.integers(0, 256)), int(rng.integers(0, 512))
        fg.cr_mult, fg.cr_luma_mult, fg.cr_offset = int(rng.integers(0, 256)), int(rng.integers(0, 256)), int(rng.integers(0, 512))
        fg.overlap = 1
        fg.clip_to_restricted_range = 0
        fg.matrix_identity = 0

    si = SideInfo(side=side, keep=keep, blocks=dict(blocks=blocks, skip=skip))
    return fr, si


def make_search_pair(seed, width=1920, height=1080, sigma=None):
    """CDEF-search workload (8-bit 4:2:0): the source is the cosine-gradient
    texture without noise; the reconstruction adds per-8x8 DC offsets in
    +/-12 and Gaussian noise with sigma drawn from {2, 4, 8}.  Returns
    (source, recon, side) where side is config-1 style side information for
    the same frame (its loop-filter part deblocks the reconstruction and its
    noskip words drive the search's block lists)."""
    rng = np.random.default_rng([seed, 0x5EA2C4])
    src = HostFrame.alloc(width, height, 8)
    params = gen_content(rng, src, 0.0, 0)
    rec = HostFrame.alloc(width, height, 8)
    sig = float(sigma if sigma is not None else rng.choice([2.0, 4.0, 8.0]))
    gen_content(rng, rec, sig, 12, params=params)
    _, side = make_frame(1, seed, width=width, height=height, stages=abi.PF_STAGE_LOOP_FILTER)
    return src, rec, side, sig


def make_lr_search_pair(seed, width=1920, height=1080, sigma=None):
    """Loop-restoration search workload (8-bit 4:2:0, luma searched): the
    source is the cosine-gradient texture; the reconstruction adds per-8x8
    DC offsets in +/-6 and Gaussian noise (sigma from {2, 4, 8}).  About one
    luma restoration unit in eight is made dark in the source (0..3) with
    the reconstruction 16..40 above it, the content on which the reference's
    horizontal-only Wiener scoring (taps without the centre's 128) can win,
    and about one in sixteen is reconstructed exactly (zero unfiltered SSE).
    Returns (source, recon, sigma)."""
    rng = np.random.default_rng([seed, 0x1E57A9])
    src = HostFrame.alloc(width, height, 8)
    params = gen_content(rng, src, 0.0, 0)
    rec = HostFrame.alloc(width, height, 8)
    sig = float(sigma if sigma is not None else rng.choice([2.0, 4.0, 8.0]))
    gen_content(rng, rec, sig, 6, params=params)
    horz, vert = abi.lr_unit_grid(width, height)
    for row in range(vert):
        for col in range(horz):
            x0, x1 = col * 64, (width if col + 1 == horz else col * 64 + 64)
            y0, y1 = row * 64, (height if row + 1 == vert else row * 64 + 64)
            y0 -= 8 if y0 > 0 else 0
            y1 -= 8 if y1 < height else 0
            s = src.planes[0][y0:y1, x0:x1]
            r = rec.planes[0][y0:y1, x0:x1]
            u = rng.random()
            if u < 0.125:
                s[:] = rng.integers(0, 4, size=s.shape)
                r[:] = np.clip(s.astype(np.int32) + rng.integers(16, 41, size=s.shape), 0, 255)
            elif u < 0.1875:
                r[:] = s
    return src, rec, sig


# ---------------------------------------------------------------------------
# Block record maps (threading.FrameWorkLoopFilterMap)

_TABLES = None


def av1_tables():
    """(block_dims[22][2], tx_dims[19][5], max_tx[22][4]) from the generated
    pf_tables.h: goav1's tile.BlockSize / TransformSize tables."""
    global _TABLES
    if _TABLES is None:
        import os
        import re

        text = open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc", "pf_tables.h")).read()

        def grab(name, cols):
            body = re.search(name + r"\[[^\]]*\]\[\d+\] = \{(.*?)\n\};", text, re.S).group(1)
            vals = [int(v) for v in re.findall(r"\d+", body)]
            return [tuple(vals[i:i + cols]) for i in range(0, len(vals), cols)]

        _TABLES = (grab("pf_block_dims", 2), grab("pf_tx_dims", 5), grab("pf_max_tx", 4))
    return _TABLES


# AV1 partitions of a square block of n 4x4 units, as (x, y, w, h) children
# in decode order; "split" recurses into the four quadrants.
def _partition_children(kind, n):
    h = n // 2
    q = n // 4
    return {
        "none": [(0, 0, n, n)],
        "horz": [(0, 0, n, h), (0, h, n, h)],
        "vert": [(0, 0, h, n), (h, 0, h, n)],
        "horz_a": [(0, 0, h, h), (h, 0, h, h), (0, h, n, h)],
        "horz_b": [(0, 0, n, h), (0, h, h, h), (h, h, h, h)],
        "vert_a": [(0, 0, h, h), (0, h, h, h), (h, 0, h, n)],
        "vert_b": [(0, 0, h, n), (h, 0, h, h), (h, h, h, h)],
        "horz_4": [(0, i * q, n, q) for i in range(4)],
        "vert_4": [(i * q, 0, q, n) for i in range(4)],
    }[kind]


def make_lf_map(seed, mi_cols, mi_rows, ss=(1, 1), mono=False, sb128=True, p_intra=0.3, p_skip=0.3, p_split=0.5,
                p_vartx=0.6):
    """A decoded block record map (threading.FrameWorkLoopFilterMap,
    threading/loop_filter_map.go:46-72) for an mi_cols x mi_rows grid: each
    64x64 or 128x128 superblock partitioned at random with AV1's partition
    types (frame-edge blocks forced to split or halve as AV1 does), each
    block intra (transform size reduced 0-2 steps) or inter (skip, or a
    random var-tx split tree), its chroma transform the largest for the
    layout (tile/tx_size.go:109-132), random segment, reference frame, mode
    class and delta-lf values.  Returns (records[mi_rows, mi_cols] of
    abi.lf_record_dtype(), decode-order origin cell indices)."""
    bdims, txd, maxtx = av1_tables()
    size_of = {d: i for i, d in enumerate(bdims)}
    layout_col = 3 if ss[0] == 0 else (1 if ss[1] else 2)
    rng = np.random.default_rng([seed, mi_cols, mi_rows, 0x1F3A])
    rec = np.zeros((mi_rows, mi_cols), abi.lf_record_dtype())
    order = []

    def emit(x, y, w, h):
        if x >= mi_cols or y >= mi_rows:
            return
        bs = size_of[(w, h)]
        intra = rng.random() < p_intra
        skip = (not intra) and rng.random() < p_skip
        tx = maxtx[bs][0]
        split = (0, 0)
        if intra:
            for _ in range(int(rng.integers(0, 3))):
                tx = txd[tx][4] if tx else tx
        elif not skip and tx and rng.random() < p_vartx:
            split = (int(rng.integers(1, 1 << 16)), int(rng.integers(0, 1 << 16)))
        x1, y1 = min(x + w, mi_cols), min(y + h, mi_rows)
        r = rec[y:y1, x:x1]
        r["mi_col"], r["mi_row"], r["mi_col_end"], r["mi_row_end"] = x, y, x1, y1
        r["block_size"], r["valid"], r["intra"], r["skip"] = bs, 1, intra, skip
        r["tx_y"], r["tx_uv"], r["has_uv"] = tx, maxtx[bs][layout_col], 0 if mono else 1
        r["segment_id"] = rng.integers(0, 8)
        r["ref_frame"] = 0 if intra else rng.integers(1, 8)
        r["mode"] = 0 if intra else rng.integers(0, 2)
        r["delta_lf_from_base"] = rng.integers(-12, 13)
        r["delta_lf"] = rng.integers(-12, 13, size=4)
        r["tx_split"] = split
        order.append(y * mi_cols + x)

    def part(x, y, n):
        if x >= mi_cols or y >= mi_rows:
            return
        has_rows, has_cols = y + n // 2 < mi_rows, x + n // 2 < mi_cols
        if n == 1:
            emit(x, y, 1, 1)
            return
        if has_rows and has_cols:
            kinds = ["none", "horz", "vert", "split"]
            if n > 2:
                kinds += ["horz_a", "horz_b", "vert_a", "vert_b"]
            if 2 < n < 32:
                kinds += ["horz_4", "vert_4"]
            kind = "split" if rng.random() < p_split and n > 2 else kinds[int(rng.integers(0, len(kinds)))]
        elif has_cols:
            kind = "horz" if rng.random() < 0.5 and n > 2 else "split"
        elif has_rows:
            kind = "vert" if rng.random() < 0.5 and n > 2 else "split"
        else:
            kind = "split"
        if kind == "split":
            h = n // 2
            for dy in (0, h):
                for dx in (0, h):
                    part(x + dx, y + dy, h)
            return
        for cx, cy, w, hh in _partition_children(kind, n):
            emit(x + cx, y + cy, w, hh)

    sb = 32 if sb128 else 16
    for y in range(0, mi_rows, sb):
        for x in range(0, mi_cols, sb):
            part(x, y, sb)
    return rec, np.array(order, np.int32)


def make_lf_levels(seed, mode="plain"):
    """pf_lf_levels: "plain" (frame levels only), "deltas" (segmentation,
    delta_lf multi and mode/ref deltas on), "single" (delta_lf single),
    "zero" (both luma levels 0)."""
    rng = np.random.default_rng([seed, 0x1E7E])
    lv = abi.pf_lf_levels()
    lv.level_y[0], lv.level_y[1] = int(rng.integers(1, 64)), int(rng.integers(1, 64))
    lv.level_u, lv.level_v = int(rng.integers(0, 64)), int(rng.integers(0, 64))
    if mode == "zero":
        lv.level_y[0] = lv.level_y[1] = 0
    if mode in ("deltas", "single"):
        lv.delta_lf_present = 1
        lv.delta_lf_multi = 1 if mode == "deltas" else 0
        lv.segmentation_enabled = 1
        lv.mode_ref_delta_enabled = 1
        for i in range(8):
            lv.ref_delta[i] = int(rng.integers(-20, 21))
            for k in range(4):
                lv.segment_delta[i][k] = int(rng.integers(-20, 21))
        lv.mode_delta[0], lv.mode_delta[1] = int(rng.integers(-20, 21)), int(rng.integers(-20, 21))
    return lv
