// pf_lfmask.cu - deblocking edge masks and level cache built on the GPU from
// goav1's block record map.
//
// FrameWorkLoopFilterMasks.BuildFromMap (internal/av1/threading/
// loop_filter_masks.go:450-680) walks the block origins of the record map and
// ORs each block's edges into the lfmask.FilterMask of its 128x128 region:
// the left/above edge of a block takes the minimum of the block's own
// transform class and the class the neighbouring block carries out of its
// right column / bottom row (read from the map, 2 luma / 1 chroma when there
// is none); inner transform edges of intra and non-skip inter blocks take the
// minimum of the two transforms either side (lfmask/mask.go:110-400).  That
// rule depends only on the cells either side of an edge, so here each 4x4
// cell decides its own edges: one CTA per 128x128 region and a thread per
// cell.  A warp is one column of cells for the vertical edges and, after a
// transpose through shared memory, one row for the horizontal edges; each
// strength lane of the mask is then one warp ballot, so every mask word is
// written once, without atomics.
//
// The level cache (populateLoopFilterLevelCacheFromMap,
// decoder/postfilter_loopfilter_masks.go:119-228) is per cell too: the luma
// bytes are the cell's own block's levels, the chroma bytes those of the
// block that comes last in raster order of origin among the blocks covering
// the chroma cell (the reference's walk writes them in that order).
//
// The errors the reference returns come from its level-cache walk, which
// visits cells in a chain per MI row (an invalid cell steps one cell, a
// valid one jumps to its MIColEnd).  k_lf_build's row CTAs find that chain
// for each row by pointer doubling in shared memory and keep its first
// error; the host takes the first row's.
#include <limits.h>
#include <string.h>

#include "pf_common.cuh"
#include "pf_tables.h"

namespace pf {

constexpr int kLfBatch = 1, kLfFilter = 2;  // error kinds: INVALID_BATCH, INVALID_FILTER

struct MapTables {
  uint8_t block[22][2];  // W4, H4
  uint8_t tx[19][5];     // W4, H4, Log2W, Log2H, Sub
};

struct MapArgs {
  const uint4* rec;  // 32-byte records, two uint4 each
  uint16_t* masks;
  uint32_t* levels;  // one 4-byte level cell per MI cell
  unsigned long long* rowErr;  // per MI row: first error (cell << 8 | kind) or all ones
  int cols, rows, sbw, regions, ssx, ssy, mono, ccols, crows;
  // ResolveBlockLevels inputs (loopfilter/level.go:86-118)
  uint8_t base[3][2];
  uint8_t lumaZero, deltaPresent, deltaMulti, segEnabled, modeRef;
  int8_t refDelta[8], modeDelta[2];
  int16_t segDelta[8][4];
  MapTables t;
};

// One decoded record (pf_lf_record, 32 bytes).
struct LfRec {
  uint32_t w[8];
  __device__ int col() const { return w[0] & 0xffff; }
  __device__ int row() const { return w[0] >> 16; }
  __device__ int colEnd() const { return w[1] & 0xffff; }
  __device__ int bs() const { return w[2] & 0xff; }
  __device__ bool valid() const { return (w[2] >> 8) & 0xff; }
  __device__ bool intra() const { return (w[2] >> 16) & 0xff; }
  __device__ bool skip() const { return w[2] >> 24; }
  __device__ int txy() const { return w[3] & 0xff; }
  __device__ int txuv() const { return (w[3] >> 8) & 0xff; }
  __device__ bool hasUV() const { return (w[3] >> 16) & 0xff; }
  __device__ int seg() const { return w[3] >> 24; }
  __device__ int ref() const { return w[4] & 0xff; }
  __device__ int mode() const { return (w[4] >> 8) & 0xff; }
  __device__ int deltaFromBase() const { return (int8_t)(w[4] >> 16); }
  __device__ int deltaMulti(int i) const {
    return i == 0 ? (int8_t)(w[4] >> 24) : (int8_t)(w[5] >> (8 * (i - 1)));
  }
  __device__ uint32_t split() const { return w[6]; }  // depth-0 bits low, depth-1 bits high
};

__device__ __forceinline__ LfRec load_rec(const MapArgs& a, int x, int y) {
  const uint4* p = a.rec + 2 * ((size_t)y * a.cols + x);
  const uint4 u = __ldg(p), v = __ldg(p + 1);
  LfRec r;
  r.w[0] = u.x, r.w[1] = u.y, r.w[2] = u.z, r.w[3] = u.w;
  r.w[4] = v.x, r.w[5] = v.y, r.w[6] = v.z, r.w[7] = v.w;
  return r;
}

// The transform leaf covering block-local cell (lx, ly) of a block whose root
// transform is `tx`, tiled from the block origin (decomp_tx,
// lfmask/mask.go:63-98; the split bits of depth 0 and 1 are indexed by the
// node's position yOff*4+xOff in the tree, a shift past 15 reading 0).
// Returns the leaf's clamped width and height classes (min(log2, 2)) and
// whether the cell is in the leaf's first column / first row.
struct Leaf {
  int cw, ch;
  bool left, top;
};

__device__ __forceinline__ Leaf tx_leaf(const MapTables& t, int tx, bool uniform, uint32_t split, int lx, int ly) {
  int lw = t.tx[tx][2], lh = t.tx[tx][3];
  int xo = lx >> lw, yo = ly >> lh;
  int xb = xo << lw, yb = yo << lh;
  if (!uniform) {
#pragma unroll
    for (int depth = 0; depth < 2; depth++) {
      const int sh = yo * 4 + xo;
      const uint32_t bits = depth ? split >> 16 : split & 0xffff;
      if (tx == 0 || sh >= 16 || !((bits >> sh) & 1)) break;
      const int w4 = 1 << lw, h4 = 1 << lh;
      const int cx = (w4 >= h4 && lx - xb >= (w4 >> 1)) ? 1 : 0;
      const int cy = (h4 >= w4 && ly - yb >= (h4 >> 1)) ? 1 : 0;
      xb += cx * (w4 >> 1);
      yb += cy * (h4 >> 1);
      xo = xo * 2 + cx;
      yo = yo * 2 + cy;
      tx = t.tx[tx][4];
      lw = t.tx[tx][2];
      lh = t.tx[tx][3];
    }
  }
  Leaf L;
  L.cw = lw < 2 ? lw : 2;
  L.ch = lh < 2 ? lh : 2;
  L.left = lx == xb;
  L.top = ly == yb;
  return L;
}

__device__ __forceinline__ int safe_tx(int tx) { return tx < 19 ? tx : 0; }

// A record's luma transform layout: intra blocks and inter blocks without
// depth-0 split bits use the root transform throughout (mask.go:113-118,
// build.go:104-111).
__device__ __forceinline__ bool uniform_tx(const LfRec& r) { return r.intra() || (r.split() & 0xffff) == 0; }

// The head of a record (words 0-3: origin, extent, size and flags,
// transforms and segment) and, when asked, its split word: what the edge
// rules read of a neighbouring cell.
__device__ __forceinline__ LfRec load_head(const MapArgs& a, int x, int y, bool split) {
  const uint4* p = a.rec + 2 * ((size_t)y * a.cols + x);
  const uint4 u = __ldg(p);
  LfRec r;
  r.w[0] = u.x, r.w[1] = u.y, r.w[2] = u.z, r.w[3] = u.w;
  r.w[4] = r.w[5] = r.w[7] = 0;
  r.w[6] = split ? __ldg((const uint32_t*)(p + 1) + 2) : 0;
  return r;
}

// The class a neighbouring block carries out of its right column (vertical)
// or bottom row (horizontal), read at map cell (x, y) whose record is `r`
// (fillLeftLumaContext / fillAboveLumaContext, loop_filter_masks.go:553-646):
// 2 when the cell holds no valid block.
__device__ int luma_edge_ctx(const MapArgs& a, const LfRec& r, int x, int y, bool vertical) {
  if (!r.valid() || r.bs() >= 22) return 2;
  const int nbw = min(a.cols - r.col(), (int)a.t.block[r.bs()][0]);
  const int nbh = min(a.rows - r.row(), (int)a.t.block[r.bs()][1]);
  if (nbw <= 0 || nbh <= 0) return 2;
  const int lx = vertical ? nbw - 1 : x - r.col();
  const int ly = vertical ? y - r.row() : nbh - 1;
  if (lx < 0 || lx >= nbw || ly < 0 || ly >= nbh) return 2;
  const Leaf L = tx_leaf(a.t, safe_tx(r.txy()), uniform_tx(r), r.split(), lx, ly);
  return vertical ? L.cw : L.ch;
}

__device__ __forceinline__ int clamp_level(int v) { return v < 0 ? 0 : (v > 63 ? 63 : v); }

// ResolveBlockLevels (loopfilter/level.go:120-190) packed as the level cell
// [Y vertical, Y horizontal, U, V].  Indices are masked so that a record the
// check kernel rejects cannot read out of range.
__device__ uint32_t block_levels(const MapArgs& a, const LfRec& r) {
  if (a.lumaZero) return 0;
  if (!a.deltaPresent && !a.segEnabled && !a.modeRef)
    return a.base[0][0] | a.base[0][1] << 8 | a.base[1][0] << 16 | a.base[2][0] << 24;
  const int nplanes = a.mono ? 1 : 3;
  const int ref = r.ref() & 7, seg = r.seg() & 7;
  uint32_t out = 0;
  for (int k = 0; k < 4; k++) {  // (Y,V) (Y,H) (U,V) (V,V)
    const int plane = k < 2 ? 0 : k - 1, edge = k < 2 ? k : 0;
    if (plane >= nplanes) break;
    const int base = a.base[plane][edge];
    if (plane && base == 0) continue;
    int dl = 0;
    if (a.deltaPresent) dl = a.deltaMulti ? r.deltaMulti(plane ? plane + 1 : edge) : r.deltaFromBase();
    const int sd = a.segEnabled ? a.segDelta[seg][plane ? plane + 1 : edge] : 0;
    int lvl = clamp_level(base + dl);
    lvl = clamp_level(lvl + sd);
    if (a.modeRef) {
      int d = a.refDelta[ref];
      if (ref > 0) d += a.modeDelta[r.mode() & 1];
      lvl = clamp_level(lvl + d * (1 << (lvl >> 5)));
    }
    out |= (uint32_t)lvl << (8 * k);
  }
  return out;
}

// Luma cell (x, y) with its record and those of its left and upper
// neighbours: the width class of the vertical edge on its left and of the
// horizontal edge on its top (-1: no edge), and the luma bytes of its level
// cell.
__device__ void luma_cell(const MapArgs& a, int x, int y, const LfRec& r, const LfRec& left, const LfRec& above,
                          int& sv, int& sh, uint32_t& lv) {
  if (!r.valid() || r.bs() >= 22) return;
  const int bx = r.col(), by = r.row();
  const int bw4 = min(a.cols - bx, (int)a.t.block[r.bs()][0]);
  const int bh4 = min(a.rows - by, (int)a.t.block[r.bs()][1]);
  const int lx = x - bx, ly = y - by;
  if (lx < 0 || ly < 0 || lx >= bw4 || ly >= bh4) return;
  const int tx = safe_tx(r.txy());
  const bool uni = uniform_tx(r);
  const bool inner = r.intra() || !r.skip();
  const Leaf L = tx_leaf(a.t, tx, uni, r.split(), lx, ly);
  if (lx == 0)
    sv = min(L.cw, bx > 0 ? luma_edge_ctx(a, left, x - 1, y, true) : 2);
  else if (L.left && inner)
    sv = min(L.cw, tx_leaf(a.t, tx, uni, r.split(), lx - 1, ly).cw);
  if (ly == 0)
    sh = min(L.ch, by > 0 ? luma_edge_ctx(a, above, x, y - 1, false) : 2);
  else if (L.top && inner)
    sh = min(L.ch, tx_leaf(a.t, tx, uni, r.split(), lx, ly - 1).ch);
  lv = block_levels(a, r) & 0xffff;
}

// Chroma level bytes of chroma cell (x, y): the covering block last in raster
// order of origin (the reference's walk writes each block's chroma rect), one
// of the records at the cell's luma group.
__device__ uint32_t chroma_levels(const MapArgs& a, int x, int y) {
  // The group is 1, 2 or 4 cells: k = j * 2 + i with i <= ssx, j <= ssy.
  uint32_t head0[4], head2[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const int i = k & 1, j = k >> 1;
    head2[k] = 0;
    if (i <= a.ssx && j <= a.ssy) {
      const uint4 u = __ldg(a.rec + 2 * ((size_t)((y << a.ssy) + j) * a.cols + (x << a.ssx) + i));
      head0[k] = u.x, head2[k] = u.z;
    }
  }
  int best = -1;
  uint32_t bestKey = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    const bool valid = (head2[k] >> 8) & 0xff;
    if (!valid || (head2[k] & 0xff) >= 22) continue;
    const uint32_t key = head0[k];  // mi_row << 16 | mi_col: raster order of origin
    if (best < 0 || key > bestKey) best = k, bestKey = key;
  }
  if (best < 0) return 0;
  return block_levels(a, load_rec(a, (x << a.ssx) + (best & 1), (y << a.ssy) + (best >> 1))) & 0xffff0000u;
}

// Chroma cell (cx, cy) with the record `r` at the bottom-right luma cell of
// its luma group: the block carrying the shared chroma there (the has_chroma
// gate of dav1d as BuildFromMap applies it, loop_filter_masks.go:508-533).
__device__ void chroma_cell(const MapArgs& a, int cx, int cy, const LfRec& r, int& sv, int& sh) {
  const int lx = (cx << a.ssx) + a.ssx, ly = (cy << a.ssy) + a.ssy;
  if (!r.valid() || !r.hasUV() || r.bs() >= 22) return;
  const int bx = r.col(), by = r.row();
  const int W4 = a.t.block[r.bs()][0], H4 = a.t.block[r.bs()][1];
  if (!((W4 > a.ssx || (bx & 1)) && (H4 > a.ssy || (by & 1)))) return;
  const int bw4 = min(a.cols - bx, W4), bh4 = min(a.rows - by, H4);
  if (lx < bx || lx >= bx + bw4 || ly < by || ly >= by + bh4) return;
  const int cbw4 = min(a.ccols - (bx >> a.ssx), (W4 + a.ssx) >> a.ssx);
  const int cbh4 = min(a.crows - (by >> a.ssy), (H4 + a.ssy) >> a.ssy);
  const int lcx = cx - (bx >> a.ssx), lcy = cy - (by >> a.ssy);
  if (lcx < 0 || lcy < 0 || lcx >= cbw4 || lcy >= cbh4) return;
  const uint8_t* d = a.t.tx[safe_tx(r.txuv())];
  const int cw = d[2] != 0, ch = d[3] != 0;
  const bool inner = r.intra() || !r.skip();
  // The two context loads depend only on the block origin: issue both.
  const bool needL = lcx == 0 && bx > 0, needA = lcy == 0 && by > 0;
  LfRec nl, na;
  if (needL) nl = load_head(a, bx - 1, min((cy << a.ssy) + a.ssy, a.rows - 1), false);
  if (needA) na = load_head(a, min((cx << a.ssx) + a.ssx, a.cols - 1), by - 1, false);
  if (lcx == 0) {
    int ctx = 1;
    if (needL && nl.valid() && nl.hasUV()) ctx = a.t.tx[safe_tx(nl.txuv())][2] != 0;
    sv = min(cw, ctx);
  } else if (inner && (lcx & (d[0] - 1)) == 0) {
    sv = cw;
  }
  if (lcy == 0) {
    int ctx = 1;
    if (needA && na.valid() && na.hasUV()) ctx = a.t.tx[safe_tx(na.txuv())][3] != 0;
    sh = min(ch, ctx);
  } else if (inner && (lcy & (d[1] - 1)) == 0) {
    sh = ch;
  }
}

// One 128x128 region (32x32 cells) per CTA, a thread per cell.
__device__ void region_masks(const MapArgs& a, int region, int8_t (*s_t)[33], uint32_t (*s_lv)[33]) {
  const int rx = region % a.sbw, ry = region / a.sbw;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* M = (uint32_t*)(a.masks + (size_t)region * PF_LF_MASK_WORDS);

  // Every record load that does not depend on another goes out first: the
  // cell's own record, its left and upper neighbours (read only when the
  // cell starts its block), and the emitter of this thread's chroma cell.
  const int x = rx * 32 + w, y = ry * 32 + lane;
  const bool in = x < a.cols && y < a.rows;
  const int cwid = 32 >> a.ssx, chgt = 32 >> a.ssy;
  const int cx = rx * cwid + w, cy = ry * chgt + lane;
  const bool cin = !a.mono && w < cwid && lane < chgt && cx < a.ccols && cy < a.crows;
  LfRec own, left, above, em;
  if (in) own = load_rec(a, x, y);
  if (in && x > 0) left = load_head(a, x - 1, y, true);
  if (in && y > 0) above = load_head(a, x, y - 1, true);
  if (cin) em = load_head(a, (cx << a.ssx) + a.ssx, (cy << a.ssy) + a.ssy, false);

  // Luma.  Warp = column w, lane = row: vertical edges of column w.
  int sv = -1, sh = -1;
  uint32_t lv = 0;
  if (in) {
    luma_cell(a, x, y, own, left, above, sv, sh, lv);
    if (!a.mono && x < a.ccols && y < a.crows) lv |= chroma_levels(a, x, y);
  }
  // Y[0][w][s] as one 32-bit word: bit = row within the region.
#pragma unroll
  for (int s = 0; s < 3; s++) {
    const uint32_t b = __ballot_sync(0xffffffffu, sv == s);
    if (lane == 0) M[w * 3 + s] = b;
  }
  s_t[lane][w] = (int8_t)sh;
  s_lv[lane][w] = lv;
  __syncthreads();
  // Warp = row w, lane = column: horizontal edges of row w, and the level
  // cells of row w stored coalesced.
  {
    const int s0 = s_t[w][lane];
#pragma unroll
    for (int s = 0; s < 3; s++) {
      const uint32_t b = __ballot_sync(0xffffffffu, s0 == s);
      if (lane == 0) M[(32 + w) * 3 + s] = b;
    }
    const int x2 = rx * 32 + lane, y2 = ry * 32 + w;
    if (x2 < a.cols && y2 < a.rows) a.levels[(size_t)y2 * a.cols + x2] = s_lv[w][lane];
  }
  __syncthreads();

  // Chroma: the region's (32 >> ssx) x (32 >> ssy) chroma cells.  UV[dir][pos][s]
  // is two 16-bit halves split at 16 >> ss of the scanned direction.
  int cv = -1, chs = -1;
  if (cin) chroma_cell(a, cx, cy, em, cv, chs);
  const int vsplit = 16 >> a.ssy, hsplit = 16 >> a.ssx;
#pragma unroll
  for (int s = 0; s < 2; s++) {
    const uint32_t b = __ballot_sync(0xffffffffu, cv == s);
    if (lane == 0) M[192 + w * 2 + s] = (b & ((1u << vsplit) - 1)) | (b >> vsplit) << 16;
  }
  s_t[lane][w] = (int8_t)chs;
  __syncthreads();
  {
    const int s0 = s_t[w][lane];
#pragma unroll
    for (int s = 0; s < 2; s++) {
      const uint32_t b = __ballot_sync(0xffffffffu, s0 == s);
      if (lane == 0) M[192 + (32 + w) * 2 + s] = (b & ((1u << hsplit) - 1)) | (b >> hsplit) << 16;
    }
  }
}

// The reference's level-cache walk over one MI row (postfilter_loopfilter_masks
// .go:146-224): each cell's successor in the chain and the error the walk
// meets if it visits the cell; ResolveBlockLevels' checks (level.go:126-175)
// come before the block-size check, as in the reference.
__device__ uint32_t walk_cell(const MapArgs& a, int c, int row) {
  const LfRec r = load_rec(a, c, row);
  if (!r.valid()) return c + 1;
  const int next = r.colEnd();
  if (next <= c || next > a.cols) return (uint32_t)c | (uint32_t)kLfBatch << 20;
  uint32_t code = 0;
  if (r.col() == c && r.row() == row) {
    if (r.ref() >= 8 || r.mode() > 1 || (!a.lumaZero && a.segEnabled && r.seg() >= 8))
      code = kLfFilter;
    else if (r.bs() >= 22 || r.txy() >= 19 || (!a.mono && r.hasUV() && r.txuv() >= 19))
      code = kLfBatch;
  }
  return (uint32_t)next | code << 20;
}

struct WalkSmem {
  int next[1024];
  int succ[1024];
  uint8_t mark[1024];
  int entry, err, exit;
};

// One MI row's walk, 1024 cells at a time: the chain from the entry cell is
// found by pointer doubling (after round r every cell within 2^(r+1) - 1
// steps of the entry is marked), an error cell ending the chain.  Writes the
// row's first error as (cell index << 8 | kind), or all ones.
__device__ void row_walk(const MapArgs& a, int row, WalkSmem& S) {
  const int i = threadIdx.x;
  if (i == 0) S.entry = 0, S.err = INT_MAX;
  for (int c0 = 0; c0 < a.cols; c0 += 1024) {
    __syncthreads();
    const int entry = S.entry;
    if (entry >= a.cols || S.err != INT_MAX) break;
    if (entry >= c0 + 1024) continue;
    const int c = c0 + i;
    const uint32_t v = c < a.cols ? walk_cell(a, c, row) : (uint32_t)(c + 1);
    const int code = v >> 20, succ = v & 0xfffff;
    S.succ[i] = v;
    S.next[i] = code ? c : succ;  // an error cell is a fixed point: the chain ends there
    S.mark[i] = c == entry;
    if (i == 0) S.exit = INT_MAX;
    __syncthreads();
#pragma unroll 1
    for (int r = 0; r < 10; r++) {
      const int n = S.next[i];
      const bool m = S.mark[i];
      const int n2 = n < c0 + 1024 ? S.next[n - c0] : n;
      __syncthreads();
      if (m && n < c0 + 1024) S.mark[n - c0] = 1;
      S.next[i] = n2;
      __syncthreads();
    }
    if (S.mark[i]) {
      if (code) atomicMin(&S.err, c);
      else if (succ >= c0 + 1024) S.exit = succ;  // the chain's last cell in this chunk
    }
    __syncthreads();
    if (i == 0) S.entry = S.err != INT_MAX ? a.cols : S.exit;
  }
  __syncthreads();
  if (i == 0) {
    unsigned long long out = ~0ull;
    if (S.err != INT_MAX)  // the error's chunk is the last one loaded
      out = (unsigned long long)((size_t)row * a.cols + S.err) << 8 | (S.succ[S.err & 1023] >> 20);
    a.rowErr[row] = out;
  }
}

// One launch: CTAs [0, regions) build the masks and level cache of one
// 128x128 region each, the rest walk one MI row each for the status.
__global__ void __launch_bounds__(1024) k_lf_build(MapArgs a) {
  __shared__ int8_t s_t[32][33];
  __shared__ uint32_t s_lv[32][33];
  __shared__ WalkSmem s_walk;
  if ((int)blockIdx.x < a.regions)
    region_masks(a, blockIdx.x, s_t, s_lv);
  else
    row_walk(a, blockIdx.x - a.regions, s_walk);
}

}  // namespace pf

void* pf_internal_search_scratch(pf_ctx* c, size_t bytes);  // pf_api.cu
int pf_internal_wait(pf_ctx* c, void* stream);  // pf_api.cu: blocking or bounded by the context's deadline
void* pf_internal_stream(pf_ctx* c);
void* pf_internal_pinned(pf_ctx* c, size_t bytes);

extern "C" int pf_lf_build(pf_ctx* ctx, const pf_lf_record* records, int32_t cols, int32_t rows,
                           uint32_t records_memory, const pf_lf_levels* lv, int32_t ss_x, int32_t ss_y, int32_t mono,
                           uint16_t* masks, uint8_t* level_cache, uint32_t out_memory) {
  using namespace pf;
  static_assert(sizeof(pf_lf_record) == 32, "pf_lf_record is 32 bytes");
  if (!ctx || !records || !lv || !masks || !level_cache) return PF_ERR_INVALID_ARG;
  if (cols <= 0 || rows <= 0 || (cols & 1) || (rows & 1) || cols > 16384 || rows > 16384) return PF_ERR_INVALID_ARG;
  if (records_memory > PF_MEM_DEVICE || out_memory > PF_MEM_DEVICE || ss_x < 0 || ss_x > 1 || ss_y < 0 ||
      ss_y > 1 || mono < 0 || mono > 1)
    return PF_ERR_INVALID_ARG;
  if (records_memory == PF_MEM_DEVICE && ((uintptr_t)records & 15)) return PF_ERR_INVALID_ARG;
  if (out_memory == PF_MEM_DEVICE && (((uintptr_t)masks & 3) || ((uintptr_t)level_cache & 3)))
    return PF_ERR_INVALID_ARG;

  MapArgs a;
  memset(&a, 0, sizeof(a));
  a.cols = cols, a.rows = rows;
  a.sbw = (cols + 31) >> 5;
  const int sbh = (rows + 31) >> 5;
  a.ssx = ss_x, a.ssy = ss_y, a.mono = mono;
  a.ccols = (cols + ss_x) >> ss_x, a.crows = (rows + ss_y) >> ss_y;
  auto clampl = [](int v) { return (uint8_t)(v < 0 ? 0 : (v > 63 ? 63 : v)); };
  a.base[0][0] = clampl(lv->level_y[0]), a.base[0][1] = clampl(lv->level_y[1]);
  a.base[1][0] = a.base[1][1] = clampl(lv->level_u);
  a.base[2][0] = a.base[2][1] = clampl(lv->level_v);
  a.lumaZero = lv->level_y[0] == 0 && lv->level_y[1] == 0;
  a.deltaPresent = lv->delta_lf_present != 0, a.deltaMulti = lv->delta_lf_multi != 0;
  a.segEnabled = lv->segmentation_enabled != 0, a.modeRef = lv->mode_ref_delta_enabled != 0;
  memcpy(a.refDelta, lv->ref_delta, 8);
  memcpy(a.modeDelta, lv->mode_delta, 2);
  if (a.segEnabled) memcpy(a.segDelta, lv->segment_delta, sizeof(a.segDelta));
  memcpy(a.t.block, pf_block_dims, sizeof(a.t.block));
  memcpy(a.t.tx, pf_tx_dims, sizeof(a.t.tx));

  const size_t cells = (size_t)cols * rows;
  const size_t recB = cells * sizeof(pf_lf_record), maskB = (size_t)a.sbw * sbh * PF_LF_MASK_WORDS * 2,
               lcB = cells * 4;
  auto up = [](size_t n) { return (n + 255) & ~(size_t)255; };
  const bool hostRec = records_memory == PF_MEM_HOST, hostOut = out_memory == PF_MEM_HOST;
  const size_t errB = up((size_t)rows * 8);
  const size_t total = errB + (hostRec ? up(recB) : 0) + (hostOut ? up(maskB) + up(lcB) : 0);
  uint8_t* scratch = (uint8_t*)pf_internal_search_scratch(ctx, total);
  unsigned long long* hostErr = (unsigned long long*)pf_internal_pinned(ctx, (size_t)rows * 8);
  if (!scratch || !hostErr) return PF_ERR_DEVICE;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  size_t off = errB;
  a.rowErr = (unsigned long long*)scratch;
  cudaError_t e = cudaSuccess;
  if (hostRec) {
    a.rec = (const uint4*)(scratch + off);
    off += up(recB);
    e = cudaMemcpyAsync((void*)a.rec, records, recB, cudaMemcpyHostToDevice, st);
  } else {
    a.rec = (const uint4*)records;
  }
  if (hostOut) {
    a.masks = (uint16_t*)(scratch + off);
    off += up(maskB);
    a.levels = (uint32_t*)(scratch + off);
  } else {
    a.masks = masks;
    a.levels = (uint32_t*)level_cache;
  }
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  a.regions = a.sbw * sbh;
  k_lf_build<<<a.regions + rows, 1024, 0, st>>>(a);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hostErr, a.rowErr, (size_t)rows * 8, cudaMemcpyDeviceToHost, st);
  if (hostOut && e == cudaSuccess) e = cudaMemcpyAsync(masks, a.masks, maskB, cudaMemcpyDeviceToHost, st);
  if (hostOut && e == cudaSuccess) e = cudaMemcpyAsync(level_cache, a.levels, lcB, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  const int w = pf_internal_wait(ctx, st);
  if (w != PF_OK) return w;
  unsigned long long err = ~0ull;
  for (int r = 0; r < rows; r++) err = hostErr[r] < err ? hostErr[r] : err;
  if (err == ~0ull) return PF_OK;
  return (err & 0xff) == kLfFilter ? PF_ERR_INVALID_FILTER : PF_ERR_INVALID_BATCH;
}
