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
// valid one jumps to its MIColEnd).  k_lf_check replays that chain for each
// row over shared memory and keeps the first error in raster order.
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
  unsigned long long* err;
  int cols, rows, sbw, ssx, ssy, mono, ccols, crows;
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

// The class a neighbouring block carries out of its right column (vertical)
// or bottom row (horizontal) at the given map cell (fillLeftLumaContext /
// fillAboveLumaContext, loop_filter_masks.go:553-646): 2 when the cell holds
// no valid block.
__device__ int luma_edge_ctx(const MapArgs& a, int x, int y, bool vertical) {
  const LfRec r = load_rec(a, x, y);
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

// Luma cell (x, y): the width class of the vertical edge on its left and of
// the horizontal edge on its top (-1: no edge), and its level cell.
__device__ void luma_cell(const MapArgs& a, int x, int y, int& sv, int& sh, uint32_t& lv) {
  const LfRec r = load_rec(a, x, y);
  if (r.valid() && r.bs() < 22) {
    const int bx = r.col(), by = r.row();
    const int bw4 = min(a.cols - bx, (int)a.t.block[r.bs()][0]);
    const int bh4 = min(a.rows - by, (int)a.t.block[r.bs()][1]);
    const int lx = x - bx, ly = y - by;
    if (lx >= 0 && ly >= 0 && lx < bw4 && ly < bh4) {
      const int tx = safe_tx(r.txy());
      const bool uni = uniform_tx(r);
      const bool inner = r.intra() || !r.skip();
      const Leaf L = tx_leaf(a.t, tx, uni, r.split(), lx, ly);
      if (lx == 0)
        sv = min(L.cw, bx > 0 ? luma_edge_ctx(a, x - 1, y, true) : 2);
      else if (L.left && inner)
        sv = min(L.cw, tx_leaf(a.t, tx, uni, r.split(), lx - 1, ly).cw);
      if (ly == 0)
        sh = min(L.ch, by > 0 ? luma_edge_ctx(a, x, y - 1, false) : 2);
      else if (L.top && inner)
        sh = min(L.ch, tx_leaf(a.t, tx, uni, r.split(), lx, ly - 1).ch);
      lv = block_levels(a, r) & 0xffff;
    }
  }
  // Chroma levels of chroma cell (x, y): the covering block last in raster
  // order of origin (the reference's walk writes each block's chroma rect).
  if (!a.mono && x < a.ccols && y < a.crows) {
    uint32_t bestKey = 0;
    bool found = false;
    LfRec best;
    for (int j = 0; j <= a.ssy; j++)
      for (int i = 0; i <= a.ssx; i++) {
        const LfRec c = load_rec(a, (x << a.ssx) + i, (y << a.ssy) + j);
        if (!c.valid() || c.bs() >= 22) continue;
        const uint32_t key = (uint32_t)c.row() << 16 | c.col();
        if (!found || key > bestKey) best = c, bestKey = key, found = true;
      }
    if (found) lv |= block_levels(a, best) & 0xffff0000u;
  }
}

// Chroma cell (cx, cy): the block carrying the shared chroma is the one at the
// bottom-right luma cell of the cell's luma group (the has_chroma gate of
// dav1d as BuildFromMap applies it, loop_filter_masks.go:508-533).
__device__ void chroma_cell(const MapArgs& a, int cx, int cy, int& sv, int& sh) {
  const int lx = (cx << a.ssx) + a.ssx, ly = (cy << a.ssy) + a.ssy;
  const LfRec r = load_rec(a, lx, ly);
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
  if (lcx == 0) {
    int ctx = 1;
    if (bx > 0) {
      const LfRec n = load_rec(a, bx - 1, min((cy << a.ssy) + a.ssy, a.rows - 1));
      if (n.valid() && n.hasUV()) ctx = a.t.tx[safe_tx(n.txuv())][2] != 0;
    }
    sv = min(cw, ctx);
  } else if (inner && (lcx & (d[0] - 1)) == 0) {
    sv = cw;
  }
  if (lcy == 0) {
    int ctx = 1;
    if (by > 0) {
      const LfRec n = load_rec(a, min((cx << a.ssx) + a.ssx, a.cols - 1), by - 1);
      if (n.valid() && n.hasUV()) ctx = a.t.tx[safe_tx(n.txuv())][3] != 0;
    }
    sh = min(ch, ctx);
  } else if (inner && (lcy & (d[1] - 1)) == 0) {
    sh = ch;
  }
}

// One CTA per 128x128 region (32x32 cells), a thread per cell.
__global__ void __launch_bounds__(1024) k_lf_masks(MapArgs a) {
  __shared__ int8_t s_t[32][33];
  __shared__ uint32_t s_lv[32][33];
  const int rx = blockIdx.x, ry = blockIdx.y;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  uint32_t* M = (uint32_t*)(a.masks + ((size_t)ry * a.sbw + rx) * PF_LF_MASK_WORDS);

  // Luma.  Warp = column w, lane = row: vertical edges of column w.
  int sv = -1, sh = -1;
  uint32_t lv = 0;
  const int x = rx * 32 + w, y = ry * 32 + lane;
  if (x < a.cols && y < a.rows) luma_cell(a, x, y, sv, sh, lv);
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
  const int cwid = 32 >> a.ssx, chgt = 32 >> a.ssy;
  int cv = -1, chs = -1;
  const int cx = rx * cwid + w, cy = ry * chgt + lane;
  if (!a.mono && w < cwid && lane < chgt && cx < a.ccols && cy < a.crows) chroma_cell(a, cx, cy, cv, chs);
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
  if (next <= c || next > a.cols) return (uint32_t)kLfBatch << 20;
  uint32_t code = 0;
  if (r.col() == c && r.row() == row) {
    if (r.ref() >= 8 || r.mode() > 1 || (!a.lumaZero && a.segEnabled && r.seg() >= 8))
      code = kLfFilter;
    else if (r.bs() >= 22 || r.txy() >= 19 || (!a.mono && r.hasUV() && r.txuv() >= 19))
      code = kLfBatch;
  }
  return (uint32_t)next | code << 20;
}

__global__ void __launch_bounds__(256) k_lf_check(MapArgs a) {
  __shared__ uint32_t s_info[256];
  __shared__ int s_pos, s_stop;
  const int row = blockIdx.x;
  if (threadIdx.x == 0) s_pos = 0, s_stop = 0;
  for (int c0 = 0; c0 < a.cols; c0 += 256) {
    __syncthreads();
    if (s_stop) break;
    const int c = c0 + threadIdx.x;
    s_info[threadIdx.x] = c < a.cols ? walk_cell(a, c, row) : 0;
    __syncthreads();
    if (threadIdx.x == 0) {
      int pos = s_pos;
      while (pos < c0 + 256 && pos < a.cols) {
        const uint32_t v = s_info[pos - c0];
        if (v >> 20) {
          atomicMin(a.err, (unsigned long long)((size_t)row * a.cols + pos) << 8 | (v >> 20));
          s_stop = 1;
          break;
        }
        pos = v & 0xfffff;  // strictly past pos: an invalid cell steps one, a valid one jumps to MIColEnd
      }
      s_pos = pos;
    }
  }
}

}  // namespace pf

void* pf_internal_search_scratch(pf_ctx* c, size_t bytes);  // pf_api.cu
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
  const size_t total = 256 + (hostRec ? up(recB) : 0) + (hostOut ? up(maskB) + up(lcB) : 0);
  uint8_t* scratch = (uint8_t*)pf_internal_search_scratch(ctx, total);
  unsigned long long* hostErr = (unsigned long long*)pf_internal_pinned(ctx, 64);
  if (!scratch || !hostErr) return PF_ERR_DEVICE;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  size_t off = 256;
  a.err = (unsigned long long*)scratch;
  cudaError_t e = cudaMemsetAsync(a.err, 0xff, 8, st);
  if (hostRec) {
    a.rec = (const uint4*)(scratch + off);
    off += up(recB);
    if (e == cudaSuccess) e = cudaMemcpyAsync((void*)a.rec, records, recB, cudaMemcpyHostToDevice, st);
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
  k_lf_check<<<rows, 256, 0, st>>>(a);
  k_lf_masks<<<dim3(a.sbw, sbh), 1024, 0, st>>>(a);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(hostErr, a.err, 8, cudaMemcpyDeviceToHost, st);
  if (hostOut && e == cudaSuccess) e = cudaMemcpyAsync(masks, a.masks, maskB, cudaMemcpyDeviceToHost, st);
  if (hostOut && e == cudaSuccess) e = cudaMemcpyAsync(level_cache, a.levels, lcB, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  const unsigned long long err = *hostErr;
  if (err == ~0ull) return PF_OK;
  return (err & 0xff) == kLfFilter ? PF_ERR_INVALID_FILTER : PF_ERR_INVALID_BATCH;
}
