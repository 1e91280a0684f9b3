// CPU oracle (test infrastructure): goav1's deblocking edge-mask and
// level-cache build from the block record map, restated block by block as
// the reference runs it.  Only tests/ and the bench's CPU baseline leg use it.
//
//   oracle_lf_build         FrameWorkLoopFilterMasks.BuildFromMap
//                           (internal/av1/threading/loop_filter_masks.go:450-551,
//                           neighbour contexts :553-680) then
//                           populateLoopFilterLevelCacheFromMap
//                           (internal/av1/decoder/postfilter_loopfilter_masks.go:119-228)
//   oracle_lf_build_ordered the decode-time build: blocks in decode order with
//                           the carried above/left contexts, the left context
//                           reset at each superblock row
//                           (loop_filter_masks.go:289-400)
//   oracle_lf_mask_block    one block's edges with explicit contexts, the
//                           lfmask functions maskEdgesIntra / maskEdgesInter /
//                           maskEdgesChroma (internal/av1/lfmask/mask.go:110-525)
//   oracle_lf_block_levels  PreparedLevelResolver.ResolveBlockLevels
//                           (internal/av1/loopfilter/level.go:86-190)
//
// Masks are lfmask.FilterMask words: Y[dir][pos][strength][half] (384) then
// UV[dir][pos][strength][half] (256) per 128x128 region.
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pf_oracle.h"
#include "pf_tables.h"

namespace {

constexpr int kOk = 0, kErrBatch = PF_ERR_INVALID_BATCH, kErrFilter = PF_ERR_INVALID_FILTER;

int imin(int a, int b) { return a < b ? a : b; }

// Y/UV edge bit setters.  `pos` is the 4x4 column (vertical edges) or row
// (horizontal edges) inside the region, `bit` the position along the edge.
void set_y(uint16_t* m, int dir, int pos, int s, int bit) {
  m[((dir * 32 + (pos & 31)) * 3 + s) * 2 + (bit >= 16)] |= (uint16_t)(1u << (bit & 15));
}
void set_uv(uint16_t* m, int dir, int pos, int s, int bit, int split) {
  const int hi = bit >= split;
  m[384 + ((dir * 32 + (pos & 31)) * 2 + s) * 2 + hi] |= (uint16_t)(1u << (hi ? bit - split : bit));
}

// dav1d's decomp_tx scratch for one block (lfmask/mask.go:63-98, :527-581):
// per block-local cell the clamped log2 width/height of its transform, and at
// each transform's first column its width (xstep) and at its first row its
// height (ystep), in 4x4 units.
struct TxGrid {
  uint8_t lw[32][32], lh[32][32], xstep[32][32], ystep[32][32];
};

void tx_leaf(TxGrid& g, int yb, int xb, int tx) {
  const uint8_t* d = pf_tx_dims[tx];
  const int w = d[0], h = d[1];
  for (int y = yb; y < yb + h; y++) {
    for (int x = xb; x < xb + w; x++) {
      g.lw[y][x] = (uint8_t)imin(d[2], 2);
      g.lh[y][x] = (uint8_t)imin(d[3], 2);
    }
    g.xstep[y][xb] = (uint8_t)w;
  }
  for (int x = xb; x < xb + w; x++) g.ystep[yb][x] = (uint8_t)h;
}

void decomp_tx(TxGrid& g, int yb, int xb, int tx, int depth, int yoff, int xoff, const uint16_t split[2]) {
  const uint8_t* d = pf_tx_dims[tx];
  bool isSplit = false;
  if (tx != 0 && depth <= 1) {
    const int sh = yoff * 4 + xoff;
    isSplit = sh < 16 && ((split[depth] >> sh) & 1);
  }
  if (!isSplit) {
    tx_leaf(g, yb, xb, tx);
    return;
  }
  const int sub = d[4], hw = d[0] >> 1, hh = d[1] >> 1;
  decomp_tx(g, yb, xb, sub, depth + 1, yoff * 2, xoff * 2, split);
  if (d[0] >= d[1]) decomp_tx(g, yb, xb + hw, sub, depth + 1, yoff * 2, xoff * 2 + 1, split);
  if (d[1] >= d[0]) {
    decomp_tx(g, yb + hh, xb, sub, depth + 1, yoff * 2 + 1, xoff * 2, split);
    if (d[0] >= d[1]) decomp_tx(g, yb + hh, xb + hw, sub, depth + 1, yoff * 2 + 1, xoff * 2 + 1, split);
  }
}

// The transform grid of a w4 x h4 (visible) block: root transforms tiled
// from the origin, each decomposed by the split bits (uniform when none).
void block_grid(TxGrid& g, int w4, int h4, int tx, const uint16_t split[2], bool uniform) {
  static const uint16_t none[2] = {0, 0};
  const uint8_t* d = pf_tx_dims[tx];
  int yoff = 0;
  for (int y = 0; y < h4; y += d[1], yoff++) {
    int xoff = 0;
    for (int x = 0; x < w4; x += d[0], xoff++) decomp_tx(g, y, x, tx, 0, yoff, xoff, uniform ? none : split);
  }
}

// maskEdgesInter (mask.go:110-332) written over the decomposed grid; for an
// unsplit block this is the reference's fast path bit for bit (a class-0
// edge, an inner edge at every multiple of the transform width).
void mask_inter(uint16_t* m, int by4, int bx4, int w4, int h4, int skip, int tx, const uint16_t split[2],
                uint8_t* a, uint8_t* l) {
  TxGrid g;
  block_grid(g, w4, h4, tx, split, split[0] == 0 || tx == 0);
  for (int y = 0; y < h4; y++) set_y(m, 0, bx4, imin(g.lw[y][0], l[y]), by4 + y);
  for (int x = 0; x < w4; x++) set_y(m, 1, by4, imin(g.lh[0][x], a[x]), bx4 + x);
  if (!skip) {
    for (int y = 0; y < h4; y++) {
      int ltx = g.lw[y][0], step = g.xstep[y][0];
      for (int x = step; x < w4; x += step) {
        const int rtx = g.lw[y][x];
        set_y(m, 0, bx4 + x, imin(rtx, ltx), by4 + y);
        ltx = rtx;
        step = g.xstep[y][x];
      }
    }
    for (int x = 0; x < w4; x++) {
      int ttx = g.lh[0][x], step = g.ystep[0][x];
      for (int y = step; y < h4; y += step) {
        const int btx = g.lh[y][x];
        set_y(m, 1, by4 + y, imin(ttx, btx), bx4 + x);
        ttx = btx;
        step = g.ystep[y][x];
      }
    }
  }
  for (int y = 0; y < h4; y++) l[y] = g.lw[y][w4 - 1];
  for (int x = 0; x < w4; x++) a[x] = g.lh[h4 - 1][x];
}

// maskEdgesIntra (mask.go:334-400).
void mask_intra(uint16_t* m, int by4, int bx4, int w4, int h4, int tx, uint8_t* a, uint8_t* l) {
  const uint8_t* d = pf_tx_dims[tx];
  const int twl = imin(2, d[2]), thl = imin(2, d[3]);
  for (int y = 0; y < h4; y++) set_y(m, 0, bx4, imin(twl, l[y]), by4 + y);
  for (int x = 0; x < w4; x++) set_y(m, 1, by4, imin(thl, a[x]), bx4 + x);
  for (int x = d[0]; x < w4; x += d[0])
    for (int y = 0; y < h4; y++) set_y(m, 0, bx4 + x, twl, by4 + y);
  for (int y = d[1]; y < h4; y += d[1])
    for (int x = 0; x < w4; x++) set_y(m, 1, by4 + y, thl, bx4 + x);
  for (int x = 0; x < w4; x++) a[x] = (uint8_t)thl;
  for (int y = 0; y < h4; y++) l[y] = (uint8_t)twl;
}

// maskEdgesChroma (mask.go:405-525); chroma 4x4 units, the lanes split at
// 16 >> ss of the scanned direction.
void mask_chroma(uint16_t* m, int cby4, int cbx4, int cw4, int ch4, int skipInter, int tx, uint8_t* a, uint8_t* l,
                 int ssx, int ssy) {
  const uint8_t* d = pf_tx_dims[tx];
  const int twl = d[2] != 0, thl = d[3] != 0;
  const int vsplit = 16 >> ssy, hsplit = 16 >> ssx;
  for (int y = 0; y < ch4; y++) set_uv(m, 0, cbx4, imin(twl, l[y]), (cby4 + y) & 31, vsplit);
  for (int x = 0; x < cw4; x++) set_uv(m, 1, cby4, imin(thl, a[x]), (cbx4 + x) & 31, hsplit);
  if (!skipInter) {
    for (int x = d[0]; x < cw4; x += d[0])
      for (int y = 0; y < ch4; y++) set_uv(m, 0, cbx4 + x, twl, (cby4 + y) & 31, vsplit);
    for (int y = d[1]; y < ch4; y += d[1])
      for (int x = 0; x < cw4; x++) set_uv(m, 1, cby4 + y, thl, (cbx4 + x) & 31, hsplit);
  }
  for (int x = 0; x < cw4; x++) a[x] = (uint8_t)thl;
  for (int y = 0; y < ch4; y++) l[y] = (uint8_t)twl;
}

struct Map {
  const pf_lf_record* r;
  int cols, rows, ssx, ssy, hasChroma, sbw;
  const pf_lf_record& at(int x, int y) const { return r[(size_t)y * cols + x]; }
};

// CreateIntra / CreateInter (lfmask/build.go:60-100, :203-236) without the
// level writes: the luma edges over the frame-clamped block, then, when the
// chroma contexts are given, the chroma edges over its chroma rectangle.
void create_block(const Map& M, uint16_t* region, const pf_lf_record& r, int bx, int by, uint8_t* ay, uint8_t* ly,
                  uint8_t* auv, uint8_t* luv) {
  const int W4 = pf_block_dims[r.block_size][0], H4 = pf_block_dims[r.block_size][1];
  const int bw4 = imin(M.cols - bx, W4), bh4 = imin(M.rows - by, H4);
  const int bx4 = bx & 31, by4 = by & 31;
  if (bw4 > 0 && bh4 > 0) {
    if (r.intra)
      mask_intra(region, by4, bx4, bw4, bh4, r.tx_y, ay, ly);
    else
      mask_inter(region, by4, bx4, bw4, bh4, r.skip ? 1 : 0, r.tx_y, r.tx_split, ay, ly);
  }
  if (!auv) return;
  const int cbw4 = imin(((M.cols + M.ssx) >> M.ssx) - (bx >> M.ssx), (W4 + M.ssx) >> M.ssx);
  const int cbh4 = imin(((M.rows + M.ssy) >> M.ssy) - (by >> M.ssy), (H4 + M.ssy) >> M.ssy);
  if (cbw4 <= 0 || cbh4 <= 0) return;
  mask_chroma(region + 0, by4 >> M.ssy, bx4 >> M.ssx, cbw4, cbh4, r.intra ? 0 : (r.skip ? 1 : 0), r.tx_uv, auv, luv,
              M.ssx, M.ssy);
}

// The right-column (vertical) or bottom-row (horizontal) context a block
// carries out (IntraEdgeContext / InterEdgeContext, lfmask/build.go:101-202),
// read at one local row / column.
int carried_luma_ctx(const Map& M, const pf_lf_record& n, int local, bool right) {
  const int nbw = imin(M.cols - n.mi_col, pf_block_dims[n.block_size][0]);
  const int nbh = imin(M.rows - n.mi_row, pf_block_dims[n.block_size][1]);
  TxGrid g;
  block_grid(g, nbw, nbh, n.tx_y, n.tx_split, n.intra || (n.tx_split[0] == 0 && n.tx_split[1] == 0));
  return right ? g.lw[local][nbw - 1] : g.lh[nbh - 1][local];
}

bool block_fits(const Map& M, const pf_lf_record& n) {
  if (n.block_size >= 22) return false;
  return imin(M.cols - n.mi_col, pf_block_dims[n.block_size][0]) > 0 &&
         imin(M.rows - n.mi_row, pf_block_dims[n.block_size][1]) > 0;
}

// buildBlockFromMap (loop_filter_masks.go:483-551).
void build_from_map_block(const Map& M, uint16_t* masks, int bx, int by) {
  const pf_lf_record& r = M.at(bx, by);
  const int W4 = pf_block_dims[r.block_size][0], H4 = pf_block_dims[r.block_size][1];
  const int bw4 = imin(M.cols - bx, W4), bh4 = imin(M.rows - by, H4);
  if (bw4 <= 0 || bh4 <= 0) return;
  uint8_t ly[32], ay[32], luv[32], auv[32];
  // fillLeftLumaContext / fillAboveLumaContext (:586-646): per row / column,
  // the block owning the neighbouring cell; 2 where there is none.
  for (int y = 0; y < bh4; y++) {
    ly[y] = 2;
    if (bx == 0) continue;
    const pf_lf_record& n = M.at(bx - 1, by + y);
    if (!n.valid || !block_fits(M, n)) continue;
    const int local = by + y - n.mi_row;
    const int nbh = imin(M.rows - n.mi_row, pf_block_dims[n.block_size][1]);
    if (local >= 0 && local < nbh) ly[y] = (uint8_t)carried_luma_ctx(M, n, local, true);
  }
  for (int x = 0; x < bw4; x++) {
    ay[x] = 2;
    if (by == 0) continue;
    const pf_lf_record& n = M.at(bx + x, by - 1);
    if (!n.valid || !block_fits(M, n)) continue;
    const int local = bx + x - n.mi_col;
    const int nbw = imin(M.cols - n.mi_col, pf_block_dims[n.block_size][0]);
    if (local >= 0 && local < nbw) ay[x] = (uint8_t)carried_luma_ctx(M, n, local, false);
  }
  uint8_t *pa = nullptr, *pl = nullptr;
  if (M.hasChroma && r.has_uv && (W4 > M.ssx || (bx & 1)) && (H4 > M.ssy || (by & 1))) {
    const int cbw4 = imin(((M.cols + M.ssx) >> M.ssx) - (bx >> M.ssx), (W4 + M.ssx) >> M.ssx);
    const int cbh4 = imin(((M.rows + M.ssy) >> M.ssy) - (by >> M.ssy), (H4 + M.ssy) >> M.ssy);
    if (cbw4 > 0 && cbh4 > 0) {
      // fillLeftChromaContext / fillAboveChromaContext (:655-680): the
      // bottom-right luma cell of the neighbouring chroma cell's group.
      for (int cy = 0; cy < cbh4; cy++) {
        luv[cy] = 1;
        if (bx == 0) continue;
        const int lr = imin((((by >> M.ssy) + cy) << M.ssy) + M.ssy, M.rows - 1);
        const pf_lf_record& n = M.at(bx - 1, lr);
        if (n.valid && n.has_uv) luv[cy] = pf_tx_dims[n.tx_uv][2] != 0;
      }
      for (int cx = 0; cx < cbw4; cx++) {
        auv[cx] = 1;
        if (by == 0) continue;
        const int lc = imin((((bx >> M.ssx) + cx) << M.ssx) + M.ssx, M.cols - 1);
        const pf_lf_record& n = M.at(lc, by - 1);
        if (n.valid && n.has_uv) auv[cx] = pf_tx_dims[n.tx_uv][3] != 0;
      }
      pa = auv, pl = luv;
    }
  }
  uint16_t* region = masks + ((size_t)(by >> 5) * M.sbw + (bx >> 5)) * PF_LF_MASK_WORDS;
  create_block(M, region, r, bx, by, ay, ly, pa, pl);
}

int clamp_level(int v) { return v < 0 ? 0 : (v > 63 ? 63 : v); }

}  // namespace

extern "C" int oracle_lf_block_levels(const pf_lf_levels* p, int mono, const pf_lf_record* r, uint8_t out[4]) {
  memset(out, 0, 4);
  if (r->ref_frame >= 8 || r->mode > 1) return kErrFilter;
  if (p->level_y[0] == 0 && p->level_y[1] == 0) return kOk;
  const int base[3][2] = {{clamp_level(p->level_y[0]), clamp_level(p->level_y[1])},
                          {clamp_level(p->level_u), clamp_level(p->level_u)},
                          {clamp_level(p->level_v), clamp_level(p->level_v)}};
  uint8_t lv[3][2] = {{0, 0}, {0, 0}, {0, 0}};
  if (!p->delta_lf_present && !p->segmentation_enabled && !p->mode_ref_delta_enabled) {
    for (int i = 0; i < 3; i++)
      for (int e = 0; e < 2; e++) lv[i][e] = (uint8_t)base[i][e];
  } else {
    for (int plane = 0; plane < (mono ? 1 : 3); plane++) {
      for (int edge = 0; edge < 2; edge++) {
        const int b = base[plane][edge];
        if (plane && b == 0) continue;
        int dl = 0;
        if (p->delta_lf_present) dl = p->delta_lf_multi ? r->delta_lf[plane ? plane + 1 : edge] : r->delta_lf_from_base;
        int sd = 0;
        if (p->segmentation_enabled) {
          if (r->segment_id >= 8) return kErrFilter;
          sd = p->segment_delta[r->segment_id][plane ? plane + 1 : edge];
        }
        int lvl = clamp_level(b + dl);
        lvl = clamp_level(lvl + sd);
        if (p->mode_ref_delta_enabled) {
          int d = p->ref_delta[r->ref_frame];
          if (r->ref_frame > 0) d += p->mode_delta[r->mode];
          lvl = clamp_level(lvl + d * (1 << (lvl >> 5)));
        }
        lv[plane][edge] = (uint8_t)lvl;
      }
    }
  }
  out[0] = lv[0][0], out[1] = lv[0][1], out[2] = lv[1][0], out[3] = lv[2][0];
  return kOk;
}

extern "C" int oracle_lf_build(const pf_lf_record* rec, int cols, int rows, const pf_lf_levels* lvp, int ssx, int ssy,
                               int mono, uint16_t* masks, uint8_t* level_cache) {
  Map M{rec, cols, rows, ssx, ssy, !mono, (cols + 31) >> 5};
  const int sbh = (rows + 31) >> 5;
  // The level walk (postfilter_loopfilter_masks.go:135-224) first, for its
  // status: the transform sizes the mask build indexes are checked with it.
  std::vector<uint8_t> lc((size_t)cols * rows * 4, 0);
  for (int row = 0; row < rows; row++) {
    for (int col = 0; col < cols;) {
      const pf_lf_record& r = M.at(col, row);
      if (!r.valid) {
        col++;
        continue;
      }
      const int next = r.mi_col_end;
      if (next <= col || next > cols) return kErrBatch;
      if (r.mi_col != col || r.mi_row != row) {
        col = next;
        continue;
      }
      uint8_t lv[4];
      const int st = oracle_lf_block_levels(lvp, mono, &r, lv);
      if (st) return st;
      if (r.block_size >= 22 || r.tx_y >= 19 || (!mono && r.has_uv && r.tx_uv >= 19)) return kErrBatch;
      const int W4 = pf_block_dims[r.block_size][0], H4 = pf_block_dims[r.block_size][1];
      const int bw4 = imin(cols - col, W4), bh4 = imin(rows - row, H4);
      for (int y = 0; y < bh4; y++)
        for (int x = 0; x < bw4; x++) {
          uint8_t* c = &lc[4 * ((size_t)(row + y) * cols + col + x)];
          c[0] = lv[0], c[1] = lv[1];
        }
      if (!mono) {
        const int cbw4 = imin(((cols + ssx) >> ssx) - (col >> ssx), (W4 + ssx) >> ssx);
        const int cbh4 = imin(((rows + ssy) >> ssy) - (row >> ssy), (H4 + ssy) >> ssy);
        for (int y = 0; y < cbh4; y++)
          for (int x = 0; x < cbw4; x++) {
            uint8_t* c = &lc[4 * ((size_t)((row >> ssy) + y) * cols + (col >> ssx) + x)];
            c[2] = lv[2], c[3] = lv[3];
          }
      }
      col = next;
    }
  }
  memset(masks, 0, (size_t)M.sbw * sbh * PF_LF_MASK_WORDS * 2);
  for (int by = 0; by < rows; by++)
    for (int bx = 0; bx < cols; bx++) {
      const pf_lf_record& r = M.at(bx, by);
      if (!r.valid || r.mi_col != bx || r.mi_row != by || r.block_size >= 22) continue;
      build_from_map_block(M, masks, bx, by);
    }
  memcpy(level_cache, lc.data(), lc.size());
  return kOk;
}

extern "C" int oracle_lf_build_ordered(const pf_lf_record* rec, int cols, int rows, const int32_t* order, int n,
                                       int sb_log2, int ssx, int ssy, int mono, uint16_t* masks) {
  Map M{rec, cols, rows, ssx, ssy, !mono, (cols + 31) >> 5};
  memset(masks, 0, (size_t)M.sbw * ((rows + 31) >> 5) * PF_LF_MASK_WORDS * 2);
  // aY/aUV span the frame width, reset once; lY/lUV one 128-region column,
  // reset at each superblock-row change (resetLeft, :289-300).
  std::vector<uint8_t> aY(cols + 32, 2), aUV(cols + 32, 1);
  uint8_t lY[64], lUV[64];
  int sbRow = -1;
  for (int i = 0; i < n; i++) {
    const int bx = order[i] % cols, by = order[i] / cols;
    const pf_lf_record& r = M.at(bx, by);
    if (r.block_size >= 22) continue;
    if (by >> sb_log2 != sbRow) {
      memset(lY, 2, sizeof(lY));
      memset(lUV, 1, sizeof(lUV));
      sbRow = by >> sb_log2;
    }
    const int W4 = pf_block_dims[r.block_size][0], H4 = pf_block_dims[r.block_size][1];
    uint8_t *pa = nullptr, *pl = nullptr;
    if (M.hasChroma && r.has_uv && (W4 > ssx || (bx & 1)) && (H4 > ssy || (by & 1))) {
      pa = &aUV[bx >> ssx];
      pl = &lUV[(by & 31) >> ssy];
    }
    uint16_t* region = masks + ((size_t)(by >> 5) * M.sbw + (bx >> 5)) * PF_LF_MASK_WORDS;
    create_block(M, region, r, bx, by, &aY[bx], &lY[by & 31], pa, pl);
  }
  return kOk;
}

extern "C" void oracle_lf_mask_block(int kind, uint16_t* region, int by4, int bx4, int w4, int h4, int skip, int tx,
                                     const uint16_t split[2], uint8_t* a, uint8_t* l, int ssx, int ssy) {
  if (kind == 0)
    mask_intra(region, by4, bx4, w4, h4, tx, a, l);
  else if (kind == 1)
    mask_inter(region, by4, bx4, w4, h4, skip, tx, split, a, l);
  else
    mask_chroma(region, by4, bx4, w4, h4, skip, tx, a, l, ssx, ssy);
}
