// pf_oracle.cpp - CPU oracle (test infrastructure only): a scalar restatement
// of goav1's post-reconstruction filter chain.  Every function names the
// reference file:line it follows (paths inside thesyncim/goav1).  It is the
// checker for the CUDA path and the CPU baseline timed by bench.py; the
// product never links it.
#include "pf_oracle.h"

#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pf_tables.h"

namespace {

// ---------------------------------------------------------------------------
// Plane access.  8-bit planes hold bytes; 10/12-bit planes little-endian
// uint16 (frame/buffer.go; cdef/filter.go:366).
struct Plane {
  uint8_t* data = nullptr;
  int64_t stride = 0;
  int bps = 1;
  int w = 0, h = 0, aw = 0, ah = 0;
  int get(int x, int y) const {
    const uint8_t* p = data + (int64_t)y * stride + (int64_t)x * bps;
    return bps == 1 ? p[0] : (int)(p[0] | (p[1] << 8));
  }
  void set(int x, int y, int v) {
    uint8_t* p = data + (int64_t)y * stride + (int64_t)x * bps;
    if (bps == 1) {
      p[0] = (uint8_t)v;
    } else {
      p[0] = (uint8_t)v;
      p[1] = (uint8_t)(v >> 8);
    }
  }
};

Plane plane_of(const pf_frame* f, int p) {
  Plane pl;
  pl.data = (uint8_t*)f->plane[p].data;
  pl.stride = f->plane[p].stride;
  pl.bps = f->bit_depth > 8 ? 2 : 1;
  pl.w = f->plane[p].width;
  pl.h = f->plane[p].height;
  pl.aw = f->plane[p].alloc_width;
  pl.ah = f->plane[p].alloc_height;
  return pl;
}

int imin(int a, int b) { return a < b ? a : b; }
int imax(int a, int b) { return a > b ? a : b; }
int iclip(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
int iabs(int v) { return v < 0 ? -v : v; }
int bitlen(unsigned v) {
  int n = 0;
  while (v) {
    n++;
    v >>= 1;
  }
  return n;
}

// ===========================================================================
// Deblocking
// ===========================================================================

// loopfilter/threshold.go:18-47 (ThresholdsForLevel).
void lf_thresholds(int level, int sharpness, int* E, int* I, int* H) {
  int shift = 0;
  if (sharpness > 0) shift++;
  if (sharpness > 4) shift++;
  int limit = level >> shift;
  if (sharpness > 0 && limit > 9 - sharpness) limit = 9 - sharpness;
  if (limit < 1) limit = 1;
  *I = limit;
  *E = 2 * (level + 2) + limit;
  *H = level >> 4;
}

// loopfilter/sb.go:348-446 (lpfUnit16); at bit depth 8 it reduces exactly to
// lpfUnit8 (sb.go:156-262): bd8 = 0 gives F = 1 and the [-128,127] / [0,255]
// clamps of clampDiff8 / clampPixel8.  One 4-sample edge unit: (x,y) is q0 of
// the first sample, (ax,ay) steps along the edge, (bx,by) across it.
void lpf_unit(Plane& pl, int x, int y, int ax, int ay, int bx, int by, int bd, int E, int I,
              int H, int wd) {
  const int bd8 = bd - 8;
  const int F = 1 << bd8;
  E <<= bd8;
  I <<= bd8;
  H <<= bd8;
  const unsigned twoI = 2u * I, twoF = 2u * F, twoH = 2u * H;
  const int maxPix = (1 << bd) - 1;
  const int diffMin = -128 << bd8, diffMax = (128 << bd8) - 1;
  for (int i = 0; i < 4; i++, x += ax, y += ay) {
    auto P = [&](int k) { return pl.get(x - (k + 1) * bx, y - (k + 1) * by); };
    auto Q = [&](int k) { return pl.get(x + k * bx, y + k * by); };
    auto SP = [&](int k, int v) { pl.set(x - (k + 1) * bx, y - (k + 1) * by, v); };
    auto SQ = [&](int k, int v) { pl.set(x + k * bx, y + k * by, v); };
    int p1 = P(1), p0 = P(0), q0 = Q(0), q1 = Q(1);
    if ((unsigned)(p1 - p0 + I) > twoI || (unsigned)(q1 - q0 + I) > twoI ||
        iabs(p0 - q0) * 2 + (iabs(p1 - q1) >> 1) > E)
      continue;
    int p2 = 0, q2 = 0, p3 = 0, q3 = 0;
    if (wd > 4) {
      p2 = P(2);
      q2 = Q(2);
      if ((unsigned)(p2 - p1 + I) > twoI || (unsigned)(q2 - q1 + I) > twoI) continue;
      if (wd > 6) {
        p3 = P(3);
        q3 = Q(3);
        if ((unsigned)(p3 - p2 + I) > twoI || (unsigned)(q3 - q2 + I) > twoI) continue;
      }
    }
    bool flat8in = false;
    if (wd >= 6) {
      flat8in = (unsigned)(p2 - p0 + F) <= twoF && (unsigned)(p1 - p0 + F) <= twoF &&
                (unsigned)(q1 - q0 + F) <= twoF && (unsigned)(q2 - q0 + F) <= twoF;
      if (wd >= 8 && flat8in)
        flat8in = (unsigned)(p3 - p0 + F) <= twoF && (unsigned)(q3 - q0 + F) <= twoF;
    }
    if (flat8in) {
      if (wd >= 16) {
        int p6 = P(6), p5 = P(5), p4 = P(4), q4 = Q(4), q5 = Q(5), q6 = Q(6);
        if ((unsigned)(p6 - p0 + F) <= twoF && (unsigned)(p5 - p0 + F) <= twoF &&
            (unsigned)(p4 - p0 + F) <= twoF && (unsigned)(q4 - q0 + F) <= twoF &&
            (unsigned)(q5 - q0 + F) <= twoF && (unsigned)(q6 - q0 + F) <= twoF) {
          SP(5, (p6 * 7 + p5 * 2 + p4 * 2 + p3 + p2 + p1 + p0 + q0 + 8) >> 4);
          SP(4, (p6 * 5 + p5 * 2 + p4 * 2 + p3 * 2 + p2 + p1 + p0 + q0 + q1 + 8) >> 4);
          SP(3, (p6 * 4 + p5 + p4 * 2 + p3 * 2 + p2 * 2 + p1 + p0 + q0 + q1 + q2 + 8) >> 4);
          SP(2, (p6 * 3 + p5 + p4 + p3 * 2 + p2 * 2 + p1 * 2 + p0 + q0 + q1 + q2 + q3 + 8) >> 4);
          SP(1, (p6 * 2 + p5 + p4 + p3 + p2 * 2 + p1 * 2 + p0 * 2 + q0 + q1 + q2 + q3 + q4 + 8) >> 4);
          SP(0, (p6 + p5 + p4 + p3 + p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1 + q2 + q3 + q4 + q5 + 8) >> 4);
          SQ(0, (p5 + p4 + p3 + p2 + p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2 + q3 + q4 + q5 + q6 + 8) >> 4);
          SQ(1, (p4 + p3 + p2 + p1 + p0 + q0 * 2 + q1 * 2 + q2 * 2 + q3 + q4 + q5 + q6 * 2 + 8) >> 4);
          SQ(2, (p3 + p2 + p1 + p0 + q0 + q1 * 2 + q2 * 2 + q3 * 2 + q4 + q5 + q6 * 3 + 8) >> 4);
          SQ(3, (p2 + p1 + p0 + q0 + q1 + q2 * 2 + q3 * 2 + q4 * 2 + q5 + q6 * 4 + 8) >> 4);
          SQ(4, (p1 + p0 + q0 + q1 + q2 + q3 * 2 + q4 * 2 + q5 * 2 + q6 * 5 + 8) >> 4);
          SQ(5, (p0 + q0 + q1 + q2 + q3 + q4 * 2 + q5 * 2 + q6 * 7 + 8) >> 4);
          continue;
        }
      }
      if (wd >= 8) {
        SP(2, (p3 * 3 + p2 * 2 + p1 + p0 + q0 + 4) >> 3);
        SP(1, (p3 * 2 + p2 + p1 * 2 + p0 + q0 + q1 + 4) >> 3);
        SP(0, (p3 + p2 + p1 + p0 * 2 + q0 + q1 + q2 + 4) >> 3);
        SQ(0, (p2 + p1 + p0 + q0 * 2 + q1 + q2 + q3 + 4) >> 3);
        SQ(1, (p1 + p0 + q0 + q1 * 2 + q2 + q3 * 2 + 4) >> 3);
        SQ(2, (p0 + q0 + q1 + q2 * 2 + q3 * 3 + 4) >> 3);
        continue;
      }
      SP(1, (p2 * 3 + p1 * 2 + p0 * 2 + q0 + 4) >> 3);
      SP(0, (p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1 + 4) >> 3);
      SQ(0, (p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2 + 4) >> 3);
      SQ(1, (p0 + q0 * 2 + q1 * 2 + q2 * 3 + 4) >> 3);
      continue;
    }
    bool hev = (unsigned)(p1 - p0 + H) > twoH || (unsigned)(q1 - q0 + H) > twoH;
    int f;
    if (hev)
      f = imin(imax(imin(imax(p1 - q1, diffMin), diffMax) + 3 * (q0 - p0), diffMin), diffMax);
    else
      f = imin(imax(3 * (q0 - p0), diffMin), diffMax);
    int f1 = imin(f + 4, diffMax) >> 3;
    int f2 = imin(f + 3, diffMax) >> 3;
    SP(0, imin(imax(p0 + f2, 0), maxPix));
    SQ(0, imin(imax(q0 - f1, 0), maxPix));
    if (!hev) {
      f = (f1 + 1) >> 1;
      SP(1, imin(imax(p1 + f, 0), maxPix));
      SQ(1, imin(imax(q1 - f, 0), maxPix));
    }
  }
}

// loopfilter/sb.go:99-113 (sbUnitWidth).
int sb_unit_width(const uint32_t vm[3], bool luma, uint32_t bit) {
  if (vm[2] & bit) return 16;
  if (vm[1] & bit) return luma ? 8 : 6;
  return 4;
}

uint32_t lane_mask(int n) { return n >= 32 ? 0xffffffffu : ((1u << n) - 1u); }

// postfilter_loopfilter_masks_sb.go:21-188 (applyLoopFilterMaskPlaneRangeSB)
// with the scalar superblock kernels loopfilter/sb.go:115-153, :302-336.
void lf_plane_range(const pf_frame* fr, const pf_loop_filter& lf, int plane, int dir, int rRow) {
  Plane pl = plane_of(fr, plane);
  const int bd = fr->bit_depth;
  const int ssx = plane ? fr->ss_x : 0, ssy = plane ? fr->ss_y : 0;
  // frameWorkLoopFilterPlaneSize (postfilter_loopfilter.go:2569-2597).
  const int posW = ((plane ? (fr->width + ssx) >> ssx : fr->width) + 3) & ~3;
  const int posH = ((plane ? (fr->height + ssy) >> ssy : fr->height) + 3) & ~3;
  const int w4 = posW >> 2, h4 = posH >> 2;
  const int cols = lf.mi_cols;
  const uint8_t* cells = lf.level_cache;
  const int comp_v = plane == 0 ? 0 : plane + 1, comp_h = plane == 0 ? 1 : plane + 1;
  const bool luma = plane == 0;
  const int regionW = 32 >> ssx, regionH = 32 >> ssy;
  const int laneV = luma ? 16 : (16 >> ssy), laneH = luma ? 16 : (16 >> ssx);
  const int nk = luma ? 3 : 2;
  for (int rCol = 0; rCol < lf.sb128_w; rCol++) {
    const uint16_t* region = lf.masks + (size_t)(rRow * lf.sb128_w + rCol) * PF_LF_MASK_WORDS;
    auto mword = [&](int d, int pos, int k, int half) -> uint32_t {
      if (luma) return region[((d * 32 + pos) * 3 + k) * 2 + half];
      return region[384 + ((d * 32 + pos) * 2 + k) * 2 + half];
    };
    const int baseRow = rRow * regionH, baseCol = rCol * regionW;
    const int nRows = imin(regionH, h4 - baseRow), nCols = imin(regionW, w4 - baseCol);
    if (nRows <= 0 || nCols <= 0) continue;
    if (dir == 0) {
      const uint32_t rowMask = lane_mask(nRows);
      for (int pos = 0; pos < nCols; pos++) {
        const int col = baseCol + pos;
        if (col == 0) continue;
        uint32_t vm[3] = {0, 0, 0};
        for (int k = 0; k < nk; k++) vm[k] = (mword(0, pos, k, 0) | (mword(0, pos, k, 1) << laneV)) & rowMask;
        uint32_t all = vm[0] | vm[1] | vm[2];
        while (all) {
          int n = __builtin_ctz(all);
          uint32_t bit = 1u << n;
          all &= ~bit;
          int li = (baseRow + n) * cols + col;
          int L = cells[4 * li + comp_v];
          if (L == 0) L = cells[4 * (li - 1) + comp_v];
          if (L == 0) continue;
          int E, I, H;
          lf_thresholds(L, lf.sharpness, &E, &I, &H);
          lpf_unit(pl, col * 4, (baseRow + n) * 4, 0, 1, 1, 0, bd, E, I, H, sb_unit_width(vm, luma, bit));
        }
      }
    } else {
      const uint32_t colMask = lane_mask(nCols);
      for (int pos = 0; pos < nRows; pos++) {
        const int row = baseRow + pos;
        if (row == 0) continue;
        uint32_t vm[3] = {0, 0, 0};
        for (int k = 0; k < nk; k++) vm[k] = (mword(1, pos, k, 0) | (mword(1, pos, k, 1) << laneH)) & colMask;
        uint32_t all = vm[0] | vm[1] | vm[2];
        while (all) {
          int n = __builtin_ctz(all);
          uint32_t bit = 1u << n;
          all &= ~bit;
          int li = row * cols + baseCol + n;
          int L = cells[4 * li + comp_h];
          if (L == 0) L = cells[4 * (li - cols) + comp_h];
          if (L == 0) continue;
          int E, I, H;
          lf_thresholds(L, lf.sharpness, &E, &I, &H);
          lpf_unit(pl, (baseCol + n) * 4, row * 4, 1, 0, 0, 1, bd, E, I, H, sb_unit_width(vm, luma, bit));
        }
      }
    }
  }
}

// postfilter_loopfilter_masks.go:229-268 (applyLoopFilterEdgesFromMasksInPlanePassOrder):
// per 128x128 region row, every plane's vertical edges then every plane's
// horizontal edges; chroma gated off when both luma frame levels are zero or
// the plane's base level is zero (:232-252, postfilter_loopfilter.go:171-191).
int do_loop_filter(const pf_frame* fr, const pf_frame_side* side) {
  const pf_loop_filter& lf = side->lf;
  if (!lf.masks || !lf.level_cache) return PF_ERR_INVALID_FILTER;
  const bool lumaZero = lf.level_y[0] == 0 && lf.level_y[1] == 0;
  const int maxPlane = fr->mono ? 0 : 2;
  for (int rRow = 0; rRow < lf.sb128_h; rRow++) {
    for (int dir = 0; dir < 2; dir++) {
      for (int plane = 0; plane <= maxPlane; plane++) {
        if (plane != 0) {
          int base = plane == 1 ? lf.level_u : lf.level_v;
          if (lumaZero || base == 0) continue;
        }
        lf_plane_range(fr, lf, plane, dir, rRow);
      }
    }
  }
  return PF_OK;
}

// ===========================================================================
// CDEF
// ===========================================================================
constexpr int kBStride = 144;         // cdef/constants.go:9-19
constexpr int kVeryLarge = 0x4000;
constexpr int kInputSize = kBStride * (128 + 4);

const int kCdefDirections[12][2] = {  // cdef/filter.go:53-66
    {1 * kBStride, 2 * kBStride},      {1 * kBStride, 2 * kBStride - 1},
    {-1 * kBStride + 1, -2 * kBStride + 2}, {1, -1 * kBStride + 2},
    {1, 2},                            {1, 1 * kBStride + 2},
    {1 * kBStride + 1, 2 * kBStride + 2}, {1 * kBStride, 2 * kBStride + 1},
    {1 * kBStride, 2 * kBStride},      {1 * kBStride, 2 * kBStride - 1},
    {-1 * kBStride + 1, -2 * kBStride + 2}, {1, -1 * kBStride + 2},
};
const int kDivTable[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};  // direction.go:13

// cdef/direction.go:432-501 (finishDirection and the three cost helpers).
int finish_direction(int32_t partial[8][15], int32_t* variance) {
  int32_t cost[8];
  for (int d = 0; d < 8; d++) {
    const int32_t* p = partial[d];
    int32_t c = 0;
    if (d == 2 || d == 6) {
      for (int i = 0; i < 8; i++) c += p[i] * p[i];
      c *= kDivTable[8];
    } else if (d == 0 || d == 4) {
      for (int i = 0; i < 7; i++) c += (p[i] * p[i] + p[14 - i] * p[14 - i]) * kDivTable[i + 1];
      c += p[7] * p[7] * kDivTable[8];
    } else {
      c = (p[3] * p[3] + p[4] * p[4] + p[5] * p[5] + p[6] * p[6] + p[7] * p[7]) * kDivTable[8] +
          (p[0] * p[0] + p[10] * p[10]) * kDivTable[2] + (p[1] * p[1] + p[9] * p[9]) * kDivTable[4] +
          (p[2] * p[2] + p[8] * p[8]) * kDivTable[6];
    }
    cost[d] = c;
  }
  int best = 0;
  int32_t bestCost = cost[0];
  for (int d = 1; d < 8; d++)
    if (cost[d] > bestCost) {
      best = d;
      bestCost = cost[d];
    }
  *variance = (bestCost - cost[(best + 4) & 7]) >> 10;
  return best;
}

// cdef/direction.go:37-79 (findDirectionScalar).
int find_dir(const uint16_t* img, int stride, int coeffShift, int32_t* variance) {
  int32_t partial[8][15];
  memset(partial, 0, sizeof(partial));
  for (int i = 0; i < 8; i++) {
    for (int j = 0; j < 8; j++) {
      int32_t x = (int32_t)(img[i * stride + j] >> coeffShift) - 128;
      partial[0][i + j] += x;
      partial[1][i + (j >> 1)] += x;
      partial[2][i] += x;
      partial[3][3 + i - (j >> 1)] += x;
      partial[4][7 + i - j] += x;
      partial[5][3 - (i >> 1) + j] += x;
      partial[6][j] += x;
      partial[7][(i >> 1) + j] += x;
    }
  }
  return finish_direction(partial, variance);
}

// cdef/filter.go:173-191 and filter_u8.go:124-134.
int constrain_shift(int threshold, int damping) {
  if (threshold == 0) return 0;
  return imax(damping - (bitlen((unsigned)threshold) - 1), 0);
}
int constrain(int diff, int threshold, int shift) {
  int a = iabs(diff);
  int l = imin(imax(threshold - (a >> shift), 0), a);
  return diff < 0 ? -l : l;
}
int cdef_round(int x, int sum) { return x + ((8 + sum - (sum < 0)) >> 4); }

// cdef/filter.go:79-169 (filterBlockPureGo).
void filter_block(uint16_t* dst, int dstStride, const uint16_t* in, int origin, int pri, int sec,
                  int dir, int priDamp, int secDamp, int coeffShift, int w, int h) {
  static const int kPriTaps[2][2] = {{4, 2}, {3, 3}};  // cdef/filter.go:68
  const int* priTaps = kPriTaps[(pri >> coeffShift) & 1];
  const int pri0 = kCdefDirections[dir + 2][0], pri1 = kCdefDirections[dir + 2][1];
  const int s0a = kCdefDirections[dir + 4][0], s0b = kCdefDirections[dir + 4][1];
  const int s1a = kCdefDirections[dir][0], s1b = kCdefDirections[dir][1];
  const int priShift = constrain_shift(pri, priDamp), secShift = constrain_shift(sec, secDamp);
  for (int r = 0; r < h; r++) {
    for (int c = 0; c < w; c++) {
      const int base = origin + r * kBStride + c;
      const int x = in[base];
      if (pri == 0 && sec == 0) {
        dst[r * dstStride + c] = (uint16_t)x;
        continue;
      }
      int sum = 0;
      int a0 = in[base + pri0], a1 = in[base - pri0], a2 = in[base + pri1], a3 = in[base - pri1];
      int b0 = in[base + s0a], b1 = in[base - s0a], b2 = in[base + s1a], b3 = in[base - s1a];
      int b4 = in[base + s0b], b5 = in[base - s0b], b6 = in[base + s1b], b7 = in[base - s1b];
      if (pri) {
        sum += priTaps[0] * (constrain(a0 - x, pri, priShift) + constrain(a1 - x, pri, priShift)) +
               priTaps[1] * (constrain(a2 - x, pri, priShift) + constrain(a3 - x, pri, priShift));
      }
      if (sec) {
        sum += 2 * (constrain(b0 - x, sec, secShift) + constrain(b1 - x, sec, secShift) +
                    constrain(b2 - x, sec, secShift) + constrain(b3 - x, sec, secShift)) +
               constrain(b4 - x, sec, secShift) + constrain(b5 - x, sec, secShift) +
               constrain(b6 - x, sec, secShift) + constrain(b7 - x, sec, secShift);
      }
      int y = cdef_round(x, sum);
      if (pri && sec) {
        const int m = kVeryLarge - 1;
        int hi = x, lo = x;
        const int t[12] = {a0, a1, a2, a3, b0, b1, b2, b3, b4, b5, b6, b7};
        for (int k = 0; k < 12; k++) {
          hi = imax(hi, t[k] & m);
          lo = imin(lo, t[k]);
        }
        y = imin(imax(y, lo), hi);
      }
      dst[r * dstStride + c] = (uint16_t)y;
    }
  }
}

// cdef/filter.go:603-612 (adjustStrength).
int adjust_strength(int strength, int32_t variance) {
  if (variance == 0) return 0;
  int i = 0;
  int32_t v = variance >> 6;
  if (v != 0) i = imin(bitlen((unsigned)v) - 1, 12);
  return (strength * (4 + i) + 8) >> 4;
}

struct CdefGrid {
  uint8_t dir[16][16];
  int32_t var[16][16];
};

// Packed strength -> (level, secondary) (cdef/strength.go:12-22).
void decode_strength(int packed, int* pri, int* sec) {
  *pri = packed >> 2;
  *sec = packed & 3;
  if (*sec == 3) *sec = 4;
}

bool cdef_plane_has_filtering(const pf_cdef& c, int plane) {  // postfilter_cdef.go:1355-1368
  int limit = imin(c.strength_count, 8);
  for (int i = 0; i < limit; i++) {
    if (plane == 0 && c.y_strength[i]) return true;
    if (plane != 0 && c.uv_strength[i]) return true;
  }
  return false;
}

// Reads a sample of the pre-CDEF snapshot as a uint16.
struct Snapshot {
  std::vector<uint16_t> pix;
  int w = 0, h = 0;
};

// postfilter_cdef.go:1101-1123 (frameWorkFillCDEFInputSentinels) and
// :1151-1249 (frameWorkCopyCDEFInput) including the row/column replicate
// quirk for non-final units whose plane ends inside the halo.
void cdef_stage_input(uint16_t* input, const Snapshot& src, int unitX, int unitY, int unitW, int unitH) {
  const int fillW = unitW + 16, fillH = unitH + 4;
  for (int row = 0; row < 2; row++)
    for (int i = 0; i < fillW; i++) input[row * kBStride + i] = kVeryLarge;
  for (int row = 2; row < 2 + unitH; row++) {
    for (int i = 0; i < 8; i++) input[row * kBStride + i] = kVeryLarge;
    for (int i = 0; i < 8; i++) input[row * kBStride + 8 + unitW + i] = kVeryLarge;
  }
  for (int row = 2 + unitH; row < fillH; row++)
    for (int i = 0; i < fillW; i++) input[row * kBStride + i] = kVeryLarge;

  const int srcX0 = imax(unitX - 8, 0), srcY0 = imax(unitY - 2, 0);
  const int srcX1 = imin(unitX + unitW + 8, src.w), srcY1 = imin(unitY + unitH + 2, src.h);
  const int copyW = srcX1 - srcX0, copyH = srcY1 - srcY0;
  if (copyW <= 0 || copyH <= 0) return;
  const int dstOff = 2 * kBStride + 8 + (srcY0 - unitY) * kBStride + (srcX0 - unitX);
  for (int r = 0; r < copyH; r++)
    for (int c = 0; c < copyW; c++)
      input[dstOff + r * kBStride + c] = src.pix[(size_t)(srcY0 + r) * src.w + srcX0 + c];
  const int wantY1 = unitY + unitH + 2;
  const bool rowExtend = srcY1 < wantY1 && srcY1 > 0 && unitY + unitH < src.h;
  if (rowExtend) {
    const int last = dstOff + (copyH - 1) * kBStride;
    for (int row = srcY1; row < wantY1; row++) {
      const int ext = dstOff + (row - srcY0) * kBStride;
      for (int c = 0; c < copyW; c++) input[ext + c] = input[last + c];
    }
  }
  const int wantX1 = unitX + unitW + 8;
  if (srcX1 < wantX1 && srcX1 > 0 && unitX + unitW < src.w) {
    const int extRows = rowExtend ? wantY1 - srcY0 : copyH;
    for (int row = 0; row < extRows; row++) {
      const int ro = dstOff + row * kBStride;
      const uint16_t last = input[ro + copyW - 1];
      for (int i = ro + copyW; i < ro + (wantX1 - srcX0); i++) input[i] = last;
    }
  }
}

// cdef/filter.go:614-633 (convertChromaDirections).
void convert_chroma_dirs(CdefGrid& g, const std::vector<std::pair<int, int>>& blocks, int xdec) {
  static const uint8_t conv422[8] = {7, 0, 2, 4, 5, 6, 6, 6};
  static const uint8_t conv440[8] = {1, 2, 2, 2, 3, 4, 6, 0};
  for (auto& b : blocks) {
    uint8_t& d = g.dir[b.first][b.second];
    d = xdec ? conv422[d] : conv440[d];
  }
}

// Per-unit filter-block loop of filterFrameBlocks + filterUnitBlocksPureGo
// (cdef/filter.go:231-241, :396-470, :490-543).
void cdef_filter_unit(uint16_t* unitDst, const uint16_t* input, const std::vector<std::pair<int, int>>& blocks,
                      CdefGrid& grid, int plane, int xdec, int ydec, int level, int secondary,
                      int damping0, int coeffShift, bool deriveDirections) {
  const int pri = level << coeffShift;
  const int sec = secondary << coeffShift;
  int damping = damping0 + coeffShift;
  if (plane != 0) damping--;
  const int bwLog2 = 3 - xdec, bhLog2 = 3 - ydec;
  const int bw = 1 << bwLog2, bh = 1 << bhLog2;
  const int origin = 2 * kBStride + 8;
  if (plane == 0 && deriveDirections) {
    for (auto& b : blocks) {
      const int srcOrigin = origin + ((b.first * kBStride) << bhLog2) + (b.second << bwLog2);
      int32_t var;
      grid.dir[b.first][b.second] = (uint8_t)find_dir(input + srcOrigin, kBStride, coeffShift, &var);
      grid.var[b.first][b.second] = var;
    }
  }
  if (deriveDirections && plane == 1 && xdec != ydec) convert_chroma_dirs(grid, blocks, xdec);
  const bool lumaAdjust = plane == 0 && (deriveDirections || pri != 0);
  for (auto& b : blocks) {
    int strength = pri;
    if (lumaAdjust) strength = adjust_strength(pri, grid.var[b.first][b.second]);
    const int dir = pri != 0 ? grid.dir[b.first][b.second] : 0;
    const int srcOrigin = origin + ((b.first * kBStride) << bhLog2) + (b.second << bwLog2);
    uint16_t* d = unitDst + ((b.first << bhLog2) * kBStride) + (b.second << bwLog2);
    filter_block(d, kBStride, input, srcOrigin, strength, sec, dir, damping, damping, coeffShift, bw, bh);
  }
}

// postfilter_cdef.go:525-710 (applyCDEFPostFilterRows, snapshot walk) and
// :960-1035 (cdefPlaneWalker.applySnapshot), :936-956 (unitStrength),
// :1041-1047 (frameWorkCDEFPlaneNeedsPrimaryDirection), :1390-1412
// (frameWorkCDEFAlignedPlane), :1544-1561 (block list from the noskip word).
int do_cdef(const pf_frame* fr, const pf_frame_side* side, int* unitsOut) {
  const pf_cdef& c = side->cdef;
  const bool mono = fr->mono;
  bool any = false;
  for (int i = 0; i < imin(c.strength_count, 8); i++)
    if (c.y_strength[i] || (!mono && c.uv_strength[i])) any = true;
  if (!any) return PF_OK;
  const int cols = (fr->width + 63) / 64, rows = (fr->height + 63) / 64;
  if (!c.index || !c.read || c.index_stride < cols || c.index_rows < rows) return PF_ERR_INVALID_CDEF;
  const bool chromaFiltering = !mono && cdef_plane_has_filtering(c, 1);
  const int coeffShift = fr->bit_depth - 8;
  std::vector<CdefGrid> grids((size_t)cols * rows);
  memset(grids.data(), 0, grids.size() * sizeof(CdefGrid));
  std::vector<uint16_t> input(kInputSize), unitDst(kInputSize);
  int units = 0;
  for (int plane = 0; plane < (mono ? 1 : 3); plane++) {
    bool process = cdef_plane_has_filtering(c, plane);
    if (plane == 0 && !process) process = chromaFiltering;
    if (!process) continue;
    const int xdec = plane ? fr->ss_x : 0, ydec = plane ? fr->ss_y : 0;
    Plane pl = plane_of(fr, plane);
    // MI-aligned plane extent (frameWorkCDEFAlignedPlane).
    int aw = ((fr->width + 7) & ~7) >> xdec, ah = ((fr->height + 7) & ~7) >> ydec;
    aw = imax(aw, pl.w);
    ah = imax(ah, pl.h);
    aw = imin(aw, (int)(pl.stride / pl.bps));
    Snapshot src;
    src.w = aw;
    src.h = ah;
    src.pix.resize((size_t)aw * ah);
    for (int y = 0; y < ah; y++)
      for (int x = 0; x < aw; x++) src.pix[(size_t)y * aw + x] = (uint16_t)pl.get(x, y);
    const int unitSizeX = 64 >> xdec, unitSizeY = 64 >> ydec;
    const int bw = 8 >> xdec, bh = 8 >> ydec;
    for (int ur = 0; ur < rows; ur++) {
      for (int uc = 0; uc < cols; uc++) {
        const int mapOff = ur * c.index_stride + uc;
        if (!c.read[mapOff]) continue;
        const int idx = c.index[mapOff];
        if (idx >= c.strength_count || idx >= 8) return PF_ERR_INVALID_CDEF;
        const int packed = plane == 0 ? c.y_strength[idx] : c.uv_strength[idx];
        bool needPrimary;
        if (plane == 0)
          needPrimary = (c.y_strength[idx] >> 2) != 0 || (chromaFiltering && (c.uv_strength[idx] >> 2) != 0);
        else
          needPrimary = (c.uv_strength[idx] >> 2) != 0;
        const bool directionOnly = plane == 0 && chromaFiltering && packed == 0 && (c.uv_strength[idx] >> 2) != 0;
        if (packed == 0 && !directionOnly) continue;
        const int unitX = (uc * 64) >> xdec, unitY = (ur * 64) >> ydec;
        const int unitW = imin(unitSizeX, src.w - unitX), unitH = imin(unitSizeY, src.h - unitY);
        if (unitW <= 0 || unitH <= 0) continue;
        const int bcols = (unitW + bw - 1) / bw, brows = (unitH + bh - 1) / bh;
        uint64_t m = ~0ull;
        if (c.noskip) {
          m = 0;
          for (int i = 0; i < 8; i++) m |= (uint64_t)c.noskip[(size_t)(ur * cols + uc) * 8 + i] << (8 * i);
        }
        std::vector<std::pair<int, int>> blocks;
        const uint64_t colMask = (1ull << bcols) - 1;
        for (int by = 0; by < brows; by++) {
          uint64_t rowBits = (m >> (by * 8)) & colMask;
          for (int bx = 0; bx < bcols; bx++)
            if (rowBits & (1ull << bx)) blocks.emplace_back(by, bx);
        }
        if (blocks.empty()) continue;
        cdef_stage_input(input.data(), src, unitX, unitY, unitW, unitH);
        if (!directionOnly && (int)blocks.size() < bcols * brows) {
          for (int r = 0; r < unitH; r++)
            for (int x = 0; x < unitW; x++)
              unitDst[r * kBStride + x] = src.pix[(size_t)(unitY + r) * src.w + unitX + x];
        }
        int level, secondary;
        decode_strength(packed, &level, &secondary);
        cdef_filter_unit(unitDst.data(), input.data(), blocks, grids[(size_t)ur * cols + uc], plane, xdec, ydec,
                         level, secondary, c.damping, coeffShift, needPrimary);
        if (directionOnly) continue;
        for (int r = 0; r < unitH; r++)
          for (int x = 0; x < unitW; x++) pl.set(unitX + x, unitY + r, unitDst[r * kBStride + x]);
        units++;
      }
    }
  }
  if (unitsOut) *unitsOut = units;
  return PF_OK;
}

// ===========================================================================
// Loop restoration
// ===========================================================================
constexpr int kLRBorder = 3, kLRCtxVert = 2, kLRExtraHorz = 4, kLRUnitOffset = 8;

struct LRGrid {
  int type = 0, unitSize = 0, W = 0, H = 0, ssx = 0, ssy = 0, horz = 0, vert = 0;
};

// tile/restoration_schedule.go:61-109 (BuildRestorationPlaneGrid) and
// :400-409 (countRestorationUnits).
LRGrid lr_grid(const pf_frame* fr, const pf_restoration& lr, int plane) {
  LRGrid g;
  g.type = lr.type[plane];
  g.unitSize = plane ? lr.unit_size_uv : lr.unit_size_y;
  g.ssx = plane ? fr->ss_x : 0;
  g.ssy = plane ? fr->ss_y : 0;
  g.W = (fr->width + g.ssx) >> g.ssx;
  g.H = (fr->height + g.ssy) >> g.ssy;
  if (g.type != PF_LR_NONE && g.unitSize > 0) {
    auto count = [&](int size) {
      int u = (size + (g.unitSize >> 1)) / g.unitSize;
      return u == 0 ? 1 : u;
    };
    g.horz = count(g.W);
    g.vert = count(g.H);
  }
  return g;
}

struct LRLines {  // tile/restoration_boundary.go:20-31
  std::vector<uint16_t> above, below;
  int stride = 0;
};

// tile/restoration_boundary.go:192-255 (SaveRestorationBoundaryLinesFromFramePlaneRows),
// :454-521 (line saves) and :879-926 (finishRestorationBoundaryLines).
// coded != null: a super-resolved frame's deblock save
// (tile/restoration_boundary.go:257-406): each saved row is the coded frame's
// row over its MI-aligned span, upscaled to the plane width g.W
// (superres.UpscalePlaneCoded); fr is then only the geometry.
void lr_save_lines(const pf_frame* fr, int plane, const LRGrid& g, LRLines& lines, bool afterCDEF,
                   const pf_frame* coded = nullptr) {
  Plane pl = plane_of(fr, plane);
  const int stripeH = 64 >> g.ssy, off = kLRUnitOffset >> g.ssy;
  const int nStripes = (g.H + off) / stripeH + 2;
  lines.stride = g.W + 2 * kLRExtraHorz;
  if (lines.above.empty()) {
    lines.above.assign((size_t)lines.stride * nStripes * kLRCtxVert, 0);
    lines.below.assign((size_t)lines.stride * nStripes * kLRCtxVert, 0);
  }
  auto finish = [&](std::vector<uint16_t>& buf, int stripe, int saved) {
    uint16_t* l0 = &buf[(size_t)(stripe * kLRCtxVert) * lines.stride];
    if (saved == 1) memcpy(l0 + lines.stride, l0, lines.stride * sizeof(uint16_t));
    for (int i = 0; i < kLRCtxVert; i++) {
      uint16_t* line = l0 + i * lines.stride;
      for (int j = 0; j < kLRExtraHorz; j++) {
        line[j] = line[kLRExtraHorz];
        line[kLRExtraHorz + g.W + j] = line[kLRExtraHorz + g.W - 1];
      }
    }
  };
  auto save_row = [&](std::vector<uint16_t>& buf, int stripe, int ctxRow, int srcRow) {
    uint16_t* line = &buf[(size_t)(stripe * kLRCtxVert + ctxRow) * lines.stride];
    if (coded) {
      Plane cp = plane_of(coded, plane);
      const int cw = (coded->width + g.ssx) >> g.ssx, aw = ((coded->width + 7) & ~7) >> g.ssx;
      std::vector<uint16_t> row(aw);
      for (int x = 0; x < aw; x++) row[x] = (uint16_t)cp.get(x, srcRow);
      oracle_superres_row(row.data(), aw, cw, line + kLRExtraHorz, g.W, coded->bit_depth);
      return;
    }
    for (int x = 0; x < g.W; x++) line[kLRExtraHorz + x] = (uint16_t)pl.get(x, srcRow);
  };
  for (int s = 0;; s++) {
    const int y0 = imax(0, s * stripeH - off);
    if (y0 >= g.H) break;
    const int y1 = imin((s + 1) * stripeH - off, g.H);
    const bool deblockAbove = s > 0, deblockBelow = y1 < g.H;
    if (!afterCDEF) {
      if (deblockAbove) {
        const int row = y0 - kLRCtxVert;
        const int n = imin(kLRCtxVert, g.H - row);
        for (int i = 0; i < n; i++) save_row(lines.above, s, i, row + i);
        finish(lines.above, s, n);
      }
      if (deblockBelow) {
        const int n = imin(kLRCtxVert, g.H - y1);
        for (int i = 0; i < n; i++) save_row(lines.below, s, i, y1 + i);
        finish(lines.below, s, n);
      }
    } else {
      if (!deblockAbove) {
        for (int i = 0; i < kLRCtxVert; i++) save_row(lines.above, s, i, y0);
        finish(lines.above, s, kLRCtxVert);
      }
      if (!deblockBelow) {
        for (int i = 0; i < kLRCtxVert; i++) save_row(lines.below, s, i, y1 - 1);
        finish(lines.below, s, kLRCtxVert);
      }
    }
  }
}

// restoration/wiener.go:59-80, :132-196, :202-211.
void wiener_rounds(int bd, int* r0, int* r1) {
  int round0 = 3, round1 = 2 * 7 - 3;
  int range = bd + 7 - round0 + 2;
  if (range > 16) {
    round0 += range - 16;
    round1 -= range - 16;
  }
  *r0 = round0;
  *r1 = round1;
}
int32_t rpot(int32_t v, int bits) { return bits <= 0 ? v : (v + (int32_t)(1 << (bits - 1))) >> bits; }
uint32_t rpotu(uint32_t v, int bits) { return bits <= 0 ? v : (v + (uint32_t)(1u << (bits - 1))) >> bits; }

void wiener_apply(const uint16_t* src, int sstride, uint16_t* dst, int dstride, int w, int h,
                  const int16_t* vf, const int16_t* hf, int bd) {
  int round0, round1;
  wiener_rounds(bd, &round0, &round1);
  std::vector<uint16_t> temp((size_t)w * (h + 6));
  const int32_t limit = 1 << (bd + 1 + 7 - round0);
  const int32_t offH = 1 << (bd + 7 - 1);
  for (int row = -3; row < h + 3; row++) {
    for (int col = 0; col < w; col++) {
      const uint16_t* s = src + (ptrdiff_t)row * sstride + col - 3;
      int32_t sum = ((int32_t)s[3] << 7) + offH;
      for (int k = 0; k < 7; k++) sum += (int32_t)s[k] * hf[k];
      int32_t v = rpot(sum, round0);
      temp[(size_t)(row + 3) * w + col] = (uint16_t)std::min(std::max(v, 0), limit - 1);
    }
  }
  const int32_t offV = 1 << (bd + round1 - 1);
  const int32_t maxV = (1 << bd) - 1;
  for (int row = 0; row < h; row++) {
    for (int col = 0; col < w; col++) {
      int32_t c3 = temp[(size_t)(row + 3) * w + col];
      int32_t sum = (c3 << 7) - offV;
      for (int k = 0; k < 7; k++) sum += (int32_t)temp[(size_t)(row + k) * w + col] * vf[k];
      int32_t v = rpot(sum, round1);
      dst[(size_t)row * dstride + col] = (uint16_t)std::min(std::max(v, 0), maxV);
    }
  }
}

// restoration/selfguided.go:111-127 (DecodeSGRXQ).
void sgr_decode_xq(const int8_t* xqd, int set, int16_t* xq) {
  const int r0 = pf_sgr_params[set][0], r1 = pf_sgr_params[set][1];
  if (r0 == 0) {
    xq[0] = 0;
    xq[1] = (int16_t)(128 - xqd[1]);
  } else if (r1 == 0) {
    xq[0] = xqd[0];
    xq[1] = 0;
  } else {
    xq[0] = xqd[0];
    xq[1] = (int16_t)(128 - xq[0] - xqd[1]);
  }
}

// restoration/selfguided.go:324-359 (calculateIntermediateFull) + :361-390 (boxsum).
void sgr_intermediate(const std::vector<int32_t>& dgd, int dgdStride, int w, int h, int bd, int set, int radiusIdx,
                      int pass, std::vector<int32_t>& A, std::vector<int32_t>& B, int bufStride) {
  std::fill(A.begin(), A.end(), 0);
  std::fill(B.begin(), B.end(), 0);
  const int r = pf_sgr_params[set][radiusIdx];
  const int s = pf_sgr_params[set][2 + radiusIdx];
  const int wext = w + 6, hext = h + 6;
  for (int row = 0; row < hext; row++) {
    const int y0 = imax(0, row - r), y1 = imin(hext - 1, row + r);
    for (int col = 0; col < wext; col++) {
      const int x0 = imax(0, col - r), x1 = imin(wext - 1, col + r);
      int32_t sum = 0, sq = 0;
      for (int y = y0; y <= y1; y++)
        for (int x = x0; x <= x1; x++) {
          int32_t v = dgd[(size_t)y * dgdStride + x];
          sum += v;
          sq += v * v;
        }
      B[(size_t)row * bufStride + col] = sum;
      A[(size_t)row * bufStride + col] = sq;
    }
  }
  const int aOrigin = 3 * bufStride + 3;
  const int step = pass ? 2 : 1;
  const uint32_t n = (uint32_t)((2 * r + 1) * (2 * r + 1));
  for (int row = -1; row < h + 1; row += step) {
    for (int col = -1; col < w + 1; col++) {
      const size_t k = (size_t)(aOrigin + row * bufStride + col);
      const uint32_t a = (uint32_t)rpot(A[k], 2 * (bd - 8));
      const uint32_t b = (uint32_t)rpot(B[k], bd - 8);
      uint32_t p = 0;
      if (a * n >= b * b) p = a * n - b * b;
      uint32_t z = rpotu(p * (uint32_t)s, 20);
      if (z > 255) z = 255;
      A[k] = pf_sgr_x_by_xplus1[z];
      B[k] = (int32_t)rpotu((uint32_t)(256 - A[k]) * (uint32_t)B[k] * (uint32_t)pf_sgr_one_by_x[n - 1], 12);
    }
  }
}

// restoration/selfguided.go:132-310 (ApplySelfguidedRestoration, selfguidedFast,
// selfguided, sgrWeightedRow with its int16 wrap).
void sgr_apply(const uint16_t* src, int sstride, uint16_t* dst, int dstride, int w, int h, int set,
               const int8_t* xqd, int bd) {
  const int dgdStride = w + 6;
  std::vector<int32_t> dgd((size_t)dgdStride * (h + 6));
  for (int row = -3; row < h + 3; row++)
    for (int col = -3; col < w + 3; col++)
      dgd[(size_t)(row + 3) * dgdStride + col + 3] = src[(ptrdiff_t)row * sstride + col];
  const int bufStride = (((w + 6) + 3) & ~3) + 16;
  std::vector<int32_t> A((size_t)bufStride * (h + 6)), B((size_t)bufStride * (h + 6));
  std::vector<int32_t> flt0((size_t)w * h, 0), flt1((size_t)w * h, 0);
  const int dgdOrigin = 3 * dgdStride + 3;
  const int aOrigin = 3 * bufStride + 3;
  if (pf_sgr_params[set][0] > 0) {
    sgr_intermediate(dgd, dgdStride, w, h, bd, set, 0, 1, A, B, bufStride);
    for (int row = 0; row < h; row++) {
      const int k0 = aOrigin + row * bufStride;
      for (int col = 0; col < w; col++) {
        const int k = k0 + col;
        int32_t a, b, shift;
        if ((row & 1) == 0) {
          a = (A[k - bufStride] + A[k + bufStride]) * 6 +
              (A[k - bufStride - 1] + A[k - bufStride + 1] + A[k + bufStride - 1] + A[k + bufStride + 1]) * 5;
          b = (B[k - bufStride] + B[k + bufStride]) * 6 +
              (B[k - bufStride - 1] + B[k - bufStride + 1] + B[k + bufStride - 1] + B[k + bufStride + 1]) * 5;
          shift = 8 + 5 - 4;
        } else {
          a = A[k] * 6 + (A[k - 1] + A[k + 1]) * 5;
          b = B[k] * 6 + (B[k - 1] + B[k + 1]) * 5;
          shift = 8 + 4 - 4;
        }
        flt0[(size_t)row * w + col] = rpot(a * dgd[dgdOrigin + row * dgdStride + col] + b, shift);
      }
    }
  }
  if (pf_sgr_params[set][1] > 0) {
    sgr_intermediate(dgd, dgdStride, w, h, bd, set, 1, 0, A, B, bufStride);
    for (int row = 0; row < h; row++) {
      const int k0 = aOrigin + row * bufStride;
      for (int col = 0; col < w; col++) {
        const int k = k0 + col;
        const int32_t a = (A[k] + A[k - 1] + A[k + 1] + A[k - bufStride] + A[k + bufStride]) * 4 +
                          (A[k - bufStride - 1] + A[k + bufStride - 1] + A[k - bufStride + 1] + A[k + bufStride + 1]) * 3;
        const int32_t b = (B[k] + B[k - 1] + B[k + 1] + B[k - bufStride] + B[k + bufStride]) * 4 +
                          (B[k - bufStride - 1] + B[k + bufStride - 1] + B[k - bufStride + 1] + B[k + bufStride + 1]) * 3;
        flt1[(size_t)row * w + col] = rpot(a * dgd[dgdOrigin + row * dgdStride + col] + b, 8 + 5 - 4);
      }
    }
  }
  int16_t xq[2];
  sgr_decode_xq(xqd, set, xq);
  const int32_t maxI = (1 << bd) - 1;
  for (int row = 0; row < h; row++) {
    for (int col = 0; col < w; col++) {
      const int32_t u = (int32_t)src[(ptrdiff_t)row * sstride + col] << 4;
      int32_t v = u << 7;
      v += xq[0] * (flt0[(size_t)row * w + col] - u);
      v += xq[1] * (flt1[(size_t)row * w + col] - u);
      const int32_t r = rpot(v, 7 + 4);
      const int32_t wv = (int32_t)(int16_t)r;
      dst[(size_t)row * dstride + col] = (uint16_t)std::min(std::max(wv, 0), maxI);
    }
  }
}

// tile/restoration_geometry.go:54-95 (UnitRect), :97-141 (ProcessingStripe),
// :163-236 (ProcessingUnit); tile/restoration_apply.go:526-674 (the striped
// unit apply with stripe-boundary setup and restore) and
// restoration_frame_bridge.go:101-204 (bordered data / dst round trip).
int do_loop_restoration(const pf_frame* fr, const pf_frame_side* side, LRLines lines[3], int* unitsOut) {
  const pf_restoration& lr = side->lr;
  const int bd = fr->bit_depth;
  int units = 0;
  for (int plane = 0; plane < (fr->mono ? 1 : 3); plane++) {
    LRGrid g = lr_grid(fr, lr, plane);
    if (g.type == PF_LR_NONE) continue;
    if (g.unitSize == 0) return PF_ERR_INVALID_PLAN;
    const int nUnits = g.horz * g.vert;
    if (!lr.units[plane] || lr.unit_count[plane] < nUnits) return PF_ERR_INVALID_PLAN;
    bool anyFiltered = false;
    for (int i = 0; i < nUnits; i++)
      if (lr.units[plane][i].type != PF_LR_NONE) anyFiltered = true;
    if (!anyFiltered) continue;
    Plane pl = plane_of(fr, plane);
    // Bordered data copy with the 3-pixel replicate extension (ExtendRestorationFrame,
    // restoration_boundary.go:126-180).
    const int B = 32;
    const int dstride = g.W + 2 * B;
    std::vector<uint16_t> data((size_t)dstride * (g.H + 2 * B), 0), out((size_t)dstride * (g.H + 2 * B), 0);
    auto D = [&](int x, int y) -> uint16_t& { return data[(size_t)(y + B) * dstride + x + B]; };
    for (int y = 0; y < g.H; y++)
      for (int x = 0; x < g.W; x++) D(x, y) = (uint16_t)pl.get(x, y);
    for (int y = 0; y < g.H; y++)
      for (int x = 0; x < kLRBorder; x++) {
        D(-kLRBorder + x, y) = D(0, y);
        D(g.W + x, y) = D(g.W - 1, y);
      }
    for (int y = -kLRBorder; y < 0; y++)
      for (int x = -kLRBorder; x < g.W + kLRBorder; x++) D(x, y) = D(x, 0);
    for (int y = g.H; y < g.H + kLRBorder; y++)
      for (int x = -kLRBorder; x < g.W + kLRBorder; x++) D(x, y) = D(x, g.H - 1);

    const int fullStripe = 64 >> g.ssy, procW = 64 >> g.ssx, runitOff = kLRUnitOffset >> g.ssy;
    for (int ur = 0; ur < g.vert; ur++) {
      for (int uc = 0; uc < g.horz; uc++) {
        const pf_lr_unit& u = lr.units[plane][ur * g.horz + uc];
        if (u.type == PF_LR_NONE) continue;
        if (u.type != PF_LR_WIENER && u.type != PF_LR_SGRPROJ) return PF_ERR_INVALID_PLAN;
        if (g.type != PF_LR_SWITCHABLE && u.type != g.type) return PF_ERR_INVALID_PLAN;
        // UnitRect.
        int x0 = uc * g.unitSize, x1 = x0 + g.unitSize;
        if (uc + 1 == g.horz) x1 = g.W;
        int y0 = ur * g.unitSize, y1 = y0 + g.unitSize;
        if (ur + 1 == g.vert) y1 = g.H;
        if (y0 > 0) y0 -= runitOff;
        if (y1 < g.H) y1 -= runitOff;
        int16_t vf[7], hf[7];
        if (u.type == PF_LR_WIENER) {
          // restoration/wiener.go:44-47 (NewWienerFilter).
          const int16_t v0 = u.wiener_v[0], v1 = u.wiener_v[1], v2 = u.wiener_v[2];
          const int16_t h0 = u.wiener_h[0], h1 = u.wiener_h[1], h2 = u.wiener_h[2];
          const int16_t vv[7] = {v0, v1, v2, (int16_t)(-2 * (v0 + v1 + v2)), v2, v1, v0};
          const int16_t hh[7] = {h0, h1, h2, (int16_t)(-2 * (h0 + h1 + h2)), h2, h1, h0};
          memcpy(vf, vv, sizeof(vf));
          memcpy(hf, hh, sizeof(hf));
        }
        for (int y = y0; y < y1;) {
          const int tileStripe = (y + runitOff) / fullStripe;
          int nominal = fullStripe;
          if (y == 0) nominal -= runitOff;
          const int sh = imin(nominal, y1 - y);
          const bool copyAbove = y != 0, copyBelow = y + nominal < g.H;
          const int lineW = (x1 - x0) + 2 * kLRExtraHorz;
          std::vector<uint16_t> saveA((size_t)3 * lineW), saveB((size_t)3 * lineW);
          // setupRestorationStripeBoundaryFromSaved (restoration_boundary.go:553-614).
          if (copyAbove) {
            for (int i = -kLRBorder; i < 0; i++) {
              const int bufRow = tileStripe * kLRCtxVert + imax(i + kLRCtxVert, 0);
              for (int k = 0; k < lineW; k++) {
                uint16_t& d = D(x0 - kLRExtraHorz + k, y + i);
                saveA[(size_t)(i + kLRBorder) * lineW + k] = d;
                d = lines[plane].above[(size_t)bufRow * lines[plane].stride + x0 + k];
              }
            }
          }
          if (copyBelow) {
            for (int i = 0; i < kLRBorder; i++) {
              const int bufRow = tileStripe * kLRCtxVert + imin(i, kLRCtxVert - 1);
              for (int k = 0; k < lineW; k++) {
                uint16_t& d = D(x0 - kLRExtraHorz + k, y + sh + i);
                saveB[(size_t)i * lineW + k] = d;
                d = lines[plane].below[(size_t)bufRow * lines[plane].stride + x0 + k];
              }
            }
          }
          for (int x = x0; x < x1; x += procW) {
            const int rem = x1 - x;
            int fw = u.type == PF_LR_WIENER ? imin(procW, (rem + 15) & ~15) : imin(procW, rem);
            const uint16_t* s = &D(x, y);
            uint16_t* o = &out[(size_t)(y + B) * dstride + x + B];
            if (u.type == PF_LR_WIENER)
              wiener_apply(s, dstride, o, dstride, fw, sh, vf, hf, bd);
            else
              sgr_apply(s, dstride, o, dstride, fw, sh, u.sgr_set, u.sgr_xqd, bd);
          }
          // restoreRestorationStripeBoundarySaved (restoration_boundary.go:652-685).
          if (copyAbove)
            for (int i = -kLRBorder; i < 0; i++)
              for (int k = 0; k < lineW; k++) D(x0 - kLRExtraHorz + k, y + i) = saveA[(size_t)(i + kLRBorder) * lineW + k];
          if (copyBelow)
            for (int i = 0; i < kLRBorder; i++) {
              if (y + sh + i >= y1 + kLRBorder) break;
              for (int k = 0; k < lineW; k++) D(x0 - kLRExtraHorz + k, y + sh + i) = saveB[(size_t)i * lineW + k];
            }
          y += sh;
        }
        // Store the record rect back (StoreBorderedSamplePlaneRectTrusted).
        for (int yy = y0; yy < y1; yy++)
          for (int xx = x0; xx < x1; xx++) pl.set(xx, yy, out[(size_t)(yy + B) * dstride + xx + B]);
        units++;
      }
    }
  }
  if (unitsOut) *unitsOut = units;
  return PF_OK;
}

// ===========================================================================
// Border extension (frame/buffer.go:301-400, ExtendBordersFrom(0))
// ===========================================================================
void extend_borders(const pf_frame* fr) {
  for (int p = 0; p < (fr->mono ? 1 : 3); p++) {
    Plane pl = plane_of(fr, p);
    const int h = imin(pl.h, pl.ah);
    for (int y = 0; y < h; y++) {
      const int v = pl.get(pl.w - 1, y);
      for (int x = pl.w; x < pl.aw; x++) pl.set(x, y, v);
    }
    for (int y = h; y < pl.ah; y++)
      memcpy(pl.data + (int64_t)y * pl.stride, pl.data + (int64_t)(h - 1) * pl.stride, (size_t)pl.aw * pl.bps);
  }
}

// ===========================================================================
// Film grain
// ===========================================================================

// filmgrain/random.go:15-72.
uint16_t lfsr_number(uint16_t& reg, int bits) {
  const uint16_t bit = ((reg >> 0) ^ (reg >> 1) ^ (reg >> 3) ^ (reg >> 12)) & 1;
  reg = (uint16_t)((reg >> 1) | (bit << 15));
  if (bits == 16) return reg;
  return (uint16_t)((reg >> (16 - bits)) & ((1 << bits) - 1));
}
uint16_t stripe_seed(uint16_t seed, int lumaLine) {
  const int n = lumaLine >> 5;
  uint16_t r = seed;
  r ^= (uint16_t)(((n * 37 + 178) & 255) << 8);
  r ^= (uint16_t)((n * 173 + 105) & 255);
  return r;
}
int rpow2(int v, int bits) { return bits <= 0 ? v : (v + (1 << (bits - 1))) >> bits; }

constexpr int kGW = 82, kGH = 73;

// filmgrain/luma.go:24-82 (GenerateLumaGrain with the generic AR loop).
void luma_grain(int16_t* g, const pf_film_grain& fg, int bd) {
  memset(g, 0, sizeof(int16_t) * kGW * kGH);
  if (fg.num_y_points == 0) return;
  uint16_t reg = fg.seed;
  const int shift = 12 - bd + fg.grain_scale_shift;
  for (int y = 0; y < kGH; y++)
    for (int x = 0; x < kGW; x++) {
      const int idx = lfsr_number(reg, 11);
      g[y * kGW + x] = (int16_t)rpow2(pf_gaussian_sequence[idx], shift);
    }
  const int lag = fg.ar_coeff_lag;
  if (lag == 0) return;
  const int cs = fg.ar_coeff_shift, ro = 1 << (cs - 1);
  const int gmin = -(1 << (bd - 1)), gmax = (1 << (bd - 1)) - 1;
  for (int y = 3; y < kGH; y++)
    for (int x = 3; x < kGW - 3; x++) {
      int sum = 0, pos = 0;
      for (int dr = -lag; dr <= 0; dr++)
        for (int dc = -lag; dc <= lag; dc++) {
          if (dr == 0 && dc == 0) break;
          sum += fg.ar_coeffs_y[pos++] * g[(y + dr) * kGW + x + dc];
        }
      g[y * kGW + x] = (int16_t)iclip(g[y * kGW + x] + ((sum + ro) >> cs), gmin, gmax);
    }
}

// filmgrain/chroma.go:29-91, :223-241.
void chroma_grain(int16_t* g, const int16_t* luma, const pf_film_grain& fg, int plane, int bd, int ssx, int ssy) {
  memset(g, 0, sizeof(int16_t) * kGW * kGH);
  uint16_t reg = (uint16_t)(fg.seed ^ (plane == 1 ? 0xb524 : 0x49d8));
  const int w = ssx ? 44 : 82, h = ssy ? 38 : 73;
  const int shift = 12 - bd + fg.grain_scale_shift;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int idx = lfsr_number(reg, 11);
      g[y * kGW + x] = (int16_t)rpow2(pf_gaussian_sequence[idx], shift);
    }
  const int lag = fg.ar_coeff_lag;
  if (lag == 0 && fg.num_y_points == 0) return;
  const int8_t* co = plane == 1 ? fg.ar_coeffs_cb : fg.ar_coeffs_cr;
  const int cs = fg.ar_coeff_shift, ro = 1 << (cs - 1);
  const int gmin = -(1 << (bd - 1)), gmax = (1 << (bd - 1)) - 1;
  for (int y = 3; y < h; y++)
    for (int x = 3; x < w - 3; x++) {
      int sum = 0, pos = 0;
      for (int dr = -lag; dr <= 0; dr++)
        for (int dc = -lag; dc <= lag; dc++) {
          if (dr == 0 && dc == 0) {
            if (fg.num_y_points != 0) {
              const int lx = ((x - 3) << ssx) + 3, ly = ((y - 3) << ssy) + 3;
              int s = 0;
              for (int dy = 0; dy <= ssy; dy++)
                for (int dx = 0; dx <= ssx; dx++) s += luma[(ly + dy) * kGW + lx + dx];
              sum += rpow2(s, ssx + ssy) * co[pos];
            }
            break;
          }
          sum += co[pos++] * g[(y + dr) * kGW + x + dc];
        }
      g[y * kGW + x] = (int16_t)iclip(g[y * kGW + x] + ((sum + ro) >> cs), gmin, gmax);
    }
}

// filmgrain/scaling.go:18-48 (BuildScalingLUT).
void scaling_lut(uint8_t* dst, const uint8_t (*pts)[2], int n) {
  memset(dst, 0, 256);
  if (n == 0) return;
  for (int x = 0; x < pts[0][0]; x++) dst[x] = pts[0][1];
  for (int p = 0; p < n - 1; p++) {
    const int dy = pts[p + 1][1] - pts[p][1], dx = pts[p + 1][0] - pts[p][0];
    const int64_t delta = (int64_t)dy * ((65536 + (dx >> 1)) / dx);
    for (int x = 0; x < dx; x++) dst[pts[p][0] + x] = (uint8_t)(pts[p][1] + (int)(((int64_t)x * delta + 32768) >> 16));
  }
  for (int x = pts[n - 1][0]; x < 256; x++) dst[x] = pts[n - 1][1];
}

// filmgrain/scaling.go:56-75 (scaleLUT).
int scale_lut(const uint8_t* lut, int index, int bd) {
  const int maxIndex = (1 << bd) - 1;
  index = iclip(index, 0, maxIndex);
  const int shift = bd - 8;
  const int x = index >> shift;
  if (bd == 8 || x == 255) return lut[x];
  const int rem = index - (x << shift);
  const int start = lut[x], end = lut[x + 1];
  return (uint8_t)(start + rpow2((end - start) * rem, shift));
}

struct FGPlaneCtx {
  Plane src;         // un-grained (post-LR) plane
  Plane dst;         // display plane
  const int16_t* grain;
  const uint8_t* lut;
};

int blend_luma(int prev, int cur, int offset, int bd) {  // filmgrain/blend.go:16-25
  int pw = 27, cw = 17;
  if (offset == 1) {
    pw = 17;
    cw = 27;
  }
  return iclip(rpow2(prev * pw + cur * cw, 5), -(1 << (bd - 1)), (1 << (bd - 1)) - 1);
}
int blend_chroma(int prev, int cur, int offset, int shift, int bd) {  // apply.go:538-546
  if (shift) return iclip(rpow2(prev * 23 + cur * 22, 5), -(1 << (bd - 1)), (1 << (bd - 1)) - 1);
  return blend_luma(prev, cur, offset, bd);
}

// filmgrain/apply.go:72-343: one 32-row stripe of one plane, every 32-pixel
// block left to right with offsets drawn in order from the stripe LFSR(s).
// The overlap blends of apply.go:206-343 are restated per sample: grain(x,y)
// is the current block's template sample, blended with the left block's for
// x < xStart and with the block above's for y < yStart (with the corner
// blending the left/top pairs first, then the two results).
void fg_stripe(const pf_frame* fr, const pf_film_grain& fg, int plane, int row, FGPlaneCtx& pc, const Plane& luma) {
  const int bd = fr->bit_depth;
  const int sx = plane ? fr->ss_x : 0, sy = plane ? fr->ss_y : 0;
  const int W = pc.src.w, Hp = pc.src.h;
  const int bh = 32 >> sy;
  const int y0 = row * bh;
  const int height = imin(bh, Hp - y0);
  const int rows = (fg.overlap && row > 0) ? 2 : 1;
  uint16_t regs[2];
  for (int i = 0; i < rows; i++) regs[i] = stripe_seed(fg.seed, (row - i) * 32);
  const int bw = 32 >> sx;
  int minV = 0, maxV = (256 << (bd - 8)) - 1;
  if (fg.clip_to_restricted_range) {
    minV = 16 << (bd - 8);
    maxV = (plane == 0 ? 235 : (fg.matrix_identity ? 235 : 240)) << (bd - 8);
  }
  const bool oddLuma = plane != 0 && sx && (fr->width & 1);
  uint8_t off[2][2] = {{0, 0}, {0, 0}};
  const int ovl = 2;  // LumaOverlapSamples
  auto gidx = [&](int offset, int bc, int br, int x, int y) {
    const int col = 3 + (ovl >> sx) * (3 + (offset >> 4)) + x + bw * bc;
    const int rr = 3 + (ovl >> sy) * (3 + (offset & 15)) + y + bh * br;
    return rr * kGW + col;
  };
  for (int bx = 0; bx < W; bx += bw) {
    const int blockW = imin(bw, W - bx);
    if (fg.overlap && bx > 0)
      for (int i = 0; i < rows; i++) off[1][i] = off[0][i];
    for (int i = 0; i < rows; i++) off[0][i] = (uint8_t)lfsr_number(regs[i], 8);
    const int yStart = (fg.overlap && row > 0) ? imin(height, ovl >> sy) : 0;
    const int xStart = (fg.overlap && bx > 0) ? imin(blockW, ovl >> sx) : 0;
    for (int y = 0; y < height; y++) {
      for (int x = 0; x < blockW; x++) {
        int g = pc.grain[gidx(off[0][0], 0, 0, x, y)];
        if (x < xStart) {
          const int left = pc.grain[gidx(off[1][0], 1, 0, x, y)];
          g = blend_chroma(left, g, x, plane ? sx : 0, bd);
        }
        if (y < yStart) {
          int top = pc.grain[gidx(off[0][1], 0, 1, x, y)];
          if (x < xStart) {
            const int topLeft = pc.grain[gidx(off[1][1], 1, 1, x, y)];
            top = blend_chroma(topLeft, top, x, plane ? sx : 0, bd);
          }
          if (plane == 0) {
            g = blend_luma(top, g, y, bd);
          } else {
            // chromaOverlapWeights / blendChromaOverlap along y (apply.go:414-422, :538-546).
            g = blend_chroma(top, g, y, sy, bd);
          }
        }
        const int px = bx + x, py = y0 + y;
        const int s = pc.src.get(px, py);
        int scale;
        if (plane == 0) {
          scale = scale_lut(pc.lut, s, bd);
        } else {
          // chromaScalingIndex (apply.go:501-520).
          const int lx = px << sx, ly = py << sy;
          int avg = luma.get(lx, ly);
          if (sx && !(oddLuma && px == W - 1)) avg = (avg + luma.get(lx + 1, ly) + 1) >> 1;
          int idx;
          if (fg.chroma_scaling_from_luma) {
            idx = avg;
          } else {
            const int lm = (plane == 1 ? fg.cb_luma_mult : fg.cr_luma_mult) - 128;
            const int cm = (plane == 1 ? fg.cb_mult : fg.cr_mult) - 128;
            const int ofs = ((plane == 1 ? fg.cb_offset : fg.cr_offset) << (bd - 8)) - (1 << bd);
            idx = iclip(((avg * lm + s * cm) >> 6) + ofs, 0, (1 << bd) - 1);
          }
          scale = scale_lut(pc.lut, idx, bd);
        }
        const int noise = rpow2(scale * g, fg.scaling_shift);
        pc.dst.set(px, py, iclip(s + noise, minV, maxV));
      }
    }
  }
}

// postfilter_filmgrain.go:192-263 (plan), :516-628 (ApplyFilmGrainPostFilter):
// scaling LUTs, luma then chroma templates, chroma planes then luma, written
// into the display frame (a copy of the post-filter frame).
int do_film_grain(const pf_frame* fr, const pf_film_grain& fg, const pf_frame* disp) {
  if (!disp) return PF_ERR_INVALID_ARG;
  const int bd = fr->bit_depth;
  // Display starts as a copy of the reference frame (frameWorkCopyPostFilterFrame).
  for (int p = 0; p < (fr->mono ? 1 : 3); p++) {
    Plane s = plane_of(fr, p), d = plane_of(disp, p);
    for (int y = 0; y < s.ah; y++) memcpy(d.data + (int64_t)y * d.stride, s.data + (int64_t)y * s.stride, (size_t)s.aw * s.bps);
  }
  if (!fg.apply) return PF_OK;
  const bool lumaActive = fg.num_y_points != 0;
  bool chromaActive[3] = {false, false, false};
  if (!fr->mono) {
    chromaActive[1] = fg.num_cb_points != 0 || fg.chroma_scaling_from_luma;
    chromaActive[2] = fg.num_cr_points != 0 || fg.chroma_scaling_from_luma;
  }
  if (!lumaActive && !chromaActive[1] && !chromaActive[2]) return PF_OK;  // no-op grain
  if (fg.scaling_shift < 8 || fg.scaling_shift > 11) return PF_ERR_INVALID_FORMAT;
  uint8_t luts[3][256];
  scaling_lut(luts[0], fg.y_points, fg.num_y_points);
  if (fg.chroma_scaling_from_luma) {
    memcpy(luts[1], luts[0], 256);
    memcpy(luts[2], luts[0], 256);
  } else {
    scaling_lut(luts[1], fg.cb_points, fg.num_cb_points);
    scaling_lut(luts[2], fg.cr_points, fg.num_cr_points);
  }
  std::vector<int16_t> lg(kGW * kGH, 0), cg[3];
  if (lumaActive) luma_grain(lg.data(), fg, bd);
  for (int p = 1; p <= 2; p++) {
    if (!chromaActive[p]) continue;
    cg[p].assign(kGW * kGH, 0);
    chroma_grain(cg[p].data(), lg.data(), fg, p, bd, fr->ss_x, fr->ss_y);
  }
  Plane luma = plane_of(fr, 0);
  for (int p = 1; p <= 2; p++) {
    if (!chromaActive[p]) continue;
    FGPlaneCtx pc{plane_of(fr, p), plane_of(disp, p), cg[p].data(), luts[p]};
    const int bh = 32 >> fr->ss_y;
    const int rows = (pc.src.h + bh - 1) / bh;
    for (int r = 0; r < rows; r++) fg_stripe(fr, fg, p, r, pc, luma);
  }
  if (lumaActive) {
    FGPlaneCtx pc{plane_of(fr, 0), plane_of(disp, 0), lg.data(), luts[0]};
    const int rows = (pc.src.h + 31) / 32;
    for (int r = 0; r < rows; r++) fg_stripe(fr, fg, 0, r, pc, luma);
  }
  return PF_OK;
}

}  // namespace

// ===========================================================================
// Driver: postfilter.go:589-782 (applySupportedPostFiltersInPlace) and
// :810-842 (the publication variant writing grain into a display copy).
// ===========================================================================
extern "C" int oracle_frame_apply(const pf_frame* fr, const pf_frame_side* side, const pf_frame* disp) {
  if (!fr || !side) return PF_ERR_INVALID_ARG;
  int st;
  LRLines lines[3];
  const bool lr = (side->stages & PF_STAGE_LOOP_RESTORATION) != 0;
  if (side->stages & PF_STAGE_LOOP_FILTER) {
    if ((st = do_loop_filter(fr, side)) != PF_OK) return st;
  }
  if (lr)
    for (int p = 0; p < (fr->mono ? 1 : 3); p++) {
      LRGrid g = lr_grid(fr, side->lr, p);
      if (g.type != PF_LR_NONE) lr_save_lines(fr, p, g, lines[p], false);
    }
  if (side->stages & PF_STAGE_CDEF) {
    if ((st = do_cdef(fr, side, nullptr)) != PF_OK) return st;
  }
  if (lr) {
    for (int p = 0; p < (fr->mono ? 1 : 3); p++) {
      LRGrid g = lr_grid(fr, side->lr, p);
      if (g.type != PF_LR_NONE) lr_save_lines(fr, p, g, lines[p], true);
    }
    if ((st = do_loop_restoration(fr, side, lines, nullptr)) != PF_OK) return st;
  }
  if (side->stages & PF_STAGE_EXTEND_BORDERS) extend_borders(fr);
  if (side->stages & PF_STAGE_FILM_GRAIN) {
    if ((st = do_film_grain(fr, side->fg, disp)) != PF_OK) return st;
  }
  return PF_OK;
}

// The decoder's order for a super-resolved frame (decoder/postfilter.go:
// 336-345, postfilter_superres.go:206-283): deblock, the deblock-row save
// (upscaled), CDEF on the coded frame; the upscale; restoration, border
// extension and grain on the upscaled frame.
extern "C" int oracle_frame_apply_superres(const pf_frame* coded, const pf_frame_side* side, const pf_frame* up,
                                           const pf_frame* disp) {
  if (!coded || !side || !up) return PF_ERR_INVALID_ARG;
  int st;
  LRLines lines[3];
  const bool lr = (side->stages & PF_STAGE_LOOP_RESTORATION) != 0;
  if (side->stages & PF_STAGE_LOOP_FILTER) {
    if ((st = do_loop_filter(coded, side)) != PF_OK) return st;
  }
  if (lr)
    for (int p = 0; p < (up->mono ? 1 : 3); p++) {
      LRGrid g = lr_grid(up, side->lr, p);
      if (g.type != PF_LR_NONE) lr_save_lines(up, p, g, lines[p], false, coded);
    }
  if (side->stages & PF_STAGE_CDEF) {
    if ((st = do_cdef(coded, side, nullptr)) != PF_OK) return st;
  }
  if ((st = oracle_superres_upscale(coded, up)) != PF_OK) return st;
  if (lr) {
    for (int p = 0; p < (up->mono ? 1 : 3); p++) {
      LRGrid g = lr_grid(up, side->lr, p);
      if (g.type != PF_LR_NONE) lr_save_lines(up, p, g, lines[p], true);
    }
    if ((st = do_loop_restoration(up, side, lines, nullptr)) != PF_OK) return st;
  }
  if (side->stages & PF_STAGE_EXTEND_BORDERS) extend_borders(up);
  if (side->stages & PF_STAGE_FILM_GRAIN) {
    if ((st = do_film_grain(up, side->fg, disp)) != PF_OK) return st;
  }
  return PF_OK;
}

extern "C" int oracle_loop_filter(const pf_frame* fr, const pf_frame_side* side) { return do_loop_filter(fr, side); }
extern "C" int oracle_cdef(const pf_frame* fr, const pf_frame_side* side) { return do_cdef(fr, side, nullptr); }

extern "C" int oracle_cdef_find_dir(const uint16_t* img, int stride, int coeff_shift, int32_t* variance) {
  return find_dir(img, stride, coeff_shift, variance);
}
extern "C" void oracle_cdef_filter_block(uint16_t* dst, const uint16_t* in, int in_origin, int pri, int sec, int dir,
                                         int pri_damping, int sec_damping, int coeff_shift, int w, int h) {
  filter_block(dst, w, in, in_origin, pri, sec, dir, pri_damping, sec_damping, coeff_shift, w, h);
}
extern "C" int oracle_cdef_adjust_strength(int strength, int32_t variance) { return adjust_strength(strength, variance); }

extern "C" void oracle_lpf_line(uint16_t* line16, int bit_depth, int level, int sharpness, int wd) {
  pf_frame f;
  memset(&f, 0, sizeof(f));
  f.bit_depth = (uint8_t)bit_depth;
  // A 16x4 plane holding the line in each of its four rows.
  std::vector<uint16_t> buf(16 * 4);
  for (int r = 0; r < 4; r++)
    for (int i = 0; i < 16; i++) buf[r * 16 + i] = line16[i];
  Plane pl;
  pl.data = (uint8_t*)buf.data();
  pl.stride = 32;
  pl.bps = 2;
  pl.w = 16;
  pl.h = 4;
  int E, I, H;
  lf_thresholds(level, sharpness, &E, &I, &H);
  lpf_unit(pl, 8, 0, 0, 1, 1, 0, bit_depth, E, I, H, wd);
  for (int i = 0; i < 16; i++) line16[i] = buf[i];
}

// The same edge unit with explicit thresholds: E (block limit), I (inner
// limit) and H (high-edge-variance threshold) at 8-bit scale, as goav1's
// Filter4/6/8/14Edge tests give them (loopfilter/loopfilter_test.go); wd is
// the dav1d width class 4, 6, 8 or 16 (the 14-tap filter).
extern "C" void oracle_lpf_line_thr(uint16_t* line16, int bit_depth, int E, int I, int H, int wd) {
  std::vector<uint16_t> buf(16 * 4);
  for (int r = 0; r < 4; r++)
    for (int i = 0; i < 16; i++) buf[r * 16 + i] = line16[i];
  Plane pl;
  pl.data = (uint8_t*)buf.data();
  pl.stride = 32;
  pl.bps = 2;
  pl.w = 16;
  pl.h = 4;
  lpf_unit(pl, 8, 0, 0, 1, 1, 0, bit_depth, E, I, H, wd);
  for (int i = 0; i < 16; i++) line16[i] = buf[i];
}

extern "C" int oracle_sgr_x_by_xplus1(int z) { return pf_sgr_x_by_xplus1[z < 0 ? 0 : (z > 255 ? 255 : z)]; }

extern "C" void oracle_lf_thresholds(int level, int sharpness, int* E, int* I, int* H) {
  lf_thresholds(level, sharpness, E, I, H);
}

// convertChromaDirections on one direction (cdef/filter.go:614-633).
extern "C" int oracle_cdef_chroma_dir(int dir, int xdec, int ydec) {
  if (xdec == ydec) return dir;
  CdefGrid g;
  memset(&g, 0, sizeof(g));
  g.dir[0][0] = (uint8_t)dir;
  std::vector<std::pair<int, int>> one(1, std::make_pair(0, 0));
  convert_chroma_dirs(g, one, xdec);
  return g.dir[0][0];
}

// Film grain on one plane with a given template and scaling table
// (filmgrain/apply.go:72-343 over every 32-row stripe): src/dst hold the
// plane's samples as uint16 with `stride` samples per row; luma (the luma
// plane, luma_stride samples per row) gives chroma its scaling index.
extern "C" int oracle_fg_apply_plane(const uint16_t* src, uint16_t* dst, int stride, const uint16_t* luma,
                                     int luma_stride, int frame_w, int frame_h, const int16_t* grain, const uint8_t* lut,
                                     const pf_film_grain* fg, int plane, int bit_depth, int ss_x, int ss_y) {
  pf_frame fr;
  memset(&fr, 0, sizeof(fr));
  fr.width = frame_w;
  fr.height = frame_h;
  fr.bit_depth = (uint8_t)bit_depth;
  fr.ss_x = (uint8_t)ss_x;
  fr.ss_y = (uint8_t)ss_y;
  const int sx = plane ? ss_x : 0, sy = plane ? ss_y : 0;
  Plane s, d, l;
  s.data = (uint8_t*)src;
  d.data = (uint8_t*)dst;
  s.stride = d.stride = (int64_t)stride * 2;
  s.bps = d.bps = 2;
  s.w = d.w = (frame_w + sx) >> sx;
  s.h = d.h = (frame_h + sy) >> sy;
  l.data = (uint8_t*)(luma ? luma : src);
  l.stride = (int64_t)(luma ? luma_stride : stride) * 2;
  l.bps = 2;
  l.w = frame_w;
  l.h = frame_h;
  FGPlaneCtx pc{s, d, grain, lut};
  const int bh = 32 >> sy;
  for (int r = 0; r < (s.h + bh - 1) / bh; r++) fg_stripe(&fr, *fg, plane, r, pc, l);
  return PF_OK;
}

extern "C" uint16_t oracle_lfsr_next(uint16_t* reg, int bits) { return lfsr_number(*reg, bits); }
extern "C" uint16_t oracle_stripe_seed(uint16_t seed, int luma_line) { return stripe_seed(seed, luma_line); }
extern "C" int oracle_scaling_lut(uint8_t* dst256, const uint8_t* points, int n) {
  scaling_lut(dst256, (const uint8_t(*)[2])points, n);
  return 0;
}
extern "C" int oracle_scale_lut(const uint8_t* lut, int index, int bit_depth) { return scale_lut(lut, index, bit_depth); }
extern "C" int oracle_luma_grain(int16_t* dst, const pf_film_grain* fg, int bit_depth) {
  luma_grain(dst, *fg, bit_depth);
  return 0;
}
extern "C" int oracle_chroma_grain(int16_t* dst, const int16_t* luma, const pf_film_grain* fg, int plane, int bit_depth,
                                   int ss_x, int ss_y) {
  chroma_grain(dst, luma, *fg, plane, bit_depth, ss_x, ss_y);
  return 0;
}
extern "C" int16_t oracle_gaussian(int index) { return pf_gaussian_sequence[index & 2047]; }
extern "C" void oracle_sgr_decode_xq(const int8_t* xqd, int set, int16_t* xq) { sgr_decode_xq(xqd, set, xq); }
extern "C" void oracle_wiener(const uint16_t* src, int sstride, uint16_t* dst, int dstride, int w, int h,
                              const int16_t* vf, const int16_t* hf, int bit_depth) {
  wiener_apply(src, sstride, dst, dstride, w, h, vf, hf, bit_depth);
}
extern "C" void oracle_sgr(const uint16_t* src, int sstride, uint16_t* dst, int dstride, int w, int h, int set,
                           const int8_t* xqd, int bit_depth) {
  sgr_apply(src, sstride, dst, dstride, w, h, set, xqd, bit_depth);
}
