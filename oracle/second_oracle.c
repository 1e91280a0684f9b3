/*
 * second_oracle.c - a second, independent CPU oracle for the filter
 * arithmetic (test infrastructure only; nothing in the product links it).
 *
 * oracle/pf_oracle.cpp restates goav1's production Go paths; the CUDA
 * kernels are checked against it at tolerance zero.  A misreading shared by
 * that restatement and the kernels would pass those checks, so the filter
 * arithmetic is restated here a second time from different sources:
 *
 *   - where goav1's own tests carry a libaom-style restatement used as their
 *     second oracle, that restatement (file:line below, paths inside
 *     thesyncim/goav1): cReferenceFilter4/6/8/14, filterBlockLibaomReference
 *     with its constrain/adjust helpers, findDirectionLibaomReference,
 *     referenceWienerPixel, frozenSGRIntermediate;
 *   - otherwise the AV1 specification's own formulation of the process,
 *     which is organised differently from goav1's: the self-guided filter
 *     with direct window box sums and the spec's formulas for s, x/(x+1)
 *     and 1/n; film grain through the spec's noise stripes and noise image
 *     (each 32-row stripe's noise built with its horizontal blends, then the
 *     vertical blend against the stripe above) instead of goav1's per-block
 *     blend of the four neighbouring offsets.
 *
 * The only table shared with the first oracle is the normative 2048-entry
 * Gaussian sequence (pf_tables.h), which tests/golden pins by goav1's own
 * checksums.  tests/test_second_oracle.py drives both oracles over random
 * inputs and asserts goav1's literal known-answer vectors against both.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "goav1pf.h"
#include "pf_tables.h"

static int so_abs(int v) { return v < 0 ? -v : v; }
static int so_clamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static int so_round2(int v, int n) { return n == 0 ? v : (v + (1 << (n - 1))) >> n; }
static int64_t so_round2_64(int64_t v, int n) { return n == 0 ? v : (v + ((int64_t)1 << (n - 1))) >> n; }

/* ======================================================================
 * Deblocking: the libaom restatements of loopfilter/loopfilter_test.go.
 * Thresholds are the 8-bit Limit / BlockLimit / HighEdgeVariance, scaled by
 * 1 << (bitDepth - 8) (:368-370, :1242-1245).
 * ====================================================================== */

/* cReferenceFilterMask2/3/4 (:2638-2642, :1266-1272, :1705-1713). */
static int so_mask(int n, const int* p, const int* q, int limit, int blimit) {
  /* p[0] = p0, p[1] = p1, ...; q likewise. */
  for (int k = 1; k < n; k++)
    if (so_abs(p[k] - p[k - 1]) > limit || so_abs(q[k] - q[k - 1]) > limit) return 0;
  return so_abs(p[0] - q[0]) * 2 + so_abs(p[1] - q[1]) / 2 <= blimit;
}

/* cReferenceFlatMask3/4 (:1274-1279, :1715-1722) over taps 1..n-1. */
static int so_flat(int n, const int* p, const int* q, int thresh) {
  for (int k = 1; k < n; k++)
    if (so_abs(p[k] - p[0]) > thresh || so_abs(q[k] - q[0]) > thresh) return 0;
  return 1;
}

/* cReferenceFilter4 (:1281-1304) on p1 p0 q0 q1. */
static void so_filter4(int* p1, int* p0, int* q0, int* q1, int hev_thr, int lo, int hi, int center) {
  const int ps1 = *p1 - center, ps0 = *p0 - center, qs0 = *q0 - center, qs1 = *q1 - center;
  const int hev = so_abs(*p1 - *p0) > hev_thr || so_abs(*q1 - *q0) > hev_thr;
  int f = hev ? so_clamp(ps1 - qs1, lo, hi) : 0;
  f = so_clamp(f + 3 * (qs0 - ps0), lo, hi);
  const int f1 = so_clamp(f + 4, lo, hi) >> 3;
  const int f2 = so_clamp(f + 3, lo, hi) >> 3;
  *p0 = so_clamp(ps0 + f2, lo, hi) + center;
  *q0 = so_clamp(qs0 - f1, lo, hi) + center;
  if (!hev) {
    const int outer = so_round2(f1, 1);
    *p1 = so_clamp(ps1 + outer, lo, hi) + center;
    *q1 = so_clamp(qs1 - outer, lo, hi) + center;
  }
}

/* One edge sample line of `width` taps (4, 6, 8 or 14), in order
 * p(n-1) .. p0 q0 .. q(n-1), filtered in place.  Returns 0, or -1 for an
 * unsupported width.  cReferenceFilterByWidth (:2593-2618) with
 * cReferenceFilter4Samples (:2620-2636), cReferenceFilter6 (:1241-1264),
 * cReferenceFilter8 (:1678-1703) and cReferenceFilter14 (:367-401). */
int so_lf_filter(int width, int* s, int bit_depth, int limit8, int blimit8, int hev8) {
  const int scale = 1 << (bit_depth - 8);
  const int limit = limit8 * scale, blimit = blimit8 * scale, hev = hev8 * scale;
  const int lo = -128 * scale, hi = 128 * scale - 1, center = 128 * scale;
  const int half = width / 2;
  int p[7], q[7];
  for (int k = 0; k < half; k++) {
    p[k] = s[half - 1 - k];
    q[k] = s[half + k];
  }
  switch (width) {
    case 4:
      if (!so_mask(2, p, q, limit, blimit)) return 0;
      so_filter4(&p[1], &p[0], &q[0], &q[1], hev, lo, hi, center);
      break;
    case 6:
      if (!so_mask(3, p, q, limit, blimit)) return 0;
      if (so_flat(3, p, q, scale)) {
        const int p2 = p[2], p1 = p[1], p0 = p[0], q0 = q[0], q1 = q[1], q2 = q[2];
        p[1] = so_round2(p2 * 3 + p1 * 2 + p0 * 2 + q0, 3);
        p[0] = so_round2(p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1, 3);
        q[0] = so_round2(p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2, 3);
        q[1] = so_round2(p0 + q0 * 2 + q1 * 2 + q2 * 3, 3);
      } else {
        so_filter4(&p[1], &p[0], &q[0], &q[1], hev, lo, hi, center);
      }
      break;
    case 8:
    case 14: {
      if (!so_mask(4, p, q, limit, blimit)) return 0;
      const int flat = so_flat(4, p, q, scale);
      int flat2 = 0;
      if (width == 14 && flat) {
        /* cReferenceFlatMask4(scale, p6, p5, p4, p0, q0, q4, q5, q6). */
        flat2 = 1;
        for (int k = 4; k < 7; k++)
          if (so_abs(p[k] - p[0]) > scale || so_abs(q[k] - q[0]) > scale) flat2 = 0;
      }
      if (width == 14 && flat && flat2) {
        const int p6 = p[6], p5 = p[5], p4 = p[4], p3 = p[3], p2 = p[2], p1 = p[1], p0 = p[0];
        const int q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3], q4 = q[4], q5 = q[5], q6 = q[6];
        p[5] = so_round2(p6 * 7 + p5 * 2 + p4 * 2 + p3 + p2 + p1 + p0 + q0, 4);
        p[4] = so_round2(p6 * 5 + p5 * 2 + p4 * 2 + p3 * 2 + p2 + p1 + p0 + q0 + q1, 4);
        p[3] = so_round2(p6 * 4 + p5 + p4 * 2 + p3 * 2 + p2 * 2 + p1 + p0 + q0 + q1 + q2, 4);
        p[2] = so_round2(p6 * 3 + p5 + p4 + p3 * 2 + p2 * 2 + p1 * 2 + p0 + q0 + q1 + q2 + q3, 4);
        p[1] = so_round2(p6 * 2 + p5 + p4 + p3 + p2 * 2 + p1 * 2 + p0 * 2 + q0 + q1 + q2 + q3 + q4, 4);
        p[0] = so_round2(p6 + p5 + p4 + p3 + p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1 + q2 + q3 + q4 + q5, 4);
        q[0] = so_round2(p5 + p4 + p3 + p2 + p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2 + q3 + q4 + q5 + q6, 4);
        q[1] = so_round2(p4 + p3 + p2 + p1 + p0 + q0 * 2 + q1 * 2 + q2 * 2 + q3 + q4 + q5 + q6 * 2, 4);
        q[2] = so_round2(p3 + p2 + p1 + p0 + q0 + q1 * 2 + q2 * 2 + q3 * 2 + q4 + q5 + q6 * 3, 4);
        q[3] = so_round2(p2 + p1 + p0 + q0 + q1 + q2 * 2 + q3 * 2 + q4 * 2 + q5 + q6 * 4, 4);
        q[4] = so_round2(p1 + p0 + q0 + q1 + q2 + q3 * 2 + q4 * 2 + q5 * 2 + q6 * 5, 4);
        q[5] = so_round2(p0 + q0 + q1 + q2 + q3 + q4 * 2 + q5 * 2 + q6 * 7, 4);
      } else if (flat) {
        /* The 8-tap flat filter (also the 14-tap's narrow fallback, :380-385). */
        const int p3 = p[3], p2 = p[2], p1 = p[1], p0 = p[0], q0 = q[0], q1 = q[1], q2 = q[2], q3 = q[3];
        p[2] = so_round2(p3 + p3 + p3 + 2 * p2 + p1 + p0 + q0, 3);
        p[1] = so_round2(p3 + p3 + p2 + 2 * p1 + p0 + q0 + q1, 3);
        p[0] = so_round2(p3 + p2 + p1 + 2 * p0 + q0 + q1 + q2, 3);
        q[0] = so_round2(p2 + p1 + p0 + 2 * q0 + q1 + q2 + q3, 3);
        q[1] = so_round2(p1 + p0 + q0 + 2 * q1 + q2 + q3 + q3, 3);
        q[2] = so_round2(p0 + q0 + q1 + 2 * q2 + q3 + q3 + q3, 3);
      } else {
        so_filter4(&p[1], &p[0], &q[0], &q[1], hev, lo, hi, center);
      }
      break;
    }
    default:
      return -1;
  }
  for (int k = 0; k < half; k++) {
    s[half - 1 - k] = p[k];
    s[half + k] = q[k];
  }
  return 0;
}

/* ======================================================================
 * CDEF: the libaom restatements of cdef/cdef_test.go.
 * ====================================================================== */
#define SO_BSTRIDE 144
#define SO_VERY_LARGE 0x4000

/* referenceCDEFDirections (:297-306), referenceCDEFPrimaryTaps and
 * referenceCDEFSecondaryTaps (:308-309). */
static const int so_dirs[8][2] = {
    {-1 * SO_BSTRIDE + 1, -2 * SO_BSTRIDE + 2}, {1, -1 * SO_BSTRIDE + 2}, {1, 2}, {1, 1 * SO_BSTRIDE + 2},
    {1 * SO_BSTRIDE + 1, 2 * SO_BSTRIDE + 2},  {1 * SO_BSTRIDE, 2 * SO_BSTRIDE + 1},
    {1 * SO_BSTRIDE, 2 * SO_BSTRIDE},          {1 * SO_BSTRIDE, 2 * SO_BSTRIDE - 1}};
static const int so_pri_taps[2][2] = {{4, 2}, {3, 3}};
static const int so_sec_taps[2] = {2, 1};

/* msbReference (:400-407). */
static int so_msb(int v) {
  int n = 0;
  while (v > 1) {
    v >>= 1;
    n++;
  }
  return n;
}

/* constrainReference (:379-386). */
static int so_constrain(int diff, int threshold, int damping) {
  if (threshold == 0) return 0;
  int shift = damping - so_msb(threshold);
  if (shift < 0) shift = 0;
  const int m = so_clamp(threshold - (so_abs(diff) >> shift), 0, so_abs(diff));
  return diff < 0 ? -m : m;
}

/* adjustStrengthReference (:388-398). */
int so_cdef_adjust_strength(int strength, int32_t variance) {
  if (variance == 0) return 0;
  int i = 0;
  const int v = variance >> 6;
  if (v != 0) i = so_msb(v) < 12 ? so_msb(v) : 12;
  return (strength * (4 + i) + 8) >> 4;
}

/* filterBlockLibaomReference (:232-295): dst[dst_origin + row*dst_stride +
 * col] for a width x height block whose input sample (0,0) is
 * input[input_origin], input stride 144. */
void so_cdef_filter_block(uint16_t* dst, int dst_stride, int dst_origin, const uint16_t* input, int input_origin,
                          int pri, int sec, int dir, int pri_damping, int sec_damping, int coeff_shift, int width,
                          int height) {
  const int clip = pri != 0 && sec != 0;
  const int* pt = so_pri_taps[(pri >> coeff_shift) & 1];
  for (int row = 0; row < height; row++) {
    for (int col = 0; col < width; col++) {
      const int base = input_origin + row * SO_BSTRIDE + col;
      const int x = input[base];
      int sum = 0, mx = x, mn = x;
      for (int k = 0; k < 2; k++) {
        if (pri != 0) {
          const int p0 = input[base + so_dirs[dir][k]], p1 = input[base - so_dirs[dir][k]];
          sum += pt[k] * so_constrain(p0 - x, pri, pri_damping);
          sum += pt[k] * so_constrain(p1 - x, pri, pri_damping);
          if (clip) {
            if (p0 != SO_VERY_LARGE && p0 > mx) mx = p0;
            if (p1 != SO_VERY_LARGE && p1 > mx) mx = p1;
            if (p0 < mn) mn = p0;
            if (p1 < mn) mn = p1;
          }
        }
        if (sec != 0) {
          const int s[4] = {input[base + so_dirs[(dir + 2) & 7][k]], input[base - so_dirs[(dir + 2) & 7][k]],
                            input[base + so_dirs[(dir + 6) & 7][k]], input[base - so_dirs[(dir + 6) & 7][k]]};
          for (int j = 0; j < 4; j++) {
            if (clip) {
              if (s[j] != SO_VERY_LARGE && s[j] > mx) mx = s[j];
              if (s[j] < mn) mn = s[j];
            }
            sum += so_sec_taps[k] * so_constrain(s[j] - x, sec, sec_damping);
          }
        }
      }
      int y = x + ((8 + sum - (sum < 0)) >> 4);
      if (clip) y = so_clamp(y, mn, mx);
      dst[dst_origin + row * dst_stride + col] = (uint16_t)y;
    }
  }
}

/* findDirectionLibaomReference (:681-728). */
int so_cdef_find_dir(const uint16_t* img, int stride, int coeff_shift, int32_t* variance) {
  int32_t cost[8] = {0};
  int partial[8][15];
  static const int div_table[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};
  memset(partial, 0, sizeof(partial));
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      const int x = (int)(img[i * stride + j] >> coeff_shift) - 128;
      partial[0][i + j] += x;
      partial[1][i + j / 2] += x;
      partial[2][i] += x;
      partial[3][3 + i - j / 2] += x;
      partial[4][7 + i - j] += x;
      partial[5][3 - i / 2 + j] += x;
      partial[6][j] += x;
      partial[7][i / 2 + j] += x;
    }
  for (int i = 0; i < 8; i++) {
    cost[2] += (int32_t)(partial[2][i] * partial[2][i]);
    cost[6] += (int32_t)(partial[6][i] * partial[6][i]);
  }
  cost[2] *= div_table[8];
  cost[6] *= div_table[8];
  for (int i = 0; i < 7; i++) {
    cost[0] += (int32_t)((partial[0][i] * partial[0][i] + partial[0][14 - i] * partial[0][14 - i]) * div_table[i + 1]);
    cost[4] += (int32_t)((partial[4][i] * partial[4][i] + partial[4][14 - i] * partial[4][14 - i]) * div_table[i + 1]);
  }
  cost[0] += (int32_t)(partial[0][7] * partial[0][7] * div_table[8]);
  cost[4] += (int32_t)(partial[4][7] * partial[4][7] * div_table[8]);
  for (int i = 1; i < 8; i += 2) {
    for (int j = 0; j < 5; j++) cost[i] += (int32_t)(partial[i][3 + j] * partial[i][3 + j]);
    cost[i] *= div_table[8];
    for (int j = 0; j < 3; j++)
      cost[i] += (int32_t)((partial[i][j] * partial[i][j] + partial[i][10 - j] * partial[i][10 - j]) *
                           div_table[2 * j + 2]);
  }
  int32_t best_cost = 0;
  int best = 0;
  for (int i = 0; i < 8; i++)
    if (cost[i] > best_cost) {
      best_cost = cost[i];
      best = i;
    }
  *variance = (best_cost - cost[(best + 4) & 7]) >> 10;
  return best;
}

/* The chroma direction of a 4:2:2 (xdec 1, ydec 0) or 4:4:0 (xdec 0,
 * ydec 1) plane from the luma direction: the AV1 specification's
 * cdef_uv_dir tables of the CDEF filter process; other layouts keep the
 * luma direction. */
int so_cdef_chroma_dir(int dir, int xdec, int ydec) {
  static const int uv422[8] = {7, 0, 2, 4, 5, 6, 6, 6};
  static const int uv440[8] = {1, 2, 2, 2, 3, 4, 6, 0};
  if (xdec && !ydec) return uv422[dir & 7];
  if (!xdec && ydec) return uv440[dir & 7];
  return dir;
}

/* ======================================================================
 * Wiener: referenceWienerPixel / referenceWienerHorizontal
 * (restoration/restoration_test.go:1884-1925), every output sample
 * recomputing its seven horizontally filtered neighbours.
 * ====================================================================== */
static void so_wiener_rounds(int bd, int* r0, int* r1) {
  *r0 = 3;
  *r1 = 11;
  if (bd == 12) {
    *r0 = 5;
    *r1 = 9;
  }
}

static int so_wiener_h(const uint16_t* src, int stride, int origin, int row, int col, const int16_t* f, int bd,
                       int round0) {
  const int32_t limit = 1 << (bd + 1 + 7 - round0);
  int32_t sum = ((int32_t)src[origin + row * stride + col] << 7) + (1 << (bd + 7 - 1));
  for (int k = 0; k < 7; k++) sum += (int32_t)src[origin + row * stride + col - 3 + k] * f[k];
  return so_clamp(so_round2(sum, round0), 0, limit - 1);
}

/* src: sample (0,0) of the unit at src[origin], with 3 samples of context
 * on every side; vf7/hf7: the 7 taps as NewWienerFilter lays them out. */
void so_wiener(const uint16_t* src, int stride, int origin, uint16_t* dst, int dst_stride, int w, int h,
               const int16_t* vf7, const int16_t* hf7, int bd) {
  int round0, round1;
  so_wiener_rounds(bd, &round0, &round1);
  const int maxv = (1 << bd) - 1;
  for (int row = 0; row < h; row++)
    for (int col = 0; col < w; col++) {
      const int center = so_wiener_h(src, stride, origin, row, col, hf7, bd, round0);
      int32_t sum = ((int32_t)center << 7) - (1 << (bd + round1 - 1));
      for (int k = 0; k < 7; k++) sum += (int32_t)so_wiener_h(src, stride, origin, row - 3 + k, col, hf7, bd, round0) * vf7[k];
      dst[row * dst_stride + col] = (uint16_t)so_clamp(so_round2(sum, round1), 0, maxv);
    }
}

/* ======================================================================
 * Self-guided filter, in the AV1 specification's formulation (the box
 * filter process and the self guided filter process of loop restoration):
 * each A/B entry from a direct (2r+1)^2 window sum of the source, the
 * strength s from the set's radius and epsilon, x/(x+1) and 1/n by formula.
 * The intermediate follows frozenSGRIntermediate
 * (restoration_test.go:456-493) in using the unscaled box sum in B.
 * ====================================================================== */

/* The sixteen parameter sets: radius and epsilon of each pass. */
static const int so_sgr_sets[16][4] = {
    {2, 12, 1, 4},  {2, 15, 1, 6},  {2, 18, 1, 8},  {2, 21, 1, 9},  {2, 24, 1, 10}, {2, 29, 1, 11},
    {2, 36, 1, 12}, {2, 45, 1, 13}, {2, 56, 1, 14}, {2, 68, 1, 15}, {0, 0, 1, 5},   {0, 0, 1, 8},
    {0, 0, 1, 11},  {0, 0, 1, 14},  {2, 30, 0, 0},  {2, 75, 0, 0}};

/* Radius and strength s = round(2^20 / (n^2 * eps)) of both passes. */
void so_sgr_params(int set, int* r0, int* s0, int* r1, int* s1) {
  int rs[2], ss[2];
  for (int pass = 0; pass < 2; pass++) {
    const int r = so_sgr_sets[set][2 * pass], eps = so_sgr_sets[set][2 * pass + 1];
    rs[pass] = r;
    ss[pass] = 0;
    if (r) {
      const int n = (2 * r + 1) * (2 * r + 1);
      const int n2e = n * n * eps;
      ss[pass] = ((1 << 20) + n2e / 2) / n2e;
    }
  }
  *r0 = rs[0];
  *s0 = ss[0];
  *r1 = rs[1];
  *s1 = ss[1];
}

/* The projection weights from the coded xqd pair (the decoder's xq). */
void so_sgr_decode_xq(const int8_t* xqd, int set, int* xq0, int* xq1) {
  const int r0 = so_sgr_sets[set][0], r1 = so_sgr_sets[set][2];
  if (r0 == 0) {
    *xq0 = 0;
    *xq1 = 128 - xqd[1];
  } else if (r1 == 0) {
    *xq0 = xqd[0];
    *xq1 = 0;
  } else {
    *xq0 = xqd[0];
    *xq1 = 128 - xqd[0] - xqd[1];
  }
}

/* x/(x+1) in 1/256 units as the spec defines it (z >= 255 gives 256). */
int so_sgr_x_by_xplus1(int z) {
  if (z >= 255) return 256;
  if (z == 0) return 1;
  return ((z << 8) + z / 2) / (z + 1);
}

/* 1/n in 1/4096 units. */
int so_sgr_one_by_n(int n) { return ((1 << 12) + n / 2) / n; }

/* The A/B grid of one pass at (i, j), i in -1..h, j in -1..w. */
static void so_sgr_ab(const uint16_t* src, int stride, int origin, int i, int j, int r, int s, int bd, int* A,
                      int* B) {
  const int n = (2 * r + 1) * (2 * r + 1);
  int64_t a = 0, b = 0;
  for (int dy = -r; dy <= r; dy++)
    for (int dx = -r; dx <= r; dx++) {
      const int c = src[origin + (i + dy) * stride + j + dx];
      a += (int64_t)c * c;
      b += c;
    }
  a = so_round2_64(a, 2 * (bd - 8));
  const int64_t d = so_round2_64(b, bd - 8);
  int64_t p = a * n - d * d;
  if (p < 0) p = 0;
  const int z = (int)so_round2_64(p * s, 20);
  const int a2 = so_sgr_x_by_xplus1(z);
  const int64_t b2 = (int64_t)((1 << 8) - a2) * b * so_sgr_one_by_n(n);
  *A = a2;
  *B = (int)so_round2_64(b2, 12);
}

/* One pass's filtered value (in 1/16 units) at (i, j). */
static int so_sgr_filtered(const uint16_t* src, int stride, int origin, int i, int j, int pass, int r, int s, int bd) {
  int a = 0, b = 0;
  for (int dy = -1; dy <= 1; dy++)
    for (int dx = -1; dx <= 1; dx++) {
      int weight;
      if (pass == 0) {
        weight = ((i + dy) & 1) ? (dx == 0 ? 6 : 5) : 0;
      } else {
        weight = (dx == 0 || dy == 0) ? 4 : 3;
      }
      if (!weight) continue;
      int A, B;
      so_sgr_ab(src, stride, origin, i + dy, j + dx, r, s, bd, &A, &B);
      a += weight * A;
      b += weight * B;
    }
  const int shift = (pass == 0 && (i & 1)) ? 4 : 5;
  const int v = a * src[origin + i * stride + j] + b;
  return so_round2(v, 8 + shift - 4);
}

/* src: sample (0,0) of the unit at src[origin], 3 samples of context on
 * every side.  The projection wraps to int16 before the clip, as goav1's
 * sgrWeightedRow does (restoration/selfguided.go:233-247). */
void so_sgr(const uint16_t* src, int stride, int origin, uint16_t* dst, int dst_stride, int w, int h, int set,
            const int8_t* xqd, int bd) {
  int r0, s0, r1, s1, xq0, xq1;
  so_sgr_params(set, &r0, &s0, &r1, &s1);
  so_sgr_decode_xq(xqd, set, &xq0, &xq1);
  const int maxv = (1 << bd) - 1;
  for (int i = 0; i < h; i++)
    for (int j = 0; j < w; j++) {
      const int u = src[origin + i * stride + j] << 4;
      int v = u << 7;
      if (r0) v += xq0 * (so_sgr_filtered(src, stride, origin, i, j, 0, r0, s0, bd) - u);
      if (r1) v += xq1 * (so_sgr_filtered(src, stride, origin, i, j, 1, r1, s1, bd) - u);
      const int wv = (int16_t)so_round2(v, 11);
      dst[i * dst_stride + j] = (uint16_t)so_clamp(wv, 0, maxv);
    }
}

/* ======================================================================
 * Film grain, in the specification's formulation: the grain generation
 * process (luma and chroma templates with the auto-regressive filter; the
 * chroma filter's last tap weighting the co-located average of the luma
 * grain) and the add-noise process (noise stripes of 34 rows per 32-row
 * luma stripe, one 8-bit random offset per 32x32 luma block, horizontal
 * overlap blends inside the stripe, vertical blends against the previous
 * stripe's two extra rows, then scaling and clipping).  Templates are
 * 73x82 int16, stride 82, as goav1 stores them.
 * ====================================================================== */
#define SO_GW 82
#define SO_GH 73

static uint16_t so_rand(uint16_t* reg, int bits) {
  const uint16_t r = *reg;
  const uint16_t bit = ((r >> 0) ^ (r >> 1) ^ (r >> 3) ^ (r >> 12)) & 1;
  *reg = (uint16_t)((r >> 1) | (bit << 15));
  return (uint16_t)((*reg >> (16 - bits)) & ((1 << bits) - 1));
}

/* Templates of all three planes (luma, cb, cr; each SO_GW * SO_GH). */
void so_grain_templates(int16_t* luma, int16_t* cb, int16_t* cr, const pf_film_grain* fg, int bd, int ssx, int ssy) {
  const int shift = 12 - bd + fg->grain_scale_shift;
  const int gmin = -(1 << (bd - 1)), gmax = (1 << (bd - 1)) - 1;
  memset(luma, 0, sizeof(int16_t) * SO_GW * SO_GH);
  memset(cb, 0, sizeof(int16_t) * SO_GW * SO_GH);
  memset(cr, 0, sizeof(int16_t) * SO_GW * SO_GH);
  uint16_t reg = fg->seed;
  for (int y = 0; y < SO_GH; y++)
    for (int x = 0; x < SO_GW; x++) {
      int g = 0;
      if (fg->num_y_points > 0) g = pf_gaussian_sequence[so_rand(&reg, 11)];
      luma[y * SO_GW + x] = (int16_t)so_round2(g, shift);
    }
  const int lag = fg->ar_coeff_lag;
  const int ar_shift = fg->ar_coeff_shift;
  for (int y = 3; y < SO_GH; y++)
    for (int x = 3; x < SO_GW - 3; x++) {
      int sum = 0, pos = 0;
      for (int dr = -lag; dr <= 0; dr++)
        for (int dc = -lag; dc <= lag; dc++) {
          if (dr == 0 && dc == 0) break;
          sum += luma[(y + dr) * SO_GW + x + dc] * fg->ar_coeffs_y[pos++];
        }
      luma[y * SO_GW + x] = (int16_t)so_clamp(luma[y * SO_GW + x] + so_round2(sum, ar_shift), gmin, gmax);
    }
  const int cw = ssx ? 44 : 82, ch = ssy ? 38 : 73;
  const int cb_on = fg->num_cb_points || fg->chroma_scaling_from_luma;
  const int cr_on = fg->num_cr_points || fg->chroma_scaling_from_luma;
  reg = (uint16_t)(fg->seed ^ 0xb524);
  for (int y = 0; y < ch; y++)
    for (int x = 0; x < cw; x++) {
      int g = 0;
      if (cb_on) g = pf_gaussian_sequence[so_rand(&reg, 11)];
      cb[y * SO_GW + x] = (int16_t)so_round2(g, shift);
    }
  reg = (uint16_t)(fg->seed ^ 0x49d8);
  for (int y = 0; y < ch; y++)
    for (int x = 0; x < cw; x++) {
      int g = 0;
      if (cr_on) g = pf_gaussian_sequence[so_rand(&reg, 11)];
      cr[y * SO_GW + x] = (int16_t)so_round2(g, shift);
    }
  for (int y = 3; y < ch; y++)
    for (int x = 3; x < cw - 3; x++) {
      int sum0 = 0, sum1 = 0, pos = 0;
      for (int dr = -lag; dr <= 0; dr++)
        for (int dc = -lag; dc <= lag; dc++) {
          const int c0 = fg->ar_coeffs_cb[pos], c1 = fg->ar_coeffs_cr[pos];
          if (dr == 0 && dc == 0) {
            if (fg->num_y_points > 0) {
              int l = 0;
              const int lx = ((x - 3) << ssx) + 3, ly = ((y - 3) << ssy) + 3;
              for (int i = 0; i <= ssy; i++)
                for (int j = 0; j <= ssx; j++) l += luma[(ly + i) * SO_GW + lx + j];
              l = so_round2(l, ssx + ssy);
              sum0 += l * c0;
              sum1 += l * c1;
            }
            break;
          }
          sum0 += c0 * cb[(y + dr) * SO_GW + x + dc];
          sum1 += c1 * cr[(y + dr) * SO_GW + x + dc];
          pos++;
        }
      if (cb_on) cb[y * SO_GW + x] = (int16_t)so_clamp(cb[y * SO_GW + x] + so_round2(sum0, ar_shift), gmin, gmax);
      if (cr_on) cr[y * SO_GW + x] = (int16_t)so_clamp(cr[y * SO_GW + x] + so_round2(sum1, ar_shift), gmin, gmax);
    }
}

/* The 256-entry scaling function of a point list (piecewise linear). */
void so_scaling_lut(uint8_t* lut, const uint8_t (*pts)[2], int n) {
  memset(lut, 0, 256);
  if (n == 0) return;
  for (int x = 0; x < pts[0][0]; x++) lut[x] = pts[0][1];
  for (int i = 0; i + 1 < n; i++) {
    const int dy = pts[i + 1][1] - pts[i][1], dx = pts[i + 1][0] - pts[i][0];
    const int delta = dy * ((65536 + (dx >> 1)) / dx);
    for (int x = 0, d = 32768; x < dx; x++, d += delta) lut[pts[i][0] + x] = (uint8_t)(pts[i][1] + (d >> 16));
  }
  for (int x = pts[n - 1][0]; x < 256; x++) lut[x] = pts[n - 1][1];
}

static int so_scale(const uint8_t* lut, int index, int bd) {
  const int shift = bd - 8;
  const int x = index >> shift;
  const int rem = index - (x << shift);
  if (bd == 8 || x == 255) return lut[x];
  return lut[x] + so_round2((lut[x + 1] - lut[x]) * rem, shift);
}

/* Noise of one plane over a frame of frame_w x frame_h luma samples:
 * noise[y * pw + x] for the plane's pw x ph samples. */
static void so_noise_image(int16_t* noise, int pw, int ph, const int16_t* grain, const pf_film_grain* fg, int frame_w,
                           int frame_h, int subx, int suby, int bd) {
  const int gmin = -(1 << (bd - 1)), gmax = (1 << (bd - 1)) - 1;
  const int nstripes = ((frame_h + 1) / 2 + 15) / 16;
  const int sw = pw + 34;
  const int srows = 34 >> suby;
  int16_t* stripes = (int16_t*)calloc((size_t)nstripes * srows * sw, sizeof(int16_t));
  for (int ln = 0; ln < nstripes; ln++) {
    uint16_t reg = fg->seed;
    reg ^= (uint16_t)(((ln * 37 + 178) & 255) << 8);
    reg ^= (uint16_t)((ln * 173 + 105) & 255);
    int16_t* st = stripes + (size_t)ln * srows * sw;
    for (int x = 0; x < (frame_w + 1) / 2; x += 16) {
      const int rnd = so_rand(&reg, 8);
      const int ox = rnd >> 4, oy = rnd & 15;
      const int pox = subx ? 6 + ox : 9 + ox * 2;
      const int poy = suby ? 6 + oy : 9 + oy * 2;
      for (int i = 0; i < (34 >> suby); i++)
        for (int j = 0; j < (34 >> subx); j++) {
          int g = grain[(poy + i) * SO_GW + pox + j];
          const int col = subx ? x + j : x * 2 + j;
          if (col >= sw) continue;
          if (!subx) {
            if (j < 2 && fg->overlap && x > 0) {
              const int old = st[i * sw + col];
              g = j == 0 ? old * 27 + g * 17 : old * 17 + g * 27;
              g = so_clamp(so_round2(g, 5), gmin, gmax);
            }
          } else {
            if (j == 0 && fg->overlap && x > 0) {
              const int old = st[i * sw + col];
              g = so_clamp(so_round2(old * 23 + g * 22, 5), gmin, gmax);
            }
          }
          st[i * sw + col] = (int16_t)g;
        }
    }
  }
  for (int y = 0; y < ph; y++) {
    const int ln = y >> (5 - suby);
    const int i = y - (ln << (5 - suby));
    for (int x = 0; x < pw; x++) {
      int g = stripes[((size_t)ln * srows + i) * sw + x];
      if (!suby) {
        if (i < 2 && ln > 0 && fg->overlap) {
          const int old = stripes[((size_t)(ln - 1) * srows + i + 32) * sw + x];
          g = i == 0 ? old * 27 + g * 17 : old * 17 + g * 27;
          g = so_clamp(so_round2(g, 5), gmin, gmax);
        }
      } else {
        if (i < 1 && ln > 0 && fg->overlap) {
          const int old = stripes[((size_t)(ln - 1) * srows + i + 16) * sw + x];
          g = so_clamp(so_round2(old * 23 + g * 22, 5), gmin, gmax);
        }
      }
      noise[(size_t)y * pw + x] = (int16_t)g;
    }
  }
  free(stripes);
}

/* Grain on one plane.  Samples are uint16 (any bit depth); src/dst have
 * `stride` samples per row and the plane's ((frame_w + subx) >> subx) x
 * ((frame_h + suby) >> suby) samples; luma (frame_w x frame_h, luma_stride)
 * gives chroma its scaling index.  grain is the plane's template, lut its
 * scaling function. */
void so_grain_apply_plane(const uint16_t* src, uint16_t* dst, int stride, const uint16_t* luma, int luma_stride,
                          int frame_w, int frame_h, const int16_t* grain, const uint8_t* lut, const pf_film_grain* fg,
                          int plane, int bd, int ssx, int ssy) {
  const int subx = plane ? ssx : 0, suby = plane ? ssy : 0;
  const int pw = (frame_w + subx) >> subx, ph = (frame_h + suby) >> suby;
  int16_t* noise = (int16_t*)malloc(sizeof(int16_t) * (size_t)pw * ph);
  so_noise_image(noise, pw, ph, grain, fg, frame_w, frame_h, subx, suby, bd);
  int minv = 0, maxl = (256 << (bd - 8)) - 1, maxc = maxl;
  if (fg->clip_to_restricted_range) {
    minv = 16 << (bd - 8);
    maxl = 235 << (bd - 8);
    maxc = fg->matrix_identity ? maxl : 240 << (bd - 8);
  }
  const int shift = fg->scaling_shift;
  for (int y = 0; y < ph; y++)
    for (int x = 0; x < pw; x++) {
      const int orig = src[y * stride + x];
      int index = orig;
      if (plane) {
        const int lx = x << subx, ly = y << suby;
        const int nx = lx + 1 < frame_w - 1 ? lx + 1 : frame_w - 1;
        const int avg = subx ? so_round2(luma[ly * luma_stride + lx] + luma[ly * luma_stride + nx], 1)
                             : luma[ly * luma_stride + lx];
        if (fg->chroma_scaling_from_luma) {
          index = avg;
        } else {
          const int lm = (plane == 1 ? fg->cb_luma_mult : fg->cr_luma_mult) - 128;
          const int cm = (plane == 1 ? fg->cb_mult : fg->cr_mult) - 128;
          const int off = (plane == 1 ? fg->cb_offset : fg->cr_offset) - 256;
          const int combined = avg * lm + orig * cm;
          index = so_clamp((combined >> 6) + off * (1 << (bd - 8)), 0, (1 << bd) - 1);
        }
      }
      const int n = so_round2(so_scale(lut, index, bd) * noise[(size_t)y * pw + x], shift);
      dst[y * stride + x] = (uint16_t)so_clamp(orig + n, minv, plane ? maxc : maxl);
    }
  free(noise);
}
