// pf_fg.cu - film-grain synthesis and reference-frame border extension.
//
// Film grain follows goav1's publication path: internal/av1/decoder/
// postfilter_filmgrain.go:192-263 (plane activity), :516-628 (LUTs, luma then
// chroma templates, chroma planes then luma, into a display copy) and the
// filmgrain package: random.go:15-72 (LFSR, stripe seeds), luma.go:24-158 and
// chroma.go:29-241 (templates with the AR recursion), scaling.go:18-121,
// apply.go:72-343, :414-546 and blend.go:16-25 (per-32x32 block offsets drawn
// in order from each stripe's LFSR, overlap blends, noise and clipping).
//
// GPU shape: the 82x73 templates are generated by one 3-warp CTA per frame.
// The Gaussian fill is split over the CTA's 96 threads: the LFSR is linear
// over GF(2)^16, so thread k starts from M^(kL) * seed (jump matrices
// precomputed on the host) and walks its L draws; the AR filter runs as a
// wavefront over t = x + 4y (every AR input of sample (y, x) has a smaller
// t), one warp per template, rows in lanes, neighbours passed between lanes
// by shuffles.  Offsets come from one thread per 32-row stripe.  The apply
// is one thread per output sample, 64x16-sample tiles per CTA.
#include <atomic>

#include "pf_common.cuh"
#include "pf_tables.h"

namespace pf {

constexpr int kGW = 82, kGH = 73;

__device__ __forceinline__ int rpow2(int v, int bits) { return bits <= 0 ? v : (v + (1 << (bits - 1))) >> bits; }

__device__ __forceinline__ uint16_t lfsr(uint16_t& reg, int bits) {
  const uint16_t bit = ((reg >> 0) ^ (reg >> 1) ^ (reg >> 3) ^ (reg >> 12)) & 1;
  reg = (uint16_t)((reg >> 1) | (bit << 15));
  return (uint16_t)((reg >> (16 - bits)) & ((1 << bits) - 1));
}

// ---- grain templates ----
//
// Shared layout of a template while it is generated: 32 lanes x 4 padded
// rows of 128 samples.  Template row y is AR row v = y - 3 (v = -3..h-4);
// it lives in padded row 4 * (v mod 32) + floor(v / 32) + 1, column x at
// x + 4.  Lane r of the AR warp owns AR rows r, r + 32, r + 64 (rows -3..-1
// ride on lanes 29..31), so the rows a lane visits are consecutive in
// memory and its position at wavefront step t is one running address,
// 508 r + t + 132.  Samples that the recursion must pass through unchanged
// (rows 0-2, the three border columns on each side, the padding) are
// stored with kNonAr added; an AR output is a plain sample.  The stored
// value then tells each step what to do, and no step needs a bounds test.
constexpr int kTplRow = 128;
constexpr int kTplPlane = 32 * 4 * kTplRow;
constexpr int kTplCol0 = 4;
constexpr int kNonAr = 16384;  // above any grain sample (|g| <= 2048)
constexpr int kFgTemplateThreads = 96;

struct TplSmem {
  int16_t g[3][kTplPlane];  // luma, Cb, Cr
  int16_t lt[kTplPlane];    // the chroma AR's luma term, chroma layout
  int16_t gauss[2048];      // the Gaussian sequence
};

__device__ __forceinline__ int tpl_at(int y, int x) {
  const int v = y - 3;
  return (4 * (v & 31) + (v >> 5) + 1) * kTplRow + x + kTplCol0;
}

__device__ __forceinline__ int tpl_decode(int s) { return s >= kNonAr / 2 ? s - kNonAr : s; }

// AR recursion of one template (luma.go:83-158 / chroma.go:92-199 generic
// form), run by one warp as a single wavefront with no barrier: AR row v
// is at column x = t - 4v at step t, so every AR input of (v, x) from the
// rows above was finished at an earlier step.  Rows v - d at column
// x + LAG reach the lane from lane r - 1 by warp shuffles out of small
// register rings: the row directly above as that lane's output of 4 - LAG
// steps back, and the rows further up as the values that lane itself
// received 4 steps back (for LAG 3 those two are passed on as one packed
// pair of int16; for LAG 2 and 3 a pair of taps costs one __dp2a_lo).
// The filter runs in transposed form: a value arriving from the rows above
// goes straight into the partial sums of the outputs x .. x + 2*LAG it
// reaches, and the lane's own output adds its in-row products to the next
// LAG outputs' sums, so the loop-carried path is shuffle -> multiply-add ->
// shift -> clip.  The partial sums rotate through acc[] with the step and
// start from the rounding offset; the rings are whole rotations long, so
// the unrolled steps rename registers.
// The wavefront starts 4*LAG steps early so that the pass-through rows
// above the first AR row are in the rings when row 0 needs them, and may
// run a few steps past the last AR output (those steps only rewrite
// pass-through samples with their own values).  LAG is a template argument
// (coefficients in registers, unrolled taps); with LAG 0 only the luma
// term remains, one sample a lane.
template <int LAG, bool kLt>
__device__ __forceinline__ void ar_warp(int16_t* g, const int16_t* lt, const FgTemplateArgs& p, int plane, int w, int h) {
  constexpr int kTaps = 2 * LAG * (LAG + 1);  // causal neighbours before the centre
  const int lane = threadIdx.x & 31;
  const int cs = p.coeff_shift, ro = 1 << (cs - 1);
  const int gmin = -(1 << (p.bd - 1)), gmax = (1 << (p.bd - 1)) - 1;
  const int8_t* cf = p.coeffs[plane];
  if constexpr (LAG == 0) {
    if constexpr (!kLt) return;
    const int coL = cf[0], aw = w - 6;
    for (int i = lane; i < aw * (h - 3); i += 32) {
      const int o = tpl_at(3 + i / aw, 3 + i % aw);
      g[o] = (int16_t)iclip(g[o] + ((lt[o] * coL + ro) >> cs), gmin, gmax);
    }
  } else {
    constexpr int W = 2 * LAG + 1;
    constexpr int U = 2 * W;  // ring length (at least 5) and unroll
    // Per output slot j (the output j columns right of the arriving value):
    // the two farthest rows' taps as a byte pair (LAG 2 and 3) and the
    // nearest row's tap (LAG 1 and 3).
    int cp[W], c1[W], cin[LAG + 1];
#pragma unroll
    for (int j = 0; j < W; j++) {
      cp[j] = 0;
      c1[j] = 0;
      if constexpr (LAG >= 2)
        cp[j] = (int)(uint8_t)cf[2 * LAG - j] | ((int)(uint8_t)cf[W + 2 * LAG - j] << 8);
      if constexpr (LAG == 3) c1[j] = cf[2 * W + 2 * LAG - j];
      if constexpr (LAG == 1) c1[j] = cf[2 * LAG - j];
    }
#pragma unroll
    for (int m = 1; m <= LAG; m++) cin[m] = cf[LAG * W + LAG - m];
    const int coL = kLt ? cf[kTaps] : 0;
    int acc[W], ring[U], ring2[U];
#pragma unroll
    for (int j = 0; j < W; j++) acc[j] = ro;
#pragma unroll
    for (int j = 0; j < U; j++) ring[j] = ring2[j] = 0;
    const int src = (lane + 31) & 31;
    const int pos0 = 508 * lane + 132;
    // The last step finishes column w - 4 of the last AR row.
    const int tend = 4 * (h - 4) + w - 3;
    for (int t0 = -4 * LAG; t0 < tend; t0 += U) {
      int16_t* gp = g + pos0 + t0;
      const int16_t* lp = kLt ? lt + pos0 + t0 : nullptr;
#pragma unroll
      for (int k = 0; k < U; k++) {
        if constexpr (LAG == 3) {
          // (row y-3, row y-2) as a pair, then row y-1.
          const int q = __shfl_sync(0xffffffffu, ring2[(k + U - 4) % U], src);
          const int v1 = __shfl_sync(0xffffffffu, ring[(k + U - 1) % U], src);
#pragma unroll
          for (int j = W - 1; j >= 0; j--) acc[(j + k) % W] = __dp2a_lo(q, cp[j], acc[(j + k) % W]);
#pragma unroll
          for (int j = W - 1; j >= 0; j--) acc[(j + k) % W] += c1[j] * v1;
          ring2[k] = (int)__byte_perm((unsigned)q, (unsigned)v1, 0x5432);
        } else if constexpr (LAG == 2) {
          const int v1 = __shfl_sync(0xffffffffu, ring[(k + U - 2) % U], src);
          const int v2 = __shfl_sync(0xffffffffu, ring2[(k + U - 4) % U], src);
          const int pr = (int)__byte_perm((unsigned)v2, (unsigned)v1, 0x5410);
          ring2[k] = v1;
#pragma unroll
          for (int j = W - 1; j >= 0; j--) acc[(j + k) % W] = __dp2a_lo(pr, cp[j], acc[(j + k) % W]);
        } else {
          const int v1 = __shfl_sync(0xffffffffu, ring[(k + U - 3) % U], src);
#pragma unroll
          for (int j = W - 1; j >= 0; j--) acc[(j + k) % W] += c1[j] * v1;
        }
        const int g0 = gp[k];
        int s = acc[k % W];
        if constexpr (kLt) s += lp[k] * coL;
        const int o = iclip(g0 + (s >> cs), gmin, gmax);
        const int out = g0 >= kNonAr / 2 ? g0 - kNonAr : o;
        gp[k] = (int16_t)out;
        ring[k] = out;
        // Output x's in-row products for columns x + 1 .. x + LAG; its slot
        // then serves column x + W.
        acc[k % W] = ro;
#pragma unroll
        for (int m = 1; m <= LAG; m++) acc[(m + k) % W] += cin[m] * out;
      }
    }
  }
}

template <bool kLt>
__device__ __forceinline__ void ar_warp_lag(int16_t* g, const int16_t* lt, const FgTemplateArgs& p, int plane, int w, int h) {
  switch (p.lag) {
    case 0: ar_warp<0, kLt>(g, lt, p, plane, w, h); break;
    case 1: ar_warp<1, kLt>(g, lt, p, plane, w, h); break;
    case 2: ar_warp<2, kLt>(g, lt, p, plane, w, h); break;
    default: ar_warp<3, kLt>(g, lt, p, plane, w, h); break;
  }
}

// Luma term of the chroma AR (chroma.go:92-199): at each chroma AR position
// the luma grain averaged over the co-located 1, 2 or 4 samples, into lt
// (chroma layout).  The luma samples read are all AR positions, which hold
// plain values.  All threads of the CTA.
__device__ __forceinline__ void luma_term(int16_t* lt, const int16_t* luma, int sx, int sy, int w, int h) {
  const int aw = w - 6;
  for (int i = threadIdx.x; i < aw * (h - 3); i += blockDim.x) {
    const int y = 3 + i / aw, x = 3 + i % aw;
    const int lx = ((x - 3) << sx) + 3, ly = ((y - 3) << sy) + 3;
    const int a = tpl_at(ly, lx);
    int s = luma[a];
    if (sx) s += luma[a + 1];
    if (sy) {
      const int b = tpl_at(ly + 1, lx);
      s += luma[b];
      if (sx) s += luma[b + 1];
    }
    lt[tpl_at(y, x)] = (int16_t)rpow2(s, sx + sy);
  }
}

// Jump matrices: g_jump[t][k][c] = M^(k*L_t) e_c for the three template
// shapes (t = 0: 82x73, 1: 44x73, 2: 44x38), L_t = ceil(samples / 96), so
// that thread k of the CTA starts its share of the draws at draw k * L_t.
// Global memory rather than constant: every thread reads its own row.
__device__ int16_t g_gauss[2048];
__device__ uint16_t g_jump[3][kFgTemplateThreads][16];
__device__ int g_jump_len[3];

__device__ __forceinline__ uint16_t gf2_apply(const uint16_t* cols, uint16_t v) {
  uint16_t r = 0;
#pragma unroll
  for (int c = 0; c < 16; c++)
    if ((v >> c) & 1) r ^= cols[c];
  return r;
}

// Gaussian fill of one template (luma.go:32-38 / chroma.go:38-44): draw i of
// the plane's LFSR goes to sample (i / w, i % w).  All threads of the CTA,
// each walking L consecutive draws from its jumped LFSR state.
__device__ __forceinline__ void gauss_fill(int16_t* g, const int16_t* gauss, uint16_t seed, int w, int h, int shape, int shift) {
  const int L = g_jump_len[shape];
  uint16_t reg = gf2_apply(g_jump[shape][threadIdx.x], seed);
  int i = threadIdx.x * L;
  const int iend = imin(i + L, w * h);
  if (i >= iend) return;
  int y = i / w, x = i - y * w;
  int row = tpl_at(y, 0);
  for (; i < iend; i++) {
    const int v = rpow2(gauss[lfsr(reg, 11)], shift);
    const bool ar = y >= 3 && x >= 3 && x < w - 3;
    g[row + x] = (int16_t)(ar ? v : v + kNonAr);
    if (++x == w) {
      x = 0;
      row = tpl_at(++y, 0);
    }
  }
}

// One frame's templates: Gaussian fills of the three planes by the whole
// CTA, the luma AR on warp 0, the luma term, then the Cb and Cr AR side by
// side on warps 1 and 2, and the templates written out (stride 82) with
// the pass-through marks taken off.
__device__ __forceinline__ void fg_templates(const FgTemplateArgs& p, int16_t* gy, int16_t* gu, int16_t* gv, TplSmem& S) {
  const int warp = threadIdx.x >> 5;
  int16_t* outs[3] = {gy, gu, gv};
  const int cw = p.ssx ? 44 : kGW, ch = p.ssy ? 38 : kGH;
  const int cshape = p.ssx ? (p.ssy ? 2 : 1) : 0;
  {
    const int4 fill = make_int4(0x40004000, 0x40004000, 0x40004000, 0x40004000);
    static_assert(kNonAr == 0x4000, "fill pattern");
    int4* g4 = reinterpret_cast<int4*>(S.g[0]);
    for (int i = threadIdx.x; i < 3 * kTplPlane / 8; i += blockDim.x) g4[i] = fill;
    const int4* src = reinterpret_cast<const int4*>(g_gauss);
    int4* dst = reinterpret_cast<int4*>(S.gauss);
    for (int i = threadIdx.x; i < 2048 / 8; i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const int shift = 12 - p.bd + p.grain_scale_shift;
  if (p.num_y_points != 0) gauss_fill(S.g[0], S.gauss, p.seed, kGW, kGH, 0, shift);
  if (p.active[1]) gauss_fill(S.g[1], S.gauss, (uint16_t)(p.seed ^ 0xb524), cw, ch, cshape, shift);
  if (p.active[2]) gauss_fill(S.g[2], S.gauss, (uint16_t)(p.seed ^ 0x49d8), cw, ch, cshape, shift);
  __syncthreads();
  if (warp == 0 && p.num_y_points != 0 && p.lag != 0) ar_warp_lag<false>(S.g[0], nullptr, p, 0, kGW, kGH);
  __syncthreads();
  const bool lumaTerm = p.num_y_points != 0;
  if (lumaTerm) {
    luma_term(S.lt, S.g[0], p.ssx, p.ssy, cw, ch);
    __syncthreads();
  }
  const bool runC = warp >= 1 && warp <= 2 && p.active[warp] && !(p.lag == 0 && p.num_y_points == 0);
  if (runC) {
    if (lumaTerm)
      ar_warp_lag<true>(S.g[warp], S.lt, p, warp, cw, ch);
    else
      ar_warp_lag<false>(S.g[warp], nullptr, p, warp, cw, ch);
  }
  __syncthreads();
  // Two samples per 32-bit store (rows of 82 samples keep pairs aligned).
  for (int pl = 0; pl < 3; pl++) {
    if (!outs[pl]) continue;
    uint32_t* o = reinterpret_cast<uint32_t*>(outs[pl]);
    for (int i = threadIdx.x; i < kGH * kGW / 2; i += blockDim.x) {
      const int y = i / (kGW / 2), x = 2 * (i - y * (kGW / 2));
      const uint32_t s = *reinterpret_cast<const uint32_t*>(&S.g[pl][tpl_at(y, x)]);
      const int lo = tpl_decode((int16_t)(s & 0xffff)), hi = tpl_decode((int16_t)(s >> 16));
      o[i] = (uint32_t)(uint16_t)lo | ((uint32_t)(uint16_t)hi << 16);
    }
  }
}

// Offsets of every 32x32 block: row r uses the LFSR seeded by stripe r
// (random.go:39-49), one Number(8) per block in order (apply.go:72-125).
__device__ __forceinline__ void fg_offsets_row(uint16_t seed, int r, int cols, uint8_t* out) {
  const int n = r;  // lumaLine >> 5 with lumaLine = 32 r
  uint16_t reg = seed;
  reg ^= (uint16_t)(((n * 37 + 178) & 255) << 8);
  reg ^= (uint16_t)((n * 173 + 105) & 255);
  for (int b = 0; b < cols; b++) out[r * cols + b] = (uint8_t)lfsr(reg, 8);
}

__device__ __forceinline__ int scale_lut(const uint8_t* lut, int index, int bd) {
  index = iclip(index, 0, (1 << bd) - 1);
  const int shift = bd - 8;
  const int x = index >> shift;
  if (bd == 8 || x == 255) return lut[x];
  const int rem = index - (x << shift);
  const int start = lut[x], end = lut[x + 1];
  return (uint8_t)(start + rpow2((end - start) * rem, shift));
}

__device__ __forceinline__ int blend_w(int prev, int cur, int pw, int cw, int bd) {
  return iclip(rpow2(prev * pw + cur * cw, 5), -(1 << (bd - 1)), (1 << (bd - 1)) - 1);
}

// Display = reference with grain added on the cropped area of active planes;
// every allocated sample of the display frame is written.
// One column x of up to 4 rows y0.. of one display plane (all inside one
// 32-row grain block row): per-block values once, then per sample.
// kFgRowGroup: rows of the column whose loads go out together (1, 2 or 4,
// the grain group's tile setting).
template <typename T, int kFgRowGroup>
__device__ __forceinline__ void fg_apply_col(const DFrame& ref, const DFrame& disp, const FgArgs& a, const uint8_t* lut,
                                             int plane, int x, int y0, int nrows) {
  // Plane descriptors and parameters by value: they live in the job table in
  // global memory, which the compiler would re-read after every store.
  const DPlane sp = ref.pl[plane];
  const DPlane dp = disp.pl[plane];
  if (x >= sp.aw) return;
  const int yend = imin(y0 + nrows, sp.ah);
  if (!a.active[plane] || x >= sp.w) {
    if (kFgRowGroup == 1) {
      for (int y = y0; y < yend; y++) row_ptr<T>(dp, y)[x] = row_ptr<T>(sp, y)[x];
      return;
    }
    // Loads of a group of rows before its stores (the compiler may not move
    // a load of the frame above a store to the display frame).
    for (int yg = y0; yg < yend; yg += kFgRowGroup) {
      T v[kFgRowGroup];
#pragma unroll
      for (int k = 0; k < kFgRowGroup; k++)
        if (yg + k < yend) v[k] = row_ptr<T>(sp, yg + k)[x];
#pragma unroll
      for (int k = 0; k < kFgRowGroup; k++)
        if (yg + k < yend) row_ptr<T>(dp, yg + k)[x] = v[k];
    }
    return;
  }
  const int bd = sizeof(T) == 1 ? 8 : ref.bd;  // a constant for 8-bit: the depth shifts fold
  const int sx = plane ? ref.ssx : 0, sy = plane ? ref.ssy : 0;
  const int bwl = 5 - sx, bhl = 5 - sy;
  const int bw = 1 << bwl, bh = 1 << bhl;
  const int row = y0 >> bhl, bcol = x >> bwl;
  const int xi = x - (bcol << bwl);
  const int ovl = 2;
  const int xStart = (a.overlap && bcol > 0) ? imin(sp.w - (bcol << bwl), ovl >> sx) : 0;
  const int yStart = (a.overlap && row > 0) ? imin(sp.h - (row << bhl), ovl >> sy) : 0;
  const uint8_t* offs = a.offsets + row * a.off_cols + bcol;
  const int16_t* gr = a.grain[plane];
  // Template column / row origins of the current, left, top and top-left blocks.
  auto gcol = [&](int offset, int bc) { return 3 + (ovl >> sx) * (3 + (offset >> 4)) + xi + bw * bc; };
  auto grow = [&](int offset, int br) { return 3 + (ovl >> sy) * (3 + (offset & 15)) + bh * br; };
  const int o00 = offs[0];
  const int c00 = gcol(o00, 0), r00 = grow(o00, 0);
  const bool left = xi < xStart;
  int c10 = 0, r10 = 0, c01 = 0, r01 = 0, c11 = 0, r11 = 0;
  if (left) {
    const int o10 = offs[-1];
    c10 = gcol(o10, 1);
    r10 = grow(o10, 0);
  }
  if (yStart > 0) {
    const int o01 = offs[-a.off_cols];
    c01 = gcol(o01, 0);
    r01 = grow(o01, 1);
    if (left) {
      const int o11 = offs[-a.off_cols - 1];
      c11 = gcol(o11, 1);
      r11 = grow(o11, 1);
    }
  }
  // Horizontal blend weights: luma 27/17 then 17/27; subsampled chroma 23/22.
  const int hpw = sx ? 23 : (xi == 1 ? 17 : 27), hcw = sx ? 22 : (xi == 1 ? 27 : 17);
  const int shift = a.scaling_shift;
  int minV = 0, maxV = (256 << (bd - 8)) - 1;
  if (a.clip_restricted) {
    minV = 16 << (bd - 8);
    maxV = (plane == 0 ? 235 : (a.matrix_identity ? 235 : 240)) << (bd - 8);
  }
  const int yclip = imin(yend, sp.h);
  const DPlane lp = ref.pl[0];
  const bool cfl = a.cfl, oddLuma = a.odd_luma;
  const int lumaMult = a.luma_mult[plane] - 128, mult = a.mult[plane] - 128;
  const int offs0 = (a.offset[plane] << (bd - 8)) - (1 << bd);
  if (kFgRowGroup == 1) {
    // One row at a time (40 registers, 6 CTAs per SM).
    for (int y = y0; y < yend; y++) {
      const int s = row_ptr<T>(sp, y)[x];
      if (y >= yclip) {
        row_ptr<T>(dp, y)[x] = (T)s;
        continue;
      }
      const int yi = y - (row << bhl);
      int g = gr[(r00 + yi) * kGW + c00];
      if (left) g = blend_w(gr[(r10 + yi) * kGW + c10], g, hpw, hcw, bd);
      if (yi < yStart) {
        int top = gr[(r01 + yi) * kGW + c01];
        if (left) top = blend_w(gr[(r11 + yi) * kGW + c11], top, hpw, hcw, bd);
        const int vpw = sy ? 23 : (yi == 1 ? 17 : 27), vcw = sy ? 22 : (yi == 1 ? 27 : 17);
        g = blend_w(top, g, vpw, vcw, bd);
      }
      int idx;
      if (plane == 0) {
        idx = s;
      } else {
        // chromaScalingIndex (apply.go:501-520) on the un-grained luma.
        const T* lrow = row_ptr<T>(lp, y << sy);
        const int lx = x << sx;
        int avg = lrow[lx];
        if (sx && !(oddLuma && x == sp.w - 1)) avg = (avg + lrow[lx + 1] + 1) >> 1;
        if (cfl) {
          idx = avg;
        } else {
          const int combined = avg * lumaMult + s * mult;
          idx = iclip((combined >> 6) + offs0, 0, (1 << bd) - 1);
        }
      }
      const int scale = scale_lut(lut, idx, bd);
      const int noise = rpow2(scale * g, shift);
      row_ptr<T>(dp, y)[x] = (T)iclip(s + noise, minV, maxV);
    }
    return;
  }
  // Groups of rows: every load of a group (frame sample, grain, co-located
  // luma) is issued before the group's first store to the display frame.
  for (int yg = y0; yg < yend; yg += kFgRowGroup) {
    int sv[kFgRowGroup], gv[kFgRowGroup], lv[kFgRowGroup];
#pragma unroll
    for (int k = 0; k < kFgRowGroup; k++) {
      const int y = yg + k;
      sv[k] = gv[k] = lv[k] = 0;
      if (y >= yend) continue;
      sv[k] = row_ptr<T>(sp, y)[x];
      if (y >= yclip) continue;
      const int yi = y - (row << bhl);
      int g = gr[(r00 + yi) * kGW + c00];
      if (left) g = blend_w(gr[(r10 + yi) * kGW + c10], g, hpw, hcw, bd);
      if (yi < yStart) {
        int top = gr[(r01 + yi) * kGW + c01];
        if (left) top = blend_w(gr[(r11 + yi) * kGW + c11], top, hpw, hcw, bd);
        const int vpw = sy ? 23 : (yi == 1 ? 17 : 27), vcw = sy ? 22 : (yi == 1 ? 27 : 17);
        g = blend_w(top, g, vpw, vcw, bd);
      }
      gv[k] = g;
      if (plane != 0) {
        // chromaScalingIndex (apply.go:501-520) on the un-grained luma.
        const T* lrow = row_ptr<T>(lp, y << sy);
        const int lx = x << sx;
        int avg = lrow[lx];
        if (sx && !(oddLuma && x == sp.w - 1)) avg = (avg + lrow[lx + 1] + 1) >> 1;
        lv[k] = avg;
      }
    }
#pragma unroll
    for (int k = 0; k < kFgRowGroup; k++) {
      const int y = yg + k;
      if (y >= yend) break;
      const int s = sv[k];
      if (y >= yclip) {
        row_ptr<T>(dp, y)[x] = (T)s;
        continue;
      }
      int idx;
      if (plane == 0 || cfl) {
        idx = plane == 0 ? s : lv[k];
      } else {
        const int combined = lv[k] * lumaMult + s * mult;
        idx = iclip((combined >> 6) + offs0, 0, (1 << bd) - 1);
      }
      const int scale = scale_lut(lut, idx, bd);
      const int noise = rpow2(scale * gv[k], shift);
      row_ptr<T>(dp, y)[x] = (T)iclip(s + noise, minV, maxV);
    }
  }
}

// fg_apply_col for four adjacent columns x .. x + 3 (x a multiple of 4,
// 8-bit planes): the four samples of a row are read and written as one
// 32-bit word, and the block set-up (offsets, template positions, blend
// weights) is shared by the four columns, which always lie in one grain
// block.  Planes whose rows are not 4-byte aligned, or a quad reaching past
// the allocated width, go column by column.
__device__ __forceinline__ void fg_apply_quad(const DFrame& ref, const DFrame& disp, const FgArgs& a,
                                              const uint8_t* lut, int plane, int x, int y0, int nrows) {
  const DPlane sp = ref.pl[plane];
  const DPlane dp = disp.pl[plane];
  if (x >= sp.aw) return;
  const DPlane lp = ref.pl[0];
  const uintptr_t al = reinterpret_cast<uintptr_t>(sp.ptr) | (uintptr_t)sp.stride |
                       reinterpret_cast<uintptr_t>(dp.ptr) | (uintptr_t)dp.stride |
                       reinterpret_cast<uintptr_t>(lp.ptr) | (uintptr_t)lp.stride;
  if (x + 4 > sp.aw || (al & 3)) {
#pragma unroll
    for (int k = 0; k < 4; k++) fg_apply_col<uint8_t, 1>(ref, disp, a, lut, plane, x + k, y0, nrows);
    return;
  }
  const int yend = imin(y0 + nrows, sp.ah);
  auto word = [](const DPlane& p, int y, int xx) { return reinterpret_cast<uint32_t*>(row_ptr<uint8_t>(p, y) + xx); };
  if (!a.active[plane] || x >= sp.w) {
    for (int y = y0; y < yend; y++) *word(dp, y, x) = *word(sp, y, x);
    return;
  }
  const int sx = plane ? ref.ssx : 0, sy = plane ? ref.ssy : 0;
  const int bwl = 5 - sx, bhl = 5 - sy;
  const int bw = 1 << bwl, bh = 1 << bhl;
  const int row = y0 >> bhl, bcol = x >> bwl;
  const int xi = x - (bcol << bwl);
  const int ovl = 2;
  const int xStart = (a.overlap && bcol > 0) ? imin(sp.w - (bcol << bwl), ovl >> sx) : 0;
  const int yStart = (a.overlap && row > 0) ? imin(sp.h - (row << bhl), ovl >> sy) : 0;
  const uint8_t* offs = a.offsets + row * a.off_cols + bcol;
  const int16_t* gr = a.grain[plane];
  auto gcol = [&](int offset, int bc) { return 3 + (ovl >> sx) * (3 + (offset >> 4)) + xi + bw * bc; };
  auto grow = [&](int offset, int br) { return 3 + (ovl >> sy) * (3 + (offset & 15)) + bh * br; };
  const int o00 = offs[0];
  const int c00 = gcol(o00, 0), r00 = grow(o00, 0);
  const bool left = xi < xStart;  // only column xi (and xi + 1 for luma) of the first quad of a block
  int c10 = 0, r10 = 0, c01 = 0, r01 = 0, c11 = 0, r11 = 0;
  if (left) {
    const int o10 = offs[-1];
    c10 = gcol(o10, 1);
    r10 = grow(o10, 0);
  }
  if (yStart > 0) {
    const int o01 = offs[-a.off_cols];
    c01 = gcol(o01, 0);
    r01 = grow(o01, 1);
    if (left) {
      const int o11 = offs[-a.off_cols - 1];
      c11 = gcol(o11, 1);
      r11 = grow(o11, 1);
    }
  }
  const int shift = a.scaling_shift;
  int minV = 0, maxV = 255;
  if (a.clip_restricted) {
    minV = 16;
    maxV = plane == 0 ? 235 : (a.matrix_identity ? 235 : 240);
  }
  const int yclip = imin(yend, sp.h);
  const bool cfl = a.cfl, oddLuma = a.odd_luma;
  const int lumaMult = a.luma_mult[plane] - 128, mult = a.mult[plane] - 128;
  const int offs0 = a.offset[plane] - 256;
  for (int y = y0; y < yend; y++) {
    const uint32_t s4 = *word(sp, y, x);
    if (y >= yclip) {
      *word(dp, y, x) = s4;
      continue;
    }
    const int yi = y - (row << bhl);
    // The co-located luma of the four chroma samples: 8 bytes (4:2:x) or 4,
    // the second word only when a column it serves is inside the crop.
    uint32_t l0 = 0, l1 = 0;
    if (plane != 0) {
      l0 = *word(lp, y << sy, x << sx);
      if (sx && x + 2 < sp.w) l1 = *word(lp, y << sy, (x << sx) + 4);
    }
    const int16_t* g00 = gr + (r00 + yi) * kGW + c00;
    uint32_t out = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const int s = (s4 >> (8 * k)) & 0xff;
      int o = s;
      if (x + k < sp.w) {
        const bool lk = xi + k < xStart;
        const int hpw = sx ? 23 : (xi + k == 1 ? 17 : 27), hcw = sx ? 22 : (xi + k == 1 ? 27 : 17);
        int g = g00[k];
        if (lk) g = blend_w(gr[(r10 + yi) * kGW + c10 + k], g, hpw, hcw, 8);
        if (yi < yStart) {
          int top = gr[(r01 + yi) * kGW + c01 + k];
          if (lk) top = blend_w(gr[(r11 + yi) * kGW + c11 + k], top, hpw, hcw, 8);
          const int vpw = sy ? 23 : (yi == 1 ? 17 : 27), vcw = sy ? 22 : (yi == 1 ? 27 : 17);
          g = blend_w(top, g, vpw, vcw, 8);
        }
        int idx;
        if (plane == 0) {
          idx = s;
        } else {
          // chromaScalingIndex (apply.go:501-520) on the un-grained luma.
          int avg;
          if (sx) {
            const uint32_t lw = k < 2 ? l0 : l1;
            const int b0 = (lw >> (16 * (k & 1))) & 0xff, b1 = (lw >> (16 * (k & 1) + 8)) & 0xff;
            avg = (oddLuma && x + k == sp.w - 1) ? b0 : (b0 + b1 + 1) >> 1;
          } else {
            avg = (l0 >> (8 * k)) & 0xff;
          }
          idx = cfl ? avg : iclip(((avg * lumaMult + s * mult) >> 6) + offs0, 0, 255);
        }
        const int noise = rpow2(lut[idx] * g, shift);
        o = iclip(s + noise, minV, maxV);
      }
      out |= (uint32_t)o << (8 * k);
    }
    *word(dp, y, x) = out;
  }
}

// frame/buffer.go:339-400: replicate the last visible column into the padding
// columns of every visible row, then the last visible row into padding rows.
template <typename T>
__device__ __forceinline__ void extend_px(const DFrame& f, int plane, int x, int y) {
  const DPlane& p = f.pl[plane];
  if (x >= p.aw || y >= p.ah) return;
  if (x < p.w && y < p.h) return;
  const int h = imin(p.h, p.ah);
  row_ptr<T>(p, y)[x] = row_ptr<T>(p, imin(y, h - 1))[imin(x, p.w - 1)];
}

// ---- batched kernels ----

__global__ void __launch_bounds__(kFgTemplateThreads) k_fg_templates_batch(BatchArgs b) {
  extern __shared__ __align__(16) unsigned char s_tpl[];
  TplSmem& S = *reinterpret_cast<TplSmem*>(s_tpl);
  const int* base = b.base + ST_FG_TEMPLATES * (b.n + 1);
  for_each_item(b, ST_FG_TEMPLATES, [&](int item) {
    const FrameJob& J = b.jobs[find_frame(base, b.n, item)];
    fg_templates(J.fgt, J.fg.grain[0], J.fg.grain[1], J.fg.grain[2], S);
  });
}

__global__ void __launch_bounds__(64) k_fg_offsets_batch(BatchArgs b) {
  const int* base = b.base + ST_FG_OFFSETS * (b.n + 1);
  for_each_item(b, ST_FG_OFFSETS, [&](int item) {
    const int fi = find_frame(base, b.n, item);
    const FrameJob& J = b.jobs[fi];
    const int r = (item - base[fi]) * 64 + threadIdx.x;
    if (r < J.fg.off_rows) fg_offsets_row(J.fgt.seed, r, J.fg.off_cols, const_cast<uint8_t*>(J.fg.offsets));
  });
}

// Display frame: 64x64-sample tiles of each plane, 256 threads x 16 rows (a
// thread's rows stay inside one grain block: blocks are 32 or 16 rows high,
// and a thread's per-column set-up is spread over 16 samples).
// The plane's scaling table is staged in shared memory per tile.
struct FgTile {
  const FrameJob* J;
  int plane, tx, ty;
};

__device__ __forceinline__ FgTile fg_locate(const BatchArgs& b, const int* base, int item) {
  const int fi = find_frame(base, b.n, item);
  const FrameJob& J = b.jobs[fi];
  int local = item - base[fi];
  int plane = 0;
  while (plane < 2 && local >= J.fg_tx[plane] * J.fg_ty[plane]) {
    local -= J.fg_tx[plane] * J.fg_ty[plane];
    plane++;
  }
  return FgTile{&J, plane, local % J.fg_tx[plane], local / J.fg_tx[plane]};
}

// kGroup rows per load group (fg_apply_col); one row at a time keeps 40
// registers (6 CTAs per SM), groups of 2 or 4 need 64 (4 CTAs per SM).
// kGroup 0: four columns by four rows a thread (fg_apply_quad, 8-bit).
template <bool kLoop, int kGroup>
__global__ void __launch_bounds__(256, kGroup == 1 ? 6 : 4) k_fg_apply_batch(BatchArgs b) {
  __shared__ uint8_t s_lut[256];
  const int* base = b.base + ST_FG_APPLY * (b.n + 1);
  for_each_item<kLoop>(
      b, ST_FG_APPLY,
      [&](int item) {
        const FgTile t = fg_locate(b, base, item);
        const FrameJob& J = *t.J;
        s_lut[threadIdx.x] = J.fg.lut[t.plane][threadIdx.x];
        __syncthreads();
        if constexpr (kGroup == 0) {
          // Four columns by four rows a thread.
          const int x = t.tx * 64 + (threadIdx.x & 15) * 4;
          const int y0 = t.ty * 64 + (threadIdx.x >> 4) * 4;
          if (J.io.bd == 8) {
            fg_apply_quad(J.io, J.disp, J.fg, s_lut, t.plane, x, y0, 4);
          } else {
#pragma unroll
            for (int k = 0; k < 4; k++) fg_apply_col<uint16_t, 1>(J.io, J.disp, J.fg, s_lut, t.plane, x + k, y0, 4);
          }
        } else {
          const int x = t.tx * 64 + (threadIdx.x & 63);
          const int y0 = t.ty * 64 + (threadIdx.x >> 6) * 16;
          if (J.io.bd == 8)
            fg_apply_col<uint8_t, kGroup>(J.io, J.disp, J.fg, s_lut, t.plane, x, y0, 16);
          else
            fg_apply_col<uint16_t, kGroup>(J.io, J.disp, J.fg, s_lut, t.plane, x, y0, 16);
        }
        __syncthreads();  // the table is rewritten by the next tile
      },
      [&](int item) {
        // The tile of the filtered frame (the grain's input).
        const FgTile t = fg_locate(b, base, item);
        const FrameJob& J = *t.J;
        const int x0 = t.tx * 64, y0 = t.ty * 64;
        if (J.io.bd == 8)
          prefetch_block<uint8_t>(J.io.pl[t.plane], x0, x0 + 64, y0, y0 + 64);
        else
          prefetch_block<uint16_t>(J.io.pl[t.plane], x0, x0 + 64, y0, y0 + 64);
      });
}

// Border extension: 64x4-sample tiles of the right strip [w, aw) x [0, h)
// then of the bottom strip [0, aw) x [h, ah), per plane.
__global__ void __launch_bounds__(256) k_extend_batch(BatchArgs b) {
  const int* base = b.base + ST_EXTEND * (b.n + 1);
  for_each_item(b, ST_EXTEND, [&](int item) {
    const int fi = find_frame(base, b.n, item);
    const FrameJob& J = b.jobs[fi];
    int local = item - base[fi];
    for (int plane = 0; plane < 3; plane++) {
      const int nr = J.ext_r[plane][0] * J.ext_r[plane][1], nb = J.ext_b[plane][0] * J.ext_b[plane][1];
      if (local >= nr + nb) {
        local -= nr + nb;
        continue;
      }
      const DPlane& p = J.io.pl[plane];
      int x, y;
      if (local < nr) {
        x = p.w + (local % J.ext_r[plane][0]) * 64 + (threadIdx.x & 63);
        y = (local / J.ext_r[plane][0]) * 4 + (threadIdx.x >> 6);
        if (y >= p.h) return;
      } else {
        local -= nr;
        x = (local % J.ext_b[plane][0]) * 64 + (threadIdx.x & 63);
        y = p.h + (local / J.ext_b[plane][0]) * 4 + (threadIdx.x >> 6);
      }
      if (J.io.bd == 8)
        extend_px<uint8_t>(J.io, plane, x, y);
      else
        extend_px<uint16_t>(J.io, plane, x, y);
      return;
    }
  });
}

// LFSR step as a GF(2)^16 map, for the host-side jump tables.
static uint16_t lfsr_step_host(uint16_t reg) {
  const uint16_t bit = ((reg >> 0) ^ (reg >> 1) ^ (reg >> 3) ^ (reg >> 12)) & 1;
  return (uint16_t)((reg >> 1) | (bit << 15));
}

cudaError_t fg_upload_tables() {
  static_assert(sizeof(pf_gaussian_sequence) == sizeof(g_gauss), "Gaussian sequence length");
  cudaError_t e = cudaMemcpyToSymbol(g_gauss, pf_gaussian_sequence, sizeof(pf_gaussian_sequence));
  if (e != cudaSuccess) return e;
  uint16_t jump[3][kFgTemplateThreads][16];
  int lens[3];
  const int samples[3] = {82 * 73, 44 * 73, 44 * 38};
  for (int t = 0; t < 3; t++) {
    const int L = (samples[t] + kFgTemplateThreads - 1) / kFgTemplateThreads;
    lens[t] = L;
    uint16_t cols[16];
    for (int c = 0; c < 16; c++) cols[c] = (uint16_t)(1u << c);
    for (int k = 0; k < kFgTemplateThreads; k++) {
      for (int c = 0; c < 16; c++) jump[t][k][c] = cols[c];
      for (int c = 0; c < 16; c++)
        for (int s = 0; s < L; s++) cols[c] = lfsr_step_host(cols[c]);
    }
  }
  e = cudaMemcpyToSymbol(g_jump, jump, sizeof(jump));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(g_jump_len, lens, sizeof(lens));
  return e;
}

cudaError_t launch_fg_templates_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  // The shared layout is above the default 48 KB: opt in once per device.
  constexpr int kMaxDevices = 64;
  static std::atomic<bool> configured[kMaxDevices];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!configured[dev].load(std::memory_order_acquire)) {
    e = cudaFuncSetAttribute(k_fg_templates_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(TplSmem));
    if (e != cudaSuccess) return e;
    configured[dev].store(true, std::memory_order_release);
  }
  k_fg_templates_batch<<<grid, kFgTemplateThreads, sizeof(TplSmem), st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_fg_offsets_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  k_fg_offsets_batch<<<grid, 64, 0, st>>>(b);
  return cudaGetLastError();
}

cudaError_t launch_fg_apply_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  const bool loop = batch_loops(b);
  static int w0 = 0, w1 = 0, w2 = 0, w4 = 0;
  switch (b.tile) {
    case 3:
      loop ? k_fg_apply_batch<true, 0><<<grid, 256, 0, st>>>(b)
           : k_fg_apply_batch<false, 0><<<grid, 256, 0, st>>>(with_wave(b, k_fg_apply_batch<false, 0>, 256, 0, w0));
      break;
    case 1:
      loop ? k_fg_apply_batch<true, 2><<<grid, 256, 0, st>>>(b)
           : k_fg_apply_batch<false, 2><<<grid, 256, 0, st>>>(with_wave(b, k_fg_apply_batch<false, 2>, 256, 0, w2));
      break;
    case 2:
      loop ? k_fg_apply_batch<true, 4><<<grid, 256, 0, st>>>(b)
           : k_fg_apply_batch<false, 4><<<grid, 256, 0, st>>>(with_wave(b, k_fg_apply_batch<false, 4>, 256, 0, w4));
      break;
    default:
      loop ? k_fg_apply_batch<true, 1><<<grid, 256, 0, st>>>(b)
           : k_fg_apply_batch<false, 1><<<grid, 256, 0, st>>>(with_wave(b, k_fg_apply_batch<false, 1>, 256, 0, w1));
  }
  return cudaGetLastError();
}

cudaError_t launch_extend_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  k_extend_batch<<<grid, 256, 0, st>>>(b);
  return cudaGetLastError();
}

}  // namespace pf
