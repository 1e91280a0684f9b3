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
// The Gaussian fill is split over 32 lanes: the LFSR is linear over
// GF(2)^16, so lane k starts from M^(kL) * seed (jump matrices precomputed on
// the host) and walks its L draws; the AR filter runs as a wavefront over
// t = x + 4y (every AR input of sample (y, x) has a smaller t), one warp per
// template, rows in lanes, neighbours read from the shared template.  Offsets
// come from one thread per 32-row stripe.  The apply is one thread per output
// sample, 64x16-sample tiles per CTA.
#include "pf_common.cuh"
#include "pf_tables.h"

namespace pf {

__constant__ int16_t c_gauss[2048];

constexpr int kGW = 82, kGH = 73;

__device__ __forceinline__ int rpow2(int v, int bits) { return bits <= 0 ? v : (v + (1 << (bits - 1))) >> bits; }

__device__ __forceinline__ uint16_t lfsr(uint16_t& reg, int bits) {
  const uint16_t bit = ((reg >> 0) ^ (reg >> 1) ^ (reg >> 3) ^ (reg >> 12)) & 1;
  reg = (uint16_t)((reg >> 1) | (bit << 15));
  return (uint16_t)((reg >> (16 - bits)) & ((1 << bits) - 1));
}

// AR recursion of one template (luma.go:83-158 / chroma.go:92-199 generic
// form), run by one warp as a wavefront with no CTA barrier.  The template's
// AR rows are taken in bands of up to 32 rows, one row per lane; at step t
// lane r (row y) handles column x = t - 4r, so every sample of the rows
// above that its output needs (columns up to x + LAG <= x + 3) was written
// to the shared template by lanes r-1.. at an earlier step, and the warp
// barrier that ends each step makes it visible.  The filter runs in
// transposed form: when the value of row y-d at column x + LAG arrives, its
// products go straight into the partial sums of the outputs x .. x + 2*LAG
// it reaches, and the lane's own output adds its in-row products to the
// next LAG outputs' sums; the output then needs only its own sum, so the
// loop-carried path is load -> one multiply-add -> round -> clip -> store.
// The 2*LAG+1 partial sums rotate through acc[] with the step (the steps
// run in groups of 2*LAG+1, slot (j + k) mod (2*LAG+1) holding output x + j
// at step k of a group), so moving to the next column renames registers
// instead of copying them.  A chroma template's luma term comes from lt[]
// (the averaged luma grain at each chroma position, filled before the
// recursion).  A lane outside the AR columns passes the template's value
// through unchanged, so the rows above always hold the template as it
// stands.  Bands run one after the other, each only as long as its own rows
// need.  LAG is a template argument (coefficients in registers, unrolled
// taps).
constexpr int kFgTemplateThreads = 96;

template <int LAG>
__device__ __forceinline__ void ar_warp(int16_t* g, const int16_t* lt, const FgTemplateArgs& p, int plane, int w, int h) {
  constexpr int kTaps = 2 * LAG * (LAG + 1);  // causal neighbours before the centre
  constexpr int W = 2 * LAG + 1;
  const int lane = threadIdx.x & 31;
  const int cs = p.coeff_shift, ro = 1 << (cs - 1);
  const int gmin = -(1 << (p.bd - 1)), gmax = (1 << (p.bd - 1)) - 1;
  int co[kTaps + 1];
#pragma unroll
  for (int i = 0; i <= kTaps; i++) co[i] = p.coeffs[plane][i];
  const int coL = lt ? co[kTaps] : 0;
  for (int y0 = 3; y0 < h; y0 += 32) {
    const int rows = imin(32, h - y0);
    const int y = y0 + lane;
    const bool row = lane < rows;
    int acc[W];
#pragma unroll
    for (int j = 0; j < W; j++) acc[j] = 0;
    // The first step brings column 0 of the rows above into the sums; the
    // last one finishes column w - 4 of the band's last row.
    const int tend = 4 * (rows - 1) + w - 3;
    for (int t0 = -LAG; t0 < tend; t0 += W) {
#pragma unroll
      for (int k = 0; k < W; k++) {
        const int t = t0 + k;
        if (t < tend) {
          const int x = t - 4 * lane;
          const int xn = x + LAG;  // the column entering the sums
          const bool inCol = row && x >= 0 && x < w;
          const int g0 = inCol ? g[y * kGW + x] : 0;
          if (row && xn >= 0 && xn < w) {
            // Farthest row first: the row directly above (written one step
            // ago when LAG = 3) enters this step's output last.
#pragma unroll
            for (int d = LAG; d >= 1; d--) {
              const int v = g[(y - d) * kGW + xn];
#pragma unroll
              for (int j = W - 1; j >= 0; j--) acc[(j + k) % W] += co[(LAG - d) * W + 2 * LAG - j] * v;
            }
          }
          int out = g0;
          if (inCol && x >= 3 && x < w - 3) {
            int sum = acc[k % W];
            if (lt) sum += lt[y * kGW + x] * coL;
            out = iclip(g0 + ((sum + ro) >> cs), gmin, gmax);
            g[y * kGW + x] = (int16_t)out;
          }
          // Output x's in-row products for columns x + 1 .. x + LAG; its
          // slot then serves column x + W.
#pragma unroll
          for (int m = 1; m <= LAG; m++) acc[(m + k) % W] += co[LAG * W + LAG - m] * out;
          acc[k % W] = 0;
        }
        __syncwarp();
      }
    }
  }
}

// Luma term of the chroma AR (chroma.go:92-199): at each chroma AR position
// the luma grain averaged over the co-located 1, 2 or 4 samples, into lt
// (same layout as the templates).  All threads of the CTA.
__device__ __forceinline__ void luma_term(int16_t* lt, const int16_t* luma, int sx, int sy, int w, int h) {
  const int aw = w - 6;
  for (int i = threadIdx.x; i < aw * (h - 3); i += blockDim.x) {
    const int y = 3 + i / aw, x = 3 + i % aw;
    const int lx = ((x - 3) << sx) + 3, ly = ((y - 3) << sy) + 3;
    int s = luma[ly * kGW + lx];
    if (sx) s += luma[ly * kGW + lx + 1];
    if (sy) {
      s += luma[(ly + 1) * kGW + lx];
      if (sx) s += luma[(ly + 1) * kGW + lx + 1];
    }
    lt[y * kGW + x] = (int16_t)rpow2(s, sx + sy);
  }
}

__device__ __forceinline__ void ar_warp_lag(int16_t* g, const int16_t* lt, const FgTemplateArgs& p, int plane, int w, int h) {
  switch (p.lag) {
    case 0: ar_warp<0>(g, lt, p, plane, w, h); break;
    case 1: ar_warp<1>(g, lt, p, plane, w, h); break;
    case 2: ar_warp<2>(g, lt, p, plane, w, h); break;
    default: ar_warp<3>(g, lt, p, plane, w, h); break;
  }
}

// Jump matrices: c_jump[t][k][c] = M^(k*L_t) e_c for the three template
// shapes (t = 0: 82x73, 1: 44x73, 2: 44x38), L_t = ceil(samples / 32).
__constant__ uint16_t c_jump[3][32][16];
__constant__ int c_jump_len[3];

__device__ __forceinline__ uint16_t gf2_apply(const uint16_t* cols, uint16_t v) {
  uint16_t r = 0;
#pragma unroll
  for (int c = 0; c < 16; c++)
    if ((v >> c) & 1) r ^= cols[c];
  return r;
}

// Gaussian fill of one template (luma.go:32-38 / chroma.go:38-44): draw i of
// the plane's LFSR goes to sample (i / w, i % w).  One warp.
__device__ __forceinline__ void gauss_fill(int16_t* g, const int16_t* gauss, uint16_t seed, int w, int h, int shape, int shift) {
  const int lane = threadIdx.x & 31;
  const int L = c_jump_len[shape];
  uint16_t reg = gf2_apply(c_jump[shape][lane], seed);
  const int n = w * h;
  int i = lane * L;
  const int iend = imin(i + L, n);
  int y = i / w, x = i - y * w;
  for (; i < iend; i++) {
    g[y * kGW + x] = (int16_t)rpow2(gauss[lfsr(reg, 11)], shift);
    if (++x == w) {
      x = 0;
      y++;
    }
  }
}

// One frame's templates: Gaussian fills by warps 0-2 (luma, Cb, Cr), then the
// AR recursions (luma on warp 0, then Cb and Cr side by side).  s_gl holds
// the Gaussian sequence while the templates are filled (lanes draw
// different entries, which constant memory would serialise), then the
// chroma AR's luma term.
__device__ __forceinline__ void fg_templates(const FgTemplateArgs& p, int16_t* gy, int16_t* gu, int16_t* gv, int16_t (*s_g)[kGW * kGH],
                             int16_t* s_gl) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int16_t* outs[3] = {gy, gu, gv};
  const int cw = p.ssx ? 44 : kGW, ch = p.ssy ? 38 : kGH;
  const int cshape = p.ssx ? (p.ssy ? 2 : 1) : 0;
  const int16_t* s_gauss = s_gl;
  for (int i = threadIdx.x; i < 2048; i += blockDim.x) s_gl[i] = c_gauss[i];
  __syncthreads();
  if (warp < 3) {
    int16_t* g = s_g[warp];
    for (int i = lane; i < kGW * kGH; i += 32) g[i] = 0;
    __syncwarp();
    const bool active = warp == 0 ? p.num_y_points != 0 : p.active[warp];
    const int shift = 12 - p.bd + p.grain_scale_shift;
    if (active) {
      if (warp == 0)
        gauss_fill(g, s_gauss, p.seed, kGW, kGH, 0, shift);
      else
        gauss_fill(g, s_gauss, (uint16_t)(p.seed ^ (warp == 1 ? 0xb524 : 0x49d8)), cw, ch, cshape, shift);
    }
    __syncwarp();
  }
  __syncthreads();
  // Luma on warp 0; then Cb and Cr side by side on warps 1 and 2 (their
  // luma term reads the finished luma template).
  if (warp == 0 && p.num_y_points != 0 && p.lag != 0) ar_warp_lag(s_g[0], nullptr, p, 0, kGW, kGH);
  __syncthreads();
  const bool lumaTerm = p.num_y_points != 0;
  if (lumaTerm) {
    luma_term(s_gl, s_g[0], p.ssx, p.ssy, cw, ch);
    __syncthreads();
  }
  const bool runC = warp >= 1 && warp <= 2 && p.active[warp] && !(p.lag == 0 && p.num_y_points == 0);
  if (runC) ar_warp_lag(s_g[warp], lumaTerm ? s_gl : nullptr, p, warp, cw, ch);
  __syncthreads();
  for (int pl = 0; pl < 3; pl++)
    if (outs[pl])
      for (int i = threadIdx.x; i < kGW * kGH; i += blockDim.x) outs[pl][i] = s_g[pl][i];
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
  __shared__ int16_t s_g[3][kGW * kGH];
  __shared__ int16_t s_gl[kGW * kGH];  // Gaussian sequence, then the luma term
  const int* base = b.base + ST_FG_TEMPLATES * (b.n + 1);
  for_each_item(b, ST_FG_TEMPLATES, [&](int item) {
    const FrameJob& J = b.jobs[find_frame(base, b.n, item)];
    fg_templates(J.fgt, J.fg.grain[0], J.fg.grain[1], J.fg.grain[2], s_g, s_gl);
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
  cudaError_t e = cudaMemcpyToSymbol(c_gauss, pf_gaussian_sequence, sizeof(pf_gaussian_sequence));
  if (e != cudaSuccess) return e;
  uint16_t jump[3][32][16];
  int lens[3];
  const int samples[3] = {82 * 73, 44 * 73, 44 * 38};
  for (int t = 0; t < 3; t++) {
    const int L = (samples[t] + 31) / 32;
    lens[t] = L;
    uint16_t cols[16];
    for (int c = 0; c < 16; c++) cols[c] = (uint16_t)(1u << c);
    for (int k = 0; k < 32; k++) {
      for (int c = 0; c < 16; c++) jump[t][k][c] = cols[c];
      for (int c = 0; c < 16; c++)
        for (int s = 0; s < L; s++) cols[c] = lfsr_step_host(cols[c]);
    }
  }
  e = cudaMemcpyToSymbol(c_jump, jump, sizeof(jump));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_jump_len, lens, sizeof(lens));
  return e;
}

cudaError_t launch_fg_templates_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  k_fg_templates_batch<<<grid, kFgTemplateThreads, 0, st>>>(b);
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
