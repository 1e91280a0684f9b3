// pf_lr.cu - loop restoration (Wiener / SGRproj) on the GPU.
//
// One CTA per (64-wide processing column, restoration stripe, plane).  The
// geometry is goav1's: tile/restoration_schedule.go:61-109, :400-409 (unit
// grid), tile/restoration_geometry.go:54-236 (unit rects shifted up by 8/4
// rows, stripes of 64/32 rows with the first one 8/4 rows shorter, 64-wide
// processing units).  Each stripe reads the post-CDEF plane with a 3-sample
// replicated frame border (restoration_boundary.go:126-180) and, across
// interior stripe boundaries, the pre-CDEF rows the CDEF kernel saved
// (setupRestorationStripeBoundaryFromSaved, restoration_boundary.go:553-614:
// rows above = saved[max(i+2,0)], rows below = saved[min(i,1)]).  The
// filters are restoration/wiener.go:59-211 and restoration/selfguided.go:
// 111-390 (box sums, a/b tables, 6/5 and 4/3 weights, projection with the
// int16 wrap).  Visible output columns depend only on +/-3 source columns,
// so the reference's rounding of the last Wiener unit width up to 16 changes
// no stored sample and is not replicated.
//
// Every sample of the tile inside the MI-aligned plane is written to the
// destination: restored samples where a Wiener/SGR unit covers the cropped
// plane, the post-CDEF sample everywhere else.
#include "pf_common.cuh"
#include "pf_tables.h"

namespace pf {

__constant__ int16_t c_sgr_params[16][4];
__constant__ uint16_t c_x_by_xplus1[256];
__constant__ uint16_t c_one_by_x[25];

constexpr int kWin = 70;  // 64 + 2*3

struct LrSmem {
  uint16_t win[kWin * kWin];
  int32_t flt0[64 * 64];     // SGR radius-2 filter output between the passes (Wiener: row-pass temp)
  uint16_t A[66 * 66];       // SGR a (<= 256)
  int32_t B[66 * 66];
  uint16_t x_by_xplus1[256];  // data-dependent lookup: smem, not constant memory
};

__device__ __forceinline__ int32_t rpot(int32_t v, int bits) {
  return bits <= 0 ? v : (v + (int32_t)(1 << (bits - 1))) >> bits;
}
__device__ __forceinline__ uint32_t rpotu(uint32_t v, int bits) {
  return bits <= 0 ? v : (v + (1u << (bits - 1))) >> bits;
}

// One restoration tile: processing column j of stripe s of `plane`.
template <typename T>
__device__ void lr_tile(const DFrame& src, const DFrame& dst, const LrArgs& a, const int* aw, const int* ah,
                        int enabled, int plane, int j, int s, LrSmem& sm) {
  uint16_t* s_win = sm.win;
  uint16_t* s_A = sm.A;
  int32_t* s_B = sm.B;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int ssx = plane ? src.ssx : 0, ssy = plane ? src.ssy : 0;
  const int PW = 64 >> ssx, SH = 64 >> ssy, off = 8 >> ssy;
  const int Wa = aw[plane], Ha = ah[plane];
  const DPlane& sp = src.pl[plane];
  const DPlane& dp = dst.pl[plane];
  const int Wc = sp.w, Hc = sp.h;
  const int x0 = j * PW;
  const int y0 = imax(0, s * SH - off);
  if (x0 >= Wa || y0 >= Ha) return;
  const int x1 = imin(x0 + PW, Wa), y1 = imin((s + 1) * SH - off, Ha);
  const int tid = threadIdx.x;
  const int tx = tid % PW, ty0 = tid / PW, rowStep = 256 / PW;
  const int bd = src.bd;

  // Which restoration unit (if any) covers this tile.
  const pf_lr_unit* u = nullptr;
  const int xf1 = imin(x1, Wc), yf1 = imin(y1, Hc);
  if (enabled && a.type[plane] != PF_LR_NONE && x0 < Wc && y0 < Hc) {
    const int us = a.unit_size[plane];
    const int ur = imin((y0 + off) / us, a.vert[plane] - 1);
    const int uc = imin(x0 / us, a.horz[plane] - 1);
    const pf_lr_unit* cand = &a.units[plane][ur * a.horz[plane] + uc];
    if (cand->type == PF_LR_WIENER || cand->type == PF_LR_SGRPROJ) u = cand;
  }
  if (!u) {
    if (tx < x1 - x0)
      for (int y = y0 + ty0; y < y1; y += rowStep) row_ptr<T>(dp, y)[x0 + tx] = row_ptr<T>(sp, y)[x0 + tx];
    return;
  }
  const int h = yf1 - y0, w = xf1 - x0;
  // ---- stage the (h+6) x (w+6) source window ----
  const int nominal = SH - (y0 == 0 ? off : 0);
  const bool copyAbove = y0 != 0, copyBelow = y0 + nominal < Hc;
  const int kAbove = s, kBelow = s + 1;  // boundary indices of the saved lines
  const int ww = w + 6, wh = h + 6;
  for (int r = warp; r < wh; r += 8) {
    const int yy = y0 - 3 + r;
    const T* srow;
    if (yy < y0 && copyAbove) {
      srow = reinterpret_cast<const T*>(a.lines[plane] + (int64_t)(kAbove * 4 + imax(yy - y0 + 2, 0)) * a.line_stride[plane]);
    } else if (yy >= yf1 && copyBelow) {
      srow = reinterpret_cast<const T*>(a.lines[plane] + (int64_t)(kBelow * 4 + 2 + imin(yy - yf1, 1)) * a.line_stride[plane]);
    } else {
      srow = row_ptr<T>(sp, iclip(yy, 0, Hc - 1));
    }
    for (int c = lane; c < ww; c += 32) s_win[r * kWin + c] = (uint16_t)srow[iclip(x0 - 3 + c, 0, Wc - 1)];
  }
  for (int i = tid; i < 256; i += 256) sm.x_by_xplus1[i] = c_x_by_xplus1[i];
  __syncthreads();

  // Pixels of the tile outside the cropped plane are copied through.
  if (tx < x1 - x0)
    for (int y = y0 + ty0; y < y1; y += rowStep)
      if (x0 + tx >= Wc || y >= Hc) row_ptr<T>(dp, y)[x0 + tx] = row_ptr<T>(sp, y)[x0 + tx];

  const int maxv = (1 << bd) - 1;
  if (u->type == PF_LR_WIENER) {
    // restoration/wiener.go:202-211 (wienerRounds), :132-196.
    int round0 = 3, round1 = 11;
    const int range = bd + 7 - round0 + 2;
    if (range > 16) {
      round0 += range - 16;
      round1 -= range - 16;
    }
    const int hv0 = u->wiener_h[0], hv1 = u->wiener_h[1], hv2 = u->wiener_h[2];
    const int hf[7] = {hv0, hv1, hv2, -2 * (hv0 + hv1 + hv2), hv2, hv1, hv0};
    const int vv0 = u->wiener_v[0], vv1 = u->wiener_v[1], vv2 = u->wiener_v[2];
    const int vf[7] = {vv0, vv1, vv2, -2 * (vv0 + vv1 + vv2), vv2, vv1, vv0};
    const int32_t limit = 1 << (bd + 1 + 7 - round0);
    const int32_t offH = 1 << (bd + 7 - 1);
    uint16_t* temp = reinterpret_cast<uint16_t*>(sm.flt0);  // (h+6) x 64
    for (int r = warp; r < wh; r += 8) {
      for (int c = lane; c < w; c += 32) {
        const uint16_t* sw = &s_win[r * kWin + c];
        int32_t sum = ((int32_t)sw[3] << 7) + offH;
#pragma unroll
        for (int k = 0; k < 7; k++) sum += (int32_t)sw[k] * hf[k];
        temp[r * 64 + c] = (uint16_t)imin(imax(rpot(sum, round0), 0), limit - 1);
      }
    }
    __syncthreads();
    const int32_t offV = 1 << (bd + round1 - 1);
    if (tx < w)
      for (int y = ty0; y < h; y += rowStep) {
        int32_t c3 = temp[(y + 3) * 64 + tx];
        int32_t sum = (c3 << 7) - offV;
#pragma unroll
        for (int k = 0; k < 7; k++) sum += (int32_t)temp[(y + k) * 64 + tx] * vf[k];
        row_ptr<T>(dp, y0 + y)[x0 + tx] = (T)imin(imax(rpot(sum, round1), 0), maxv);
      }
    return;
  }

  // ---- SGRproj (restoration/selfguided.go:132-359) ----
  const int set = u->sgr_set;
  const int r0 = c_sgr_params[set][0], r1 = c_sgr_params[set][1];
  // restoration/selfguided.go:111-127 (DecodeSGRXQ).
  int xq0, xq1;
  if (r0 == 0) {
    xq0 = 0;
    xq1 = 128 - u->sgr_xqd[1];
  } else if (r1 == 0) {
    xq0 = u->sgr_xqd[0];
    xq1 = 0;
  } else {
    xq0 = u->sgr_xqd[0];
    xq1 = 128 - xq0 - u->sgr_xqd[1];
  }
  int32_t* flt0 = sm.flt0;  // [y * 64 + x]
  if (r0 == 0)
    for (int y = warp; y < h; y += 8)
      for (int x = lane; x < w; x += 32) flt0[y * 64 + x] = 0;
  const int nrows = h + 2, ncols = w + 2;
  for (int pass = 0; pass < 2; pass++) {
    const int r = pass == 0 ? r0 : r1;
    if (r == 0) continue;
    const int sv = c_sgr_params[set][2 + pass];
    const uint32_t n = (uint32_t)((2 * r + 1) * (2 * r + 1));
    const int step = pass == 0 ? 2 : 1;  // the r = 2 pass computes rows -1, 1, 3, ...
    // a/b for rows -1..h and cols -1..w at [(row+1)*66 + col+1].  Box sums:
    // each lane slides a (2r+1)-row column sum down its window column; the
    // (2r+1)-wide row sum comes from the neighbouring lanes by shuffles, so
    // a warp yields 32-2r output columns per row.
    const int outPer = 32 - 2 * r;
    const int nch = (ncols + outPer - 1) / outPer;
    const int nseg = (nrows + 15) / 16;
    for (int item = warp; item < nch * nseg; item += 8) {
      const int q = item % nch, seg = item / nch;
      const int cc = q * outPer + lane - r;   // output column of this lane
      const int wc = cc + 2;                  // its window column (centre)
      const bool colIn = wc >= 0 && wc < ww;
      const int rs = seg * 16, re = imin(rs + 16, nrows);
      int rr = rs + (step == 2 ? (rs & 1) : 0);
      uint32_t vs = 0, vq = 0;
      if (colIn && rr < re)
        for (int dy = -r; dy <= r; dy++) {
          const uint32_t v = s_win[(rr + 2 + dy) * kWin + wc];
          vs += v;
          vq += v * v;
        }
      for (; rr < re; rr += step) {
        uint32_t bs = 0, bq = 0;
        for (int dx = -r; dx <= r; dx++) {
          bs += __shfl_sync(0xffffffffu, vs, imin(imax(lane + dx, 0), 31));
          bq += __shfl_sync(0xffffffffu, vq, imin(imax(lane + dx, 0), 31));
        }
        if (lane >= r && lane < 32 - r && cc < ncols) {
          const int32_t sum = (int32_t)bs, sq = (int32_t)bq;
          const uint32_t av = (uint32_t)rpot(sq, 2 * (bd - 8));
          const uint32_t bv = (uint32_t)rpot(sum, bd - 8);
          uint32_t p = 0;
          if (av * n >= bv * bv) p = av * n - bv * bv;
          uint32_t z = rpotu(p * (uint32_t)sv, 20);
          if (z > 255) z = 255;
          const int32_t A = sm.x_by_xplus1[z];
          s_A[rr * 66 + cc] = (uint16_t)A;
          s_B[rr * 66 + cc] = (int32_t)rpotu((uint32_t)(256 - A) * (uint32_t)sum * (uint32_t)c_one_by_x[n - 1], 12);
        }
        // Slide the column sums down to the next computed row.
        if (colIn && rr + step < re) {
          for (int k = 0; k < step; k++) {
            const uint32_t vin = s_win[(rr + 2 + r + 1 + k) * kWin + wc];
            const uint32_t vout = s_win[(rr + 2 - r + k) * kWin + wc];
            vs += vin - vout;
            vq += vin * vin - vout * vout;
          }
        }
      }
    }
    __syncthreads();
    if (tx < w) {
      for (int y = ty0; y < h; y += rowStep) {
        const uint16_t* A = &s_A[(y + 1) * 66 + tx + 1];
        const int32_t* B = &s_B[(y + 1) * 66 + tx + 1];
        const int32_t dg = s_win[(y + 3) * kWin + tx + 3];
        if (pass == 0) {
          int32_t av, bv, shift;
          if ((y & 1) == 0) {
            av = (A[-66] + A[66]) * 6 + (A[-67] + A[-65] + A[65] + A[67]) * 5;
            bv = (B[-66] + B[66]) * 6 + (B[-67] + B[-65] + B[65] + B[67]) * 5;
            shift = 9;
          } else {
            av = A[0] * 6 + (A[-1] + A[1]) * 5;
            bv = B[0] * 6 + (B[-1] + B[1]) * 5;
            shift = 8;
          }
          flt0[y * 64 + tx] = rpot(av * dg + bv, shift);
        } else {
          // restoration/selfguided.go:233-247: projection with the int16 wrap.
          const int32_t av = (A[0] + A[-1] + A[1] + A[-66] + A[66]) * 4 + (A[-67] + A[65] + A[-65] + A[67]) * 3;
          const int32_t bv = (B[0] + B[-1] + B[1] + B[-66] + B[66]) * 4 + (B[-67] + B[65] + B[-65] + B[67]) * 3;
          const int32_t f1 = rpot(av * dg + bv, 9);
          const int32_t uu = dg << 4;
          const int32_t v = (uu << 7) + xq0 * (flt0[y * 64 + tx] - uu) + xq1 * (f1 - uu);
          const int32_t wv = (int32_t)(int16_t)rpot(v, 11);
          row_ptr<T>(dp, y0 + y)[x0 + tx] = (T)imin(imax(wv, 0), maxv);
        }
      }
    }
    __syncthreads();
  }
  if (r1 == 0 && tx < w) {
    // Only the radius-2 filter: project with xq1 = 0.
    for (int y = ty0; y < h; y += rowStep) {
      const int32_t uu = (int32_t)s_win[(y + 3) * kWin + tx + 3] << 4;
      const int32_t v = (uu << 7) + xq0 * (flt0[y * 64 + tx] - uu);
      const int32_t wv = (int32_t)(int16_t)rpot(v, 11);
      row_ptr<T>(dp, y0 + y)[x0 + tx] = (T)imin(imax(wv, 0), maxv);
    }
  }
}

cudaError_t lr_upload_tables() {
  cudaError_t e = cudaMemcpyToSymbol(c_sgr_params, pf_sgr_params, sizeof(pf_sgr_params));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_x_by_xplus1, pf_sgr_x_by_xplus1, sizeof(pf_sgr_x_by_xplus1));
  if (e == cudaSuccess) e = cudaMemcpyToSymbol(c_one_by_x, pf_sgr_one_by_x, sizeof(pf_sgr_one_by_x));
  return e;
}

// Batched restoration: each work item is one (processing column, stripe)
// tile of one plane of one frame.  Frames without restoration get the copy
// of the CDEF output back into the frame.
__global__ void __launch_bounds__(256, 4) k_lr_batch(BatchArgs b) {
  extern __shared__ __align__(16) uint8_t lr_smem_raw[];
  LrSmem& sm = *reinterpret_cast<LrSmem*>(lr_smem_raw);
  const int* base = b.base + ST_LR * (b.n + 1);
  for_each_item(base[b.n], b.counters ? b.counters + ST_LR : nullptr, [&](int item) {
    const int fi = find_frame(base, b.n, item);
    const FrameJob& J = b.jobs[fi];
    int local = item - base[fi];
    int plane = 0;
    while (plane < 2 && local >= J.lr_cols[plane] * J.lr_rows[plane]) {
      local -= J.lr_cols[plane] * J.lr_rows[plane];
      plane++;
    }
    const int j = local % J.lr_cols[plane], s = local / J.lr_cols[plane];
    if (J.io.bd == 8)
      lr_tile<uint8_t>(J.scr, J.io, J.lr, J.aw, J.ah, J.do_lr, plane, j, s, sm);
    else
      lr_tile<uint16_t>(J.scr, J.io, J.lr, J.aw, J.ah, J.do_lr, plane, j, s, sm);
  });
}

cudaError_t launch_lr_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_lr_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LrSmem));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  k_lr_batch<<<grid, 256, sizeof(LrSmem), st>>>(b);
  return cudaGetLastError();
}

}  // namespace pf
