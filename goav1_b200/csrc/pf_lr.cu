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
constexpr int kLrMaxRun = 16;  // rows of one thread's output run (see lr_wiener_window)

struct LrSmem {
  uint16_t win[kWin * kWin];
  union {
    // SGR a (<= 256) / b tables: radius 1 for rows -1..h, radius 2 for the
    // rows -1, 1, 3, ... it is computed on; columns -1..w.
    struct {
      uint16_t A1[66 * 66];
      int32_t B1[66 * 66];
      uint16_t A2[33 * 66];
      int32_t B2[33 * 66];
    } sgr;
    uint16_t wtemp[kWin * 64];  // Wiener row-pass output, (h+6) x 64
  };
  uint16_t x_by_xplus1[256];  // data-dependent lookup: smem, not constant memory
};

__device__ __forceinline__ int32_t rpot(int32_t v, int bits) {
  return bits <= 0 ? v : (v + (int32_t)(1 << (bits - 1))) >> bits;
}
__device__ __forceinline__ uint32_t rpotu(uint32_t v, int bits) {
  return bits <= 0 ? v : (v + (1u << (bits - 1))) >> bits;
}

// Wiener filter of the staged window (restoration/wiener.go:132-211): the
// block's sample (0,0) sits at sm.win[3 * kWin + 3], w x h <= 64 x 64, with
// the 3-sample halo around it.  hf/vf are the 7 horizontal / vertical taps.
// out(y, x, v) receives every output sample; thread tid produces column
// x = tid % PW over a run of consecutive rows (the h rows split into 256 / PW
// runs).  Every thread of the CTA calls it; it leaves the window untouched
// and ends without a barrier.
template <class Out>
__device__ __forceinline__ void lr_wiener_window(LrSmem& sm, int w, int h, int bd, const int* hf, const int* vf, int PW,
                                 Out&& out) {
  const uint16_t* s_win = sm.win;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tid = threadIdx.x, tx = tid % PW, ty0 = tid / PW, rpg = (h + 256 / PW - 1) / (256 / PW);
  const int wh = h + 6;
  const int maxv = (1 << bd) - 1;
  // restoration/wiener.go:202-211 (wienerRounds), :132-196.
  int round0 = 3, round1 = 11;
  const int range = bd + 7 - round0 + 2;
  if (range > 16) {
    round0 += range - 16;
    round1 -= range - 16;
  }
  const int32_t limit = 1 << (bd + 1 + 7 - round0);
  const int32_t offH = 1 << (bd + 7 - 1);
  uint16_t* temp = sm.wtemp;  // (h+6) x 64
  // Row pass: a lane takes the column pair (2 lane, 2 lane + 1) of a row,
  // its eight window samples read as four aligned 32-bit words (kWin and
  // the column are even); the taps are symmetric (hf[k] == hf[6 - k]), so
  // the mirrored samples are summed first.
  const int hc = hf[3] + 128;
  for (int r = warp; r < wh; r += 8) {
    const int c = 2 * lane;
    if (c < w) {
      const uint32_t* sw = reinterpret_cast<const uint32_t*>(&s_win[r * kWin + c]);
      const uint32_t p01 = sw[0], p23 = sw[1], p45 = sw[2], p67 = sw[3];
      const int32_t v0 = p01 & 0xffff, v1 = p01 >> 16, v2 = p23 & 0xffff, v3 = p23 >> 16;
      const int32_t v4 = p45 & 0xffff, v5 = p45 >> 16, v6 = p67 & 0xffff, v7 = p67 >> 16;
      const int32_t s0 = offH + v3 * hc + (v0 + v6) * hf[0] + (v1 + v5) * hf[1] + (v2 + v4) * hf[2];
      const int32_t s1 = offH + v4 * hc + (v1 + v7) * hf[0] + (v2 + v6) * hf[1] + (v3 + v5) * hf[2];
      const uint32_t o0 = (uint32_t)imin(imax(rpot(s0, round0), 0), limit - 1);
      const uint32_t o1 = (uint32_t)imin(imax(rpot(s1, round0), 0), limit - 1);
      *reinterpret_cast<uint32_t*>(&temp[r * 64 + c]) = o0 | (o1 << 16);
    }
  }
  __syncthreads();
  const int32_t offV = 1 << (bd + round1 - 1);
  // Each thread a run of consecutive output rows of column tx: the seven
  // vertical taps slide down in registers, one new row read per output.  A
  // run is at most kLrMaxRun rows (h <= 64 over 4 runs per column at PW 64,
  // over 8 at PW 32), and the loop is unrolled to that bound so that the
  // slide is register renaming.
  const int ya = ty0 * rpg, yb = imin(h, ya + rpg);
  if (tx < w && ya < yb) {
    int32_t t[7];
#pragma unroll
    for (int k = 0; k < 6; k++) t[k] = temp[(ya + k) * 64 + tx];
#pragma unroll
    for (int i = 0; i < kLrMaxRun; i++) {
      const int y = ya + i;
      if (y >= yb) break;
      t[6] = temp[(y + 6) * 64 + tx];
      int32_t sum = (t[3] << 7) - offV + t[3] * vf[3];
#pragma unroll
      for (int k = 0; k < 3; k++) sum += (t[k] + t[6 - k]) * vf[k];
      out(y, tx, imin(imax(rpot(sum, round1), 0), maxv));
#pragma unroll
      for (int k = 0; k < 6; k++) t[k] = t[k + 1];
    }
  }
}

// a and b of one SGR box (restoration/selfguided.go:132-231): the box's sum
// and sum of squares, area N (9 or 25), strength sv.
template <int N>
__device__ __forceinline__ void sgr_ab(uint32_t bs, uint32_t bq, int bd, int sv, const uint16_t* xbx, uint16_t* A,
                                       int32_t* B) {
  const int32_t sum = (int32_t)bs, sq = (int32_t)bq;
  const uint32_t av = (uint32_t)rpot(sq, 2 * (bd - 8));
  const uint32_t bv = (uint32_t)rpot(sum, bd - 8);
  uint32_t p = 0;
  if (av * N >= bv * bv) p = av * N - bv * bv;
  uint32_t z = rpotu(p * (uint32_t)sv, 20);
  if (z > 255) z = 255;
  const int32_t a = xbx[z];
  *A = (uint16_t)a;
  *B = (int32_t)rpotu((uint32_t)(256 - a) * (uint32_t)sum * (uint32_t)c_one_by_x[N - 1], 12);
}

// Self-guided filter of the staged window (restoration/selfguided.go:111-390)
// for a parameter set whose radius-2 (R2) and radius-1 (R1) filters are on
// or off, with the decoded projection weights xq0 / xq1; same window,
// thread mapping and out() contract as lr_wiener_window.  sm.x_by_xplus1
// must hold the table.  Ends with a barrier.
//
// Box sums: one sweep down the window for both radii.  A warp takes a chunk
// of 32 - 2*halo box columns and a segment of box rows; each lane slides the
// 3-row and 5-row column sums of its window column down the segment (two
// window loads a row: the rows entering the 5-row sum and leaving the 3-row
// one; the other two moves reuse the previous row's), and the row sums come
// from the neighbouring lanes by shuffles.  Radius 1 has a box on every row,
// radius 2 on the rows -1, 1, 3, ....  Filters: one pass, each thread a run
// of rows of one column, the a/b neighbourhoods of both radii sliding down
// in registers, projected straight to out().
template <bool R2, bool R1, class Out>
__device__ __forceinline__ void lr_sgr_window_t(LrSmem& sm, int w, int h, int bd, int s2, int s1, int xq0, int xq1,
                                                int PW, Out&& out) {
  const uint16_t* s_win = sm.win;
  uint16_t* A1 = sm.sgr.A1;
  int32_t* B1 = sm.sgr.B1;
  uint16_t* A2 = sm.sgr.A2;
  int32_t* B2 = sm.sgr.B2;
  const uint16_t* xbx = sm.x_by_xplus1;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int tid = threadIdx.x, tx = tid % PW, ty0 = tid / PW, rpg = (h + 256 / PW - 1) / (256 / PW);
  const int ya = ty0 * rpg, yb = imin(h, ya + rpg);
  const int ww = w + 6;
  const int maxv = (1 << bd) - 1;
  constexpr int kHalo = R2 ? 2 : 1;
  constexpr int kOutPer = 32 - 2 * kHalo;
  constexpr unsigned kAll = 0xffffffffu;
  const int nrows = h + 2, ncols = w + 2;
  const int nch = (ncols + kOutPer - 1) / kOutPer;
  const int segLen = (nrows + 7) >> 3;  // 8 row segments per column chunk
  for (int item = warp; item < nch * 8; item += 8) {
    const int seg = item / nch, q = item - seg * nch;
    const int cc = q * kOutPer + lane - kHalo;  // box column + 1 of this lane
    const int wc = cc + 2;                      // its window column
    const bool colIn = wc >= 0 && wc < ww;
    const bool store = lane >= kHalo && lane < 32 - kHalo && cc < ncols;
    const int rs = seg * segLen, re = imin(rs + segLen, nrows);
    if (rs >= re) continue;
    auto ld = [&](int r) -> uint32_t { return colIn ? (uint32_t)s_win[r * kWin + wc] : 0u; };
    // Box row rr (= row + 1) covers window rows rr+1 .. rr+3 (radius 1) and
    // rr .. rr+4 (radius 2).
    const uint32_t v0 = ld(rs), v1 = ld(rs + 1), v2 = ld(rs + 2), v3 = ld(rs + 3), v4 = ld(rs + 4);
    uint32_t c3s = v1 + v2 + v3, c3q = v1 * v1 + v2 * v2 + v3 * v3;
    uint32_t c5s = c3s + v0 + v4, c5q = c3q + v0 * v0 + v4 * v4;
    uint32_t enter3 = v4, leave5 = v0;  // window rows rr+4 (enters the 3-row sum) and rr (leaves the 5-row one)
    for (int rr = rs; rr < re; rr++) {
      if (R1) {
        const uint32_t bs = c3s + __shfl_up_sync(kAll, c3s, 1) + __shfl_down_sync(kAll, c3s, 1);
        const uint32_t bq = c3q + __shfl_up_sync(kAll, c3q, 1) + __shfl_down_sync(kAll, c3q, 1);
        if (store) sgr_ab<9>(bs, bq, bd, s1, xbx, &A1[rr * 66 + cc], &B1[rr * 66 + cc]);
      }
      if (R2 && (rr & 1) == 0) {
        const uint32_t bs = c5s + __shfl_up_sync(kAll, c5s, 1) + __shfl_down_sync(kAll, c5s, 1) +
                            __shfl_up_sync(kAll, c5s, 2) + __shfl_down_sync(kAll, c5s, 2);
        const uint32_t bq = c5q + __shfl_up_sync(kAll, c5q, 1) + __shfl_down_sync(kAll, c5q, 1) +
                            __shfl_up_sync(kAll, c5q, 2) + __shfl_down_sync(kAll, c5q, 2);
        if (store) sgr_ab<25>(bs, bq, bd, s2, xbx, &A2[(rr >> 1) * 66 + cc], &B2[(rr >> 1) * 66 + cc]);
      }
      if (rr + 1 < re) {
        const uint32_t l3 = ld(rr + 1);
        if (R1) {
          c3s += enter3 - l3;
          c3q += enter3 * enter3 - l3 * l3;
        }
        if (R2) {
          const uint32_t e5 = ld(rr + 5);
          c5s += e5 - leave5;
          c5q += e5 * e5 - leave5 * leave5;
          enter3 = e5;
        } else {
          enter3 = ld(rr + 4 + 1);
        }
        leave5 = l3;
      }
    }
  }
  __syncthreads();
  if (tx < w && ya < yb) {
    // Radius 2: even y weighs table rows y and y + 2 (6 centre / 5 corners,
    // shift 9), odd y row y + 1 (6 / 5, shift 8); the tables hold the even
    // rows k at k / 2.  Radius 1: rows y, y + 1, y + 2 (4 cross / 3
    // corners).  A table row enters as its 3-sum S and centre C over columns
    // tx .. tx + 2: 6 C + 5 (S - C) = 5 S + C, and the radius-1 weights sum
    // to 4 S(y+1) + 3 (S(y) + S(y+2)) + C(y) + C(y+2).
    struct SC {
      int32_t sa, ca, sb, cb;
    };
    auto row2 = [&](int i) {
      const int o = i * 66 + tx;
      const int32_t a0 = A2[o], a1 = A2[o + 1], a2 = A2[o + 2];
      const int32_t b0 = B2[o], b1 = B2[o + 1], b2 = B2[o + 2];
      return SC{a0 + a1 + a2, a1, b0 + b1 + b2, b1};
    };
    auto row1 = [&](int k) {
      const int o = k * 66 + tx;
      const int32_t a0 = A1[o], a1 = A1[o + 1], a2 = A1[o + 2];
      const int32_t b0 = B1[o], b1 = B1[o + 1], b2 = B1[o + 2];
      return SC{a0 + a1 + a2, a1, b0 + b1 + b2, b1};
    };
    // For y = ya: the pair (ya / 2, ya / 2 + 1) when ya is even, the one
    // row (ya + 1) / 2 in d2 when it is odd.
    SC u2{}, d2{}, u1{}, m1{};
    if (R2) {
      u2 = row2(ya >> 1);
      d2 = row2((ya >> 1) + 1);
    }
    if (R1) {
      u1 = row1(ya);
      m1 = row1(ya + 1);
    }
#pragma unroll
    for (int i = 0; i < kLrMaxRun; i++) {
      const int y = ya + i;
      if (y >= yb) break;
      const int32_t dg = s_win[(y + 3) * kWin + tx + 3];
      const int32_t uu = dg << 4;
      int32_t v = uu << 7;
      if (R2) {
        int32_t av, bv, shift;
        if ((y & 1) == 0) {
          if (i != 0) {
            u2 = d2;
            d2 = row2((y >> 1) + 1);
          }
          av = 5 * (u2.sa + d2.sa) + u2.ca + d2.ca;
          bv = 5 * (u2.sb + d2.sb) + u2.cb + d2.cb;
          shift = 9;
        } else {
          av = 5 * d2.sa + d2.ca;
          bv = 5 * d2.sb + d2.cb;
          shift = 8;
        }
        v += xq0 * (rpot(av * dg + bv, shift) - uu);
      }
      if (R1) {
        const SC d1 = row1(y + 2);
        const int32_t av = 4 * m1.sa + 3 * (u1.sa + d1.sa) + u1.ca + d1.ca;
        const int32_t bv = 4 * m1.sb + 3 * (u1.sb + d1.sb) + u1.cb + d1.cb;
        v += xq1 * (rpot(av * dg + bv, 9) - uu);
        u1 = m1;
        m1 = d1;
      }
      // restoration/selfguided.go:233-247: projection with the int16 wrap.
      const int32_t wv = (int32_t)(int16_t)rpot(v, 11);
      out(y, tx, imin(imax(wv, 0), maxv));
    }
  }
  __syncthreads();
}

// The self-guided filter with parameter set `set` and the coded xqd pair
// (restoration/selfguided.go:111-127, DecodeSGRXQ), dispatched on which of
// its two radii are on (r0 is 0 or 2, r1 is 0 or 1).
template <class Out>
__device__ __forceinline__ void lr_sgr_window(LrSmem& sm, int w, int h, int bd, int set, int xqd0, int xqd1, int PW,
                                              Out&& out) {
  const int r0 = c_sgr_params[set][0], r1 = c_sgr_params[set][1];
  const int s0 = c_sgr_params[set][2], s1 = c_sgr_params[set][3];
  if (r0 == 0)
    lr_sgr_window_t<false, true>(sm, w, h, bd, s0, s1, 0, 128 - xqd1, PW, out);
  else if (r1 == 0)
    lr_sgr_window_t<true, false>(sm, w, h, bd, s0, s1, xqd0, 0, PW, out);
  else
    lr_sgr_window_t<true, true>(sm, w, h, bd, s0, s1, xqd0, 128 - xqd0 - xqd1, PW, out);
}

// One restoration tile: processing column j of stripe s of `plane`.
template <typename T>
__device__ void lr_tile(const DFrame& src, const DFrame& dst, const LrArgs& a, const int* aw, const int* ah,
                        int enabled, int plane, int j, int s, LrSmem& sm) {
  uint16_t* s_win = sm.win;
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
  const int bd = sizeof(T) == 1 ? 8 : src.bd;  // a constant for 8-bit: the rounding shifts fold

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
    copy_block<T>(sp, dp, x0, x1, y0, y1);
    return;
  }
  const int h = yf1 - y0, w = xf1 - x0;
  // ---- stage the (h+6) x (w+6) source window ----
  const int nominal = SH - (y0 == 0 ? off : 0);
  const bool copyAbove = y0 != 0, copyBelow = y0 + nominal < Hc;
  const int kAbove = s, kBelow = s + 1;  // boundary indices of the saved lines
  const int ww = w + 6, wh = h + 6;
  auto srcRow = [&](int r) -> const T* {
    const int yy = y0 - 3 + r;
    if (yy < y0 && copyAbove)
      return reinterpret_cast<const T*>(a.lines[plane] + (int64_t)(kAbove * 4 + imax(yy - y0 + 2, 0)) * a.line_stride[plane]);
    if (yy >= yf1 && copyBelow)
      return reinterpret_cast<const T*>(a.lines[plane] + (int64_t)(kBelow * 4 + 2 + imin(yy - yf1, 1)) * a.line_stride[plane]);
    return row_ptr<T>(sp, iclip(yy, 0, Hc - 1));
  };
  // A warp's rows r and r+8 and each lane's three columns are loaded before
  // any is stored: six loads in flight per lane (ww <= 70 < 96).
  for (int r0 = warp; r0 < wh; r0 += 16) {
    uint16_t v[2][3];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int r = r0 + 8 * q;
      if (r < wh) {
        const T* srow = srcRow(r);
#pragma unroll
        for (int k = 0; k < 3; k++) {
          const int c = lane + 32 * k;
          if (c < ww) v[q][k] = (uint16_t)srow[iclip(x0 - 3 + c, 0, Wc - 1)];
        }
      }
    }
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int k = 0; k < 3; k++)
        if (r0 + 8 * q < wh && lane + 32 * k < ww) s_win[(r0 + 8 * q) * kWin + lane + 32 * k] = v[q][k];
  }
  for (int i = tid; i < 256; i += 256) sm.x_by_xplus1[i] = c_x_by_xplus1[i];
  __syncthreads();

  // Pixels of the tile outside the cropped plane are copied through.
  if ((x1 > Wc || y1 > Hc) && tx < x1 - x0)
    for (int y = y0 + ty0; y < y1; y += rowStep)
      if (x0 + tx >= Wc || y >= Hc) row_ptr<T>(dp, y)[x0 + tx] = row_ptr<T>(sp, y)[x0 + tx];

  auto store = [&](int y, int x, int v) { row_ptr<T>(dp, y0 + y)[x0 + x] = (T)v; };
  if (u->type == PF_LR_WIENER) {
    const int hv0 = u->wiener_h[0], hv1 = u->wiener_h[1], hv2 = u->wiener_h[2];
    const int hf[7] = {hv0, hv1, hv2, -2 * (hv0 + hv1 + hv2), hv2, hv1, hv0};
    const int vv0 = u->wiener_v[0], vv1 = u->wiener_v[1], vv2 = u->wiener_v[2];
    const int vf[7] = {vv0, vv1, vv2, -2 * (vv0 + vv1 + vv2), vv2, vv1, vv0};
    lr_wiener_window(sm, w, h, bd, hf, vf, PW, store);
    return;
  }
  // ---- SGRproj (restoration/selfguided.go:132-359) ----
  lr_sgr_window(sm, w, h, bd, u->sgr_set, u->sgr_xqd[0], u->sgr_xqd[1], PW, store);
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
struct LrTile {
  const FrameJob* J;
  int plane, j, s;
};

__device__ __forceinline__ LrTile lr_locate(const BatchArgs& b, const int* base, int item) {
  const int fi = find_frame(base, b.n, item);
  const FrameJob& J = b.jobs[fi];
  int local = item - base[fi];
  int plane = 0;
  while (plane < 2 && local >= J.lr_cols[plane] * J.lr_rows[plane]) {
    local -= J.lr_cols[plane] * J.lr_rows[plane];
    plane++;
  }
  return LrTile{&J, plane, local % J.lr_cols[plane], local / J.lr_cols[plane]};
}

template <bool kLoop>
__global__ void __launch_bounds__(256, 4) k_lr_batch(BatchArgs b) {
  extern __shared__ __align__(16) uint8_t lr_smem_raw[];
  LrSmem& sm = *reinterpret_cast<LrSmem*>(lr_smem_raw);
  const int* base = b.base + ST_LR * (b.n + 1);
  for_each_item<kLoop>(
      b, ST_LR,
      [&](int item) {
        const LrTile t = lr_locate(b, base, item);
        const FrameJob& J = *t.J;
        if (J.io.bd == 8)
          lr_tile<uint8_t>(J.scr, J.io, J.lr, J.aw, J.ah, J.do_lr, t.plane, t.j, t.s, sm);
        else
          lr_tile<uint16_t>(J.scr, J.io, J.lr, J.aw, J.ah, J.do_lr, t.plane, t.j, t.s, sm);
      },
      [&](int item) {
        // The tile's stripe of the CDEF output with its 3-sample halo.
        const LrTile t = lr_locate(b, base, item);
        const FrameJob& J = *t.J;
        const int ssx = t.plane ? J.io.ssx : 0, ssy = t.plane ? J.io.ssy : 0;
        const int PW = 64 >> ssx, SH = 64 >> ssy, off = 8 >> ssy;
        const int x0 = t.j * PW, y0 = t.s * SH - off;
        if (J.io.bd == 8)
          prefetch_block<uint8_t>(J.scr.pl[t.plane], x0 - 3, x0 + PW + 3, y0 - 3, y0 + SH + 3);
        else
          prefetch_block<uint16_t>(J.scr.pl[t.plane], x0 - 3, x0 + PW + 3, y0 - 3, y0 + SH + 3);
      });
}

cudaError_t launch_lr_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_lr_batch<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LrSmem));
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k_lr_batch<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LrSmem));
    if (e != cudaSuccess) return e;
    configured = true;
  }
  static int wave = 0;
  if (batch_loops(b))
    k_lr_batch<true><<<grid, 256, sizeof(LrSmem), st>>>(b);
  else
    k_lr_batch<false><<<grid, 256, sizeof(LrSmem), st>>>(with_wave(b, k_lr_batch<false>, 256, sizeof(LrSmem), wave));
  return cudaGetLastError();
}

// ---- encoder loop-restoration unit search ----
// encoder/restoration.go:149-210 (SearchWienerUnitU8), :216-263
// (SearchSGRProjUnitU8) and the unit loops of EncodeLoopRestorationKeyframe
// (encoder/keyframe_lossy.go:2313-2383, :2422-2453), luma of 8-bit frames.
//
// Two launches.  k_lr_search_sse: one CTA per (unit, job); job 0 measures
// the unfiltered SSE, the six horizontal-only Wiener candidates and the
// exact Wiener filter of the pick, jobs 1..4 one exact SGR preset each, into
// a table of 32-bit SSEs (a unit holds at most 95 x 95 samples, so every sum
// stays below 2^32).  When the output is wanted, each exact filter also
// stores its filtered unit in a candidate buffer ([unit][job][64 x 64]
// bytes, 10 MB at 1080p, so it stays in L2).  k_lr_search_decide: one CTA
// per unit replays the reference's decisions over the table, writes the
// unit record and copies the winner's samples (or the unfiltered ones) into
// the output plane.

// The candidate tap sets and presets of encoder/restoration.go:166-173 and
// :235-240, in the reference's order (first strictly better wins).
__constant__ int8_t c_lrs_wiener[PF_LR_WIENER_CANDIDATES][3] = {
    {0, -3, 12}, {0, -5, 18}, {0, -2, 8}, {0, 2, 10}, {1, 4, 14}, {0, -1, 4}};
__constant__ int8_t c_lrs_sgr[PF_LR_SGR_PRESETS][3] = {{0, 8, 24}, {2, 16, 40}, {10, 0, 48}, {14, 24, 72}};

constexpr uint32_t kLrsNone = 0xffffffffu;

struct LrsSse {
  uint32_t base;
  uint32_t wiener[PF_LR_WIENER_CANDIDATES];  // horizontal approximation
  uint32_t wexact;                           // exact Wiener of the pick
  uint32_t sgr[PF_LR_SGR_PRESETS];
  int32_t wpick;
};

struct LrsArgs {
  const uint8_t* src;
  int64_t sstride;
  const uint8_t* rec;
  int64_t rstride;
  uint8_t* dst;  // null: search only
  int64_t dstride;
  int W, H, horz, vert;
  LrsSse* table;
  pf_lr_search_unit* out;
  uint8_t* cand;  // [unit][1 + PF_LR_SGR_PRESETS][64 * 64]; null: search only
};

constexpr int kLrsJobs = 1 + PF_LR_SGR_PRESETS;

__device__ __forceinline__ uint8_t* lrs_cand(const LrsArgs& a, int unit, int job) {
  return a.cand + ((size_t)unit * kLrsJobs + job) * 4096;
}

struct LrsSmem {
  LrSmem lr;
  uint8_t src[64 * 64];
  uint32_t red[8 * 8];
};

// tile/restoration_geometry.go:54-92 for luma units of 64.
__device__ __forceinline__ void lrs_rect(const LrsArgs& a, int col, int row, int& x0, int& y0, int& x1, int& y1) {
  x0 = col * 64;
  x1 = col + 1 == a.horz ? a.W : x0 + 64;
  y0 = row * 64;
  y1 = row + 1 == a.vert ? a.H : y0 + 64;
  if (y0 > 0) y0 -= 8;
  if (y1 < a.H) y1 -= 8;
}

// Sums N per-thread values over the CTA; every thread gets the totals.
template <int N>
__device__ __forceinline__ void lrs_block_sum(uint32_t (&v)[N], uint32_t* red) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int i = 0; i < N; i++) {
    uint32_t x = v[i];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) red[warp * N + i] = x;
  }
  __syncthreads();
#pragma unroll
  for (int i = 0; i < N; i++) {
    uint32_t x = 0;
    for (int k = 0; k < 8; k++) x += red[k * N + i];
    v[i] = x;
  }
  __syncthreads();
}

// The unit's recon window with a 3-sample edge-clamped border (the bordered
// copy of keyframe_lossy.go:2313-2330) into sm.lr.win; the SGR table when
// `tables`; the unit's source samples into sm.src when `source`.
__device__ __forceinline__ void lrs_stage(const LrsArgs& a, LrsSmem& sm, int x0, int y0, int w, int h, bool tables,
                                          bool source) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Six loads in flight per lane, as in lr_tile.
  for (int r0 = warp; r0 < h + 6; r0 += 16) {
    uint8_t v[2][3];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int r = r0 + 8 * q;
      if (r < h + 6) {
        const uint8_t* row = a.rec + (int64_t)iclip(y0 - 3 + r, 0, a.H - 1) * a.rstride;
#pragma unroll
        for (int k = 0; k < 3; k++)
          if (lane + 32 * k < w + 6) v[q][k] = row[iclip(x0 - 3 + lane + 32 * k, 0, a.W - 1)];
      }
    }
#pragma unroll
    for (int q = 0; q < 2; q++)
#pragma unroll
      for (int k = 0; k < 3; k++)
        if (r0 + 8 * q < h + 6 && lane + 32 * k < w + 6) sm.lr.win[(r0 + 8 * q) * kWin + lane + 32 * k] = v[q][k];
  }
  if (source)
    for (int r = warp; r < h; r += 8) {
      const uint8_t* row = a.src + (int64_t)(y0 + r) * a.sstride + x0;
      for (int c = lane; c < w; c += 32) sm.src[r * 64 + c] = row[c];
    }
  if (tables) sm.lr.x_by_xplus1[threadIdx.x] = c_x_by_xplus1[threadIdx.x];
  __syncthreads();
}

// The same sets as compile-time values, for the unrolled candidate loop.
__host__ __device__ constexpr int lrs_tap(int c, int k) {
  constexpr int8_t t[PF_LR_WIENER_CANDIDATES][3] = {{0, -3, 12}, {0, -5, 18}, {0, -2, 8},
                                                    {0, 2, 10},  {1, 4, 14},  {0, -1, 4}};
  return t[c][k];
}

// One candidate's horizontal-only prediction (encoder/restoration.go:181-198)
// from the symmetric pair sums p06, p15, p24 and the centre p3.
template <int C>
__device__ __forceinline__ int lrs_hpred(int p06, int p15, int p24, int p3) {
  constexpr int t0 = lrs_tap(C, 0), t1 = lrs_tap(C, 1), t2 = lrs_tap(C, 2), t3 = -2 * (t0 + t1 + t2);
  const int hs = t0 * p06 + t1 * p15 + t2 * p24 + t3 * p3;
  return iclip((hs + 64) >> 7, 0, 255);
}

template <int C>
__device__ __forceinline__ void lrs_hsse(uint32_t* acc, int s, int p06, int p15, int p24, int p3) {
  const int d = s - lrs_hpred<C>(p06, p15, p24, p3);
  acc[1 + C] += (uint32_t)(d * d);
  if constexpr (C + 1 < PF_LR_WIENER_CANDIDATES) lrs_hsse<C + 1>(acc, s, p06, p15, p24, p3);
}

__device__ __forceinline__ void lrs_taps(int c, int* f) {
  const int t0 = c_lrs_wiener[c][0], t1 = c_lrs_wiener[c][1], t2 = c_lrs_wiener[c][2];
  f[0] = f[6] = t0;
  f[1] = f[5] = t1;
  f[2] = f[4] = t2;
  f[3] = -2 * (t0 + t1 + t2);  // restoration/wiener.go:44-47 (NewWienerFilter)
}

// SearchWienerUnitU8's choice over the table (encoder/restoration.go:161-209).
__device__ __forceinline__ int lrs_wiener_pick(const uint32_t* cand, uint32_t base, int area) {
  int pick = -1;
  uint64_t best = base;
  if (base != 0)
    for (int c = 0; c < PF_LR_WIENER_CANDIDATES; c++)
      if ((uint64_t)cand[c] + (uint64_t)area < best) {
        best = cand[c];
        pick = c;
      }
  return pick;
}

__global__ void __launch_bounds__(256, 3) k_lr_search_sse(LrsArgs a) {
  extern __shared__ __align__(16) uint8_t lrs_smem_raw[];
  LrsSmem& sm = *reinterpret_cast<LrsSmem*>(lrs_smem_raw);
  const int unit = blockIdx.x, job = blockIdx.y;
  int x0, y0, x1, y1;
  lrs_rect(a, unit % a.horz, unit / a.horz, x0, y0, x1, y1);
  const int w = x1 - x0, h = y1 - y0;
  const bool fits = w <= 64 && h <= 64;  // restoration/wiener.go:198-200
  LrsSse& T = a.table[unit];
  const int tid = threadIdx.x;
  if (job > 0) {
    // SearchSGRProjUnitU8, one preset (encoder/restoration.go:242-261).
    const int p = job - 1;
    if (!fits) {
      if (tid == 0) T.sgr[p] = kLrsNone;
      return;
    }
    lrs_stage(a, sm, x0, y0, w, h, true, true);
    uint32_t acc[1] = {0};
    uint8_t* keep = a.cand ? lrs_cand(a, unit, job) : nullptr;
    lr_sgr_window(sm.lr, w, h, 8, c_lrs_sgr[p][0], c_lrs_sgr[p][1], c_lrs_sgr[p][2], 64, [&](int y, int x, int v) {
      const int d = (int)sm.src[y * 64 + x] - v;
      acc[0] += (uint32_t)(d * d);
      if (keep) keep[y * 64 + x] = (uint8_t)v;
    });
    lrs_block_sum(acc, sm.red);
    if (tid == 0) T.sgr[p] = acc[0];
    return;
  }
  // Job 0: SearchWienerUnitU8 (encoder/restoration.go:149-210).
  uint32_t acc[1 + PF_LR_WIENER_CANDIDATES];
#pragma unroll
  for (int i = 0; i <= PF_LR_WIENER_CANDIDATES; i++) acc[i] = 0;
  if (fits) {
    lrs_stage(a, sm, x0, y0, w, h, false, true);
    const int tx = tid & 63;
    if (tx < w)
      for (int y = tid >> 6; y < h; y += 4) {
        const uint16_t* wr = &sm.lr.win[(y + 3) * kWin + tx];
        const int s = sm.src[y * 64 + tx];
        const int d0 = s - (int)wr[3];
        acc[0] += (uint32_t)(d0 * d0);
        lrs_hsse<0>(acc, s, wr[0] + wr[6], wr[1] + wr[5], wr[2] + wr[4], wr[3]);
      }
  } else {
    // Units larger than 64x64 (the last row or column of some frame sizes):
    // the search still runs on them, straight from the frame.
    for (int i = tid; i < w * h; i += 256) {
      const int y = y0 + i / w, x = x0 + i % w;
      const uint8_t* rr = a.rec + (int64_t)y * a.rstride;
      const int s = a.src[(int64_t)y * a.sstride + x];
      const int d0 = s - (int)rr[x];
      acc[0] += (uint32_t)(d0 * d0);
      int px[7];
#pragma unroll
      for (int k = 0; k < 7; k++) px[k] = rr[iclip(x + k - 3, 0, a.W - 1)];
      lrs_hsse<0>(acc, s, px[0] + px[6], px[1] + px[5], px[2] + px[4], px[3]);
    }
  }
  lrs_block_sum(acc, sm.red);
  const int pick = lrs_wiener_pick(acc + 1, acc[0], w * h);
  uint32_t ex[1] = {kLrsNone};
  if (pick >= 0 && fits) {
    // The exact filter of the pick (keyframe_lossy.go:2344-2366).
    int fv[7];
    lrs_taps(pick, fv);
    ex[0] = 0;
    uint8_t* keep = a.cand ? lrs_cand(a, unit, 0) : nullptr;
    lr_wiener_window(sm.lr, w, h, 8, fv, fv, 64, [&](int y, int x, int v) {
      const int d = (int)sm.src[y * 64 + x] - v;
      ex[0] += (uint32_t)(d * d);
      if (keep) keep[y * 64 + x] = (uint8_t)v;
    });
    lrs_block_sum(ex, sm.red);
  }
  if (tid == 0) {
    T.base = acc[0];
    for (int c = 0; c < PF_LR_WIENER_CANDIDATES; c++) T.wiener[c] = acc[1 + c];
    T.wexact = ex[0];
    T.wpick = pick;
  }
}

// The unit's decision (keyframe_lossy.go:2338-2382) and, with a.dst, the
// unit filtered by it (:2422-2453).
__global__ void __launch_bounds__(256) k_lr_search_decide(LrsArgs a) {
  const int unit = blockIdx.x, tid = threadIdx.x;
  int x0, y0, x1, y1;
  lrs_rect(a, unit % a.horz, unit / a.horz, x0, y0, x1, y1);
  const int w = x1 - x0, h = y1 - y0;
  const bool fits = w <= 64 && h <= 64;
  const LrsSse& T = a.table[unit];
  const uint64_t base = T.base;
  const int wpick = T.wpick;
  uint64_t best = ~0ull;
  int type = PF_LR_NONE;
  if (wpick >= 0 && fits) {
    best = T.wexact;
    type = PF_LR_WIENER;
  }
  int spick = -1;
  uint64_t sbest = fits ? base : ~0ull;
  if (fits && base != 0)
    for (int p = 0; p < PF_LR_SGR_PRESETS; p++)
      if ((uint64_t)T.sgr[p] + (uint64_t)(w * h) < sbest) {
        sbest = T.sgr[p];
        spick = p;
      }
  if (spick >= 0 && sbest < best) {
    best = sbest;
    type = PF_LR_SGRPROJ;
  }
  if (tid == 0) {
    pf_lr_search_unit r;
    memset(&r, 0, sizeof(r));
    r.x0 = x0;
    r.y0 = y0;
    r.x1 = x1;
    r.y1 = y1;
    r.base_sse = base;
    r.sse = type == PF_LR_NONE ? base : best;
    r.wiener_sse = wpick >= 0 && fits ? (uint64_t)T.wexact : ~0ull;
    r.sgr_sse = sbest;
    r.wiener_candidate = (int8_t)wpick;
    r.sgr_preset = (int8_t)spick;
    r.unit.type = (uint8_t)type;
    if (type == PF_LR_WIENER)
      for (int k = 0; k < 3; k++) r.unit.wiener_v[k] = r.unit.wiener_h[k] = c_lrs_wiener[wpick][k];
    if (type == PF_LR_SGRPROJ) {
      r.unit.sgr_set = (uint8_t)c_lrs_sgr[spick][0];
      r.unit.sgr_xqd[0] = c_lrs_sgr[spick][1];
      r.unit.sgr_xqd[1] = c_lrs_sgr[spick][2];
    }
    a.out[unit] = r;
  }
  if (!a.dst) return;
  // keyframe_lossy.go:2422-2453: the decided filter's samples, kept by the
  // measuring CTA; NONE units keep the reconstruction.
  const uint8_t* from = type == PF_LR_WIENER ? lrs_cand(a, unit, 0)
                        : type == PF_LR_SGRPROJ ? lrs_cand(a, unit, 1 + spick) : nullptr;
  if (from) {
    const int x = tid & 63;
    if (x < w)
      for (int y = tid >> 6; y < h; y += 4) a.dst[(int64_t)(y0 + y) * a.dstride + x0 + x] = from[y * 64 + x];
    return;
  }
  for (int y = tid >> 5; y < h; y += 8)
    for (int x = tid & 31; x < w; x += 32)
      a.dst[(int64_t)(y0 + y) * a.dstride + x0 + x] = a.rec[(int64_t)(y0 + y) * a.rstride + x0 + x];
}

static int lrs_check(const pf_frame* f, const pf_frame* ref) {
  // goav1's keyframe encoder works on 8-bit 4:2:0 pictures (SourceFrame420).
  if (f->bit_depth != 8 || f->ss_x != 1 || f->ss_y != 1 || f->mono || f->width != ref->width ||
      f->height != ref->height)
    return PF_ERR_UNSUPPORTED;
  if (f->memory != ref->memory || f->memory > PF_MEM_DEVICE) return PF_ERR_INVALID_ARG;
  const pf_plane& pl = f->plane[0];
  if (!pl.data || pl.width != ref->width || pl.height != ref->height || pl.stride < pl.width)
    return PF_ERR_SHORT_BUFFER;
  return PF_OK;
}

}  // namespace pf

void* pf_internal_search_scratch(pf_ctx* c, size_t bytes);  // pf_api.cu
int pf_internal_wait(pf_ctx* c, void* stream);  // pf_api.cu: blocking or bounded by the context's deadline
void* pf_internal_stream(pf_ctx* c);
void* pf_internal_pinned(pf_ctx* c, size_t bytes);

extern "C" int pf_lr_search(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const pf_frame* restored,
                            pf_lr_search_unit* units, int32_t max_units) {
  using namespace pf;
  if (!ctx || !source || !recon) return PF_ERR_INVALID_ARG;
  if (recon->width <= 0 || recon->height <= 0) return PF_ERR_INVALID_ARG;
  int stt = lrs_check(recon, recon);
  if (stt == PF_OK) stt = lrs_check(source, recon);
  if (stt == PF_OK && restored) stt = lrs_check(restored, recon);
  if (stt != PF_OK) return stt;
  const int W = recon->width, H = recon->height;
  const int horz = imax((W + 32) / 64, 1), vert = imax((H + 32) / 64, 1), n = horz * vert;
  if (units && max_units < n) return PF_ERR_SHORT_BUFFER;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  const bool host = recon->memory == PF_MEM_HOST;
  const pf_plane &sp = source->plane[0], &rp = recon->plane[0];
  // In place (restored's luma is recon's): the unit filters read a copy.
  const bool alias = restored && restored->plane[0].data == rp.data;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t plane = al((size_t)W * H);
  size_t off = 0;
  const size_t oTab = off;
  off += al(sizeof(LrsSse) * n);
  const size_t oOut = off;
  off += al(sizeof(pf_lr_search_unit) * n);
  const size_t oSrc = off;
  off += host ? plane : 0;
  const size_t oRec = off;
  off += host || alias ? plane : 0;
  const size_t oDst = off;
  off += host && restored ? plane : 0;
  const size_t oCand = off;
  off += restored ? (size_t)n * kLrsJobs * 4096 : 0;
  uint8_t* base = (uint8_t*)pf_internal_search_scratch(ctx, off);
  if (!base) return PF_ERR_DEVICE;
  LrsArgs a;
  a.W = W;
  a.H = H;
  a.horz = horz;
  a.vert = vert;
  a.table = (LrsSse*)(base + oTab);
  a.out = (pf_lr_search_unit*)(base + oOut);
  a.cand = restored ? base + oCand : nullptr;
  cudaError_t e = cudaSuccess;
  const cudaMemcpyKind up = host ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
  if (host) {
    a.src = base + oSrc;
    a.sstride = W;
    e = cudaMemcpy2DAsync(base + oSrc, W, sp.data, sp.stride, W, H, up, st);
  } else {
    a.src = (const uint8_t*)sp.data;
    a.sstride = sp.stride;
  }
  if (host || alias) {
    a.rec = base + oRec;
    a.rstride = W;
    if (e == cudaSuccess) e = cudaMemcpy2DAsync(base + oRec, W, rp.data, rp.stride, W, H, up, st);
  } else {
    a.rec = (const uint8_t*)rp.data;
    a.rstride = rp.stride;
  }
  a.dst = nullptr;
  a.dstride = 0;
  if (restored) {
    a.dst = host ? base + oDst : (uint8_t*)restored->plane[0].data;
    a.dstride = host ? W : restored->plane[0].stride;
  }
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  static bool configured = false;
  if (!configured) {
    if (cudaFuncSetAttribute(k_lr_search_sse, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sizeof(LrsSmem)) !=
        cudaSuccess)
      return PF_ERR_DEVICE;
    configured = true;
  }
  k_lr_search_sse<<<dim3(n, 1 + PF_LR_SGR_PRESETS), 256, sizeof(LrsSmem), st>>>(a);
  k_lr_search_decide<<<n, 256, 0, st>>>(a);
  e = cudaGetLastError();
  if (e == cudaSuccess && host && restored)
    e = cudaMemcpy2DAsync(restored->plane[0].data, restored->plane[0].stride, a.dst, W, W, H,
                          cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && units)
    e = cudaMemcpyAsync(units, a.out, sizeof(pf_lr_search_unit) * n, cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  return pf_internal_wait(ctx, st);
}

