// pf_deblock.cu - AV1 deblocking on the GPU.
//
// Follows goav1's mask-driven deblock: internal/av1/decoder/
// postfilter_loopfilter_masks.go:229-268 (all vertical edges of the frame,
// then all horizontal edges; chroma gated off when both luma frame levels or
// the plane's base level are zero), postfilter_loopfilter_masks_sb.go:21-188
// (the per-128x128-region bitmask walk, edges outside the 4-aligned crop and
// column/row 0 dropped), loopfilter/sb.go:99-153 (width class from the mask
// lanes, level fallback to the left/above cell) and sb.go:156-446 (the
// 4/6/8/16-wide edge kernels).
//
// Same-direction edges never overlap (AV1 ties filter width to transform
// spacing), so every 4-sample edge unit of one direction is independent: one
// thread owns one unit (4 lines), warps run along the edge grid so the 32
// threads of a warp touch one 128-byte span per row.
#include <type_traits>

#include "pf_common.cuh"

namespace pf {

// loopfilter/sb.go:348-446 (lpfUnit16); reduces to lpfUnit8 at bd == 8.
// q points at q0 of the first line; sa steps along the edge, sb across it
// (both in elements).
// The inner samples of the unit's four lines: P[i][k] = p_k, Q[i][k] = q_k of
// line i (k < 4).  `q` points at q0 of line 0; dir 0 (vertical edge) steps
// lines by rows, dir 1 by columns.  With `words`, eight 4-sample words are
// read (4 bytes, or 8 for 16-bit samples): for a vertical edge the p3..p0
// and q0..q3 runs of each line, for a horizontal edge the four lines'
// samples of each of the eight rows; else sample by sample.
template <typename T>
__device__ __forceinline__ void lpf_inner(const T* q, int stride, int dir, bool words, int (&P)[4][4],
                                          int (&Q)[4][4]) {
  if (!words) {
    const int sa = dir == 0 ? stride : 1, sb = dir == 0 ? 1 : stride;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        P[i][k] = q[i * sa - (k + 1) * sb];
        Q[i][k] = q[i * sa + k * sb];
      }
    return;
  }
  typedef typename std::conditional<sizeof(T) == 1, uint32_t, uint2>::type W;
  auto lane = [](const W& w, int j) -> int {
    if constexpr (sizeof(T) == 1) {
      return (w >> (8 * j)) & 0xff;
    } else {
      return ((j < 2 ? w.x : w.y) >> (16 * (j & 1))) & 0xffff;
    }
  };
  W v[8];
  if (dir == 0) {
#pragma unroll
    for (int i = 0; i < 4; i++) {
      v[2 * i] = *reinterpret_cast<const W*>(q + (int64_t)i * stride - 4);
      v[2 * i + 1] = *reinterpret_cast<const W*>(q + (int64_t)i * stride);
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        P[i][k] = lane(v[2 * i], 3 - k);
        Q[i][k] = lane(v[2 * i + 1], k);
      }
  } else {
#pragma unroll
    for (int j = 0; j < 8; j++) v[j] = *reinterpret_cast<const W*>(q + (int64_t)(j - 4) * stride);
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        P[i][k] = lane(v[3 - k], i);
        Q[i][k] = lane(v[4 + k], i);
      }
  }
}

template <typename T>
__device__ __forceinline__ void lpf_unit(T* q, int sa, int sb, int bd, int E, int I, int H, int wd,
                                         const int (&P)[4][4], const int (&Q)[4][4]) {
  const int bd8 = bd - 8;
  const int F = 1 << bd8;
  E <<= bd8;
  I <<= bd8;
  H <<= bd8;
  const unsigned twoI = 2u * I, twoF = 2u * F, twoH = 2u * H;
  const int maxPix = (1 << bd) - 1;
  const int diffMin = -128 << bd8, diffMax = (128 << bd8) - 1;
  // The four lines never overlap, so the inner samples of all four (P, Q:
  // p3..q3) were read by the caller before any line is filtered.
#pragma unroll
  for (int i = 0; i < 4; i++, q += sa) {
    const int p1 = P[i][1], p0 = P[i][0], q0 = Q[i][0], q1 = Q[i][1];
    if ((unsigned)(p1 - p0 + I) > twoI || (unsigned)(q1 - q0 + I) > twoI ||
        abs(p0 - q0) * 2 + (abs(p1 - q1) >> 1) > E)
      continue;
    int p2 = 0, q2 = 0, p3 = 0, q3 = 0;
    if (wd > 4) {
      p2 = P[i][2];
      q2 = Q[i][2];
      if ((unsigned)(p2 - p1 + I) > twoI || (unsigned)(q2 - q1 + I) > twoI) continue;
      if (wd > 6) {
        p3 = P[i][3];
        q3 = Q[i][3];
        if ((unsigned)(p3 - p2 + I) > twoI || (unsigned)(q3 - q2 + I) > twoI) continue;
      }
    }
    bool flat8in = false;
    if (wd >= 6) {
      flat8in = (unsigned)(p2 - p0 + F) <= twoF && (unsigned)(p1 - p0 + F) <= twoF &&
                (unsigned)(q1 - q0 + F) <= twoF && (unsigned)(q2 - q0 + F) <= twoF;
      if (wd >= 8 && flat8in) flat8in = (unsigned)(p3 - p0 + F) <= twoF && (unsigned)(q3 - q0 + F) <= twoF;
    }
    if (flat8in) {
      if (wd >= 16) {
        const int p6 = q[-7 * sb], p5 = q[-6 * sb], p4 = q[-5 * sb];
        const int q4 = q[4 * sb], q5 = q[5 * sb], q6 = q[6 * sb];
        if ((unsigned)(p6 - p0 + F) <= twoF && (unsigned)(p5 - p0 + F) <= twoF &&
            (unsigned)(p4 - p0 + F) <= twoF && (unsigned)(q4 - q0 + F) <= twoF &&
            (unsigned)(q5 - q0 + F) <= twoF && (unsigned)(q6 - q0 + F) <= twoF) {
          // The twelve outputs as one running sum: each output's 16-weight
          // window differs from the previous one by two samples in, two out.
          int t = p6 * 7 + p5 * 2 + p4 * 2 + p3 + p2 + p1 + p0 + q0 + 8;
          q[-6 * sb] = (T)(t >> 4);
          t += p3 + q1 - 2 * p6;
          q[-5 * sb] = (T)(t >> 4);
          t += p2 + q2 - p6 - p5;
          q[-4 * sb] = (T)(t >> 4);
          t += p1 + q3 - p6 - p4;
          q[-3 * sb] = (T)(t >> 4);
          t += p0 + q4 - p6 - p3;
          q[-2 * sb] = (T)(t >> 4);
          t += q0 + q5 - p6 - p2;
          q[-sb] = (T)(t >> 4);
          t += q1 + q6 - p6 - p1;
          q[0] = (T)(t >> 4);
          t += q2 + q6 - p5 - p0;
          q[sb] = (T)(t >> 4);
          t += q3 + q6 - p4 - q0;
          q[2 * sb] = (T)(t >> 4);
          t += q4 + q6 - p3 - q1;
          q[3 * sb] = (T)(t >> 4);
          t += q5 + q6 - p2 - q2;
          q[4 * sb] = (T)(t >> 4);
          t += 2 * q6 - p1 - q3;
          q[5 * sb] = (T)(t >> 4);
          continue;
        }
      }
      if (wd >= 8) {
        q[-3 * sb] = (T)((p3 * 3 + p2 * 2 + p1 + p0 + q0 + 4) >> 3);
        q[-2 * sb] = (T)((p3 * 2 + p2 + p1 * 2 + p0 + q0 + q1 + 4) >> 3);
        q[-sb] = (T)((p3 + p2 + p1 + p0 * 2 + q0 + q1 + q2 + 4) >> 3);
        q[0] = (T)((p2 + p1 + p0 + q0 * 2 + q1 + q2 + q3 + 4) >> 3);
        q[sb] = (T)((p1 + p0 + q0 + q1 * 2 + q2 + q3 * 2 + 4) >> 3);
        q[2 * sb] = (T)((p0 + q0 + q1 + q2 * 2 + q3 * 3 + 4) >> 3);
        continue;
      }
      q[-2 * sb] = (T)((p2 * 3 + p1 * 2 + p0 * 2 + q0 + 4) >> 3);
      q[-sb] = (T)((p2 + p1 * 2 + p0 * 2 + q0 * 2 + q1 + 4) >> 3);
      q[0] = (T)((p1 + p0 * 2 + q0 * 2 + q1 * 2 + q2 + 4) >> 3);
      q[sb] = (T)((p0 + q0 * 2 + q1 * 2 + q2 * 3 + 4) >> 3);
      continue;
    }
    const bool hev = (unsigned)(p1 - p0 + H) > twoH || (unsigned)(q1 - q0 + H) > twoH;
    int f;
    if (hev)
      f = imin(imax(imin(imax(p1 - q1, diffMin), diffMax) + 3 * (q0 - p0), diffMin), diffMax);
    else
      f = imin(imax(3 * (q0 - p0), diffMin), diffMax);
    const int f1 = imin(f + 4, diffMax) >> 3;
    const int f2 = imin(f + 3, diffMax) >> 3;
    q[-sb] = (T)imin(imax(p0 + f2, 0), maxPix);
    q[0] = (T)imin(imax(q0 - f1, 0), maxPix);
    if (!hev) {
      f = (f1 + 1) >> 1;
      q[-2 * sb] = (T)imin(imax(p1 + f, 0), maxPix);
      q[sb] = (T)imin(imax(q1 - f, 0), maxPix);
    }
  }
}

// One thread per 4x4 edge unit (c4, r4) of `plane`; dir 0 filters the
// unit's left (vertical) edge, dir 1 its top (horizontal) edge.
template <typename T>
__device__ __forceinline__ void deblock_unit(const DFrame& f, const LfArgs& a, int dir, int plane, int c4, int r4) {
  if (a.gate_chroma[plane]) return;
  const int ssx = plane ? f.ssx : 0, ssy = plane ? f.ssy : 0;
  // frameWorkLoopFilterPlaneSize: edge positions inside the 4-aligned crop.
  const int w4 = ((plane ? (f.width + ssx) >> ssx : f.width) + 3) >> 2;
  const int h4 = ((plane ? (f.height + ssy) >> ssy : f.height) + 3) >> 2;
  if (c4 >= w4 || r4 >= h4) return;
  if (dir == 0 ? c4 == 0 : r4 == 0) return;
  const bool luma = plane == 0;
  const int regionW = 32 >> ssx, regionH = 32 >> ssy;
  const int rCol = c4 / regionW, rRow = r4 / regionH;
  const int pcol = c4 - rCol * regionW, prow = r4 - rRow * regionH;
  const uint16_t* region = a.masks + (size_t)(rRow * a.sb128_w + rCol) * PF_LF_MASK_WORDS;
  const int pos = dir == 0 ? pcol : prow;
  const int bit = dir == 0 ? prow : pcol;
  // The cell's and its left / upper neighbour's levels (sb.go:122-128,
  // :142-148) and the unit's inner samples depend only on the cell: their
  // loads go out with the mask words' instead of after them.  The inner
  // samples p3..q3 of the four lines lie inside the allocated plane for
  // every unit past the first column / row (edge positions are inside the
  // 4-aligned crop, which the 8-aligned allocation covers).
  const int comp = plane == 0 ? dir : plane + 1;
  const int li = r4 * a.mi_cols + c4;
  const int L0 = __ldg(&a.level_cache[4 * li + comp]);
  const int L1 = __ldg(&a.level_cache[4 * (dir == 0 ? li - 1 : li - a.mi_cols) + comp]);
  const DPlane& pl = f.pl[plane];
  const int pos0 = dir == 0 ? c4 * 4 : r4 * 4;
  const int lim = dir == 0 ? pl.aw : pl.ah;
  const int along = dir == 0 ? r4 * 4 + 3 : c4 * 4 + 3;
  const int alongLim = dir == 0 ? pl.ah : pl.aw;
  if (pos0 - 4 < 0 || pos0 + 3 >= lim || along >= alongLim) return;
  const int sstride = (int)(pl.stride / sizeof(T));
  T* q = row_ptr<T>(pl, r4 * 4) + c4 * 4;
  const bool words = (((uintptr_t)pl.ptr | (uintptr_t)pl.stride) & (4 * sizeof(T) - 1)) == 0;
  int P[4][4], Q[4][4];
  lpf_inner<T>(q, sstride, dir, words, P, Q);
  // The width class: the widest mask lane with this unit's bit set; every
  // lane's word is read up front so the loads go out together.
  int k = -1;
  if (luma) {
    const int half = bit >> 4, b = bit & 15;
    const uint16_t* m = &region[((dir * 32 + pos) * 3) * 2 + half];
    const int w0 = __ldg(&m[0]), w1 = __ldg(&m[2]), w2 = __ldg(&m[4]);
    k = ((w2 >> b) & 1) ? 2 : ((w1 >> b) & 1) ? 1 : ((w0 >> b) & 1) ? 0 : -1;
  } else {
    const int lane = dir == 0 ? (16 >> ssy) : (16 >> ssx);
    const int half = bit / lane, b = bit - half * lane;
    const uint16_t* m = &region[384 + ((dir * 32 + pos) * 2) * 2 + half];
    const int w0 = __ldg(&m[0]), w1 = __ldg(&m[2]);
    k = ((w1 >> b) & 1) ? 1 : ((w0 >> b) & 1) ? 0 : -1;
  }
  if (k < 0) return;
  const int wd = k == 2 ? 16 : (k == 1 ? (luma ? 8 : 6) : 4);
  // Level with the left / above fallback: the neighbour's when this cell's
  // is 0 (c4 > 0 for vertical, r4 > 0 for horizontal edges here).
  const int L = L0 != 0 ? L0 : L1;
  if (L == 0) return;
  // loopfilter/threshold.go:18-47.
  const int sh = a.sharpness;
  int limit = L >> ((sh > 0) + (sh > 4));
  if (sh > 0 && limit > 9 - sh) limit = 9 - sh;
  if (limit < 1) limit = 1;
  const int E = 2 * (L + 2) + limit, I = limit, H = L >> 4;
  // The masks are trusted like the reference trusts them, but a 14-tap edge
  // whose outer taps would leave the allocated plane (only a malformed mask
  // can ask for one; the reference would fault on it) is skipped instead of
  // touched.
  if (wd == 16 && (pos0 - 7 < 0 || pos0 + 6 >= lim)) return;
  const int bd = sizeof(T) == 1 ? 8 : f.bd;  // a constant for 8-bit: the depth shifts fold
  if (dir == 0)
    lpf_unit<T>(q, sstride, 1, bd, E, I, H, wd, P, Q);
  else
    lpf_unit<T>(q, 1, sstride, bd, E, I, H, wd, P, Q);
}

// Batched deblocking: each work item is one tile of edge units of one plane
// of one frame (db_tile_w x db_tile_h units, 32x8 by default); 256 threads,
// one edge unit each.
struct DbTile {
  const FrameJob* J;
  int plane, tx, ty;
};

__device__ __forceinline__ DbTile db_locate(const BatchArgs& b, const int* base, int item) {
  const int fi = find_frame(base, b.n, item);
  const FrameJob& J = b.jobs[fi];
  int local = item - base[fi];
  int plane = 0;
  while (plane < 2 && local >= J.db_tx[plane] * J.db_ty[plane]) {
    local -= J.db_tx[plane] * J.db_ty[plane];
    plane++;
  }
  return DbTile{&J, plane, local % J.db_tx[plane], local / J.db_tx[plane]};
}

template <bool kLoop>
__global__ void __launch_bounds__(256, 4) k_deblock_batch(BatchArgs b, int dir) {
  const int stage = dir == 0 ? ST_DEBLOCK_V : ST_DEBLOCK_H;
  const int* base = b.base + stage * (b.n + 1);
  for_each_item<kLoop>(
      b, stage,
      [&](int item) {
        const DbTile t = db_locate(b, base, item);
        const FrameJob& J = *t.J;
        const int tw = db_tile_w(J.db_tile), lg = 31 - __clz(tw);
        const int c4 = t.tx * tw + (threadIdx.x & (tw - 1)), r4 = t.ty * (256 >> lg) + (threadIdx.x >> lg);
        if (J.io.bd == 8)
          deblock_unit<uint8_t>(J.io, J.lf, dir, t.plane, c4, r4);
        else
          deblock_unit<uint16_t>(J.io, J.lf, dir, t.plane, c4, r4);
      },
      [&](int item) {
        // The tile's samples and the 8 on each side its edges can reach.
        const DbTile t = db_locate(b, base, item);
        const int tw = db_tile_w(t.J->db_tile), th = 256 / tw;
        const int x0 = t.tx * tw * 4, y0 = t.ty * th * 4;
        if (t.J->io.bd == 8)
          prefetch_block<uint8_t>(t.J->io.pl[t.plane], x0 - 8, x0 + tw * 4 + 8, y0 - 8, y0 + th * 4 + 8);
        else
          prefetch_block<uint16_t>(t.J->io.pl[t.plane], x0 - 8, x0 + tw * 4 + 8, y0 - 8, y0 + th * 4 + 8);
      });
}

cudaError_t launch_deblock_batch(const BatchArgs& b, int total, int grid, int dir, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  static int wave = 0;
  if (batch_loops(b))
    k_deblock_batch<true><<<grid, 256, 0, st>>>(b, dir);
  else
    k_deblock_batch<false><<<grid, 256, 0, st>>>(with_wave(b, k_deblock_batch<false>, 256, 0, wave), dir);
  return cudaGetLastError();
}

}  // namespace pf
