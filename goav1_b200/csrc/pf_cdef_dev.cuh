// pf_cdef_dev.cuh - CDEF device helpers shared by the decoder-side CDEF
// kernel (pf_cdef.cu) and the encoder strength search (pf_search.cu).
// Arithmetic follows goav1's cdef/direction.go:37-79, :432-501 and
// cdef/filter.go:79-191, :603-612.
#pragma once

#include "pf_common.cuh"

namespace pf {

constexpr int kVeryLarge = 0x4000;
constexpr int kSW = 80;   // smem row stride (64 + 2*8)
constexpr int kSH = 68;   // smem rows (64 + 2*2)

// (dy, dx) of the two taps of each CDEF direction entry, cdef/filter.go:53-66.
static __constant__ int8_t c_cdef_dir[12][2][2] = {
    {{1, 0}, {2, 0}},   {{1, 0}, {2, -1}}, {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}},
    {{0, 1}, {0, 2}},   {{0, 1}, {1, 2}},  {{1, 1}, {2, 2}},   {{1, 0}, {2, 1}},
    {{1, 0}, {2, 0}},   {{1, 0}, {2, -1}}, {{-1, 1}, {-2, 2}}, {{0, 1}, {-1, 2}},
};

__device__ __forceinline__ int dir_off(int e, int k) { return c_cdef_dir[e][k][0] * kSW + c_cdef_dir[e][k][1]; }

// Direction cost over one 8x8 block (cdef/direction.go:37-79 partial sums,
// :469-501 cost): for direction D the samples (i, j), shifted to 8 bits
// and less 128, are summed into partials p[dir_k(D, i, j)], and the cost is
// the weighted sum of their squares.  dir_k is that index; dir_count is how
// many samples each partial sums.
__host__ __device__ constexpr int dir_k(int D, int i, int j) {
  return D == 0 ? i + j : D == 1 ? i + (j >> 1) : D == 2 ? i : D == 3 ? 3 + i - (j >> 1) :
         D == 4 ? 7 + i - j : D == 5 ? 3 - (i >> 1) + j : D == 6 ? j : (i >> 1) + j;
}
__host__ __device__ constexpr int dir_count(int D, int k) {
  int n = 0;
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) n += dir_k(D, i, j) == k;
  return n;
}

// The direction cost on packed sample pairs: w[i][m] holds samples (i, 2m) and
// (i, 2m + 1) of the block in its low and high halves, raw.  Each pair is
// added as one 32-bit word into the accumulator of its even sample's index
// (the odd sample's index differs from it by the same -1, 0 or +1 for every
// pair of a direction), with the samples shifted to 8 bits and left biased
// by +128: a half never sums more than eight values below 256, so it never
// carries into the other.  The halves are then split into the partial sums,
// the bias taken off by each sum's sample count, and the cost formed from
// them (direction.go:469-501), so the result is the same integer as summing
// the shifted, unbiased samples one by one.
template <int D>
__host__ __device__ __forceinline__ int32_t dir_cost_pairs(const uint32_t (&w)[8][4], int shift) {
  constexpr int kDelta = dir_k(D, 0, 1) - dir_k(D, 0, 0);
  const uint32_t mask = (0xffffu >> shift) * 0x10001u;
  uint32_t acc[15];
#pragma unroll
  for (int k = 0; k < 15; k++) acc[k] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++)
#pragma unroll
    for (int m = 0; m < 4; m++) acc[dir_k(D, i, 2 * m)] += (w[i][m] >> shift) & mask;
  int32_t p[15];
#pragma unroll
  for (int k = 0; k < 15; k++) {
    int32_t v = (int32_t)(acc[k] & 0xffffu);
    if (k - kDelta >= 0 && k - kDelta < 15) v += (int32_t)(acc[k - kDelta] >> 16);
    p[k] = v - 128 * dir_count(D, k);
  }
  if (D == 2 || D == 6) {
    int32_t s = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += p[i] * p[i];
    return s * 105;
  }
  if (D == 0 || D == 4) {
    const int32_t div[8] = {840, 420, 280, 210, 168, 140, 120, 105};
    int32_t s = 0;
#pragma unroll
    for (int i = 0; i < 7; i++) s += (p[i] * p[i] + p[14 - i] * p[14 - i]) * div[i];
    return s + p[7] * p[7] * 105;
  }
  return (p[3] * p[3] + p[4] * p[4] + p[5] * p[5] + p[6] * p[6] + p[7] * p[7]) * 105 +
         (p[0] * p[0] + p[10] * p[10]) * 420 + (p[1] * p[1] + p[9] * p[9]) * 210 +
         (p[2] * p[2] + p[8] * p[8]) * 140;
}

template <int D>
__device__ __forceinline__ int32_t dir_cost_packed(const uint16_t* blk, int shift) {
  uint32_t w[8][4];
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const uint4 row = *reinterpret_cast<const uint4*>(blk + i * kSW);
    w[i][0] = row.x, w[i][1] = row.y, w[i][2] = row.z, w[i][3] = row.w;
  }
  return dir_cost_pairs<D>(w, shift);
}

__device__ __forceinline__ int32_t dir_cost_any(int d, const uint16_t* blk, int shift) {
  switch (d) {
    case 0: return dir_cost_packed<0>(blk, shift);
    case 1: return dir_cost_packed<1>(blk, shift);
    case 2: return dir_cost_packed<2>(blk, shift);
    case 3: return dir_cost_packed<3>(blk, shift);
    case 4: return dir_cost_packed<4>(blk, shift);
    case 5: return dir_cost_packed<5>(blk, shift);
    case 6: return dir_cost_packed<6>(blk, shift);
    default: return dir_cost_packed<7>(blk, shift);
  }
}

__device__ __forceinline__ int constrain(int diff, int threshold, int shift) {
  const int a = abs(diff);
  const int l = imin(imax(threshold - (a >> shift), 0), a);
  return diff < 0 ? -l : l;
}

__device__ __forceinline__ int constrain_shift(int threshold, int damping) {
  if (threshold == 0) return 0;
  return imax(damping - (31 - __clz(threshold)), 0);
}

__device__ __forceinline__ int adjust_strength(int strength, int32_t variance) {
  if (variance == 0) return 0;
  const int32_t v = variance >> 6;
  const int i = v != 0 ? imin(31 - __clz(v), 12) : 0;
  return (strength * (4 + i) + 8) >> 4;
}

// One sample of cdef/filter.go:79-169; c points at the centre sample in smem.
// po/so: the primary tap offsets (entry dir+2) and the two secondary entries
// (dir+4, dir) as smem offsets; the constrain shifts are precomputed.
// kMask: the input may hold the VeryLarge sentinel, which the clamp's max
// must ignore; an input without sentinels skips the masking.
template <bool kMask = true>
__device__ __forceinline__ int cdef_filter_px(const uint16_t* c, int pri, int priShift, int sec, int secShift,
                                              int2 po, int2 s0, int2 s1, int coeffShift) {
  const int x = c[0];
  int sum = 0;
  int hi = x, lo = x;
  if (pri) {
    const int odd = (pri >> coeffShift) & 1;
    const int t0 = odd ? 3 : 4, t1 = odd ? 3 : 2;
    const int a0 = c[po.x], a1 = c[-po.x], a2 = c[po.y], a3 = c[-po.y];
    sum += t0 * (constrain(a0 - x, pri, priShift) + constrain(a1 - x, pri, priShift)) +
           t1 * (constrain(a2 - x, pri, priShift) + constrain(a3 - x, pri, priShift));
    if (sec) {
      const int m = kMask ? kVeryLarge - 1 : 0xffff;
      hi = __vimax3_s32(__vimax3_s32(hi, a0 & m, a1 & m), a2 & m, a3 & m);
      lo = __vimin3_s32(__vimin3_s32(lo, a0, a1), a2, a3);
    }
  }
  if (sec) {
    const int b0 = c[s0.x], b1 = c[-s0.x], b2 = c[s1.x], b3 = c[-s1.x];
    const int b4 = c[s0.y], b5 = c[-s0.y], b6 = c[s1.y], b7 = c[-s1.y];
    sum += 2 * (constrain(b0 - x, sec, secShift) + constrain(b1 - x, sec, secShift) +
                constrain(b2 - x, sec, secShift) + constrain(b3 - x, sec, secShift)) +
           constrain(b4 - x, sec, secShift) + constrain(b5 - x, sec, secShift) + constrain(b6 - x, sec, secShift) +
           constrain(b7 - x, sec, secShift);
    if (pri) {
      // 3-way DPX min/max: half the instructions of a two-operand chain.
      const int m = kMask ? kVeryLarge - 1 : 0xffff;
      hi = __vimax3_s32(__vimax3_s32(hi, b0 & m, b1 & m), __vimax3_s32(b2 & m, b3 & m, b4 & m),
                        __vimax3_s32(b5 & m, b6 & m, b7 & m));
      lo = __vimin3_s32(__vimin3_s32(lo, b0, b1), __vimin3_s32(b2, b3, b4), __vimin3_s32(b5, b6, b7));
    }
  }
  int y = x + ((8 + sum - (sum < 0)) >> 4);
  if (pri && sec) y = imin(imax(y, lo), hi);
  return y;
}

// cdef_filter_px for 8-bit input without sentinels, with constrain() read
// from tables: tp (primary, the block's strength) and ts (secondary) point at
// the entry for a difference of 0 of 511-entry tables covering -255..255,
// built from constrain() itself, so the result is the same sample.
__device__ __forceinline__ int cdef_filter_px_tab(const uint16_t* c, int pri, const int16_t* tp, int sec,
                                                  const int16_t* ts, int2 po, int2 s0, int2 s1) {
  const int x = c[0];
  int sum = 0;
  int hi = x, lo = x;
  if (pri) {
    const int odd = pri & 1;
    const int t0 = odd ? 3 : 4, t1 = odd ? 3 : 2;
    const int a0 = c[po.x], a1 = c[-po.x], a2 = c[po.y], a3 = c[-po.y];
    sum += t0 * (tp[a0 - x] + tp[a1 - x]) + t1 * (tp[a2 - x] + tp[a3 - x]);
    if (sec) {
      hi = __vimax3_s32(__vimax3_s32(hi, a0, a1), a2, a3);
      lo = __vimin3_s32(__vimin3_s32(lo, a0, a1), a2, a3);
    }
  }
  if (sec) {
    const int b0 = c[s0.x], b1 = c[-s0.x], b2 = c[s1.x], b3 = c[-s1.x];
    const int b4 = c[s0.y], b5 = c[-s0.y], b6 = c[s1.y], b7 = c[-s1.y];
    sum += 2 * (ts[b0 - x] + ts[b1 - x] + ts[b2 - x] + ts[b3 - x]) + ts[b4 - x] + ts[b5 - x] + ts[b6 - x] +
           ts[b7 - x];
    if (pri) {
      hi = __vimax3_s32(__vimax3_s32(hi, b0, b1), __vimax3_s32(b2, b3, b4), __vimax3_s32(b5, b6, b7));
      lo = __vimin3_s32(__vimin3_s32(lo, b0, b1), __vimin3_s32(b2, b3, b4), __vimin3_s32(b5, b6, b7));
    }
  }
  int y = x + ((8 + sum - (sum < 0)) >> 4);
  if (pri && sec) y = imin(imax(y, lo), hi);
  return y;
}

// cdef_filter_px for 8-bit input that may hold the VeryLarge sentinel, with
// constrain() read from 513-entry tables: tp / ts point at the entry for a
// difference of 0, and differences beyond +/-255 (only a sentinel makes one,
// and at 8-bit strengths <= 15 constrain() is 0 there) clamp to the end
// entries, which hold 0.  The clamp-range masking is cdef_filter_px's.
__device__ __forceinline__ int cdef_filter_px_tab8(const uint16_t* c, int pri, const int16_t* tp, int sec,
                                                   const int16_t* ts, int2 po, int2 s0, int2 s1) {
  const int x = c[0];
  auto lut = [](const int16_t* t, int d) { return (int)t[imin(imax(d, -256), 256)]; };
  int sum = 0;
  int hi = x, lo = x;
  constexpr int m = kVeryLarge - 1;
  if (pri) {
    const int odd = pri & 1;
    const int t0 = odd ? 3 : 4, t1 = odd ? 3 : 2;
    const int a0 = c[po.x], a1 = c[-po.x], a2 = c[po.y], a3 = c[-po.y];
    sum += t0 * (lut(tp, a0 - x) + lut(tp, a1 - x)) + t1 * (lut(tp, a2 - x) + lut(tp, a3 - x));
    if (sec) {
      hi = __vimax3_s32(__vimax3_s32(hi, a0 & m, a1 & m), a2 & m, a3 & m);
      lo = __vimin3_s32(__vimin3_s32(lo, a0, a1), a2, a3);
    }
  }
  if (sec) {
    const int b0 = c[s0.x], b1 = c[-s0.x], b2 = c[s1.x], b3 = c[-s1.x];
    const int b4 = c[s0.y], b5 = c[-s0.y], b6 = c[s1.y], b7 = c[-s1.y];
    sum += 2 * (lut(ts, b0 - x) + lut(ts, b1 - x) + lut(ts, b2 - x) + lut(ts, b3 - x)) + lut(ts, b4 - x) +
           lut(ts, b5 - x) + lut(ts, b6 - x) + lut(ts, b7 - x);
    if (pri) {
      hi = __vimax3_s32(__vimax3_s32(hi, b0 & m, b1 & m), __vimax3_s32(b2 & m, b3 & m, b4 & m),
                        __vimax3_s32(b5 & m, b6 & m, b7 & m));
      lo = __vimin3_s32(__vimin3_s32(lo, b0, b1), __vimin3_s32(b2, b3, b4), __vimin3_s32(b5, b6, b7));
    }
  }
  int y = x + ((8 + sum - (sum < 0)) >> 4);
  if (pri && sec) y = imin(imax(y, lo), hi);
  return y;
}

}  // namespace pf
