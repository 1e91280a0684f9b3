// pf_search.cu - the encoder's CDEF strength search on the GPU.
//
// Follows goav1's cdefSearcher (internal/av1/encoder/cdef_search.go) over a
// trial list: level 1's (:98-110: all 64 packed strengths in the svtPfGI
// order, chroma the same list, row subsampling 1) for pf_cdef_search and the
// learned search, any level's for pf_cdef_search_ex (chroma trials the level
// does not measure, luma rows every subsamplingFactor-th with the SSE scaled
// back).  Trial indices past the list hold kNotATrial, which no selection
// step picks, so the selection over all 64 indices equals finish's over the
// list (:892-899: endGI = len(filterMap)):
//   k_cdef_search   one CTA per 64x64 filter block: the noskip 8x8 list
//                   (computeCDEFList, :410-447), the VeryLarge-padded input
//                   (loadCDEFInput, :479-506), luma directions from the
//                   reconstruction, then for each tested trial the SSE of
//                   the filtered block against the source (searchRow,
//                   :649-745; FilterBlocksU8SubsampledTrusted with row step 1,
//                   cdef/filter_search.go:20-74).  The work is split into
//                   (trial, 8-row group) tasks spread over the warps, so a
//                   block that tests few trials (the learned search) still
//                   keeps every warp busy.  An untested trial gets the
//                   reference's untested-chroma figure (cdefDefaultMSEUV*64,
//                   :669-672) in both planes.
//   k_sel_greedy    finish (:886-945): jointStrengthSearchDual /
//                   searchOneDual (:780-869) for one nb = 1 << cluster index,
//                   all 5*nb greedy and refinement steps inside one launch.
//                   Eight CTAs of a thread-block cluster each own a slice of
//                   the filter blocks (SSE rows in shared memory), compute
//                   partial savings sav[j][k] = sum_i max(0, best_i -
//                   m0[i][j] - m1[i][k]) (the reference's form), and reduce
//                   them through distributed shared memory.
//   k_sel_finish    the RD choice of nb and the per-block preset index.
#include <cooperative_groups.h>
#include <string.h>

#include <vector>

#include "pf_cdef_dev.cuh"
#include "pf_search.cuh"

namespace cg = cooperative_groups;

namespace pf {

constexpr int kLearnedSlices = 4;
constexpr int kTrialsPerSlice = 16;

__global__ void __launch_bounds__(256) k_cdef_search(SearchArgs a) {
  __shared__ uint16_t s_in[kSH * kSW];
  __shared__ __align__(16) uint8_t s_src[64 * 64];
  __shared__ __align__(16) uint8_t s_rec[64 * 64];  // the reconstruction itself (unfiltered trials measure it)
  __shared__ int32_t s_cost[64 * 8];
  __shared__ uint8_t s_dir[64];
  __shared__ int8_t s_ai[64];   // adjustStrength index, -1 for zero variance
  __shared__ int2 s_ofs[12];
  __shared__ uint32_t s_sse[2][64];  // luma; U+V
  __shared__ uint8_t s_list[2][64];  // tested trials, ascending
  __shared__ int s_cnt[2];
  // constrain() of the plane's damping: primary strength k at row k (0..15),
  // secondary strengths 1, 2, 4 at rows 16..18; entry kTab0 is a difference
  // of 0, entries kTab0 -/+ 256 stand for every difference beyond +/-255
  // (both 0).  A row is a copy of the context's table for its strength and
  // shift, two entries in, so its 32-bit words stay aligned.
  constexpr int kTabStride = 520, kTab0 = 257;
  __shared__ __align__(16) int16_t s_tab[19][kTabStride];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int slices = a.slices > 1 ? a.slices : 1;
  const int fb = blockIdx.x / slices, slice = blockIdx.x - fb * slices;
  const int fbr = fb / a.nhfb, fbc = fb - fbr * a.nhfb;
  const int lr = 16 * fbr, lc = 16 * fbc;
  const int nhb = imin(16, a.miCols - lc), nvb = imin(16, a.miRows - lr);
  const int nfb = a.nhfb * a.nvfb;
  uint64_t* m0 = a.mse + (size_t)fb * 64;
  uint64_t* m1 = a.mse + (size_t)nfb * 64 + (size_t)fb * 64;
  const uint64_t listed = fb_listed(a, fb, lr, lc);
  const int count = a.trials.count;
  if (listed == 0) {
    if (tid < 64 && slice == 0) {
      m0[tid] = tid < count ? 0 : (uint64_t)kNotATrial;
      m1[tid] = tid < count ? 0 : (uint64_t)kNotATrial;
    }
    if (tid == 0 && slice == 0) a.skip[fb] = 1;
    return;
  }
  const uint64_t listMask = count >= 64 ? ~0ull : (1ull << count) - 1;
  const uint64_t mask0 = a.tmask ? a.tmask[2 * fb] : listMask;
  const uint64_t mask1 = a.tmask ? a.tmask[2 * fb + 1] : a.trials.uvMask;
  const int ssY = a.trials.ss;
  // The slices this block uses: one per kTrialsPerSlice tested trials (a
  // block with a handful of trials is measured by one CTA, a fallback block
  // by all of its CTAs); the others have nothing to do.
  const int used = imin(slices, 1 + (__popcll(mask0) + __popcll(mask1)) / kTrialsPerSlice);
  if (slice >= used) return;
  if (tid == 0) {
    if (slice == 0) a.skip[fb] = 0;
    // This slice's share of the tested trials: list positions slice,
    // slice + used, ...
    int c0 = 0, c1 = 0, n0 = 0, n1 = 0;
    for (int g = 0; g < 64; g++) {
      if ((mask0 >> g) & 1) {
        if (n0 % used == slice) s_list[0][c0++] = (uint8_t)g;
        n0++;
      }
      if ((mask1 >> g) & 1) {
        if (n1 % used == slice) s_list[1][c1++] = (uint8_t)g;
        n1++;
      }
    }
    s_cnt[0] = c0;
    s_cnt[1] = c1;
  }
  if (tid < 12) s_ofs[tid] = make_int2(dir_off(tid, 0), dir_off(tid, 1));
  if (tid < 128) s_sse[tid >> 6][tid & 63] = 0;
  const int damping = a.damping;
  for (int pli = 0; pli < 3; pli++) {
    const int dec = pli ? 1 : 0;
    const int P = pli ? 1 : 0;
    const int x0 = (lc * 4) >> dec, y0 = (lr * 4) >> dec;
    const int w = (nhb * 4) >> dec, h = (nvb * 4) >> dec;
    const DPlane& rp = a.rec.pl[pli];
    const DPlane& sp = a.src.pl[pli];
    const int planeW = rp.w, planeH = rp.h;
    __syncthreads();  // the previous plane's tasks are done with the buffers
    // A slice with none of the block's tested trials in this plane skips it
    // (the chroma planes share one count); the chroma trials still need the
    // luma directions, which the features kernel left in a.dirs.
    if (s_cnt[P] == 0 && !(pli == 0 && s_cnt[1] > 0 && !a.dirs)) {
      if (pli == 0 && s_cnt[1] > 0 && tid < 64 && ((listed >> tid) & 1)) {
        s_dir[tid] = a.dirs[(size_t)fb * 64 + tid];
        s_ai[tid] = a.ais[(size_t)fb * 64 + tid];
      }
      continue;
    }
    // loadCDEFInput: frame samples where they exist, VeryLarge elsewhere.
    // A row wholly inside the plane whose start is 4-byte aligned is read
    // four samples at a time (w + 16 is a multiple of 4).
    for (int r = warp; r < h + 4; r += 8) {
      const int yy = y0 - 2 + r;
      const bool rowIn = yy >= 0 && yy < planeH;
      const uint8_t* srow = rowIn ? row_ptr<uint8_t>(rp, yy) : nullptr;
      const int xs = x0 - 8;
      if (rowIn && xs >= 0 && xs + w + 16 <= planeW && (((uintptr_t)(srow + xs)) & 3) == 0) {
        const uint32_t* q = reinterpret_cast<const uint32_t*>(srow + xs);
        for (int c4 = lane; c4 < (w + 16) >> 2; c4 += 32) {
          const uint32_t v = q[c4];
          uint16_t* d = &s_in[r * kSW + 4 * c4];
          d[0] = v & 0xff;
          d[1] = (v >> 8) & 0xff;
          d[2] = (v >> 16) & 0xff;
          d[3] = v >> 24;
        }
      } else {
        for (int c = lane; c < w + 16; c += 32) {
          const int xx = xs + c;
          s_in[r * kSW + c] = (rowIn && xx >= 0 && xx < planeW) ? srow[xx] : (uint16_t)kVeryLarge;
        }
      }
    }
    for (int r = warp; r < h; r += 8) {
      const uint8_t* srow = row_ptr<uint8_t>(sp, y0 + r) + x0;
      const uint8_t* rrow = row_ptr<uint8_t>(rp, y0 + r) + x0;
      if ((((uintptr_t)srow | (uintptr_t)rrow) & 3) == 0) {
        for (int c4 = lane; c4 < w >> 2; c4 += 32) {
          reinterpret_cast<uint32_t*>(&s_src[r * 64])[c4] = reinterpret_cast<const uint32_t*>(srow)[c4];
          reinterpret_cast<uint32_t*>(&s_rec[r * 64])[c4] = reinterpret_cast<const uint32_t*>(rrow)[c4];
        }
      } else {
        for (int c = lane; c < w; c += 32) {
          s_src[r * 64 + c] = srow[c];
          s_rec[r * 64 + c] = rrow[c];
        }
      }
    }
    if (pli == 0 && a.dirs) {
      // Directions already found by the features kernel (same arithmetic).
      if (tid < 64 && ((listed >> tid) & 1)) {
        s_dir[tid] = a.dirs[(size_t)fb * 64 + tid];
        s_ai[tid] = a.ais[(size_t)fb * 64 + tid];
      }
    } else if (pli == 0) {
      // Luma directions of the listed blocks, from the reconstruction.
      // A warp takes one direction for 32 blocks (no divergence between
      // the eight direction templates).
      for (int wi = tid; wi < 64 * 8; wi += 256) {
        const int d = wi >> 6, b = wi & 63;
        if ((listed >> b) & 1)
          s_cost[b * 8 + d] = dir_cost8_dev(d, row_ptr<uint8_t>(rp, y0 + (b >> 3) * 8) + x0 + (b & 7) * 8, rp.stride);
      }
      __syncthreads();
      if (tid < 64 && ((listed >> tid) & 1)) {
        int best = 0;
        int32_t bc = s_cost[tid * 8];
        for (int d = 1; d < 8; d++)
          if (s_cost[tid * 8 + d] > bc) {
            best = d;
            bc = s_cost[tid * 8 + d];
          }
        const int32_t var = (bc - s_cost[tid * 8 + ((best + 4) & 7)]) >> 10;
        s_dir[tid] = (uint8_t)best;
        int ai = -1;
        if (var != 0) {
          ai = 0;
          const int32_t v = var >> 6;
          if (v) ai = imin(31 - __clz(v), 12);
        }
        s_ai[tid] = (int8_t)ai;
      }
    }
    const int bl = 3 - dec;
    const int dmp = pli ? damping - 1 : damping;
    if (pli < 2) {  // chroma planes share one damping
      // Rows of 256 32-bit words (entries -255 .. 256 at kTab0 - 255 ..),
      // then entry kTab0 - 256 (a difference below -255) set to 0.
      for (int i = tid; i < 19 * 256; i += 256) {
        const int t = i >> 8, wd = i & 255;
        const int k = t < 16 ? t : (t == 16 ? 1 : (t == 17 ? 2 : 4));
        const uint32_t* src = reinterpret_cast<const uint32_t*>(a.ctab + (size_t)(k * 8 + constrain_shift(k, dmp)) * 512);
        reinterpret_cast<uint32_t*>(&s_tab[t][kTab0 - 255])[wd] = src[wd];
      }
      if (tid < 19) s_tab[tid][kTab0 - 256] = 0;
    }
    __syncthreads();
    const int ngrp = (h + 7) >> 3;
    const int ntask = s_cnt[P] * ngrp;
    // Luma rows every ssY-th (the subsampled search), chroma every row.
    const int step = P ? 1 : ssY;
    for (int task = warp; task < ntask; task += 8) {
      const int g = s_list[P][task / ngrp];
      const int grp = task - (task / ngrp) * ngrp;
      const int packed = P ? a.trials.uv[g] : a.trials.y[g];
      const int pri = packed >> 2;
      int sec = packed & 3;
      if (sec == 3) sec = 4;
      const int16_t* ts = &s_tab[sec == 1 ? 16 : (sec == 2 ? 17 : 18)][kTab0];
      uint32_t sse = 0;
      for (int xx = lane; xx < w; xx += 32) {
        for (int yb = grp * 8; yb < imin(grp * 8 + 8, h); yb += 1 << bl) {
          const int b = ((yb >> bl) << 3) + (xx >> bl);
          if (!((listed >> b) & 1)) continue;
          int strength = pri;
          if (pli == 0 && pri != 0) {
            const int ai = s_ai[b];
            strength = ai < 0 ? 0 : (pri * (4 + ai) + 8) >> 4;
          }
          const bool filt = (strength | sec) != 0;
          const int dir = pri != 0 ? s_dir[b] : 0;
          const int16_t* tp = &s_tab[strength][kTab0];
          const int2 po = s_ofs[dir + 2], q0 = s_ofs[dir + 4], q1 = s_ofs[dir];
          for (int yy = yb; yy < yb + (1 << bl); yy += step) {
            // An unfiltered block keeps the reconstruction (cdefDist8 against
            // recon / the copyFB trial buffer), which below the crop is not
            // the VeryLarge-padded input.
            int v = s_rec[yy * 64 + xx];
            if (filt)
              // The 8-bit trial buffer keeps the low byte (cdef/filter_u8.go:151),
              // which matters only below the crop where the centre is VeryLarge.
              v = (uint8_t)cdef_filter_px_tab8(&s_in[(2 + yy) * kSW + 8 + xx], strength, tp, sec, ts, po, q0, q1);
            const int e = (int)s_src[yy * 64 + xx] - v;
            sse += (uint32_t)(e * e);
          }
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sse += __shfl_xor_sync(0xffffffffu, sse, o);
      if (lane == 0) atomicAdd(&s_sse[P][g], sse);
    }
  }
  __syncthreads();
  if (tid < 64) {
    // Each entry written once: a tested trial by the slice that measured
    // it, the rest by slice 0.
    const uint64_t below = (1ull << tid) - 1;
    const bool t0 = (mask0 >> tid) & 1, t1 = (mask1 >> tid) & 1;
    const bool own0 = t0 && __popcll(mask0 & below) % used == slice;
    const bool own1 = t1 && __popcll(mask1 & below) % used == slice;
    if (tid >= count) {
      if (slice == 0) m0[tid] = m1[tid] = kNotATrial;
    } else {
      // A subsampled luma SSE is scaled back by the row step (searchRow, :722-734).
      if (own0) m0[tid] = (uint64_t)s_sse[0][tid] * (uint64_t)ssY;
      else if (!t0 && slice == 0) m0[tid] = (uint64_t)kUntestedMSE;
      if (own1) m1[tid] = (uint64_t)s_sse[1][tid];
      else if (!t1 && slice == 0) m1[tid] = (uint64_t)kUntestedMSE;
    }
  }
}

// ---- greedy preset selection (finish) ----

struct SelShared {
  unsigned long long part[4096];       // this CTA's partial savings (or column sums)
  unsigned long long col[128];
  unsigned long long candV[2], candSB[2];
  int candI[2];
  unsigned long long redV[kSelThreads / 32];
  int redI[kSelThreads / 32];
  unsigned long long redS[kSelThreads / 32];
  int lev0[8], lev1[8];
  unsigned long long tot;
};

// First maximum wins: larger value, or equal value at a lower index.
__device__ __forceinline__ void argmax_merge(unsigned long long& v, int& i, unsigned long long v2, int i2) {
  if (i == 0x7fffffff || v2 > v || (v2 == v && i2 < i)) {
    v = v2;
    i = i2;
  }
}

// The non-skip filter blocks in order (computeCDEFList's non-empty units):
// a ballot per warp and a running base; returns their count.  All threads
// of the block call it; `wsum` is one int per warp of scratch.
__device__ int compact_blocks(const uint8_t* skip, int nfb, int* list, int* wsum) {
  const int t = threadIdx.x, nw = blockDim.x >> 5;
  int base = 0;
  for (int b0 = 0; b0 < nfb; b0 += blockDim.x) {
    const int fb = b0 + t;
    const bool keep = fb < nfb && !skip[fb];
    const unsigned m = __ballot_sync(0xffffffffu, keep);
    __syncthreads();  // the previous chunk of blocks is done with wsum
    if ((t & 31) == 0) wsum[t >> 5] = __popc(m);
    __syncthreads();
    int off = base;
    for (int w = 0; w < (t >> 5); w++) off += wsum[w];
    off += __popc(m & ((1u << (t & 31)) - 1));
    if (keep) list[off] = fb;
    for (int w = 0; w < nw; w++) base += wsum[w];
  }
  __syncthreads();
  return base;
}

// One cluster per configuration nb = 1 << (blockIdx.x / cluster size); the
// cluster size (16, or 8 where a 16-CTA cluster cannot be placed) is read at
// run time.  kRows: the filter blocks' SSE rows (as 32-bit values; an 8-bit
// 64x64 block's SSE is below 2^28) are copied into shared memory.
template <bool kRows>
__global__ void __launch_bounds__(kSelThreads) k_sel_greedy(SelArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  SelShared& S = *reinterpret_cast<SelShared*>(smem);
  int* s_sb = reinterpret_cast<int*>(smem + sizeof(SelShared));  // [nfb] non-skip blocks
  uint32_t* s_best = reinterpret_cast<uint32_t*>(s_sb + ((a.nfb + 3) & ~3));
  uint32_t* s_min1 = s_best + a.cap;
  uint32_t* s_rows = s_min1 + a.cap;  // [cap][128] when kRows
  cg::cluster_group cl = cg::this_cluster();
  const int CS = (int)cl.num_blocks();
  const int rank = (int)cl.block_rank();
  const int cfg = blockIdx.x / CS;
  const int nb = 1 << cfg;
  const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
  const int n = compact_blocks(a.skip, a.nfb, s_sb, S.redI);
  SelOut* out = a.out;
  if (n == 0) {
    if (rank == 0 && t == 0) {
      for (int g = 0; g < 8; g++) out->lev0[cfg][g] = out->lev1[cfg][g] = 0;
      out->tot[cfg] = 0;
    }
    return;
  }
  const int per = (n + CS - 1) / CS;
  const int i0 = imin(n, rank * per), i1 = imin(n, i0 + per), cnt = i1 - i0;
  const int pairs = 4096 / CS;
  const uint64_t* M0 = a.mse;
  const uint64_t* M1 = a.mse + (size_t)a.nfb * 64;
  auto row = [&](int il, int pl, int j) -> uint32_t {
    if (kRows) return s_rows[il * 128 + pl * 64 + j];
    const int fb = s_sb[i0 + il];
    return (uint32_t)(pl ? M1 : M0)[(size_t)fb * 64 + j];
  };
  if (kRows)
    for (int e = t; e < cnt * 128; e += kSelThreads) {
      const int il = e >> 7, pl = (e >> 6) & 1, j = e & 63;
      const int fb = s_sb[i0 + il];
      s_rows[e] = (uint32_t)(pl ? M1 : M0)[(size_t)fb * 64 + j];
    }
  __syncthreads();
  for (int il = t; il < cnt; il += kSelThreads) {
    uint32_t m = 0xffffffffu;
    for (int k = 0; k < 64; k++) m = min(m, row(il, 1, k));
    s_min1[il] = m;
  }
  if (t < 8) S.lev0[t] = S.lev1[t] = 0;
  __syncthreads();
  const int steps = a.refine ? 5 * nb : nb;
  for (int k = 0; k < steps; k++) {
    const int nbCur = k < nb ? k : nb - 1;
    const int par = k & 1;
    if (nbCur == 0) {
      // First pick: the luma and chroma strengths with the least total SSE.
      if (t < 128) {
        unsigned long long s = 0;
        for (int il = 0; il < cnt; il++) s += row(il, t >> 6, t & 63);
        S.part[t] = s;
      }
      cl.sync();
      if (t < 128) {
        unsigned long long s0 = 0, s1 = 0, s2 = 0, s3 = 0;
        for (int r = 0; r < CS; r += 4) {
          s0 += cl.map_shared_rank(&S.part[0], r)[t];
          s1 += cl.map_shared_rank(&S.part[0], r + 1)[t];
          s2 += cl.map_shared_rank(&S.part[0], r + 2)[t];
          s3 += cl.map_shared_rank(&S.part[0], r + 3)[t];
        }
        S.col[t] = (s0 + s1) + (s2 + s3);
      }
      __syncthreads();
      if (t == 0) {
        int b0 = 0, b1 = 0;
        for (int j = 1; j < 64; j++) {
          if (S.col[j] < S.col[b0]) b0 = j;
          if (S.col[64 + j] < S.col[64 + b1]) b1 = j;
        }
        S.lev0[0] = b0;
        S.lev1[0] = b1;
        S.tot = S.col[b0] + S.col[64 + b1];
      }
      cl.sync();  // every CTA has read the others' column sums
    } else {
      // best_i over the strengths selected so far, and its sum.
      unsigned long long sb = 0;
      for (int il = t; il < cnt; il += kSelThreads) {
        uint32_t best = row(il, 0, S.lev0[0]) + row(il, 1, S.lev1[0]);
        for (int g = 1; g < nbCur; g++) best = min(best, row(il, 0, S.lev0[g]) + row(il, 1, S.lev1[g]));
        s_best[il] = best;
        sb += best;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sb += __shfl_xor_sync(0xffffffffu, sb, o);
      if (lane == 0) S.redS[warp] = sb;
      __syncthreads();
      if (warp == 0) {
        unsigned long long v = lane < kSelThreads / 32 ? S.redS[lane] : 0;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) S.candSB[par] = v;
      }
      // Partial savings of this CTA's blocks: thread t owns (j, k0..k0+7).
      // A block saves below 2^29, so eight blocks sum exactly in 32 bits
      // before joining the 64-bit totals.
      const int j = t >> 3, k0 = (t & 7) * 8;
      unsigned long long acc[8];
      uint32_t acc32[8];
#pragma unroll
      for (int q = 0; q < 8; q++) acc[q] = acc32[q] = 0;
      for (int il0 = 0; il0 < cnt; il0 += 8) {
        const int il1 = imin(cnt, il0 + 8);
        for (int il = il0; il < il1; il++) {
          const uint32_t bi = s_best[il], a0 = row(il, 0, j);
          if (a0 + s_min1[il] >= bi) continue;  // no k can save anything
          const uint32_t rem = bi - a0;
#pragma unroll
          for (int q = 0; q < 8; q++) {
            const uint32_t v = row(il, 1, k0 + q);
            acc32[q] += v < rem ? rem - v : 0u;
          }
        }
#pragma unroll
        for (int q = 0; q < 8; q++) {
          acc[q] += acc32[q];
          acc32[q] = 0;
        }
      }
#pragma unroll
      for (int q = 0; q < 8; q++) S.part[j * 64 + k0 + q] = acc[q];
      cl.sync();
      // Reduce this CTA's slice across the cluster; first maximum wins.
      unsigned long long bv = 0;
      int bi = 0x7fffffff;
      for (int e = rank * pairs + t; e < (rank + 1) * pairs; e += kSelThreads) {
        // Four independent remote reads in flight (CS is a multiple of 4).
        unsigned long long v0 = 0, v1 = 0, v2 = 0, v3 = 0;
        for (int r = 0; r < CS; r += 4) {
          v0 += cl.map_shared_rank(&S.part[0], r)[e];
          v1 += cl.map_shared_rank(&S.part[0], r + 1)[e];
          v2 += cl.map_shared_rank(&S.part[0], r + 2)[e];
          v3 += cl.map_shared_rank(&S.part[0], r + 3)[e];
        }
        argmax_merge(bv, bi, (v0 + v1) + (v2 + v3), e);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long v2 = __shfl_xor_sync(0xffffffffu, bv, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, bi, o);
        argmax_merge(bv, bi, v2, i2);
      }
      if (lane == 0) {
        S.redV[warp] = bv;
        S.redI[warp] = bi;
      }
      __syncthreads();
      if (warp == 0) {
        unsigned long long v = 0;
        int i = 0x7fffffff;
        if (lane < kSelThreads / 32) {
          v = S.redV[lane];
          i = S.redI[lane];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const unsigned long long v2 = __shfl_xor_sync(0xffffffffu, v, o);
          const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
          argmax_merge(v, i, v2, i2);
        }
        if (lane == 0) {
          S.candV[par] = v;
          S.candI[par] = i;
        }
      }
      cl.sync();
      if (warp == 0) {
        // Lane r reads rank r's candidate and partial sum of best_i.
        unsigned long long v = 0, sbr = 0;
        int i = 0x7fffffff;
        if (lane < CS) {
          const SelShared* R = cl.map_shared_rank(&S, lane);
          v = R->candV[par];
          i = R->candI[par];
          sbr = R->candSB[par];
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const unsigned long long v2 = __shfl_xor_sync(0xffffffffu, v, o);
          const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
          argmax_merge(v, i, v2, i2);
          sbr += __shfl_xor_sync(0xffffffffu, sbr, o);
        }
        if (lane == 0) {
          S.lev0[nbCur] = i >> 6;
          S.lev1[nbCur] = i & 63;
          S.tot = sbr - v;
        }
      }
    }
    // Refinement passes drop the oldest pick (jointStrengthSearchDual).
    if (t == 0 && k + 1 >= nb && k + 1 < steps)
      for (int g = 0; g < nb - 1; g++) {
        S.lev0[g] = S.lev0[g + 1];
        S.lev1[g] = S.lev1[g + 1];
      }
    __syncthreads();
  }
  if (rank == 0 && t == 0) {
    for (int g = 0; g < 8; g++) {
      out->lev0[cfg][g] = g < nb ? S.lev0[g] : 0;
      out->lev1[cfg][g] = g < nb ? S.lev1[g] : 0;
    }
    out->tot[cfg] = S.tot;
  }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

// RD choice of nb (finish, :914-931) and the per-block preset index.
__global__ void __launch_bounds__(256) k_sel_finish(SelArgs a, int maxCfg, unsigned long long lambda, uint8_t* fbIndex,
                                                    FinishOut* fo) {
  __shared__ int s_best, s_n;
  const SelOut* st = a.out;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  {
    int c = 0;
    for (int fb = threadIdx.x; fb < a.nfb; fb += blockDim.x) c += !a.skip[fb];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&s_n, c);
  }
  __syncthreads();
  const int n = s_n;
  if (threadIdx.x == 0) {
    unsigned long long bestTot = 1ull << 63;
    int best = 0;
    for (int c = 0; c <= maxCfg; c++) {
      const int nb = 1 << c;
      const long long rate = (long long)(n * c + nb * 6 * 2) << 9;
      const unsigned long long cost =
          (unsigned long long)((rate * (long long)lambda + (1 << 8)) >> 9) + ((st->tot[c] * 16ull) << 7);
      if (cost < bestTot) {
        bestTot = cost;
        best = c;
      }
    }
    s_best = best;
    if (blockIdx.x == 0) {
      fo->bits = best;
      fo->cost = bestTot;
      for (int j = 0; j < (1 << best); j++) {
        fo->ys[j] = st->lev0[best][j];
        fo->uvs[j] = a.uvFromY ? st->lev0[best][j] : st->lev1[best][j];
      }
    }
  }
  __syncthreads();
  const int c = s_best, nb = 1 << c;
  const uint64_t* M0 = a.mse;
  const uint64_t* M1 = a.mse + (size_t)a.nfb * 64;
  for (int fb = blockIdx.x * blockDim.x + threadIdx.x; fb < a.nfb; fb += gridDim.x * blockDim.x) {
    if (a.skip[fb]) {
      fbIndex[fb] = 0;
      continue;
    }
    int bg = 0;
    unsigned long long bm = 1ull << 63;
    for (int g = 0; g < nb; g++) {
      const int uvg = a.uvFromY ? st->lev0[c][g] : st->lev1[c][g];
      const unsigned long long v = M0[(size_t)fb * 64 + st->lev0[c][g]] + M1[(size_t)fb * 64 + uvg];
      if (v < bm) {
        bg = g;
        bm = v;
      }
    }
    fbIndex[fb] = (uint8_t)bg;
  }
}

size_t sel_smem_bytes(int nfb, bool rows) {
  const int cap = (nfb + kSelMinCluster - 1) / kSelMinCluster;
  return sizeof(SelShared) + (size_t)((nfb + 3) & ~3) * 4 + (size_t)cap * 8 + (rows ? (size_t)cap * 512 : 0);
}

cudaError_t launch_search(const SearchArgs& a, cudaStream_t st) {
  k_cdef_search<<<a.nhfb * a.nvfb * (a.slices > 1 ? a.slices : 1), 256, 0, st>>>(a);
  return cudaGetLastError();
}

// Launches k_sel_greedy with 16-CTA clusters when the device can place one
// with this much shared memory, else with 8-CTA clusters.
template <bool kRows>
static cudaError_t launch_greedy(const SelArgs& s, int maxCfg, size_t bytes, cudaStream_t st) {
  const void* fn = (const void*)k_sel_greedy<kRows>;
  // The attributes and the cluster size are settled once per device and
  // shared-memory size (host queries cost more than the short launches).
  static thread_local int lastDev = -1;
  static thread_local size_t lastBytes = 0;
  static thread_local int lastCs = 0;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev == lastDev && bytes <= lastBytes && lastCs) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = lastCs;
    attr[0].val.clusterDim.y = attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(lastCs * (maxCfg + 1));
    cfg.blockDim = dim3(kSelThreads);
    cfg.dynamicSmemBytes = bytes;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_sel_greedy<kRows>, s);
  }
  cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e != cudaSuccess) return e;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  cudaLaunchConfig_t cfg = {};
  cfg.blockDim = dim3(kSelThreads);
  cfg.dynamicSmemBytes = bytes;
  cfg.stream = st;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int cs = kSelMaxCluster;
  for (; cs > kSelMinCluster; cs >>= 1) {
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3(cs * (maxCfg + 1));
    int nclusters = 0;
    if (cudaOccupancyMaxActiveClusters(&nclusters, fn, &cfg) == cudaSuccess && nclusters >= 1) break;
    cudaGetLastError();  // a refused query leaves no sticky error
  }
  attr[0].val.clusterDim.x = cs;
  attr[0].val.clusterDim.y = attr[0].val.clusterDim.z = 1;
  cfg.gridDim = dim3(cs * (maxCfg + 1));
  e = cudaLaunchKernelEx(&cfg, k_sel_greedy<kRows>, s);
  if (e == cudaSuccess) {
    lastDev = dev;
    lastBytes = bytes;
    lastCs = cs;
  }
  return e;
}

cudaError_t launch_select(SelArgs s, int maxCfg, unsigned long long lambda, uint8_t* fbIndex, FinishOut* fo,
                          cudaStream_t st) {
  s.cap = (s.nfb + kSelMinCluster - 1) / kSelMinCluster;
  const bool rows = sel_smem_bytes(s.nfb, true) <= kSelMaxSmem;
  const size_t bytes = sel_smem_bytes(s.nfb, rows);
  if (bytes > kSelMaxSmem) return cudaErrorInvalidValue;
  const cudaError_t e = rows ? launch_greedy<true>(s, maxCfg, bytes, st) : launch_greedy<false>(s, maxCfg, bytes, st);
  if (e != cudaSuccess) return e;
  k_sel_finish<<<imax(1, (s.nfb + 255) / 256), 256, 0, st>>>(s, maxCfg, lambda, fbIndex, fo);
  return cudaGetLastError();
}

}  // namespace pf

using namespace pf;

// ---------------------------------------------------------------------------
// Host side: the search entry points.  Scratch comes from a cache the context
// keeps (grown, never shrunk); host frames are staged like pf_frame_apply's.

void* pf_internal_search_scratch(pf_ctx* c, size_t bytes);  // pf_api.cu
void* pf_internal_stream(pf_ctx* c);
cudaEvent_t* pf_internal_events(pf_ctx* c);  // pf_api.cu: null unless the context times stages
const int16_t* pf_internal_ctab(pf_ctx* c);  // pf_api.cu
void* pf_internal_pinned(pf_ctx* c, size_t bytes);
void* pf_internal_cached_upload(pf_ctx* c, const void* host, size_t bytes, size_t extra, cudaStream_t st,
                                int* changed);
int pf_internal_wait(pf_ctx* c, void* stream);  // pf_api.cu: blocking or bounded by the context's deadline

static void* stage_frame(const pf_frame* f, void* dst, int64_t* strides, cudaStream_t st, cudaError_t* e) {
  size_t off = 0;
  for (int p = 0; p < 3; p++) {
    strides[p] = ((int64_t)f->plane[p].alloc_width + 255) & ~(int64_t)255;
    off += (size_t)strides[p] * f->plane[p].alloc_height;
  }
  if (!dst) return (void*)off;
  uint8_t* base = (uint8_t*)dst;
  for (int p = 0; p < 3 && *e == cudaSuccess; p++) {
    *e = cudaMemcpy2DAsync(base, strides[p], f->plane[p].data, f->plane[p].stride, f->plane[p].alloc_width,
                           f->plane[p].alloc_height, cudaMemcpyHostToDevice, st);
    base += (size_t)strides[p] * f->plane[p].alloc_height;
  }
  return dst;
}

static DFrame search_dframe(const pf_frame* f, uint8_t* const* ptrs, const int64_t* strides) {
  DFrame d;
  memset(&d, 0, sizeof(d));
  d.width = f->width;
  d.height = f->height;
  d.bd = 8;
  d.ssx = d.ssy = 1;
  for (int p = 0; p < 3; p++) {
    d.pl[p].ptr = ptrs[p];
    d.pl[p].stride = strides[p];
    d.pl[p].w = f->plane[p].width;
    d.pl[p].h = f->plane[p].height;
    d.pl[p].aw = f->plane[p].alloc_width;
    d.pl[p].ah = f->plane[p].alloc_height;
  }
  return d;
}

// Validation, staging and scratch shared by the search entry points.
// Scratch: [staged src | staged rec | noskip | mse | skip | SelOut |
//           FinishOut | fbIndex | caller's extra bytes].
struct Staged {
  SearchArgs a;
  SelArgs s;
  uint8_t* idx;
  FinishOut* fo;
  uint8_t* extra;
  uint8_t* pin;  // page-locked staging: noskip words up, then the results down
  int nfb, maxCfg;
  cudaStream_t st;
  pf_ctx* ctx;
};

static int check_search_frame(const pf_frame* f, const pf_frame* recon) {
  // goav1's searcher works on 8-bit 4:2:0 pictures (SourceFrame420).
  if (f->bit_depth != 8 || f->ss_x != 1 || f->ss_y != 1 || f->mono || f->width != recon->width ||
      f->height != recon->height)
    return PF_ERR_UNSUPPORTED;
  if (f->memory != recon->memory || f->memory > PF_MEM_DEVICE) return PF_ERR_INVALID_ARG;
  for (int p = 0; p < 3; p++) {
    const int w = p ? (recon->width + 1) >> 1 : recon->width, h = p ? (recon->height + 1) >> 1 : recon->height;
    const int aw8 = ((recon->width + 7) & ~7) >> (p ? 1 : 0), ah8 = ((recon->height + 7) & ~7) >> (p ? 1 : 0);
    const pf_plane& pl = f->plane[p];
    if (!pl.data || pl.width != w || pl.height != h || pl.alloc_width < aw8 || pl.alloc_height < ah8 ||
        pl.stride < pl.alloc_width)
      return PF_ERR_SHORT_BUFFER;
  }
  return PF_OK;
}

static void level1_trials(TrialList* t);

// source may be null (features only: the source is never read).
static int stage_search(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                        int damping, int maxCfg, size_t extra, Staged* S) {
  int stt = check_search_frame(recon, recon);
  if (stt == PF_OK && source) stt = check_search_frame(source, recon);
  if (stt != PF_OK) return stt;
  if (damping < 3 || damping > 6) return PF_ERR_INVALID_CDEF;
  const int miCols = ((recon->width + 7) >> 3) << 1, miRows = ((recon->height + 7) >> 3) << 1;
  const int nhfb = (miCols + 15) / 16, nvfb = (miRows + 15) / 16, nfb = nhfb * nvfb;
  if (sel_smem_bytes(nfb, false) > kSelMaxSmem) return PF_ERR_UNSUPPORTED;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  const bool host = recon->memory == PF_MEM_HOST;
  int64_t sS[3] = {0, 0, 0}, rS[3];
  cudaError_t e = cudaSuccess;
  const size_t srcBytes = host && source ? (size_t)stage_frame(source, nullptr, sS, st, &e) : 0;
  const size_t recBytes = host ? (size_t)stage_frame(recon, nullptr, rS, st, &e) : 0;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  const size_t oSrc = off; off += al(srcBytes);
  const size_t oRec = off; off += al(recBytes);
  const size_t oNs = off; off += al((size_t)nfb * 8);
  const size_t oMse = off; off += al((size_t)2 * nfb * 64 * 8);
  const size_t oSkip = off; off += al(nfb);
  const size_t oSel = off; off += al(sizeof(SelOut));
  const size_t oFin = off; off += al(sizeof(FinishOut));
  const size_t oIdx = off; off += al(nfb);
  const size_t oExtra = off; off += al(extra);
  uint8_t* base = (uint8_t*)pf_internal_search_scratch(ctx, off);
  if (!base) return PF_ERR_DEVICE;
  uint8_t* sp[3] = {nullptr, nullptr, nullptr};
  uint8_t* rpp[3];
  if (host) {
    if (source) stage_frame(source, base + oSrc, sS, st, &e);
    stage_frame(recon, base + oRec, rS, st, &e);
    size_t o1 = 0, o2 = 0;
    for (int p = 0; p < 3; p++) {
      if (source) {
        sp[p] = base + oSrc + o1;
        o1 += (size_t)sS[p] * source->plane[p].alloc_height;
      }
      rpp[p] = base + oRec + o2;
      o2 += (size_t)rS[p] * recon->plane[p].alloc_height;
    }
  } else {
    for (int p = 0; p < 3; p++) {
      if (source) {
        sp[p] = (uint8_t*)source->plane[p].data;
        sS[p] = source->plane[p].stride;
      }
      rpp[p] = (uint8_t*)recon->plane[p].data;
      rS[p] = recon->plane[p].stride;
    }
  }
  // The noskip words may live in host or device memory: copy them into the
  // scratch either way; host words go through page-locked staging so the
  // copy does not hold the host.
  // One page-locked block for the call (requested once, so it never moves
  // while a copy is queued): the noskip words, then the selection results.
  uint8_t* pin = (uint8_t*)pf_internal_pinned(ctx, al((size_t)nfb * 8) + al(sizeof(FinishOut)) + al(nfb));
  if (!pin) return PF_ERR_DEVICE;
  S->pin = pin;
  const uint8_t* ns = nullptr;
  if (noskip && e == cudaSuccess) {
    cudaPointerAttributes at;
    const bool dev = cudaPointerGetAttributes(&at, noskip) == cudaSuccess &&
                     (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    if (dev) {
      e = cudaMemcpyAsync(base + oNs, noskip, (size_t)nfb * 8, cudaMemcpyDeviceToDevice, st);
    } else {
      memcpy(pin, noskip, (size_t)nfb * 8);
      e = cudaMemcpyAsync(base + oNs, pin, (size_t)nfb * 8, cudaMemcpyHostToDevice, st);
    }
    ns = base + oNs;
  }
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  SearchArgs& a = S->a;
  a.src = source ? search_dframe(source, sp, sS) : search_dframe(recon, rpp, rS);
  a.rec = search_dframe(recon, rpp, rS);
  a.noskip = ns;
  a.tmask = nullptr;
  a.miCols = miCols;
  a.miRows = miRows;
  a.nhfb = nhfb;
  a.nvfb = nvfb;
  a.damping = damping;
  a.mse = (uint64_t*)(base + oMse);
  a.skip = base + oSkip;
  a.dirs = nullptr;
  a.ais = nullptr;
  a.ctab = pf_internal_ctab(ctx);
  a.slices = 1;
  level1_trials(&a.trials);
  SelArgs& s = S->s;
  s.mse = a.mse;
  s.skip = a.skip;
  s.nfb = nfb;
  s.cap = 0;
  s.refine = 1;
  s.uvFromY = 0;
  s.out = (SelOut*)(base + oSel);
  S->idx = base + oIdx;
  S->fo = (FinishOut*)(base + oFin);
  S->extra = base + oExtra;
  S->nfb = nfb;
  S->maxCfg = maxCfg;
  S->st = st;
  S->ctx = ctx;
  return PF_OK;
}

// The level-1 list (cdef_search.go:98-110).
static void level1_trials(TrialList* t) {
  memset(t, 0, sizeof(*t));
  for (int g = 0; g < 64; g++) t->y[g] = t->uv[g] = (int8_t)trial_strength(g);
  t->uvMask = ~0ull;
  t->count = 64;
  t->ss = 1;
}

static int search_damping(const pf_cdef_search_params* params) {
  return params->damping ? params->damping : 3 + (params->qindex >> 6);
}

static int search_max_cfg(const pf_cdef_search_params* params) {
  return params->max_presets >= 8 ? 3 : params->max_presets >= 4 ? 2 : params->max_presets >= 2 ? 1 : 0;
}

// Search (with S.a.tmask already set by the caller, or null), selection,
// results to the host.
static int search_finish(Staged& S, const pf_cdef_search_params* params, uint64_t* mse_out, uint8_t* fb_index_out,
                         pf_cdef_search_result* result, cudaEvent_t* ev = nullptr) {
  const cudaStream_t st = S.st;
  if (launch_search(S.a, st) != cudaSuccess) return PF_ERR_DEVICE;
  if (ev && cudaEventRecord(ev[3], st) != cudaSuccess) return PF_ERR_DEVICE;
  if (launch_select(S.s, S.maxCfg, (unsigned long long)params->lambda, S.idx, S.fo, st) != cudaSuccess)
    return PF_ERR_DEVICE;
  if (ev && cudaEventRecord(ev[4], st) != cudaSuccess) return PF_ERR_DEVICE;
  // The small results come back through the page-locked block (a pageable
  // destination would make each copy a staged, synchronous one).
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  uint8_t* pfo = S.pin + al((size_t)S.nfb * 8);
  uint8_t* pidx = pfo + al(sizeof(FinishOut));
  if (cudaMemcpyAsync(pfo, S.fo, sizeof(FinishOut), cudaMemcpyDeviceToHost, st) != cudaSuccess) return PF_ERR_DEVICE;
  if (mse_out &&
      cudaMemcpyAsync(mse_out, S.a.mse, (size_t)2 * S.nfb * 64 * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PF_ERR_DEVICE;
  if (fb_index_out && cudaMemcpyAsync(pidx, S.idx, S.nfb, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PF_ERR_DEVICE;
  const int w = pf_internal_wait(S.ctx, st);
  if (w != PF_OK) return w;
  FinishOut fo;
  memcpy(&fo, pfo, sizeof(fo));
  if (fb_index_out) memcpy(fb_index_out, pidx, S.nfb);
  if (result) {
    memset(result, 0, sizeof(*result));
    result->bits = (uint8_t)fo.bits;
    result->strength_count = (uint8_t)(1 << fo.bits);
    // Presets map back through the luma list, chroma's too (finish,
    // cdef_search.go:937-940).
    for (int j = 0; j < (1 << fo.bits); j++) {
      result->y_strength[j] = (uint8_t)S.a.trials.y[fo.ys[j]];
      result->uv_strength[j] = (uint8_t)S.a.trials.y[fo.uvs[j]];
    }
    result->cost = (double)fo.cost;
  }
  return PF_OK;
}

extern "C" int pf_cdef_search(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                              const pf_cdef_search_params* params, uint64_t* mse_out, uint8_t* fb_index_out,
                              pf_cdef_search_result* result) {
  if (!ctx || !source || !recon || !params) return PF_ERR_INVALID_ARG;
  Staged S;
  const int stt = stage_search(ctx, source, recon, noskip, search_damping(params), search_max_cfg(params), 0, &S);
  if (stt != PF_OK) return stt;
  return search_finish(S, params, mse_out, fb_index_out, result);
}

extern "C" int pf_cdef_search_ex(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                                 const pf_cdef_search_params* params, const pf_cdef_search_ctrls* ctrls,
                                 uint64_t* mse_out, uint8_t* fb_index_out, pf_cdef_search_result* result) {
  if (!ctx || !source || !recon || !params || !ctrls) return PF_ERR_INVALID_ARG;
  if (ctrls->count < 1 || ctrls->count > PF_CDEF_MAX_TRIALS || ctrls->subsampling < 1) return PF_ERR_INVALID_ARG;
  TrialList t;
  memset(&t, 0, sizeof(t));
  for (int g = 0; g < ctrls->count; g++) {
    if (ctrls->y[g] < 0 || ctrls->y[g] > 63 || ctrls->uv[g] < -1 || ctrls->uv[g] > 63) return PF_ERR_INVALID_CDEF;
    t.y[g] = ctrls->y[g];
    t.uv[g] = ctrls->uv[g];
    if (ctrls->uv[g] >= 0) t.uvMask |= 1ull << g;
  }
  t.count = ctrls->count;
  t.ss = ctrls->subsampling < 4 ? ctrls->subsampling : 4;  // BLOCK_8X8 caps the luma step (searchRow, :694-699)
  Staged S;
  const int stt = stage_search(ctx, source, recon, noskip, search_damping(params), search_max_cfg(params), 0, &S);
  if (stt != PF_OK) return stt;
  S.a.trials = t;
  S.s.uvFromY = ctrls->uv_from_y ? 1 : 0;
  return search_finish(S, params, mse_out, fb_index_out, result);
}

// ---------------------------------------------------------------------------
// Search controls per level and the picture plan (host logic).

extern "C" int pf_cdef_search_level_rtc(int32_t islice, int32_t screen) {
  // svtRTCCDEFSearchLevel (cdef_search.go:208-221).
  if (islice) return 5;
  return screen ? 7 : 8;
}

namespace {
// One level's controls: first- and second-pass luma and chroma lists and the
// flags updateOnRefInfo and the plan read (svtCDEFSearchCtrls,
// cdef_search.go:55-70, filled as setSVTCDEFSearchControls does, :72-202).
struct LevelCtrls {
  bool enabled = false, useRef = false, bestRef = false, skipDetector = false, uvFromY = false;
  int first = 0, second = 0, ss = 1;
  int8_t fs1[64] = {}, fs2[64] = {}, uv1[64] = {}, uv2[64] = {};
  int predY = 0;
};

// The first-pass primaries of levels 1-8 (indices into svtPfGI, p * 4).
const int8_t* level_primaries(int level, int* n) {
  static const int8_t l1[16] = {0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15};
  static const int8_t l2[12] = {0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14};
  static const int8_t l3[5] = {0, 4, 8, 12, 15};
  static const int8_t l45[3] = {0, 7, 15};
  static const int8_t l678[2] = {0, 15};
  switch (level) {
    case 1: *n = 16; return l1;
    case 2: *n = 12; return l2;
    case 3: *n = 5; return l3;
    case 4:
    case 5: *n = 3; return l45;
    default: *n = 2; return l678;
  }
}

LevelCtrls level_ctrls(int level, bool isBase, bool notHighest) {
  LevelCtrls c;
  c.enabled = true;
  int n;
  const int8_t* pri = level_primaries(level, &n);
  c.first = n;
  for (int i = 0; i < n; i++) c.fs1[i] = c.uv1[i] = (int8_t)(4 * pri[i]);
  if (level <= 4) {
    // Second pass: each first-pass strength's three secondaries.
    c.second = 3 * n;
    for (int i = 0; i < n; i++)
      for (int j = 1; j < 4; j++) c.fs2[3 * i + j - 1] = (int8_t)(c.fs1[i] + j);
    for (int i = 0; i < c.second; i++) c.uv2[i] = level == 1 ? c.fs2[i] : (int8_t)-1;
    return c;
  }
  // Levels 5-8: secondary 2 of each first-pass strength, chroma untested there.
  c.second = n;
  for (int i = 0; i < n; i++) {
    c.fs2[i] = (int8_t)(c.fs1[i] + 2);
    c.uv2[i] = -1;
  }
  if (level == 5) {
    c.bestRef = !notHighest;
    return c;
  }
  if (level == 8) c.uv1[0] = c.uv1[1] = -1;
  c.uv1[2] = -1;
  c.ss = 4;
  if (level == 6) c.bestRef = !notHighest;
  if (level == 7) {
    c.useRef = !notHighest;
    c.bestRef = !isBase;
    c.skipDetector = !isBase;
  }
  if (level == 8) {
    c.useRef = !isBase;
    c.bestRef = !isBase;
    c.uvFromY = true;
    for (int i = 0; i < c.first; i++) c.uv1[i] = -1;
    for (int i = 0; i < c.second; i++) c.uv2[i] = -1;
  }
  return c;
}

// updateOnRefInfo (cdef_search.go:237-272): false when CDEF turns off.
bool on_ref_info(LevelCtrls& c, const pf_cdef_ref_strengths& ref) {
  if (c.useRef) {
    int lo = 63, hi = 0;
    for (int i = 0; i < ref.count; i++) {
      lo = ref.y[i] < lo ? ref.y[i] : lo;
      hi = ref.y[i] > hi ? ref.y[i] : hi;
    }
    c.predY = (lo + hi) / 2 < 63 ? (lo + hi) / 2 : 63;
    c.first = c.second = 0;
    return c.predY != 0;
  }
  if (c.bestRef) {
    c.first = 1;
    c.second = 0;
    if ((int8_t)ref.y[0] != c.fs1[0]) c.fs1[c.first++] = (int8_t)ref.y[0];
    if ((int8_t)ref.uv[0] == c.uv1[0]) c.uv1[0] = c.uv1[1] = -1;
    return c.first != 1;
  }
  return true;
}
}  // namespace

extern "C" int pf_cdef_plan_picture(int32_t level, int32_t islice, int32_t is_base, int32_t not_highest_layer,
                                    const pf_cdef_ref_strengths* ref, int32_t ref_skip_percent, pf_cdef_plan* plan) {
  if (!plan) return PF_ERR_INVALID_ARG;
  if (level == 9) return PF_ERR_UNSUPPORTED;
  if (level < 0 || level > 9) return PF_ERR_INVALID_ARG;
  memset(plan, 0, sizeof(*plan));
  if (level == 0) return PF_OK;
  LevelCtrls c = level_ctrls(level, is_base != 0, not_highest_layer != 0);
  bool on = c.enabled;
  // planSVTCDEF (cdef_frame.go:34-54): on inter pictures, the skip detector,
  // else the reference's strengths.
  if (!islice) {
    if (ref_skip_percent > 75 && c.skipDetector) {
      on = false;
    } else if (c.useRef || c.bestRef) {
      if (!ref || ref->count < 1 || ref->count > 8) return PF_ERR_INVALID_ARG;
      on = on_ref_info(c, *ref);
    }
  }
  plan->on = on;
  plan->search = on && !c.useRef;
  if (on && c.useRef) plan->y_strength = (uint8_t)c.predY;  // predUVF is 0
  pf_cdef_search_ctrls& t = plan->ctrls;
  t.count = c.first + c.second;
  for (int g = 0; g < t.count; g++) {
    t.y[g] = g < c.first ? c.fs1[g] : c.fs2[g - c.first];
    t.uv[g] = g < c.first ? c.uv1[g] : c.uv2[g - c.first];
  }
  t.subsampling = c.ss;
  t.uv_from_y = c.uvFromY;
  return PF_OK;
}

// Host or device bytes into a host vector.
static bool read_small(const uint8_t* p, size_t n, std::vector<uint8_t>* out) {
  out->resize(n);
  cudaPointerAttributes at;
  const bool dev = cudaPointerGetAttributes(&at, p) == cudaSuccess &&
                   (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
  cudaGetLastError();
  if (!dev) {
    memcpy(out->data(), p, n);
    return true;
  }
  return cudaMemcpy(out->data(), p, n, cudaMemcpyDeviceToHost) == cudaSuccess;
}

extern "C" int pf_cdef_apply(pf_ctx* ctx, const pf_frame* recon, const uint8_t* noskip,
                             const pf_cdef_search_params* params, const pf_cdef_search_result* result,
                             const uint8_t* fb_index) {
  if (!ctx || !recon || !params || !result) return PF_ERR_INVALID_ARG;
  const int stt = check_search_frame(recon, recon);
  if (stt != PF_OK) return stt;
  if (result->bits > 3) return PF_ERR_INVALID_CDEF;
  const int count = 1 << result->bits;
  // cdef_apply.go:262-271: nothing to do when every strength is zero.
  bool zero = true;
  for (int i = 0; i < count; i++)
    if (result->y_strength[i] || result->uv_strength[i]) zero = false;
  if (zero) return PF_OK;
  const int ucols = (recon->width + 63) / 64, urows = (recon->height + 63) / 64, n = ucols * urows;
  std::vector<uint8_t> ns, idx, read(n, 1), index(n, 0);
  if (noskip && !read_small(noskip, (size_t)n * 8, &ns)) return PF_ERR_DEVICE;
  if (fb_index && !read_small(fb_index, n, &idx)) return PF_ERR_DEVICE;
  // cdef_apply.go:202-235 (markFromLoopFilterMap, noskip-grid branch): a
  // unit is coded, with its searched index, when an in-frame 8x8 block of it
  // carries residual.
  const int cols8 = (recon->width + 7) >> 3, rows8 = (recon->height + 7) >> 3;
  for (int uy = 0; uy < urows; uy++)
    for (int ux = 0; ux < ucols; ux++) {
      const int u = uy * ucols + ux;
      if (noskip) {
        uint64_t inFrame = 0, word = 0;
        for (int by = 0; by < 8 && uy * 8 + by < rows8; by++)
          for (int bx = 0; bx < 8 && ux * 8 + bx < cols8; bx++) inFrame |= 1ull << (by * 8 + bx);
        for (int b = 0; b < 8; b++) word |= (uint64_t)ns[(size_t)u * 8 + b] << (8 * b);
        read[u] = (word & inFrame) != 0;
      }
      index[u] = read[u] && fb_index ? idx[u] : 0;
    }
  pf_frame_side side;
  memset(&side, 0, sizeof(side));
  side.stages = PF_STAGE_CDEF;
  side.side_memory = PF_MEM_HOST;
  pf_cdef& c = side.cdef;
  c.damping = (uint8_t)search_damping(params);
  c.bits = result->bits;
  c.strength_count = (uint8_t)count;
  memcpy(c.y_strength, result->y_strength, 8);
  memcpy(c.uv_strength, result->uv_strength, 8);
  c.index = index.data();
  c.read = read.data();
  c.index_stride = ucols;
  c.index_rows = urows;
  c.noskip = noskip ? ns.data() : nullptr;
  const int r = pf_frame_apply(ctx, recon, &side, nullptr, nullptr);
  if (r != PF_OK) return r;
  return pf_sync(ctx);
}

extern "C" int pf_cdef_features(pf_ctx* ctx, const pf_frame* recon, const uint8_t* noskip, int32_t qindex,
                                int32_t damping, float* features) {
  if (!ctx || !recon || !features) return PF_ERR_INVALID_ARG;
  if (qindex < 0 || qindex > 255) return PF_ERR_INVALID_ARG;
  const int dmp = damping ? damping : 3 + (qindex >> 6);
  Staged S;
  const int miCols = ((recon->width + 7) >> 3) << 1, miRows = ((recon->height + 7) >> 3) << 1;
  const int nfb = ((miCols + 15) / 16) * ((miRows + 15) / 16);
  const size_t xBytes = (size_t)nfb * PF_MLP_FEATURES * sizeof(float);
  const int stt = stage_search(ctx, nullptr, recon, noskip, dmp, 0, xBytes, &S);
  if (stt != PF_OK) return stt;
  float* X = (float*)S.extra;
  if (launch_features(S.a, qindex, X, true, S.st) != cudaSuccess) return PF_ERR_DEVICE;
  if (cudaMemcpyAsync(features, X, xBytes, cudaMemcpyDeviceToHost, S.st) != cudaSuccess) return PF_ERR_DEVICE;
  return pf_internal_wait(ctx, S.st);
}

extern "C" int pf_cdef_search_learned(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon,
                                      const uint8_t* noskip, const pf_cdef_search_params* params,
                                      const pf_cdef_mlp* model, float threshold, int32_t candidates,
                                      int32_t flags, uint64_t* mse_out, uint8_t* fb_index_out,
                                      pf_cdef_search_result* result, pf_cdef_learned_stats* stats) {
  if (!ctx || !source || !recon || !params || !model) return PF_ERR_INVALID_ARG;
  if (flags & ~PF_LEARNED_REFINE) return PF_ERR_INVALID_ARG;
  if (candidates < 1 || candidates > 8 || !(threshold >= 0.f)) return PF_ERR_INVALID_ARG;
  if (params->qindex < 0 || params->qindex > 255) return PF_ERR_INVALID_ARG;
  const int miCols = ((recon->width + 7) >> 3) << 1, miRows = ((recon->height + 7) >> 3) << 1;
  const int nfb = ((miCols + 15) / 16) * ((miRows + 15) / 16);
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  const size_t xBytes = al((size_t)nfb * PF_MLP_FEATURES * sizeof(float));
  const size_t mBytes = al((size_t)nfb * 2 * sizeof(uint64_t));
  const size_t dBytes = al((size_t)nfb * 128);
  Staged S;
  const int stt = stage_search(ctx, source, recon, noskip, search_damping(params), search_max_cfg(params),
                               xBytes + mBytes + dBytes, &S);
  if (stt != PF_OK) return stt;
  float* X = (float*)S.extra;
  uint64_t* masks = (uint64_t*)(S.extra + xBytes);
  int changed = 0;
  uint8_t* mbase = (uint8_t*)pf_internal_cached_upload(ctx, model, sizeof(pf_cdef_mlp), mlp_expanded_bytes(), S.st,
                                                       &changed);
  if (!mbase) return PF_ERR_DEVICE;
  const pf_cdef_mlp* dmodel = (const pf_cdef_mlp*)mbase;
  float* W = (float*)(mbase + ((sizeof(pf_cdef_mlp) + 255) & ~(size_t)255));
  S.a.dirs = S.extra + xBytes + mBytes;
  S.a.ais = (int8_t*)(S.extra + xBytes + mBytes + (size_t)nfb * 64);
  // With stage timing on: events around features, network, trial search
  // and selection (read into stats->stage_ms).
  cudaEvent_t* ev = stats ? pf_internal_events(ctx) : nullptr;
  if (ev && cudaEventRecord(ev[0], S.st) != cudaSuccess) return PF_ERR_DEVICE;
  if (launch_features(S.a, params->qindex, X, false, S.st) != cudaSuccess) return PF_ERR_DEVICE;
  if (ev && cudaEventRecord(ev[1], S.st) != cudaSuccess) return PF_ERR_DEVICE;
  if (launch_mlp_masks(dmodel, W, changed != 0, X, nfb, threshold, candidates, masks, S.st) != cudaSuccess)
    return PF_ERR_DEVICE;
  if (ev && cudaEventRecord(ev[2], S.st) != cudaSuccess) return PF_ERR_DEVICE;
  S.a.tmask = masks;
  // A block's tested trials vary from a few to all 64 (a fallback head):
  // four CTAs share each block's list, so the fallback blocks do not set
  // the launch's length alone.
  S.a.slices = kLearnedSlices;
  S.s.refine = (flags & PF_LEARNED_REFINE) ? 1 : 0;
  const int r = search_finish(S, params, mse_out, fb_index_out, result, ev);
  if (r != PF_OK) return r;
  // The statistics are read back after the search (no host wait between the
  // network and the search it steers).
  if (stats) {
    std::vector<uint64_t> hm((size_t)nfb * 2);
    std::vector<uint8_t> skip(nfb);
    if (cudaMemcpy(hm.data(), masks, (size_t)nfb * 16, cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(skip.data(), S.a.skip, nfb, cudaMemcpyDeviceToHost) != cudaSuccess)
      return PF_ERR_DEVICE;
    memset(stats, 0, sizeof(*stats));
    for (int i = 0; i < 4; i++) {
      float ms = -1.f;
      if (ev && cudaEventElapsedTime(&ms, ev[i], ev[i + 1]) != cudaSuccess) {
        ms = -1.f;
        (void)cudaGetLastError();
      }
      stats->stage_ms[i] = ev ? ms : -1.f;
    }
    for (int fb = 0; fb < nfb; fb++) {
      if (skip[fb]) continue;
      stats->blocks++;
      const int c0 = __builtin_popcountll(hm[2 * fb]), c1 = __builtin_popcountll(hm[2 * fb + 1]);
      if (c0 == 64) stats->fallback_luma++;
      if (c1 == 64) stats->fallback_chroma++;
      stats->trials_luma += c0;
      stats->trials_chroma += c1;
    }
  }
  return PF_OK;
}
