// pf_search.cu - the encoder's CDEF strength search on the GPU.
//
// Follows goav1's cdefSearcher (internal/av1/encoder/cdef_search.go) at
// level-1 controls (:98-110: all 64 packed strengths in the svtPfGI order,
// chroma the same list, row subsampling 1):
//   k_cdef_search   one CTA per 64x64 filter block: the noskip 8x8 list
//                   (computeCDEFList, :410-447), the VeryLarge-padded input
//                   (loadCDEFInput, :479-506), luma directions from the
//                   reconstruction, then for each of the 64 trials the SSE of
//                   the filtered block against the source (searchRow,
//                   :649-745; FilterBlocksU8SubsampledTrusted with row step 1,
//                   cdef/filter_search.go:20-74).  Warps own trials, lanes own
//                   pixels, the SSE is a warp reduction.
//   k_sel_*         finish (:886-945): jointStrengthSearchDual / searchOneDual
//                   (:780-869) for nb = 1, 2, 4, 8 as a chain of GPU steps.
//                   sav[j][k] = sum_i max(0, best_i - m0[i][j] - m1[i][k]) is
//                   the reference's savings form; FB chunks add their partial
//                   sums atomically, one CTA picks the argmax.
//   k_sel_finish    the RD choice of nb and the per-block preset index.
#include <string.h>

#include <vector>

#include "pf_cdef_dev.cuh"

namespace pf {

struct SearchArgs {
  DFrame src, rec;          // 8-bit 4:2:0
  const uint8_t* noskip;    // 8 bytes per filter block, or null (all blocks)
  int miCols, miRows, nhfb, nvfb;
  int damping;
  uint64_t* mse;            // [2][nfb][64]
  uint8_t* skip;            // [nfb]
};

// Trial gi -> packed strength (level-1 lists, svtPfGI then pf+1..pf+3).
__host__ __device__ __forceinline__ int trial_strength(int g) {
  if (g < 16) return g * 4;
  const int k = g - 16;
  return (k / 3) * 4 + (k % 3) + 1;
}

// Direction cost of direction D over an 8-bit 8x8 block in global memory.
template <int D>
__device__ __forceinline__ int32_t dir_cost8(const uint8_t* blk, int64_t stride) {
  int32_t p[15];
#pragma unroll
  for (int k = 0; k < 15; k++) p[k] = 0;
#pragma unroll
  for (int i = 0; i < 8; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) {
      const int32_t x = (int32_t)blk[i * stride + j] - 128;
      if (D == 0) p[i + j] += x;
      if (D == 1) p[i + (j >> 1)] += x;
      if (D == 2) p[i] += x;
      if (D == 3) p[3 + i - (j >> 1)] += x;
      if (D == 4) p[7 + i - j] += x;
      if (D == 5) p[3 - (i >> 1) + j] += x;
      if (D == 6) p[j] += x;
      if (D == 7) p[(i >> 1) + j] += x;
    }
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
         (p[0] * p[0] + p[10] * p[10]) * 420 + (p[1] * p[1] + p[9] * p[9]) * 210 + (p[2] * p[2] + p[8] * p[8]) * 140;
}

__device__ int32_t dir_cost8_any(int d, const uint8_t* blk, int64_t stride) {
  switch (d) {
    case 0: return dir_cost8<0>(blk, stride);
    case 1: return dir_cost8<1>(blk, stride);
    case 2: return dir_cost8<2>(blk, stride);
    case 3: return dir_cost8<3>(blk, stride);
    case 4: return dir_cost8<4>(blk, stride);
    case 5: return dir_cost8<5>(blk, stride);
    case 6: return dir_cost8<6>(blk, stride);
    default: return dir_cost8<7>(blk, stride);
  }
}

__global__ void __launch_bounds__(256) k_cdef_search(SearchArgs a) {
  __shared__ uint16_t s_in[kSH * kSW];
  __shared__ uint8_t s_src[64 * 64];
  __shared__ uint8_t s_rec[64 * 64];  // the reconstruction itself (unfiltered trials measure it)
  __shared__ int32_t s_cost[64 * 8];
  __shared__ uint8_t s_dir[64];
  __shared__ int8_t s_ai[64];   // adjustStrength index, -1 for zero variance
  __shared__ int2 s_ofs[12];
  __shared__ uint32_t s_m1[64];  // U+V SSE per trial
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int fb = blockIdx.x;
  const int fbr = fb / a.nhfb, fbc = fb - fbr * a.nhfb;
  const int lr = 16 * fbr, lc = 16 * fbc;
  const int nhb = imin(16, a.miCols - lc), nvb = imin(16, a.miRows - lr);
  const int nfb = a.nhfb * a.nvfb;
  uint64_t* m0 = a.mse + (size_t)fb * 64;
  uint64_t* m1 = a.mse + (size_t)nfb * 64 + (size_t)fb * 64;
  uint64_t word = ~0ull;
  if (a.noskip) {
    word = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) word |= (uint64_t)a.noskip[(size_t)fb * 8 + i] << (8 * i);
  }
  uint64_t listed = 0;
  for (int r = 0; r < imin(a.miRows - lr, 16); r += 2)
    for (int c = 0; c < imin(a.miCols - lc, 16); c += 2) {
      const int b = (r >> 1) * 8 + (c >> 1);
      listed |= word & (1ull << b);
    }
  if (listed == 0) {
    if (tid < 64) {
      m0[tid] = 0;
      m1[tid] = 0;
    }
    if (tid == 0) a.skip[fb] = 1;
    return;
  }
  if (tid == 0) a.skip[fb] = 0;
  if (tid < 12) s_ofs[tid] = make_int2(dir_off(tid, 0), dir_off(tid, 1));
  if (tid < 64) s_m1[tid] = 0;
  const int damping = a.damping;
  for (int pli = 0; pli < 3; pli++) {
    const int dec = pli ? 1 : 0;
    const int x0 = (lc * 4) >> dec, y0 = (lr * 4) >> dec;
    const int w = (nhb * 4) >> dec, h = (nvb * 4) >> dec;
    const DPlane& rp = a.rec.pl[pli];
    const DPlane& sp = a.src.pl[pli];
    const int planeW = rp.w, planeH = rp.h;
    // loadCDEFInput: frame samples where they exist, VeryLarge elsewhere.
    for (int r = warp; r < h + 4; r += 8) {
      const int yy = y0 - 2 + r;
      const bool rowIn = yy >= 0 && yy < planeH;
      const uint8_t* srow = rowIn ? row_ptr<uint8_t>(rp, yy) : nullptr;
      for (int c = lane; c < w + 16; c += 32) {
        const int xx = x0 - 8 + c;
        s_in[r * kSW + c] = (rowIn && xx >= 0 && xx < planeW) ? srow[xx] : (uint16_t)kVeryLarge;
      }
    }
    for (int r = warp; r < h; r += 8)
      for (int c = lane; c < w; c += 32) {
        s_src[r * 64 + c] = row_ptr<uint8_t>(sp, y0 + r)[x0 + c];
        s_rec[r * 64 + c] = row_ptr<uint8_t>(rp, y0 + r)[x0 + c];
      }
    if (pli == 0) {
      // Luma directions of the listed blocks, from the reconstruction.
      for (int wi = tid; wi < 64 * 8; wi += 256) {
        const int b = wi >> 3, d = wi & 7;
        if ((listed >> b) & 1)
          s_cost[wi] = dir_cost8_any(d, row_ptr<uint8_t>(rp, y0 + (b >> 3) * 8) + x0 + (b & 7) * 8, rp.stride);
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
    __syncthreads();
    const int bl = 3 - dec;
    const int dmp = pli ? damping - 1 : damping;
    for (int t = 0; t < 8; t++) {
      const int g = warp + 8 * t;
      const int packed = trial_strength(g);
      const int pri = packed >> 2;
      int sec = packed & 3;
      if (sec == 3) sec = 4;
      const int secShift = constrain_shift(sec, dmp);
      uint32_t sse = 0;
      for (int yy = 0; yy < h; yy++) {
        for (int xx = lane; xx < w; xx += 32) {
          const int b = ((yy >> bl) << 3) + (xx >> bl);
          if (!((listed >> b) & 1)) continue;
          int strength = pri;
          if (pli == 0 && pri != 0) {
            const int ai = s_ai[b];
            strength = ai < 0 ? 0 : (pri * (4 + ai) + 8) >> 4;
          }
          const uint16_t* c = &s_in[(2 + yy) * kSW + 8 + xx];
          // An unfiltered block keeps the reconstruction (cdefDist8 against
          // recon / the copyFB trial buffer), which below the crop is not the
          // VeryLarge-padded input.
          int v = s_rec[yy * 64 + xx];
          if (strength | sec) {
            const int dir = pri != 0 ? s_dir[b] : 0;
            // The 8-bit trial buffer keeps the low byte (cdef/filter_u8.go:151),
            // which matters only below the crop where the centre is VeryLarge.
            v = (uint8_t)cdef_filter_px(c, strength, constrain_shift(strength, dmp), sec, secShift, s_ofs[dir + 2],
                                        s_ofs[dir + 4], s_ofs[dir], 0);
          }
          const int e = (int)s_src[yy * 64 + xx] - v;
          sse += (uint32_t)(e * e);
        }
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) sse += __shfl_xor_sync(0xffffffffu, sse, o);
      if (lane == 0) {
        if (pli == 0)
          m0[g] = sse;
        else
          s_m1[g] += sse;
      }
    }
    __syncthreads();
  }
  if (tid < 64) m1[tid] = s_m1[tid];
}

// ---- greedy preset selection (finish) ----

struct SelState {
  int lev0[4][8], lev1[4][8];     // per configuration nb = 1 << c
  unsigned long long tot[4];
  unsigned long long sav[4][64 * 64];
  unsigned long long sumBest[4];
  unsigned long long colsum[4][2][64];
};

struct SelArgs {
  const uint64_t* mse;   // [2][nfb][64]
  const int* sb;         // non-skip filter blocks
  int n, nfb;
  SelState* st;
};

// One step's partial sums over a chunk of filter blocks: for nbCur == 0 the
// per-strength column sums, else sumBest and the savings matrix.
__global__ void __launch_bounds__(256) k_sel_accum(SelArgs a, int cfg, int nbCur) {
  SelState* st = a.st;
  const int per = (a.n + gridDim.x - 1) / gridDim.x;
  const int i0 = blockIdx.x * per, i1 = imin(a.n, i0 + per);
  if (i0 >= i1) return;
  const uint64_t* M0 = a.mse;
  const uint64_t* M1 = a.mse + (size_t)a.nfb * 64;
  if (nbCur == 0) {
    if (threadIdx.x < 128) {
      const int pl = threadIdx.x >> 6, j = threadIdx.x & 63;
      const uint64_t* M = pl ? M1 : M0;
      unsigned long long s = 0;
      for (int i = i0; i < i1; i++) s += M[(size_t)a.sb[i] * 64 + j];
      atomicAdd(&st->colsum[cfg][pl][j], s);
    }
    return;
  }
  __shared__ unsigned long long s_best[256];
  __shared__ unsigned long long s_part;
  if (threadIdx.x == 0) s_part = 0;
  __syncthreads();
  unsigned long long localSav[16];
#pragma unroll
  for (int q = 0; q < 16; q++) localSav[q] = 0;
  for (int base = i0; base < i1; base += 256) {
    const int cnt = imin(256, i1 - base);
    __syncthreads();
    if ((int)threadIdx.x < cnt) {
      const int fb = a.sb[base + threadIdx.x];
      unsigned long long best = M0[(size_t)fb * 64 + st->lev0[cfg][0]] + M1[(size_t)fb * 64 + st->lev1[cfg][0]];
      for (int g = 1; g < nbCur; g++) {
        const unsigned long long c = M0[(size_t)fb * 64 + st->lev0[cfg][g]] + M1[(size_t)fb * 64 + st->lev1[cfg][g]];
        if (c < best) best = c;
      }
      s_best[threadIdx.x] = best;
      atomicAdd(&s_part, best);
    }
    __syncthreads();
    for (int ii = 0; ii < cnt; ii++) {
      const int fb = a.sb[base + ii];
      const unsigned long long best = s_best[ii];
#pragma unroll
      for (int q = 0; q < 16; q++) {
        const int p = threadIdx.x + 256 * q;
        const int j = p >> 6, k = p & 63;
        const unsigned long long v0 = M0[(size_t)fb * 64 + j];
        if (v0 >= best) continue;
        const unsigned long long rem = best - v0, v1 = M1[(size_t)fb * 64 + k];
        if (v1 < rem) localSav[q] += rem - v1;
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 16; q++)
    if (localSav[q]) atomicAdd(&st->sav[cfg][threadIdx.x + 256 * q], localSav[q]);
  __syncthreads();
  if (threadIdx.x == 0) atomicAdd(&st->sumBest[cfg], s_part);
}

// Picks the step's winner, clears the accumulators, and shifts the selected
// list left when the next step is a refinement pass.
__global__ void __launch_bounds__(1024) k_sel_pick(SelArgs a, int cfg, int nbCur, int shiftAfter, int nb) {
  SelState* st = a.st;
  __shared__ unsigned long long s_v[1024];
  __shared__ int s_i[1024];
  const int t = threadIdx.x;
  if (a.n == 0) {
    if (t == 0) {
      st->lev0[cfg][nbCur] = st->lev1[cfg][nbCur] = 0;
      st->tot[cfg] = 0;
    }
  } else if (nbCur == 0) {
    if (t == 0) {
      int b0 = 0, b1 = 0;
      for (int j = 1; j < 64; j++) {
        if (st->colsum[cfg][0][j] < st->colsum[cfg][0][b0]) b0 = j;
        if (st->colsum[cfg][1][j] < st->colsum[cfg][1][b1]) b1 = j;
      }
      st->lev0[cfg][0] = b0;
      st->lev1[cfg][0] = b1;
      st->tot[cfg] = st->colsum[cfg][0][b0] + st->colsum[cfg][1][b1];
    }
  } else {
    // argmax over row-major (j, k), the first maximum wins (strict >).
    unsigned long long bv = 0;
    int bi = 0x7fffffff;
    for (int p = t; p < 4096; p += 1024) {
      const unsigned long long v = st->sav[cfg][p];
      if (bi == 0x7fffffff || v > bv) {
        bv = v;
        bi = p;
      }
    }
    s_v[t] = bv;
    s_i[t] = bi;
    __syncthreads();
    for (int o = 512; o > 0; o >>= 1) {
      if (t < o) {
        const unsigned long long v2 = s_v[t + o];
        const int i2 = s_i[t + o];
        if (v2 > s_v[t] || (v2 == s_v[t] && i2 < s_i[t])) {
          s_v[t] = v2;
          s_i[t] = i2;
        }
      }
      __syncthreads();
    }
    if (t == 0) {
      st->lev0[cfg][nbCur] = s_i[0] >> 6;
      st->lev1[cfg][nbCur] = s_i[0] & 63;
      st->tot[cfg] = st->sumBest[cfg] - s_v[0];
    }
  }
  __syncthreads();
  for (int p = t; p < 4096; p += 1024) st->sav[cfg][p] = 0;
  if (t < 128) st->colsum[cfg][t >> 6][t & 63] = 0;
  if (t == 0) st->sumBest[cfg] = 0;
  if (shiftAfter && t == 0) {
    for (int j = 0; j < nb - 1; j++) {
      st->lev0[cfg][j] = st->lev0[cfg][j + 1];
      st->lev1[cfg][j] = st->lev1[cfg][j + 1];
    }
  }
}

struct FinishOut {
  int bits;
  int ys[8], uvs[8];
  unsigned long long cost;
};

// RD choice of nb (finish, :914-931) and the per-block preset index.
__global__ void __launch_bounds__(256) k_sel_finish(SelArgs a, int maxCfg, unsigned long long lambda, uint8_t* fbIndex,
                                                    FinishOut* out) {
  __shared__ int s_best;
  const SelState* st = a.st;
  if (threadIdx.x == 0) {
    unsigned long long bestTot = 1ull << 63;
    int best = 0;
    for (int c = 0; c <= maxCfg; c++) {
      const int nb = 1 << c;
      const long long rate = (long long)(a.n * c + nb * 6 * 2) << 9;
      const unsigned long long cost =
          (unsigned long long)((rate * (long long)lambda + (1 << 8)) >> 9) + ((st->tot[c] * 16ull) << 7);
      if (cost < bestTot) {
        bestTot = cost;
        best = c;
      }
    }
    s_best = best;
    if (blockIdx.x == 0) {
      out->bits = best;
      out->cost = bestTot;
      for (int j = 0; j < (1 << best); j++) {
        out->ys[j] = st->lev0[best][j];
        out->uvs[j] = st->lev1[best][j];
      }
    }
  }
  __syncthreads();
  const int c = s_best, nb = 1 << c;
  const uint64_t* M0 = a.mse;
  const uint64_t* M1 = a.mse + (size_t)a.nfb * 64;
  for (int fb = blockIdx.x * blockDim.x + threadIdx.x; fb < a.nfb; fb += gridDim.x * blockDim.x) fbIndex[fb] = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += gridDim.x * blockDim.x) {
    const int fb = a.sb[i];
    int bg = 0;
    unsigned long long bm = 1ull << 63;
    for (int g = 0; g < nb; g++) {
      const unsigned long long v = M0[(size_t)fb * 64 + st->lev0[c][g]] + M1[(size_t)fb * 64 + st->lev1[c][g]];
      if (v < bm) {
        bg = g;
        bm = v;
      }
    }
    fbIndex[fb] = (uint8_t)bg;
  }
}

// Compacts the non-skip filter blocks into a list (order preserved).
__global__ void k_sel_list(const uint8_t* skip, int nfb, int* sb, int* n) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    int c = 0;
    for (int fb = 0; fb < nfb; fb++)
      if (!skip[fb]) sb[c++] = fb;
    *n = c;
  }
}

}  // namespace pf

using namespace pf;

// ---------------------------------------------------------------------------
// Host side: the search entry point.  Scratch comes from a small cache the
// entry point keeps per process (grown, never shrunk); frames are staged like
// pf_frame_apply's.

namespace {
struct SearchBufs {
  void* p = nullptr;
  size_t n = 0;
};
}  // namespace

void* pf_internal_search_scratch(pf_ctx* c, size_t bytes);  // pf_api.cu
void* pf_internal_stream(pf_ctx* c);

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

extern "C" int pf_cdef_search(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                              const pf_cdef_search_params* params, uint64_t* mse_out, uint8_t* fb_index_out,
                              pf_cdef_search_result* result) {
  if (!ctx || !source || !recon || !params) return PF_ERR_INVALID_ARG;
  // goav1's searcher works on 8-bit 4:2:0 pictures (SourceFrame420).
  if (recon->bit_depth != 8 || source->bit_depth != 8 || recon->ss_x != 1 || recon->ss_y != 1 || recon->mono ||
      source->width != recon->width || source->height != recon->height || source->ss_x != 1 || source->ss_y != 1)
    return PF_ERR_UNSUPPORTED;
  if (recon->memory != source->memory || recon->memory > PF_MEM_DEVICE) return PF_ERR_INVALID_ARG;
  for (int p = 0; p < 3; p++) {
    const int w = p ? (recon->width + 1) >> 1 : recon->width, h = p ? (recon->height + 1) >> 1 : recon->height;
    const int aw8 = ((recon->width + 7) & ~7) >> (p ? 1 : 0), ah8 = ((recon->height + 7) & ~7) >> (p ? 1 : 0);
    for (const pf_frame* f : {source, recon}) {
      const pf_plane& pl = f->plane[p];
      if (!pl.data || pl.width != w || pl.height != h || pl.alloc_width < aw8 || pl.alloc_height < ah8 ||
          pl.stride < pl.alloc_width)
        return PF_ERR_SHORT_BUFFER;
    }
  }
  const int miCols = ((recon->width + 7) >> 3) << 1, miRows = ((recon->height + 7) >> 3) << 1;
  const int nhfb = (miCols + 15) / 16, nvfb = (miRows + 15) / 16, nfb = nhfb * nvfb;
  const int damping = params->damping ? params->damping : 3 + (params->qindex >> 6);
  if (damping < 3 || damping > 6) return PF_ERR_INVALID_CDEF;
  const int maxCfg = params->max_presets >= 8 ? 3 : params->max_presets >= 4 ? 2 : params->max_presets >= 2 ? 1 : 0;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  const bool host = recon->memory == PF_MEM_HOST;
  // Scratch: [staged src | staged rec | noskip | mse | skip | sb list | n | SelState | FinishOut | fbIndex].
  int64_t sS[3], rS[3];
  cudaError_t e = cudaSuccess;
  const size_t srcBytes = host ? (size_t)stage_frame(source, nullptr, sS, st, &e) : 0;
  const size_t recBytes = host ? (size_t)stage_frame(recon, nullptr, rS, st, &e) : 0;
  auto al = [](size_t v) { return (v + 255) & ~(size_t)255; };
  size_t off = 0;
  const size_t oSrc = off; off += al(srcBytes);
  const size_t oRec = off; off += al(recBytes);
  const size_t oNs = off; off += al((size_t)nfb * 8);
  const size_t oMse = off; off += al((size_t)2 * nfb * 64 * 8);
  const size_t oSkip = off; off += al(nfb);
  const size_t oSb = off; off += al((size_t)nfb * 4);
  const size_t oN = off; off += 256;
  const size_t oSel = off; off += al(sizeof(SelState));
  const size_t oFin = off; off += al(sizeof(FinishOut));
  const size_t oIdx = off; off += al(nfb);
  uint8_t* base = (uint8_t*)pf_internal_search_scratch(ctx, off);
  if (!base) return PF_ERR_DEVICE;
  uint8_t* sp[3];
  uint8_t* rpp[3];
  if (host) {
    stage_frame(source, base + oSrc, sS, st, &e);
    stage_frame(recon, base + oRec, rS, st, &e);
    size_t o1 = 0, o2 = 0;
    for (int p = 0; p < 3; p++) {
      sp[p] = base + oSrc + o1;
      rpp[p] = base + oRec + o2;
      o1 += (size_t)sS[p] * source->plane[p].alloc_height;
      o2 += (size_t)rS[p] * recon->plane[p].alloc_height;
    }
  } else {
    for (int p = 0; p < 3; p++) {
      sp[p] = (uint8_t*)source->plane[p].data;
      sS[p] = source->plane[p].stride;
      rpp[p] = (uint8_t*)recon->plane[p].data;
      rS[p] = recon->plane[p].stride;
    }
  }
  // The noskip words may live in host or device memory: copy them into the
  // scratch either way (cudaMemcpyDefault resolves the direction).
  const uint8_t* ns = nullptr;
  if (noskip) {
    if (e == cudaSuccess) e = cudaMemcpyAsync(base + oNs, noskip, (size_t)nfb * 8, cudaMemcpyDefault, st);
    ns = base + oNs;
  }
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  SearchArgs a;
  a.src = search_dframe(source, sp, sS);
  a.rec = search_dframe(recon, rpp, rS);
  a.noskip = ns;
  a.miCols = miCols;
  a.miRows = miRows;
  a.nhfb = nhfb;
  a.nvfb = nvfb;
  a.damping = damping;
  a.mse = (uint64_t*)(base + oMse);
  a.skip = base + oSkip;
  k_cdef_search<<<nfb, 256, 0, st>>>(a);
  k_sel_list<<<1, 32, 0, st>>>(a.skip, nfb, (int*)(base + oSb), (int*)(base + oN));
  if (cudaMemsetAsync(base + oSel, 0, sizeof(SelState), st) != cudaSuccess) return PF_ERR_DEVICE;
  // The number of non-skip blocks is needed on the host to size the steps.
  int n = 0;
  if (cudaMemcpyAsync(&n, base + oN, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return PF_ERR_DEVICE;
  SelArgs s;
  s.mse = a.mse;
  s.sb = (const int*)(base + oSb);
  s.n = n;
  s.nfb = nfb;
  s.st = (SelState*)(base + oSel);
  const int grid = imax(1, imin(148, n));
  for (int c = 0; c <= maxCfg; c++) {
    const int nb = 1 << c;
    // jointStrengthSearchDual: nb greedy steps, then 4*nb refinements.
    const int steps = nb + 4 * nb;
    for (int k = 0; k < steps; k++) {
      const int nbCur = k < nb ? k : nb - 1;
      const int shiftAfter = (k + 1 >= nb && k + 1 < steps) ? 1 : 0;
      k_sel_accum<<<grid, 256, 0, st>>>(s, c, nbCur);
      k_sel_pick<<<1, 1024, 0, st>>>(s, c, nbCur, shiftAfter, nb);
    }
  }
  k_sel_finish<<<imax(1, (nfb + 255) / 256), 256, 0, st>>>(s, maxCfg, (unsigned long long)params->lambda,
                                                           base + oIdx, (FinishOut*)(base + oFin));
  if (cudaGetLastError() != cudaSuccess) return PF_ERR_DEVICE;
  FinishOut fo;
  if (cudaMemcpyAsync(&fo, base + oFin, sizeof(fo), cudaMemcpyDeviceToHost, st) != cudaSuccess) return PF_ERR_DEVICE;
  if (mse_out &&
      cudaMemcpyAsync(mse_out, a.mse, (size_t)2 * nfb * 64 * 8, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PF_ERR_DEVICE;
  if (fb_index_out && cudaMemcpyAsync(fb_index_out, base + oIdx, nfb, cudaMemcpyDeviceToHost, st) != cudaSuccess)
    return PF_ERR_DEVICE;
  if (cudaStreamSynchronize(st) != cudaSuccess) return PF_ERR_DEVICE;
  if (result) {
    memset(result, 0, sizeof(*result));
    result->bits = (uint8_t)fo.bits;
    result->strength_count = (uint8_t)(1 << fo.bits);
    for (int j = 0; j < (1 << fo.bits); j++) {
      result->y_strength[j] = (uint8_t)trial_strength(fo.ys[j]);
      result->uv_strength[j] = (uint8_t)trial_strength(fo.uvs[j]);
    }
    result->cost = (double)fo.cost;
  }
  return PF_OK;
}
