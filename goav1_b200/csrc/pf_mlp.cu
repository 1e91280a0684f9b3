// pf_mlp.cu - learned CDEF strength selection: per-filter-block features,
// the 40-64-64-128 network (bf16 weights, fp32 arithmetic) and its training
// kernels.  No counterpart in goav1; the search it steers is the one in
// pf_search.cu (encoder/cdef_search.go level-1 trials and finish()).
//
//   k_cdef_features  one CTA per 64x64 filter block: CDEF direction costs and
//                    variances of the searched 8x8 blocks (cdef/direction.go
//                    arithmetic, as the search computes them), pixel
//                    statistics of the deblocked reconstruction, all
//                    accumulated as exact integers; 33 features per block.
//   k_feat_frame     frame means of seven of them (features 33..39).
//   k_mlp_masks      forward pass per 32 blocks, softmax heads, and the
//                    tested-trial masks: the top `candidates` trials of each
//                    head, or all 64 trials of a head whose top-1
//                    probability is below the threshold.
//   k_mlp_train_step forward + backward over 32 samples per CTA, partial
//                    gradients per CTA (no atomics: the reduction order is
//                    fixed, so training is deterministic).
//   k_mlp_reduce     sums the partials in CTA order, Adam on fp32 master
//                    weights, bf16 round-to-nearest-even copies for the next
//                    forward pass.
// The network is 14,848 MACs per sample: far too small for the tensor cores
// to matter (a 1080p frame is 510 samples, 7.6 M MACs); the kernels use
// fp32 FMA over bf16 weights converted once into shared memory.
#include <cuda_bf16.h>
#include <string.h>

#include <vector>

#include "pf_cdef_dev.cuh"
#include "pf_search.cuh"

namespace pf {

constexpr int kF = PF_MLP_FEATURES, kH = PF_MLP_HIDDEN, kC = PF_MLP_CLASSES, kO = PF_MLP_OUTPUTS;
constexpr int kNW1 = kH * kF, kNW2 = kH * kH, kNW3 = kO * kH;
constexpr int kNW = kNW1 + kNW2 + kNW3;
constexpr int kNP = PF_MLP_PARAMS;
constexpr int kTile = 32;  // samples per CTA
constexpr int kMlpThreads = 256;
constexpr int kPerFb = 33;  // per-block features; 33..39 are frame means

// ---------------------------------------------------------------------------
// Features.

struct FeatAcc {
  unsigned long long dcost[8], dhist[8];
  unsigned long long varsum, nvar0, adjsum;
  unsigned long long bvar;                 // sum over blocks of 64*sum(x^2) - sum(x)^2
  unsigned long long gH, cH, gV, cV;       // |horizontal| / |vertical| neighbour differences
  unsigned long long bH, cbH, bV, cbV;     // the ones across an 8-sample boundary
  unsigned long long lap, clap;            // |3x3 Laplacian|
  unsigned long long sumY;
  unsigned long long uvar, vvar;           // 4x4 chroma blocks: 16*sum(x^2) - sum(x)^2
  unsigned long long clapUV, cclapUV, cgUV, ccgUV;
};

__device__ __forceinline__ void acc_add(unsigned long long* p, unsigned long long v) {
  if (v) atomicAdd(p, v);
}

__global__ void __launch_bounds__(256, 4) k_cdef_features(SearchArgs a, int qindex, float* X) {
  __shared__ FeatAcc A;
  __shared__ int32_t s_cost[64 * 8];
  __shared__ uint8_t s_y[64 * 64];      // the filter block's luma (allocated part)
  __shared__ uint8_t s_c[2][32 * 32];   // and chroma
  const int tid = threadIdx.x;
  const int fb = blockIdx.x;
  const int fbr = fb / a.nhfb, fbc = fb - fbr * a.nhfb;
  const int lr = 16 * fbr, lc = 16 * fbc;
  const uint64_t listed = fb_listed(a, fb, lr, lc);
  float* out = X + (size_t)fb * kF;
  if (listed == 0) {
    if (tid < kPerFb) out[tid] = 0.f;
    return;
  }
  {
    unsigned long long* z = reinterpret_cast<unsigned long long*>(&A);
    for (int i = tid; i < (int)(sizeof(FeatAcc) / 8); i += 256) z[i] = 0;
  }
  const DPlane& Y = a.rec.pl[0];
  const int x0 = lc * 4, y0 = lr * 4;
  const int W = a.rec.width, H = a.rec.height;
  const int wc = imin(64, W - x0), hc = imin(64, H - y0);
  const int x0c = x0 >> 1, y0c = y0 >> 1;
  const int wcc = imin(32, a.rec.pl[1].w - x0c), hcc = imin(32, a.rec.pl[1].h - y0c);
  // Stage the block once, row-coalesced: every statistic reads shared memory.
  {
    const int rh = imin(64, Y.ah - y0), rw = imin(64, Y.aw - x0);
    for (int e = tid; e < rh * 64; e += 256) {
      const int i = e >> 6, j = e & 63;
      s_y[e] = j < rw ? row_ptr<uint8_t>(Y, y0 + i)[x0 + j] : 0;
    }
    for (int pl = 1; pl < 3; pl++) {
      const DPlane& Cp = a.rec.pl[pl];
      const int ch = imin(32, Cp.ah - y0c), cw = imin(32, Cp.aw - x0c);
      for (int e = tid; e < ch * 32; e += 256) {
        const int i = e >> 5, j = e & 31;
        s_c[pl - 1][e] = j < cw ? row_ptr<uint8_t>(Cp, y0c + i)[x0c + j] : 0;
      }
    }
  }
  __syncthreads();
  // Direction costs of the searched blocks (the search's own arithmetic).
  // A warp takes one direction for 32 blocks (no divergence between the
  // eight direction templates).
  for (int wi = tid; wi < 64 * 8; wi += 256) {
    const int d = wi >> 6, b = wi & 63;
    if ((listed >> b) & 1) s_cost[b * 8 + d] = dir_cost8_dev(d, &s_y[(b >> 3) * 8 * 64 + (b & 7) * 8], 64);
  }
  __syncthreads();
  if (tid < 64) {
    // Per searched 8x8 block (two warps, a lane per block), then warp sums:
    // one shared atomic per warp and counter.
    const bool on = (listed >> tid) & 1;
    unsigned long long dc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    unsigned long long var64 = 0, nvar0 = 0, adj = 0, bvar = 0, cv[2] = {0, 0};
    int best = 0;
    if (on) {
      int32_t bc = s_cost[tid * 8];
      for (int d = 1; d < 8; d++)
        if (s_cost[tid * 8 + d] > bc) {
          best = d;
          bc = s_cost[tid * 8 + d];
        }
      const int32_t var = (bc - s_cost[tid * 8 + ((best + 4) & 7)]) >> 10;
      for (int d = 0; d < 8; d++) dc[d] = (unsigned long long)s_cost[tid * 8 + d];
      var64 = (unsigned long long)var;
      int ai = -1;
      if (var == 0) {
        nvar0 = 1;
      } else {
        const int32_t v = var >> 6;
        ai = v ? imin(31 - __clz(v), 12) : 0;
        adj = (unsigned long long)(4 + ai);
      }
      if (a.dirs) {
        a.dirs[(size_t)fb * 64 + tid] = (uint8_t)best;
        a.ais[(size_t)fb * 64 + tid] = (int8_t)ai;
      }
      // 8x8 luma variance and 4x4 chroma variances of the block.
      const uint8_t* by = &s_y[(tid >> 3) * 8 * 64 + (tid & 7) * 8];
      long long s = 0, q = 0;
      for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
          const int x = by[i * 64 + j];
          s += x;
          q += x * x;
        }
      bvar = (unsigned long long)(64 * q - s * s);
      for (int pl = 0; pl < 2; pl++) {
        const uint8_t* bc2 = &s_c[pl][(tid >> 3) * 4 * 32 + (tid & 7) * 4];
        int cs = 0, cq = 0;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) {
            const int x = bc2[i * 32 + j];
            cs += x;
            cq += x * x;
          }
        cv[pl] = (unsigned long long)(16 * cq - cs * cs);
      }
    }
    // Direction histogram: each lane's best direction as a ballot per value.
    unsigned long long hist[8];
#pragma unroll
    for (int d = 0; d < 8; d++) hist[d] = __popc(__ballot_sync(0xffffffffu, on && best == d));
    unsigned long long v[15] = {dc[0], dc[1], dc[2], dc[3], dc[4], dc[5], dc[6], dc[7], var64, nvar0, adj, bvar,
                                cv[0], cv[1], 0};
#pragma unroll
    for (int k = 0; k < 14; k++)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((tid & 31) == 0) {
#pragma unroll
      for (int d = 0; d < 8; d++) {
        acc_add(&A.dcost[d], v[d]);
        acc_add(&A.dhist[d], hist[d]);
      }
      acc_add(&A.varsum, v[8]);
      acc_add(&A.nvar0, v[9]);
      acc_add(&A.adjsum, v[10]);
      acc_add(&A.bvar, v[11]);
      acc_add(&A.uvar, v[12]);
      acc_add(&A.vvar, v[13]);
    }
  }
  // Pixel statistics over the cropped luma region.
  {
    unsigned long long gH = 0, cH = 0, gV = 0, cV = 0, bH = 0, cbH = 0, bV = 0, cbV = 0, lap = 0, clap = 0,
                       sy = 0;
    for (int e = tid; e < hc * 64; e += 256) {
      const int i = e >> 6, j = e & 63;
      if (j >= wc) continue;
      const uint8_t* r0 = &s_y[i * 64];
      const int x = r0[j];
      sy += x;
      if (j + 1 < wc) {
        const unsigned d = abs(r0[j + 1] - x);
        gH += d;
        cH++;
        if (((x0 + j + 1) & 7) == 0) {
          bH += d;
          cbH++;
        }
      }
      if (i + 1 < hc) {
        const unsigned d = abs(r0[64 + j] - x);
        gV += d;
        cV++;
        if (((y0 + i + 1) & 7) == 0) {
          bV += d;
          cbV++;
        }
      }
      if (i >= 1 && i + 1 < hc && j >= 1 && j + 1 < wc) {
        const uint8_t* ru = r0 - 64;
        const uint8_t* rd = r0 + 64;
        const int L = ru[j - 1] - 2 * ru[j] + ru[j + 1] - 2 * r0[j - 1] + 4 * x - 2 * r0[j + 1] + rd[j - 1] -
                      2 * rd[j] + rd[j + 1];
        lap += (unsigned)abs(L);
        clap++;
      }
    }
    // Chroma: Laplacian and neighbour differences over the cropped region.
    unsigned long long cl = 0, ccl = 0, cg = 0, ccg = 0;
    for (int e = tid; e < 2 * hcc * 32; e += 256) {
      const int pl = e / (hcc * 32), r = e - pl * hcc * 32;
      const int i = r >> 5, j = r & 31;
      if (j >= wcc) continue;
      const uint8_t* r0 = &s_c[pl][i * 32];
      const int x = r0[j];
      if (j + 1 < wcc) {
        cg += (unsigned)abs(r0[j + 1] - x);
        ccg++;
      }
      if (i + 1 < hcc) {
        cg += (unsigned)abs(r0[32 + j] - x);
        ccg++;
      }
      if (i >= 1 && i + 1 < hcc && j >= 1 && j + 1 < wcc) {
        const uint8_t* ru = r0 - 32;
        const uint8_t* rd = r0 + 32;
        const int L = ru[j - 1] - 2 * ru[j] + ru[j + 1] - 2 * r0[j - 1] + 4 * x - 2 * r0[j + 1] + rd[j - 1] -
                      2 * rd[j] + rd[j + 1];
        cl += (unsigned)abs(L);
        ccl++;
      }
    }
    // Warp sums first: one shared atomic per warp and counter.
    unsigned long long v[15] = {gH, cH, gV, cV, bH, cbH, bV, cbV, lap, clap, sy, cl, ccl, cg, ccg};
#pragma unroll
    for (int k = 0; k < 15; k++)
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    if ((tid & 31) == 0) {
      unsigned long long* dst[15] = {&A.gH, &A.cH, &A.gV, &A.cV, &A.bH, &A.cbH, &A.bV, &A.cbV, &A.lap, &A.clap,
                                     &A.sumY, &A.clapUV, &A.cclapUV, &A.cgUV, &A.ccgUV};
#pragma unroll
      for (int k = 0; k < 15; k++) acc_add(dst[k], v[k]);
    }
  }
  __syncthreads();
  if (tid < kPerFb) {
    // Thread i writes feature i (same expressions as the oracle's).
    const float nb = (float)__popcll(listed);
    auto cnt = [](unsigned long long c) { return (float)(c ? c : 1ull); };
    float f;
    const int i = tid;
    if (i < 8) {
      unsigned long long ds = 0;
      for (int d = 0; d < 8; d++) ds += A.dcost[d];
      f = ds ? (float)A.dcost[i] / (float)ds : 0.125f;
    } else if (i < 16) {
      f = (float)A.dhist[i - 8] / nb;
    } else {
      switch (i) {
        case 16: f = log2f(1.f + (float)A.varsum / nb); break;
        case 17: f = (float)A.nvar0 / nb; break;
        case 18: f = (float)A.adjsum / (16.f * nb); break;
        case 19: f = log2f(1.f + (float)A.bvar / (4096.f * nb)); break;
        case 20: f = log2f(1.f + (float)A.gH / cnt(A.cH)); break;
        case 21: f = log2f(1.f + (float)A.gV / cnt(A.cV)); break;
        case 22: f = log2f(1.f + (float)A.lap / cnt(A.clap)); break;
        case 23: f = ((float)A.bH / cnt(A.cbH) - (float)(A.gH - A.bH) / cnt(A.cH - A.cbH)) / 8.f; break;
        case 24: f = ((float)A.bV / cnt(A.cbV) - (float)(A.gV - A.bV) / cnt(A.cV - A.cbV)) / 8.f; break;
        case 25: f = log2f(1.f + (float)A.uvar / (256.f * nb)); break;
        case 26: f = log2f(1.f + (float)A.vvar / (256.f * nb)); break;
        case 27: f = log2f(1.f + (float)A.clapUV / cnt(A.cclapUV)); break;
        case 28: f = log2f(1.f + (float)A.cgUV / cnt(A.ccgUV)); break;
        case 29: f = nb / 64.f; break;
        case 30: f = (float)qindex / 255.f; break;
        case 31: f = (float)(a.damping - 3) / 3.f; break;
        default: f = (float)A.sumY / (255.f * (float)(wc * hc)); break;
      }
    }
    out[i] = f;
  }
}

// Frame means of features 16, 19, 22, 23, 24, 25, 27 over the searched
// blocks (features 33..39 of every block).  Fixed-order sums: 256 threads
// stride over the blocks, then a tree in shared memory, so every caller gets
// the same bits.
__constant__ int c_frame_feat[7] = {16, 19, 22, 23, 24, 25, 27};

struct FrameMeanSmem {
  double sum[7][256];
  int cnt[256];
  float mean[7];
};

__device__ void frame_means(const float* X, int nfb, FrameMeanSmem& M) {
  const int t = threadIdx.x;  // blockDim.x == 256
  double acc[7] = {0, 0, 0, 0, 0, 0, 0};
  int c = 0;
  for (int fb = t; fb < nfb; fb += 256) {
    const float* f = X + (size_t)fb * kF;
    if (f[29] > 0.f) {
      c++;
      for (int i = 0; i < 7; i++) acc[i] += (double)f[c_frame_feat[i]];
    }
  }
  for (int i = 0; i < 7; i++) M.sum[i][t] = acc[i];
  M.cnt[t] = c;
  __syncthreads();
  for (int o = 128; o > 0; o >>= 1) {
    if (t < o) {
      for (int i = 0; i < 7; i++) M.sum[i][t] += M.sum[i][t + o];
      M.cnt[t] += M.cnt[t + o];
    }
    __syncthreads();
  }
  if (t < 7) M.mean[t] = M.cnt[0] ? (float)(M.sum[t][0] / (double)M.cnt[0]) : 0.f;
  __syncthreads();
}

__global__ void __launch_bounds__(256) k_feat_frame(float* X, int nfb) {
  __shared__ FrameMeanSmem M;
  frame_means(X, nfb, M);
  for (int e = threadIdx.x; e < nfb * 7; e += 256) X[(size_t)(e / 7) * kF + kPerFb + e % 7] = M.mean[e % 7];
}

// ---------------------------------------------------------------------------
// The network.

template <int TILE>
struct MlpTileT {
  float w1[kNW1], w2[kNW2], w3[kNW3];
  float b1[kH], b2[kH], b3[kO];
  float x[TILE][kF + 1];
  float h1[TILE][kH + 1];
  float h2[TILE][kH + 1];
  float z[TILE][kO + 1];   // logits, then probabilities, then dL/dz
  float dh2[TILE][kH + 1];
  float dh1[TILE][kH + 1];
  float lossh[TILE][2];
  float loss[TILE];
  int y[TILE][2];
};
using MlpTile = MlpTileT<kTile>;  // training tile
constexpr int kInferTile = 8;    // inference: more CTAs, less serial work each
using MlpInfer = MlpTileT<kInferTile>;

__device__ __forceinline__ float bf16_to_f(uint16_t b) { return __uint_as_float((uint32_t)b << 16); }

// Loads the weights (bf16 -> fp32) and the normalised features of `count`
// samples (rows[first + s], or first + s), then the three layers.  Lanes of
// a warp are samples, warps are output groups: a weight is a broadcast and
// an activation row a conflict-free column.
// Weights widened once to fp32 for the inference kernels: [w1 | w2 | w3 |
// b1 | b2 | b3 | feat_shift | feat_scale], the layout of MlpTileT's weight
// block followed by the normalisation.
constexpr int kExpanded = kNP + 2 * kF;

__global__ void k_mlp_expand(const pf_cdef_mlp* M, float* W) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kExpanded) return;
  if (p < kNW)
    W[p] = bf16_to_f(reinterpret_cast<const uint16_t*>(M)[p]);
  else if (p < kNP)
    W[p] = reinterpret_cast<const float*>(&M->b1[0])[p - kNW];
  else
    W[p] = reinterpret_cast<const float*>(&M->feat_shift[0])[p - kNP];  // shift, then scale
}

template <int TILE>
__device__ void mlp_forward(MlpTileT<TILE>& T, const pf_cdef_mlp* M, const float* X, const int* rows, int first, int count,
                            const float* means = nullptr, const float* Wf = nullptr) {
  const int t = threadIdx.x;
  const float* shift = M ? M->feat_shift : Wf + kNP;
  const float* scale = M ? M->feat_scale : Wf + kNP + kF;
  if (Wf) {
    // fp32 weights and biases, contiguous like the tile's: 16-byte copies.
    const float4* src = reinterpret_cast<const float4*>(Wf);
    float4* dst = reinterpret_cast<float4*>(&T.w1[0]);
    for (int e = t; e < kNP / 4; e += kMlpThreads) dst[e] = src[e];
  } else {
    for (int e = t; e < kNW1; e += kMlpThreads) T.w1[e] = bf16_to_f(M->w1[e]);
    for (int e = t; e < kNW2; e += kMlpThreads) T.w2[e] = bf16_to_f(M->w2[e]);
    for (int e = t; e < kNW3; e += kMlpThreads) T.w3[e] = bf16_to_f(M->w3[e]);
    if (t < kH) {
      T.b1[t] = M->b1[t];
      T.b2[t] = M->b2[t];
    }
    if (t < kO) T.b3[t] = M->b3[t];
  }
  for (int e = t; e < TILE * kF; e += kMlpThreads) {
    const int s = e / kF, k = e - s * kF;
    float v = 0.f;
    if (s < count) {
      const int r = rows ? rows[first + s] : first + s;
      const float f = (means && k >= kPerFb) ? means[k - kPerFb] : X[(size_t)r * kF + k];
      v = (f - shift[k]) * scale[k];
    }
    T.x[s][k] = v;
  }
  __syncthreads();
  constexpr int G = kMlpThreads / TILE;  // output groups
  const int s = t % TILE, og = t / TILE;
  for (int q = 0; q < kH / G; q++) {
    const int o = og * (kH / G) + q;
    float acc = T.b1[o];
    for (int k = 0; k < kF; k++) acc = __fmaf_rn(T.w1[o * kF + k], T.x[s][k], acc);
    T.h1[s][o] = acc > 0.f ? acc : 0.f;
  }
  __syncthreads();
  for (int q = 0; q < kH / G; q++) {
    const int o = og * (kH / G) + q;
    float acc = T.b2[o];
    for (int k = 0; k < kH; k++) acc = __fmaf_rn(T.w2[o * kH + k], T.h1[s][k], acc);
    T.h2[s][o] = acc > 0.f ? acc : 0.f;
  }
  __syncthreads();
  for (int q = 0; q < kO / G; q++) {
    const int o = og * (kO / G) + q;
    float acc = T.b3[o];
    for (int k = 0; k < kH; k++) acc = __fmaf_rn(T.w3[o * kH + k], T.h2[s][k], acc);
    T.z[s][o] = acc;
  }
  __syncthreads();
}

// Softmax of both heads in place, one warp per (sample, head): lane l holds
// classes l and l + 32; the maximum and the sum are butterfly reductions
// (sum order: e[l] + e[l+32], then xor-partners at distances 16..1).  With
// labels, the per-sample loss (log-sum-exp minus the label's logit, both
// heads).
template <int TILE>
__device__ void mlp_softmax(MlpTileT<TILE>& T, bool withLoss) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int task = warp; task < 2 * TILE; task += kMlpThreads / 32) {
    const int s = task >> 1, hd = task & 1;
    float* z = &T.z[s][hd * kC];
    const float z0 = z[lane], z1 = z[lane + 32];
    float m = fmaxf(z0, z1);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    const float e0 = expf(z0 - m), e1 = expf(z1 - m);
    float sum = e0 + e1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (withLoss && lane == 0) T.lossh[s][hd] = m + logf(sum) - z[T.y[s][hd]];
    __syncwarp();
    const float inv = 1.f / sum;
    z[lane] = e0 * inv;
    z[lane + 32] = e1 * inv;
  }
  __syncthreads();
  if (withLoss && threadIdx.x < TILE) T.loss[threadIdx.x] = T.lossh[threadIdx.x][0] + T.lossh[threadIdx.x][1];
  __syncthreads();
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_masks(const float* W, const float* X, int nfb,
                                                           float threshold, int candidates, uint64_t* masks) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpInfer& T = *reinterpret_cast<MlpInfer*>(smem);
  __shared__ FrameMeanSmem FM;
  __shared__ uint64_t s_m[kInferTile][2];
  __shared__ int s_conf[kInferTile][2];
  const int first = blockIdx.x * kInferTile, count = imin(kInferTile, nfb - first);
  frame_means(X, nfb, FM);  // features 33..39 (the features kernel leaves them unset)
  mlp_forward(T, nullptr, X, nullptr, first, count, FM.mean, W);
  mlp_softmax(T, false);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int task = warp; task < 2 * kInferTile; task += kMlpThreads / 32) {
    const int s = task >> 1, hd = task & 1;
    float p0 = T.z[s][hd * kC + lane], p1 = T.z[s][hd * kC + lane + 32];
    uint64_t m = 0;
    float top = 0.f;
    for (int c = 0; c < candidates; c++) {
      // Largest remaining probability, the lower class on ties.
      float v = p0;
      int i = lane;
      if (p1 > v) {
        v = p1;
        i = lane + 32;
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const float v2 = __shfl_xor_sync(0xffffffffu, v, o);
        const int i2 = __shfl_xor_sync(0xffffffffu, i, o);
        if (v2 > v || (v2 == v && i2 < i)) {
          v = v2;
          i = i2;
        }
      }
      if (c == 0) top = v;
      m |= 1ull << i;
      if (i == lane) p0 = -1.f;
      if (i == lane + 32) p1 = -1.f;
    }
    if (lane == 0) {
      s_m[s][hd] = m;
      s_conf[s][hd] = top >= threshold;
    }
  }
  __syncthreads();
  const int t = threadIdx.x;
  if (t < count) {
    // Each head falls back on its own: an unsure luma head measures all 64
    // luma trials while a confident chroma head keeps its candidates.
    masks[2 * (size_t)(first + t)] = s_conf[t][0] ? s_m[t][0] : ~0ull;
    masks[2 * (size_t)(first + t) + 1] = s_conf[t][1] ? s_m[t][1] : ~0ull;
  }
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_probs(const float* W, const float* X, int n, float* P) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpInfer& T = *reinterpret_cast<MlpInfer*>(smem);
  const int first = blockIdx.x * kInferTile, count = imin(kInferTile, n - first);
  mlp_forward(T, nullptr, X, nullptr, first, count, nullptr, W);
  mlp_softmax(T, false);
  for (int e = threadIdx.x; e < count * kO; e += kMlpThreads) P[(size_t)first * kO + e] = T.z[e / kO][e % kO];
}

// Forward and backward over samples rows[first + 32*blockIdx.x + s] (s <
// count), gradients of (sum of losses) / total written per CTA to
// G[blockIdx.x][PF_MLP_PARAMS], summed losses to L[blockIdx.x].
__global__ void __launch_bounds__(kMlpThreads) k_mlp_train_step(const pf_cdef_mlp* M, const float* X,
                                                                const uint8_t* labels, const int* rows, int first,
                                                                int total, float* G, float* L, int* stepCounter) {
  extern __shared__ __align__(16) unsigned char smem[];
  MlpTile& T = *reinterpret_cast<MlpTile*>(smem);
  const int t = threadIdx.x;
  const int f0 = first + blockIdx.x * kTile;
  const int count = imin(kTile, total - blockIdx.x * kTile);
  if (stepCounter && blockIdx.x == 0 && t == 0) atomicAdd(stepCounter, 1);
  if (t < kTile) {
    const int r = t < count ? (rows ? rows[f0 + t] : f0 + t) : 0;
    T.y[t][0] = t < count ? labels[2 * (size_t)r] : 0;
    T.y[t][1] = t < count ? labels[2 * (size_t)r + 1] : 0;
  }
  mlp_forward(T, M, X, rows, f0, count);
  mlp_softmax(T, true);
  const float invB = 1.f / (float)total;
  for (int e = t; e < kTile * kO; e += kMlpThreads) {
    const int s = e >> 7, o = e & 127;
    const int hd = o >> 6, c = o & 63;
    T.z[s][o] = s < count ? (T.z[s][o] - (c == T.y[s][hd] ? 1.f : 0.f)) * invB : 0.f;
  }
  __syncthreads();
  float* g = G + (size_t)blockIdx.x * kNP;
  float* gw1 = g;
  float* gw2 = g + kNW1;
  float* gw3 = g + kNW1 + kNW2;
  float* gb1 = g + kNW;
  float* gb2 = gb1 + kH;
  float* gb3 = gb2 + kH;
  for (int e = t; e < kNW3; e += kMlpThreads) {
    const int o = e >> 6, k = e & 63;
    float acc = 0.f;
    for (int s = 0; s < kTile; s++) acc = __fmaf_rn(T.z[s][o], T.h2[s][k], acc);
    gw3[e] = acc;
  }
  if (t < kO) {
    float acc = 0.f;
    for (int s = 0; s < kTile; s++) acc += T.z[s][t];
    gb3[t] = acc;
  }
  for (int e = t; e < kTile * kH; e += kMlpThreads) {
    const int s = e >> 6, k = e & 63;
    float acc = 0.f;
    if (T.h2[s][k] > 0.f)
      for (int o = 0; o < kO; o++) acc = __fmaf_rn(T.w3[o * kH + k], T.z[s][o], acc);
    T.dh2[s][k] = acc;
  }
  __syncthreads();
  for (int e = t; e < kNW2; e += kMlpThreads) {
    const int o = e >> 6, k = e & 63;
    float acc = 0.f;
    for (int s = 0; s < kTile; s++) acc = __fmaf_rn(T.dh2[s][o], T.h1[s][k], acc);
    gw2[e] = acc;
  }
  if (t < kH) {
    float acc = 0.f;
    for (int s = 0; s < kTile; s++) acc += T.dh2[s][t];
    gb2[t] = acc;
  }
  for (int e = t; e < kTile * kH; e += kMlpThreads) {
    const int s = e >> 6, k = e & 63;
    float acc = 0.f;
    if (T.h1[s][k] > 0.f)
      for (int o = 0; o < kH; o++) acc = __fmaf_rn(T.w2[o * kH + k], T.dh2[s][o], acc);
    T.dh1[s][k] = acc;
  }
  __syncthreads();
  for (int e = t; e < kNW1; e += kMlpThreads) {
    const int o = e / kF, k = e - o * kF;
    float acc = 0.f;
    for (int s = 0; s < kTile; s++) acc = __fmaf_rn(T.dh1[s][o], T.x[s][k], acc);
    gw1[e] = acc;
  }
  if (t < kH) {
    float acc = 0.f;
    for (int s = 0; s < kTile; s++) acc += T.dh1[s][t];
    gb1[t] = acc;
  }
  if (t == 0) {
    float acc = 0.f;
    for (int s = 0; s < count; s++) acc += T.loss[s];
    L[blockIdx.x] = acc;
  }
}

struct AdamState {
  float* master;  // fp32 weights and biases, PF_MLP_PARAMS
  float* m;
  float* v;
  float lr, beta1, beta2, eps, wd;
};

__device__ __forceinline__ uint16_t f_to_bf16(float f) { return __bfloat16_as_ushort(__float2bfloat16_rn(f)); }

// Sums the per-CTA partials in CTA order; with an Adam state, updates the
// master weights and the bf16 model, else writes the sums to `out`.
__global__ void __launch_bounds__(256) k_mlp_reduce(const float* G, const float* L, int tiles, float lossScale,
                                                    float* out, float* lossOut, AdamState A, const int* step,
                                                    pf_cdef_mlp* M, const int* epoch) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0) {
    float acc = 0.f;
    for (int c = 0; c < tiles; c++) acc += L[c];
    if (epoch)
      lossOut[*epoch] += acc * lossScale;
    else
      *lossOut = acc * lossScale;
  }
  if (p >= kNP) return;
  float g = 0.f;
  for (int c = 0; c < tiles; c++) g += G[(size_t)c * kNP + p];
  if (!A.master) {
    out[p] = g;
    return;
  }
  const int k = *step;
  const float m = A.m[p] = A.beta1 * A.m[p] + (1.f - A.beta1) * g;
  const float v = A.v[p] = A.beta2 * A.v[p] + (1.f - A.beta2) * g * g;
  const float mh = m / (1.f - powf(A.beta1, (float)k));
  const float vh = v / (1.f - powf(A.beta2, (float)k));
  float w = A.master[p];
  if (p < kNW) w -= A.lr * A.wd * w;
  w -= A.lr * mh / (sqrtf(vh) + A.eps);
  A.master[p] = w;
  if (p < kNW)
    reinterpret_cast<uint16_t*>(M)[p] = f_to_bf16(w);
  else
    reinterpret_cast<float*>(&M->b1[0])[p - kNW] = w;  // b1, b2, b3 are contiguous
}

__global__ void k_epoch_inc(int* epoch) { (*epoch)++; }

__global__ void k_master_init(const pf_cdef_mlp* M, float* master) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kNP) return;
  master[p] = p < kNW ? bf16_to_f(reinterpret_cast<const uint16_t*>(M)[p])
                      : reinterpret_cast<const float*>(&M->b1[0])[p - kNW];
}

static cudaError_t set_tile_smem(const void* fn, size_t bytes = sizeof(MlpTile)) {
  return cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

cudaError_t launch_features(const SearchArgs& a, int qindex, float* X, bool frameMeans, cudaStream_t st) {
  const int nfb = a.nhfb * a.nvfb;
  k_cdef_features<<<nfb, 256, 0, st>>>(a, qindex, X);
  if (frameMeans) k_feat_frame<<<1, 256, 0, st>>>(X, nfb);
  return cudaGetLastError();
}

size_t mlp_expanded_bytes() { return (size_t)kExpanded * sizeof(float); }

cudaError_t launch_mlp_masks(const pf_cdef_mlp* dmodel, float* W, bool expand, const float* X, int nfb,
                             float threshold, int candidates, uint64_t* masks, cudaStream_t st) {
  static thread_local int ready = -1;  // device whose attribute is set
  int dev = 0;
  cudaGetDevice(&dev);
  if (ready != dev) {
    const cudaError_t e = set_tile_smem((const void*)k_mlp_masks, sizeof(MlpInfer));
    if (e != cudaSuccess) return e;
    ready = dev;
  }
  if (expand) k_mlp_expand<<<(kExpanded + 255) / 256, 256, 0, st>>>(dmodel, W);
  k_mlp_masks<<<(nfb + kInferTile - 1) / kInferTile, kMlpThreads, sizeof(MlpInfer), st>>>(W, X, nfb, threshold,
                                                                                       candidates, masks);
  return cudaGetLastError();
}

}  // namespace pf

using namespace pf;

void* pf_internal_stream(pf_ctx* c);  // pf_api.cu

namespace {

// Device buffers of one training / inference call (freed on scope exit).
struct Scratch {
  std::vector<void*> ptrs;
  cudaError_t err = cudaSuccess;
  template <typename T>
  T* get(size_t count) {
    void* p = nullptr;
    if (err == cudaSuccess) err = cudaMalloc(&p, count * sizeof(T) + 16);
    if (err != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    return (T*)p;
  }
  ~Scratch() {
    for (void* p : ptrs) cudaFree(p);
  }
};

uint64_t splitmix(uint64_t* s) {
  uint64_t z = (*s += 0x9e3779b97f4a7c15ull);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

int check_labels(const uint8_t* labels, int n) {
  for (int i = 0; i < 2 * n; i++)
    if (labels[i] >= PF_MLP_CLASSES) return PF_ERR_INVALID_ARG;
  return PF_OK;
}

}  // namespace

extern "C" int pf_cdef_mlp_forward(pf_ctx* ctx, const pf_cdef_mlp* model, const float* features, int32_t n,
                                   float* probs) {
  if (!ctx || !model || n < 0 || (n > 0 && (!features || !probs))) return PF_ERR_INVALID_ARG;
  if (n == 0) return PF_OK;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  Scratch S;
  pf_cdef_mlp* dm = S.get<pf_cdef_mlp>(1);
  float* W = S.get<float>(kExpanded);
  float* X = S.get<float>((size_t)n * kF);
  float* P = S.get<float>((size_t)n * kO);
  if (S.err != cudaSuccess) return PF_ERR_DEVICE;
  if (cudaMemcpyAsync(dm, model, sizeof(*model), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(X, features, (size_t)n * kF * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      set_tile_smem((const void*)k_mlp_probs, sizeof(MlpInfer)) != cudaSuccess)
    return PF_ERR_DEVICE;
  k_mlp_expand<<<(kExpanded + 255) / 256, 256, 0, st>>>(dm, W);
  k_mlp_probs<<<(n + kInferTile - 1) / kInferTile, kMlpThreads, sizeof(MlpInfer), st>>>(W, X, n, P);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(probs, P, (size_t)n * kO * 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return PF_ERR_DEVICE;
  return PF_OK;
}

extern "C" int pf_cdef_mlp_gradients(pf_ctx* ctx, const pf_cdef_mlp* model, const float* features,
                                     const uint8_t* labels, int32_t n, float* loss, pf_cdef_mlp_grads* grads) {
  if (!ctx || !model || !features || !labels || !loss || !grads || n <= 0) return PF_ERR_INVALID_ARG;
  if (check_labels(labels, n) != PF_OK) return PF_ERR_INVALID_ARG;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  const int tiles = (n + kTile - 1) / kTile;
  Scratch S;
  pf_cdef_mlp* dm = S.get<pf_cdef_mlp>(1);
  float* X = S.get<float>((size_t)n * kF);
  uint8_t* Y = S.get<uint8_t>((size_t)n * 2);
  float* G = S.get<float>((size_t)tiles * kNP);
  float* L = S.get<float>(tiles);
  float* out = S.get<float>(kNP + 1);
  if (S.err != cudaSuccess) return PF_ERR_DEVICE;
  if (cudaMemcpyAsync(dm, model, sizeof(*model), cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(X, features, (size_t)n * kF * 4, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaMemcpyAsync(Y, labels, (size_t)n * 2, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      set_tile_smem((const void*)k_mlp_train_step) != cudaSuccess)
    return PF_ERR_DEVICE;
  k_mlp_train_step<<<tiles, kMlpThreads, sizeof(MlpTile), st>>>(dm, X, Y, nullptr, 0, n, G, L, nullptr);
  AdamState none;
  memset(&none, 0, sizeof(none));
  k_mlp_reduce<<<(kNP + 255) / 256, 256, 0, st>>>(G, L, tiles, 1.f / (float)n, out, out + kNP, none, nullptr, nullptr,
                                                  nullptr);
  if (cudaGetLastError() != cudaSuccess ||
      cudaMemcpyAsync(grads, out, sizeof(*grads), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaMemcpyAsync(loss, out + kNP, 4, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return PF_ERR_DEVICE;
  return PF_OK;
}

extern "C" int pf_cdef_mlp_train(pf_ctx* ctx, pf_cdef_mlp* model, const float* features, const uint8_t* labels,
                                 int32_t n, const pf_cdef_mlp_train_params* prm, float* epoch_loss) {
  if (!ctx || !model || !features || !labels || !prm || n <= 0) return PF_ERR_INVALID_ARG;
  if (prm->epochs <= 0 || prm->batch <= 0 || prm->batch % kTile || !(prm->lr > 0.f)) return PF_ERR_INVALID_ARG;
  if (check_labels(labels, n) != PF_OK) return PF_ERR_INVALID_ARG;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  const int B = prm->batch, steps = (n + B - 1) / B, tilesMax = B / kTile;
  Scratch S;
  pf_cdef_mlp* dm = S.get<pf_cdef_mlp>(1);
  float* X = S.get<float>((size_t)n * kF);
  uint8_t* Y = S.get<uint8_t>((size_t)n * 2);
  int* perm = S.get<int>(n);
  float* G = S.get<float>((size_t)tilesMax * kNP);
  float* L = S.get<float>(tilesMax);
  float* master = S.get<float>(kNP);
  float* m = S.get<float>(kNP);
  float* v = S.get<float>(kNP);
  int* counters = S.get<int>(2);  // Adam step, epoch
  float* eloss = S.get<float>(prm->epochs);
  if (S.err != cudaSuccess) return PF_ERR_DEVICE;
  cudaError_t e = cudaMemcpyAsync(dm, model, sizeof(*model), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(X, features, (size_t)n * kF * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(Y, labels, (size_t)n * 2, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(m, 0, kNP * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(v, 0, kNP * 4, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(counters, 0, 8, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(eloss, 0, (size_t)prm->epochs * 4, st);
  if (e == cudaSuccess) e = set_tile_smem((const void*)k_mlp_train_step);
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  k_master_init<<<(kNP + 255) / 256, 256, 0, st>>>(dm, master);
  AdamState A;
  A.master = master;
  A.m = m;
  A.v = v;
  A.lr = prm->lr;
  A.beta1 = prm->beta1;
  A.beta2 = prm->beta2;
  A.eps = prm->eps;
  A.wd = prm->weight_decay;
  // One epoch (every step's forward/backward and Adam update) is captured
  // once as a CUDA graph and replayed; only the shuffled order changes.
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  for (int s = 0; s < steps; s++) {
    const int first = s * B, total = imin(B, n - first);
    const int tiles = (total + kTile - 1) / kTile;
    k_mlp_train_step<<<tiles, kMlpThreads, sizeof(MlpTile), st>>>(dm, X, Y, perm, first, total, G, L, counters);
    k_mlp_reduce<<<(kNP + 255) / 256, 256, 0, st>>>(G, L, tiles, 1.f / (float)n, nullptr, eloss, A, counters, dm,
                                                    counters + 1);
  }
  k_epoch_inc<<<1, 1, 0, st>>>(counters + 1);
  e = cudaStreamEndCapture(st, &graph);
  if (e == cudaSuccess) e = cudaGraphInstantiate(&exec, graph, 0);
  std::vector<int> order(n);
  uint64_t rs = prm->seed;
  for (int ep = 0; ep < prm->epochs && e == cudaSuccess; ep++) {
    for (int i = 0; i < n; i++) order[i] = i;
    for (int i = n - 1; i > 0; i--) {
      const int j = (int)(splitmix(&rs) % (uint64_t)(i + 1));
      const int tmp = order[i];
      order[i] = order[j];
      order[j] = tmp;
    }
    e = cudaMemcpyAsync(perm, order.data(), (size_t)n * 4, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaGraphLaunch(exec, st);
    // The host order buffer is reused next epoch: wait for the copy.
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  }
  if (exec) cudaGraphExecDestroy(exec);
  if (graph) cudaGraphDestroy(graph);
  if (e == cudaSuccess) e = cudaMemcpyAsync(model, dm, sizeof(*model), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess && epoch_loss)
    e = cudaMemcpyAsync(epoch_loss, eloss, (size_t)prm->epochs * 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  return e == cudaSuccess ? PF_OK : PF_ERR_DEVICE;
}
