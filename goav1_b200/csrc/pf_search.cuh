// pf_search.cuh - shared declarations of the encoder CDEF strength search
// (pf_search.cu) and the learned strength selection built on it (pf_mlp.cu).
#pragma once

#include "pf_cdef_dev.cuh"
#include "pf_common.cuh"

namespace pf {

// goav1's cdefDefaultMSEUV * 64 (encoder/cdef_search.go:669-672): the SSE
// recorded for a trial that was not measured.
constexpr uint32_t kUntestedMSE = 1040400u * 64u;

constexpr int kSelMaxCluster = 16;  // CTAs per greedy-selection cluster (non-portable size)
constexpr int kSelMinCluster = 8;   // fallback where a 16-CTA cluster cannot be placed
constexpr int kSelThreads = 512;
constexpr size_t kSelMaxSmem = 200 * 1024;

// Trial gi -> packed strength (level-1 lists: svtPfGI = 4*i for i < 16, then
// pf+1..pf+3 for each first-pass pf; encoder/cdef_search.go:72-110).
__host__ __device__ __forceinline__ int trial_strength(int g) {
  if (g < 16) return g * 4;
  const int k = g - 16;
  return (k / 3) * 4 + (k % 3) + 1;
}

// The trials a search measures (a level's controls, cdefSearchJob in
// encoder/cdef_search.go:581-596): trial g tests luma packed strength y[g]
// and chroma uv[g] (uvMask bit clear: not measured); luma rows every ss-th.
struct TrialList {
  int8_t y[64];
  int8_t uv[64];
  uint64_t uvMask;
  int count;
  int ss;
};

// SSE-table entry of a trial index past the list (PF_CDEF_NOT_A_TRIAL): no
// selection step can pick it (see k_sel_greedy).
constexpr uint32_t kNotATrial = 0x7fffffffu;

struct SearchArgs {
  DFrame src, rec;          // 8-bit 4:2:0
  const uint8_t* noskip;    // 8 bytes per filter block, or null (all blocks)
  const uint64_t* tmask;    // [nfb][2] tested luma / chroma trials, or null (all 64)
  int miCols, miRows, nhfb, nvfb;
  int damping;
  uint64_t* mse;            // [2][nfb][64]
  uint8_t* skip;            // [nfb]
  // Per 8x8 luma block of each filter block: CDEF direction and
  // adjustStrength index (-1 for zero variance).  Written by the features
  // kernel when non-null; read by the search instead of its own direction
  // pass when non-null.
  uint8_t* dirs;            // [nfb][64]
  int8_t* ais;              // [nfb][64]
  TrialList trials;         // tmask searches use the level-1 list
  // constrain() tables of the context ([strength 16][shift 8][512], entry
  // 255 + d for a difference d, entry 511 = 0: CdefArgs.ctab).
  const int16_t* ctab;
  // CTAs per filter block: slice s of a block measures the tested trials at
  // positions s, s + slices, ... of its list (1: one CTA measures them all).
  int slices;
};

struct SelOut {
  int lev0[4][8], lev1[4][8];  // per configuration nb = 1 << c
  unsigned long long tot[4];
};

struct FinishOut {
  int bits;
  int ys[8], uvs[8];
  unsigned long long cost;
};

struct SelArgs {
  const uint64_t* mse;   // [2][nfb][64]
  const uint8_t* skip;   // [nfb]; the kernels list the non-skip blocks themselves
  int nfb, cap;
  int refine;            // 1: the reference's 4*nb refinement passes after the nb greedy picks
  int uvFromY;           // the presets' chroma trials are their luma trials (finish, :920-925)
  SelOut* out;
};

// The 8x8 luma blocks of filter block fb that the search measures
// (computeCDEFList, encoder/cdef_search.go:410-447: noskip blocks inside the
// MI grid), as a bit per block (bit = 8 * row + column).
__device__ __forceinline__ uint64_t fb_listed(const SearchArgs& a, int fb, int lr, int lc) {
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
  return listed;
}

// cdef/direction.go:37-79 (partial sums) and :469-501 (cost), 8-bit samples
// read straight from the frame or a staged copy; shared by the search and
// the features.  The samples go in as packed pairs (dir_cost_pairs): two
// 32-bit loads a row when the rows are 4-byte aligned, bytes otherwise.
template <int D>
__device__ __forceinline__ int32_t dir_cost8(const uint8_t* blk, int64_t stride) {
  uint32_t w[8][4];
  if (((reinterpret_cast<uintptr_t>(blk) | (uintptr_t)stride) & 3) == 0) {
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const uint32_t* r = reinterpret_cast<const uint32_t*>(blk + i * stride);
      const uint32_t lo = r[0], hi = r[1];
      w[i][0] = __byte_perm(lo, 0, 0x4140), w[i][1] = __byte_perm(lo, 0, 0x4342);
      w[i][2] = __byte_perm(hi, 0, 0x4140), w[i][3] = __byte_perm(hi, 0, 0x4342);
    }
  } else {
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
      for (int m = 0; m < 4; m++) w[i][m] = blk[i * stride + 2 * m] | ((uint32_t)blk[i * stride + 2 * m + 1] << 16);
  }
  return dir_cost_pairs<D>(w, 0);
}

__device__ __forceinline__ int32_t dir_cost8_dev(int d, const uint8_t* blk, int64_t stride) {
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

size_t sel_smem_bytes(int nfb, bool rows);
cudaError_t launch_search(const SearchArgs& a, cudaStream_t st);
// The greedy selection for nb = 1..(1 << maxCfg) and the RD finish;
// everything stays on the device (no host round trip).
cudaError_t launch_select(SelArgs s, int maxCfg, unsigned long long lambda, uint8_t* fbIndex, FinishOut* fo,
                          cudaStream_t st);

// pf_mlp.cu: per-filter-block features of a.rec (X: [nfb][PF_MLP_FEATURES]);
// the frame means (features 33..39) only with frameMeans (the mask kernel
// computes them itself).
cudaError_t launch_features(const SearchArgs& a, int qindex, float* X, bool frameMeans, cudaStream_t st);
// pf_mlp.cu: the network over X and the tested-trial masks ([nfb][2]).
size_t mlp_expanded_bytes();  // fp32 copy of the network's parameters
// W: the fp32 copy, refreshed from dmodel first when `expand` is set.
cudaError_t launch_mlp_masks(const pf_cdef_mlp* dmodel, float* W, bool expand, const float* X, int nfb,
                             float threshold, int candidates, uint64_t* masks, cudaStream_t st);

}  // namespace pf
