// pf_diag.cu - measured instruction-issue ceilings for the integer roofline.
//
// The post-filter kernels are integer stencils whose time is set by how many
// warp instructions they issue, not by DRAM bytes.  Their roofline therefore
// needs a measured issue ceiling beside the copy bandwidth: this file runs
// fixed instruction streams over every SM and reports warp instructions per
// second.
//   kind 0: lop3.b32 only        (the integer ALU pipe: logic, add, min/max)
//   kind 1: mad.lo.u32 only      (the integer multiply-add path)
//   kind 2: the two interleaved
//   kind 3: fma.rn.f32 only      (the FP32 pipe, which accepts a warp
//                                 instruction every cycle: the issue ceiling
//                                 of one instruction per clock per SM
//                                 sub-partition)
// Each op is an inline-PTX instruction on a register the next op of its chain
// reads, with eight independent chains per thread and 2,048 threads per SM,
// so the count of issued instructions is the count written here (the loop's
// own counter and branch add under 2 %).
#include <cuda_runtime.h>
#include <stdint.h>

#include "goav1pf.h"

namespace {

constexpr int kOpsPerIter = 8 * 16;  // chains x unrolled rounds

__global__ void __launch_bounds__(256) k_issue_f32(uint32_t* sink, int iters, uint32_t salt) {
  float a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = (float)(threadIdx.x * (2 * k + 1) + blockIdx.x + salt) * 1e-3f;
  const float m = 0.999f + 1e-6f * (float)salt;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
      for (int k = 0; k < 8; k++) asm volatile("fma.rn.f32 %0, %0, %1, %2;" : "+f"(a[k]) : "f"(m), "f"(a[(k + 1) & 7]));
    }
  }
  float x = 0.f;
#pragma unroll
  for (int k = 0; k < 8; k++) x += a[k];
  if (x == 1234.5f) sink[blockIdx.x * blockDim.x + threadIdx.x] = 1u;  // keeps the chains live
}

template <int KIND>
__global__ void __launch_bounds__(256) k_issue(uint32_t* sink, int iters, uint32_t salt) {
  uint32_t a[8];
#pragma unroll
  for (int k = 0; k < 8; k++) a[k] = threadIdx.x * (2 * k + 1) + blockIdx.x + salt;
  const uint32_t m = 0x9E3779B1u ^ salt;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int r = 0; r < 16; r++) {
#pragma unroll
      for (int k = 0; k < 8; k++) {
        if (KIND == 0 || (KIND == 2 && (k & 1)))
          asm volatile("lop3.b32 %0, %0, %1, %2, 0x96;" : "+r"(a[k]) : "r"(m), "r"(a[(k + 1) & 7]));
        else
          asm volatile("mad.lo.u32 %0, %0, %1, %2;" : "+r"(a[k]) : "r"(m), "r"(a[(k + 1) & 7]));
      }
    }
  }
  uint32_t x = 0;
#pragma unroll
  for (int k = 0; k < 8; k++) x ^= a[k];
  if (x == 0x7f4a7c15u) sink[blockIdx.x * blockDim.x + threadIdx.x] = x;  // keeps the chains live
}

}  // namespace

extern "C" int pf_diag_issue_rate(int kind, double* warp_inst_per_s, double* ms) {
  if (kind < 0 || kind > 3 || !warp_inst_per_s) return PF_ERR_INVALID_ARG;
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return PF_ERR_DEVICE;
  const int threads = 256, blocks = sms * 8, iters = 2048;
  uint32_t* sink = nullptr;
  cudaStream_t st = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = PF_ERR_DEVICE;
  float best = 0.0f;
  if (cudaMalloc(&sink, sizeof(uint32_t) * blocks * threads) != cudaSuccess) return PF_ERR_DEVICE;
  if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess || cudaEventCreate(&e0) != cudaSuccess ||
      cudaEventCreate(&e1) != cudaSuccess)
    goto done;
  // One warm-up launch, then the fastest of three timed launches.
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(e0, st);
    if (kind == 0)
      k_issue<0><<<blocks, threads, 0, st>>>(sink, iters, (uint32_t)rep);
    else if (kind == 1)
      k_issue<1><<<blocks, threads, 0, st>>>(sink, iters, (uint32_t)rep);
    else if (kind == 2)
      k_issue<2><<<blocks, threads, 0, st>>>(sink, iters, (uint32_t)rep);
    else
      k_issue_f32<<<blocks, threads, 0, st>>>(sink, iters, (uint32_t)rep);
    cudaEventRecord(e1, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) goto done;
    float t = 0.0f;
    if (cudaEventElapsedTime(&t, e0, e1) != cudaSuccess) goto done;
    if (rep > 0 && (best == 0.0f || t < best)) best = t;
  }
  if (best > 0.0f) {
    const double warps = (double)blocks * threads / 32.0;
    *warp_inst_per_s = warps * iters * kOpsPerIter / (best * 1e-3);
    if (ms) *ms = best;
    rc = PF_OK;
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (st) cudaStreamDestroy(st);
  cudaFree(sink);
  return rc;
}
