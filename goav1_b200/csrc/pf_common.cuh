// pf_common.cuh - device-side frame views and launch parameter blocks shared
// by the post-filter kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "goav1pf.h"

namespace pf {

// One plane in device memory.  stride in bytes; w/h cropped; aw/ah allocated.
struct DPlane {
  uint8_t* ptr;
  int64_t stride;
  int w, h, aw, ah;
};

struct DFrame {
  DPlane pl[3];
  int width, height;  // cropped luma
  int bd, ssx, ssy, mono;
};

template <typename T>
__device__ __forceinline__ T* row_ptr(const DPlane& p, int y) {
  return reinterpret_cast<T*>(p.ptr + (int64_t)y * p.stride);
}

// Copies column x of rows y, y+step, ... < yEnd from one plane to another,
// four rows' loads issued before their stores (the planes may not alias).
template <typename T>
__device__ __forceinline__ void copy_column(const DPlane& from, const DPlane& to, int x, int y, int yEnd, int step) {
  for (; y < yEnd; y += 4 * step) {
    T v[4];
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (y + k * step < yEnd) v[k] = row_ptr<T>(from, y + k * step)[x];
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (y + k * step < yEnd) row_ptr<T>(to, y + k * step)[x] = v[k];
  }
}

// Copies the block [x0, x1) x [y0, y1) of one plane to another (the planes
// may not alias) with the whole CTA: 16-byte words, up to four per thread in
// flight, when both rows' starts and strides are 16-byte aligned and a row is
// a whole number of words; otherwise column by column.
template <typename T>
__device__ __forceinline__ void copy_block(const DPlane& from, const DPlane& to, int x0, int x1, int y0, int y1) {
  if (x1 <= x0 || y1 <= y0) return;
  const int rowBytes = (x1 - x0) * (int)sizeof(T);
  const uint8_t* s0 = from.ptr + (int64_t)y0 * from.stride + (int64_t)x0 * sizeof(T);
  uint8_t* d0 = to.ptr + (int64_t)y0 * to.stride + (int64_t)x0 * sizeof(T);
  if (((reinterpret_cast<uintptr_t>(s0) | reinterpret_cast<uintptr_t>(d0) | (uintptr_t)from.stride |
        (uintptr_t)to.stride | (uintptr_t)rowBytes) & 15) == 0) {
    const int wpr = rowBytes >> 4, total = (y1 - y0) * wpr;
    for (int i0 = threadIdx.x; i0 < total; i0 += 4 * blockDim.x) {
      uint4 v[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int i = i0 + k * blockDim.x;
        if (i < total) {
          const int r = i / wpr, c = i - r * wpr;
          v[k] = *reinterpret_cast<const uint4*>(s0 + (int64_t)r * from.stride + c * 16);
        }
      }
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int i = i0 + k * blockDim.x;
        if (i < total) {
          const int r = i / wpr, c = i - r * wpr;
          *reinterpret_cast<uint4*>(d0 + (int64_t)r * to.stride + c * 16) = v[k];
        }
      }
    }
    return;
  }
  const int w = x1 - x0;
  for (int i = threadIdx.x; i < w * (y1 - y0); i += blockDim.x) {
    const int r = i / w, c = i - r * w;
    row_ptr<T>(to, y0 + r)[x0 + c] = row_ptr<T>(from, y0 + r)[x0 + c];
  }
}

__host__ __device__ __forceinline__ int imin(int a, int b) { return a < b ? a : b; }
__host__ __device__ __forceinline__ int imax(int a, int b) { return a > b ? a : b; }
__host__ __device__ __forceinline__ int iclip(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// ---- per-frame parameter blocks (passed by value to kernels) ----

struct LfArgs {
  const uint16_t* masks;
  const uint8_t* level_cache;
  int sb128_w, sb128_h, mi_cols, mi_rows;
  int sharpness;
  int gate_chroma[3];  // 1 = skip plane (chroma gating)
};

struct CdefArgs {
  const uint8_t* index;
  const uint8_t* read;
  const uint8_t* noskip;  // may be null
  int index_stride, ucols, urows;
  int damping;
  int filter;           // 0 = copy only (CDEF stage off)
  int chroma_filtering;
  int plane_process[3];
  uint8_t y_strength[8], uv_strength[8];
  int strength_count;
  // Loop-restoration boundary lines (pre-CDEF rows), per plane.
  uint8_t* lines[3];    // [boundary k][4 rows][stride] samples of T
  int64_t line_stride[3];  // bytes per line row
  int save_lines[3];
  // constrain() of every 8-bit strength (0..15) and shift (0..7): table
  // [strength][shift] of 512 entries, entry 255 + d for a difference d in
  // -255..255 (entry 511 is 0).
  const int16_t* ctab;
};

struct LrArgs {
  const pf_lr_unit* units[3];
  int type[3];          // frame type per plane
  int unit_size[3];
  int horz[3], vert[3];
  const uint8_t* lines[3];
  int64_t line_stride[3];
};

struct FgArgs {
  int16_t* grain[3];      // 73*82 templates
  const uint8_t* offsets; // [rows][blocks] offsets of the stripe LFSRs
  int off_rows, off_cols;
  uint8_t lut[3][256];
  int active[3];
  int scaling_shift;
  int overlap;
  int clip_restricted;
  int matrix_identity;
  int cfl;
  int mult[3], luma_mult[3], offset[3];
  int odd_luma;
};

struct FgTemplateArgs {
  uint16_t seed;
  int bd;
  int num_y_points;
  int grain_scale_shift;
  int lag, coeff_shift;
  int8_t coeffs[3][25];
  int active[3];
  int ssx, ssy;
};

// ---- batched execution: one launch per stage over the frames of a batch ----

enum Stage {
  ST_FG_TEMPLATES = 0,
  ST_DEBLOCK_V,
  ST_DEBLOCK_H,
  ST_CDEF,
  ST_LR,
  ST_EXTEND,
  ST_FG_OFFSETS,
  ST_FG_APPLY,
  ST_COUNT
};

// Work items of a stage are numbered frame after frame; base[f] is the first
// item of frame f (base[n] = total).  Each stage decodes its local index.
struct FrameJob {
  DFrame io;    // the frame, filtered in place
  DFrame scr;   // CDEF output scratch (same geometry)
  DFrame disp;  // film-grain display frame
  LfArgs lf;
  CdefArgs cdef;
  LrArgs lr;
  FgArgs fg;
  FgTemplateArgs fgt;
  int aw[3], ah[3];          // MI-aligned plane extents
  int db_tile;               // deblocking tile shape (db_tile_w / db_tile_h)
  int db_tx[3], db_ty[3];    // deblock tiles per plane (0 = gated)
  int lr_cols[3], lr_rows[3];  // restoration tiles (processing column x stripe)
  int fg_tx[3], fg_ty[3];    // 64x64-sample tiles of the display planes
  int ext_r[3][2], ext_b[3][2];  // extension tiles: right strip, bottom strip
  int do_lr;
};

struct BatchArgs {
  const FrameJob* jobs;
  const int* base;  // ST_COUNT arrays of n+1 ints, stage-major
  int n;
  int* counters;    // ST_COUNT work counters (persistent mode), or null
  // The launch's schedule (pf_schedule): consecutive work items a CTA takes
  // at a time (one launch grid slot, or one counter grab when persistent),
  // and how many items ahead of the current one the CTA prefetches into L2.
  int chunk;
  int ahead;
  int tile;  // the stage's tile setting (pf_schedule.tile; deblocking reads it from the job)
  // The frames [f0, f1) this launch covers (a frame group of the batch;
  // items base[f0] .. base[f1] - 1 of each stage).
  int f0, f1;
  // CTAs of this launch resident at once (SMs x CTAs per SM): with one item
  // per CTA, `ahead` counts in these waves.
  int wave;
};

// Deblocking tile shapes (pf_schedule.tile): width x height in 4x4 edge
// units, 256 units (one per thread) a tile.
__host__ __device__ __forceinline__ int db_tile_w(int tile) { return tile == 1 ? 64 : tile == 2 ? 16 : tile == 3 ? 8 : 32; }
__host__ __device__ __forceinline__ int db_tile_h(int tile) { return 256 / db_tile_w(tile); }

// Prefetches the samples [x0, x1) x [y0, y1) of a plane (clamped to its
// allocation) into L2, one 128-byte line per thread at a time.  A hint only:
// nothing is read into registers and nothing is ordered.
template <typename T>
__device__ __forceinline__ void prefetch_block(const DPlane& p, int x0, int x1, int y0, int y1) {
  x0 = x0 < 0 ? 0 : x0;
  y0 = y0 < 0 ? 0 : y0;
  x1 = x1 > p.aw ? p.aw : x1;
  y1 = y1 > p.ah ? p.ah : y1;
  if (x1 <= x0 || y1 <= y0) return;
  const uintptr_t row0 = reinterpret_cast<uintptr_t>(p.ptr) + (uintptr_t)x0 * sizeof(T);
  const uintptr_t l0 = row0 & ~(uintptr_t)127;
  const int lines = (int)(((row0 + (uintptr_t)(x1 - x0) * sizeof(T) - 1) >> 7) - (l0 >> 7)) + 1;
  const int n = lines * (y1 - y0);
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int r = i / lines, l = i - r * lines;
    const uintptr_t a = ((row0 + (uintptr_t)(y0 + r) * (uintptr_t)p.stride) & ~(uintptr_t)127) + (uintptr_t)l * 128;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(a));
  }
}

__device__ __forceinline__ int find_frame(const int* base, int n, int item) {
  int lo = 0, hi = n;  // base[lo] <= item < base[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&base[mid]) <= item) lo = mid; else hi = mid;
  }
  return lo;
}

// Runs f(item) for the CTA's work items: a chunk of b.chunk consecutive
// items per CTA (grid = ceil(total / chunk)), or a persistent CTA draining
// the stage's queue a chunk at a time through an atomic counter.  Inside a
// chunk, prefetch(item) warms L2 with the input of the item b.ahead places
// on.  Every item is independent of the others, so no schedule changes a
// result.  The loop's position lives in shared memory, so that nothing but
// f's own state is held in registers across f.
// kLoop = false compiles only the one-item-per-CTA schedule (the launcher's
// choice when the stage has no chunks and no persistent CTAs), which keeps
// the loop's bookkeeping out of the kernel's register allocation.
template <bool kLoop = true, typename F, typename P>
__device__ __forceinline__ void for_each_item(const BatchArgs& b, int stage, F f, P prefetch) {
  const int* base = b.base + stage * (b.n + 1);
  const int lo = __ldg(&base[b.f0]), total = __ldg(&base[b.f1]);
  const int chunk = b.chunk > 1 ? b.chunk : 1;
  int* counter = b.counters ? b.counters + stage : nullptr;
  if (!kLoop || (counter == nullptr && chunk == 1)) {
    // One item per CTA: the item `ahead` waves on, which a CTA starting
    // about when this one ends will take, is prefetched first.
    const int it = lo + (int)blockIdx.x;
    if (b.ahead > 0) {
      const int next = it + b.ahead * b.wave;
      if (next < total) prefetch(next);
    }
    if (it < total) f(it);
    return;
  }
  // Next item, end of the chunk, first item of the chunk, end of the
  // range, chunk, start of the range.
  __shared__ int s_pos[6];
  if (threadIdx.x == 0) {
    const int first = lo + (counter ? atomicAdd(counter, chunk) : (int)blockIdx.x * chunk);
    s_pos[0] = s_pos[2] = first;
    s_pos[1] = first + chunk < total ? first + chunk : total;
    s_pos[3] = total;
    s_pos[4] = chunk;
    s_pos[5] = lo;
  }
  __syncthreads();
  for (;;) {
    int it = s_pos[0];
    if (it >= s_pos[1]) {
      // Chunk done: the next one (persistent CTAs) or the end.
      if (b.counters == nullptr) break;
      __syncthreads();
      if (threadIdx.x == 0) {
        const int n = s_pos[3], c = s_pos[4];
        const int first = s_pos[5] + atomicAdd(b.counters + stage, c);
        s_pos[0] = s_pos[2] = first;
        s_pos[1] = first + c < n ? first + c : n;
      }
      __syncthreads();
      it = s_pos[0];
      if (it >= s_pos[3]) break;
    }
    if (b.ahead > 0) {
      const int last = s_pos[1];
      if (it == s_pos[2])
        for (int k = 1; k <= b.ahead && it + k < last; k++) prefetch(it + k);
      else if (it + b.ahead < last)
        prefetch(it + b.ahead);
    }
    f(it);
    __syncthreads();
    if (threadIdx.x == 0) s_pos[0] = s_pos[0] + 1;
    __syncthreads();
  }
}

template <bool kLoop = true, typename F>
__device__ __forceinline__ void for_each_item(const BatchArgs& b, int stage, F f) {
  auto none = [](int) {};
  for_each_item<kLoop>(b, stage, f, none);
}

// Whether a launch needs the looping form of for_each_item.
inline bool batch_loops(const BatchArgs& b) { return b.counters != nullptr || b.chunk > 1; }

// CTAs of `kernel` the current device holds at once (SMs x CTAs per SM at
// `threads` threads and `smem` dynamic shared bytes): a launch's wave.
template <class K>
inline int resident_ctas(K kernel, int threads, size_t smem) {
  int occ = 0, dev = 0, sms = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, threads, smem) != cudaSuccess || occ < 1) {
    (void)cudaGetLastError();
    occ = 1;
  }
  return occ * (sms > 0 ? sms : 1);
}

// The launch arguments with `wave` filled in when the one-item-per-CTA form
// prefetches waves ahead (the count is settled once per kernel).
template <class K>
inline BatchArgs with_wave(const BatchArgs& b, K kernel, int threads, size_t smem, int& cached) {
  BatchArgs a = b;
  if (a.ahead > 0 && !batch_loops(a)) {
    if (!cached) cached = resident_ctas(kernel, threads, smem);
    a.wave = cached;
  }
  return a;
}

}  // namespace pf
