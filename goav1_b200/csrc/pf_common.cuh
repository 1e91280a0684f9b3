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
  int db_tx[3], db_ty[3];    // deblock tiles (32x8 edge units) per plane (0 = gated)
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
};

__device__ __forceinline__ int find_frame(const int* base, int n, int item) {
  int lo = 0, hi = n;  // base[lo] <= item < base[hi]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (__ldg(&base[mid]) <= item) lo = mid; else hi = mid;
  }
  return lo;
}

// Runs f(item) for the CTA's work items: one item per CTA (grid = total), or
// a persistent CTA draining the stage's queue through an atomic counter.
template <typename F>
__device__ __forceinline__ void for_each_item(int total, int* counter, F f) {
  if (counter == nullptr) {
    if ((int)blockIdx.x < total) f((int)blockIdx.x);
    return;
  }
  __shared__ int s_item;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= total) break;
    f(it);
  }
}

}  // namespace pf
