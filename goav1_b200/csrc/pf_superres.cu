// pf_superres.cu - AV1 super-resolution upscaling on the GPU.
//
// superres.UpscalePlaneCoded (internal/av1/superres/superres.go:40-107) as
// the decoder runs it between CDEF and loop restoration
// (internal/av1/decoder/postfilter_superres.go:206-283): each plane's coded
// samples, read over the MI-aligned span (the columns past the crop are the
// genuine coded samples, not a clamp of the last cropped column), are
// resampled to the upscaled width with the normative 8-tap, 64-phase filter;
// the step and initial phase come from the cropped coded width
// (av1_get_upscale_convolve_step / get_upscale_convolve_x0 as restated there).
//
// One CTA per output row of one plane, the source row staged in shared
// memory; a thread per output sample.  The filter travels in the kernel
// arguments and is copied to shared memory (the 32 lanes of a warp read 32
// different phases, each as one 16-byte word).
#include <string.h>

#include "pf_common.cuh"
#include "pf_tables.h"

namespace pf {

constexpr int kSrScaleBits = 14, kSrExtraBits = kSrScaleBits - 6;

struct SrPlane {
  const uint8_t* src;
  int64_t sstride;
  uint8_t* dst;
  int64_t dstride;
  int srcWidth, dstWidth, rows, step, x0;
};

struct SrArgs {
  SrPlane pl[3];
  int nplanes, bd;
  int rowBase[4];  // prefix of the planes' rows over the grid
  int16_t filter[64][8];
};

// One output row.  The source row (the MI-aligned span) is staged in shared
// memory first; each output reads its phase's 8 taps as one 16-byte word.
template <typename T>
__device__ __forceinline__ void sr_row(const SrPlane& p, const uint8_t* srcRow, uint8_t* dstRow, const int16_t (*f)[8],
                                       uint16_t* s_row, int maxv) {
  const T* srow = reinterpret_cast<const T*>(srcRow);
  T* drow = reinterpret_cast<T*>(dstRow);
  const int last = p.srcWidth - 1;
  for (int x = threadIdx.x; x < p.srcWidth; x += blockDim.x) s_row[x] = srow[x];
  __syncthreads();
  for (int x = threadIdx.x; x < p.dstWidth; x += blockDim.x) {
    // superres.go:78-107 (upscaleRowPureGo).
    const int srcX = -(1 << kSrScaleBits) + p.x0 + x * p.step;
    const int px = srcX >> kSrScaleBits;
    const uint4 tw = *reinterpret_cast<const uint4*>(f[(srcX & ((1 << kSrScaleBits) - 1)) >> kSrExtraBits]);
    const int tap[8] = {(int16_t)(tw.x & 0xffff), (int16_t)(tw.x >> 16), (int16_t)(tw.y & 0xffff), (int16_t)(tw.y >> 16),
                        (int16_t)(tw.z & 0xffff), (int16_t)(tw.z >> 16), (int16_t)(tw.w & 0xffff), (int16_t)(tw.w >> 16)};
    const int base = px - 3;
    int sum = 0;
    if (base >= 0 && base + 7 <= last) {
#pragma unroll
      for (int k = 0; k < 8; k++) sum += (int)s_row[base + k] * tap[k];
    } else {
#pragma unroll
      for (int k = 0; k < 8; k++) sum += (int)s_row[iclip(base + k, 0, last)] * tap[k];
    }
    drow[x] = (T)iclip((sum + 64) >> 7, 0, maxv);
  }
}

// Rows of at most kSrMaxSpan source samples (the upscaler's frames are at
// most 16384 wide, so a coded span is at most 16384 * 8 / 9 + 8 samples).
constexpr int kSrMaxSpan = 14600;

__global__ void __launch_bounds__(256) k_superres(SrArgs a) {
  __shared__ __align__(16) int16_t s_f[64][8];
  extern __shared__ uint16_t s_row[];
  for (int i = threadIdx.x; i < 64 * 8; i += blockDim.x) s_f[i >> 3][i & 7] = a.filter[i >> 3][i & 7];
  const int r = blockIdx.x;
  int p = 0;
  while (p + 1 < a.nplanes && r >= a.rowBase[p + 1]) p++;
  const int y = r - a.rowBase[p];
  const int maxv = (1 << a.bd) - 1;
  const SrPlane& q = a.pl[p];
  const uint8_t* srow = q.src + (int64_t)y * q.sstride;
  uint8_t* drow = q.dst + (int64_t)y * q.dstride;
  if (a.bd == 8)
    sr_row<uint8_t>(q, srow, drow, s_f, s_row, maxv);
  else
    sr_row<uint16_t>(q, srow, drow, s_f, s_row, maxv);
}

// Restoration stripe-boundary rows of a super-resolved frame
// (tile/restoration_boundary.go:257-406, SaveRestorationBoundaryLinesFromFramePlaneSuperRes):
// the deblocked coded rows b-2 .. b+1 around each stripe boundary b are
// upscaled into the rows the restoration kernel reads (k*4 + j for boundary
// k; when row b+1 is past the plane, row b stands in for it, as
// finishRestorationBoundaryLines does).  One CTA per (plane, boundary, row).
struct SrLinesArgs {
  SrPlane pl[3];       // src: the deblocked coded plane; dst: the plane's lines, dstride per line
  int nb[3];           // boundary slots per plane
  int sh[3], off[3];   // stripe height and offset per plane
  int nplanes, bd;
  int16_t filter[64][8];
};

__global__ void __launch_bounds__(256) k_superres_lines(SrLinesArgs a) {
  __shared__ __align__(16) int16_t s_f[64][8];
  extern __shared__ uint16_t s_row[];
  for (int i = threadIdx.x; i < 64 * 8; i += blockDim.x) s_f[i >> 3][i & 7] = a.filter[i >> 3][i & 7];
  int r = blockIdx.x, p = 0;
  while (p + 1 < a.nplanes && r >= a.nb[p] * 4) {
    r -= a.nb[p] * 4;
    p++;
  }
  const int k = r >> 2, j = r & 3;
  const SrPlane& q = a.pl[p];
  const int b = k * a.sh[p] - a.off[p], y = b - 2 + j;
  // Block-uniform exits, before any barrier.
  if (k < 1 || b >= q.rows || y >= q.rows) return;
  const uint8_t* srow = q.src + (int64_t)y * q.sstride;
  uint8_t* line = q.dst + (int64_t)(k * 4 + j) * q.dstride;
  const int maxv = (1 << a.bd) - 1;
  if (a.bd == 8)
    sr_row<uint8_t>(q, srow, line, s_f, s_row, maxv);
  else
    sr_row<uint16_t>(q, srow, line, s_f, s_row, maxv);
  if (j == 2 && b + 1 >= q.rows) {
    // The stand-in row: copy what this CTA just wrote.
    __syncthreads();
    const int bps = a.bd == 8 ? 1 : 2;
    for (int x = threadIdx.x; x < q.dstWidth * bps; x += blockDim.x) line[q.dstride + x] = line[x];
  }
}

cudaError_t launch_superres_frame(const uint8_t* const* src, const int64_t* sstride, uint8_t* const* dst,
                                  const int64_t* dstride, const pf_frame* coded, int upW, cudaStream_t st);
cudaError_t launch_superres_lines(const uint8_t* const* src, const int64_t* sstride, uint8_t* const* lines,
                                  const int64_t* lstride, const int* nb, const pf_frame* coded, int upW,
                                  cudaStream_t st);

// Per-plane geometry of an upscale from `coded` (its width the coded width)
// to a plane width derived from upW.
static void sr_planes(const pf_frame* coded, int upW, int* cw, int* aw, int* dw, int* rows) {
  for (int p = 0; p < (coded->mono ? 1 : 3); p++) {
    const int sx = p ? coded->ss_x : 0, sy = p ? coded->ss_y : 0;
    cw[p] = (coded->width + sx) >> sx;
    aw[p] = ((coded->width + 7) & ~7) >> sx;
    dw[p] = (upW + sx) >> sx;
    rows[p] = (coded->height + sy) >> sy;
  }
}

static void sr_phase_dev(int coded, int dst, int* step, int* x0) {
  const int s = ((coded << kSrScaleBits) + dst / 2) / dst;
  const int err = dst * s - (coded << kSrScaleBits);
  int x = ((-((dst - coded) << (kSrScaleBits - 1))) + dst / 2) / dst;
  x += (1 << (kSrExtraBits - 1)) - err / 2;
  *step = s;
  *x0 = x & ((1 << kSrScaleBits) - 1);
}

cudaError_t launch_superres_lines(const uint8_t* const* src, const int64_t* sstride, uint8_t* const* lines,
                                  const int64_t* lstride, const int* nb, const pf_frame* coded, int upW,
                                  cudaStream_t st) {
  SrLinesArgs a;
  memset(&a, 0, sizeof(a));
  memcpy(a.filter, pf_superres_filter, sizeof(a.filter));
  int cw[3], aw[3], dw[3], rows[3], total = 0, span = 0;
  sr_planes(coded, upW, cw, aw, dw, rows);
  a.nplanes = coded->mono ? 1 : 3;
  a.bd = coded->bit_depth;
  for (int p = 0; p < a.nplanes; p++) {
    SrPlane& q = a.pl[p];
    sr_phase_dev(cw[p], dw[p], &q.step, &q.x0);
    q.src = src[p];
    q.sstride = sstride[p];
    q.dst = lines[p];
    q.dstride = lstride[p];
    q.srcWidth = aw[p];
    q.dstWidth = dw[p];
    q.rows = rows[p];
    const int sy = p ? coded->ss_y : 0;
    a.sh[p] = 64 >> sy;
    a.off[p] = 8 >> sy;
    a.nb[p] = lines[p] ? nb[p] : 0;
    total += a.nb[p] * 4;
    span = aw[p] > span ? aw[p] : span;
  }
  if (total == 0) return cudaSuccess;
  k_superres_lines<<<total, 256, (size_t)span * sizeof(uint16_t), st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_superres_frame(const uint8_t* const* src, const int64_t* sstride, uint8_t* const* dst,
                                  const int64_t* dstride, const pf_frame* coded, int upW, cudaStream_t st) {
  SrArgs a;
  memset(&a, 0, sizeof(a));
  memcpy(a.filter, pf_superres_filter, sizeof(a.filter));
  int cw[3], aw[3], dw[3], rows[3], span = 0;
  sr_planes(coded, upW, cw, aw, dw, rows);
  a.nplanes = coded->mono ? 1 : 3;
  a.bd = coded->bit_depth;
  for (int p = 0; p < a.nplanes; p++) {
    SrPlane& q = a.pl[p];
    sr_phase_dev(cw[p], dw[p], &q.step, &q.x0);
    q.src = src[p];
    q.sstride = sstride[p];
    q.dst = dst[p];
    q.dstride = dstride[p];
    q.srcWidth = aw[p];
    q.dstWidth = dw[p];
    q.rows = rows[p];
    a.rowBase[p + 1] = a.rowBase[p] + rows[p];
    span = aw[p] > span ? aw[p] : span;
  }
  k_superres<<<a.rowBase[a.nplanes], 256, (size_t)span * sizeof(uint16_t), st>>>(a);
  return cudaGetLastError();
}

}  // namespace pf

void* pf_internal_search_scratch(pf_ctx* c, size_t bytes);  // pf_api.cu
int pf_internal_wait(pf_ctx* c, void* stream);  // pf_api.cu: blocking or bounded by the context's deadline
void* pf_internal_stream(pf_ctx* c);

// Step and initial phase of one plane (superres.go:45-51).
static void sr_phase(int coded, int dst, int* step, int* x0) {
  const int s = ((coded << pf::kSrScaleBits) + dst / 2) / dst;
  const int err = dst * s - (coded << pf::kSrScaleBits);
  int x = ((-((dst - coded) << (pf::kSrScaleBits - 1))) + dst / 2) / dst;
  x += (1 << (pf::kSrExtraBits - 1)) - err / 2;
  *step = s;
  *x0 = x & ((1 << pf::kSrScaleBits) - 1);
}

extern "C" int pf_superres_upscale(pf_ctx* ctx, const pf_frame* coded, const pf_frame* upscaled) {
  using namespace pf;
  if (!ctx || !coded || !upscaled) return PF_ERR_INVALID_ARG;
  if (coded->memory > PF_MEM_DEVICE || coded->memory != upscaled->memory) return PF_ERR_INVALID_ARG;
  if (coded->bit_depth != 8 && coded->bit_depth != 10 && coded->bit_depth != 12) return PF_ERR_INVALID_FORMAT;
  if (coded->bit_depth != upscaled->bit_depth || coded->ss_x != upscaled->ss_x || coded->ss_y != upscaled->ss_y ||
      coded->mono != upscaled->mono || coded->height != upscaled->height || coded->width <= 0 ||
      coded->height <= 0 || upscaled->width <= coded->width || upscaled->width > 16384)
    return PF_ERR_INVALID_FORMAT;
  const int bps = coded->bit_depth > 8 ? 2 : 1;
  const int nplanes = coded->mono ? 1 : 3;
  SrArgs a;
  memset(&a, 0, sizeof(a));
  memcpy(a.filter, pf_superres_filter, sizeof(a.filter));
  a.nplanes = nplanes;
  a.bd = coded->bit_depth;
  int cw[3], aw[3], dw[3], rows[3];
  size_t hostBytes = 0;
  for (int p = 0; p < nplanes; p++) {
    const int sx = p ? coded->ss_x : 0, sy = p ? coded->ss_y : 0;
    cw[p] = (coded->width + sx) >> sx;
    aw[p] = ((coded->width + 7) & ~7) >> sx;  // the MI-aligned span the decoder reads
    dw[p] = (upscaled->width + sx) >> sx;
    rows[p] = (coded->height + sy) >> sy;
    const pf_plane &sp = coded->plane[p], &dp = upscaled->plane[p];
    if (!sp.data || !dp.data || sp.width != cw[p] || sp.height != rows[p] || sp.alloc_width < aw[p] ||
        sp.alloc_height < rows[p] || sp.stride < (int64_t)sp.alloc_width * bps || dp.width != dw[p] ||
        dp.height != rows[p] || dp.alloc_width < dw[p] || dp.alloc_height < rows[p] ||
        dp.stride < (int64_t)dp.alloc_width * bps)
      return PF_ERR_SHORT_BUFFER;
    a.rowBase[p + 1] = a.rowBase[p] + rows[p];
    hostBytes += ((size_t)aw[p] * bps + 255) / 256 * 256 * rows[p] + ((size_t)dw[p] * bps + 255) / 256 * 256 * rows[p];
  }
  const bool host = coded->memory == PF_MEM_HOST;
  const cudaStream_t st = (cudaStream_t)pf_internal_stream(ctx);
  uint8_t* scratch = nullptr;
  if (host) {
    scratch = (uint8_t*)pf_internal_search_scratch(ctx, hostBytes + 256);
    if (!scratch) return PF_ERR_DEVICE;
  }
  size_t off = 0;
  cudaError_t e = cudaSuccess;
  for (int p = 0; p < nplanes; p++) {
    SrPlane& q = a.pl[p];
    const pf_plane &sp = coded->plane[p], &dp = upscaled->plane[p];
    sr_phase(cw[p], dw[p], &q.step, &q.x0);
    q.srcWidth = aw[p];
    q.dstWidth = dw[p];
    q.rows = rows[p];
    if (host) {
      const int64_t ss = ((int64_t)aw[p] * bps + 255) / 256 * 256, ds = ((int64_t)dw[p] * bps + 255) / 256 * 256;
      q.src = scratch + off;
      q.sstride = ss;
      off += (size_t)ss * rows[p];
      q.dst = scratch + off;
      q.dstride = ds;
      off += (size_t)ds * rows[p];
      if (e == cudaSuccess)
        e = cudaMemcpy2DAsync((void*)q.src, ss, sp.data, sp.stride, (size_t)aw[p] * bps, rows[p],
                              cudaMemcpyHostToDevice, st);
    } else {
      q.src = (const uint8_t*)sp.data;
      q.sstride = sp.stride;
      q.dst = (uint8_t*)dp.data;
      q.dstride = dp.stride;
    }
  }
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  int span = 0;
  for (int p = 0; p < nplanes; p++) span = aw[p] > span ? aw[p] : span;
  if (span > kSrMaxSpan) return PF_ERR_INVALID_FORMAT;
  const size_t smem = (size_t)span * sizeof(uint16_t);  // at most 29 KB: no opt-in needed
  k_superres<<<a.rowBase[nplanes], 256, smem, st>>>(a);
  e = cudaGetLastError();
  if (host)
    for (int p = 0; p < nplanes && e == cudaSuccess; p++)
      e = cudaMemcpy2DAsync(upscaled->plane[p].data, upscaled->plane[p].stride, a.pl[p].dst, a.pl[p].dstride,
                            (size_t)dw[p] * bps, rows[p], cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return PF_ERR_DEVICE;
  return pf_internal_wait(ctx, st);
}
