// pf_api.cu - the C ABI of the B200 post-filter chain (include/goav1pf.h).
//
// Replaces goav1's decoderFrameWorkReusableSupportedPostFilterRunner
// (decoder_postfilter_bind.go:398-440): validate everything before touching
// the frame (postfilter.go:596-613), then run deblock -> CDEF (with the
// loop-restoration boundary-line save fused in) -> loop restoration ->
// border extension on the reference frame in place, and film grain into the
// display frame (postfilter.go:589-782, :810-842).
//
// Buffers: the frame is deblocked in place; CDEF writes a scratch frame the
// context owns; loop restoration (or a plain copy when it is off) writes the
// result back into the frame.  Host frames are staged through device buffers
// the context keeps and grows; nothing is allocated per call once warm.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pf_common.cuh"

namespace pf {
cudaError_t launch_deblock(const DFrame& f, const LfArgs& a, cudaStream_t st);
cudaError_t launch_cdef(const DFrame& in, const DFrame& out, const CdefArgs& a, cudaStream_t st);
cudaError_t launch_lr(const DFrame& src, const DFrame& dst, const LrArgs& a, int enabled, cudaStream_t st);
cudaError_t lr_upload_tables();
cudaError_t fg_upload_tables();
cudaError_t launch_fg_templates(const FgTemplateArgs& p, int16_t* gy, int16_t* gu, int16_t* gv, cudaStream_t st);
cudaError_t launch_fg_offsets(uint16_t seed, int rows, int cols, uint8_t* out, cudaStream_t st);
cudaError_t launch_fg_apply(const DFrame& ref, const DFrame& disp, const FgArgs& a, cudaStream_t st);
cudaError_t launch_extend(const DFrame& f, cudaStream_t st);
}  // namespace pf

using namespace pf;

namespace {

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  cudaError_t ensure(size_t need) {
    if (need <= n) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
    need = (need + 4095) & ~(size_t)4095;
    cudaError_t e = cudaMalloc(&p, need);
    if (e == cudaSuccess) n = need;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
};

int bps_of(const pf_frame* f) { return f->bit_depth > 8 ? 2 : 1; }

}  // namespace

struct pf_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int timing = 0;
  cudaEvent_t ev[6] = {};
  DevBuf io, disp, scratch, lines, grain, offsets;
  DevBuf masks, lc, index, read, noskip, units[3];
};

// ---------------------------------------------------------------------------
// Validation (no device work; mirrors the reference's error taxonomy).

static int plane_dims_ok(const pf_frame* f) {
  if (f->bit_depth != 8 && f->bit_depth != 10 && f->bit_depth != 12) return 0;
  if (f->ss_x > 1 || f->ss_y > 1 || f->mono > 1 || f->width <= 0 || f->height <= 0) return 0;
  if (f->mono) return 0;  // monochrome frames are not supported by this runner
  const int bps = bps_of(f);
  for (int p = 0; p < 3; p++) {
    const pf_plane& pl = f->plane[p];
    const int sx = p ? f->ss_x : 0, sy = p ? f->ss_y : 0;
    const int w = (f->width + sx) >> sx, h = (f->height + sy) >> sy;
    if (!pl.data || pl.width != w || pl.height != h) return 0;
    const int aw8 = ((f->width + 7) & ~7) >> sx, ah8 = ((f->height + 7) & ~7) >> sy;
    if (pl.alloc_width < aw8 || pl.alloc_height < ah8) return 0;
    if (pl.stride < (int64_t)pl.alloc_width * bps) return 0;
    if (bps == 2 && ((uintptr_t)pl.data & 1)) return 0;
  }
  return 1;
}

static int frames_same_geometry(const pf_frame* a, const pf_frame* b) {
  if (a->width != b->width || a->height != b->height || a->bit_depth != b->bit_depth || a->ss_x != b->ss_x ||
      a->ss_y != b->ss_y || a->mono != b->mono)
    return 0;
  for (int p = 0; p < 3; p++)
    if (a->plane[p].alloc_width != b->plane[p].alloc_width || a->plane[p].alloc_height != b->plane[p].alloc_height)
      return 0;
  return 1;
}

static void lr_grid(const pf_frame* f, const pf_restoration& lr, int p, int* horz, int* vert, int* us) {
  const int sx = p ? f->ss_x : 0, sy = p ? f->ss_y : 0;
  const int W = (f->width + sx) >> sx, H = (f->height + sy) >> sy;
  *us = p ? lr.unit_size_uv : lr.unit_size_y;
  *horz = *vert = 0;
  if (lr.type[p] == PF_LR_NONE || *us == 0) return;
  int h = (W + (*us >> 1)) / *us, v = (H + (*us >> 1)) / *us;
  *horz = h ? h : 1;
  *vert = v ? v : 1;
}

extern "C" int pf_frame_validate(const pf_frame* f, const pf_frame_side* s, const pf_frame* display) {
  if (!f || !s) return PF_ERR_INVALID_ARG;
  if (s->stages & ~0x1Fu) return PF_ERR_UNSUPPORTED;
  if (f->memory > PF_MEM_DEVICE || s->side_memory > PF_MEM_DEVICE) return PF_ERR_INVALID_ARG;
  if (!plane_dims_ok(f)) return PF_ERR_SHORT_BUFFER;
  const bool hostSide = s->side_memory == PF_MEM_HOST;
  const int miCols = ((f->width + 7) >> 3) << 1, miRows = ((f->height + 7) >> 3) << 1;
  if (s->stages & PF_STAGE_LOOP_FILTER) {
    const pf_loop_filter& lf = s->lf;
    if (lf.sharpness > 7 || lf.level_y[0] > 63 || lf.level_y[1] > 63 || lf.level_u > 63 || lf.level_v > 63)
      return PF_ERR_INVALID_FILTER;
    if (!lf.masks || !lf.level_cache || lf.mi_cols != miCols || lf.mi_rows != miRows ||
        lf.sb128_w != (miCols + 31) / 32 || lf.sb128_h != (miRows + 31) / 32)
      return PF_ERR_INVALID_FILTER;
    if (hostSide) {
      for (int i = 0; i < 4 * miCols * miRows; i++)
        if (lf.level_cache[i] > 63) return PF_ERR_INVALID_FILTER;
    }
  }
  const int ucols = (f->width + 63) / 64, urows = (f->height + 63) / 64;
  if (s->stages & PF_STAGE_CDEF) {
    const pf_cdef& c = s->cdef;
    if (c.strength_count == 0 || c.strength_count > 8 || c.damping < 3 || c.damping > 6) return PF_ERR_INVALID_CDEF;
    for (int i = 0; i < c.strength_count; i++)
      if (c.y_strength[i] > 0x3f || c.uv_strength[i] > 0x3f) return PF_ERR_INVALID_CDEF;
    if (!c.index || !c.read || c.index_stride < ucols || c.index_rows < urows) return PF_ERR_INVALID_CDEF;
    if (hostSide) {
      for (int r = 0; r < urows; r++)
        for (int k = 0; k < ucols; k++)
          if (c.read[r * c.index_stride + k] && c.index[r * c.index_stride + k] >= c.strength_count)
            return PF_ERR_INVALID_CDEF;
    }
  }
  if (s->stages & PF_STAGE_LOOP_RESTORATION) {
    const pf_restoration& lr = s->lr;
    for (int p = 0; p < 3; p++) {
      if (lr.type[p] > PF_LR_SGRPROJ) return PF_ERR_INVALID_PLAN;
      if (lr.type[p] == PF_LR_NONE) continue;
      int horz, vert, us;
      lr_grid(f, lr, p, &horz, &vert, &us);
      const int minUs = p ? (64 >> std::max((int)f->ss_x, (int)f->ss_y)) : 64;
      if (us < minUs || us > 256 || (us & (us - 1))) return PF_ERR_INVALID_PLAN;
      if (!lr.units[p] || lr.unit_count[p] < horz * vert) return PF_ERR_INVALID_PLAN;
      if (hostSide) {
        for (int i = 0; i < horz * vert; i++) {
          const pf_lr_unit& u = lr.units[p][i];
          if (u.type == PF_LR_NONE) continue;
          if (u.type != PF_LR_WIENER && u.type != PF_LR_SGRPROJ) return PF_ERR_INVALID_PLAN;
          if (lr.type[p] != PF_LR_SWITCHABLE && u.type != lr.type[p]) return PF_ERR_INVALID_PLAN;
          if (u.type == PF_LR_SGRPROJ && u.sgr_set > 15) return PF_ERR_INVALID_PLAN;
          if (u.type == PF_LR_WIENER) {
            for (int k = 0; k < 2; k++) {
              const int8_t* t = k ? u.wiener_h : u.wiener_v;
              if (t[0] < -5 || t[0] > 10 || t[1] < -23 || t[1] > 8 || t[2] < -17 || t[2] > 46)
                return PF_ERR_INVALID_PLAN;
            }
          }
        }
      }
    }
  }
  if (s->stages & PF_STAGE_FILM_GRAIN) {
    const pf_film_grain& g = s->fg;
    if (g.apply) {
      if (g.num_y_points > 14 || g.num_cb_points > 10 || g.num_cr_points > 10 || g.ar_coeff_lag > 3 ||
          g.grain_scale_shift > 3)
        return PF_ERR_INVALID_FORMAT;
      const bool active = g.num_y_points || g.num_cb_points || g.num_cr_points || g.chroma_scaling_from_luma;
      if (active && (g.scaling_shift < 8 || g.scaling_shift > 11)) return PF_ERR_INVALID_FORMAT;
      if (active && (g.ar_coeff_lag > 0 || g.num_y_points) && (g.ar_coeff_shift < 6 || g.ar_coeff_shift > 9))
        return PF_ERR_INVALID_FORMAT;
      const uint8_t(*sets[3])[2] = {g.y_points, g.cb_points, g.cr_points};
      const int counts[3] = {g.num_y_points, g.num_cb_points, g.num_cr_points};
      for (int k = 0; k < 3; k++)
        for (int i = 1; i < counts[k]; i++)
          if (sets[k][i][0] <= sets[k][i - 1][0]) return PF_ERR_INVALID_FORMAT;
    }
    if (!display) return PF_ERR_INVALID_ARG;
    if (display->memory > PF_MEM_DEVICE || !plane_dims_ok(display) || !frames_same_geometry(f, display))
      return PF_ERR_SHORT_BUFFER;
  }
  return PF_OK;
}

// ---------------------------------------------------------------------------

static DFrame dframe_from(const pf_frame* f, void* const* ptrs, const int64_t* strides) {
  DFrame d;
  memset(&d, 0, sizeof(d));
  d.width = f->width;
  d.height = f->height;
  d.bd = f->bit_depth;
  d.ssx = f->ss_x;
  d.ssy = f->ss_y;
  d.mono = f->mono;
  for (int p = 0; p < 3; p++) {
    d.pl[p].ptr = (uint8_t*)ptrs[p];
    d.pl[p].stride = strides[p];
    d.pl[p].w = f->plane[p].width;
    d.pl[p].h = f->plane[p].height;
    d.pl[p].aw = f->plane[p].alloc_width;
    d.pl[p].ah = f->plane[p].alloc_height;
  }
  return d;
}

// Lays out a device frame with f's geometry inside buf (each plane 256-byte
// aligned, stride rounded to 256 bytes).
static cudaError_t layout_like(const pf_frame* f, DevBuf& buf, void** ptrs, int64_t* strides) {
  const int bps = bps_of(f);
  size_t off[3], total = 0;
  for (int p = 0; p < 3; p++) {
    strides[p] = ((int64_t)f->plane[p].alloc_width * bps + 255) & ~(int64_t)255;
    off[p] = total;
    total += (size_t)strides[p] * f->plane[p].alloc_height;
    total = (total + 255) & ~(size_t)255;
  }
  cudaError_t e = buf.ensure(total);
  if (e != cudaSuccess) return e;
  for (int p = 0; p < 3; p++) ptrs[p] = (uint8_t*)buf.p + off[p];
  return cudaSuccess;
}

template <typename TT>
static const TT* side_ptr(pf_ctx* c, DevBuf& b, const TT* src, size_t bytes, bool host, cudaError_t* e) {
  if (!host || !src) return src;
  *e = b.ensure(bytes);
  if (*e != cudaSuccess) return nullptr;
  *e = cudaMemcpyAsync(b.p, src, bytes, cudaMemcpyHostToDevice, c->stream);
  return (const TT*)b.p;
}

static void build_scaling_lut(uint8_t* dst, const uint8_t (*pts)[2], int n) {
  // filmgrain/scaling.go:18-48 (BuildScalingLUT).
  memset(dst, 0, 256);
  if (n == 0) return;
  for (int x = 0; x < pts[0][0]; x++) dst[x] = pts[0][1];
  for (int p = 0; p < n - 1; p++) {
    const int dy = pts[p + 1][1] - pts[p][1], dx = pts[p + 1][0] - pts[p][0];
    const int64_t delta = (int64_t)dy * ((65536 + (dx >> 1)) / dx);
    for (int x = 0; x < dx; x++) dst[pts[p][0] + x] = (uint8_t)(pts[p][1] + (int)(((int64_t)x * delta + 32768) >> 16));
  }
  for (int x = pts[n - 1][0]; x < 256; x++) dst[x] = pts[n - 1][1];
}

#define CK(expr)                       \
  do {                                 \
    cudaError_t _e = (expr);           \
    if (_e != cudaSuccess) {           \
      last_error(_e);                  \
      return PF_ERR_DEVICE;            \
    }                                  \
  } while (0)

static void last_error(cudaError_t e) {
  if (getenv("PF_DEBUG")) fprintf(stderr, "goav1pf: CUDA error %s\n", cudaGetErrorString(e));
}

extern "C" int pf_abi_version(void) { return PF_ABI_VERSION; }

extern "C" const char* pf_status_string(int s) {
  switch (s) {
    case PF_OK: return "ok";
    case PF_ERR_INVALID_CDEF: return "cdef: invalid input";
    case PF_ERR_INVALID_FILTER: return "loopfilter: invalid filter";
    case PF_ERR_INVALID_PLAN: return "restoration: invalid plan";
    case PF_ERR_UNSUPPORTED: return "decoder: unsupported post-filter";
    case PF_ERR_SHORT_BUFFER: return "frame: short buffer";
    case PF_ERR_INVALID_FORMAT: return "frame: invalid format";
    case PF_ERR_INVALID_ARG: return "invalid argument";
    case PF_ERR_DEVICE: return "CUDA error";
    case PF_ERR_TIMEOUT: return "device wait timed out";
    case PF_ERR_NO_DEVICE: return "no usable CUDA device";
    default: return "unknown status";
  }
}

extern "C" pf_ctx* pf_create(const pf_config* cfg, int* status) {
  int dev = cfg ? cfg->device : 0;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= dev) {
    if (status) *status = PF_ERR_NO_DEVICE;
    return nullptr;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess || prop.major < 10) {
    if (status) *status = PF_ERR_NO_DEVICE;
    return nullptr;
  }
  if (cudaSetDevice(dev) != cudaSuccess) {
    if (status) *status = PF_ERR_DEVICE;
    return nullptr;
  }
  pf_ctx* c = new pf_ctx();
  c->device = dev;
  c->timing = cfg ? cfg->timing : 0;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess || lr_upload_tables() != cudaSuccess ||
      fg_upload_tables() != cudaSuccess) {
    delete c;
    if (status) *status = PF_ERR_DEVICE;
    return nullptr;
  }
  for (int i = 0; i < 6; i++) cudaEventCreate(&c->ev[i]);
  if (status) *status = PF_OK;
  return c;
}

extern "C" void pf_destroy(pf_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  DevBuf* bufs[] = {&c->io, &c->disp, &c->scratch, &c->lines, &c->grain, &c->offsets, &c->masks,
                    &c->lc, &c->index, &c->read, &c->noskip, &c->units[0], &c->units[1], &c->units[2]};
  for (DevBuf* b : bufs) b->release();
  for (int i = 0; i < 6; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" int pf_sync(pf_ctx* c) {
  if (!c) return PF_ERR_INVALID_ARG;
  return cudaStreamSynchronize(c->stream) == cudaSuccess ? PF_OK : PF_ERR_DEVICE;
}

extern "C" void* pf_stream(pf_ctx* c) { return c ? (void*)c->stream : nullptr; }

// Queues the chain for one validated frame whose planes are at io (device).
static int run_chain(pf_ctx* c, const pf_frame* f, const DFrame& io, const pf_frame_side* s, const DFrame* disp,
                     pf_stats* stats) {
  const cudaStream_t st = c->stream;
  const bool host = s->side_memory == PF_MEM_HOST;
  const int bps = bps_of(f);
  cudaError_t e = cudaSuccess;
  const int miCols = ((f->width + 7) >> 3) << 1, miRows = ((f->height + 7) >> 3) << 1;
  const int ucols = (f->width + 63) / 64, urows = (f->height + 63) / 64;
  uint32_t done = 0;
  if (c->timing) cudaEventRecord(c->ev[0], st);

  // ---- deblocking ----
  if (s->stages & PF_STAGE_LOOP_FILTER) {
    const pf_loop_filter& lf = s->lf;
    LfArgs a;
    memset(&a, 0, sizeof(a));
    a.masks = side_ptr(c, c->masks, lf.masks, (size_t)lf.sb128_w * lf.sb128_h * PF_LF_MASK_WORDS * 2, host, &e);
    CK(e);
    a.level_cache = side_ptr(c, c->lc, lf.level_cache, (size_t)4 * miCols * miRows, host, &e);
    CK(e);
    a.sb128_w = lf.sb128_w;
    a.sb128_h = lf.sb128_h;
    a.mi_cols = lf.mi_cols;
    a.mi_rows = lf.mi_rows;
    a.sharpness = lf.sharpness;
    const bool lumaZero = lf.level_y[0] == 0 && lf.level_y[1] == 0;
    a.gate_chroma[0] = 0;
    a.gate_chroma[1] = f->mono || lumaZero || lf.level_u == 0;
    a.gate_chroma[2] = f->mono || lumaZero || lf.level_v == 0;
    CK(launch_deblock(io, a, st));
    done |= PF_STAGE_LOOP_FILTER;
  }
  if (c->timing) cudaEventRecord(c->ev[1], st);

  // ---- CDEF (+ LR boundary lines) ----
  const bool doLR = (s->stages & PF_STAGE_LOOP_RESTORATION) &&
                    (s->lr.type[0] != PF_LR_NONE || s->lr.type[1] != PF_LR_NONE || s->lr.type[2] != PF_LR_NONE);
  bool cdefAny = false;
  const pf_cdef& cd = s->cdef;
  if (s->stages & PF_STAGE_CDEF) {
    for (int i = 0; i < std::min((int)cd.strength_count, 8); i++)
      if (cd.y_strength[i] || (!f->mono && cd.uv_strength[i])) cdefAny = true;
  }
  void* sptr[3];
  int64_t sstride[3];
  DFrame B;
  if (cdefAny || doLR) {
    CK(layout_like(f, c->scratch, sptr, sstride));
    B = dframe_from(f, sptr, sstride);
    CdefArgs a;
    memset(&a, 0, sizeof(a));
    a.filter = cdefAny ? 1 : 0;
    a.ucols = ucols;
    a.urows = urows;
    std::vector<uint8_t> zeros;
    if (cdefAny) {
      a.index = side_ptr(c, c->index, cd.index, (size_t)cd.index_stride * cd.index_rows, host, &e);
      CK(e);
      a.read = side_ptr(c, c->read, cd.read, (size_t)cd.index_stride * cd.index_rows, host, &e);
      CK(e);
      a.noskip = cd.noskip ? side_ptr(c, c->noskip, cd.noskip, (size_t)ucols * urows * 8, host, &e) : nullptr;
      CK(e);
      a.index_stride = cd.index_stride;
    } else {
      // Copy-only pass: an all-zero Read map (no unit filters).
      CK(c->read.ensure((size_t)ucols * urows));
      CK(cudaMemsetAsync(c->read.p, 0, (size_t)ucols * urows, st));
      a.read = (const uint8_t*)c->read.p;
      a.index = (const uint8_t*)c->read.p;
      a.index_stride = ucols;
    }
    a.damping = cd.damping;
    a.strength_count = cd.strength_count;
    for (int i = 0; i < 8; i++) {
      a.y_strength[i] = cd.y_strength[i];
      a.uv_strength[i] = cd.uv_strength[i];
    }
    bool uvAny = false, yAny = false;
    for (int i = 0; i < std::min((int)cd.strength_count, 8); i++) {
      uvAny |= cd.uv_strength[i] != 0;
      yAny |= cd.y_strength[i] != 0;
    }
    a.chroma_filtering = !f->mono && uvAny;
    a.plane_process[0] = yAny || a.chroma_filtering;
    a.plane_process[1] = a.plane_process[2] = uvAny;
    if (doLR) {
      size_t total = 0;
      size_t offs[3];
      for (int p = 0; p < 3; p++) {
        offs[p] = total;
        if (s->lr.type[p] == PF_LR_NONE) continue;
        const int sy = p ? f->ss_y : 0;
        const int SH = 64 >> sy, off = 8 >> sy;
        const int nb = (f->plane[p].height + off) / SH + 2;
        const int64_t ls = ((int64_t)f->plane[p].width * bps + 255) & ~(int64_t)255;
        a.line_stride[p] = ls;
        total += (size_t)nb * 4 * ls;
      }
      CK(c->lines.ensure(total));
      for (int p = 0; p < 3; p++) {
        if (s->lr.type[p] == PF_LR_NONE) continue;
        a.lines[p] = (uint8_t*)c->lines.p + offs[p];
        a.save_lines[p] = 1;
      }
    }
    CK(launch_cdef(io, B, a, st));
    if (cdefAny) done |= PF_STAGE_CDEF;
    if (c->timing) cudaEventRecord(c->ev[2], st);
    // ---- loop restoration (or copy back) ----
    LrArgs la;
    memset(&la, 0, sizeof(la));
    if (doLR) {
      for (int p = 0; p < 3; p++) {
        la.type[p] = s->lr.type[p];
        if (la.type[p] == PF_LR_NONE) continue;
        int horz, vert, us;
        lr_grid(f, s->lr, p, &horz, &vert, &us);
        la.horz[p] = horz;
        la.vert[p] = vert;
        la.unit_size[p] = us;
        la.units[p] = side_ptr(c, c->units[p], s->lr.units[p], sizeof(pf_lr_unit) * horz * vert, host, &e);
        CK(e);
        la.lines[p] = a.lines[p];
        la.line_stride[p] = a.line_stride[p];
      }
    }
    CK(launch_lr(B, io, la, doLR ? 1 : 0, st));
    if (doLR) done |= PF_STAGE_LOOP_RESTORATION;
  } else if (c->timing) {
    cudaEventRecord(c->ev[2], st);
  }
  if (c->timing) cudaEventRecord(c->ev[3], st);

  // ---- border extension ----
  if (s->stages & PF_STAGE_EXTEND_BORDERS) {
    CK(launch_extend(io, st));
    done |= PF_STAGE_EXTEND_BORDERS;
  }
  if (c->timing) cudaEventRecord(c->ev[4], st);

  // ---- film grain into the display frame ----
  if ((s->stages & PF_STAGE_FILM_GRAIN) && disp) {
    const pf_film_grain& g = s->fg;
    FgArgs a;
    memset(&a, 0, sizeof(a));
    a.active[0] = g.apply && g.num_y_points != 0;
    a.active[1] = g.apply && !f->mono && (g.num_cb_points != 0 || g.chroma_scaling_from_luma);
    a.active[2] = g.apply && !f->mono && (g.num_cr_points != 0 || g.chroma_scaling_from_luma);
    if (a.active[0] || a.active[1] || a.active[2]) {
      CK(c->grain.ensure(3 * 82 * 73 * sizeof(int16_t)));
      int16_t* gbase = (int16_t*)c->grain.p;
      FgTemplateArgs t;
      memset(&t, 0, sizeof(t));
      t.seed = g.seed;
      t.bd = f->bit_depth;
      t.num_y_points = g.num_y_points;
      t.grain_scale_shift = g.grain_scale_shift;
      t.lag = g.ar_coeff_lag;
      t.coeff_shift = g.ar_coeff_shift;
      memcpy(t.coeffs[0], g.ar_coeffs_y, 24);
      memcpy(t.coeffs[1], g.ar_coeffs_cb, 25);
      memcpy(t.coeffs[2], g.ar_coeffs_cr, 25);
      t.active[0] = a.active[0];
      t.active[1] = a.active[1];
      t.active[2] = a.active[2];
      t.ssx = f->ss_x;
      t.ssy = f->ss_y;
      CK(launch_fg_templates(t, gbase, gbase + 82 * 73, gbase + 2 * 82 * 73, st));
      const int rows = (f->height + 31) / 32, cols = (f->width + 31) / 32;
      CK(c->offsets.ensure((size_t)rows * cols));
      CK(launch_fg_offsets(g.seed, rows, cols, (uint8_t*)c->offsets.p, st));
      for (int p = 0; p < 3; p++) a.grain[p] = gbase + p * 82 * 73;
      a.offsets = (const uint8_t*)c->offsets.p;
      a.off_rows = rows;
      a.off_cols = cols;
      build_scaling_lut(a.lut[0], g.y_points, g.num_y_points);
      if (g.chroma_scaling_from_luma) {
        memcpy(a.lut[1], a.lut[0], 256);
        memcpy(a.lut[2], a.lut[0], 256);
      } else {
        build_scaling_lut(a.lut[1], g.cb_points, g.num_cb_points);
        build_scaling_lut(a.lut[2], g.cr_points, g.num_cr_points);
      }
      a.scaling_shift = g.scaling_shift;
      a.overlap = g.overlap;
      a.clip_restricted = g.clip_to_restricted_range;
      a.matrix_identity = g.matrix_identity;
      a.cfl = g.chroma_scaling_from_luma;
      a.mult[1] = g.cb_mult;
      a.luma_mult[1] = g.cb_luma_mult;
      a.offset[1] = g.cb_offset;
      a.mult[2] = g.cr_mult;
      a.luma_mult[2] = g.cr_luma_mult;
      a.offset[2] = g.cr_offset;
      a.odd_luma = f->ss_x && (f->width & 1);
      CK(launch_fg_apply(io, *disp, a, st));
      done |= PF_STAGE_FILM_GRAIN;
    } else {
      // No-op grain: the display picture is the reference picture.
      FgArgs z;
      memset(&z, 0, sizeof(z));
      CK(launch_fg_apply(io, *disp, z, st));
    }
  }
  if (c->timing) cudaEventRecord(c->ev[5], st);
  if (stats) {
    stats->completed = done;
  }
  return PF_OK;
}

static void read_stage_times(pf_ctx* c, pf_stats* stats) {
  if (!stats || !c->timing) return;
  for (int i = 0; i < 5; i++) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]);
    stats->stage_ms[i] = ms;
  }
}

extern "C" int pf_frame_apply(pf_ctx* c, const pf_frame* f, const pf_frame_side* s, const pf_frame* display,
                              pf_stats* stats) {
  if (!c) return PF_ERR_INVALID_ARG;
  int st = pf_frame_validate(f, s, display);
  if (st != PF_OK) return st;
  CK(cudaSetDevice(c->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  const int bps = bps_of(f);
  void* ioPtr[3];
  int64_t ioStride[3];
  if (f->memory == PF_MEM_HOST) {
    CK(layout_like(f, c->io, ioPtr, ioStride));
    for (int p = 0; p < 3; p++)
      CK(cudaMemcpy2DAsync(ioPtr[p], ioStride[p], f->plane[p].data, f->plane[p].stride,
                           (size_t)f->plane[p].alloc_width * bps, f->plane[p].alloc_height, cudaMemcpyHostToDevice,
                           c->stream));
  } else {
    for (int p = 0; p < 3; p++) {
      ioPtr[p] = f->plane[p].data;
      ioStride[p] = f->plane[p].stride;
    }
  }
  DFrame io = dframe_from(f, ioPtr, ioStride);
  const bool wantDisp = (s->stages & PF_STAGE_FILM_GRAIN) && display;
  DFrame disp;
  void* dPtr[3];
  int64_t dStride[3];
  if (wantDisp) {
    if (display->memory == PF_MEM_HOST) {
      CK(layout_like(display, c->disp, dPtr, dStride));
    } else {
      for (int p = 0; p < 3; p++) {
        dPtr[p] = display->plane[p].data;
        dStride[p] = display->plane[p].stride;
      }
    }
    disp = dframe_from(display, dPtr, dStride);
  }
  st = run_chain(c, f, io, s, wantDisp ? &disp : nullptr, stats);
  if (st != PF_OK) return st;
  if (f->memory == PF_MEM_HOST)
    for (int p = 0; p < 3; p++)
      CK(cudaMemcpy2DAsync(f->plane[p].data, f->plane[p].stride, ioPtr[p], ioStride[p],
                           (size_t)f->plane[p].alloc_width * bps, f->plane[p].alloc_height, cudaMemcpyDeviceToHost,
                           c->stream));
  if (wantDisp && display->memory == PF_MEM_HOST)
    for (int p = 0; p < 3; p++)
      CK(cudaMemcpy2DAsync(display->plane[p].data, display->plane[p].stride, dPtr[p], dStride[p],
                           (size_t)display->plane[p].alloc_width * bps, display->plane[p].alloc_height,
                           cudaMemcpyDeviceToHost, c->stream));
  if (f->memory == PF_MEM_HOST || (wantDisp && display->memory == PF_MEM_HOST) || s->side_memory == PF_MEM_HOST ||
      c->timing) {
    CK(cudaStreamSynchronize(c->stream));
    read_stage_times(c, stats);
  }
  CK(cudaGetLastError());
  return PF_OK;
}

extern "C" int pf_batch_apply(pf_ctx* c, const pf_batch_item* items, int32_t n, pf_stats* stats) {
  if (!c || (!items && n > 0) || n < 0) return PF_ERR_INVALID_ARG;
  for (int i = 0; i < n; i++) {
    int st = pf_frame_validate(items[i].frame, items[i].side, items[i].display);
    if (st != PF_OK) return st;
    if (items[i].frame->memory != PF_MEM_DEVICE || items[i].side->side_memory != PF_MEM_DEVICE) return PF_ERR_INVALID_ARG;
  }
  for (int i = 0; i < n; i++) {
    int st = pf_frame_apply(c, items[i].frame, items[i].side, items[i].display, stats);
    if (st != PF_OK) return st;
  }
  return PF_OK;
}

extern "C" int pf_cdef_search(pf_ctx* c, const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                              const pf_cdef_search_params* params, uint64_t* mse_out, uint8_t* fb_index_out,
                              pf_cdef_search_result* result) {
  (void)c;
  (void)source;
  (void)recon;
  (void)noskip;
  (void)params;
  (void)mse_out;
  (void)fb_index_out;
  (void)result;
  return PF_ERR_UNSUPPORTED;
}
