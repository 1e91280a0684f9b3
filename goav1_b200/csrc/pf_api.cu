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
#include <new>
#include <thread>
#include <utility>
#include <vector>

#include "pf_common.cuh"
#include "pf_wait.h"

namespace pf {
cudaError_t launch_deblock_batch(const BatchArgs& b, int total, int grid, int dir, cudaStream_t st);
cudaError_t launch_cdef_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
size_t cdef_tables_bytes();
cudaError_t launch_cdef_tables(int16_t* dst, cudaStream_t st);
cudaError_t launch_lr_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t launch_fg_templates_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t launch_fg_offsets_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t launch_fg_apply_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t launch_extend_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t lr_upload_tables();
cudaError_t fg_upload_tables();
cudaError_t launch_superres_frame(const uint8_t* const* src, const int64_t* sstride, uint8_t* const* dst,
                                  const int64_t* dstride, const pf_frame* coded, int upW, cudaStream_t st);
cudaError_t launch_superres_lines(const uint8_t* const* src, const int64_t* sstride, uint8_t* const* lines,
                                  const int64_t* lstride, const int* nb, const pf_frame* coded, int upW,
                                  cudaStream_t st);
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

// Page-locked host allocator whose element construction leaves bytes as they
// are (staging that is always overwritten is not zero-filled first).
template <class T>
struct PinnedAlloc {
  using value_type = T;
  PinnedAlloc() = default;
  template <class U>
  PinnedAlloc(const PinnedAlloc<U>&) {}
  T* allocate(size_t n) {
    void* p = nullptr;
    if (cudaMallocHost(&p, n * sizeof(T)) != cudaSuccess) throw std::bad_alloc();
    return static_cast<T*>(p);
  }
  void deallocate(T* p, size_t) { cudaFreeHost(p); }
  template <class U>
  void construct(U* p) {
    ::new ((void*)p) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new ((void*)p) U(std::forward<A>(a)...);
  }
  bool operator==(const PinnedAlloc&) const { return true; }
  bool operator!=(const PinnedAlloc&) const { return false; }
};
using PinnedBytes = std::vector<uint8_t, PinnedAlloc<uint8_t>>;

}  // namespace

struct pf_ctx {
  int device = 0;
  int sm_count = 148;
  int64_t wait_timeout_us = 0;    // 0: synchronous calls block; else PF_ERR_TIMEOUT at the deadline
  cudaStream_t stream = nullptr;  // main stream (returned by pf_stream)
  cudaStream_t side = nullptr;    // film-grain templates/offsets overlap the chain here
  int timing = 0;
  cudaEvent_t ev[8] = {};
  cudaEvent_t fork = nullptr, join = nullptr;
  DevBuf io, disp;           // staging of host frames
  DevBuf sr_up, sr_lines;    // super-resolved frames: upscaled staging, upscaled boundary rows
  DevBuf arena;              // per-frame scratch: CDEF output, LR lines, grain, offsets
  DevBuf sidebuf;            // host side information copied up
  DevBuf jobs, bases, counters;
  DevBuf search;             // encoder CDEF search scratch
  DevBuf ctab;               // CDEF constrain() tables (CdefArgs.ctab)
  DevBuf model;              // the learned search's network, uploaded when it changes
  std::vector<uint8_t> model_shadow;  // host copy of what `model` holds
  void* pinned = nullptr;    // page-locked staging for small host inputs
  size_t pinned_n = 0;
  void* model_pin = nullptr; // page-locked staging of the network upload
  std::vector<FrameJob> hjobs;
  std::vector<int> hbase;
  // Side information of the current batch, page-locked so its upload is an
  // asynchronous DMA; side_done marks the upload's end, and the buffer is
  // not rewritten before it (side_pending).
  PinnedBytes hside;
  cudaEvent_t side_done = nullptr;
  bool side_pending = false;
  // The schedule of each stage's launch (pf_schedule): persistent-CTA count
  // (0 = one CTA per chunk), work items per chunk, items prefetched ahead,
  // and the deblocking tile shape.
  int persistent[ST_COUNT] = {};
  int chunk[ST_COUNT] = {1, 1, 1, 1, 1, 1, 1, 1};
  int ahead[ST_COUNT] = {};
  int tile[ST_COUNT] = {};  // launch-level tile setting (grain apply: rows per load group)
  int db_tile = 0;          // deblocking tile shape (per job: it sets the tile counts)
  // Frame groups (pf_set_frame_groups): 2 runs the batch's two halves on the
  // main stream and stream2.
  int frame_groups = 1;
  cudaStream_t stream2 = nullptr;
  cudaEvent_t gfork = nullptr, gjoin = nullptr;
  // CUDA graphs of pf_batch_apply, one per batch signature (see run_batch).
  int graphs = 0;
  std::vector<struct GraphEntry*> gcache;
  uint64_t gclock = 0;
  // Host-frame batches (run_host_pipeline): copy streams and a ring of
  // staging slots, each a chunk of frames on the device with the page-locked
  // tables of its launch.
  cudaStream_t h2d = nullptr, d2h = nullptr;
  // Recorded after the border extension when mark_chain is set: the reference
  // frame is final there, so its download can overlap the grain stage.
  cudaEvent_t chain_done = nullptr;
  bool mark_chain = false;
  struct HostSlot {
    DevBuf io, disp;
    void* pjobs = nullptr;
    size_t njobs = 0;
    void* pbase = nullptr;
    size_t nbase = 0;
    PinnedBytes side;  // the chunk's side information, written in place
    DevBuf djobs, dbases, dside;  // the chunk's tables on the device
    cudaEvent_t up = nullptr, comp = nullptr, down = nullptr;
    bool used = false;
  } hslot[3];
  int host_chunk = 4;
};

// One captured batch signature, in two slots used in turn: each slot is a
// graph and the page-locked copies of the job table, prefix arrays and side
// information its copy nodes read when it runs.  A replay waits for the
// slot's previous run (its event) before rewriting those buffers, so the host
// can prepare one batch while the previous one is still on the GPU.
struct GraphSlot {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t done = nullptr;
  void* pjobs = nullptr;
  void* pbase = nullptr;
  void* pside = nullptr;
};

struct GraphEntry {
  std::vector<int64_t> key;
  void* bufs[5] = {};  // the context scratch the captured kernels address
  GraphSlot slot[2];
  int next = 0;
  uint64_t used = 0;
  ~GraphEntry() {
    for (GraphSlot& g : slot) {
      if (g.done) cudaEventSynchronize(g.done);
      if (g.exec) cudaGraphExecDestroy(g.exec);
      if (g.graph) cudaGraphDestroy(g.graph);
      if (g.done) cudaEventDestroy(g.done);
      if (g.pjobs) cudaFreeHost(g.pjobs);
      if (g.pbase) cudaFreeHost(g.pbase);
      if (g.pside) cudaFreeHost(g.pside);
    }
  }
};

// ---------------------------------------------------------------------------
// Validation (no device work; mirrors the reference's error taxonomy).

// Whether any of n bytes exceeds 63 (bit 6 or 7 set), read 8 bytes at a
// time without an early exit so the compiler vectorises the scan of a
// frame's level cache (half a megabyte at 1080p).
static bool any_byte_above_63(const uint8_t* p, size_t n) {
  uint64_t acc = 0;
  size_t i = 0;
  for (; i + 8 <= n; i += 8) {
    uint64_t w;
    memcpy(&w, p + i, 8);
    acc |= w;
  }
  for (; i < n; i++) acc |= p[i];
  return (acc & 0xC0C0C0C0C0C0C0C0ull) != 0;
}

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

// Whether any plane of `a` shares bytes with any plane of `b` (each plane
// spans stride x (alloc_height - 1) + its row).
static bool frames_overlap(const pf_frame* a, const pf_frame* b) {
  const int ba = a->bit_depth > 8 ? 2 : 1, bb = b->bit_depth > 8 ? 2 : 1;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      const pf_plane &p = a->plane[i], &q = b->plane[j];
      if (!p.data || !q.data || p.alloc_height <= 0 || q.alloc_height <= 0) continue;
      const uintptr_t p0 = (uintptr_t)p.data, q0 = (uintptr_t)q.data;
      const uintptr_t p1 = p0 + (uintptr_t)(p.stride * (p.alloc_height - 1) + (int64_t)p.alloc_width * ba);
      const uintptr_t q1 = q0 + (uintptr_t)(q.stride * (q.alloc_height - 1) + (int64_t)q.alloc_width * bb);
      if (p0 < q1 && q0 < p1) return true;
    }
  return false;
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
    if (hostSide && any_byte_above_63(lf.level_cache, (size_t)4 * miCols * miRows)) return PF_ERR_INVALID_FILTER;
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
    // The display picture is a separate output (PostFilterOutput): grain
    // reads the reference's luma for chroma scaling while it writes display.
    if (display->memory == f->memory && frames_overlap(f, display)) return PF_ERR_INVALID_ARG;
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

namespace pf {
// The 256-entry scaling table of a piecewise-linear point list
// (filmgrain/scaling.go:18-48, BuildScalingLUT); also used by
// pf_film_grain_static.
void build_scaling_lut(uint8_t* dst, const uint8_t (*pts)[2], int n) {
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
}  // namespace pf

// The last failing CUDA call of this thread, for pf_status_detail().
static thread_local char g_detail[256];

static void last_error(cudaError_t e, const char* expr, int line) {
  snprintf(g_detail, sizeof(g_detail), "%s (%s) at pf_api.cu:%d: %s", cudaGetErrorName(e), cudaGetErrorString(e),
           line, expr);
  if (getenv("PF_DEBUG")) fprintf(stderr, "goav1pf: %s\n", g_detail);
}

#define CK(expr)                        \
  do {                                  \
    cudaError_t _e = (expr);            \
    if (_e != cudaSuccess) {            \
      last_error(_e, #expr, __LINE__);  \
      return PF_ERR_DEVICE;             \
    }                                   \
  } while (0)

extern "C" const char* pf_status_detail(void) { return g_detail; }

// A synchronous call's wait on its own device work: blocking, or polled with
// the context's deadline (pf_config.wait_timeout_us).  PF_OK, PF_ERR_TIMEOUT
// (the work stays queued) or PF_ERR_DEVICE.
template <class Q, class B>
static int ctx_wait(pf_ctx* c, Q query, B block, const char* what, int line) {
  if (c->wait_timeout_us <= 0) {
    const cudaError_t e = block();
    if (e != cudaSuccess) {
      last_error(e, what, line);
      return PF_ERR_DEVICE;
    }
    return PF_OK;
  }
  cudaError_t failed = cudaSuccess;
  const int r = wait_until(
      [&]() {
        const cudaError_t e = query();
        if (e == cudaSuccess) return (int)kWaitReady;
        if (e == cudaErrorNotReady) {
          cudaGetLastError();  // not an error: keep it out of later launch checks
          return (int)kWaitPending;
        }
        failed = e;
        return (int)kWaitFailed;
      },
      c->wait_timeout_us);
  if (r == kWaitTimedOut) {
    snprintf(g_detail, sizeof(g_detail), "%s at pf_api.cu:%d: still running after %lld us", what, line,
             (long long)c->wait_timeout_us);
    return PF_ERR_TIMEOUT;
  }
  if (r == kWaitError) {
    last_error(failed, what, line);
    return PF_ERR_DEVICE;
  }
  return PF_OK;
}

static int wait_stream(pf_ctx* c, cudaStream_t st, int line) {
  return ctx_wait(
      c, [&]() { return cudaStreamQuery(st); }, [&]() { return cudaStreamSynchronize(st); }, "stream wait", line);
}

static int wait_event(pf_ctx* c, cudaEvent_t ev, int line) {
  return ctx_wait(
      c, [&]() { return cudaEventQuery(ev); }, [&]() { return cudaEventSynchronize(ev); }, "event wait", line);
}

#define CKW(expr)                  \
  do {                             \
    const int _w = (expr);         \
    if (_w != PF_OK) return _w;    \
  } while (0)

// The other entry points' waits (pf_search.cu, pf_lr.cu, ...).
int pf_internal_wait(pf_ctx* c, void* stream) { return wait_stream(c, (cudaStream_t)stream, __LINE__); }

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
    case PF_ERR_INVALID_BATCH: return "threading: invalid batch";
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
  if (cfg && cfg->wait_timeout_us < 0) {
    if (status) *status = PF_ERR_INVALID_ARG;
    return nullptr;
  }
  pf_ctx* c = new pf_ctx();
  c->device = dev;
  c->timing = cfg ? cfg->timing : 0;
  c->wait_timeout_us = cfg ? cfg->wait_timeout_us : 0;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess || lr_upload_tables() != cudaSuccess ||
      fg_upload_tables() != cudaSuccess) {
    delete c;
    if (status) *status = PF_ERR_DEVICE;
    return nullptr;
  }
  for (int i = 0; i < 8; i++) cudaEventCreate(&c->ev[i]);
  cudaEventCreateWithFlags(&c->fork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&c->join, cudaEventDisableTiming);
  cudaStreamCreateWithFlags(&c->side, cudaStreamNonBlocking);
  cudaStreamCreateWithFlags(&c->stream2, cudaStreamNonBlocking);
  cudaEventCreateWithFlags(&c->gfork, cudaEventDisableTiming);
  cudaEventCreateWithFlags(&c->gjoin, cudaEventDisableTiming);
  c->sm_count = prop.multiProcessorCount;
  // The CDEF kernel's constrain() tables, built once on the context's stream
  // (every later launch is ordered after it).
  if (c->ctab.ensure(cdef_tables_bytes()) != cudaSuccess ||
      launch_cdef_tables((int16_t*)c->ctab.p, c->stream) != cudaSuccess) {
    pf_destroy(c);
    if (status) *status = PF_ERR_DEVICE;
    return nullptr;
  }
  if (status) *status = PF_OK;
  return c;
}

extern "C" void pf_destroy(pf_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->device);
  cudaStreamSynchronize(c->stream);
  cudaStreamSynchronize(c->side);
  if (c->stream2) cudaStreamSynchronize(c->stream2);
  if (c->h2d) cudaStreamSynchronize(c->h2d);
  if (c->d2h) cudaStreamSynchronize(c->d2h);
  DevBuf* bufs[] = {&c->io,     &c->disp,     &c->arena,  &c->sidebuf, &c->jobs,    &c->bases,
                    &c->counters, &c->search, &c->sr_up,   &c->sr_lines, &c->ctab};
  for (DevBuf* b : bufs) b->release();
  for (pf_ctx::HostSlot& h : c->hslot) {
    h.io.release();
    h.disp.release();
    if (h.pjobs) cudaFreeHost(h.pjobs);
    if (h.pbase) cudaFreeHost(h.pbase);
    PinnedBytes().swap(h.side);
    h.djobs.release();
    h.dbases.release();
    h.dside.release();
    if (h.up) cudaEventDestroy(h.up);
    if (h.comp) cudaEventDestroy(h.comp);
    if (h.down) cudaEventDestroy(h.down);
  }
  if (c->h2d) cudaStreamDestroy(c->h2d);
  if (c->d2h) cudaStreamDestroy(c->d2h);
  c->model.release();
  for (GraphEntry* g : c->gcache) delete g;
  c->gcache.clear();
  if (c->pinned) cudaFreeHost(c->pinned);
  if (c->model_pin) cudaFreeHost(c->model_pin);
  for (int i = 0; i < 8; i++)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  cudaEventDestroy(c->fork);
  cudaEventDestroy(c->join);
  if (c->chain_done) cudaEventDestroy(c->chain_done);
  if (c->side_done) cudaEventDestroy(c->side_done);
  if (c->gfork) cudaEventDestroy(c->gfork);
  if (c->gjoin) cudaEventDestroy(c->gjoin);
  if (c->stream2) cudaStreamDestroy(c->stream2);
  cudaStreamDestroy(c->side);
  cudaStreamDestroy(c->stream);
  delete c;
}

extern "C" int pf_sync(pf_ctx* c) {
  if (!c) return PF_ERR_INVALID_ARG;
  return wait_stream(c, c->stream, __LINE__);
}

extern "C" void* pf_stream(pf_ctx* c) { return c ? (void*)c->stream : nullptr; }


// ---------------------------------------------------------------------------
// Job preparation.

struct FrameRef {
  const pf_frame* f;
  const pf_frame_side* s;
  const pf_frame* display;  // may be null
  void* io[3];
  int64_t ioStride[3];
  void* dp[3];
  int64_t dStride[3];
  // Restoration stripe-boundary rows made elsewhere (a super-resolved frame's
  // upscaled deblock rows); null: the CDEF pass saves them.
  uint8_t* ext_lines[3];
  int64_t ext_line_stride[3];
};

static size_t align256(size_t v) { return (v + 255) & ~(size_t)255; }

static bool cdef_any(const pf_frame* f, const pf_frame_side* s) {
  if (!(s->stages & PF_STAGE_CDEF)) return false;
  for (int i = 0; i < std::min((int)s->cdef.strength_count, 8); i++)
    if (s->cdef.y_strength[i] || (!f->mono && s->cdef.uv_strength[i])) return true;
  return false;
}

static bool lr_any(const pf_frame_side* s) {
  return (s->stages & PF_STAGE_LOOP_RESTORATION) &&
         (s->lr.type[0] != PF_LR_NONE || s->lr.type[1] != PF_LR_NONE || s->lr.type[2] != PF_LR_NONE);
}

static bool fg_active(const pf_frame* f, const pf_frame_side* s, int act[3]) {
  const pf_film_grain& g = s->fg;
  act[0] = g.apply && g.num_y_points != 0;
  act[1] = g.apply && !f->mono && (g.num_cb_points != 0 || g.chroma_scaling_from_luma);
  act[2] = g.apply && !f->mono && (g.num_cr_points != 0 || g.chroma_scaling_from_luma);
  return (s->stages & PF_STAGE_FILM_GRAIN) && (act[0] || act[1] || act[2]);
}

// Scratch bytes one frame needs in the arena.
static size_t frame_scratch(const pf_frame* f, const pf_frame_side* s) {
  const int bps = bps_of(f);
  size_t n = 0;
  if (cdef_any(f, s) || lr_any(s)) {
    for (int p = 0; p < 3; p++)
      n += align256((size_t)align256((size_t)f->plane[p].alloc_width * bps) * f->plane[p].alloc_height);
  }
  if (lr_any(s)) {
    for (int p = 0; p < 3; p++) {
      if (s->lr.type[p] == PF_LR_NONE) continue;
      const int sy = p ? f->ss_y : 0;
      const int nb = (f->plane[p].height + (8 >> sy)) / (64 >> sy) + 2;
      n += align256((size_t)nb * 4 * align256((size_t)f->plane[p].width * bps));
    }
  }
  int act[3];
  if (fg_active(f, s, act)) {
    n += align256(3 * 82 * 73 * sizeof(int16_t));
    n += align256((size_t)((f->height + 31) / 32) * ((f->width + 31) / 32));
  }
  return n;
}

// Host side-information bytes to copy up for one frame.
static size_t frame_side_bytes(const pf_frame* f, const pf_frame_side* s) {
  if (s->side_memory != PF_MEM_HOST) return 0;
  size_t n = 0;
  const int miCols = ((f->width + 7) >> 3) << 1, miRows = ((f->height + 7) >> 3) << 1;
  const int ucols = (f->width + 63) / 64, urows = (f->height + 63) / 64;
  if (s->stages & PF_STAGE_LOOP_FILTER)
    n += align256((size_t)s->lf.sb128_w * s->lf.sb128_h * PF_LF_MASK_WORDS * 2) + align256((size_t)4 * miCols * miRows);
  if (cdef_any(f, s))
    n += 2 * align256((size_t)s->cdef.index_stride * s->cdef.index_rows) + align256((size_t)ucols * urows * 8);
  if (lr_any(s))
    for (int p = 0; p < 3; p++)
      if (s->lr.type[p] != PF_LR_NONE) n += align256(sizeof(pf_lr_unit) * s->lr.unit_count[p]);
  return n;
}

struct Cursor {
  uint8_t* base;
  size_t off;
  void* take(size_t n) {
    void* p = base + off;
    off += align256(n);
    return p;
  }
};

template <class Bytes>
static const void* put_side(Bytes& hs, Cursor& dev, const void* src, size_t n) {
  if (!src || n == 0) return src;
  void* d = dev.take(n);
  const size_t at = (uint8_t*)d - dev.base;
  if (hs.size() < at + n) hs.resize(at + n);
  memcpy(hs.data() + at, src, n);
  return d;
}

template <class Bytes>
static void fill_job(const FrameRef& r, Cursor& arena, Cursor& side, Bytes& hs, FrameJob& J, int counts[ST_COUNT],
                     int dbTile) {
  const pf_frame* f = r.f;
  const pf_frame_side* s = r.s;
  const int bps = bps_of(f);
  const bool host = s->side_memory == PF_MEM_HOST;
  memset(&J, 0, sizeof(J));
  J.io = dframe_from(f, r.io, r.ioStride);
  const int miCols = ((f->width + 7) >> 3) << 1, miRows = ((f->height + 7) >> 3) << 1;
  const int ucols = (f->width + 63) / 64, urows = (f->height + 63) / 64;
  for (int p = 0; p < 3; p++) {
    const int xdec = p ? f->ss_x : 0, ydec = p ? f->ss_y : 0;
    J.aw[p] = ((f->width + 7) & ~7) >> xdec;
    J.ah[p] = ((f->height + 7) & ~7) >> ydec;
  }
  for (int k = 0; k < ST_COUNT; k++) counts[k] = 0;

  // Deblocking.
  if (s->stages & PF_STAGE_LOOP_FILTER) {
    const pf_loop_filter& lf = s->lf;
    LfArgs& a = J.lf;
    a.masks = host ? (const uint16_t*)put_side(hs, side, lf.masks, (size_t)lf.sb128_w * lf.sb128_h * PF_LF_MASK_WORDS * 2)
                   : lf.masks;
    a.level_cache = host ? (const uint8_t*)put_side(hs, side, lf.level_cache, (size_t)4 * miCols * miRows) : lf.level_cache;
    a.sb128_w = lf.sb128_w;
    a.sb128_h = lf.sb128_h;
    a.mi_cols = lf.mi_cols;
    a.mi_rows = lf.mi_rows;
    a.sharpness = lf.sharpness;
    const bool lumaZero = lf.level_y[0] == 0 && lf.level_y[1] == 0;
    a.gate_chroma[1] = f->mono || lumaZero || lf.level_u == 0;
    a.gate_chroma[2] = f->mono || lumaZero || lf.level_v == 0;
    int tiles = 0;
    J.db_tile = dbTile;
    for (int p = 0; p < 3; p++) {
      if (a.gate_chroma[p]) continue;
      const int sx = p ? f->ss_x : 0, sy = p ? f->ss_y : 0;
      const int w4 = (((f->width + sx) >> sx) + 3) >> 2, h4 = (((f->height + sy) >> sy) + 3) >> 2;
      J.db_tx[p] = (w4 + db_tile_w(dbTile) - 1) / db_tile_w(dbTile);
      J.db_ty[p] = (h4 + db_tile_h(dbTile) - 1) / db_tile_h(dbTile);
      tiles += J.db_tx[p] * J.db_ty[p];
    }
    counts[ST_DEBLOCK_V] = counts[ST_DEBLOCK_H] = tiles;
  }

  // CDEF (+ restoration boundary lines) and restoration (or copy back).
  const bool cdefOn = cdef_any(f, s), lrOn = lr_any(s);
  if (cdefOn || lrOn) {
    void* sp[3];
    int64_t ss[3];
    for (int p = 0; p < 3; p++) {
      ss[p] = (int64_t)align256((size_t)f->plane[p].alloc_width * bps);
      sp[p] = arena.take((size_t)ss[p] * f->plane[p].alloc_height);
    }
    J.scr = dframe_from(f, sp, ss);
    CdefArgs& a = J.cdef;
    const pf_cdef& cd = s->cdef;
    a.filter = cdefOn ? 1 : 0;
    a.ucols = ucols;
    a.urows = urows;
    if (cdefOn) {
      const size_t n = (size_t)cd.index_stride * cd.index_rows;
      a.index = host ? (const uint8_t*)put_side(hs, side, cd.index, n) : cd.index;
      a.read = host ? (const uint8_t*)put_side(hs, side, cd.read, n) : cd.read;
      a.noskip = cd.noskip ? (host ? (const uint8_t*)put_side(hs, side, cd.noskip, (size_t)ucols * urows * 8) : cd.noskip)
                           : nullptr;
      a.index_stride = cd.index_stride;
    }
    a.damping = cd.damping;
    a.strength_count = cdefOn ? cd.strength_count : 0;
    bool uvAny = false, yAny = false;
    for (int i = 0; i < 8; i++) {
      a.y_strength[i] = cd.y_strength[i];
      a.uv_strength[i] = cd.uv_strength[i];
    }
    for (int i = 0; i < std::min((int)cd.strength_count, 8); i++) {
      uvAny |= cd.uv_strength[i] != 0;
      yAny |= cd.y_strength[i] != 0;
    }
    a.chroma_filtering = cdefOn && !f->mono && uvAny;
    a.plane_process[0] = cdefOn && (yAny || a.chroma_filtering);
    a.plane_process[1] = a.plane_process[2] = cdefOn && uvAny;
    J.do_lr = lrOn ? 1 : 0;
    if (lrOn) {
      for (int p = 0; p < 3; p++) {
        if (s->lr.type[p] == PF_LR_NONE) continue;
        const int sy = p ? f->ss_y : 0;
        const int nb = (f->plane[p].height + (8 >> sy)) / (64 >> sy) + 2;
        if (r.ext_lines[p]) {
          a.line_stride[p] = r.ext_line_stride[p];
          a.lines[p] = r.ext_lines[p];
          a.save_lines[p] = 0;
        } else {
          a.line_stride[p] = (int64_t)align256((size_t)f->plane[p].width * bps);
          a.lines[p] = (uint8_t*)arena.take((size_t)nb * 4 * a.line_stride[p]);
          a.save_lines[p] = 1;
        }
        LrArgs& l = J.lr;
        l.type[p] = s->lr.type[p];
        int horz, vert, us;
        lr_grid(f, s->lr, p, &horz, &vert, &us);
        l.horz[p] = horz;
        l.vert[p] = vert;
        l.unit_size[p] = us;
        l.units[p] = host ? (const pf_lr_unit*)put_side(hs, side, s->lr.units[p], sizeof(pf_lr_unit) * horz * vert)
                          : s->lr.units[p];
        l.lines[p] = a.lines[p];
        l.line_stride[p] = a.line_stride[p];
      }
    }
    counts[ST_CDEF] = ucols * urows;
    int tiles = 0;
    for (int p = 0; p < (f->mono ? 1 : 3); p++) {
      const int sx = p ? f->ss_x : 0, sy = p ? f->ss_y : 0;
      const int PW = 64 >> sx, SH = 64 >> sy, off = 8 >> sy;
      J.lr_cols[p] = (J.aw[p] + PW - 1) / PW;
      J.lr_rows[p] = (J.ah[p] + off + SH - 1) / SH;
      tiles += J.lr_cols[p] * J.lr_rows[p];
    }
    counts[ST_LR] = tiles;
  }

  // Border extension.
  if (s->stages & PF_STAGE_EXTEND_BORDERS) {
    int tiles = 0;
    for (int p = 0; p < (f->mono ? 1 : 3); p++) {
      const pf_plane& pl = f->plane[p];
      J.ext_r[p][0] = (pl.alloc_width - pl.width + 63) / 64;
      J.ext_r[p][1] = J.ext_r[p][0] ? (pl.height + 3) / 4 : 0;
      J.ext_b[p][0] = (pl.alloc_width + 63) / 64;
      J.ext_b[p][1] = (pl.alloc_height - pl.height + 3) / 4;
      tiles += J.ext_r[p][0] * J.ext_r[p][1] + J.ext_b[p][0] * J.ext_b[p][1];
    }
    counts[ST_EXTEND] = tiles;
  }

  // Film grain into the display frame.
  if ((s->stages & PF_STAGE_FILM_GRAIN) && r.display) {
    J.disp = dframe_from(r.display, r.dp, r.dStride);
    int act[3];
    const bool on = fg_active(f, s, act);
    FgArgs& a = J.fg;
    if (on) {
      const pf_film_grain& g = s->fg;
      int16_t* gbase = (int16_t*)arena.take(3 * 82 * 73 * sizeof(int16_t));
      const int rows = (f->height + 31) / 32, cols = (f->width + 31) / 32;
      a.offsets = (const uint8_t*)arena.take((size_t)rows * cols);
      for (int p = 0; p < 3; p++) {
        a.grain[p] = gbase + p * 82 * 73;
        a.active[p] = act[p];
      }
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
      FgTemplateArgs& t = J.fgt;
      t.seed = g.seed;
      t.bd = f->bit_depth;
      t.num_y_points = g.num_y_points;
      t.grain_scale_shift = g.grain_scale_shift;
      t.lag = g.ar_coeff_lag;
      t.coeff_shift = g.ar_coeff_shift;
      memcpy(t.coeffs[0], g.ar_coeffs_y, 24);
      memcpy(t.coeffs[1], g.ar_coeffs_cb, 25);
      memcpy(t.coeffs[2], g.ar_coeffs_cr, 25);
      for (int p = 0; p < 3; p++) t.active[p] = act[p];
      t.ssx = f->ss_x;
      t.ssy = f->ss_y;
      counts[ST_FG_TEMPLATES] = 1;
      counts[ST_FG_OFFSETS] = (rows + 63) / 64;
    }
    int tiles = 0;
    for (int p = 0; p < (f->mono ? 1 : 3); p++) {
      J.fg_tx[p] = (f->plane[p].alloc_width + 63) / 64;
      J.fg_ty[p] = (f->plane[p].alloc_height + 63) / 64;
      tiles += J.fg_tx[p] * J.fg_ty[p];
    }
    counts[ST_FG_APPLY] = tiles;
  }
}

// Queues the copies of the host tables (from the given host buffers) and
// every stage's launch on the context's streams.
// djobs / dbases: device copies of the tables when the caller uploaded them
// already (null: copy hjobs / hbase / hside into the context's buffers here).
static int enqueue_batch(pf_ctx* c, const FrameJob* hjobs, const int* hbase, const uint8_t* hside, size_t nside,
                         int n, bool fg, const void* djobs = nullptr, const void* dbases = nullptr) {
  const cudaStream_t st = c->stream;
  if (!djobs) {
    if (nside) {
      CK(cudaMemcpyAsync(c->sidebuf.p, hside, nside, cudaMemcpyHostToDevice, st));
      if (hside == c->hside.data()) {
        if (!c->side_done) CK(cudaEventCreateWithFlags(&c->side_done, cudaEventDisableTiming));
        CK(cudaEventRecord(c->side_done, st));
        c->side_pending = true;
      }
    }
    CK(cudaMemcpyAsync(c->jobs.p, hjobs, sizeof(FrameJob) * n, cudaMemcpyHostToDevice, st));
    CK(cudaMemcpyAsync(c->bases.p, hbase, sizeof(int) * c->hbase.size(), cudaMemcpyHostToDevice, st));
    djobs = c->jobs.p;
    dbases = c->bases.p;
  }
  // Frame groups: with two, the batch's frames are split where half of its
  // restoration tiles lie, and each half runs the chain on its own stream,
  // so one half's stage overlaps the other's (the tail of each launch is
  // filled by the other stream's CTAs).
  const int groups = c->frame_groups > 1 && n >= 2 ? 2 : 1;
  int fmid = n;
  if (groups == 2) {
    const int* lrBase = hbase + (size_t)ST_LR * (n + 1);
    const int half = lrBase[n] / 2;
    fmid = 1;
    while (fmid < n - 1 && lrBase[fmid] < half) fmid++;
  }
  bool persistent = false;
  for (int k = 0; k < ST_COUNT; k++) persistent |= c->persistent[k] > 0;
  if (persistent) CK(cudaMemsetAsync(c->counters.p, 0, sizeof(int) * ST_COUNT * groups, st));
  BatchArgs b;
  b.jobs = (const FrameJob*)djobs;
  b.base = (const int*)dbases;
  b.n = n;
  b.wave = 0;
  auto count = [&](int k, int f0, int f1) {
    return hbase[(size_t)k * (n + 1) + f1] - hbase[(size_t)k * (n + 1) + f0];
  };
  auto args = [&](int k, int f0, int f1, int grp, int* grid) {
    BatchArgs a = b;
    a.f0 = f0;
    a.f1 = f1;
    const int t = count(k, f0, f1);
    a.chunk = c->chunk[k];
    a.ahead = c->ahead[k];
    a.tile = c->tile[k];
    const int chunks = (t + a.chunk - 1) / a.chunk;
    if (c->persistent[k] > 0 && chunks > c->persistent[k]) {
      *grid = c->persistent[k];
      a.counters = (int*)c->counters.p + grp * ST_COUNT;
    } else {
      *grid = chunks;
      a.counters = nullptr;
    }
    return a;
  };
  int g;
  // Film-grain templates and offsets depend on nothing else: side stream.
  if (fg) {
    CK(cudaEventRecord(c->fork, st));
    CK(cudaStreamWaitEvent(c->side, c->fork, 0));
    BatchArgs a = args(ST_FG_TEMPLATES, 0, n, 0, &g);
    CK(launch_fg_templates_batch(a, count(ST_FG_TEMPLATES, 0, n), g, c->side));
    a = args(ST_FG_OFFSETS, 0, n, 0, &g);
    CK(launch_fg_offsets_batch(a, count(ST_FG_OFFSETS, 0, n), g, c->side));
    CK(cudaEventRecord(c->join, c->side));
  }
  // Stage events: per stage with one group; with two only the whole batch
  // is timed (it reads as the deblocking stage's time, the others as zero).
  const bool stageEv = c->timing && groups == 1;
  if (c->timing) CK(cudaEventRecord(c->ev[0], st));
  if (groups == 2) {
    CK(cudaEventRecord(c->gfork, st));
    CK(cudaStreamWaitEvent(c->stream2, c->gfork, 0));
  }
  for (int gi = 0; gi < groups; gi++) {
    const cudaStream_t gs = gi ? c->stream2 : st;
    const int f0 = gi ? fmid : 0, f1 = groups == 2 && gi == 0 ? fmid : n;
    BatchArgs a = args(ST_DEBLOCK_V, f0, f1, gi, &g);
    CK(launch_deblock_batch(a, count(ST_DEBLOCK_V, f0, f1), g, 0, gs));
    a = args(ST_DEBLOCK_H, f0, f1, gi, &g);
    CK(launch_deblock_batch(a, count(ST_DEBLOCK_H, f0, f1), g, 1, gs));
    if (stageEv) CK(cudaEventRecord(c->ev[1], gs));
    a = args(ST_CDEF, f0, f1, gi, &g);
    CK(launch_cdef_batch(a, count(ST_CDEF, f0, f1), g, gs));
    if (stageEv) CK(cudaEventRecord(c->ev[2], gs));
    a = args(ST_LR, f0, f1, gi, &g);
    CK(launch_lr_batch(a, count(ST_LR, f0, f1), g, gs));
    if (stageEv) CK(cudaEventRecord(c->ev[3], gs));
    a = args(ST_EXTEND, f0, f1, gi, &g);
    CK(launch_extend_batch(a, count(ST_EXTEND, f0, f1), g, gs));
    if (stageEv) CK(cudaEventRecord(c->ev[4], gs));
    if (c->mark_chain && gi == 0) {
      // While capturing, an external event node: each replay records it
      // for the copy stream that waits on it outside the graph.
      cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
      CK(cudaStreamIsCapturing(gs, &cap));
      CK(cap == cudaStreamCaptureStatusActive ? cudaEventRecordWithFlags(c->chain_done, gs, cudaEventRecordExternal)
                                               : cudaEventRecord(c->chain_done, gs));
    }
    if (fg) CK(cudaStreamWaitEvent(gs, c->join, 0));
    a = args(ST_FG_APPLY, f0, f1, gi, &g);
    CK(launch_fg_apply_batch(a, count(ST_FG_APPLY, f0, f1), g, gs));
  }
  if (groups == 2) {
    CK(cudaEventRecord(c->gjoin, c->stream2));
    CK(cudaStreamWaitEvent(st, c->gjoin, 0));
    if (c->timing)
      for (int i = 1; i < 5; i++) CK(cudaEventRecord(c->ev[i], st));  // after ev[0]: zero-length stages
  }
  if (c->timing) CK(cudaEventRecord(c->ev[5], st));
  return PF_OK;
}

// The batch signature: everything that shapes the launch sequence (grid
// sizes follow from the prefix arrays and the persistent settings, copy
// sizes from n and the side-information bytes).
static std::vector<int64_t> batch_key(const pf_ctx* c, int n, bool fg) {
  std::vector<int64_t> k;
  k.reserve(8 + ST_COUNT + c->hbase.size());
  k.push_back(n);
  k.push_back((int64_t)c->hside.size());
  k.push_back(fg);
  for (int i = 0; i < ST_COUNT; i++) {
    k.push_back(c->persistent[i]);
    k.push_back(c->chunk[i]);
    k.push_back(c->ahead[i]);
    k.push_back(c->tile[i]);
  }
  k.push_back(c->db_tile);
  k.push_back(c->frame_groups);
  k.push_back(c->mark_chain);
  for (int v : c->hbase) k.push_back(v);
  return k;
}

// Replays the graph captured for this batch signature (capturing the slot on
// its first use; at most 8 signatures kept, least recently used dropped).  A
// graph addresses the context's scratch buffers, so it is recaptured after
// any of them moved.
static int replay_or_capture(pf_ctx* c, int n, bool fg) {
  const cudaStream_t st = c->stream;
  const std::vector<int64_t> key = batch_key(c, n, fg);
  void* bufs[5] = {c->arena.p, c->sidebuf.p, c->jobs.p, c->bases.p, c->counters.p};
  const size_t nj = sizeof(FrameJob) * n, nb = sizeof(int) * c->hbase.size(), ns = c->hside.size();
  GraphEntry* e = nullptr;
  for (GraphEntry* x : c->gcache)
    if (x->key == key && memcmp(x->bufs, bufs, sizeof(bufs)) == 0) e = x;
  if (!e) {
    if (c->gcache.size() >= 8) {
      auto lru = std::min_element(c->gcache.begin(), c->gcache.end(),
                                  [](const GraphEntry* a, const GraphEntry* b) { return a->used < b->used; });
      delete *lru;
      c->gcache.erase(lru);
    }
    e = new GraphEntry();
    e->key = key;
    memcpy(e->bufs, bufs, sizeof(bufs));
    c->gcache.push_back(e);
  }
  e->used = ++c->gclock;
  GraphSlot& g = e->slot[e->next];
  e->next ^= 1;
  if (!g.exec) {
    if (cudaMallocHost(&g.pjobs, nj + 16) != cudaSuccess || cudaMallocHost(&g.pbase, nb + 16) != cudaSuccess ||
        cudaMallocHost(&g.pside, ns + 16) != cudaSuccess)
      return PF_ERR_DEVICE;
    CK(cudaEventCreateWithFlags(&g.done, cudaEventDisableTiming));
  } else {
    CKW(wait_event(c, g.done, __LINE__));  // the slot's previous run has read its tables
  }
  memcpy(g.pjobs, c->hjobs.data(), nj);
  memcpy(g.pbase, c->hbase.data(), nb);
  if (ns) memcpy(g.pside, c->hside.data(), ns);
  if (!g.exec) {
    CK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int est =
        enqueue_batch(c, (const FrameJob*)g.pjobs, (const int*)g.pbase, (const uint8_t*)g.pside, ns, n, fg);
    const cudaError_t ce = cudaStreamEndCapture(st, &g.graph);
    cudaError_t ie = cudaSuccess;
    if (est == PF_OK && ce == cudaSuccess) ie = cudaGraphInstantiate(&g.exec, g.graph, 0);
    if (est != PF_OK || ce != cudaSuccess || ie != cudaSuccess) {
      if (g.graph) cudaGraphDestroy(g.graph);
      g.graph = nullptr;
      g.exec = nullptr;
      if (est != PF_OK) return est;
      CK(ce != cudaSuccess ? ce : ie);
    }
  }
  CK(cudaGraphLaunch(g.exec, st));
  CK(cudaEventRecord(g.done, st));
  return PF_OK;
}

// Builds the job table and prefix arrays of n validated frames into c->hjobs
// / hbase and their host side information into hs (the device buffers they
// address are sized here); *fg tells whether any frame has film grain.
// sideDev: where the side information goes on the device (the context's
// buffer, or a host-pipeline slot's).
template <class Bytes>
static int prepare_batch(pf_ctx* c, const FrameRef* refs, int n, Bytes& hs, DevBuf& sideDev, uint32_t* completed,
                         bool* fg) {
  size_t arenaBytes = 0, sideBytes = 0;
  for (int i = 0; i < n; i++) {
    arenaBytes += frame_scratch(refs[i].f, refs[i].s);
    sideBytes += frame_side_bytes(refs[i].f, refs[i].s);
  }
  CK(c->arena.ensure(arenaBytes + 256));
  CK(sideDev.ensure(sideBytes + 256));
  Cursor arena{(uint8_t*)c->arena.p, 0}, side{(uint8_t*)sideDev.p, 0};
  c->hjobs.resize(n);
  c->hbase.assign((size_t)ST_COUNT * (n + 1), 0);
  hs.clear();
  uint32_t done = 0;
  for (int i = 0; i < n; i++) {
    int counts[ST_COUNT];
    fill_job(refs[i], arena, side, hs, c->hjobs[i], counts, c->db_tile);
    c->hjobs[i].cdef.ctab = (const int16_t*)c->ctab.p;
    for (int k = 0; k < ST_COUNT; k++) c->hbase[(size_t)k * (n + 1) + i + 1] = c->hbase[(size_t)k * (n + 1) + i] + counts[k];
    const pf_frame_side* s = refs[i].s;
    if (counts[ST_DEBLOCK_V]) done |= PF_STAGE_LOOP_FILTER;
    if (cdef_any(refs[i].f, s)) done |= PF_STAGE_CDEF;
    if (lr_any(s)) done |= PF_STAGE_LOOP_RESTORATION;
    if (s->stages & PF_STAGE_EXTEND_BORDERS) done |= PF_STAGE_EXTEND_BORDERS;
    if (counts[ST_FG_TEMPLATES]) done |= PF_STAGE_FILM_GRAIN;
  }
  CK(c->jobs.ensure(sizeof(FrameJob) * n));
  CK(c->bases.ensure(sizeof(int) * c->hbase.size()));
  CK(c->counters.ensure(sizeof(int) * ST_COUNT * 2));  // one set per frame group
  *fg = c->hbase[(size_t)ST_FG_TEMPLATES * (n + 1) + n] > 0;
  *completed = done;
  return PF_OK;
}

static void add_stats(const pf_ctx* c, int n, uint32_t done, pf_stats* stats) {
  if (!stats) return;
  auto total = [&](int k) { return c->hbase[(size_t)k * (n + 1) + n]; };
  stats->completed |= done;
  stats->cdef_units += total(ST_CDEF);
  stats->lr_units += total(ST_LR);
  stats->fg_rows += total(ST_FG_OFFSETS);
}

// Builds the job table for n validated frames and queues every stage.
static int run_batch(pf_ctx* c, const FrameRef* refs, int n, pf_stats* stats, bool useGraph = false) {
  uint32_t done = 0;
  bool fg = false;
  // The previous batch's side information may still be on its way up.
  if (c->side_pending) {
    CKW(wait_event(c, c->side_done, __LINE__));
    c->side_pending = false;
  }
  int st = prepare_batch(c, refs, n, c->hside, c->sidebuf, &done, &fg);
  if (st != PF_OK) return st;
  const int est = (useGraph && !c->timing)
                      ? replay_or_capture(c, n, fg)
                      : enqueue_batch(c, c->hjobs.data(), c->hbase.data(), c->hside.data(), c->hside.size(), n, fg);
  if (est != PF_OK) return est;
  if (stats) {
    stats->completed = 0;
    stats->cdef_units = stats->lr_units = stats->fg_rows = 0;
  }
  add_stats(c, n, done, stats);
  return PF_OK;
}

static void read_stage_times(pf_ctx* c, pf_stats* stats) {
  if (!stats || !c->timing) return;
  for (int i = 0; i < 5; i++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c->ev[i], c->ev[i + 1]) != cudaSuccess) {
      ms = -1.f;
      (void)cudaGetLastError();  // a timing read is not a device fault
    }
    stats->stage_ms[i] = ms;
  }
}

// Byte offset of each plane from plane 0 when a host frame's planes lie back
// to back in one buffer, as goav1's frame.Bind lays them out (Y, U, V
// consecutive, each stride x aligned height: frame/buffer.go:141-236), with
// 16-byte multiples for the offsets and strides and rows padded by less than
// 256 bytes; -1 otherwise.
static int64_t contiguous_span(const pf_frame* f, int64_t off[3]) {
  const int bps = bps_of(f);
  const uint8_t* base = (const uint8_t*)f->plane[0].data;
  int64_t at = 0;
  for (int p = 0; p < 3; p++) {
    const pf_plane& pl = f->plane[p];
    const int64_t row = (int64_t)pl.alloc_width * bps;
    if ((const uint8_t*)pl.data != base + at || pl.stride < row || pl.stride - row >= 256 || pl.stride % 16 ||
        at % 16)
      return -1;
    off[p] = at;
    at += pl.stride * pl.alloc_height;
  }
  return at;
}

// Device layout of a host frame's planes at `base`: the host layout itself
// when its planes are back to back (the frame then moves as one copy), else
// each plane 256-byte aligned, with the host pitch when rows are packed
// (pitch = row bytes, a multiple of 16: the plane moves as one contiguous
// copy) or rows padded to 256 bytes.
static size_t host_frame_layout(const pf_frame* f, uint8_t* base, void** ptrs, int64_t* strides) {
  int64_t off[3];
  const int64_t span = contiguous_span(f, off);
  if (span > 0) {
    for (int p = 0; p < 3; p++) {
      strides[p] = f->plane[p].stride;
      if (ptrs) ptrs[p] = base + off[p];
    }
    return align256((size_t)span);
  }
  const int bps = bps_of(f);
  size_t total = 0;
  for (int p = 0; p < 3; p++) {
    const pf_plane& pl = f->plane[p];
    const int64_t row = (int64_t)pl.alloc_width * bps;
    strides[p] = pl.stride == row && row % 16 == 0 ? row : (row + 255) & ~(int64_t)255;
    if (ptrs) ptrs[p] = base + total;
    total = align256(total + (size_t)strides[p] * pl.alloc_height);
  }
  return total;
}

// Host <-> device copies of a frame laid out by host_frame_layout: one copy
// for a back-to-back frame, else one per plane (2-D when the pitches differ).
static cudaError_t copy_planes(const pf_frame* f, void* const* dev, const int64_t* ds, bool up, cudaStream_t st) {
  int64_t off[3];
  const int64_t span = contiguous_span(f, off);
  if (span > 0 && (uint8_t*)dev[1] - (uint8_t*)dev[0] == off[1] && (uint8_t*)dev[2] - (uint8_t*)dev[0] == off[2] &&
      ds[0] == f->plane[0].stride && ds[1] == f->plane[1].stride && ds[2] == f->plane[2].stride)
    return up ? cudaMemcpyAsync(dev[0], f->plane[0].data, (size_t)span, cudaMemcpyHostToDevice, st)
              : cudaMemcpyAsync(f->plane[0].data, dev[0], (size_t)span, cudaMemcpyDeviceToHost, st);
  const int bps = bps_of(f);
  for (int p = 0; p < 3; p++) {
    const pf_plane& pl = f->plane[p];
    const size_t w = (size_t)pl.alloc_width * bps;
    cudaError_t e;
    if (ds[p] == pl.stride && (size_t)pl.stride == w) {
      const size_t bytes = w * pl.alloc_height;
      e = up ? cudaMemcpyAsync(dev[p], pl.data, bytes, cudaMemcpyHostToDevice, st)
             : cudaMemcpyAsync(pl.data, dev[p], bytes, cudaMemcpyDeviceToHost, st);
    } else {
      e = up ? cudaMemcpy2DAsync(dev[p], ds[p], pl.data, pl.stride, w, pl.alloc_height, cudaMemcpyHostToDevice, st)
             : cudaMemcpy2DAsync(pl.data, pl.stride, dev[p], ds[p], w, pl.alloc_height, cudaMemcpyDeviceToHost, st);
    }
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

extern "C" int pf_frame_apply(pf_ctx* c, const pf_frame* f, const pf_frame_side* s, const pf_frame* display,
                              pf_stats* stats) {
  if (!c) return PF_ERR_INVALID_ARG;
  FrameRef r;
  memset(&r, 0, sizeof(r));
  // A host frame's upload goes out first, once the frame's own planes are
  // known to be what it describes (the copy reads exactly those); the
  // side information's validation (a scan of its level cache on the host)
  // then runs while the frame is on its way.  A rejected call has only
  // written the context's staging.
  const bool early = f && s && f->memory == PF_MEM_HOST && plane_dims_ok(f);
  if (early) {
    CK(cudaSetDevice(c->device));
    CK(c->io.ensure(host_frame_layout(f, nullptr, nullptr, r.ioStride) + 256));
    host_frame_layout(f, (uint8_t*)c->io.p, r.io, r.ioStride);
    CK(copy_planes(f, r.io, r.ioStride, true, c->stream));
  }
  int st = pf_frame_validate(f, s, display);
  if (st != PF_OK) return st;
  CK(cudaSetDevice(c->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  const int bps = bps_of(f);
  r.f = f;
  r.s = s;
  const bool wantDisp = (s->stages & PF_STAGE_FILM_GRAIN) && display;
  r.display = wantDisp ? display : nullptr;
  if (f->memory == PF_MEM_HOST) {
    if (!early) return PF_ERR_SHORT_BUFFER;  // unreachable: validation checks the planes too
  } else {
    for (int p = 0; p < 3; p++) {
      r.io[p] = f->plane[p].data;
      r.ioStride[p] = f->plane[p].stride;
    }
  }
  if (wantDisp) {
    if (display->memory == PF_MEM_HOST) {
      CK(c->disp.ensure(host_frame_layout(display, nullptr, nullptr, r.dStride) + 256));
      host_frame_layout(display, (uint8_t*)c->disp.p, r.dp, r.dStride);
    } else {
      for (int p = 0; p < 3; p++) {
        r.dp[p] = display->plane[p].data;
        r.dStride[p] = display->plane[p].stride;
      }
    }
  }
  // Host reference and display frames: the reference frame goes down on the
  // copy stream as soon as the border extension has run, beside the grain
  // stage and ahead of the display frame's download.
  const bool split = f->memory == PF_MEM_HOST && wantDisp && display->memory == PF_MEM_HOST;
  if (split && !c->d2h) {
    CK(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
  }
  if (split && !c->chain_done) CK(cudaEventCreateWithFlags(&c->chain_done, cudaEventDisableTiming));
  c->mark_chain = split;
  st = run_batch(c, &r, 1, stats, c->graphs != 0);
  c->mark_chain = false;
  if (st != PF_OK) return st;
  if (split) {
    CK(cudaStreamWaitEvent(c->d2h, c->chain_done, 0));
    CK(copy_planes(f, r.io, r.ioStride, false, c->d2h));
  } else if (f->memory == PF_MEM_HOST) {
    CK(copy_planes(f, r.io, r.ioStride, false, c->stream));
  }
  if (wantDisp && display->memory == PF_MEM_HOST) CK(copy_planes(display, r.dp, r.dStride, false, c->stream));
  if (f->memory == PF_MEM_HOST || (wantDisp && display->memory == PF_MEM_HOST) || c->timing) {
    CKW(wait_stream(c, c->stream, __LINE__));
    if (split) CKW(wait_stream(c, c->d2h, __LINE__));
    read_stage_times(c, stats);
  }
  CK(cudaGetLastError());
  return PF_OK;
}

static cudaError_t pinned_ensure(void** p, size_t* n, size_t need) {
  if (need <= *n) return cudaSuccess;
  if (*p) cudaFreeHost(*p);
  *p = nullptr;
  *n = 0;
  need = (need + 4095) & ~(size_t)4095;
  const cudaError_t e = cudaMallocHost(p, need);
  if (e == cudaSuccess) *n = need;
  return e;
}

// A batch of host frames: chunks of c->host_chunk frames flow through a
// ring of three device slots, the upload of one chunk (stream h2d), the
// filtering of the previous one (the main stream) and the download of the
// one before (stream d2h) overlapping.  The chain itself is run_batch's,
// unchanged; only the frames' home differs.  Page-locked host frames let the
// copies run asynchronously; pageable ones are still correct, copied
// synchronously.
static int run_host_pipeline(pf_ctx* c, const pf_batch_item* items, int n, pf_stats* stats) {
  if (!c->h2d) {
    CK(cudaStreamCreateWithFlags(&c->h2d, cudaStreamNonBlocking));
    CK(cudaStreamCreateWithFlags(&c->d2h, cudaStreamNonBlocking));
    for (pf_ctx::HostSlot& h : c->hslot) {
      CK(cudaEventCreateWithFlags(&h.up, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h.comp, cudaEventDisableTiming));
      CK(cudaEventCreateWithFlags(&h.down, cudaEventDisableTiming));
    }
  }
  const int chunk = std::max(1, c->host_chunk);
  const int nchunks = (n + chunk - 1) / chunk;
  // The shared scratch is sized for the largest chunk before anything is
  // queued, so it never moves while a chunk is in flight.
  size_t maxArena = 0, maxSide = 0;
  for (int k = 0; k < nchunks; k++) {
    size_t a = 0, b = 0;
    for (int i = k * chunk; i < std::min(n, (k + 1) * chunk); i++) {
      a += frame_scratch(items[i].frame, items[i].side);
      b += frame_side_bytes(items[i].frame, items[i].side);
    }
    maxArena = std::max(maxArena, a);
    maxSide = std::max(maxSide, b);
  }
  CK(c->arena.ensure(maxArena + 256));
  for (pf_ctx::HostSlot& h : c->hslot)
    if (h.dside.n < maxSide + 256) {
      if (h.used) CKW(wait_event(c, h.comp, __LINE__));
      CK(h.dside.ensure(maxSide + 256));
    }
  if (stats) memset(stats, 0, sizeof(*stats));
  std::vector<FrameRef> refs((size_t)chunk);
  for (int k = 0; k < nchunks; k++) {
    pf_ctx::HostSlot& h = c->hslot[k % 3];
    const int i0 = k * chunk, m = std::min(chunk, n - i0);
    // The slot's tables were read by its previous chunk's launch.
    if (h.used) CKW(wait_event(c, h.comp, __LINE__));
    size_t ioBytes = 0, dBytes = 0;
    for (int i = 0; i < m; i++) {
      const pf_batch_item& it = items[i0 + i];
      int64_t st[3];
      ioBytes += host_frame_layout(it.frame, nullptr, nullptr, st);
      if ((it.side->stages & PF_STAGE_FILM_GRAIN) && it.display)
        dBytes += host_frame_layout(it.display, nullptr, nullptr, st);
    }
    if (h.used && (ioBytes > h.io.n || dBytes > h.disp.n)) CKW(wait_event(c, h.down, __LINE__));
    CK(h.io.ensure(ioBytes + 256));
    CK(h.disp.ensure(dBytes + 256));
    if (h.used) CK(cudaStreamWaitEvent(c->h2d, h.down, 0));
    size_t oi = 0, od = 0;
    for (int i = 0; i < m; i++) {
      const pf_batch_item& it = items[i0 + i];
      FrameRef& r = refs[i];
      memset(&r, 0, sizeof(r));
      r.f = it.frame;
      r.s = it.side;
      const bool wantDisp = (it.side->stages & PF_STAGE_FILM_GRAIN) && it.display;
      r.display = wantDisp ? it.display : nullptr;
      oi += host_frame_layout(it.frame, (uint8_t*)h.io.p + oi, r.io, r.ioStride);
      if (wantDisp) od += host_frame_layout(it.display, (uint8_t*)h.disp.p + od, r.dp, r.dStride);
      CK(copy_planes(it.frame, r.io, r.ioStride, true, c->h2d));
    }
    // The chunk's tables go up with its frames, on the upload stream, into
    // the slot's own device buffers: the launch then waits for nothing but
    // the upload event, and no small copy queues behind the next chunk's
    // frames on the copy engine.
    uint32_t done = 0;
    bool fg = false;
    int st;
    try {
      st = prepare_batch(c, refs.data(), m, h.side, h.dside, &done, &fg);  // side information straight into pinned memory
    } catch (const std::bad_alloc&) {
      return PF_ERR_DEVICE;
    }
    if (st != PF_OK) return st;
    const size_t nj = sizeof(FrameJob) * m, nb = sizeof(int) * c->hbase.size();
    CK(pinned_ensure(&h.pjobs, &h.njobs, nj + 16));
    CK(pinned_ensure(&h.pbase, &h.nbase, nb + 16));
    CK(h.djobs.ensure(nj + 16));
    CK(h.dbases.ensure(nb + 16));
    memcpy(h.pjobs, c->hjobs.data(), nj);
    memcpy(h.pbase, c->hbase.data(), nb);
    if (!h.side.empty()) CK(cudaMemcpyAsync(h.dside.p, h.side.data(), h.side.size(), cudaMemcpyHostToDevice, c->h2d));
    CK(cudaMemcpyAsync(h.djobs.p, h.pjobs, nj, cudaMemcpyHostToDevice, c->h2d));
    CK(cudaMemcpyAsync(h.dbases.p, h.pbase, nb, cudaMemcpyHostToDevice, c->h2d));
    CK(cudaEventRecord(h.up, c->h2d));
    CK(cudaStreamWaitEvent(c->stream, h.up, 0));
    st = enqueue_batch(c, (const FrameJob*)h.pjobs, (const int*)h.pbase, nullptr, 0, m, fg, h.djobs.p, h.dbases.p);
    if (st != PF_OK) return st;
    add_stats(c, m, done, stats);
    CK(cudaEventRecord(h.comp, c->stream));
    CK(cudaStreamWaitEvent(c->d2h, h.comp, 0));
    for (int i = 0; i < m; i++) {
      CK(copy_planes(refs[i].f, refs[i].io, refs[i].ioStride, false, c->d2h));
      if (refs[i].display) CK(copy_planes(refs[i].display, refs[i].dp, refs[i].dStride, false, c->d2h));
    }
    CK(cudaEventRecord(h.down, c->d2h));
    h.used = true;
  }
  CKW(wait_stream(c, c->d2h, __LINE__));
  CKW(wait_stream(c, c->stream, __LINE__));
  read_stage_times(c, stats);
  CK(cudaGetLastError());
  return PF_OK;
}

// A super-resolved frame (FrameSize.SuperResEnabled): the decoder's order,
// internal/av1/decoder/postfilter.go:336-345 and postfilter_superres.go:
// deblock and CDEF on the coded frame, the restoration stripe-boundary rows
// saved from the deblocked coded rows and upscaled
// (tile/restoration_boundary.go:257-406), the CDEF output upscaled
// (superres.UpscalePlaneCoded), then restoration, border extension and grain
// on the upscaled frame.
// A super-resolved frame's arguments checked, and its side information split
// into the coded-grid stages (sa: deblocking, CDEF) and the upscaled-grid
// ones (sb: restoration, extension, grain).
static int superres_validate(const pf_frame* coded, const pf_frame_side* s, const pf_frame* up,
                             const pf_frame* display, pf_frame_side* sa, pf_frame_side* sb) {
  if (!coded || !s || !up) return PF_ERR_INVALID_ARG;
  if (s->stages & ~0x1Fu) return PF_ERR_UNSUPPORTED;
  if (coded->memory > PF_MEM_DEVICE || up->memory != coded->memory) return PF_ERR_INVALID_ARG;
  if (up->bit_depth != coded->bit_depth || up->ss_x != coded->ss_x || up->ss_y != coded->ss_y ||
      up->mono != coded->mono || up->height != coded->height || up->width <= coded->width || up->width > 16384)
    return PF_ERR_INVALID_FORMAT;
  *sa = *s;
  *sb = *s;
  sa->stages = s->stages & (PF_STAGE_LOOP_FILTER | PF_STAGE_CDEF);
  sb->stages = s->stages & (PF_STAGE_LOOP_RESTORATION | PF_STAGE_EXTEND_BORDERS | PF_STAGE_FILM_GRAIN);
  const bool wantDisp = (sb->stages & PF_STAGE_FILM_GRAIN) && display;
  if (wantDisp && display->memory != up->memory) return PF_ERR_INVALID_ARG;
  int st = pf_frame_validate(coded, sa, nullptr);
  if (st == PF_OK) st = pf_frame_validate(up, sb, display);
  return st;
}

// Rows of upscaled restoration boundary lines a super-resolved frame needs
// per plane (0: none), and their pitch.
static size_t superres_line_bytes(const pf_frame* up, const pf_frame_side* sb, int nb[3], int64_t lstride[3]) {
  size_t total = 0;
  const int bps = bps_of(up);
  for (int p = 0; p < 3; p++) {
    nb[p] = 0;
    lstride[p] = 0;
    if (!lr_any(sb) || p >= (up->mono ? 1 : 3) || sb->lr.type[p] == PF_LR_NONE) continue;
    const int sy = p ? up->ss_y : 0;
    nb[p] = (up->plane[p].height + (8 >> sy)) / (64 >> sy) + 2;
    lstride[p] = (int64_t)align256((size_t)up->plane[p].width * bps);
    total += align256((size_t)nb[p] * 4 * lstride[p]);
  }
  return total;
}

extern "C" int pf_frame_apply_superres(pf_ctx* c, const pf_frame* coded, const pf_frame_side* s,
                                       const pf_frame* up, const pf_frame* display, pf_stats* stats) {
  if (!c) return PF_ERR_INVALID_ARG;
  pf_frame_side sa, sb;
  int st = superres_validate(coded, s, up, display, &sa, &sb);
  if (st != PF_OK) return st;
  const bool wantDisp = (sb.stages & PF_STAGE_FILM_GRAIN) && display;
  CK(cudaSetDevice(c->device));
  if (stats) memset(stats, 0, sizeof(*stats));
  const int bps = bps_of(coded);
  const int nplanes = coded->mono ? 1 : 3;
  const bool host = coded->memory == PF_MEM_HOST;
  const cudaStream_t cs = c->stream;
  void *cio[3] = {}, *uio[3] = {}, *dio[3] = {};
  int64_t cst[3] = {}, ust[3] = {}, dst3[3] = {};
  if (host) {
    CK(layout_like(coded, c->io, cio, cst));
    CK(layout_like(up, c->sr_up, uio, ust));
    if (wantDisp) CK(layout_like(display, c->disp, dio, dst3));
    // Both frames go up: the upscale writes only the upscaled crop, and what
    // lies around it must come back as the caller left it.
    for (int p = 0; p < 3; p++) {
      CK(cudaMemcpy2DAsync(cio[p], cst[p], coded->plane[p].data, coded->plane[p].stride,
                           (size_t)coded->plane[p].alloc_width * bps, coded->plane[p].alloc_height,
                           cudaMemcpyHostToDevice, cs));
      CK(cudaMemcpy2DAsync(uio[p], ust[p], up->plane[p].data, up->plane[p].stride,
                           (size_t)up->plane[p].alloc_width * bps, up->plane[p].alloc_height,
                           cudaMemcpyHostToDevice, cs));
    }
  } else {
    for (int p = 0; p < 3; p++) {
      cio[p] = coded->plane[p].data;
      cst[p] = coded->plane[p].stride;
      uio[p] = up->plane[p].data;
      ust[p] = up->plane[p].stride;
      if (wantDisp) {
        dio[p] = display->plane[p].data;
        dst3[p] = display->plane[p].stride;
      }
    }
  }
  auto ref_of = [](const pf_frame* f, const pf_frame_side* side, void* const* io, const int64_t* ios) {
    FrameRef x;
    memset(&x, 0, sizeof(x));
    x.f = f;
    x.s = side;
    for (int p = 0; p < 3; p++) {
      x.io[p] = io[p];
      x.ioStride[p] = ios[p];
    }
    return x;
  };
  uint32_t done = 0;
  if (sa.stages & PF_STAGE_LOOP_FILTER) {
    pf_frame_side s1 = sa;
    s1.stages = PF_STAGE_LOOP_FILTER;
    const FrameRef x = ref_of(coded, &s1, cio, cst);
    if ((st = run_batch(c, &x, 1, nullptr)) != PF_OK) return st;
    done |= PF_STAGE_LOOP_FILTER;
  }
  // The deblocked coded rows around the stripe boundaries, upscaled.
  uint8_t* lines[3] = {};
  int64_t lstride[3] = {};
  if (lr_any(&sb)) {
    int nb[3];
    const size_t total = superres_line_bytes(up, &sb, nb, lstride);
    CK(c->sr_lines.ensure(total + 256));
    size_t off = 0;
    for (int p = 0; p < nplanes; p++)
      if (nb[p]) {
        lines[p] = (uint8_t*)c->sr_lines.p + off;
        off += align256((size_t)nb[p] * 4 * lstride[p]);
      }
    CK(launch_superres_lines((const uint8_t* const*)cio, cst, lines, lstride, nb, coded, up->width, cs));
  }
  if ((sa.stages & PF_STAGE_CDEF) && cdef_any(coded, &sa)) {
    pf_frame_side s2 = sa;
    s2.stages = PF_STAGE_CDEF;
    const FrameRef x = ref_of(coded, &s2, cio, cst);
    if ((st = run_batch(c, &x, 1, nullptr)) != PF_OK) return st;
    done |= PF_STAGE_CDEF;
  }
  CK(launch_superres_frame((const uint8_t* const*)cio, cst, (uint8_t* const*)uio, ust, coded, up->width, cs));
  if (sb.stages) {
    FrameRef x = ref_of(up, &sb, uio, ust);
    x.display = wantDisp ? display : nullptr;
    for (int p = 0; p < 3; p++) {
      x.dp[p] = dio[p];
      x.dStride[p] = dst3[p];
      x.ext_lines[p] = lines[p];
      x.ext_line_stride[p] = lstride[p];
    }
    if ((st = run_batch(c, &x, 1, stats)) != PF_OK) return st;
  }
  if (host) {
    auto down = [&](const pf_frame* f, void* const* dev, const int64_t* ds) -> cudaError_t {
      for (int p = 0; p < nplanes; p++) {
        const cudaError_t e = cudaMemcpy2DAsync(f->plane[p].data, f->plane[p].stride, dev[p], ds[p],
                                                (size_t)f->plane[p].alloc_width * bps, f->plane[p].alloc_height,
                                                cudaMemcpyDeviceToHost, cs);
        if (e != cudaSuccess) return e;
      }
      return cudaSuccess;
    };
    CK(down(coded, cio, cst));
    CK(down(up, uio, ust));
    if (wantDisp) CK(down(display, dio, dst3));
  }
  CKW(wait_stream(c, cs, __LINE__));
  if (stats) {
    stats->completed |= done;
    read_stage_times(c, stats);
  }
  CK(cudaGetLastError());
  return PF_OK;
}

// A batch of super-resolved frames: each stage of the chain runs as one
// launch over every frame that has it (deblocking over the coded frames,
// then CDEF, then restoration / extension / grain over the upscaled ones);
// the boundary-line upscale and the frame upscale are launched per frame
// between them, in the decoder's order.  Device frames: returns once the
// work is queued; host frames: one pf_frame_apply_superres per item.
extern "C" int pf_batch_apply_superres(pf_ctx* c, const pf_superres_item* items, int32_t n, pf_stats* stats) {
  if (!c || !items || n <= 0) return PF_ERR_INVALID_ARG;
  std::vector<pf_frame_side> sa((size_t)n), sb((size_t)n);
  for (int i = 0; i < n; i++) {
    if (!items[i].coded || items[i].coded->memory != items[0].coded->memory) return PF_ERR_INVALID_ARG;
    const int st = superres_validate(items[i].coded, items[i].side, items[i].up, items[i].display, &sa[i], &sb[i]);
    if (st != PF_OK) return st;
  }
  if (stats) memset(stats, 0, sizeof(*stats));
  if (items[0].coded->memory == PF_MEM_HOST) {
    for (int i = 0; i < n; i++) {
      pf_stats one;
      const int st = pf_frame_apply_superres(c, items[i].coded, items[i].side, items[i].up, items[i].display,
                                             stats ? &one : nullptr);
      if (st != PF_OK) return st;
      if (stats) {
        stats->completed |= one.completed;
        stats->cdef_units += one.cdef_units;
        stats->lr_units += one.lr_units;
        stats->fg_rows += one.fg_rows;
      }
    }
    return PF_OK;
  }
  CK(cudaSetDevice(c->device));
  const cudaStream_t cs = c->stream;
  auto ref_of = [](const pf_frame* f, const pf_frame_side* side) {
    FrameRef x;
    memset(&x, 0, sizeof(x));
    x.f = f;
    x.s = side;
    for (int p = 0; p < 3; p++) {
      x.io[p] = f->plane[p].data;
      x.ioStride[p] = f->plane[p].stride;
    }
    return x;
  };
  pf_stats acc;
  memset(&acc, 0, sizeof(acc));
  auto run = [&](std::vector<FrameRef>& refs) {
    if (refs.empty()) return (int)PF_OK;
    pf_stats one;
    const int st = run_batch(c, refs.data(), (int)refs.size(), &one);
    acc.completed |= one.completed;
    acc.cdef_units += one.cdef_units;
    acc.lr_units += one.lr_units;
    acc.fg_rows += one.fg_rows;
    return st;
  };
  std::vector<pf_frame_side> s1((size_t)n), s2((size_t)n);
  std::vector<FrameRef> refs;
  refs.reserve((size_t)n);
  // Deblocking, every coded frame in one launch per pass.
  for (int i = 0; i < n; i++)
    if (sa[i].stages & PF_STAGE_LOOP_FILTER) {
      s1[i] = sa[i];
      s1[i].stages = PF_STAGE_LOOP_FILTER;
      refs.push_back(ref_of(items[i].coded, &s1[i]));
    }
  int st = run(refs);
  if (st != PF_OK) return st;
  // The deblocked rows around each frame's stripe boundaries, upscaled, into
  // one buffer for the whole batch.
  std::vector<int> nb((size_t)n * 3);
  std::vector<int64_t> lstride((size_t)n * 3);
  std::vector<size_t> loff((size_t)n);
  size_t ltotal = 0;
  for (int i = 0; i < n; i++) {
    loff[i] = ltotal;
    ltotal += superres_line_bytes(items[i].up, &sb[i], &nb[3 * i], &lstride[3 * i]);
  }
  if (ltotal) CK(c->sr_lines.ensure(ltotal + 256));
  std::vector<uint8_t*> lines((size_t)n * 3, nullptr);
  for (int i = 0; i < n; i++) {
    if (!lr_any(&sb[i])) continue;
    size_t off = loff[i];
    for (int p = 0; p < 3; p++)
      if (nb[3 * i + p]) {
        lines[3 * i + p] = (uint8_t*)c->sr_lines.p + off;
        off += align256((size_t)nb[3 * i + p] * 4 * lstride[3 * i + p]);
      }
    const pf_frame* cf = items[i].coded;
    void* cio[3] = {cf->plane[0].data, cf->plane[1].data, cf->plane[2].data};
    const int64_t cst[3] = {cf->plane[0].stride, cf->plane[1].stride, cf->plane[2].stride};
    CK(launch_superres_lines((const uint8_t* const*)cio, cst, &lines[3 * i], &lstride[3 * i], &nb[3 * i], cf,
                             items[i].up->width, cs));
  }
  // CDEF over the coded frames.
  refs.clear();
  for (int i = 0; i < n; i++)
    if ((sa[i].stages & PF_STAGE_CDEF) && cdef_any(items[i].coded, &sa[i])) {
      s2[i] = sa[i];
      s2[i].stages = PF_STAGE_CDEF;
      refs.push_back(ref_of(items[i].coded, &s2[i]));
    }
  if ((st = run(refs)) != PF_OK) return st;
  // Upscale, then the upscaled-grid stages over every frame.
  refs.clear();
  for (int i = 0; i < n; i++) {
    const pf_frame* cf = items[i].coded;
    const pf_frame* uf = items[i].up;
    void* cio[3] = {cf->plane[0].data, cf->plane[1].data, cf->plane[2].data};
    const int64_t cst[3] = {cf->plane[0].stride, cf->plane[1].stride, cf->plane[2].stride};
    void* uio[3] = {uf->plane[0].data, uf->plane[1].data, uf->plane[2].data};
    const int64_t ust[3] = {uf->plane[0].stride, uf->plane[1].stride, uf->plane[2].stride};
    CK(launch_superres_frame((const uint8_t* const*)cio, cst, (uint8_t* const*)uio, ust, cf, uf->width, cs));
    if (!sb[i].stages) continue;
    FrameRef x = ref_of(uf, &sb[i]);
    const bool wantDisp = (sb[i].stages & PF_STAGE_FILM_GRAIN) && items[i].display;
    x.display = wantDisp ? items[i].display : nullptr;
    for (int p = 0; p < 3; p++) {
      if (wantDisp) {
        x.dp[p] = items[i].display->plane[p].data;
        x.dStride[p] = items[i].display->plane[p].stride;
      }
      x.ext_lines[p] = lines[3 * i + p];
      x.ext_line_stride[p] = lstride[3 * i + p];
    }
    refs.push_back(x);
  }
  if ((st = run(refs)) != PF_OK) return st;
  if (stats) *stats = acc;
  CK(cudaGetLastError());
  return PF_OK;
}

// Validates a batch's frames on up to 8 host threads (the level-cache scan of
// a host frame is half a megabyte at 1080p) and returns the status of the
// first failing frame in batch order, as a serial scan would.
static int validate_items(const pf_batch_item* items, int n) {
  std::vector<int> st((size_t)n, PF_OK);
  int threads = std::min(8, (n + 3) / 4);
  threads = std::min(threads, (int)std::max(1u, std::thread::hardware_concurrency()));
  bool serial = threads <= 1;
  if (!serial) {
    std::vector<std::thread> pool;
    try {
      for (int t = 0; t < threads; t++)
        pool.emplace_back([&st, items, n, threads, t] {
          for (int i = t; i < n; i += threads) st[i] = pf_frame_validate(items[i].frame, items[i].side, items[i].display);
        });
    } catch (...) {
      serial = true;
    }
    for (std::thread& th : pool) th.join();
    if (serial)
      for (int i = 0; i < n; i++) st[i] = PF_OK;
  }
  for (int i = 0; i < n; i++) {
    if (serial) st[i] = pf_frame_validate(items[i].frame, items[i].side, items[i].display);
    if (st[i] != PF_OK) return st[i];
  }
  return PF_OK;
}

extern "C" int pf_batch_apply(pf_ctx* c, const pf_batch_item* items, int32_t n, pf_stats* stats) {
  if (!c || (!items && n > 0) || n < 0) return PF_ERR_INVALID_ARG;
  if (n > 65535) return PF_ERR_INVALID_ARG;
  const int vst = validate_items(items, n);
  if (vst != PF_OK) return vst;
  std::vector<FrameRef> refs((size_t)n);
  for (int i = 0; i < n; i++) {
    const pf_batch_item& it = items[i];
    const bool wantDisp = (it.side->stages & PF_STAGE_FILM_GRAIN) && it.display;
    // Every frame and display of a batch lives on the same side: all in
    // device memory, or all in host memory (run_host_pipeline).
    const int home = items[0].frame->memory;
    if (it.frame->memory != home || (wantDisp && it.display->memory != home)) return PF_ERR_INVALID_ARG;
    FrameRef& r = refs[i];
    memset(&r, 0, sizeof(r));
    r.f = it.frame;
    r.s = it.side;
    r.display = wantDisp ? it.display : nullptr;
    for (int p = 0; p < 3; p++) {
      r.io[p] = it.frame->plane[p].data;
      r.ioStride[p] = it.frame->plane[p].stride;
      if (wantDisp) {
        r.dp[p] = it.display->plane[p].data;
        r.dStride[p] = it.display->plane[p].stride;
      }
    }
  }
  CK(cudaSetDevice(c->device));
  if (n > 0 && items[0].frame->memory == PF_MEM_HOST) return run_host_pipeline(c, items, n, stats);
  if (stats) memset(stats, 0, sizeof(*stats));
  int st = run_batch(c, refs.data(), n, stats, c->graphs != 0);
  if (st != PF_OK) return st;
  bool hostSide = false;
  for (int i = 0; i < n; i++) hostSide |= items[i].side->side_memory == PF_MEM_HOST;
  if (hostSide || c->timing) {
    CKW(wait_stream(c, c->stream, __LINE__));
    read_stage_times(c, stats);
  }
  CK(cudaGetLastError());
  return PF_OK;
}

// Scratch and stream of a context for the encoder search (pf_search.cu).
void* pf_internal_search_scratch(pf_ctx* c, size_t bytes) {
  if (c->search.ensure(bytes) != cudaSuccess) return nullptr;
  return c->search.p;
}
void* pf_internal_stream(pf_ctx* c) { return (void*)c->stream; }
// The context's stage events when it times stages (pf_config.timing), else null.
cudaEvent_t* pf_internal_events(pf_ctx* c) { return c->timing ? c->ev : nullptr; }
// The context's CDEF constrain() tables (CdefArgs.ctab).
const int16_t* pf_internal_ctab(pf_ctx* c) { return (const int16_t*)c->ctab.p; }

// Page-locked host staging of at least `bytes` (grown, never shrunk), so
// small host inputs go up with an asynchronous copy.  Valid until the next
// call; the entry points using it end with a stream synchronisation.
void* pf_internal_pinned(pf_ctx* c, size_t bytes) {
  if (bytes > c->pinned_n) {
    if (c->pinned) cudaFreeHost(c->pinned);
    c->pinned = nullptr;
    c->pinned_n = 0;
    const size_t n = (bytes + 4095) & ~(size_t)4095;
    if (cudaMallocHost(&c->pinned, n) != cudaSuccess) return nullptr;
    c->pinned_n = n;
  }
  return c->pinned;
}

// Device copy of `bytes` of host data that rarely changes (the learned
// search's network): uploaded only when it differs from the last upload
// (*changed = 1 then).  `extra` device bytes follow it (256-aligned) for
// data derived from it, which the caller refreshes when it changed.
void* pf_internal_cached_upload(pf_ctx* c, const void* host, size_t bytes, size_t extra, cudaStream_t st,
                                int* changed) {
  *changed = 0;
  const size_t need = ((bytes + 255) & ~(size_t)255) + extra;
  if (need > c->model.n) c->model_shadow.clear();  // a new buffer holds nothing yet
  if (c->model.ensure(need) != cudaSuccess) return nullptr;
  if (c->model_shadow.size() == bytes && memcmp(c->model_shadow.data(), host, bytes) == 0) return c->model.p;
  *changed = 1;
  if (c->model_shadow.size() != bytes) {
    if (c->model_pin) cudaFreeHost(c->model_pin);
    c->model_pin = nullptr;
    if (cudaMallocHost(&c->model_pin, bytes) != cudaSuccess) return nullptr;
  }
  c->model_shadow.assign((const uint8_t*)host, (const uint8_t*)host + bytes);
  memcpy(c->model_pin, host, bytes);
  if (cudaMemcpyAsync(c->model.p, c->model_pin, bytes, cudaMemcpyHostToDevice, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess) {
    c->model_shadow.clear();
    return nullptr;
  }
  return c->model.p;
}

// ---------------------------------------------------------------------------
// Batch scheduling: graphs, persistent CTAs and the autotuner.

extern "C" int pf_batch_graphs(pf_ctx* c, int32_t enable) {
  if (!c || (enable != 0 && enable != 1)) return PF_ERR_INVALID_ARG;
  c->graphs = enable;
  if (!enable) {
    for (GraphEntry* g : c->gcache) delete g;
    c->gcache.clear();
  }
  return PF_OK;
}

// The stages each tunable group sets.
static const int kTuneStages[PF_TUNE_GROUPS][2] = {
    {ST_DEBLOCK_V, ST_DEBLOCK_H}, {ST_CDEF, -1}, {ST_LR, -1}, {ST_FG_APPLY, -1}};
static const int kTuneStatIndex[PF_TUNE_GROUPS] = {0, 1, 2, 4};  // pf_stats.stage_ms

static bool schedule_ok(int group, const pf_schedule& s) {
  return s.ctas >= 0 && s.ctas <= (1 << 20) && s.units_per_cta >= 1 && s.units_per_cta <= 16 && s.staging >= 0 &&
         s.staging <= 3 && (s.units_per_cta == 1 || s.staging < s.units_per_cta) && s.tile >= 0 &&
         s.tile <= (group == PF_TUNE_DEBLOCK || group == PF_TUNE_FILM_GRAIN ? 3 : 0);
}

extern "C" int pf_set_schedule(pf_ctx* c, int32_t group, const pf_schedule* s) {
  if (!c || !s || group < 0 || group >= PF_TUNE_GROUPS || !schedule_ok(group, *s)) return PF_ERR_INVALID_ARG;
  for (int k : kTuneStages[group])
    if (k >= 0) {
      c->persistent[k] = s->ctas;
      c->chunk[k] = s->units_per_cta;
      c->ahead[k] = s->staging;
      c->tile[k] = group == PF_TUNE_DEBLOCK ? 0 : s->tile;
    }
  if (group == PF_TUNE_DEBLOCK) c->db_tile = s->tile;
  return PF_OK;
}

extern "C" int pf_get_schedule(const pf_ctx* c, int32_t group, pf_schedule* s) {
  if (!c || !s || group < 0 || group >= PF_TUNE_GROUPS) return PF_ERR_INVALID_ARG;
  const int k = kTuneStages[group][0];
  s->ctas = c->persistent[k];
  s->units_per_cta = c->chunk[k];
  s->staging = c->ahead[k];
  s->tile = group == PF_TUNE_DEBLOCK ? c->db_tile : c->tile[k];
  return PF_OK;
}

extern "C" int pf_set_frame_groups(pf_ctx* c, int32_t groups) {
  if (!c || (groups != 1 && groups != 2)) return PF_ERR_INVALID_ARG;
  c->frame_groups = groups;
  return PF_OK;
}

extern "C" int pf_set_persistent(pf_ctx* c, int32_t group, int32_t ctas) {
  if (!c || group < 0 || group >= PF_TUNE_GROUPS || ctas < 0 || ctas > (1 << 20)) return PF_ERR_INVALID_ARG;
  for (int k : kTuneStages[group])
    if (k >= 0) c->persistent[k] = ctas;
  return PF_OK;
}

extern "C" int pf_autotune(pf_ctx* c, const pf_batch_item* items, int32_t n, int32_t reps, pf_tune_result* out) {
  if (!c || !items || n <= 0 || reps <= 0 || reps > 1000 || !out) return PF_ERR_INVALID_ARG;
  const int savedTiming = c->timing;
  c->timing = 1;  // per-stage CUDA events; no graphs while timing
  c->frame_groups = 1;  // per-stage times need one group
  memset(out, 0, sizeof(*out));
  int status = PF_OK;
  // Median stage time of group gi under schedule s.
  auto measure = [&](int gi, const pf_schedule& s, float* med) {
    pf_set_schedule(c, gi, &s);
    std::vector<float> t;
    for (int r = 0; r <= reps && status == PF_OK; r++) {  // run 0 warms up
      pf_stats st;
      status = pf_batch_apply(c, items, n, &st);
      if (r > 0 && status == PF_OK) t.push_back(st.stage_ms[kTuneStatIndex[gi]]);
    }
    if (status != PF_OK) return false;
    std::sort(t.begin(), t.end());
    *med = t[t.size() / 2];
    return true;
  };
  for (int gi = 0; gi < PF_TUNE_GROUPS && status == PF_OK; gi++) {
    pf_schedule best{0, 1, 0, 0};
    float bestMs = 0;
    if (!measure(gi, best, &bestMs)) break;
    out->ms_default[gi] = bestMs;
    // One dimension at a time, each from the best schedule so far.
    auto tryOne = [&](pf_schedule cand) {
      if (!schedule_ok(gi, cand) || status != PF_OK) return;
      float ms;
      if (measure(gi, cand, &ms) && ms < bestMs) {
        bestMs = ms;
        best = cand;
      }
    };
    for (int t = 1; t <= 3; t++) {  // tile settings the group has (schedule_ok)
      pf_schedule s = best;
      s.tile = t;
      tryOne(s);
    }
    for (int u : {2, 4, 8}) {
      pf_schedule s = best;
      s.units_per_cta = u;
      s.staging = 0;
      tryOne(s);
    }
    for (int d = 1; d <= 2; d++) {  // items (one per CTA: waves) prefetched ahead
      pf_schedule s = best;
      s.staging = d;
      tryOne(s);
    }
    for (int m : {1, 2, 4, 8, 16}) {
      pf_schedule s = best;
      s.ctas = m * c->sm_count;
      tryOne(s);
    }
    if (status != PF_OK) break;
    pf_set_schedule(c, gi, &best);
    out->chosen[gi] = best;
    out->ms[gi] = bestMs;
  }
  // Frame groups last, on the whole batch's time.
  for (int groups = 1; groups <= 2 && status == PF_OK; groups++) {
    c->frame_groups = groups;
    std::vector<float> t;
    for (int r = 0; r <= reps && status == PF_OK; r++) {
      pf_stats st;
      status = pf_batch_apply(c, items, n, &st);
      float sum = 0.f;
      for (int i = 0; i < 5; i++) sum += st.stage_ms[i];
      if (r > 0 && status == PF_OK) t.push_back(sum);
    }
    if (status != PF_OK) break;
    std::sort(t.begin(), t.end());
    out->ms_groups[groups - 1] = t[t.size() / 2];
  }
  c->frame_groups = out->ms_groups[1] < out->ms_groups[0] ? 2 : 1;
  out->frame_groups = c->frame_groups;
  c->timing = savedTiming;
  return status;
}
