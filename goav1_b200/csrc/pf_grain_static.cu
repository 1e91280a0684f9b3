// pf_grain_static.cu - film-grain synthesis that allocates nothing.
//
// pf_frame_apply keeps its scratch (grain templates, block offsets, the job
// table) in device buffers a pf_ctx allocates with cudaMalloc.  Some callers
// cannot make that call: a presentation thread that adds grain right before a
// frame is shown must not stall on cudaMalloc/cudaFree, which can synchronise
// the whole device; and an application whose device memory is already handed
// out by another allocator (a caching allocator that reserved the device up
// front) may have nothing left for a raw cudaMalloc.  pf_film_grain_static
// serves them: the caller passes the input (reference) and output (display)
// frames, and every byte of scratch lives in g_grain_scratch below, a
// file-scope device array of fixed size that each GPU loading this library
// holds until the process exits.
//
// The array is shared by every call on a device and keeps whatever the last
// call left in it.  Nothing in it has to start at zero: each call rewrites the
// job record, the stage table, all three templates and every offset it reads.
// Calls whose work overlaps on the GPU (two streams, or two threads) race on
// the array; callers must order them, e.g. by issuing them on one stream.
#include <mutex>

#include <string.h>

#include "pf_common.cuh"

namespace pf {
cudaError_t fg_upload_tables();
cudaError_t launch_fg_templates_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t launch_fg_offsets_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
cudaError_t launch_fg_apply_batch(const BatchArgs& b, int total, int grid, cudaStream_t st);
}  // namespace pf

using namespace pf;

namespace {

// Scratch layout (bytes): [job record | stage table | 3 grain templates | offsets].
constexpr size_t kJobBytes = 8192;
constexpr size_t kBaseOff = kJobBytes;
constexpr size_t kGrainOff = kBaseOff + 256;
constexpr size_t kGrainBytes = 36096;  // 3 * 82 * 73 int16, rounded up to 256
constexpr size_t kOffsetsOff = kGrainOff + kGrainBytes;
static_assert(sizeof(FrameJob) <= kJobBytes, "job record does not fit its scratch slot");
static_assert(kOffsetsOff + PF_GRAIN_STATIC_MAX_BLOCKS <= PF_GRAIN_STATIC_SCRATCH_BYTES, "scratch too small");

}  // namespace

static __device__ __align__(256) uint8_t g_grain_scratch[PF_GRAIN_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
uint8_t* g_scratch_addr[kMaxDevices];  // device address of g_grain_scratch, per device

// Once per device, with that device current: the device address of the
// scratch array (host code cannot use the symbol itself as an address) and
// the grain tables in constant memory.
int setup_device(int dev, uint8_t** out) {
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_grain_scratch) != cudaSuccess || !p) return PF_ERR_DEVICE;
    if (fg_upload_tables() != cudaSuccess) return PF_ERR_DEVICE;
    g_scratch_addr[dev] = (uint8_t*)p;
  }
  *out = g_scratch_addr[dev];
  return PF_OK;
}

DFrame device_frame(const pf_frame* f) {
  DFrame d;
  memset(&d, 0, sizeof(d));
  d.width = f->width;
  d.height = f->height;
  d.bd = f->bit_depth;
  d.ssx = f->ss_x;
  d.ssy = f->ss_y;
  d.mono = f->mono;
  for (int p = 0; p < 3; p++) {
    d.pl[p].ptr = (uint8_t*)f->plane[p].data;
    d.pl[p].stride = f->plane[p].stride;
    d.pl[p].w = f->plane[p].width;
    d.pl[p].h = f->plane[p].height;
    d.pl[p].aw = f->plane[p].alloc_width;
    d.pl[p].ah = f->plane[p].alloc_height;
  }
  return d;
}

// The 256-entry scaling table of a piecewise-linear point list (the AV1
// film-grain scaling function; filmgrain/scaling.go:18-48 in goav1).
void scaling_table(uint8_t* dst, const uint8_t (*pts)[2], int n) {
  memset(dst, 0, 256);
  if (n == 0) return;
  for (int x = 0; x < pts[0][0]; x++) dst[x] = pts[0][1];
  for (int i = 0; i + 1 < n; i++) {
    const int dx = pts[i + 1][0] - pts[i][0], dy = pts[i + 1][1] - pts[i][1];
    const int64_t slope = (int64_t)dy * ((65536 + (dx >> 1)) / dx);
    for (int x = 0; x < dx; x++) dst[pts[i][0] + x] = (uint8_t)(pts[i][1] + (int)(((int64_t)x * slope + 32768) >> 16));
  }
  for (int x = pts[n - 1][0]; x < 256; x++) dst[x] = pts[n - 1][1];
}

}  // namespace

extern "C" int pf_film_grain_static(const pf_frame* ref, const pf_film_grain* fg, const pf_frame* display,
                                    void* stream) {
  if (!ref || !fg || !display) return PF_ERR_INVALID_ARG;
  pf_frame_side side;
  memset(&side, 0, sizeof(side));
  side.stages = PF_STAGE_FILM_GRAIN;
  side.side_memory = PF_MEM_DEVICE;
  side.fg = *fg;
  int st = pf_frame_validate(ref, &side, display);
  if (st != PF_OK) return st;
  if (ref->memory != PF_MEM_DEVICE || display->memory != PF_MEM_DEVICE) return PF_ERR_INVALID_ARG;
  const int rows = (ref->height + 31) / 32, cols = (ref->width + 31) / 32;
  if ((int64_t)rows * cols > PF_GRAIN_STATIC_MAX_BLOCKS) return PF_ERR_SHORT_BUFFER;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return PF_ERR_DEVICE;
  uint8_t* scratch = nullptr;
  st = setup_device(dev, &scratch);
  if (st != PF_OK) return st;

  // The one-frame job: film grain only.
  FrameJob J;
  memset(&J, 0, sizeof(J));
  J.io = device_frame(ref);
  J.disp = device_frame(display);
  FgArgs& a = J.fg;
  const int act[3] = {fg->apply && fg->num_y_points != 0,
                      fg->apply && !ref->mono && (fg->num_cb_points != 0 || fg->chroma_scaling_from_luma),
                      fg->apply && !ref->mono && (fg->num_cr_points != 0 || fg->chroma_scaling_from_luma)};
  const bool on = act[0] || act[1] || act[2];
  int counts[ST_COUNT] = {};
  if (on) {
    int16_t* grain = (int16_t*)(scratch + kGrainOff);
    for (int p = 0; p < 3; p++) {
      a.grain[p] = grain + p * 82 * 73;
      a.active[p] = act[p];
    }
    a.offsets = scratch + kOffsetsOff;
    a.off_rows = rows;
    a.off_cols = cols;
    scaling_table(a.lut[0], fg->y_points, fg->num_y_points);
    if (fg->chroma_scaling_from_luma) {
      memcpy(a.lut[1], a.lut[0], 256);
      memcpy(a.lut[2], a.lut[0], 256);
    } else {
      scaling_table(a.lut[1], fg->cb_points, fg->num_cb_points);
      scaling_table(a.lut[2], fg->cr_points, fg->num_cr_points);
    }
    a.scaling_shift = fg->scaling_shift;
    a.overlap = fg->overlap;
    a.clip_restricted = fg->clip_to_restricted_range;
    a.matrix_identity = fg->matrix_identity;
    a.cfl = fg->chroma_scaling_from_luma;
    a.mult[1] = fg->cb_mult;
    a.luma_mult[1] = fg->cb_luma_mult;
    a.offset[1] = fg->cb_offset;
    a.mult[2] = fg->cr_mult;
    a.luma_mult[2] = fg->cr_luma_mult;
    a.offset[2] = fg->cr_offset;
    a.odd_luma = ref->ss_x && (ref->width & 1);
    FgTemplateArgs& t = J.fgt;
    t.seed = fg->seed;
    t.bd = ref->bit_depth;
    t.num_y_points = fg->num_y_points;
    t.grain_scale_shift = fg->grain_scale_shift;
    t.lag = fg->ar_coeff_lag;
    t.coeff_shift = fg->ar_coeff_shift;
    memcpy(t.coeffs[0], fg->ar_coeffs_y, 24);
    memcpy(t.coeffs[1], fg->ar_coeffs_cb, 25);
    memcpy(t.coeffs[2], fg->ar_coeffs_cr, 25);
    for (int p = 0; p < 3; p++) t.active[p] = act[p];
    t.ssx = ref->ss_x;
    t.ssy = ref->ss_y;
    counts[ST_FG_TEMPLATES] = 1;
    counts[ST_FG_OFFSETS] = (rows + 63) / 64;
  }
  int tiles = 0;
  for (int p = 0; p < (ref->mono ? 1 : 3); p++) {
    J.fg_tx[p] = (ref->plane[p].alloc_width + 63) / 64;
    J.fg_ty[p] = (ref->plane[p].alloc_height + 63) / 64;
    tiles += J.fg_tx[p] * J.fg_ty[p];
  }
  counts[ST_FG_APPLY] = tiles;
  int base[ST_COUNT * 2];
  for (int k = 0; k < ST_COUNT; k++) {
    base[2 * k] = 0;
    base[2 * k + 1] = counts[k];
  }
  // Pageable host sources: each copy returns once its bytes are staged, so
  // the stack records above may go out of scope afterwards.
  const cudaStream_t s = (cudaStream_t)stream;
  if (cudaMemcpyAsync(scratch, &J, sizeof(J), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyAsync(scratch + kBaseOff, base, sizeof(base), cudaMemcpyHostToDevice, s) != cudaSuccess)
    return PF_ERR_DEVICE;
  BatchArgs b;
  b.jobs = (const FrameJob*)scratch;
  b.base = (const int*)(scratch + kBaseOff);
  b.n = 1;
  b.counters = nullptr;
  if (launch_fg_templates_batch(b, counts[ST_FG_TEMPLATES], counts[ST_FG_TEMPLATES], s) != cudaSuccess ||
      launch_fg_offsets_batch(b, counts[ST_FG_OFFSETS], counts[ST_FG_OFFSETS], s) != cudaSuccess ||
      launch_fg_apply_batch(b, counts[ST_FG_APPLY], counts[ST_FG_APPLY], s) != cudaSuccess)
    return PF_ERR_DEVICE;
  return PF_OK;
}
