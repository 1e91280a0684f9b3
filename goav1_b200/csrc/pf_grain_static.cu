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
// The job record and stage table reach the array through a one-CTA kernel
// that takes them as its by-value argument, so no host buffer is read after
// the call returns.  Calls whose work overlaps on the GPU (two streams, or two
// threads) race on the array; callers must order them, e.g. by issuing them
// on one stream.
#include <mutex>

#include <string.h>

#include "pf_common.cuh"

namespace pf {
cudaError_t fg_upload_tables();
void build_scaling_lut(uint8_t* dst, const uint8_t (*pts)[2], int n);
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
bool g_tables_loaded[kMaxDevices];  // grain tables in this device's constant memory

// Per call, with the call's device current: the device address of the
// scratch array (host code cannot use the symbol itself as an address).  The
// first call on a device also loads the grain tables into constant memory and
// waits for that upload to land, so a first call made on a non-blocking
// stream cannot read the tables before they are written.  Tables live in the
// library's module: after cudaDeviceReset the process must not call this
// entry point again on that device.
int setup_device(int dev, uint8_t** out) {
  void* p = nullptr;
  if (cudaGetSymbolAddress(&p, g_grain_scratch) != cudaSuccess || !p) return PF_ERR_DEVICE;
  std::lock_guard<std::mutex> lock(g_setup_mu);
  if (!g_tables_loaded[dev]) {
    if (fg_upload_tables() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) return PF_ERR_DEVICE;
    g_tables_loaded[dev] = true;
  }
  *out = (uint8_t*)p;
  return PF_OK;
}

// The job record and the stage prefix table, written into the scratch array
// by one CTA from its kernel argument.
struct StaticRecord {
  FrameJob job;
  int base[ST_COUNT * 2];
};
static_assert(sizeof(FrameJob) % 4 == 0, "record is copied as 32-bit words");
static_assert(sizeof(StaticRecord) <= 4096, "record must fit the kernel parameter space");

__global__ void k_grain_static_record(StaticRecord r, uint8_t* scratch) {
  const uint32_t* job = (const uint32_t*)&r.job;
  uint32_t* dj = (uint32_t*)scratch;
  for (int i = threadIdx.x; i < (int)(sizeof(FrameJob) / 4); i += blockDim.x) dj[i] = job[i];
  int* db = (int*)(scratch + kBaseOff);
  for (int i = threadIdx.x; i < ST_COUNT * 2; i += blockDim.x) db[i] = r.base[i];
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
  StaticRecord R;
  memset(&R, 0, sizeof(R));
  FrameJob& J = R.job;
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
    build_scaling_lut(a.lut[0], fg->y_points, fg->num_y_points);
    if (fg->chroma_scaling_from_luma) {
      memcpy(a.lut[1], a.lut[0], 256);
      memcpy(a.lut[2], a.lut[0], 256);
    } else {
      build_scaling_lut(a.lut[1], fg->cb_points, fg->num_cb_points);
      build_scaling_lut(a.lut[2], fg->cr_points, fg->num_cr_points);
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
  for (int k = 0; k < ST_COUNT; k++) {
    R.base[2 * k] = 0;
    R.base[2 * k + 1] = counts[k];
  }
  const cudaStream_t s = (cudaStream_t)stream;
  k_grain_static_record<<<1, 128, 0, s>>>(R, scratch);
  if (cudaGetLastError() != cudaSuccess) return PF_ERR_DEVICE;
  BatchArgs b;
  b.jobs = (const FrameJob*)scratch;
  b.base = (const int*)(scratch + kBaseOff);
  b.n = 1;
  b.counters = nullptr;
  b.chunk = 1;
  b.ahead = 0;
  b.tile = 0;
  b.f0 = 0;
  b.f1 = 1;
  b.wave = 0;
  if (launch_fg_templates_batch(b, counts[ST_FG_TEMPLATES], counts[ST_FG_TEMPLATES], s) != cudaSuccess ||
      launch_fg_offsets_batch(b, counts[ST_FG_OFFSETS], counts[ST_FG_OFFSETS], s) != cudaSuccess ||
      launch_fg_apply_batch(b, counts[ST_FG_APPLY], counts[ST_FG_APPLY], s) != cudaSuccess)
    return PF_ERR_DEVICE;
  return PF_OK;
}
