/*
 * goav1pf.h - C ABI of the B200 AV1 post-reconstruction filter chain.
 *
 * This is the drop-in boundary for goav1's decoder post-filter runner and its
 * encoder CDEF strength search.  Every entry point takes plain pointers and
 * sizes; nothing here names a PyTorch or CUDA-runtime type, so cgo, ctypes or
 * any C caller can bind it directly.
 *
 * Reference interfaces each part replaces (paths inside thesyncim/goav1):
 *   - pf_frame_apply      internal/av1/decoder/work.go:151-155
 *                          (FrameWorkPostFilterRunner.Apply) as implemented by
 *                          decoderFrameWorkReusableSupportedPostFilterRunner,
 *                          decoder_postfilter_bind.go:398-440; its display
 *                          output replaces PostFilterOutput()
 *                          (decoder_postfilter_bind.go:252-256, :434-439).
 *   - pf_cdef_search      internal/av1/encoder/cdef_search.go:580-634
 *                          (cdefSearcher.search) + :886-945 (finish).
 *   - pf_cdef_apply       internal/av1/encoder/cdef_apply.go:202-371
 *                          (cdefApplier.markFromLoopFilterMap + apply).
 *   - pf_superres_upscale internal/av1/superres/superres.go:40-107 as called
 *                          from decoder/postfilter_superres.go:206-283;
 *     pf_frame_apply_superres  the runner's Apply for super-resolved frames
 *                          (decoder/postfilter.go:336-345 stage order).
 *   - pf_lr_search        internal/av1/encoder/restoration.go:149-263
 *                          (SearchWienerUnitU8, SearchSGRProjUnitU8) and the
 *                          unit loops of EncodeLoopRestorationKeyframe,
 *                          encoder/keyframe_lossy.go:2313-2383, :2422-2453.
 *   - pf_lf_build         internal/av1/threading/loop_filter_masks.go:450-551
 *                          (FrameWorkLoopFilterMasks.BuildFromMap) and
 *                          decoder/postfilter_loopfilter_masks.go:119-228
 *                          (populateLoopFilterLevelCacheFromMap), as the
 *                          encoder's mask-driven deblock calls them
 *                          (encoder/loopfilter_apply.go:576-589).
 *   - status codes        sentinel errors: cdef.ErrInvalidCDEF
 *                          (cdef/direction.go:11), loopfilter.ErrInvalidFilter,
 *                          tile.ErrInvalidPlan, decoder.ErrUnsupportedPostFilter,
 *                          frame.ErrShortBuffer.
 *
 * Side-information layouts are the reference's own decode-time products, so a
 * Go runner passes its slices through unchanged:
 *   - loop-filter edge masks: lfmask.FilterMask per 128x128 region
 *     (lfmask/mask.go:25-41): Y[2][32][3][2] then UV[2][32][2][2] uint16;
 *   - level cache: 4 bytes per 4x4 MI cell [YV, YH, U, V]
 *     (threading/loop_filter_masks.go:20-27, lfmask/build.go:25-32);
 *   - CDEF noskip words: 8 bytes per 64x64 unit, bit by*8+bx
 *     (threading/loop_filter_noskip.go:5-19);
 *   - CDEF index map: Index[] / Read[] per unit (threading/cdef_index.go:13-18).
 */
#ifndef GOAV1PF_H
#define GOAV1PF_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PF_ABI_VERSION 3

/* ---- status codes (negative = error; the frame is untouched on every error
 *      reported before any kernel was queued, mirroring the reference's
 *      validate-before-mutate rule, postfilter.go:596-613) ---- */
enum {
  PF_OK = 0,
  PF_ERR_INVALID_CDEF = -1,      /* cdef.ErrInvalidCDEF */
  PF_ERR_INVALID_FILTER = -2,    /* loopfilter.ErrInvalidFilter */
  PF_ERR_INVALID_PLAN = -3,      /* tile.ErrInvalidPlan (loop restoration) */
  PF_ERR_UNSUPPORTED = -4,       /* decoder.ErrUnsupportedPostFilter */
  PF_ERR_SHORT_BUFFER = -5,      /* frame.ErrShortBuffer */
  PF_ERR_INVALID_FORMAT = -6,    /* frame.ErrInvalidFormat (film grain) */
  PF_ERR_INVALID_ARG = -7,       /* null pointer, bad size or enum */
  PF_ERR_DEVICE = -8,            /* a CUDA call failed */
  PF_ERR_TIMEOUT = -9,           /* a bounded device wait ran out */
  PF_ERR_NO_DEVICE = -10,        /* no usable sm_100 device */
  PF_ERR_INVALID_BATCH = -11     /* threading.ErrInvalidBatch (block record map) */
};

/* ---- stage bits (FrameWorkPostFilterStage, postfilter.go:13-21) ---- */
enum {
  PF_STAGE_LOOP_FILTER = 1u << 0,
  PF_STAGE_CDEF = 1u << 1,
  PF_STAGE_LOOP_RESTORATION = 1u << 2,
  PF_STAGE_FILM_GRAIN = 1u << 3,
  /* Edge-replicate the planes into their allocated padding after loop
   * restoration (frame.Frame.ExtendBordersFrom, applied when the frame
   * refreshes a reference slot, postfilter.go:769-771). */
  PF_STAGE_EXTEND_BORDERS = 1u << 4
};

enum { PF_MEM_HOST = 0, PF_MEM_DEVICE = 1 };

/* Restoration types (parser.RestorationType, parser/restoration.go). */
enum {
  PF_LR_NONE = 0,
  PF_LR_SWITCHABLE = 1,
  PF_LR_WIENER = 2,
  PF_LR_SGRPROJ = 3
};

/* One plane of a frame.  data points at sample (0,0); 10/12-bit samples are
 * little-endian uint16 (frame/buffer.go, cdef/filter.go:366). */
typedef struct pf_plane {
  void* data;
  int64_t stride;        /* bytes between rows */
  int32_t width;         /* cropped (visible) width in samples */
  int32_t height;        /* cropped (visible) height */
  int32_t alloc_width;   /* allocated width in samples (>= 8-aligned width) */
  int32_t alloc_height;  /* allocated rows (>= 8-aligned height) */
} pf_plane;

/* A frame (frame.Frame, frame/buffer.go:128-141).  width/height are the
 * cropped luma size (FrameSize.CodedWidth x Height: the chain filters coded
 * frames; pf_superres_upscale resamples one to FrameSize.UpscaledWidth).
 * Chroma planes are ((width+ss_x)>>ss_x) x ((height+ss_y)>>ss_y). */
typedef struct pf_frame {
  int32_t width;
  int32_t height;
  uint8_t bit_depth;     /* 8, 10 or 12 */
  uint8_t ss_x;
  uint8_t ss_y;
  uint8_t mono;
  uint8_t memory;        /* PF_MEM_HOST or PF_MEM_DEVICE */
  uint8_t reserved[3];
  pf_plane plane[3];
} pf_frame;

/* lfmask.FilterMask: 384 uint16 of Y masks then 256 of UV masks. */
#define PF_LF_MASK_WORDS 640

typedef struct pf_loop_filter {
  uint8_t level_y[2];    /* LoopFilterParams.LevelY (vertical, horizontal) */
  uint8_t level_u;
  uint8_t level_v;
  uint8_t sharpness;
  uint8_t reserved[3];
  const uint16_t* masks; /* sb128_w*sb128_h*PF_LF_MASK_WORDS */
  int32_t sb128_w;
  int32_t sb128_h;
  const uint8_t* level_cache; /* 4*mi_cols*mi_rows */
  int32_t mi_cols;       /* ((width+7)>>3)<<1, the decoder's MI grid */
  int32_t mi_rows;       /* ((height+7)>>3)<<1 */
} pf_loop_filter;

typedef struct pf_cdef {
  uint8_t damping;       /* CDEFParams.Damping (3..6) */
  uint8_t bits;
  uint8_t strength_count;
  uint8_t reserved;
  uint8_t y_strength[8]; /* packed pri<<2 | sec code */
  uint8_t uv_strength[8];
  const uint8_t* index;  /* unit grid, row stride = index_stride */
  const uint8_t* read;   /* 0/1 per unit */
  int32_t index_stride;
  int32_t index_rows;
  const uint8_t* noskip; /* 8 bytes per unit, unit_cols*unit_rows, or NULL =
                            every block filtered */
} pf_cdef;

/* One decoded restoration unit (tile.RestorationUnit). */
typedef struct pf_lr_unit {
  uint8_t type;          /* PF_LR_NONE / PF_LR_WIENER / PF_LR_SGRPROJ */
  uint8_t sgr_set;       /* SGRProjInfo.ParamsIndex */
  int8_t sgr_xqd[2];     /* SGRProjInfo.XQD */
  int8_t wiener_v[3];    /* taps 0..2 of the vertical filter */
  int8_t wiener_h[3];    /* taps 0..2 of the horizontal filter */
} pf_lr_unit;

typedef struct pf_restoration {
  uint8_t type[3];       /* frame type per plane (PF_LR_*) */
  uint8_t reserved;
  uint16_t unit_size_y;
  uint16_t unit_size_uv;
  const pf_lr_unit* units[3]; /* horz*vert units per plane, raster order */
  int32_t unit_count[3];      /* entries available in units[p] */
} pf_restoration;

/* parser.FilmGrainParams (parser/film_grain.go:21-56). */
typedef struct pf_film_grain {
  uint8_t apply;
  uint8_t chroma_scaling_from_luma;
  uint16_t seed;
  uint8_t num_y_points;
  uint8_t y_points[14][2];
  uint8_t num_cb_points;
  uint8_t cb_points[10][2];
  uint8_t num_cr_points;
  uint8_t cr_points[10][2];
  uint8_t scaling_shift;
  uint8_t ar_coeff_lag;
  int8_t ar_coeffs_y[24];
  int8_t ar_coeffs_cb[25];
  int8_t ar_coeffs_cr[25];
  uint8_t ar_coeff_shift;
  uint8_t grain_scale_shift;
  uint8_t cb_mult;
  uint8_t cb_luma_mult;
  uint16_t cb_offset;
  uint8_t cr_mult;
  uint8_t cr_luma_mult;
  uint16_t cr_offset;
  uint8_t overlap;
  uint8_t clip_to_restricted_range;
  uint8_t matrix_identity; /* ColorConfig.MatrixCoefficients == identity */
  uint8_t reserved;
} pf_film_grain;

/* Everything the runner needs for one frame (FrameWorkPostFilterContext,
 * work.go:85-101, reduced to its post-filter inputs). */
typedef struct pf_frame_side {
  uint32_t stages;       /* PF_STAGE_* still to run */
  uint32_t side_memory;  /* PF_MEM_HOST: the side-info arrays below are host
                            memory (copied up each call); PF_MEM_DEVICE: they
                            are already device resident */
  pf_loop_filter lf;
  pf_cdef cdef;
  pf_restoration lr;
  pf_film_grain fg;
} pf_frame_side;

/* Per-call counters (FrameWorkCDEFPostFilterResult & co.). */
typedef struct pf_stats {
  uint32_t completed;    /* PF_STAGE_* bits run */
  uint32_t cdef_units;
  uint32_t lr_units;
  uint32_t fg_rows;
  float stage_ms[5];     /* device time per stage when timing is on */
} pf_stats;

typedef struct pf_config {
  int32_t device;        /* CUDA ordinal */
  int32_t timing;        /* 1 = record per-stage CUDA events */
  int64_t max_width;     /* largest luma frame the context will see (0 = grow) */
  int64_t max_height;
  int64_t wait_timeout_us; /* 0: a call that waits for its device work (pf_sync,
                              host-frame pf_frame_apply / pf_batch_apply, the
                              searches, pf_superres_upscale, pf_lf_build)
                              blocks until it is done; > 0: each such wait
                              polls and the call returns PF_ERR_TIMEOUT once
                              this many microseconds have passed in it.  The
                              queued work, copies into the caller's host
                              buffers included, still runs: call pf_sync
                              before reusing those buffers or reading the
                              call's outputs. */
} pf_config;

typedef struct pf_ctx pf_ctx;

/* Library identity. */
int pf_abi_version(void);
const char* pf_status_string(int status);
/* The failing CUDA call behind the last PF_ERR_DEVICE of this thread
 * (call, source line, CUDA error), or "" if none. */
const char* pf_status_detail(void);

/* Context life cycle.  One context per decoder; calls on one context are
 * serialised by the caller (the reference calls Apply once per frame on the
 * decoder goroutine).  pf_create returns NULL and writes *status on error. */
pf_ctx* pf_create(const pf_config* cfg, int* status);
void pf_destroy(pf_ctx* ctx);

/* Runs the stages named in side->stages on `frame` in place (deblock, CDEF,
 * loop restoration, border extension; the result is the publishable
 * reference frame) and, when PF_STAGE_FILM_GRAIN is set and grain applies,
 * writes the grained display picture into `display` (which must have the
 * same geometry and share no memory with `frame`: PF_ERR_INVALID_ARG).  Host frames are copied to the device and back inside the
 * call; device frames are filtered where they lie.  Returns when the work is
 * complete (host frames) or queued on the context's stream (device frames;
 * pf_sync waits for it). */
int pf_frame_apply(pf_ctx* ctx, const pf_frame* frame, const pf_frame_side* side,
                   const pf_frame* display, pf_stats* stats);

/* Validation alone: the status pf_frame_apply would return before touching
 * anything. */
int pf_frame_validate(const pf_frame* frame, const pf_frame_side* side,
                      const pf_frame* display);

int pf_sync(pf_ctx* ctx);

/* The CUDA stream the context queues on (cudaStream_t as void*), so a caller
 * that owns device frames can order its own work around the chain. */
void* pf_stream(pf_ctx* ctx);

/* ---- batched persistent queue: many frames, one launch per stage ---- */
typedef struct pf_batch_item {
  const pf_frame* frame;
  const pf_frame_side* side;
  const pf_frame* display;
} pf_batch_item;

/* Filters n frames of any size, bit depth and chroma format; equivalent to
 * n pf_frame_apply calls.  Device-resident frames: work units of all frames
 * share one launch per stage (see batch scheduling below); the call returns
 * once the work is queued (host side information: once it is done).
 * Host-resident frames (every frame and display of the batch in host
 * memory): the frames go through in chunks of 4, the upload of one chunk,
 * the filtering of the previous one and the download of the one before that
 * overlapping on three streams; the call returns when every frame and
 * display is back in host memory.  Page-locked host memory lets the copies
 * overlap; pageable memory works, with synchronous copies.  A batch mixing
 * host and device frames gets PF_ERR_INVALID_ARG. */
int pf_batch_apply(pf_ctx* ctx, const pf_batch_item* items, int32_t n, pf_stats* stats);

/* ---- batch scheduling (no counterpart in the reference) ----
 * pf_batch_apply queues one launch per stage for all frames of a batch; each
 * work item (a tile or unit of one plane of one frame) is found from per-stage
 * prefix counts.  Two knobs shape those launches:
 *   - CUDA graphs (pf_batch_graphs): the first batch of a given signature
 *     (frame count, each frame's work per stage, side-information bytes and
 *     the schedules) is captured as a graph and later batches of
 *     that signature replay it, with only their job tables refreshed.  Up to
 *     8 signatures are kept; a change of the context's scratch buffers
 *     recaptures.  Graphs are not used while the context times stages.
 *     The switch covers batches of device frames and single-frame calls
 *     (pf_frame_apply, a batch of one); host-frame batches pipeline their
 *     chunks without graphs.
 *   - The schedule of each stage group (pf_schedule, pf_set_schedule):
 *       ctas           persistent CTAs draining the stage's items through an
 *                      atomic counter (0 = one CTA per chunk);
 *       units_per_cta  consecutive work items (tiles / 64x64 units, in the
 *                      stage's numbering: along a row first) a CTA takes at
 *                      a time, 1..16, amortising per-item set-up;
 *       staging        0..3: with one item per CTA, the CTA first prefetches
 *                      into L2 the input rows of the item that many waves
 *                      on (a wave: the CTAs the device holds at once), which
 *                      a CTA starting about when this one ends will take;
 *                      with larger chunks, the item that many places on
 *                      inside the chunk (then below units_per_cta);
 *       tile           deblocking: the tile shape, 0 = 32x8, 1 = 64x4,
 *                      2 = 16x16, 3 = 8x32 edge units a tile (one thread
 *                      each); grain apply: rows of a column whose loads are
 *                      issued together, 0 = 1 (40 registers, 6 CTAs per SM),
 *                      1 = 2, 2 = 4 (64 registers, 4 CTAs per SM), 3 = four
 *                      columns by four rows a thread, 8-bit samples moved as
 *                      32-bit words (64 registers); 0 for the other groups.
 *     Work items are independent, so every schedule gives the same samples.
 * pf_autotune searches the schedule of each group on a given batch, one
 * dimension at a time (tile setting, units per CTA, staging depth, persistent
 * CTAs at 0, 1, 2, 4, 8 and 16 per SM), keeping after each the candidate
 * with the lowest median stage time over reps timed runs (one untimed run
 * first), then the frame-group count (1 or 2) by the whole batch's median
 * time, and leaves the winners set on the context.  It runs the batch in
 * place, so pass frames whose contents may be overwritten (copies).
 * out->ms_default is each group's time with the default schedule
 * {0, 1, 0, 0}. */
enum { PF_TUNE_DEBLOCK = 0, PF_TUNE_CDEF = 1, PF_TUNE_RESTORATION = 2, PF_TUNE_FILM_GRAIN = 3, PF_TUNE_GROUPS = 4 };

typedef struct pf_schedule {
  int32_t ctas;           /* persistent CTAs (0 = one CTA per chunk) */
  int32_t units_per_cta;  /* work items per chunk, 1..16 */
  int32_t staging;        /* prefetch distance 0..3 (< units_per_cta when > 1) */
  int32_t tile;           /* deblocking 0..3, grain apply 0..3, else 0 */
} pf_schedule;

typedef struct pf_tune_result {
  pf_schedule chosen[PF_TUNE_GROUPS];  /* the schedule left set per group */
  float ms[PF_TUNE_GROUPS];            /* its median stage time */
  float ms_default[PF_TUNE_GROUPS];    /* the default schedule's */
  int32_t frame_groups;                /* the frame-group count left set (1 or 2) */
  float ms_groups[2];                  /* median batch time with 1 and 2 groups */
} pf_tune_result;

int pf_batch_graphs(pf_ctx* ctx, int32_t enable);
/* Sets / reads one group's schedule (PF_ERR_INVALID_ARG outside the ranges
 * above).  pf_set_persistent(ctx, g, n) sets only the ctas field. */
int pf_set_schedule(pf_ctx* ctx, int32_t group, const pf_schedule* schedule);
int pf_get_schedule(const pf_ctx* ctx, int32_t group, pf_schedule* schedule);
int pf_set_persistent(pf_ctx* ctx, int32_t group, int32_t ctas);
/* Frame groups: 2 splits each batch where half of its restoration tiles lie
 * and runs the two halves' chains on two streams, so each half's launches
 * overlap the other's tails; 1 (the default) runs the batch as one group.
 * The output is the same either way.  With 2, a context that times stages
 * reports the whole batch as stage_ms[0] (the other stages 0). */
int pf_set_frame_groups(pf_ctx* ctx, int32_t groups);
int pf_autotune(pf_ctx* ctx, const pf_batch_item* items, int32_t n, int32_t reps,
                pf_tune_result* out);

/* ---- encoder CDEF strength search (cdef_search.go) ---- */
typedef struct pf_cdef_search_params {
  int32_t qindex;        /* frame base_q_idx */
  int32_t damping;       /* 0 = derive 3 + (qindex >> 6) */
  int32_t max_presets;   /* nb_strengths limit: 1, 2, 4 or 8 */
  double lambda;         /* RD lambda of svtRDCost */
} pf_cdef_search_params;

typedef struct pf_cdef_search_result {
  uint8_t bits;
  uint8_t strength_count;
  uint8_t y_strength[8];
  uint8_t uv_strength[8];
  uint8_t reserved[2];
  double cost;
} pf_cdef_search_result;

/* Exhaustive per-64x64 search: for every filter block and every one of the
 * 64 packed strengths, the SSE against `source` of the CDEF-filtered
 * `recon` (luma, and U+V summed for chroma) is written to mse_out
 * (uint64, [2][n_fb][64]); then the greedy preset selection picks the frame
 * presets and fb_index_out gets each unit's preset.  recon is the deblocked
 * frame; source and recon are both host or both device frames.  noskip is
 * as in pf_cdef, in host or device memory (it is copied), or NULL to search
 * every 8x8 block.  Entry i of the 64 trials is the packed strength of the
 * reference's level-1 list: 4*i for i < 16, then 4*(k/3) + k%3 + 1 for
 * k = i - 16.  Only 8-bit 4:2:0 frames are searched (goav1's
 * SourceFrame420); others get PF_ERR_UNSUPPORTED.  mse_out and fb_index_out
 * are host buffers (either may be NULL). */
int pf_cdef_search(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon,
                   const uint8_t* noskip, const pf_cdef_search_params* params,
                   uint64_t* mse_out, uint8_t* fb_index_out,
                   pf_cdef_search_result* result);

/* The search controls of one picture (goav1's svtCDEFSearchCtrls after
 * updateOnRefInfo, as cdefSearcher.search reads them,
 * internal/av1/encoder/cdef_search.go:581-596): trial i measures luma packed
 * strength y[i] and chroma packed strength uv[i] (-1: chroma not measured,
 * its SSE is the untested figure 1040400 * 64); luma rows are measured every
 * `subsampling`-th row (capped at 4) with the SSE scaled back by that factor;
 * uv_from_y makes each preset's chroma strength its luma strength. */
#define PF_CDEF_MAX_TRIALS 64
typedef struct pf_cdef_search_ctrls {
  int32_t count;                    /* trials, first pass then second: 1..64 */
  int8_t y[PF_CDEF_MAX_TRIALS];
  int8_t uv[PF_CDEF_MAX_TRIALS];
  int32_t subsampling;              /* subsamplingFactor: 1 or 4 */
  int32_t uv_from_y;
} pf_cdef_search_ctrls;

/* SSE-table entries at and beyond ctrls->count (not trials of the list). */
#define PF_CDEF_NOT_A_TRIAL 0x7fffffffu

/* The LAST reference's signalled strengths (svtCDEFRefStrengths,
 * cdef_search.go:224-235): count = 1 << cdef_bits. */
typedef struct pf_cdef_ref_strengths {
  uint8_t count;
  uint8_t y[8];
  uint8_t uv[8];
} pf_cdef_ref_strengths;

/* A picture's CDEF plan (svtCDEFFramePlan, encoder/cdef_frame.go:13-54). */
typedef struct pf_cdef_plan {
  int32_t on;              /* CDEF is on for the picture (cdef_level != 0) */
  int32_t search;          /* the strengths come from pf_cdef_search_ex(ctrls) */
  uint8_t y_strength;      /* on && !search (use_reference_cdef_fs): the one */
  uint8_t uv_strength;     /*   strength pair the picture signals (bits 0)    */
  uint8_t reserved[2];
  pf_cdef_search_ctrls ctrls;
} pf_cdef_plan;

/* The search level goav1's real-time encoder picks
 * (svtRTCCDEFSearchLevel, cdef_search.go:208-221): 5 on intra pictures,
 * otherwise 7 for screen content and 8 for camera content. */
int pf_cdef_search_level_rtc(int32_t islice, int32_t screen);

/* planSVTCDEF (encoder/cdef_frame.go:34-54) at search level 1-8: the level's
 * controls (setSVTCDEFSearchControls, cdef_search.go:72-202), then, on
 * inter pictures, the skip detector (CDEF off when more than 75 % of the
 * LAST reference was coded skip and the level uses it) or updateOnRefInfo
 * (cdef_search.go:237-272) with `ref`, which inter pictures at levels 5-8
 * need.  Level 0 gives a plan with CDEF off; level 9 (the QP-derived
 * strengths) is PF_ERR_UNSUPPORTED.  Host logic only: no device call. */
int pf_cdef_plan_picture(int32_t level, int32_t islice, int32_t is_base, int32_t not_highest_layer,
                         const pf_cdef_ref_strengths* ref, int32_t ref_skip_percent, pf_cdef_plan* plan);

/* pf_cdef_search over an explicit trial list (cdefSearcher.search with any
 * level's controls, cdef_search.go:581-634): mse_out entries
 * [plane][fb][i] for i < ctrls->count as pf_cdef_search describes (untested
 * chroma trials at 1040400 * 64; luma at the subsampled, rescaled SSE),
 * entries from ctrls->count on hold PF_CDEF_NOT_A_TRIAL; the greedy
 * selection runs over the list and result's strengths are ctrls->y of the
 * chosen trials (chroma too, as finish maps them, :937-940; luma's with
 * uv_from_y). */
int pf_cdef_search_ex(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                      const pf_cdef_search_params* params, const pf_cdef_search_ctrls* ctrls, uint64_t* mse_out,
                      uint8_t* fb_index_out, pf_cdef_search_result* result);

/* The encoder's CDEF application (cdefApplier.apply,
 * internal/av1/encoder/cdef_apply.go:258-371): filters `recon` in place with
 * the searched parameters, leaving it equal to the decoder's post-CDEF
 * output.  The per-unit index map is the one the decoder rebuilds while
 * parsing (markFromLoopFilterMap, :202-235): a 64x64 unit is filtered, with
 * fb_index[unit] (0 when fb_index is NULL, as for result->bits == 0), when
 * any of its in-frame 8x8 blocks has its noskip bit set; noskip NULL
 * filters every unit.  Damping is params->damping, or 3 + (qindex >> 6)
 * when 0 (cdef_frame.go:62).  A result whose strengths are all zero leaves
 * recon untouched (:262-271).  8-bit 4:2:0 frames only; recon is a host or
 * device frame, noskip and fb_index host or device memory.  Returns when
 * the frame is filtered. */
int pf_cdef_apply(pf_ctx* ctx, const pf_frame* recon, const uint8_t* noskip,
                  const pf_cdef_search_params* params, const pf_cdef_search_result* result,
                  const uint8_t* fb_index);

/* ---- super-resolution upscale (superres.UpscalePlaneCoded) ----
 * The normative horizontal upscaler the decoder runs between CDEF and loop
 * restoration on super-resolved frames (internal/av1/superres/superres.go:
 * 40-107, called from internal/av1/decoder/postfilter_superres.go:206-283).
 * For each plane, the coded frame's samples over the MI-aligned span
 * (((width + 7) & ~7) >> ss_x columns, so the columns past the crop are the
 * coded buffer's own samples) and the crop height are resampled to the
 * upscaled plane width with the 8-tap, 64-phase filter; the step and the
 * initial phase come from the cropped coded width.  coded->width is
 * FrameSize.CodedWidth, upscaled->width FrameSize.UpscaledWidth (greater);
 * both frames have the same height, bit depth and chroma layout and are both
 * host or both device frames.  The cropped upscaled planes are written.
 * Mismatched frames give PF_ERR_INVALID_FORMAT (frame.ErrInvalidFormat /
 * ErrInvalidPlane), planes too small for that geometry PF_ERR_SHORT_BUFFER. */
int pf_superres_upscale(pf_ctx* ctx, const pf_frame* coded, const pf_frame* upscaled);

/* pf_frame_apply for a super-resolved frame (FrameSize.SuperResEnabled): the
 * decoder's stage order with the upscale between CDEF and restoration
 * (internal/av1/decoder/postfilter.go:336-345, postfilter_superres.go).
 * Deblocking and CDEF run on `coded` in place (its width the coded width,
 * side->lf and side->cdef in its geometry); the restoration stripe-boundary
 * rows are the deblocked coded rows, upscaled
 * (tile/restoration_boundary.go:257-406); the CDEF output is upscaled into
 * `upscaled` (width FrameSize.UpscaledWidth); restoration (side->lr on the
 * upscaled grid), border extension and grain then run on `upscaled`, grain
 * into `display` (upscaled geometry).  All frames host or all device; the
 * same status codes as pf_frame_apply and pf_superres_upscale, returned
 * before anything is touched.  Returns when the frames are filtered. */
int pf_frame_apply_superres(pf_ctx* ctx, const pf_frame* coded, const pf_frame_side* side,
                            const pf_frame* upscaled, const pf_frame* display, pf_stats* stats);

/* A batch of super-resolved frames (pf_batch_apply for frames with
 * FrameSize.SuperResEnabled): the same result as pf_frame_apply_superres on
 * each item in turn.  Device frames: deblocking runs as one launch per pass
 * over every coded frame, then the boundary rows and CDEF, then the upscale
 * of each frame, then restoration, border extension and grain as one launch
 * per stage over every upscaled frame; the call returns once the work is
 * queued (host side information: once it is copied).  Host frames: one
 * pf_frame_apply_superres per item.  Every frame of the batch in host memory
 * or every one in device memory (else PF_ERR_INVALID_ARG); an item's
 * arguments are checked as pf_frame_apply_superres checks them, and the
 * first failing item's status is returned before anything is queued. */
typedef struct pf_superres_item {
  const pf_frame* coded;      /* coded-width frame, deblocked and CDEF-filtered in place */
  const pf_frame_side* side;  /* lf / cdef on the coded grid, lr on the upscaled grid */
  const pf_frame* up;         /* upscaled frame: restoration, extension, grain */
  const pf_frame* display;    /* grain output (upscaled geometry), or null */
} pf_superres_item;

int pf_batch_apply_superres(pf_ctx* ctx, const pf_superres_item* items, int32_t n, pf_stats* stats);

/* ---- deblocking masks and level cache from the block record map ----
 * The record map is threading.FrameWorkLoopFilterMap
 * (threading/loop_filter_map.go:46-72): one record per 4x4 MI cell, row-major
 * with stride mi_cols, each block's record repeated in every cell it covers
 * (its visible part).  pf_lf_build turns it into the two products
 * pf_frame_apply's deblocking reads (pf_loop_filter.masks and .level_cache):
 *   - the lfmask.FilterMask edge bitmasks of every 128x128 region, as
 *     BuildFromMap builds them: each block's left/above edge width class is
 *     the minimum of its own transform class and the neighbouring block's
 *     right/bottom transform class read from the map (2 luma, 1 chroma at the
 *     frame edge or next to an invalid cell); inner transform edges of intra
 *     and non-skip inter blocks; chroma edges from the block that carries the
 *     shared chroma (lfmask/build.go:60-100, :203-236, lfmask/mask.go);
 *   - the level cache, each block's four levels (ResolveBlockLevels,
 *     loopfilter/level.go:120-190) over its luma cells (bytes 0-1) and its
 *     chroma cells (bytes 2-3, chroma coordinates with the luma stride),
 *     blocks later in raster order of their origin overwriting earlier ones.
 * Both outputs are overwritten whole: masks
 * ceil(mi_cols/32)*ceil(mi_rows/32)*PF_LF_MASK_WORDS uint16, level_cache
 * 4*mi_cols*mi_rows bytes.  A map whose records partition the grid (as the
 * decoder writes it) gives the reference's output bit for bit. */
typedef struct pf_lf_record {      /* threading.FrameWorkLoopFilterBlockRecord */
  uint16_t mi_col;                 /* Block.MICol, MIRow: the block's origin cell */
  uint16_t mi_row;
  uint16_t mi_col_end;             /* Block.MIColEnd, MIRowEnd (exclusive, clamped to the grid) */
  uint16_t mi_row_end;
  uint8_t block_size;              /* tile.BlockSize: 0 = 128x128 ... 21 = 4x4 */
  uint8_t valid;
  uint8_t intra;
  uint8_t skip;                    /* SkipTransform */
  uint8_t tx_y;                    /* TransformTree.Y (tile.TransformSize: 0 = 4x4 ... 18 = 64x16) */
  uint8_t tx_uv;                   /* TransformTree.UV */
  uint8_t has_uv;                  /* TransformTree.HasUV */
  uint8_t segment_id;
  uint8_t ref_frame;               /* 0 intra, 1..7 LAST..ALTREF */
  uint8_t mode;                    /* loopfilter.ModeDeltaClass: 0 GLOBALMV, 1 other inter modes */
  int8_t delta_lf_from_base;       /* DeltaLFFromBase */
  int8_t delta_lf[4];              /* DeltaLF (delta_lf_multi: YV, YH, U, V) */
  uint8_t reserved0;
  uint16_t tx_split[2];            /* TransformTree.Split: var-tx split bits, depth 0 and 1 */
  uint32_t reserved1;
} pf_lf_record;                    /* 32 bytes */

typedef struct pf_lf_levels {      /* loopfilter.PrepareLevelResolver inputs (level.go:86-118) */
  uint8_t level_y[2];              /* LoopFilterParams.LevelY */
  uint8_t level_u;
  uint8_t level_v;
  uint8_t delta_lf_present;        /* DeltaParams.DeltaLFPresent */
  uint8_t delta_lf_multi;          /* DeltaParams.DeltaLFMulti */
  uint8_t segmentation_enabled;    /* SegmentationParams.Enabled */
  uint8_t mode_ref_delta_enabled;  /* LoopFilterParams.ModeRefDeltaEnabled */
  int8_t ref_delta[8];             /* Deltas.Ref */
  int8_t mode_delta[2];            /* Deltas.Mode */
  uint8_t reserved[2];
  int16_t segment_delta[8][4];     /* per segment DeltaLFYV, DeltaLFYH, DeltaLFU, DeltaLFV */
} pf_lf_levels;

/* Builds the masks and level cache on the GPU.  records: mi_cols*mi_rows
 * records in records_memory (PF_MEM_HOST: copied up in the call); masks and
 * level_cache: both in out_memory.  ss_x/ss_y/mono: the sequence's chroma
 * layout (lfmask.Layout; no chroma edges or chroma levels when mono).
 * Returns when the outputs are written.  Errors, as the reference's walk
 * meets them in raster order of the level-cache population:
 *   - PF_ERR_INVALID_BATCH: a visited record's MIColEnd is not past its cell
 *     or past the grid, or its block size (or transform size, which the
 *     reference indexes without a check) is out of range;
 *   - PF_ERR_INVALID_FILTER: ref_frame > 7 or mode > 1, or segment_id > 7
 *     with segmentation on (ResolveBlockLevels);
 *   - PF_ERR_INVALID_ARG: null pointers, odd or zero mi_cols/mi_rows (the
 *     decoder's MI grid is always even), mi_cols or mi_rows above 16384, a
 *     bad memory kind or layout.
 * On an error the outputs are unspecified (the reference leaves them
 * partly written). */
int pf_lf_build(pf_ctx* ctx, const pf_lf_record* records, int32_t mi_cols, int32_t mi_rows,
                uint32_t records_memory, const pf_lf_levels* levels, int32_t ss_x, int32_t ss_y, int32_t mono,
                uint16_t* masks, uint8_t* level_cache, uint32_t out_memory);

/* ---- film grain with no allocation ----
 * No counterpart in the reference; this entry point exists for callers that
 * cannot call cudaMalloc: a presentation thread adding grain right before
 * display, which must not stall on an allocation that can synchronise the
 * device, or an application whose device memory is already owned by another
 * allocator.  It writes display = ref with film grain applied, exactly as
 * pf_frame_apply with only PF_STAGE_FILM_GRAIN does, but allocates nothing:
 * its scratch (grain templates, block offsets, the job record) is one
 * file-scope device array of PF_GRAIN_STATIC_SCRATCH_BYTES that every GPU
 * loading the library holds until the process exits.
 *   - ref and display are device frames (PF_MEM_DEVICE) of equal geometry on
 *     the current CUDA device; fg is the frame's grain parameters.
 *   - Frames with more than PF_GRAIN_STATIC_MAX_BLOCKS 32x32 luma blocks
 *     (ceil(width/32) * ceil(height/32), e.g. 8192x8192) are rejected with
 *     PF_ERR_SHORT_BUFFER before anything is queued.
 *   - The first call on a device sets up that device: it loads the grain
 *     tables into constant memory and waits for the device to finish
 *     (cudaDeviceSynchronize), so make that first call before any stream
 *     capture.  Every call looks up the array's device address (host code
 *     cannot use the symbol as an address).  The tables live in the library's
 *     module, so after cudaDeviceReset this entry point must not be called
 *     again on that device.
 *   - The job record reaches the array as a kernel argument: nothing the
 *     call reads from host memory is needed after it returns.
 *   - Work is queued on `stream` (a cudaStream_t, or NULL for the legacy
 *     default stream); the call returns without waiting for it.
 *   - Every call shares the one array and it keeps the last call's contents;
 *     calls whose work overlaps on the GPU race, so order them (one stream).
 */
#define PF_GRAIN_STATIC_SCRATCH_BYTES 131072
#define PF_GRAIN_STATIC_MAX_BLOCKS 65536
int pf_film_grain_static(const pf_frame* ref, const pf_film_grain* fg, const pf_frame* display, void* stream);

/* ---- learned CDEF strength selection ----
 * No counterpart in the reference.  A small network predicts, per 64x64
 * filter block, which of the 64 level-1 trials (the pf_cdef_search order)
 * is best for luma and for chroma, from 40 statistics of the deblocked
 * reconstruction.  pf_cdef_search_learned then measures only the predicted
 * trials of a confident head, all 64 trials of a head whose top-1
 * probability is below the threshold, and runs the same greedy preset
 * selection and RD choice as pf_cdef_search over that table; the bitstream
 * syntax (CDEFParams and the per-block index) is unchanged.
 *
 * Network: 40 features -> 64 ReLU -> 64 ReLU -> 64 luma + 64 chroma logits,
 * two softmax heads.  Weights are bf16 (bit patterns in uint16_t, row-major
 * [out][in]), biases and arithmetic fp32 (fused multiply-add over the inputs
 * in index order).  Features are normalised as (x - feat_shift) * feat_scale
 * before the first layer. */
#define PF_MLP_FEATURES 40
#define PF_MLP_HIDDEN 64
#define PF_MLP_CLASSES 64
#define PF_MLP_OUTPUTS (2 * PF_MLP_CLASSES)
#define PF_MLP_PARAMS                                                            \
  (PF_MLP_HIDDEN * PF_MLP_FEATURES + PF_MLP_HIDDEN * PF_MLP_HIDDEN +             \
   PF_MLP_OUTPUTS * PF_MLP_HIDDEN + 2 * PF_MLP_HIDDEN + PF_MLP_OUTPUTS)

typedef struct pf_cdef_mlp {
  uint16_t w1[PF_MLP_HIDDEN * PF_MLP_FEATURES];
  uint16_t w2[PF_MLP_HIDDEN * PF_MLP_HIDDEN];
  uint16_t w3[PF_MLP_OUTPUTS * PF_MLP_HIDDEN]; /* rows 0..63 luma, 64..127 chroma */
  float b1[PF_MLP_HIDDEN];
  float b2[PF_MLP_HIDDEN];
  float b3[PF_MLP_OUTPUTS];
  float feat_shift[PF_MLP_FEATURES];
  float feat_scale[PF_MLP_FEATURES];
} pf_cdef_mlp;

/* Gradients of the mean loss with respect to every parameter, fp32, in the
 * order w1, w2, w3, b1, b2, b3 (PF_MLP_PARAMS floats). */
typedef struct pf_cdef_mlp_grads {
  float w1[PF_MLP_HIDDEN * PF_MLP_FEATURES];
  float w2[PF_MLP_HIDDEN * PF_MLP_HIDDEN];
  float w3[PF_MLP_OUTPUTS * PF_MLP_HIDDEN];
  float b1[PF_MLP_HIDDEN];
  float b2[PF_MLP_HIDDEN];
  float b3[PF_MLP_OUTPUTS];
} pf_cdef_mlp_grads;

typedef struct pf_cdef_mlp_train_params {
  int32_t epochs;
  int32_t batch;        /* samples per Adam step (a multiple of 32) */
  float lr;             /* Adam step size */
  float beta1, beta2, eps;
  float weight_decay;   /* decoupled, on the weights only */
  uint32_t seed;        /* shuffling */
} pf_cdef_mlp_train_params;

typedef struct pf_cdef_learned_stats {
  int32_t blocks;           /* non-skip filter blocks */
  int32_t fallback_luma;    /* blocks whose luma head measured all 64 trials */
  int32_t fallback_chroma;  /* blocks whose chroma head measured all 64 trials */
  int32_t trials_luma;      /* luma trials measured, all blocks */
  int32_t trials_chroma;    /* chroma trials measured, all blocks */
  float stage_ms[4];        /* device time of features, network, trial search,
                               selection when the context times stages, else -1 */
} pf_cdef_learned_stats;

/* Per-filter-block features of an 8-bit 4:2:0 deblocked reconstruction
 * (host or device frame; noskip as in pf_cdef_search).  features is a host
 * buffer of n_fb * PF_MLP_FEATURES floats, n_fb = ceil(w/64) * ceil(h/64);
 * a block with no searched 8x8 block gets zeros in its first 33 features. */
int pf_cdef_features(pf_ctx* ctx, const pf_frame* recon, const uint8_t* noskip,
                     int32_t qindex, int32_t damping, float* features);

/* Forward pass over n host feature rows; probs (host, n * PF_MLP_OUTPUTS)
 * receives the two softmax heads. */
int pf_cdef_mlp_forward(pf_ctx* ctx, const pf_cdef_mlp* model, const float* features,
                        int32_t n, float* probs);

/* Mean cross-entropy of both heads over n samples (labels: n pairs of luma,
 * chroma trial indices) and its gradients, computed by the training
 * kernels in one batch. */
int pf_cdef_mlp_gradients(pf_ctx* ctx, const pf_cdef_mlp* model, const float* features,
                          const uint8_t* labels, int32_t n, float* loss,
                          pf_cdef_mlp_grads* grads);

/* Adam training on the GPU from `model` (updated in place: bf16 weights are
 * the rounded fp32 master weights).  epoch_loss (host, epochs floats, may be
 * NULL) receives each epoch's mean loss. */
int pf_cdef_mlp_train(pf_ctx* ctx, pf_cdef_mlp* model, const float* features,
                      const uint8_t* labels, int32_t n, const pf_cdef_mlp_train_params* params,
                      float* epoch_loss);

/* The learned search: arguments and outputs as pf_cdef_search, plus the
 * network, the confidence threshold (a head falls back to all 64 trials
 * when its top-1 probability is below it; above 1 every head falls back)
 * and the number of top trials measured by a confident head (1..8).
 * Unmeasured entries of mse_out hold 66585600 (the reference's
 * untested-trial figure).  The preset selection is the reference's greedy
 * over that table; without PF_LEARNED_REFINE in flags it stops after the nb
 * greedy picks (no 4*nb refinement passes: 8 sequential steps instead of 40
 * for 8 presets; on the evaluation frames the refinement changed no
 * frame's luma SSE by more than 0.001 %). */
#define PF_LEARNED_REFINE 1
int pf_cdef_search_learned(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon,
                           const uint8_t* noskip, const pf_cdef_search_params* params,
                           const pf_cdef_mlp* model, float threshold, int32_t candidates,
                           int32_t flags, uint64_t* mse_out, uint8_t* fb_index_out,
                           pf_cdef_search_result* result, pf_cdef_learned_stats* stats);

/* ---- encoder loop-restoration unit search (encoder/restoration.go) ----
 * Replaces the per-unit loop of EncodeLoopRestorationKeyframe
 * (internal/av1/encoder/keyframe_lossy.go:2313-2383, the bordered copy and
 * the search, and
 * :2422-2453, the application): luma restoration units of 64 samples
 * (tile.RestorationPlaneGrid, tile/restoration_geometry.go:54-92: the last
 * unit of a row or column takes the remainder, interior unit edges move up
 * by 8 rows), each searched with
 *   - SearchWienerUnitU8 (encoder/restoration.go:149-210): SSE of the
 *     unfiltered recon, then the 6 fixed symmetric tap sets of
 *     PF_LR_WIENER_CANDIDATES, scored by a horizontal-only 7-tap pass with
 *     (sum + 64) >> 7 and edge-clamped columns; a set is taken when its SSE
 *     + w*h is below the best so far;
 *   - the exact Wiener filter (restoration/wiener_u8.go:36-56, both
 *     directions the picked taps) on the 3-sample edge-clamped frame, whose
 *     SSE becomes the unit's best;
 *   - SearchSGRProjUnitU8 (encoder/restoration.go:216-263): the exact
 *     self-guided filter (restoration/selfguided_u8.go:36) for each preset
 *     of PF_LR_SGR_PRESETS under the same acceptance rule; SGRProj replaces
 *     Wiener when its SSE is strictly lower.
 * Units wider or taller than 64 stay PF_LR_NONE (the reference's filters
 * reject them).  Only 8-bit 4:2:0 frames are searched (SourceFrame420);
 * only luma is read or written.
 * source, recon and restored (may be NULL) are all host or all device
 * frames of equal geometry; restored may be recon itself.  When restored is
 * given, its luma plane receives the reconstruction with every unit's
 * decision applied (unfiltered samples for PF_LR_NONE units); its chroma
 * planes are not touched.  units (host, may be NULL) receives one record
 * per unit in raster order; max_units must cover horz*vert units, where
 * horz = max((width + 32) / 64, 1) and vert = max((height + 32) / 64, 1). */
#define PF_LR_WIENER_CANDIDATES 6
#define PF_LR_SGR_PRESETS 4
typedef struct pf_lr_search_unit {
  int32_t x0, y0, x1, y1;   /* unit rectangle on the luma plane */
  uint64_t base_sse;        /* unfiltered recon against source */
  uint64_t sse;             /* SSE of the unit as decided (base_sse for NONE) */
  uint64_t wiener_sse;      /* exact Wiener SSE of the search's pick; UINT64_MAX
                               when the Wiener search took no set or the unit
                               is larger than 64x64 */
  uint64_t sgr_sse;         /* SearchSGRProjUnitU8's best SSE (base_sse when
                               no preset was taken; UINT64_MAX when the unit
                               is larger than 64x64) */
  int8_t wiener_candidate;  /* index of the picked Wiener set, -1 = none */
  int8_t sgr_preset;        /* index of the picked SGR preset, -1 = none */
  uint8_t reserved[2];
  pf_lr_unit unit;          /* the decision, as the bitstream codes it */
} pf_lr_search_unit;
int pf_lr_search(pf_ctx* ctx, const pf_frame* source, const pf_frame* recon, const pf_frame* restored,
                 pf_lr_search_unit* units, int32_t max_units);

/* ---- measurement ----
 * No counterpart in the reference.  The warp-instruction issue rate of the
 * current device, measured by a fixed inline-PTX instruction stream over every
 * SM (kind 0: integer logic ops only, the ALU pipe; kind 1: 32-bit integer
 * multiply-adds only; kind 2: the two interleaved; kind 3: FP32 fused
 * multiply-adds, a pipe that takes an instruction every cycle, so its rate
 * is the issue ceiling).  The post-filter kernels are bound by instruction
 * issue, not by DRAM bytes, so their roofline is reported against this
 * ceiling as well as against copy bandwidth.  Synchronous; allocates and
 * frees a small buffer.  *ms receives the fastest launch's time. */
int pf_diag_issue_rate(int32_t kind, double* warp_inst_per_s, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* GOAV1PF_H */
