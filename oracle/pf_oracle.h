/*
 * pf_oracle.h - CPU oracle for the AV1 post-filter chain (test infrastructure).
 *
 * A plain, scalar C++ restatement of goav1's canonical Go paths, used only as
 * the checker in tests/ and as the CPU-baseline leg of bench.py.  Nothing in
 * the product (goav1_b200/) links or calls it.  Each function cites the
 * reference file:line it follows (paths inside thesyncim/goav1).
 *
 * Parity pinning: the reference is pure Go and no Go toolchain exists here,
 * so the reference cannot be run.  The oracle is pinned by the literal
 * known-answer tests of goav1's own test files (LFSR draws, Gaussian table
 * checksums, scaling-LUT points, CDEF direction patterns, the filter14 row-7
 * case, SGR tables, Wiener taps) and by the libaom restatements those tests
 * use as second oracles; see tests/test_oracle_kat.py.
 */
#ifndef PF_ORACLE_H
#define PF_ORACLE_H

#include "goav1pf.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Whole chain on a host frame, in place; display written when FG applies.
 * Returns a PF_* status. */
int oracle_frame_apply(const pf_frame* frame, const pf_frame_side* side,
                       const pf_frame* display);

/* Single-stage entry points (same semantics, one stage). */
int oracle_loop_filter(const pf_frame* frame, const pf_frame_side* side);
int oracle_cdef(const pf_frame* frame, const pf_frame_side* side);

/* ---- kernel-level entry points for known-answer tests ---- */
/* cdef/direction.go:37-79, :432-467.  img: 8x8 uint16, row stride. */
int oracle_cdef_find_dir(const uint16_t* img, int stride, int coeff_shift, int32_t* variance);
/* cdef/filter.go:79-169.  in: CDEF input buffer with origin at in_origin and
 * stride 144; writes w*h samples to dst (stride w). */
void oracle_cdef_filter_block(uint16_t* dst, const uint16_t* in, int in_origin,
                              int pri, int sec, int dir, int pri_damping,
                              int sec_damping, int coeff_shift, int w, int h);
/* cdef/filter.go:603-612 */
int oracle_cdef_adjust_strength(int strength, int32_t variance);
/* loopfilter/sb.go:348-446 on a line of 16 samples (q0 at index 8). */
void oracle_lpf_line(uint16_t* line16, int bit_depth, int level, int sharpness, int wd);
/* restoration/selfguided.go's x/(x+1) table entry (z clamped to 0..255). */
int oracle_sgr_x_by_xplus1(int z);
/* loopfilter/threshold.go:18-47: E (block limit), I (limit), H (hev). */
void oracle_lf_thresholds(int level, int sharpness, int* E, int* I, int* H);
/* The same with explicit 8-bit-scale thresholds E, I, H; wd 4, 6, 8 or 16. */
void oracle_lpf_line_thr(uint16_t* line16, int bit_depth, int E, int I, int H, int wd);
/* cdef/filter.go:614-633 on one direction. */
int oracle_cdef_chroma_dir(int dir, int xdec, int ydec);
/* filmgrain/apply.go:72-343 on one plane (uint16 samples) with a given
 * template (73x82, stride 82) and scaling table. */
int oracle_fg_apply_plane(const uint16_t* src, uint16_t* dst, int stride, const uint16_t* luma, int luma_stride,
                          int frame_w, int frame_h, const int16_t* grain, const uint8_t* lut,
                          const pf_film_grain* fg, int plane, int bit_depth, int ss_x, int ss_y);
/* filmgrain/random.go */
uint16_t oracle_lfsr_next(uint16_t* reg, int bits);
uint16_t oracle_stripe_seed(uint16_t seed, int luma_line);
/* filmgrain/scaling.go:18-48 */
int oracle_scaling_lut(uint8_t* dst256, const uint8_t* points, int n);
int oracle_scale_lut(const uint8_t* lut, int index, int bit_depth);
/* filmgrain/luma.go:24-82, chroma.go:29-91 */
int oracle_luma_grain(int16_t* dst /*73*82*/, const pf_film_grain* fg, int bit_depth);
int oracle_chroma_grain(int16_t* dst /*73*82*/, const int16_t* luma, const pf_film_grain* fg,
                        int plane, int bit_depth, int ss_x, int ss_y);
int16_t oracle_gaussian(int index);
/* restoration/selfguided.go:111-127 */
void oracle_sgr_decode_xq(const int8_t* xqd, int set, int16_t* xq);
/* restoration/wiener.go:59-80 on a (w+6)x(h+6) window (stride sstride,
 * origin at the window's (3,3)). */
void oracle_wiener(const uint16_t* src, int sstride, uint16_t* dst, int dstride,
                   int w, int h, const int16_t* vfilter7, const int16_t* hfilter7,
                   int bit_depth);
/* restoration/selfguided.go:132-210 */
void oracle_sgr(const uint16_t* src, int sstride, uint16_t* dst, int dstride,
                int w, int h, int set, const int8_t* xqd, int bit_depth);

/* Encoder CDEF search (encoder/cdef_search.go); see pf_cdef_search. */
int oracle_cdef_search(const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                       const pf_cdef_search_params* params, uint64_t* mse_out,
                       uint8_t* fb_index_out, pf_cdef_search_result* result);

/* finish() alone (encoder/cdef_search.go:886-945) over a given SSE table
 * ([2][nfb][64]; skip[fb] != 0 leaves a block out). */
int oracle_cdef_select(const uint64_t* mse, const uint8_t* skip, int nfb, const pf_cdef_search_params* params,
                       uint8_t* fb_index_out, pf_cdef_search_result* result);
/* The same with the refinement passes switched by `refine` (0: stop after
 * the nb greedy picks, as the learned search does by default). */
int oracle_cdef_select_ex(const uint64_t* mse, const uint8_t* skip, int nfb, const pf_cdef_search_params* params,
                          int refine, uint8_t* fb_index_out, pf_cdef_search_result* result);

/* The same over an explicit trial list (pf_cdef_search_ex), its selection,
 * and the picture plan (pf_cdef_plan_picture). */
int oracle_cdef_search_ex(const pf_frame* source, const pf_frame* recon, const uint8_t* noskip,
                          const pf_cdef_search_params* params, const pf_cdef_search_ctrls* ctrls, uint64_t* mse_out,
                          uint8_t* fb_index_out, pf_cdef_search_result* result);
int oracle_cdef_select_ctrls(const uint64_t* mse, const uint8_t* skip, int nfb, const pf_cdef_search_params* params,
                             const pf_cdef_search_ctrls* ctrls, int refine, uint8_t* fb_index_out,
                             pf_cdef_search_result* result);
int oracle_cdef_plan_picture(int level, int islice, int is_base, int not_highest_layer,
                             const pf_cdef_ref_strengths* ref, int ref_skip_percent, pf_cdef_plan* plan);

/* Learned CDEF selection (oracle/learned_oracle.cpp); see pf_cdef_features
 * and the pf_cdef_mlp_* entry points.  grads: PF_MLP_PARAMS floats. */
int oracle_cdef_features(const pf_frame* recon, const uint8_t* noskip, int qindex, int damping, float* X);
void oracle_mlp_forward(const pf_cdef_mlp* m, const float* X, int n, float* probs);
void oracle_mlp_gradients(const pf_cdef_mlp* m, const float* X, const uint8_t* labels, int n, float* loss,
                          float* grads);
void oracle_mlp_loss_grad_f64(const double* params, const double* shift, const double* scale, const float* X,
                              const uint8_t* labels, int n, double* loss, double* grads);

/* Encoder loop-restoration unit search and application
 * (oracle/lr_search_oracle.cpp); see pf_lr_search.  Host frames. */
int oracle_lr_search(const pf_frame* source, const pf_frame* recon, const pf_frame* restored,
                     pf_lr_search_unit* units, int max_units);

/* Super-resolution upscale (oracle/superres_oracle.cpp): one row, and every
 * plane of a host frame as pf_superres_upscale takes it. */
void oracle_superres_row(const uint16_t* src, int src_width, int coded_width, uint16_t* dst, int dst_width,
                         int bit_depth);
int oracle_superres_upscale(const pf_frame* coded, const pf_frame* upscaled);
/* The chain on a super-resolved frame (see pf_frame_apply_superres). */
int oracle_frame_apply_superres(const pf_frame* coded, const pf_frame_side* side, const pf_frame* upscaled,
                                const pf_frame* display);

/* Deblocking masks and level cache from the block record map
 * (oracle/lfmask_oracle.cpp). */
int oracle_lf_build(const pf_lf_record* rec, int cols, int rows, const pf_lf_levels* lv, int ssx, int ssy, int mono,
                    uint16_t* masks, uint8_t* level_cache);
int oracle_lf_build_ordered(const pf_lf_record* rec, int cols, int rows, const int32_t* order, int n, int sb_log2,
                            int ssx, int ssy, int mono, uint16_t* masks);
void oracle_lf_mask_block(int kind, uint16_t* region, int by4, int bx4, int w4, int h4, int skip, int tx,
                          const uint16_t split[2], uint8_t* a, uint8_t* l, int ssx, int ssy);
int oracle_lf_block_levels(const pf_lf_levels* p, int mono, const pf_lf_record* r, uint8_t out[4]);

/* ---- the second oracle (oracle/second_oracle.c) ----
 * Independent restatements of the filter arithmetic: goav1's in-test libaom
 * restatements and the AV1 specification's formulation. */
int so_lf_filter(int width, int* samples, int bit_depth, int limit, int blimit, int hev);
void so_cdef_filter_block(uint16_t* dst, int dst_stride, int dst_origin, const uint16_t* input, int input_origin,
                          int pri, int sec, int dir, int pri_damping, int sec_damping, int coeff_shift, int width,
                          int height);
int so_cdef_find_dir(const uint16_t* img, int stride, int coeff_shift, int32_t* variance);
int so_cdef_adjust_strength(int strength, int32_t variance);
int so_cdef_chroma_dir(int dir, int xdec, int ydec);
void so_wiener(const uint16_t* src, int stride, int origin, uint16_t* dst, int dst_stride, int w, int h,
               const int16_t* vf7, const int16_t* hf7, int bit_depth);
void so_sgr_params(int set, int* r0, int* s0, int* r1, int* s1);
void so_sgr_decode_xq(const int8_t* xqd, int set, int* xq0, int* xq1);
int so_sgr_x_by_xplus1(int z);
int so_sgr_one_by_n(int n);
void so_sgr(const uint16_t* src, int stride, int origin, uint16_t* dst, int dst_stride, int w, int h, int set,
            const int8_t* xqd, int bit_depth);
void so_grain_templates(int16_t* luma, int16_t* cb, int16_t* cr, const pf_film_grain* fg, int bit_depth, int ss_x,
                        int ss_y);
void so_scaling_lut(uint8_t* lut, const uint8_t (*points)[2], int n);
void so_grain_apply_plane(const uint16_t* src, uint16_t* dst, int stride, const uint16_t* luma, int luma_stride,
                          int frame_w, int frame_h, const int16_t* grain, const uint8_t* lut, const pf_film_grain* fg,
                          int plane, int bit_depth, int ss_x, int ss_y);

#ifdef __cplusplus
}
#endif

#endif
