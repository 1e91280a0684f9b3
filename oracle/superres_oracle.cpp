// superres_oracle.cpp - CPU oracle of the AV1 super-resolution upscale (test
// infrastructure: only tests/ use it).
//
// A scalar restatement of internal/av1/superres/superres.go:40-107
// (UpscalePlaneCoded, upscaleRowPureGo) and of the per-plane geometry the
// decoder hands it (internal/av1/decoder/postfilter_superres.go:244-272: the
// MI-aligned source span, the cropped coded width for the phase math, the
// crop height).  Pinned by the reference's known-answer rows
// (superres_test.go:10-47 and the libaom-captured row of
// superres_aligned_libaom_test.go:17-51, in tests/golden/kats.json).
#include <stdint.h>

#include "pf_oracle.h"
#include "pf_tables.h"

namespace {

int clampi(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

}  // namespace

// One row: src holds src_width samples, coded_width of them cropped.
extern "C" void oracle_superres_row(const uint16_t* src, int src_width, int coded_width, uint16_t* dst,
                                    int dst_width, int bit_depth) {
  const int scaleBits = 14, extraBits = 8;
  const int step = ((coded_width << scaleBits) + dst_width / 2) / dst_width;
  const int err = dst_width * step - (coded_width << scaleBits);
  int x0 = ((-((dst_width - coded_width) << (scaleBits - 1))) + dst_width / 2) / dst_width;
  x0 += (1 << (extraBits - 1)) - err / 2;
  x0 &= (1 << scaleBits) - 1;
  const int maxv = (1 << bit_depth) - 1, last = src_width - 1;
  for (int x = 0; x < dst_width; x++) {
    const int srcX = -(1 << scaleBits) + x0 + x * step;
    const int px = srcX >> scaleBits;
    const int16_t* f = pf_superres_filter[(srcX & ((1 << scaleBits) - 1)) >> extraBits];
    int sum = 0;
    for (int k = 0; k < 8; k++) sum += (int)src[clampi(px - 3 + k, 0, last)] * f[k];
    dst[x] = (uint16_t)clampi((sum + 64) >> 7, 0, maxv);
  }
}

// Every plane of a host frame (the layout pf_superres_upscale takes).
extern "C" int oracle_superres_upscale(const pf_frame* coded, const pf_frame* up) {
  const int bps = coded->bit_depth > 8 ? 2 : 1;
  const int nplanes = coded->mono ? 1 : 3;
  for (int p = 0; p < nplanes; p++) {
    const int sx = p ? coded->ss_x : 0, sy = p ? coded->ss_y : 0;
    const int cw = (coded->width + sx) >> sx, aw = ((coded->width + 7) & ~7) >> sx;
    const int dw = (up->width + sx) >> sx, rows = (coded->height + sy) >> sy;
    uint16_t src[8192], dst[16384];
    if (aw > 8192 || dw > 16384) return PF_ERR_INVALID_ARG;
    for (int y = 0; y < rows; y++) {
      const uint8_t* sr = (const uint8_t*)coded->plane[p].data + (int64_t)y * coded->plane[p].stride;
      uint8_t* dr = (uint8_t*)up->plane[p].data + (int64_t)y * up->plane[p].stride;
      for (int x = 0; x < aw; x++) src[x] = bps == 1 ? sr[x] : ((const uint16_t*)sr)[x];
      oracle_superres_row(src, aw, cw, dst, dw, coded->bit_depth);
      for (int x = 0; x < dw; x++) {
        if (bps == 1)
          dr[x] = (uint8_t)dst[x];
        else
          ((uint16_t*)dr)[x] = dst[x];
      }
    }
  }
  return PF_OK;
}
