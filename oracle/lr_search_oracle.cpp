// lr_search_oracle.cpp - CPU oracle of the encoder's loop-restoration unit
// search (test infrastructure: only tests/ and bench.py's CPU leg use it).
//
// A scalar restatement of internal/av1/encoder/restoration.go:149-210
// (SearchWienerUnitU8), :216-263 (SearchSGRProjUnitU8) and of the unit loops
// of EncodeLoopRestorationKeyframe (internal/av1/encoder/keyframe_lossy.go:
// 2310-2330 bordered copy, :2332-2383 search, :2422-2453 application), over
// the unit grid of tile/restoration_geometry.go:54-92.  The exact filters are
// the oracle's own restatements of restoration/wiener.go and
// restoration/selfguided.go (oracle_wiener, oracle_sgr), which the U8
// entry points restoration/wiener_u8.go:36 and selfguided_u8.go:36 equal at
// 8 bits by their contracts.
//
// Parity pinning: the reference's only test of this path
// (encoder_public_test.go:1867-1893) is an encode/decode round trip; its
// filters are pinned through the oracle's known-answer tests, and the search
// logic is checked here against a direct Python restatement on small frames.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "pf_oracle.h"

namespace {

const int16_t kWienerSets[PF_LR_WIENER_CANDIDATES][3] = {{0, -3, 12}, {0, -5, 18}, {0, -2, 8},
                                                         {0, 2, 10},  {1, 4, 14},  {0, -1, 4}};
const int kSgrPresets[PF_LR_SGR_PRESETS][3] = {{0, 8, 24}, {2, 16, 40}, {10, 0, 48}, {14, 24, 72}};

inline int clampi(int v, int lo, int hi) { return v < lo ? lo : v > hi ? hi : v; }

// restoration/wiener.go:44-47.
void new_wiener_filter(const int16_t* t, int16_t* f) {
  f[0] = f[6] = t[0];
  f[1] = f[5] = t[1];
  f[2] = f[4] = t[2];
  f[3] = (int16_t)(-2 * (t[0] + t[1] + t[2]));
}

struct Plane8 {
  const uint8_t* p;
  int64_t stride;
  uint8_t at(int x, int y) const { return p[(int64_t)y * stride + x]; }
};

// SearchWienerUnitU8 (encoder/restoration.go:149-210).
int search_wiener_unit(const Plane8& src, const Plane8& rec, int W, int H, int x0, int y0, int w, int h,
                       uint64_t* base_out) {
  uint64_t base = 0;
  for (int y = y0; y < y0 + h; y++)
    for (int x = x0; x < x0 + w; x++) {
      const int d = (int)src.at(x, y) - (int)rec.at(x, y);
      base += (uint64_t)(d * d);
    }
  *base_out = base;
  if (w <= 0 || h <= 0 || x0 + w > W || y0 + h > H || base == 0) return -1;
  uint64_t best = base;
  int pick = -1;
  for (int c = 0; c < PF_LR_WIENER_CANDIDATES; c++) {
    int16_t f[7];
    new_wiener_filter(kWienerSets[c], f);
    uint64_t sse = 0;
    for (int y = y0; y < y0 + h; y++)
      for (int x = x0; x < x0 + w; x++) {
        int hs = 0;
        for (int k = -3; k <= 3; k++) hs += f[k + 3] * (int)rec.at(clampi(x + k, 0, W - 1), y);
        const int pred = clampi((hs + 64) >> 7, 0, 255);
        const int d = (int)src.at(x, y) - pred;
        sse += (uint64_t)(d * d);
      }
    if (sse + (uint64_t)(w * h) < best) {
      best = sse;
      pick = c;
    }
  }
  return pick;
}

uint64_t block_sse(const Plane8& src, int x0, int y0, const uint16_t* out, int w, int h) {
  uint64_t sse = 0;
  for (int y = 0; y < h; y++)
    for (int x = 0; x < w; x++) {
      const int d = (int)src.at(x0 + x, y0 + y) - (int)out[y * w + x];
      sse += (uint64_t)(d * d);
    }
  return sse;
}

}  // namespace

extern "C" int oracle_lr_search(const pf_frame* source, const pf_frame* recon, const pf_frame* restored,
                                pf_lr_search_unit* units, int max_units) {
  if (!source || !recon || recon->bit_depth != 8 || source->bit_depth != 8) return PF_ERR_UNSUPPORTED;
  const int W = recon->width, H = recon->height;
  const int horz = W + 32 >= 64 ? (W + 32) / 64 : 1, vert = H + 32 >= 64 ? (H + 32) / 64 : 1;
  const int n = horz * vert;
  if (units && max_units < n) return PF_ERR_SHORT_BUFFER;
  const Plane8 src{(const uint8_t*)source->plane[0].data, source->plane[0].stride};
  const Plane8 rec{(const uint8_t*)recon->plane[0].data, recon->plane[0].stride};
  // keyframe_lossy.go:2310-2330: the 3-sample edge-clamped bordered recon.
  const int pad = 3, bs = W + 2 * pad;
  std::vector<uint16_t> bord((size_t)bs * (H + 2 * pad));
  for (int y = 0; y < H + 2 * pad; y++)
    for (int x = 0; x < bs; x++) bord[(size_t)y * bs + x] = rec.at(clampi(x - pad, 0, W - 1), clampi(y - pad, 0, H - 1));
  std::vector<pf_lr_search_unit> rec_units(n);
  std::vector<uint16_t> out(64 * 64);
  for (int i = 0; i < n; i++) {
    const int col = i % horz, row = i / horz;
    // tile/restoration_geometry.go:54-92.
    int x0 = col * 64, x1 = col + 1 == horz ? W : x0 + 64;
    int y0 = row * 64, y1 = row + 1 == vert ? H : y0 + 64;
    if (y0 > 0) y0 -= 8;
    if (y1 < H) y1 -= 8;
    const int w = x1 - x0, h = y1 - y0;
    const bool fits = w <= 64 && h <= 64;  // validRestorationBlock / validSGRBlock
    pf_lr_search_unit& r = rec_units[i];
    memset(&r, 0, sizeof(r));
    r.x0 = x0;
    r.y0 = y0;
    r.x1 = x1;
    r.y1 = y1;
    const uint16_t* origin = &bord[(size_t)(y0 + pad) * bs + x0 + pad];
    uint64_t base = 0;
    const int wpick = search_wiener_unit(src, rec, W, H, x0, y0, w, h, &base);
    r.base_sse = base;
    r.wiener_candidate = (int8_t)wpick;
    uint64_t best = ~0ull;
    int type = PF_LR_NONE;
    r.wiener_sse = ~0ull;
    if (wpick >= 0 && fits) {
      int16_t f[7];
      new_wiener_filter(kWienerSets[wpick], f);
      oracle_wiener(origin, bs, out.data(), w, w, h, f, f, 8);
      best = block_sse(src, x0, y0, out.data(), w, h);
      r.wiener_sse = best;
      type = PF_LR_WIENER;
    }
    // SearchSGRProjUnitU8 (encoder/restoration.go:216-263).
    int spick = -1;
    r.sgr_sse = ~0ull;
    if (fits) {
      uint64_t sbest = base;
      if (base != 0)
        for (int p = 0; p < PF_LR_SGR_PRESETS; p++) {
          const int8_t xqd[2] = {(int8_t)kSgrPresets[p][1], (int8_t)kSgrPresets[p][2]};
          oracle_sgr(origin, bs, out.data(), w, w, h, kSgrPresets[p][0], xqd, 8);
          const uint64_t sse = block_sse(src, x0, y0, out.data(), w, h);
          if (sse + (uint64_t)(w * h) < sbest) {
            sbest = sse;
            spick = p;
          }
        }
      r.sgr_sse = sbest;
      if (spick >= 0 && sbest < best) {
        best = sbest;
        type = PF_LR_SGRPROJ;
      }
    }
    r.sgr_preset = (int8_t)spick;
    r.sse = type == PF_LR_NONE ? base : best;
    r.unit.type = (uint8_t)type;
    if (type == PF_LR_WIENER)
      for (int k = 0; k < 3; k++) r.unit.wiener_v[k] = r.unit.wiener_h[k] = (int8_t)kWienerSets[wpick][k];
    if (type == PF_LR_SGRPROJ) {
      r.unit.sgr_set = (uint8_t)kSgrPresets[spick][0];
      r.unit.sgr_xqd[0] = (int8_t)kSgrPresets[spick][1];
      r.unit.sgr_xqd[1] = (int8_t)kSgrPresets[spick][2];
    }
  }
  // keyframe_lossy.go:2422-2453: every decided unit filtered from the
  // bordered copy into the output plane; NONE units keep the recon.
  if (restored) {
    uint8_t* dst = (uint8_t*)restored->plane[0].data;
    const int64_t ds = restored->plane[0].stride;
    for (int y = 0; y < H; y++) memmove(dst + (int64_t)y * ds, rec.p + (int64_t)y * rec.stride, W);
    for (int i = 0; i < n; i++) {
      const pf_lr_search_unit& r = rec_units[i];
      const int w = r.x1 - r.x0, h = r.y1 - r.y0;
      const uint16_t* origin = &bord[(size_t)(r.y0 + pad) * bs + r.x0 + pad];
      if (r.unit.type == PF_LR_WIENER) {
        int16_t f[7];
        new_wiener_filter(kWienerSets[r.wiener_candidate], f);
        oracle_wiener(origin, bs, out.data(), w, w, h, f, f, 8);
      } else if (r.unit.type == PF_LR_SGRPROJ) {
        oracle_sgr(origin, bs, out.data(), w, w, h, r.unit.sgr_set, r.unit.sgr_xqd, 8);
      } else {
        continue;
      }
      for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) dst[(int64_t)(r.y0 + y) * ds + r.x0 + x] = (uint8_t)out[y * w + x];
    }
  }
  if (units) memcpy(units, rec_units.data(), sizeof(pf_lr_search_unit) * n);
  return PF_OK;
}
