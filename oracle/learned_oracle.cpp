// learned_oracle.cpp - CPU oracle of the learned CDEF strength selection
// (test infrastructure: only tests/ and bench.py's CPU leg use it).
//
// The learned selection has no counterpart in goav1, so this file restates
// the repository's own definitions, not a reference function:
//   oracle_cdef_features      the 40 per-filter-block features.  The CDEF
//                             direction costs follow cdef/direction.go:37-79
//                             and :432-501 over the blocks computeCDEFList
//                             (encoder/cdef_search.go:410-447) selects; the
//                             rest are integer pixel statistics.
//   oracle_mlp_forward        the network (bf16 weights widened to fp32,
//                             fused multiply-adds over the inputs in index
//                             order, ReLU, two softmax heads summed in the
//                             GPU warp's butterfly order).
//   oracle_mlp_gradients      mean two-head cross-entropy and its gradients,
//                             accumulated in the GPU kernels' order (tiles of
//                             32 samples, fused multiply-adds), so fp32
//                             results agree up to the exp/log rounding.
//   oracle_mlp_loss_grad_f64  the same mathematics in double on unrounded
//                             parameters, for finite-difference checks.
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "pf_oracle.h"

namespace {

constexpr int kF = PF_MLP_FEATURES, kH = PF_MLP_HIDDEN, kC = PF_MLP_CLASSES, kO = PF_MLP_OUTPUTS;
constexpr int kNW1 = kH * kF, kNW2 = kH * kH, kNW3 = kO * kH, kNW = kNW1 + kNW2 + kNW3;
constexpr int kNP = PF_MLP_PARAMS;
constexpr int kTile = 32;

inline const uint8_t* px(const pf_plane& p, int y, int x) { return (const uint8_t*)p.data + (int64_t)y * p.stride + x; }

int32_t dir_cost(const pf_plane& Y, int y0, int x0, int d) {
  int32_t p[15] = {0};
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      const int32_t x = (int32_t)*px(Y, y0 + i, x0 + j) - 128;
      int k;
      switch (d) {
        case 0: k = i + j; break;
        case 1: k = i + (j >> 1); break;
        case 2: k = i; break;
        case 3: k = 3 + i - (j >> 1); break;
        case 4: k = 7 + i - j; break;
        case 5: k = 3 - (i >> 1) + j; break;
        case 6: k = j; break;
        default: k = (i >> 1) + j; break;
      }
      p[k] += x;
    }
  int32_t s = 0;
  if (d == 2 || d == 6) {
    for (int i = 0; i < 8; i++) s += p[i] * p[i];
    return s * 105;
  }
  if (d == 0 || d == 4) {
    static const int32_t div[8] = {840, 420, 280, 210, 168, 140, 120, 105};
    for (int i = 0; i < 7; i++) s += (p[i] * p[i] + p[14 - i] * p[14 - i]) * div[i];
    return s + p[7] * p[7] * 105;
  }
  return (p[3] * p[3] + p[4] * p[4] + p[5] * p[5] + p[6] * p[6] + p[7] * p[7]) * 105 +
         (p[0] * p[0] + p[10] * p[10]) * 420 + (p[1] * p[1] + p[9] * p[9]) * 210 + (p[2] * p[2] + p[8] * p[8]) * 140;
}

int lap3(const pf_plane& P, int y, int x) {
  const int L = *px(P, y - 1, x - 1) - 2 * *px(P, y - 1, x) + *px(P, y - 1, x + 1) - 2 * *px(P, y, x - 1) +
                4 * *px(P, y, x) - 2 * *px(P, y, x + 1) + *px(P, y + 1, x - 1) - 2 * *px(P, y + 1, x) +
                *px(P, y + 1, x + 1);
  return abs(L);
}

float bf16f(uint16_t b) {
  uint32_t u = (uint32_t)b << 16;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

}  // namespace

extern "C" int oracle_cdef_features(const pf_frame* rec, const uint8_t* noskip, int qindex, int damping,
                                    float* X) {
  if (rec->bit_depth != 8 || rec->ss_x != 1 || rec->ss_y != 1) return PF_ERR_UNSUPPORTED;
  const int dmp = damping ? damping : 3 + (qindex >> 6);
  const int W = rec->width, H = rec->height;
  const int miCols = ((W + 7) >> 3) << 1, miRows = ((H + 7) >> 3) << 1;
  const int nhfb = (miCols + 15) / 16, nvfb = (miRows + 15) / 16, nfb = nhfb * nvfb;
  const pf_plane& Y = rec->plane[0];
  for (int fb = 0; fb < nfb; fb++) {
    float* out = X + (size_t)fb * kF;
    const int fbr = fb / nhfb, fbc = fb % nhfb;
    const int lr = 16 * fbr, lc = 16 * fbc;
    uint64_t word = ~0ull, listed = 0;
    if (noskip) {
      word = 0;
      for (int i = 0; i < 8; i++) word |= (uint64_t)noskip[(size_t)fb * 8 + i] << (8 * i);
    }
    for (int r = 0; r < std::min(miRows - lr, 16); r += 2)
      for (int c = 0; c < std::min(miCols - lc, 16); c += 2) listed |= word & (1ull << ((r >> 1) * 8 + (c >> 1)));
    if (!listed) {
      for (int i = 0; i < 33; i++) out[i] = 0.f;
      continue;
    }
    const int x0 = lc * 4, y0 = lr * 4;
    const int wc = std::min(64, W - x0), hc = std::min(64, H - y0);
    unsigned long long dcost[8] = {0}, dhist[8] = {0}, varsum = 0, nvar0 = 0, adjsum = 0, bvar = 0;
    for (int b = 0; b < 64; b++) {
      if (!((listed >> b) & 1)) continue;
      const int by = y0 + (b >> 3) * 8, bx = x0 + (b & 7) * 8;
      int32_t c[8];
      for (int d = 0; d < 8; d++) c[d] = dir_cost(Y, by, bx, d);
      int best = 0;
      for (int d = 1; d < 8; d++)
        if (c[d] > c[best]) best = d;
      const int32_t var = (c[best] - c[(best + 4) & 7]) >> 10;
      for (int d = 0; d < 8; d++) dcost[d] += (unsigned long long)c[d];
      dhist[best]++;
      varsum += (unsigned long long)var;
      if (var == 0) {
        nvar0++;
      } else {
        const int32_t v = var >> 6;
        int ai = 0;
        if (v) {
          ai = 31 - __builtin_clz((unsigned)v);
          if (ai > 12) ai = 12;
        }
        adjsum += (unsigned long long)(4 + ai);
      }
      long long s = 0, q = 0;
      for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) {
          const int x = *px(Y, by + i, bx + j);
          s += x;
          q += x * x;
        }
      bvar += (unsigned long long)(64 * q - s * s);
    }
    unsigned long long gH = 0, cH = 0, gV = 0, cV = 0, bH = 0, cbH = 0, bV = 0, cbV = 0, lap = 0, clap = 0, sy = 0;
    for (int i = 0; i < hc; i++)
      for (int j = 0; j < wc; j++) {
        const int x = *px(Y, y0 + i, x0 + j);
        sy += x;
        if (j + 1 < wc) {
          const unsigned d = abs(*px(Y, y0 + i, x0 + j + 1) - x);
          gH += d;
          cH++;
          if (((x0 + j + 1) & 7) == 0) {
            bH += d;
            cbH++;
          }
        }
        if (i + 1 < hc) {
          const unsigned d = abs(*px(Y, y0 + i + 1, x0 + j) - x);
          gV += d;
          cV++;
          if (((y0 + i + 1) & 7) == 0) {
            bV += d;
            cbV++;
          }
        }
        if (i >= 1 && i + 1 < hc && j >= 1 && j + 1 < wc) {
          lap += (unsigned)lap3(Y, y0 + i, x0 + j);
          clap++;
        }
      }
    const int x0c = x0 >> 1, y0c = y0 >> 1;
    const int wcc = std::min(32, rec->plane[1].width - x0c), hcc = std::min(32, rec->plane[1].height - y0c);
    unsigned long long cvar[2] = {0, 0}, cl = 0, ccl = 0, cg = 0, ccg = 0;
    for (int pl = 1; pl < 3; pl++) {
      const pf_plane& P = rec->plane[pl];
      for (int b = 0; b < 64; b++) {
        if (!((listed >> b) & 1)) continue;
        int s = 0, q = 0;
        for (int i = 0; i < 4; i++)
          for (int j = 0; j < 4; j++) {
            const int x = *px(P, y0c + (b >> 3) * 4 + i, x0c + (b & 7) * 4 + j);
            s += x;
            q += x * x;
          }
        cvar[pl - 1] += (unsigned long long)(16 * q - s * s);
      }
      for (int i = 0; i < hcc; i++)
        for (int j = 0; j < wcc; j++) {
          const int x = *px(P, y0c + i, x0c + j);
          if (j + 1 < wcc) {
            cg += (unsigned)abs(*px(P, y0c + i, x0c + j + 1) - x);
            ccg++;
          }
          if (i + 1 < hcc) {
            cg += (unsigned)abs(*px(P, y0c + i + 1, x0c + j) - x);
            ccg++;
          }
          if (i >= 1 && i + 1 < hcc && j >= 1 && j + 1 < wcc) {
            cl += (unsigned)lap3(P, y0c + i, x0c + j);
            ccl++;
          }
        }
    }
    const float nb = (float)__builtin_popcountll(listed);
    unsigned long long ds = 0;
    for (int d = 0; d < 8; d++) ds += dcost[d];
    auto cnt = [](unsigned long long c) { return (float)(c ? c : 1ull); };
    for (int d = 0; d < 8; d++) out[d] = ds ? (float)dcost[d] / (float)ds : 0.125f;
    for (int d = 0; d < 8; d++) out[8 + d] = (float)dhist[d] / nb;
    out[16] = log2f(1.f + (float)varsum / nb);
    out[17] = (float)nvar0 / nb;
    out[18] = (float)adjsum / (16.f * nb);
    out[19] = log2f(1.f + (float)bvar / (4096.f * nb));
    out[20] = log2f(1.f + (float)gH / cnt(cH));
    out[21] = log2f(1.f + (float)gV / cnt(cV));
    out[22] = log2f(1.f + (float)lap / cnt(clap));
    out[23] = ((float)bH / cnt(cbH) - (float)(gH - bH) / cnt(cH - cbH)) / 8.f;
    out[24] = ((float)bV / cnt(cbV) - (float)(gV - bV) / cnt(cV - cbV)) / 8.f;
    out[25] = log2f(1.f + (float)cvar[0] / (256.f * nb));
    out[26] = log2f(1.f + (float)cvar[1] / (256.f * nb));
    out[27] = log2f(1.f + (float)cl / cnt(ccl));
    out[28] = log2f(1.f + (float)cg / cnt(ccg));
    out[29] = nb / 64.f;
    out[30] = (float)qindex / 255.f;
    out[31] = (float)(dmp - 3) / 3.f;
    out[32] = (float)sy / (255.f * (float)(wc * hc));
  }
  // Frame means of features 16, 19, 22, 23, 24, 25, 27 over searched blocks.
  static const int ff[7] = {16, 19, 22, 23, 24, 25, 27};
  double sum[7] = {0, 0, 0, 0, 0, 0, 0};
  int c = 0;
  for (int fb = 0; fb < nfb; fb++) {
    const float* f = X + (size_t)fb * kF;
    if (f[29] > 0.f) {
      c++;
      for (int i = 0; i < 7; i++) sum[i] += (double)f[ff[i]];
    }
  }
  for (int fb = 0; fb < nfb; fb++)
    for (int i = 0; i < 7; i++) X[(size_t)fb * kF + 33 + i] = c ? (float)(sum[i] / (double)c) : 0.f;
  return PF_OK;
}

namespace {

// Widened parameters in the flat order w1, w2, w3, b1, b2, b3.
std::vector<float> widen(const pf_cdef_mlp* m) {
  std::vector<float> p(kNP);
  for (int i = 0; i < kNW1; i++) p[i] = bf16f(m->w1[i]);
  for (int i = 0; i < kNW2; i++) p[kNW1 + i] = bf16f(m->w2[i]);
  for (int i = 0; i < kNW3; i++) p[kNW1 + kNW2 + i] = bf16f(m->w3[i]);
  for (int i = 0; i < kH; i++) p[kNW + i] = m->b1[i];
  for (int i = 0; i < kH; i++) p[kNW + kH + i] = m->b2[i];
  for (int i = 0; i < kO; i++) p[kNW + 2 * kH + i] = m->b3[i];
  return p;
}

struct Act {
  float x[kF], h1[kH], h2[kH], z[kO], p[kO], loss;
};

void forward(const float* P, const float* shift, const float* scale, const float* xin, Act& A, const uint8_t* y) {
  const float* w1 = P;
  const float* w2 = P + kNW1;
  const float* w3 = P + kNW1 + kNW2;
  const float* b1 = P + kNW;
  const float* b2 = b1 + kH;
  const float* b3 = b2 + kH;
  for (int k = 0; k < kF; k++) A.x[k] = (xin[k] - shift[k]) * scale[k];
  for (int o = 0; o < kH; o++) {
    float acc = b1[o];
    for (int k = 0; k < kF; k++) acc = fmaf(w1[o * kF + k], A.x[k], acc);
    A.h1[o] = acc > 0.f ? acc : 0.f;
  }
  for (int o = 0; o < kH; o++) {
    float acc = b2[o];
    for (int k = 0; k < kH; k++) acc = fmaf(w2[o * kH + k], A.h1[k], acc);
    A.h2[o] = acc > 0.f ? acc : 0.f;
  }
  for (int o = 0; o < kO; o++) {
    float acc = b3[o];
    for (int k = 0; k < kH; k++) acc = fmaf(w3[o * kH + k], A.h2[k], acc);
    A.z[o] = acc;
  }
  A.loss = 0.f;
  float l[2] = {0.f, 0.f};
  for (int hd = 0; hd < 2; hd++) {
    const float* z = A.z + hd * kC;
    float m = z[0];
    for (int o = 1; o < kC; o++) m = fmaxf(m, z[o]);
    // The GPU's warp order: e[l] + e[l+32] per lane, then xor butterflies.
    float e[kC], v[32], nv[32];
    for (int o = 0; o < kC; o++) e[o] = expf(z[o] - m);
    for (int i = 0; i < 32; i++) v[i] = e[i] + e[i + 32];
    for (int d = 16; d > 0; d >>= 1) {
      for (int i = 0; i < 32; i++) nv[i] = v[i] + v[i ^ d];
      memcpy(v, nv, sizeof(v));
    }
    const float sum = v[0];
    if (y) l[hd] = m + logf(sum) - z[y[hd]];
    const float inv = 1.f / sum;
    for (int o = 0; o < kC; o++) A.p[hd * kC + o] = e[o] * inv;
  }
  if (y) A.loss = l[0] + l[1];
}

}  // namespace

extern "C" void oracle_mlp_forward(const pf_cdef_mlp* m, const float* X, int n, float* probs) {
  const std::vector<float> P = widen(m);
  Act A;
  for (int i = 0; i < n; i++) {
    forward(P.data(), m->feat_shift, m->feat_scale, X + (size_t)i * kF, A, nullptr);
    memcpy(probs + (size_t)i * kO, A.p, sizeof(A.p));
  }
}

extern "C" void oracle_mlp_gradients(const pf_cdef_mlp* m, const float* X, const uint8_t* labels, int n,
                                     float* loss, float* grads) {
  const std::vector<float> P = widen(m);
  const float* w2 = P.data() + kNW1;
  const float* w3 = P.data() + kNW1 + kNW2;
  const float invB = 1.f / (float)n;
  const int tiles = (n + kTile - 1) / kTile;
  std::vector<float> G((size_t)tiles * kNP), L(tiles);
  std::vector<Act> A(kTile);
  std::vector<float> dz((size_t)kTile * kO), dh2((size_t)kTile * kH), dh1((size_t)kTile * kH);
  for (int t = 0; t < tiles; t++) {
    const int count = std::min(kTile, n - t * kTile);
    for (int s = 0; s < count; s++) {
      const int r = t * kTile + s;
      forward(P.data(), m->feat_shift, m->feat_scale, X + (size_t)r * kF, A[s], labels + 2 * (size_t)r);
      for (int o = 0; o < kO; o++) {
        const int hd = o >> 6, c = o & 63;
        dz[s * kO + o] = (A[s].p[o] - (c == labels[2 * (size_t)r + hd] ? 1.f : 0.f)) * invB;
      }
    }
    float* g = G.data() + (size_t)t * kNP;
    float* gw1 = g;
    float* gw2 = g + kNW1;
    float* gw3 = g + kNW1 + kNW2;
    float* gb1 = g + kNW;
    float* gb2 = gb1 + kH;
    float* gb3 = gb2 + kH;
    for (int o = 0; o < kO; o++)
      for (int k = 0; k < kH; k++) {
        float acc = 0.f;
        for (int s = 0; s < count; s++) acc = fmaf(dz[s * kO + o], A[s].h2[k], acc);
        gw3[o * kH + k] = acc;
      }
    for (int o = 0; o < kO; o++) {
      float acc = 0.f;
      for (int s = 0; s < count; s++) acc += dz[s * kO + o];
      gb3[o] = acc;
    }
    for (int s = 0; s < count; s++)
      for (int k = 0; k < kH; k++) {
        float acc = 0.f;
        if (A[s].h2[k] > 0.f)
          for (int o = 0; o < kO; o++) acc = fmaf(w3[o * kH + k], dz[s * kO + o], acc);
        dh2[s * kH + k] = acc;
      }
    for (int o = 0; o < kH; o++)
      for (int k = 0; k < kH; k++) {
        float acc = 0.f;
        for (int s = 0; s < count; s++) acc = fmaf(dh2[s * kH + o], A[s].h1[k], acc);
        gw2[o * kH + k] = acc;
      }
    for (int o = 0; o < kH; o++) {
      float acc = 0.f;
      for (int s = 0; s < count; s++) acc += dh2[s * kH + o];
      gb2[o] = acc;
    }
    for (int s = 0; s < count; s++)
      for (int k = 0; k < kH; k++) {
        float acc = 0.f;
        if (A[s].h1[k] > 0.f)
          for (int o = 0; o < kH; o++) acc = fmaf(w2[o * kH + k], dh2[s * kH + o], acc);
        dh1[s * kH + k] = acc;
      }
    for (int o = 0; o < kH; o++)
      for (int k = 0; k < kF; k++) {
        float acc = 0.f;
        for (int s = 0; s < count; s++) acc = fmaf(dh1[s * kH + o], A[s].x[k], acc);
        gw1[o * kF + k] = acc;
      }
    for (int o = 0; o < kH; o++) {
      float acc = 0.f;
      for (int s = 0; s < count; s++) acc += dh1[s * kH + o];
      gb1[o] = acc;
    }
    float acc = 0.f;
    for (int s = 0; s < count; s++) acc += A[s].loss;
    L[t] = acc;
  }
  float lsum = 0.f;
  for (int t = 0; t < tiles; t++) lsum += L[t];
  *loss = lsum * invB;
  for (int p = 0; p < kNP; p++) {
    float acc = 0.f;
    for (int t = 0; t < tiles; t++) acc += G[(size_t)t * kNP + p];
    grads[p] = acc;
  }
}

extern "C" void oracle_mlp_loss_grad_f64(const double* P, const double* shift, const double* scale, const float* X,
                                         const uint8_t* labels, int n, double* loss, double* grads) {
  const double* w1 = P;
  const double* w2 = P + kNW1;
  const double* w3 = P + kNW1 + kNW2;
  const double* b1 = P + kNW;
  const double* b2 = b1 + kH;
  const double* b3 = b2 + kH;
  double* gw1 = grads;
  double* gw2 = grads + kNW1;
  double* gw3 = grads + kNW1 + kNW2;
  double* gb1 = grads + kNW;
  double* gb2 = gb1 + kH;
  double* gb3 = gb2 + kH;
  memset(grads, 0, sizeof(double) * kNP);
  double L = 0;
  for (int i = 0; i < n; i++) {
    double x[kF], h1[kH], h2[kH], z[kO], dz[kO], d2[kH], d1[kH];
    for (int k = 0; k < kF; k++) x[k] = ((double)X[(size_t)i * kF + k] - shift[k]) * scale[k];
    for (int o = 0; o < kH; o++) {
      double a = b1[o];
      for (int k = 0; k < kF; k++) a += w1[o * kF + k] * x[k];
      h1[o] = a > 0 ? a : 0;
    }
    for (int o = 0; o < kH; o++) {
      double a = b2[o];
      for (int k = 0; k < kH; k++) a += w2[o * kH + k] * h1[k];
      h2[o] = a > 0 ? a : 0;
    }
    for (int o = 0; o < kO; o++) {
      double a = b3[o];
      for (int k = 0; k < kH; k++) a += w3[o * kH + k] * h2[k];
      z[o] = a;
    }
    for (int hd = 0; hd < 2; hd++) {
      const double* zz = z + hd * kC;
      double m = zz[0];
      for (int o = 1; o < kC; o++) m = zz[o] > m ? zz[o] : m;
      double s = 0;
      for (int o = 0; o < kC; o++) s += exp(zz[o] - m);
      const int y = labels[2 * (size_t)i + hd];
      L += m + log(s) - zz[y];
      for (int o = 0; o < kC; o++) dz[hd * kC + o] = (exp(zz[o] - m) / s - (o == y ? 1.0 : 0.0)) / n;
    }
    for (int o = 0; o < kO; o++) {
      gb3[o] += dz[o];
      for (int k = 0; k < kH; k++) gw3[o * kH + k] += dz[o] * h2[k];
    }
    for (int k = 0; k < kH; k++) {
      double a = 0;
      for (int o = 0; o < kO; o++) a += w3[o * kH + k] * dz[o];
      d2[k] = h2[k] > 0 ? a : 0;
    }
    for (int o = 0; o < kH; o++) {
      gb2[o] += d2[o];
      for (int k = 0; k < kH; k++) gw2[o * kH + k] += d2[o] * h1[k];
    }
    for (int k = 0; k < kH; k++) {
      double a = 0;
      for (int o = 0; o < kH; o++) a += w2[o * kH + k] * d2[o];
      d1[k] = h1[k] > 0 ? a : 0;
    }
    for (int o = 0; o < kH; o++) {
      gb1[o] += d1[o];
      for (int k = 0; k < kF; k++) gw1[o * kF + k] += d1[o] * x[k];
    }
  }
  *loss = L / n;
}
