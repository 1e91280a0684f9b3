// cdef_search_oracle.cpp - CPU oracle for goav1's encoder CDEF strength
// search (internal/av1/encoder/cdef_search.go), test infrastructure only.
//
// The search runs over a trial list (cdefSearchJob, cdef_search.go:581-596):
// trial gi tests luma packed strength fsY[gi] and chroma fsUV[gi] (-1: not
// tested, the chroma SSE is cdefDefaultMSEUV * 64), luma rows measured every
// subsamplingFactor-th row with the SSE scaled back (:694-701, :722-734).
// Per 64x64 filter block and trial the SSE of the CDEF-filtered
// reconstruction against the source over the block's non-skip 8x8 blocks
// (cdef_search.go:649-745) goes to mse[0] (luma) or mse[1] (U+V); finish
// (:886-945) picks the frame presets greedily over the list and maps them
// back through fsY (chroma too, or luma's with uvFromY).  The controls of
// each search level and the picture plan (setSVTCDEFSearchControls :72-202,
// updateOnRefInfo :237-272, planSVTCDEF in cdef_frame.go:34-54) are
// restated in oracle_cdef_plan_picture.  Level 1 (all 64 strengths, chroma
// the same list, subsampling 1) is oracle_cdef_search.
#include <stdint.h>
#include <string.h>

#include <vector>

#include "pf_oracle.h"

namespace {

constexpr int kBS = 144;  // cdef/constants.go BStride
constexpr int kVL = 0x4000;

int imin(int a, int b) { return a < b ? a : b; }
int imax(int a, int b) { return a > b ? a : b; }
int iabs(int v) { return v < 0 ? -v : v; }
int bitlen(unsigned v) {
  int n = 0;
  while (v) {
    n++;
    v >>= 1;
  }
  return n;
}

const int kDirs[12][2] = {  // cdef/filter.go:53-66
    {1 * kBS, 2 * kBS},   {1 * kBS, 2 * kBS - 1}, {-1 * kBS + 1, -2 * kBS + 2}, {1, -1 * kBS + 2},
    {1, 2},               {1, 1 * kBS + 2},       {1 * kBS + 1, 2 * kBS + 2},   {1 * kBS, 2 * kBS + 1},
    {1 * kBS, 2 * kBS},   {1 * kBS, 2 * kBS - 1}, {-1 * kBS + 1, -2 * kBS + 2}, {1, -1 * kBS + 2},
};

int constrain(int d, int t, int s) {
  const int a = iabs(d);
  const int l = imin(imax(t - (a >> s), 0), a);
  return d < 0 ? -l : l;
}
int cshift(int t, int damping) { return t == 0 ? 0 : imax(damping - (bitlen((unsigned)t) - 1), 0); }

// cdef/filter.go:79-169 on one sample (8-bit search input).
int filter_px(const uint16_t* in, int base, int pri, int sec, int dir, int damping) {
  const int x = in[base];
  const int ps = cshift(pri, damping), ss = cshift(sec, damping);
  const int t0 = (pri & 1) ? 3 : 4, t1 = (pri & 1) ? 3 : 2;
  int sum = 0, hi = x, lo = x;
  const int p0 = kDirs[dir + 2][0], p1 = kDirs[dir + 2][1];
  const int s0a = kDirs[dir + 4][0], s0b = kDirs[dir + 4][1], s1a = kDirs[dir][0], s1b = kDirs[dir][1];
  const int taps[12] = {in[base + p0],  in[base - p0],  in[base + p1],  in[base - p1],
                        in[base + s0a], in[base - s0a], in[base + s1a], in[base - s1a],
                        in[base + s0b], in[base - s0b], in[base + s1b], in[base - s1b]};
  if (pri)
    sum += t0 * (constrain(taps[0] - x, pri, ps) + constrain(taps[1] - x, pri, ps)) +
           t1 * (constrain(taps[2] - x, pri, ps) + constrain(taps[3] - x, pri, ps));
  if (sec)
    sum += 2 * (constrain(taps[4] - x, sec, ss) + constrain(taps[5] - x, sec, ss) + constrain(taps[6] - x, sec, ss) +
                constrain(taps[7] - x, sec, ss)) +
           constrain(taps[8] - x, sec, ss) + constrain(taps[9] - x, sec, ss) + constrain(taps[10] - x, sec, ss) +
           constrain(taps[11] - x, sec, ss);
  int y = x + ((8 + sum - (sum < 0)) >> 4);
  if (pri && sec) {
    for (int k = 0; k < 12; k++) {
      if (pri == 0 && k < 4) continue;
      hi = imax(hi, taps[k] & (kVL - 1));
      lo = imin(lo, taps[k]);
    }
    y = imin(imax(y, lo), hi);
  }
  return y;
}

// cdef/direction.go:37-79, :432-501.
int find_dir(const uint8_t* p, int stride, int32_t* var) {
  int32_t partial[8][15];
  memset(partial, 0, sizeof(partial));
  for (int i = 0; i < 8; i++)
    for (int j = 0; j < 8; j++) {
      const int32_t x = (int32_t)p[i * stride + j] - 128;
      partial[0][i + j] += x;
      partial[1][i + (j >> 1)] += x;
      partial[2][i] += x;
      partial[3][3 + i - (j >> 1)] += x;
      partial[4][7 + i - j] += x;
      partial[5][3 - (i >> 1) + j] += x;
      partial[6][j] += x;
      partial[7][(i >> 1) + j] += x;
    }
  static const int div[9] = {0, 840, 420, 280, 210, 168, 140, 120, 105};
  int32_t cost[8];
  for (int d = 0; d < 8; d++) {
    const int32_t* q = partial[d];
    int32_t c = 0;
    if (d == 2 || d == 6) {
      for (int i = 0; i < 8; i++) c += q[i] * q[i];
      c *= div[8];
    } else if (d == 0 || d == 4) {
      for (int i = 0; i < 7; i++) c += (q[i] * q[i] + q[14 - i] * q[14 - i]) * div[i + 1];
      c += q[7] * q[7] * div[8];
    } else {
      c = (q[3] * q[3] + q[4] * q[4] + q[5] * q[5] + q[6] * q[6] + q[7] * q[7]) * div[8] +
          (q[0] * q[0] + q[10] * q[10]) * div[2] + (q[1] * q[1] + q[9] * q[9]) * div[4] +
          (q[2] * q[2] + q[8] * q[8]) * div[6];
    }
    cost[d] = c;
  }
  int best = 0;
  for (int d = 1; d < 8; d++)
    if (cost[d] > cost[best]) best = d;
  *var = (cost[best] - cost[(best + 4) & 7]) >> 10;
  return best;
}

int adjust(int s, int32_t v) {  // cdef/filter.go:603-612
  if (v == 0) return 0;
  int i = 0;
  if (v >> 6) i = imin(bitlen((unsigned)(v >> 6)) - 1, 12);
  return (s * (4 + i) + 8) >> 4;
}

struct P8 {
  const uint8_t* d;
  int64_t s;
  int w, h;
  int at(int x, int y) const { return d[(int64_t)y * s + x]; }
};

P8 plane8(const pf_frame* f, int p) {
  return P8{(const uint8_t*)f->plane[p].data, f->plane[p].stride, f->plane[p].width, f->plane[p].height};
}

// The level-1 trial list (gi -> packed strength), cdef_search.go:98-110.
void level1_ctrls(pf_cdef_search_ctrls* c) {
  memset(c, 0, sizeof(*c));
  for (int i = 0; i < 16; i++) c->y[i] = (int8_t)(i * 4);
  int k = 16;
  for (int i = 0; i < 16; i++)
    for (int j = 1; j < 4; j++) c->y[k++] = (int8_t)(i * 4 + j);
  for (int g = 0; g < 64; g++) c->uv[g] = c->y[g];
  c->count = 64;
  c->subsampling = 1;
}

uint64_t rdcost(uint64_t lambda, int64_t rate, uint64_t dist) {  // cdef_search.go:302-304
  return (uint64_t)((rate * (int64_t)lambda + (1 << 8)) >> 9) + (dist << 7);
}

// cdef_search.go:780-869 (searchOneDual).
uint64_t search_one_dual(const std::vector<const uint64_t*>& m0, const std::vector<const uint64_t*>& m1, int* lev0,
                         int* lev1, int nb, int end) {
  const int n = (int)m0.size();
  if (end <= 0) {
    lev0[nb] = lev1[nb] = 0;
    return (uint64_t)1 << 63;
  }
  if (n == 0) {
    lev0[nb] = lev1[nb] = 0;
    return 0;
  }
  if (nb == 0) {
    uint64_t s0[64] = {}, s1[64] = {};
    for (int i = 0; i < n; i++)
      for (int j = 0; j < end; j++) {
        s0[j] += m0[i][j];
        s1[j] += m1[i][j];
      }
    int b0 = 0, b1 = 0;
    for (int j = 1; j < end; j++) {
      if (s0[j] < s0[b0]) b0 = j;
      if (s1[j] < s1[b1]) b1 = j;
    }
    lev0[0] = b0;
    lev1[0] = b1;
    return s0[b0] + s1[b1];
  }
  static uint64_t sav[64][64];
  for (int j = 0; j < end; j++)
    for (int k = 0; k < end; k++) sav[j][k] = 0;
  uint64_t sumBest = 0;
  for (int i = 0; i < n; i++) {
    uint64_t best = m0[i][lev0[0]] + m1[i][lev1[0]];
    for (int g = 1; g < nb; g++) {
      const uint64_t c = m0[i][lev0[g]] + m1[i][lev1[g]];
      if (c < best) best = c;
    }
    sumBest += best;
    for (int j = 0; j < end; j++) {
      const uint64_t v0 = m0[i][j];
      if (v0 >= best) continue;
      const uint64_t rem = best - v0;
      for (int k = 0; k < end; k++)
        if (m1[i][k] < rem) sav[j][k] += rem - m1[i][k];
    }
  }
  uint64_t bestSav = sav[0][0];
  int bj = 0, bk = 0;
  for (int j = 0; j < end; j++)
    for (int k = 0; k < end; k++)
      if (sav[j][k] > bestSav) {
        bestSav = sav[j][k];
        bj = j;
        bk = k;
      }
  lev0[nb] = bj;
  lev1[nb] = bk;
  return sumBest - bestSav;
}

}  // namespace

// Per filter block and plane group: cdef_search.go:649-745 (searchRow), with
// loadCDEFInput (:479-506, VeryLarge outside the cropped plane), the luma
// direction search on the reconstruction, FilterBlocksU8SubsampledTrusted
// with row step 1 (cdef/filter_search.go:20-74: in place, skip when the
// adjusted strength and the secondary are both zero) and computeCDEFDist8.
extern "C" int oracle_cdef_search_ex(const pf_frame* src, const pf_frame* rec, const uint8_t* noskip,
                                     const pf_cdef_search_params* prm, const pf_cdef_search_ctrls* ctrls,
                                     uint64_t* mse_out, uint8_t* fb_index_out, pf_cdef_search_result* result) {
  if (!src || !rec || !prm || !ctrls || !mse_out || rec->bit_depth != 8 || rec->ss_x != 1 || rec->ss_y != 1)
    return PF_ERR_INVALID_ARG;
  const int total = ctrls->count;
  if (total < 1 || total > 64 || ctrls->subsampling < 1) return PF_ERR_INVALID_ARG;
  const int W = rec->width, H = rec->height;
  const int miCols = ((W + 7) >> 3) << 1, miRows = ((H + 7) >> 3) << 1;
  const int nhfb = (miCols + 15) / 16, nvfb = (miRows + 15) / 16, nfb = nhfb * nvfb;
  const int damping = prm->damping ? prm->damping : 3 + (prm->qindex >> 6);
  // Luma rows every ss-th (BLOCK_8X8 caps it at 4); chroma every row.
  const int ssY = imin(ctrls->subsampling, 4);
  std::vector<uint16_t> in(kBS * (128 + 4));
  std::vector<uint8_t> tmp(64 * 64);
  std::vector<uint8_t> skipFB(nfb, 0);
  for (int fbr = 0; fbr < nvfb; fbr++) {
    for (int fbc = 0; fbc < nhfb; fbc++) {
      const int fb = fbr * nhfb + fbc;
      const int lr = 16 * fbr, lc = 16 * fbc;
      const int nhb = imin(16, miCols - lc), nvb = imin(16, miRows - lr);
      // computeCDEFList (cdef_search.go:410-447) from the noskip word.
      uint64_t word = ~0ull;
      if (noskip) {
        word = 0;
        for (int i = 0; i < 8; i++) word |= (uint64_t)noskip[(size_t)fb * 8 + i] << (8 * i);
      }
      std::vector<std::pair<int, int>> dlist;
      for (int r = 0; r < imin(miRows - lr, 16); r += 2)
        for (int c = 0; c < imin(miCols - lc, 16); c += 2)
          if ((word >> ((r >> 1) * 8 + (c >> 1))) & 1) dlist.emplace_back(r >> 1, c >> 1);
      uint64_t* m0 = mse_out + (size_t)fb * 64;
      uint64_t* m1 = mse_out + (size_t)nfb * 64 + (size_t)fb * 64;
      for (int g = total; g < 64; g++) m0[g] = m1[g] = PF_CDEF_NOT_A_TRIAL;
      if (dlist.empty()) {
        skipFB[fb] = 1;
        for (int g = 0; g < total; g++) m0[g] = m1[g] = 0;
        continue;
      }
      uint8_t dir[8][8] = {};
      int32_t var[8][8] = {};
      for (int g = 0; g < total; g++) m1[g] = 0;
      for (int pli = 0; pli < 3; pli++) {
        const int dec = pli ? 1 : 0;
        const int x0 = (lc * 4) >> dec, y0 = (lr * 4) >> dec;
        const int w = (nhb * 4) >> dec, h = (nvb * 4) >> dec;
        const P8 rp = plane8(rec, pli), sp = plane8(src, pli);
        const int planeW = pli ? (W + 1) >> 1 : W, planeH = pli ? (H + 1) >> 1 : H;
        // loadCDEFInput.
        const int origin = 2 * kBS + 8;
        for (int r = -2; r < h + 2; r++)
          for (int c = -8; c < w + 8; c++) {
            const int yy = y0 + r, xx = x0 + c;
            in[origin + r * kBS + c] =
                (yy >= 0 && yy < planeH && xx >= 0 && xx < planeW) ? (uint16_t)rp.at(xx, yy) : (uint16_t)kVL;
          }
        if (pli == 0)
          for (auto& b : dlist)
            dir[b.first][b.second] =
                (uint8_t)find_dir(rp.d + (int64_t)(y0 + 8 * b.first) * rp.s + x0 + 8 * b.second, (int)rp.s,
                                  &var[b.first][b.second]);
        const int bl = 3 - dec, bsz = 1 << bl;
        const int ss = pli ? 1 : ssY;
        for (int g = 0; g < total; g++) {
          if (pli && ctrls->uv[g] < 0) {
            m1[g] = (uint64_t)1040400 * 64;  // cdefDefaultMSEUV * 64 (:669-672)
            continue;
          }
          const int packed = pli ? ctrls->uv[g] : ctrls->y[g];
          const int pri = packed >> 2;
          int sec = packed & 3;
          if (sec == 3) sec = 4;
          uint64_t sse = 0;
          for (auto& b : dlist) {
            const int strength = (pli == 0 && pri != 0) ? adjust(pri, var[b.first][b.second]) : pri;
            const int d = pri != 0 ? dir[b.first][b.second] : 0;
            const int dmp = pli ? damping - 1 : damping;
            for (int i = 0; i < bsz; i += ss)
              for (int j = 0; j < bsz; j++) {
                const int yy = (b.first << bl) + i, xx = (b.second << bl) + j;
                int v;
                if (strength == 0 && sec == 0)
                  v = rp.at(x0 + xx, y0 + yy);
                else  // the 8-bit trial buffer stores byte(...) (cdef/filter_u8.go:151)
                  v = (uint8_t)filter_px(in.data(), origin + yy * kBS + xx, strength, sec, d, dmp);
                const int e = sp.at(x0 + xx, y0 + yy) - v;
                sse += (uint64_t)(e * e);
              }
          }
          if (pli == 0)
            m0[g] = sse * ss;
          else
            m1[g] += sse * ss;
        }
      }
    }
  }
  return oracle_cdef_select_ctrls(mse_out, skipFB.data(), nfb, prm, ctrls, 1, fb_index_out, result);
}

// Level 1 (cdef_search.go:98-110): all 64 strengths in the svtPfGI order,
// chroma the same list, every row measured.
extern "C" int oracle_cdef_search(const pf_frame* src, const pf_frame* rec, const uint8_t* noskip,
                                  const pf_cdef_search_params* prm, uint64_t* mse_out, uint8_t* fb_index_out,
                                  pf_cdef_search_result* result) {
  pf_cdef_search_ctrls c;
  level1_ctrls(&c);
  return oracle_cdef_search_ex(src, rec, noskip, prm, &c, mse_out, fb_index_out, result);
}

// finish (cdef_search.go:886-945) over a given SSE table, at level 1.
extern "C" int oracle_cdef_select(const uint64_t* mse, const uint8_t* skip, int nfb, const pf_cdef_search_params* prm,
                                  uint8_t* fb_index_out, pf_cdef_search_result* result) {
  return oracle_cdef_select_ex(mse, skip, nfb, prm, 1, fb_index_out, result);
}

// refine = 0 stops each configuration after its nb greedy picks (the
// learned search's selection); refine = 1 is finish() itself.
extern "C" int oracle_cdef_select_ex(const uint64_t* mse, const uint8_t* skip, int nfb,
                                     const pf_cdef_search_params* prm, int refine, uint8_t* fb_index_out,
                                     pf_cdef_search_result* result) {
  pf_cdef_search_ctrls c;
  level1_ctrls(&c);
  return oracle_cdef_select_ctrls(mse, skip, nfb, prm, &c, refine, fb_index_out, result);
}

// finish over the first ctrls->count trials (endGI = len(filterMap)); the
// presets map back through the luma list fsY, chroma's too (:937-940), or
// copy luma's with uvFromY (:920-925).
extern "C" int oracle_cdef_select_ctrls(const uint64_t* mse, const uint8_t* skip, int nfb,
                                        const pf_cdef_search_params* prm, const pf_cdef_search_ctrls* ctrls,
                                        int refine, uint8_t* fb_index_out, pf_cdef_search_result* result) {
  const int end = ctrls->count;
  std::vector<const uint64_t*> s0, s1;
  std::vector<int> sbIndex;
  for (int fb = 0; fb < nfb; fb++) {
    if (fb_index_out) fb_index_out[fb] = 0;
    if (skip[fb]) continue;
    s0.push_back(mse + (size_t)fb * 64);
    s1.push_back(mse + (size_t)nfb * 64 + (size_t)fb * 64);
    sbIndex.push_back(fb);
  }
  const int sbCount = (int)s0.size();
  const int maxBits = prm->max_presets >= 8 ? 3 : prm->max_presets >= 4 ? 2 : prm->max_presets >= 2 ? 1 : 0;
  uint64_t bestTot = (uint64_t)1 << 63;
  int bestBits = 0, ys[8] = {}, uvs[8] = {};
  const uint64_t lambda = (uint64_t)prm->lambda;
  for (int i = 0; i <= maxBits; i++) {
    int lev0[8] = {}, lev1[8] = {};
    const int nb = 1 << i;
    uint64_t tot = (uint64_t)1 << 63;
    for (int k = 0; k < nb; k++) tot = search_one_dual(s0, s1, lev0, lev1, k, end);
    for (int k = 0; refine && k < 4 * nb; k++) {
      for (int j = 0; j < nb - 1; j++) {
        lev0[j] = lev0[j + 1];
        lev1[j] = lev1[j + 1];
      }
      tot = search_one_dual(s0, s1, lev0, lev1, nb - 1, end);
    }
    const int totalBits = sbCount * i + nb * 6 * 2;
    const uint64_t cost = rdcost(lambda, (int64_t)totalBits << 9, tot * 16);
    if (cost < bestTot) {
      bestTot = cost;
      bestBits = i;
      for (int j = 0; j < nb; j++) {
        ys[j] = lev0[j];
        uvs[j] = ctrls->uv_from_y ? lev0[j] : lev1[j];
      }
    }
  }
  const int nb = 1 << bestBits;
  for (int i = 0; i < sbCount; i++) {
    int bg = 0;
    uint64_t bm = (uint64_t)1 << 63;
    for (int g = 0; g < nb; g++) {
      const uint64_t c = s0[i][ys[g]] + s1[i][uvs[g]];
      if (c < bm) {
        bg = g;
        bm = c;
      }
    }
    if (fb_index_out) fb_index_out[sbIndex[i]] = (uint8_t)bg;
  }
  if (result) {
    memset(result, 0, sizeof(*result));
    result->bits = (uint8_t)bestBits;
    result->strength_count = (uint8_t)nb;
    for (int j = 0; j < nb; j++) {
      result->y_strength[j] = (uint8_t)ctrls->y[ys[j]];
      result->uv_strength[j] = (uint8_t)ctrls->y[uvs[j]];
    }
    result->cost = (double)bestTot;
  }
  return PF_OK;
}

// ---------------------------------------------------------------------------
// Search controls per level and the picture plan.
namespace {
const int8_t kPfGI[16] = {0, 4, 8, 12, 16, 20, 24, 28, 32, 36, 40, 44, 48, 52, 56, 60};  // svtPfGI

struct Ctrls {  // svtCDEFSearchCtrls (cdef_search.go:55-70)
  bool enabled = false;
  int first = 0, second = 0;
  int8_t fs[64] = {}, fs2[64] = {}, fsuv[64] = {}, fs2uv[64] = {};
  bool useRef = false, bestRef = false, skipDet = false, uvFromY = false, qp = false;
  int ss = 0;
  int predY = 0, predUV = 0;
};

// setSVTCDEFSearchControls (cdef_search.go:72-202).
Ctrls controls(int level, bool isBase, bool notHighest) {
  Ctrls c;
  auto secondPass = [&]() {
    int sf = 0;
    for (int i = 0; i < c.first; i++)
      for (int j = 1; j < 4; j++) c.fs2[sf++] = (int8_t)(c.fs[i] + j);
  };
  auto uvFirst = [&]() {
    for (int i = 0; i < c.first; i++) c.fsuv[i] = c.fs[i];
  };
  auto uvSecondOff = [&]() {
    for (int i = 0; i < c.second; i++) c.fs2uv[i] = -1;
  };
  auto firstFrom = [&](std::initializer_list<int> gs) {
    int i = 0;
    for (int g : gs) c.fs[i++] = kPfGI[g];
    c.first = i;
  };
  switch (level) {
    case 1:
      c.enabled = true;
      firstFrom({0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 14, 15});
      c.second = c.first * 3;
      secondPass();
      uvFirst();
      for (int i = 0; i < c.second; i++) c.fs2uv[i] = c.fs2[i];
      c.ss = 1;
      break;
    case 2:
    case 3:
    case 4:
      c.enabled = true;
      if (level == 2) firstFrom({0, 1, 2, 4, 5, 6, 8, 9, 10, 12, 13, 14});
      if (level == 3) firstFrom({0, 4, 8, 12, 15});
      if (level == 4) firstFrom({0, 7, 15});
      c.second = c.first * 3;
      secondPass();
      uvFirst();
      uvSecondOff();
      c.ss = 1;
      break;
    case 5:
      c.enabled = true;
      firstFrom({0, 7, 15});
      c.second = c.first;
      for (int i = 0; i < 3; i++) c.fs2[i] = (int8_t)(c.fs[i] + 2);
      uvFirst();
      uvSecondOff();
      c.bestRef = !notHighest;
      c.ss = 1;
      break;
    case 6:
    case 7:
    case 8:
      c.enabled = true;
      c.first = 2;
      c.second = 2;
      c.fs[0] = kPfGI[0];
      c.fs[1] = kPfGI[15];
      c.fs2[0] = (int8_t)(kPfGI[0] + 2);
      c.fs2[1] = (int8_t)(kPfGI[15] + 2);
      if (level == 8) {
        c.fsuv[0] = c.fsuv[1] = -1;
      } else {
        c.fsuv[0] = c.fs[0];
        c.fsuv[1] = c.fs[1];
      }
      c.fsuv[2] = -1;
      c.fs2uv[0] = c.fs2uv[1] = -1;
      c.ss = 4;
      if (level == 6) c.bestRef = !notHighest;
      if (level == 7) {
        c.useRef = !notHighest;
        c.bestRef = !isBase;
        c.skipDet = !isBase;
      }
      if (level == 8) {
        c.useRef = !isBase;
        c.bestRef = !isBase;
        c.uvFromY = true;
      }
      break;
    default:
      break;
  }
  if (c.uvFromY && !c.qp) {
    for (int i = 0; i < c.first; i++) c.fsuv[i] = -1;
    for (int i = 0; i < c.second; i++) c.fs2uv[i] = -1;
  }
  return c;
}

// updateOnRefInfo (cdef_search.go:237-272).
bool update_on_ref(Ctrls& c, const pf_cdef_ref_strengths& ref) {
  if (c.useRef) {
    int lo = 63, hi = 0;
    for (int i = 0; i < ref.count; i++) {
      lo = imin(lo, ref.y[i]);
      hi = imax(hi, ref.y[i]);
    }
    c.predY = imin(63, (lo + hi) / 2);
    c.predUV = 0;
    c.first = 0;
    c.second = 0;
    return c.predY != 0 || c.predUV != 0;
  }
  if (c.bestRef) {
    c.first = 1;
    c.second = 0;
    if ((int8_t)ref.y[0] != c.fs[0]) {
      c.fs[1] = (int8_t)ref.y[0];
      c.first++;
    }
    if ((int8_t)ref.uv[0] == c.fsuv[0]) {
      c.fsuv[0] = -1;
      c.fsuv[1] = -1;
    }
    return c.first != 1;
  }
  return true;
}
}  // namespace

// planSVTCDEF (cdef_frame.go:34-54) at an explicit search level, and the
// job's trial list (cdef_search.go:585-596).
extern "C" int oracle_cdef_plan_picture(int level, int islice, int is_base, int not_highest_layer,
                                        const pf_cdef_ref_strengths* ref, int ref_skip_percent, pf_cdef_plan* plan) {
  if (!plan || level < 0 || level > 8) return PF_ERR_INVALID_ARG;
  memset(plan, 0, sizeof(*plan));
  if (level == 0) return PF_OK;
  Ctrls c = controls(level, is_base != 0, not_highest_layer != 0);
  bool on = c.enabled;
  if (!islice && on) {
    if (ref_skip_percent > 75 && c.skipDet) {
      on = false;
    } else if (c.useRef || c.bestRef) {
      if (!ref) return PF_ERR_INVALID_ARG;
      on = update_on_ref(c, *ref);
    }
  }
  plan->on = on;
  plan->search = on && !c.useRef;
  if (on && c.useRef) {
    plan->y_strength = (uint8_t)c.predY;
    plan->uv_strength = (uint8_t)c.predUV;
  }
  pf_cdef_search_ctrls& t = plan->ctrls;
  t.count = c.first + c.second;
  for (int g = 0; g < t.count; g++) {
    t.y[g] = g < c.first ? c.fs[g] : c.fs2[g - c.first];
    t.uv[g] = g < c.first ? c.fsuv[g] : c.fs2uv[g - c.first];
  }
  t.subsampling = c.ss;
  t.uv_from_y = c.uvFromY;
  return PF_OK;
}
