// pf_cdef.cu - CDEF on the GPU, one CTA per 64x64 filter unit (all planes).
//
// Semantics follow goav1's snapshot walk: internal/av1/decoder/
// postfilter_cdef.go:525-710 (applyCDEFPostFilterRows), :936-1035
// (unitStrength, applySnapshot), :1041-1047 (luma direction gate),
// :1101-1249 (VeryLarge halo fill and the row/column replicate quirk of
// frameWorkCopyCDEFInput), :1390-1412 (MI-aligned plane extent), :1544-1561
// (block list from the noskip word); and the kernels cdef/direction.go:37-79,
// :432-501, cdef/filter.go:79-169, :231-241, :396-543, :603-633.
//
// The kernel reads the deblocked frame (never written here) and writes every
// sample of the unit's MI-aligned extent to the output frame, filtered or
// copied, so the output is a pure function of the pre-CDEF frame exactly as
// in the reference's immutable-snapshot walk.  It also saves, straight from
// the pre-CDEF input, the four rows around each loop-restoration stripe
// boundary that falls inside the unit (tile/restoration_boundary.go:192-255):
// the boundary-line save is fused into the CDEF pass instead of a separate
// frame sweep.
#include "pf_cdef_dev.cuh"

namespace pf {

// 8-bit units without sentinels read constrain() from tables: one per
// primary strength used in the unit (8-bit strengths are 1..15) and one for
// the secondary strength, 511 entries each (differences -255..255).
constexpr int kTabLen = 512;
constexpr int kSecTab = 16;

struct CdefSmem {
  alignas(16) uint16_t in[kSH * kSW];
  int32_t cost[64 * 8];
  int32_t var[64];
  int32_t blk[64];   // per block: filter flag << 16 | priShift << 12 | strength << 4 | dir
  int2 ofs[12];      // direction tap offsets in smem units (cdef/filter.go:53-66)
  uint8_t dir[64];
  alignas(16) int16_t tab[kSecTab + 1][kTabLen];
  uint32_t strengths;    // bit k: a block of the plane filters with primary strength k
  int8_t slot[16];       // table of each primary strength
  int8_t slot_str[16];   // strength of each table
};

// One 64x64 filter unit (uc, ur), all planes.  aw/ah: MI-aligned extents
// (frameWorkCDEFAlignedPlane).
template <typename T>
__device__ void cdef_unit(const DFrame& in, const DFrame& out, const CdefArgs& a, const int* aw, const int* ah,
                          int uc, int ur, CdefSmem& sm) {
  uint16_t* s_in = sm.in;
  uint8_t* s_dir = sm.dir;
  int32_t* s_var = sm.var;
  int32_t* s_cost = sm.cost;
  const int tid = threadIdx.x;
  if (tid < 12) sm.ofs[tid] = make_int2(dir_off(tid, 0), dir_off(tid, 1));
  const int coeffShift = sizeof(T) == 1 ? 0 : in.bd - 8;
  // The index map is only present when CDEF filters; the copy-only pass (CDEF
  // off, loop restoration on) reads no side information.
  const int mapOff = ur * a.index_stride + uc;
  const bool rd = a.filter && a.read[mapOff] != 0;
  const int idx = a.filter ? a.index[mapOff] : 0;
  uint64_t word = ~0ull;
  if (a.filter && a.noskip) {
    const uint8_t* w = a.noskip + (size_t)(ur * a.ucols + uc) * 8;
    word = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) word |= (uint64_t)w[i] << (8 * i);
  }
  const int nplanes = in.mono ? 1 : 3;
  for (int plane = 0; plane < nplanes; plane++) {
    const int xdec = plane ? in.ssx : 0, ydec = plane ? in.ssy : 0;
    const int Wa = aw[plane], Ha = ah[plane];
    const int unitX = (uc * 64) >> xdec, unitY = (ur * 64) >> ydec;
    const int unitW = imin(64 >> xdec, Wa - unitX), unitH = imin(64 >> ydec, Ha - unitY);
    if (unitW <= 0 || unitH <= 0) continue;
    const DPlane& ip = in.pl[plane];
    const DPlane& op = out.pl[plane];
    // ---- activity of this (unit, plane), postfilter_cdef.go:936-956 ----
    bool active = false, needPrimary = false, directionOnly = false;
    int packed = 0;
    if (a.filter && a.plane_process[plane] && rd && idx < a.strength_count) {
      packed = plane == 0 ? a.y_strength[idx] : a.uv_strength[idx];
      if (plane == 0)
        needPrimary = (a.y_strength[idx] >> 2) != 0 || (a.chroma_filtering && (a.uv_strength[idx] >> 2) != 0);
      else
        needPrimary = (a.uv_strength[idx] >> 2) != 0;
      directionOnly = plane == 0 && a.chroma_filtering && packed == 0 && (a.uv_strength[idx] >> 2) != 0;
      active = packed != 0 || directionOnly;
    }
    const int bwLog2 = 3 - xdec, bhLog2 = 3 - ydec;
    const int bcols = (unitW + (1 << bwLog2) - 1) >> bwLog2, brows = (unitH + (1 << bhLog2) - 1) >> bhLog2;
    uint64_t listed = 0;
    if (active) {
      const uint64_t colMask = (1ull << bcols) - 1;
      for (int by = 0; by < brows; by++) listed |= ((word >> (by * 8)) & colMask) << (by * 8);
      if (listed == 0) active = false;
    }
    const int uwMax = 64 >> xdec;
    const int rowStep = 256 / uwMax;
    const int tx = tid % uwMax, ty0 = tid / uwMax;
    if (!active) {
      // Copy-through (inactive unit / plane or the CDEF stage is off).
      copy_block<T>(ip, op, unitX, unitX + unitW, unitY, unitY + unitH);
    } else {
      // ---- stage the unit + halo (frameWorkFillCDEFInputSentinels /
      //      frameWorkCopyCDEFInput with the replicate quirk) ----
      const int srcX0 = imax(unitX - 8, 0), srcY0 = imax(unitY - 2, 0);
      const int srcX1 = imin(unitX + unitW + 8, Wa), srcY1 = imin(unitY + unitH + 2, Ha);
      const int wantY1 = unitY + unitH + 2, wantX1 = unitX + unitW + 8;
      const bool rowExt = srcY1 < wantY1 && srcY1 > 0 && unitY + unitH < Ha;
      const bool colExt = srcX1 < wantX1 && srcX1 > 0 && unitX + unitW < Wa;
      const int extRowsEnd = srcY0 + (rowExt ? wantY1 - srcY0 : srcY1 - srcY0);
      const int fillW = unitW + 16, fillH = unitH + 4;
      const int warp = tid >> 5, lane = tid & 31;
      const bool interior = srcX0 == unitX - 8 && srcX1 == wantX1 && srcY0 == unitY - 2 && srcY1 == wantY1;
      const uint8_t* tile0 = reinterpret_cast<const uint8_t*>(row_ptr<T>(ip, unitY - 2) + (unitX - 8));
      // Words of 8 samples: 8 bytes (8-bit, rows start 8 bytes before a
      // 64-sample unit) or 16 bytes (10/12-bit).
      constexpr int kWord = 8 * sizeof(T);
      if (interior && fillW % 8 == 0 &&
          ((reinterpret_cast<uintptr_t>(tile0) | (uintptr_t)ip.stride) & (kWord - 1)) == 0) {
        // Interior unit with aligned rows: the whole halo is frame data, a
        // thread's few words unrolled so their loads are in flight together.
        const int wpr = fillW / 8, total = fillH * wpr;
        constexpr int kMaxItems = (kSH * (kSW / 8) + 255) / 256;
#pragma unroll
        for (int k = 0; k < kMaxItems; k++) {
          const int i = tid + 256 * k;
          if (i < total) {
            const int r = i / wpr, cw = i - r * wpr;
            const uint8_t* src = tile0 + (int64_t)r * ip.stride + cw * kWord;
            uint4 v;
            if (sizeof(T) == 1) {
              const uint2 w = *reinterpret_cast<const uint2*>(src);
              v = make_uint4(__byte_perm(w.x, 0, 0x4140), __byte_perm(w.x, 0, 0x4342), __byte_perm(w.y, 0, 0x4140),
                             __byte_perm(w.y, 0, 0x4342));
            } else {
              v = *reinterpret_cast<const uint4*>(src);
            }
            *reinterpret_cast<uint4*>(&s_in[r * kSW + cw * 8]) = v;
          }
        }
      } else if (interior) {
        // Interior unit: the whole halo is frame data.
        for (int r = warp; r < fillH; r += 8) {
          const T* src = row_ptr<T>(ip, unitY - 2 + r) + (unitX - 8);
          uint16_t* dst = &s_in[r * kSW];
          for (int c = lane; c < fillW; c += 32) dst[c] = src[c];
        }
      } else {
        for (int r = warp; r < fillH; r += 8) {
          const int sy = unitY - 2 + r;
          int ry = -1;
          if (sy >= srcY0 && sy < srcY1) ry = sy;
          else if (rowExt && sy >= srcY1 && sy < wantY1) ry = srcY1 - 1;
          const bool extRow = colExt && sy >= srcY0 && sy < extRowsEnd;
          const int ryExt = ry < 0 ? srcY1 - 1 : ry;
          uint16_t* dst = &s_in[r * kSW];
          for (int c = lane; c < fillW; c += 32) {
            const int sx = unitX - 8 + c;
            int v = kVeryLarge;
            if (sx >= srcX0 && sx < srcX1) {
              if (ry >= 0) v = row_ptr<T>(ip, ry)[sx];
            } else if (extRow && sx >= srcX1 && sx < wantX1) {
              v = row_ptr<T>(ip, ryExt)[srcX1 - 1];
            }
            dst[c] = (uint16_t)v;
          }
        }
      }
      __syncthreads();
      // ---- luma direction search on listed blocks (needPrimary) ----
      if (plane == 0 && needPrimary) {
        // A warp takes one direction for 32 blocks, so the direction's
        // template runs without divergence.
        for (int w = tid; w < 64 * 8; w += 256) {
          const int d = w >> 6, b = w & 63;
          const int by = b >> 3, bx = b & 7;
          if ((listed >> b) & 1)
            s_cost[b * 8 + d] = dir_cost_any(d, &s_in[(2 + by * 8) * kSW + 8 + bx * 8], coeffShift);
        }
        __syncthreads();
        if (tid < 64 && ((listed >> tid) & 1)) {
          int best = 0;
          int32_t bestCost = s_cost[tid * 8];
          for (int d = 1; d < 8; d++) {
            const int32_t c = s_cost[tid * 8 + d];
            if (c > bestCost) {
              best = d;
              bestCost = c;
            }
          }
          s_dir[tid] = (uint8_t)best;
          s_var[tid] = (bestCost - s_cost[tid * 8 + ((best + 4) & 7)]) >> 10;
        }
        __syncthreads();
      }
      if (plane == 1 && needPrimary && xdec != ydec) {
        // cdef/filter.go:614-633: U converts the shared grid in place (V reuses it).
        if (tid < 64 && ((listed >> tid) & 1)) {
          const uint8_t conv422[8] = {7, 0, 2, 4, 5, 6, 6, 6};
          const uint8_t conv440[8] = {1, 2, 2, 2, 3, 4, 6, 0};
          s_dir[tid] = xdec ? conv422[s_dir[tid]] : conv440[s_dir[tid]];
        }
        __syncthreads();
      }
      // ---- filter ----
      int lvl = packed >> 2, sec = packed & 3;
      if (sec == 3) sec = 4;
      const int pri = lvl << coeffShift;
      sec <<= coeffShift;
      int damping = a.damping + coeffShift;
      if (plane != 0) damping--;
      const bool lumaAdjust = plane == 0 && (needPrimary || pri != 0);
      // Per-block parameters once (cdef/filter.go:490-543): adjusted luma
      // strength, direction (0 when the primary strength is zero), shift.
      // 8-bit units whose halo is all frame data: constrain() from tables.
      const bool useTab = sizeof(T) == 1 && interior;
      if (tid == 0) sm.strengths = 0;
      __syncthreads();
      if (tid < 64) {
        const int b = tid;
        int pk = 0;
        if (!directionOnly && ((listed >> b) & 1)) {
          const int strength = lumaAdjust ? adjust_strength(pri, s_var[b]) : pri;
          const int dir = pri != 0 ? s_dir[b] : 0;
          pk = (1 << 16) | (constrain_shift(strength, damping) << 12) | (strength << 4) | dir;
          if (useTab && strength) atomicOr(&sm.strengths, 1u << strength);
        }
        sm.blk[b] = pk;
      }
      __syncthreads();
      const int secShift = constrain_shift(sec, damping);
      // The output row base in registers: the plane descriptor sits in the
      // job table, which the compiler would re-read after every store.
      uint8_t* const obase = op.ptr;
      const int64_t ostride = op.stride;
      if (useTab) {
        const uint32_t used = sm.strengths;
        const int ntab = __popc(used);
        if (tid < 16) {
          const bool on = (used >> tid) & 1;
          const int k = __popc(used & ((1u << tid) - 1));
          sm.slot[tid] = on ? (int8_t)k : (int8_t)-1;
          if (on) sm.slot_str[k] = (int8_t)tid;
        }
        __syncthreads();
        // Each table is a copy of the context's precomputed one for its
        // strength and shift (64 16-byte words; zeros for no secondary).
        for (int i = tid; i < (ntab + 1) * (kTabLen / 8); i += 256) {
          const int t = i / (kTabLen / 8), wd = i - t * (kTabLen / 8);
          const int st = t < ntab ? sm.slot_str[t] : sec;
          const int sh = t < ntab ? constrain_shift(st, damping) : secShift;
          uint4 v = make_uint4(0, 0, 0, 0);
          if (st) v = reinterpret_cast<const uint4*>(a.ctab + (size_t)(st * 8 + sh) * kTabLen)[wd];
          reinterpret_cast<uint4*>(&sm.tab[t < ntab ? t : kSecTab][0])[wd] = v;
        }
        __syncthreads();
      }
      if (tx < unitW) {
        // A thread takes one column over a run of whole block rows (16 or
        // 8 luma rows, 4 or 8 chroma rows), so each block's parameters
        // (strength, direction taps, table) are read once per block, not
        // once per sample; a warp still covers 32 adjacent columns of one
        // row at a time.
        const int rpt = (64 >> ydec) / rowStep;
        const int ya = ty0 * rpt, yb = imin(unitH, ya + rpt);
        const int bh = 1 << bhLog2;
        for (int yblk = ya; yblk < yb; yblk += bh) {
          const int b = ((yblk >> bhLog2) << 3) + (tx >> bwLog2);
          const int pk = sm.blk[b];
          const int yend = imin(yblk + bh, yb);
          const int strength = (pk >> 4) & 255, dir = pk & 7;
          const bool filt = (pk >> 16) && (strength | sec);
          const int2 po = sm.ofs[dir + 2], s0 = sm.ofs[dir + 4], s1 = sm.ofs[dir];
          const int16_t* tp = (useTab && strength) ? &sm.tab[sm.slot[strength]][255] : nullptr;
          const int16_t* ts = &sm.tab[kSecTab][255];
          const int priShift = (pk >> 12) & 15;
          for (int y = yblk; y < yend; y++) {
            const uint16_t* c = &s_in[(2 + y) * kSW + 8 + tx];
            int v = c[0];
            if (filt) {
              if (useTab)
                v = cdef_filter_px_tab(c, strength, tp, sec, ts, po, s0, s1);
              else if (interior)  // no VeryLarge sentinel anywhere in the halo
                v = cdef_filter_px<false>(c, strength, priShift, sec, secShift, po, s0, s1, coeffShift);
              else
                v = cdef_filter_px<true>(c, strength, priShift, sec, secShift, po, s0, s1, coeffShift);
            }
            reinterpret_cast<T*>(obase + (int64_t)(unitY + y) * ostride)[unitX + tx] = (T)v;
          }
        }
      }
      __syncthreads();
    }
    // ---- fused loop-restoration boundary-line save (pre-CDEF rows) ----
    // Rows b-2 .. b+1 around each stripe boundary b = k*SH - off (k >= 1)
    // inside the unit; the rows of one boundary are spread over the CTA.
    if (a.save_lines[plane]) {
      const int Hc = ip.h, Wc = ip.w;
      const int SHs = 64 >> ydec, off = 8 >> ydec;
      const int yEnd = imin(unitY + unitH, Hc);
      if (unitY < yEnd) {
        const int k0 = imax((unitY + off + 2) / SHs, 1), k1 = (yEnd - 1 + off + 2) / SHs;
        for (int k = k0; k <= k1; k++) {
          const int b = k * SHs - off;
          if (b >= Hc) break;
          const int ya = imax(unitY, b - 2), yb = imin(yEnd - 1, b + 1);
          // At most 4 rows of at most 64 samples: one sample per thread,
          // from the staged unit when this plane was staged (the rows lie
          // inside the unit, so they are frame samples there too).
          const int r = tid >> (6 - xdec), c = tid & (uwMax - 1);
          const int y = ya + r, x = unitX + c;
          if (y <= yb && c < unitW && x < Wc) {
            const int j = y - (b - 2);
            const T v = active ? (T)s_in[(y - unitY + 2) * kSW + 8 + c] : row_ptr<T>(ip, y)[x];
            reinterpret_cast<T*>(a.lines[plane] + (int64_t)(k * 4 + j) * a.line_stride[plane])[x] = v;
            if (j == 2 && b + 1 >= Hc)
              reinterpret_cast<T*>(a.lines[plane] + (int64_t)(k * 4 + 3) * a.line_stride[plane])[x] = v;
          }
        }
      }
      if (active) __syncthreads();  // the next plane restages s_in
    }
  }
}

// Batched CDEF: each work item is one 64x64 unit of one frame.
template <bool kLoop>
__global__ void __launch_bounds__(256, 4) k_cdef_batch(BatchArgs b) {
  __shared__ CdefSmem sm;
  const int* base = b.base + ST_CDEF * (b.n + 1);
  for_each_item<kLoop>(
      b, ST_CDEF,
      [&](int item) {
        const int fi = find_frame(base, b.n, item);
        const FrameJob& J = b.jobs[fi];
        const int local = item - base[fi];
        const int uc = local % J.cdef.ucols, ur = local / J.cdef.ucols;
        if (J.io.bd == 8)
          cdef_unit<uint8_t>(J.io, J.scr, J.cdef, J.aw, J.ah, uc, ur, sm);
        else
          cdef_unit<uint16_t>(J.io, J.scr, J.cdef, J.aw, J.ah, uc, ur, sm);
      },
      [&](int item) {
        // Every plane's unit with its 8-column / 2-row halo.
        const int fi = find_frame(base, b.n, item);
        const FrameJob& J = b.jobs[fi];
        const int local = item - base[fi];
        const int uc = local % J.cdef.ucols, ur = local / J.cdef.ucols;
        for (int plane = 0; plane < (J.io.mono ? 1 : 3); plane++) {
          const int xdec = plane ? J.io.ssx : 0, ydec = plane ? J.io.ssy : 0;
          const int x = (uc * 64) >> xdec, y = (ur * 64) >> ydec;
          if (J.io.bd == 8)
            prefetch_block<uint8_t>(J.io.pl[plane], x - 8, x + (64 >> xdec) + 8, y - 2, y + (64 >> ydec) + 2);
          else
            prefetch_block<uint16_t>(J.io.pl[plane], x - 8, x + (64 >> xdec) + 8, y - 2, y + (64 >> ydec) + 2);
        }
      });
}

// The constrain() tables of CdefArgs.ctab, from constrain() itself: one
// CTA per (strength, shift).
__global__ void __launch_bounds__(kTabLen) k_cdef_tables(int16_t* t) {
  const int st = blockIdx.x >> 3, sh = blockIdx.x & 7, i = threadIdx.x;
  t[(size_t)blockIdx.x * kTabLen + i] = (int16_t)(i < 511 ? constrain(i - 255, st, sh) : 0);
}

size_t cdef_tables_bytes() { return (size_t)16 * 8 * kTabLen * sizeof(int16_t); }

cudaError_t launch_cdef_tables(int16_t* dst, cudaStream_t st) {
  k_cdef_tables<<<16 * 8, kTabLen, 0, st>>>(dst);
  return cudaGetLastError();
}

cudaError_t launch_cdef_batch(const BatchArgs& b, int total, int grid, cudaStream_t st) {
  if (total <= 0) return cudaSuccess;
  static int wave = 0;
  if (batch_loops(b))
    k_cdef_batch<true><<<grid, 256, 0, st>>>(b);
  else
    k_cdef_batch<false><<<grid, 256, 0, st>>>(with_wave(b, k_cdef_batch<false>, 256, 0, wave));
  return cudaGetLastError();
}

}  // namespace pf
