// te_pair.cu — persistent pair-tile transfer-entropy kernel for multi-bin data.
//
// What it computes (reference: tenex/csrc/full_smem.cu:166-276 and
// tenex/csrc/adaptive_smem.cu:158-273): for every ordered pair (source y ->
// target x) in a pair-free id range, the joint counts
//   c3[xt1, xt, yt] = #{s < N : x[s+lag] = xt1, x[s] = xt, y[s] = yt}
// (exact int), the marginals c1[xt], c2a[xt1,xt], c2b[xt,yt], and
//   TE = (1/N) * sum_{c3>0} c3 * log2(c3*c1 / (c2a*c2b)).
//
// How (B200 design, not the reference's one-CTA-per-pair layout):
//   * Work item = one target and a chunk of W sources. The CTA stages the
//     target's joint state z[s] = x[s+lag]*b_t + x[s] into shared memory once
//     per item (u8 when b_t <= 16, else u16) with the target-only marginals
//     c2a (= row sums of c3 over yt) and c1, so sources never re-read it.
//     Series too long for that are staged in tiles of samples, the CTA's groups
//     walking the tiles together.
//   * Shared memory after the target block is cut into histogram slots sized
//     for the item (b_t^2 * b_s cells); a slot belongs to a group of G warps
//     (G = 1: warp-private histograms for the common small pairs). Counters are
//     32-bit unless 32-bit slots would need groups of more than 4 warps, then
//     16-bit halves of a word (N < 65536; two cells per word collide more
//     often, so packing is the fallback, not the rule). Where the item's slots
//     still fit at that size, table rows get an odd stride in words (b_s | 1,
//     or the half-word row | 1): rows then start in different banks, so lanes
//     that share a popular source bin but differ in target state land in
//     different banks instead of the same one or two. Pairs whose histogram
//     fits no shared-memory slot (coarsening off) run in a second
//     instantiation on per-CTA slots in global memory.
//   * Every sample is one red.shared.add (16 samples per uint4 of source bins).
//     The hardware merges lanes that add to the same word, so the cost of a
//     warp-wide reduction is the largest number of distinct words in one bank;
//     warp-level aggregation of equal cells would not lower it.
//   * The entropy pass reads each column once to form c2b, once more to form
//     the terms (ratio c3 * (1/c2b) * (c1/c2a), lg2.approx; exact 0 where
//     c3*c1 == c2a*c2b) and clears shared slots for the next source. Series of
//     2^24 samples or more take a float64 pass (float32 holds the counts exactly
//     only below 2^24).
//   * Items are handed out by an atomic ticket, targets in blocks of ~20% of L2 and
//     chunk-major within a block, so the CTAs resident at one moment share a
//     small set of source rows in L2. Sources are ordered by bin count, so one
//     item's slots are sized for sources of similar b.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstddef>
#include <mutex>

#include "common.cuh"

namespace tenex {

enum { kOutPairfree = 0, kOutMatrix = 1, kOutStats = 2 };

struct TeParams {
  const uint8_t* bins;
  int64_t ld;
  const int32_t* npv;
  int n;
  int N;          // samples per pair (row_len - lag), < 2^31
  int lag;
  int ztile;      // samples of the target staged at a time (N: the whole series)
  int big;        // N >= 2^24: float64 entropy pass
  int64_t p0, p1;  // pair-free id range [p0, p1)
  int t_first;
  int n_targets;
  int W;          // sources per item
  int n_chunks;   // items per target
  int tblock;     // targets per L2 block of the item order (pair-free mode)
  // global-memory overflow launch: pairs whose histogram does not fit shared
  // memory (only with coarsening off), one 32-bit slot of gslot_words per CTA
  int overflow;   // an overflow launch exists: both launches filter pairs by slot_fits
  uint32_t* gslots;
  int64_t gslot_words;
  // overflow launch, whole series staged: per-CTA c2b counts (gc2b_words each,
  // zero between pairs) for the entropy from the pair's samples
  uint32_t* gc2b;
  int64_t gc2b_words;
  int64_t n_items;
  int zbytes;     // bytes per z entry reserved (1 or 2)
  int bmax;       // max n_per_var (sizes the c1 row)
  // largest target b whose marginal tables (c2a, c1/c2a: 12 B x b^2) live in shared
  // memory; = bmax unless those tables for bmax would crowd out the histograms
  // (coarsening off, b in the hundreds). Pairs of larger targets run in the
  // overflow launch with the target's tables in gmarg (per CTA: 3 x bmax^2 words).
  int mbmax;
  int32_t* gmarg;
  int64_t gmarg_words;
  int smem_bytes;
  int out_mode;
  float* out;
  int64_t out_ld;
  const float* obs;
  double* sum;
  double* sumsq;
  int32_t* cnt_ge;
  int32_t* counts_dbg;
  int64_t counts_stride;
  const int32_t* order; // (n,) genes stably sorted by bin-count class (pair-free mode)
  // pair-list mode (pairs != nullptr): item q is pairs[item_start[q] .. item_start[q+1])
  // of one target; output index = position in the list
  const int64_t* pairs;
  const int64_t* item_start;
  WsHeader* ws;
};

// Workspace: header | order (n int32), 256-byte aligned (bmax kept in the
// signature for callers; the layout no longer depends on it).
__host__ __device__ inline int64_t ws_order_off(int n, int bmax) {
  (void)n;
  (void)bmax;
  return round_up((int64_t)sizeof(WsHeader), 256);
}
__host__ __device__ inline int64_t ws_total(int n, int bmax) {
  return round_up(ws_order_off(n, bmax) + (int64_t)n * 4, 256);
}

namespace {

constexpr int kMaxWarps = 32;

// Histogram layouts (see the file comment).
enum { kSlot32 = 0, kSlot16 = 1, kGmem = 2 };

struct SmemLayout {
  int z_off, c2a_off, c1_off, q_off, red_off, misc_off, slot_off;
};

// ztile: samples staged at a time (the z region holds ztile entries of zbytes);
// c1 holds bmax entries, the marginal tables mbmax^2.
__host__ __device__ inline SmemLayout smem_layout(int ztile, int zbytes, int bmax, int mbmax) {
  SmemLayout L;
  int off = 0;
  L.misc_off = off;  off += 64;                               // int misc[16]
  L.red_off = off;   off += kMaxWarps * 8;                    // double red[32]
  L.c1_off = off;    off += (int)round_up((int64_t)bmax * 4, 16);            // int c1[bt]
  L.c2a_off = off;   off += (int)round_up((int64_t)mbmax * mbmax * 4, 16);   // int c2a[bt^2]
  L.q_off = off;     off += (int)round_up((int64_t)mbmax * mbmax * 8, 16);   // {c1/c2a, c2a}
  L.z_off = off;     off += (int)round_up((int64_t)ztile * zbytes, 16);
  L.slot_off = (int)round_up(off, 128);
  return L;
}

// Slot cell (z, y): PACK16 -> 16-bit half (y & 1) of word z*hb + (y >> 1),
// else word z*bs + y.
template <bool PACK16>
__device__ __forceinline__ uint32_t cell_get(const uint32_t* slot, uint32_t z, uint32_t y,
                                             uint32_t bs, uint32_t hb) {
  if (PACK16) {
    const uint32_t w = slot[z * hb + (y >> 1)];
    return (y & 1u) ? (w >> 16) : (w & 0xffffu);
  }
  return slot[z * bs + y];
}

// Counts one sample: one reduction per sample (inline PTX, no return value).
// kSlot16 adds 1 or 1 << 16 to the word holding the cell's 16-bit half. base is
// the slot's address: the 32-bit shared window address, or (kGmem, the
// global-memory overflow slot) the global address.
template <int MODE>
__device__ __forceinline__ void hist_add(uint64_t base, uint32_t z, uint32_t y, uint32_t bs,
                                         uint32_t hb) {
  uint32_t off, inc = 1u;
  if (MODE == kSlot16) {
    off = (z * hb + (y >> 1)) << 2;
    inc = (y & 1u) * 0xffffu + 1u;
  } else {
    off = (z * bs + y) << 2;
  }
  if (MODE == kGmem)
    asm volatile("red.global.add.u32 [%0], %1;" ::"l"(base + off), "r"(inc) : "memory");
  else
    asm volatile("red.shared.add.u32 [%0], %1;" ::"r"((uint32_t)base + off), "r"(inc) : "memory");
}

template <int MODE>
__device__ __forceinline__ void hist16_z8(uint64_t slot, uint4 yv, uint4 zv, uint32_t bs,
                                          uint32_t hb) {
  const uint32_t ys[4] = {yv.x, yv.y, yv.z, yv.w};
  const uint32_t zs[4] = {zv.x, zv.y, zv.z, zv.w};
#pragma unroll
  for (int w = 0; w < 4; ++w) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t y = __byte_perm(ys[w], 0, 0x4440 + b);
      const uint32_t z = __byte_perm(zs[w], 0, 0x4440 + b);
      hist_add<MODE>(slot, z, y, bs, hb);
    }
  }
}

// Same for a group whose target states were sorted at staging (sort_state_groups):
// zv holds the states in ascending order and pm the sample each came from (nibble
// j: original position of sorted entry j), so the source's 16 bytes are put in
// the same order with three byte permutes per four samples. At each step the
// warp's lanes then hold states of similar rank, whose cells spread over fewer
// distinct words per bank than cells of unrelated states. The counts do not
// depend on the order of the samples.
template <int MODE>
__device__ __forceinline__ void hist16_z8_sorted(uint64_t slot, uint4 yv, uint4 zv, uint2 pm,
                                                 uint32_t bs, uint32_t hb) {
  const uint32_t zs[4] = {zv.x, zv.y, zv.z, zv.w};
  uint32_t ys[4];
#pragma unroll
  for (int w = 0; w < 4; ++w) {
    const uint32_t nib = ((w < 2 ? pm.x : pm.y) >> (16 * (w & 1))) & 0xffffu;
    const uint32_t sa = nib & 0x7777u;                   // byte within 8 of the pair
    const uint32_t sb = 0x3210u | ((nib & 0x8888u) >> 1);  // low (i) or high (i + 4) pair
    const uint32_t lo = __byte_perm(yv.x, yv.y, sa);
    const uint32_t hi = __byte_perm(yv.z, yv.w, sa);
    ys[w] = __byte_perm(lo, hi, sb);
  }
#pragma unroll
  for (int w = 0; w < 4; ++w) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t y = __byte_perm(ys[w], 0, 0x4440 + b);
      const uint32_t z = __byte_perm(zs[w], 0, 0x4440 + b);
      hist_add<MODE>(slot, z, y, bs, hb);
    }
  }
}

template <int MODE>
__device__ __forceinline__ void hist16_z16(uint64_t slot, uint4 yv, uint4 za, uint4 zb,
                                           uint32_t bs, uint32_t hb) {
  const uint32_t ys[4] = {yv.x, yv.y, yv.z, yv.w};
  const uint32_t zs[8] = {za.x, za.y, za.z, za.w, zb.x, zb.y, zb.z, zb.w};
#pragma unroll
  for (int w = 0; w < 4; ++w) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t y = __byte_perm(ys[w], 0, 0x4440 + b);
      const uint32_t zw = zs[(w * 4 + b) >> 1];
      const uint32_t z = (b & 1) ? (zw >> 16) : (zw & 0xffffu);
      hist_add<MODE>(slot, z, y, bs, hb);
    }
  }
}

// Histogram of one source against the staged target over n samples (all group
// lanes): zsm[i] is the target state of sample i of srow (both 16-byte aligned).
template <int MODE>
__device__ __forceinline__ void hist_source(uint64_t slot32, const unsigned char* zsm, bool z8,
                                            const uint2* zperm, const uint8_t* srow, int n,
                                            int lane_g, int gthreads, uint32_t bs, uint32_t hb) {
  const int nvec = n >> 4;
  const uint4* yv = reinterpret_cast<const uint4*>(srow);
  const uint4* zv = reinterpret_cast<const uint4*>(zsm);
  int v = lane_g;
  if (z8) {
    if (v < nvec && zperm != nullptr) {
      uint4 ycur = dev::ldg_nc_v4(yv + v);
      for (; v < nvec; v += gthreads) {
        const int vn = v + gthreads;
        uint4 ynext = ycur;
        if (vn < nvec) ynext = dev::ldg_nc_v4(yv + vn);
        hist16_z8_sorted<MODE>(slot32, ycur, zv[v], zperm[v], bs, hb);
        ycur = ynext;
      }
    } else if (v < nvec) {
      uint4 ycur = dev::ldg_nc_v4(yv + v);
      for (; v < nvec; v += gthreads) {
        const int vn = v + gthreads;
        uint4 ynext = ycur;
        if (vn < nvec) ynext = dev::ldg_nc_v4(yv + vn);
        hist16_z8<MODE>(slot32, ycur, zv[v], bs, hb);
        ycur = ynext;
      }
    }
    for (int s = (nvec << 4) + lane_g; s < n; s += gthreads)
      hist_add<MODE>(slot32, zsm[s], srow[s], bs, hb);
  } else {
    const uint16_t* z16 = reinterpret_cast<const uint16_t*>(zsm);
    if (v < nvec) {
      uint4 ycur = dev::ldg_nc_v4(yv + v);
      for (; v < nvec; v += gthreads) {
        const int vn = v + gthreads;
        uint4 ynext = ycur;
        if (vn < nvec) ynext = dev::ldg_nc_v4(yv + vn);
        hist16_z16<MODE>(slot32, ycur, zv[2 * v], zv[2 * v + 1], bs, hb);
        ycur = ynext;
      }
    }
    for (int s = (nvec << 4) + lane_g; s < n; s += gthreads)
      hist_add<MODE>(slot32, z16[s], srow[s], bs, hb);
  }
}

__device__ __forceinline__ void group_sync(int G, int g, int gthreads) {
  if (G == 1) __syncwarp();
  else dev::named_bar(1 + g, gthreads);
}

// Whether pair (bt, bs) fits one group's shared-memory slot of slot_region bytes
// (32-bit counters, or 16-bit halves when N < 65536); pairs that do not go to
// the global-memory overflow launch. Same rule on host and device.
__host__ __device__ inline bool slot_fits(int64_t bt, int64_t bs, int N, int64_t slot_region) {
  const int64_t w32 = round_up(bt * bt * bs, 4);
  if (w32 * 4 <= slot_region) return true;
  const int64_t w16 = round_up(bt * bt * ((bs + 1) / 2), 4);
  return N < 65536 && w16 * 4 <= slot_region;
}

// Whether pair (bt, bs) runs in the shared-memory launch: its histogram fits a
// slot and the target's marginal tables fit shared memory (bt <= mbmax). Every
// other pair runs in the overflow launch. Same rule on host and device, and
// monotone in bs, so sources sorted by b split each target's chunk in one place.
__host__ __device__ inline bool in_smem(int64_t bt, int64_t bs, int N, int mbmax,
                                        int64_t slot_region) {
  return bt <= mbmax && slot_fits(bt, bs, N, slot_region);
}

// Per-lane part of sum c3 * log2(c3 * c1 / (c2a * c2b)) over the pair's cells.
// Cell (z = xt1*bt + xt, y) is tab[z * stride + y] (PACK16: the 16-bit half
// (y & 1) of word z * stride + (y >> 1)); stride >= the row's words (padding
// words stay zero). Columns (xt, y) are
// spread over the group's lanes; CLEAR zeroes every word after reading it.
// term = c3 * log2(c3 * c1 / (c2a * c2b)), the ratio formed as
// c3 * (1/c2b) * (c1/c2a) (one reciprocal per column, c1/c2a staged per target)
// except where c3 * c1 == c2a * c2b, whose term is exactly 0 as in the
// reference's formula (constant or duplicated sources give TE = 0, not a
// rounding residue). Empty cells take log2(1) = 0 (no branch).
template <bool PACK16, bool CLEAR>
__device__ __forceinline__ float entropy_cols(uint32_t* tab, int bt, int bs, int stride,
                                              const int* c1i, const float2* qa, int lane_g,
                                              int gthreads) {
  float acc = 0.f;
  // every word of a row, padding included (zero, so skipped by the s == 0 test):
  // consecutive lanes then read consecutive words, one wavefront per warp
  const int ncy = stride;
  const int ncols = bt * ncy;
  for (int col = lane_g; col < ncols; col += gthreads) {
    const int j = col / ncy;
    const int wk = col - j * ncy;
    uint32_t s = 0;
    for (int i = 0; i < bt; ++i) s += tab[(i * bt + j) * stride + wk];
    if (s == 0u) continue;
    const float c1j = (float)c1i[j];
    if (PACK16) {
      const float blo = (float)(s & 0xffffu), bhi = (float)(s >> 16);
      const float inv_lo = __frcp_rn(blo), inv_hi = __frcp_rn(bhi);
      for (int i = 0; i < bt; ++i) {
        const int idx = (i * bt + j) * stride + wk;
        const uint32_t w = tab[idx];
        if (CLEAR) tab[idx] = 0u;
        const float2 q = qa[i * bt + j];  // {c1/c2a, c2a}
        const float clo = (float)(w & 0xffffu), chi = (float)(w >> 16);
        const bool elo = clo == 0.f || clo * c1j == q.y * blo;
        const bool ehi = chi == 0.f || chi * c1j == q.y * bhi;
        const float rlo = elo ? 1.f : clo * inv_lo * q.x;
        const float rhi = ehi ? 1.f : chi * inv_hi * q.x;
        acc = fmaf(clo, __log2f(rlo), acc);
        acc = fmaf(chi, __log2f(rhi), acc);
      }
    } else {
      const float b = (float)s;
      const float inv = __frcp_rn(b);
      for (int i = 0; i < bt; ++i) {
        const int idx = (i * bt + j) * stride + wk;
        const uint32_t w = tab[idx];
        if (CLEAR) tab[idx] = 0u;
        const float2 q = qa[i * bt + j];
        const float c = (float)w;
        const bool e = w == 0u || c * c1j == q.y * b;
        const float r = e ? 1.f : c * inv * q.x;
        acc = fmaf(c, __log2f(r), acc);
      }
    }
  }
  return acc;
}

// Same sum for series of 2^24 samples or more, in float64 from the integer
// counts (32-bit counters only; the zero-term test on exact 64-bit products).
template <bool CLEAR>
__device__ double entropy_cols_f64(uint32_t* tab, int bt, int bs, int stride, const int* c1i,
                                   const int* c2ai, int lane_g, int gthreads) {
  double acc = 0.0;
  const int ncols = bt * stride;  // padding words included, as in entropy_cols
  for (int col = lane_g; col < ncols; col += gthreads) {
    const int j = col / stride;
    const int y = col - j * stride;
    uint64_t s = 0;
    for (int i = 0; i < bt; ++i) s += tab[(i * bt + j) * stride + y];
    if (s == 0u) continue;
    const uint64_t c1j = (uint64_t)(uint32_t)c1i[j];
    for (int i = 0; i < bt; ++i) {
      const int idx = (i * bt + j) * stride + y;
      const uint64_t c = tab[idx];
      if (CLEAR) tab[idx] = 0u;
      const uint64_t c2a = (uint64_t)(uint32_t)c2ai[i * bt + j];
      if (c == 0u || c * c1j == c2a * s) continue;
      acc += (double)c * log2(((double)c * (double)c1j) / ((double)c2a * (double)s));
    }
  }
  return acc;
}

// Everything a group needs about the current item.
struct ItemCtx {
  int tgt;
  int64_t lo, base;
  int n_src;
  int bt;
  bool z8;
  const unsigned char* zsm;
  const int* c1i;
  const int* c2ai;
  const float2* qa;
  double* red;
  int slot_region;    // shared-memory slot region (overflow split rule)
  bool pad;           // table rows at an odd stride (row words | 1)
  const uint2* zperm; // sorted 16-sample groups of 1-byte states, or nullptr
};

// Words per table row: b_s (32-bit counters) or (b_s + 1) / 2 (16-bit halves),
// made odd when the item's slots were carved at the padded size.
// The global-memory overflow launch never pads (its slots are sized b_max^3).
template <int MODE>
__device__ __forceinline__ uint32_t row_words(uint32_t bs, bool pad) {
  const uint32_t w = MODE == kSlot16 ? (bs + 1) >> 1 : bs;
  return (MODE != kGmem && pad) ? (w | 1u) : w;
}

// Source r of the item for this launch: its id and pair id, or false if the
// pair is not this launch's (the target itself, outside [p0, p1), or, with an
// overflow launch, on the other launch's side of the shared-memory fit rule).
template <int MODE>
__device__ __forceinline__ bool pair_of(const TeParams& P, const ItemCtx& it, int r, int* src_o,
                                        int64_t* p_o) {
  int64_t p;
  int src;
  if (P.pairs) {
    p = it.lo + r;
    src = (int)P.pairs[2 * p + 1];
  } else {
    src = P.order[it.lo + r];
    p = it.base + (src < it.tgt ? src : src - 1);
    if (src == it.tgt || p < P.p0 || p >= P.p1) return false;
  }
  if (P.overflow && in_smem(it.bt, P.npv[src], P.N, P.mbmax, it.slot_region) == (MODE == kGmem))
    return false;
  *src_o = src;
  *p_o = p;
  return true;
}

// Overflow launch (whole CTA on one pair, histogram in a global-memory slot),
// whole series staged: sum c3 * log2(c3 * c1 / (c2a * c2b)) from the pair's N
// samples instead of its b_t^2 * b_s cells (up to 16.4M at b = 254, with at most N
// of them nonzero). c2b is counted from the samples into the CTA's c2b scratch;
// then each sample claims its cell with an exchange against 0, so each nonzero
// cell is evaluated once (and the slot is left clear for the next pair); the terms
// (same expression and exact-zero rule as the cell pass) are summed in 2^-32 fixed
// point, so the total does not depend on which sample claimed a cell or on the
// order of the additions: bitwise reproducible. Returns the CTA's total.
__device__ double entropy_samples_gmem(uint32_t* tab, uint32_t* c2b, const unsigned char* zsm,
                                       bool z8, const uint8_t* srow, int N, int bt, int bs,
                                       const int* c1i, const float2* qa, int tid, int nthreads,
                                       double* red) {
  const uint16_t* z16 = reinterpret_cast<const uint16_t*>(zsm);
  for (int s = tid; s < N; s += nthreads) {
    const uint32_t z = z8 ? zsm[s] : z16[s];
    const uint32_t x0 = z % (uint32_t)bt;
    atomicAdd(&c2b[x0 * (uint32_t)bs + srow[s]], 1u);
  }
  __syncthreads();
  long long acc = 0;
  for (int s = tid; s < N; s += nthreads) {
    const uint32_t z = z8 ? zsm[s] : z16[s];
    const uint32_t y = srow[s];
    const uint32_t c = atomicExch(&tab[z * (uint32_t)bs + y], 0u);
    if (c == 0u) continue;
    const uint32_t x0 = z % (uint32_t)bt;
    const float b = (float)c2b[x0 * (uint32_t)bs + y];
    const float2 q = qa[z];  // {c1/c2a, c2a}
    const float cf = (float)c;
    const bool e = cf * (float)c1i[x0] == q.y * b;
    const float r = e ? 1.f : cf * __frcp_rn(b) * q.x;
    const float term = cf * __log2f(r);
    acc += __float2ll_rn(term * 4294967296.0f);  // |term| * 2^32 < 2^63 for N < 2^24
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  long long* red64 = reinterpret_cast<long long*>(red);
  if ((tid & 31) == 0) red64[tid >> 5] = acc;
  __syncthreads();
  long long tot = 0;
  for (int w = 0; w < (nthreads >> 5); ++w) tot += red64[w];
  // c2b back to zero for the next pair (b_t * b_s words)
  for (int i = tid; i < bt * bs; i += nthreads) c2b[i] = 0u;
  __syncthreads();
  return (double)tot * (1.0 / 4294967296.0);
}

// After the histogram of source src (pair id p) is complete in the group's
// table: optional raw-count export, the entropy pass and the output.
template <int MODE>
__device__ __forceinline__ void finish_pair(const TeParams& P, const ItemCtx& it, uint32_t* slot,
                                            int G, int g, int lane_g, int tid, int warp, int src,
                                            int64_t p, float obs_m) {
  const int gthreads = G * 32;
  const int bt = it.bt;
  const int bt2 = bt * bt;
  const int bs = P.npv[src];
  constexpr bool PACK16 = MODE == kSlot16;
  group_sync(G, g, gthreads);
  uint32_t* tab = slot;  // counts read by the entropy pass
  const int stride = (int)row_words<MODE>((uint32_t)bs, it.pad);

  // -- optional raw-count export (parity checks only) --------------------
  if (P.counts_dbg != nullptr) {
    int32_t* cd = P.counts_dbg + (p - P.p0) * P.counts_stride;
    const int ncell = bt2 * bs;
    for (int c = lane_g; c < ncell; c += gthreads) {
      const int z = c / bs, y = c - z * bs;
      cd[c] = (int32_t)(PACK16 ? cell_get<true>(tab, z, y, stride, stride)
                               : tab[z * stride + y]);
    }
    group_sync(G, g, gthreads);
  }

  // -- entropy pass (shared slots are cleared for the next source) ---------
  double tot;
  bool cta_total = false;  // tot already holds the whole CTA's sum
  if (MODE == kGmem && P.gc2b != nullptr && !P.big && P.ztile >= P.N) {
    tot = entropy_samples_gmem(tab, P.gc2b + (int64_t)blockIdx.x * P.gc2b_words, it.zsm, it.z8,
                               P.bins + (int64_t)src * P.ld, P.N, bt, bs, it.c1i, it.qa, tid,
                               G * 32, it.red);
    cta_total = true;
  } else if (P.big) {
    tot = dev::warp_sum(entropy_cols_f64<true>(tab, bt, bs, stride, it.c1i, it.c2ai, lane_g,
                                                gthreads));
  } else {
    tot = dev::warp_sum((double)entropy_cols<PACK16, true>(tab, bt, bs, stride, it.c1i, it.qa,
                                                            lane_g, gthreads));
  }
  if (G > 1 && !cta_total) {
    if ((tid & 31) == 0) it.red[warp] = tot;
    dev::named_bar(1 + g, gthreads);
    if (lane_g == 0) {
      tot = 0.0;
      for (int w = 0; w < G; ++w) tot += it.red[g * G + w];
    }
  }
  if (lane_g == 0) {
    const float te = (float)(tot / (double)P.N);
    if (P.out_mode == kOutPairfree) {
      P.out[p - P.p0] = te;
    } else if (P.out_mode == kOutMatrix) {
      P.out[(int64_t)src * P.out_ld + it.tgt] = te;
    } else {
      // one addend per cell per launch: reductions without a return value
      // (no load-to-store stall) give the same float64 sums as += would
      const int64_t m = (int64_t)src * P.n + it.tgt;
      const double td = (double)te;
      atomicAdd(P.sum + m, td);
      atomicAdd(P.sumsq + m, td * td);
      if (te >= obs_m) atomicAdd(P.cnt_ge + m, 1);
    }
  }
  group_sync(G, g, gthreads);
}

// Address of the group's table for hist_add.
template <int MODE>
__device__ __forceinline__ uint64_t table_addr(uint32_t* slot, int tid) {
  uint64_t a;
  if (MODE == kGmem) asm("cvta.to.global.u64 %0, %1;" : "=l"(a) : "l"(slot));
  else a = (uint64_t)__cvta_generic_to_shared(slot);
  return a;
}

// Stages target states of samples [s0, s0 + n) into zsm (all CTA threads);
// COUNT also adds them to the c2a counts.
// Sorts every full 16-sample group of 1-byte target states in place (ascending,
// ties by position) and records in perm[v] where each sorted entry came from
// (nibble j = original position of entry j). One thread per group: a bitonic
// network on keys state << 4 | position, in registers.
__device__ __forceinline__ void sort_state_groups(unsigned char* zsm, uint2* perm, int nvec,
                                                  int tid, int nthreads) {
  uint4* zv = reinterpret_cast<uint4*>(zsm);
  for (int v = tid; v < nvec; v += nthreads) {
    const uint4 q = zv[v];
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
    uint32_t k[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) k[i] = (((w[i >> 2] >> (8 * (i & 3))) & 0xffu) << 4) | i;
#pragma unroll
    for (int size = 2; size <= 16; size <<= 1) {
#pragma unroll
      for (int stride = size >> 1; stride > 0; stride >>= 1) {
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int j = i ^ stride;
          if (j > i) {
            const uint32_t a = k[i], b = k[j];
            const uint32_t lo = min(a, b), hi = max(a, b);
            const bool up = (i & size) == 0;
            k[i] = up ? lo : hi;
            k[j] = up ? hi : lo;
          }
        }
      }
    }
    uint32_t o[4] = {0u, 0u, 0u, 0u}, p0 = 0u, p1 = 0u;
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      o[i >> 2] |= (k[i] >> 4) << (8 * (i & 3));
      if (i < 8) p0 |= (k[i] & 15u) << (4 * i);
      else p1 |= (k[i] & 15u) << (4 * (i - 8));
    }
    zv[v] = make_uint4(o[0], o[1], o[2], o[3]);
    perm[v] = make_uint2(p0, p1);
  }
}

template <bool COUNT>
__device__ __forceinline__ void stage_z(const uint8_t* trow, int lag, int bt, bool z8, int s0,
                                        int n, unsigned char* zsm, int* c2ai, int tid,
                                        int nthreads) {
  if (z8) {
    for (int s = tid; s < n; s += nthreads) {
      const uint32_t z = (uint32_t)trow[s0 + s + lag] * bt + trow[s0 + s];
      zsm[s] = (unsigned char)z;
      if (COUNT) atomicAdd(&c2ai[z], 1);
    }
  } else {
    uint16_t* z16 = reinterpret_cast<uint16_t*>(zsm);
    for (int s = tid; s < n; s += nthreads) {
      const uint32_t z = (uint32_t)trow[s0 + s + lag] * bt + trow[s0 + s];
      z16[s] = (uint16_t)z;
      if (COUNT) atomicAdd(&c2ai[z], 1);
    }
  }
}

// One group's pass over its sources of the current item. Whole series staged
// (ztile == N): each group walks its sources on its own. Tiled: the CTA's
// groups take one source each per round and walk the sample tiles together.
template <int MODE>
__device__ __forceinline__ void run_sources(const TeParams& P, const ItemCtx& it, uint32_t* slot,
                                            unsigned char* zsm, int G, int g, int n_groups,
                                            int lane_g, int tid, int warp, int nthreads) {
  const int gthreads = G * 32;
  const int N = P.N;
  const uint64_t slot_addr = table_addr<MODE>(slot, tid);
  if (P.ztile >= N) {
    for (int r = g; r < it.n_src; r += n_groups) {
      int src;
      int64_t p;
      if (!pair_of<MODE>(P, it, r, &src, &p)) continue;  // group-uniform skip
      // surrogate statistics: the observed TE is loaded now, so its latency hides
      // behind the histogram pass instead of stalling the epilogue
      float obs_m = 0.f;
      if (P.out_mode == kOutStats && lane_g == 0) obs_m = __ldg(P.obs + (int64_t)src * P.n + it.tgt);
      const uint32_t rw = row_words<MODE>((uint32_t)P.npv[src], it.pad);
      hist_source<MODE>(slot_addr, it.zsm, it.z8, it.zperm, P.bins + (int64_t)src * P.ld, N,
                        lane_g, gthreads, rw, rw);
      finish_pair<MODE>(P, it, slot, G, g, lane_g, tid, warp, src, p, obs_m);
    }
    return;
  }
  const uint8_t* trow = P.bins + (int64_t)it.tgt * P.ld;
  for (int r0 = 0; r0 < it.n_src; r0 += n_groups) {
    int src = 0;
    int64_t p = 0;
    const bool act = r0 + g < it.n_src && pair_of<MODE>(P, it, r0 + g, &src, &p);
    float obs_m = 0.f;
    if (act && P.out_mode == kOutStats && lane_g == 0)
      obs_m = __ldg(P.obs + (int64_t)src * P.n + it.tgt);
    const uint32_t rw = row_words<MODE>(act ? (uint32_t)P.npv[src] : 1u, it.pad);
    const uint8_t* srow = P.bins + (int64_t)src * P.ld;
    for (int s0 = 0; s0 < N; s0 += P.ztile) {
      const int n = min(P.ztile, N - s0);
      __syncthreads();  // every group is done with the previous tile
      stage_z<false>(trow, P.lag, it.bt, it.z8, s0, n, zsm, nullptr, tid, nthreads);
      __syncthreads();
      if (act)
        hist_source<MODE>(slot_addr, zsm, it.z8, nullptr, srow + s0, n, lane_g, gthreads, rw, rw);
    }
    if (act) finish_pair<MODE>(P, it, slot, G, g, lane_g, tid, warp, src, p, obs_m);
  }
}

}  // namespace

// GMEM = false: the shared-memory launch; true: the global-memory overflow launch
// (separate code, so the common kernel carries none of the overflow path).
template <bool GMEM>
__global__ void __launch_bounds__(1024, 1) te_pair_tile_kernel(TeParams P) {
  extern __shared__ __align__(16) unsigned char smem[];
  const SmemLayout SL = smem_layout(P.ztile, P.zbytes, P.bmax, P.mbmax);
  int* misc = reinterpret_cast<int*>(smem + SL.misc_off);
  double* red = reinterpret_cast<double*>(smem + SL.red_off);
  int* c1i = reinterpret_cast<int*>(smem + SL.c1_off);
  int* const c2a_sm = reinterpret_cast<int*>(smem + SL.c2a_off);
  float2* const qa_sm = reinterpret_cast<float2*>(smem + SL.q_off);
  // a target beyond mbmax (overflow launch only) keeps its tables in this CTA's
  // global scratch: c2a (bmax^2 ints), then {c1/c2a, c2a} (bmax^2 float2)
  int* const c2a_gm = GMEM && P.gmarg ? P.gmarg + (int64_t)blockIdx.x * P.gmarg_words : nullptr;
  float2* const qa_gm =
      c2a_gm ? reinterpret_cast<float2*>(c2a_gm + 2 * (((int64_t)P.bmax * P.bmax + 1) / 2))
             : nullptr;
  unsigned char* zsm = smem + SL.z_off;
  uint32_t* slots = reinterpret_cast<uint32_t*>(smem + SL.slot_off);
  const int slot_region = P.smem_bytes - SL.slot_off;

  const int tid = threadIdx.x;
  const int nthreads = blockDim.x;
  const int warp = tid >> 5;
  const int n_warps = nthreads >> 5;
  const int nm1 = P.n - 1;
  const int N = P.N;
  const bool tiled = P.ztile < N;

  if (*(volatile int*)&P.ws->bad_data != 0) return;  // validation failed: do nothing
  uint32_t* gslot = GMEM ? P.gslots + (int64_t)blockIdx.x * P.gslot_words : nullptr;
  if (GMEM) {
    for (int64_t i = tid; i < P.gslot_words; i += nthreads) gslot[i] = 0u;
    if (P.gc2b)
      for (int64_t i = tid; i < P.gc2b_words; i += nthreads)
        P.gc2b[(int64_t)blockIdx.x * P.gc2b_words + i] = 0u;
    __syncthreads();
  }

  for (;;) {
    if (tid == 0) misc[0] = (int)atomicAdd(GMEM ? &P.ws->ov_ticket : &P.ws->ticket, 1u);
    __syncthreads();
    const int64_t q = (int64_t)misc[0];
    if (q >= P.n_items) break;
    int tgt;
    int64_t lo, hi, base = 0;
    if (P.pairs) {
      lo = P.item_start[q];
      hi = P.item_start[q + 1];
      if (lo < 0 || hi > P.p1 || lo > hi) {  // malformed item table: skip, report
        if (tid == 0) atomicExch(&P.ws->bad_data, 2);
        __syncthreads();
        continue;
      }
      tgt = lo < hi ? (int)P.pairs[2 * lo] : 0;
    } else {
      // pair-free: chunk `chunk` covers positions [chunk*W, (chunk+1)*W) of the
      // source order (genes grouped by bin count, so one item's histogram slots
      // are sized for sources of similar b); sources outside [p0, p1) or equal
      // to the target are skipped below
      // Item order: targets in blocks of tblock rows (sized to stay in L2); within
      // a block, chunk-major, so one source chunk is shared by the CTAs resident
      // at one moment and the block's target rows are re-read from L2, not HBM.
      const int64_t per_block = (int64_t)P.tblock * P.n_chunks;
      const int blk = (int)(q / per_block);
      const int tb0 = blk * P.tblock;
      const int tbs = min(P.tblock, P.n_targets - tb0);
      const int64_t rem = q - (int64_t)blk * per_block;
      const int chunk = (int)(rem / tbs);
      tgt = P.t_first + tb0 + (int)(rem - (int64_t)chunk * tbs);
      base = (int64_t)tgt * nm1;
      lo = (int64_t)chunk * P.W;
      hi = min((int64_t)(chunk + 1) * P.W, (int64_t)P.n);
      if (base + nm1 <= P.p0 || base >= P.p1) lo = hi;  // target outside the range
      // sources are sorted by bin count: skip a chunk this launch has no pair of
      if (P.overflow && lo < hi) {
        const int btq = P.npv[tgt];
        if (!GMEM && !in_smem(btq, P.npv[P.order[lo]], N, P.mbmax, slot_region)) lo = hi;
        if (GMEM && in_smem(btq, P.npv[P.order[hi - 1]], N, P.mbmax, slot_region)) lo = hi;
      }
    }
    if (lo >= hi) {
      __syncthreads();
      continue;
    }
    const int n_src = (int)(hi - lo);
    if (P.pairs && (tgt < 0 || tgt >= P.n)) {
      if (tid == 0) atomicExch(&P.ws->bad_data, 2);
      __syncthreads();
      continue;
    }
    const int bt = P.npv[tgt];
    const int bt2 = bt * bt;
    // the target's marginal tables: shared memory, or (bt > mbmax: every pair of
    // this target is an overflow pair) the CTA's global scratch
    int* const c2ai = bt <= P.mbmax ? c2a_sm : c2a_gm;
    float2* const qa = bt <= P.mbmax ? qa_sm : qa_gm;

    // ---- max b_s over this launch's sources (pair lists: also check indices) --
    unsigned my_max = 1;
    int mine = 0;
    bool bad = tgt < 0 || tgt >= P.n;
    for (int r = tid; r < n_src; r += nthreads) {
      int src;
      if (P.pairs) {
        src = (int)P.pairs[2 * (lo + r) + 1];
        bad |= P.pairs[2 * (lo + r)] != tgt || src < 0 || src >= P.n;
        if (src < 0 || src >= P.n) src = 0;
      } else {
        src = P.order[lo + r];
        const int64_t p = base + (src < tgt ? src : src - 1);
        if (src == tgt || p < P.p0 || p >= P.p1) continue;
      }
      const int bsrc = P.npv[src];
      if (!bad && P.overflow && in_smem(bt, bsrc, N, P.mbmax, slot_region) == GMEM) continue;
      my_max = max(my_max, (unsigned)bsrc);
      mine = 1;
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0) atomicExch(&P.ws->bad_data, 2);
      __syncthreads();
      continue;
    }
    if (P.overflow && !__syncthreads_or(mine)) continue;  // no pair of this launch (uniform)
    my_max = dev::warp_max(my_max);
    if ((tid & 31) == 0) reinterpret_cast<unsigned*>(red)[warp] = my_max;
    for (int i = tid; i < bt2; i += nthreads) c2ai[i] = 0;
    __syncthreads();
    if (tid < 32) {
      unsigned v = tid < n_warps ? reinterpret_cast<unsigned*>(red)[tid] : 1u;
      v = dev::warp_max(v);
      if (tid == 0) misc[1] = (int)v;
    }

    // ---- the target: z[s] = x[s+lag]*bt + x[s] staged (whole series) and the
    // c2a counts (tiled series: counted here, staged tile by tile later) ------
    const uint8_t* trow = P.bins + (int64_t)tgt * P.ld;
    const bool z8 = bt <= 16;
    if (!tiled) {
      stage_z<true>(trow, P.lag, bt, z8, 0, N, zsm, c2ai, tid, nthreads);
    } else {
      for (int s = tid; s < N; s += nthreads)
        atomicAdd(&c2ai[(uint32_t)trow[s + P.lag] * bt + trow[s]], 1);
    }
    __syncthreads();
    // 1-byte states of a whole staged series in a region sized for 2-byte ones:
    // the spare half holds the permutation of each 16-sample group sorted by
    // state (the shared-memory launch only; the overflow launch's entropy pass
    // pairs zsm[s] with sample s of the source)
    const uint2* zperm = nullptr;
    if (!GMEM && z8 && !tiled && P.zbytes == 2 && N >= 16) {
      uint2* pm = reinterpret_cast<uint2*>(zsm + round_up((int64_t)N, 16));
      sort_state_groups(zsm, pm, N >> 4, tid, nthreads);
      zperm = pm;
      __syncthreads();
    }
    const int bsmax = misc[1];
    for (int j = tid; j < bt; j += nthreads) {
      int s = 0;
      for (int i = 0; i < bt; ++i) s += c2ai[i * bt + j];
      c1i[j] = s;
    }

    // ---- carve slots: 32-bit counters when groups of <= 4 warps fit --------
    // (the overflow launch: the whole CTA on one 32-bit slot in global memory)
    const int words32 = (int)round_up((int64_t)bt2 * bsmax, 4);
    const int words16 = (int)round_up((int64_t)bt2 * ((bsmax + 1) >> 1), 4);
    const int fit32 = GMEM ? 1 : slot_region / (words32 * 4);
    const int fit16 = GMEM ? 0 : slot_region / (words16 * 4);
    const bool pack16 = !GMEM && (N < 65536) && fit32 * 4 < n_warps && fit16 >= 1;
    const int fit = pack16 ? fit16 : fit32;
    int slot_words = pack16 ? words16 : words32;
    if (fit < 1) {
      if (tid == 0) atomicExch(&P.ws->bad_item, 1);
      __syncthreads();
      continue;
    }
    int G = 1;
    while (n_warps / G > fit) G <<= 1;
    while (G > 1 && G < n_warps && n_warps / G > 15) G <<= 1;
    const int n_groups = n_warps / G;
    // odd row stride where the same groups' slots still fit at the padded size
    // (the group size and the counter width stay as chosen above)
    bool pad = false;
    if (!GMEM) {
      const int64_t rw = pack16 ? ((((int64_t)bsmax + 1) >> 1) | 1) : ((int64_t)bsmax | 1);
      const int padded = (int)round_up((int64_t)bt2 * rw, 4);
      if ((int64_t)n_groups * padded * 4 <= slot_region) {
        slot_words = padded;
        pad = true;
      }
    }
    const int g = warp / G;
    const int lane_g = tid - g * G * 32;
    uint32_t* slot = GMEM ? gslot : slots + (int64_t)g * slot_words;
    if (!GMEM)
      for (int i = tid; i < n_groups * slot_words; i += nthreads) slots[i] = 0u;
    __syncthreads();
    for (int z = tid; z < bt2; z += nthreads) {
      const float c2a = (float)c2ai[z];
      qa[z] = make_float2(c2a > 0.f ? __fdiv_rn((float)c1i[z % bt], c2a) : 0.f, c2a);
    }
    __syncthreads();

    ItemCtx it;
    it.tgt = tgt;
    it.lo = lo;
    it.base = base;
    it.n_src = n_src;
    it.bt = bt;
    it.z8 = z8;
    it.zsm = zsm;
    it.c1i = c1i;
    it.c2ai = c2ai;
    it.qa = qa;
    it.red = red;
    it.slot_region = slot_region;
    it.pad = pad;
    it.zperm = zperm;
    if (GMEM)
      run_sources<kGmem>(P, it, slot, zsm, G, g, n_groups, lane_g, tid, warp, nthreads);
    else if (pack16)
      run_sources<kSlot16>(P, it, slot, zsm, G, g, n_groups, lane_g, tid, warp, nthreads);
    else
      run_sources<kSlot32>(P, it, slot, zsm, G, g, n_groups, lane_g, tid, warp, nthreads);
    __syncthreads();
  }
}

// Per-gene pre-pass: validation (every bin of gene g in [0, row_len) below
// n_per_var[g], and 1 <= n_per_var[g] <= b_max; sets ws->bad_data otherwise).
// One CTA per gene.
__global__ void gene_prepass_kernel(const uint8_t* bins, int64_t ld, const int32_t* npv,
                                    int b_max, int n, int64_t row_len, WsHeader* ws) {
  const int g = blockIdx.x;
  if (g >= n) return;
  const int b = npv[g];
  const uint8_t* row = bins + (int64_t)g * ld;
  const int64_t nvec = row_len >> 4;
  bool bad = b < 1 || b > b_max;
  const uint4* rv = reinterpret_cast<const uint4*>(row);
  for (int64_t v = threadIdx.x; v < nvec; v += blockDim.x) {
    const uint4 q = __ldg(rv + v);
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
      for (int bb = 0; bb < 4; ++bb) bad |= ((w[k] >> (8 * bb)) & 0xffu) >= (uint32_t)b;
  }
  for (int64_t i = (nvec << 4) + threadIdx.x; i < row_len; i += blockDim.x) bad |= row[i] >= b;
  if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(&ws->bad_data, 1);
}

// Source order for pair-free items: genes stably sorted by bin count, so a work
// item's sources have similar b (its histogram slots are sized for them) and the
// pairs that overflow shared memory form a suffix of every target's order. One CTA of 1024 threads;
// deterministic (ballot + block scan, no atomics on the order).
__device__ __forceinline__ int order_class(int b) {
  return b < 0 ? 0 : (b > 255 ? 255 : b);  // out-of-range counts (rejected later) stay in bounds
}

__global__ void __launch_bounds__(1024) source_order_kernel(const int32_t* __restrict__ npv,
                                                            int n, int32_t* __restrict__ order) {
  constexpr int kClasses = 256;
  __shared__ int present[kClasses];
  __shared__ int wsum[32];
  __shared__ int base_sh;
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5, nw = blockDim.x >> 5;
  for (int c = tid; c < kClasses; c += blockDim.x) present[c] = 0;
  if (tid == 0) base_sh = 0;
  __syncthreads();
  for (int g = tid; g < n; g += blockDim.x) present[order_class(npv[g])] = 1;
  __syncthreads();
  for (int c = 0; c < kClasses; ++c) {
    if (!present[c]) continue;  // uniform: read after the barrier above
    for (int start = 0; start < n; start += blockDim.x) {
      const int g = start + tid;
      const int flag = (g < n) && order_class(npv[g]) == c;
      const unsigned m = __ballot_sync(0xffffffffu, flag);
      const int pre = __popc(m & ((1u << lane) - 1u));
      if (lane == 0) wsum[w] = __popc(m);
      __syncthreads();
      int wpre = 0, tot = 0;
      for (int k = 0; k < nw; ++k) {
        const int v = wsum[k];
        wpre += k < w ? v : 0;
        tot += v;
      }
      const int b0 = base_sh;
      if (flag) order[b0 + wpre + pre] = g;
      __syncthreads();
      if (tid == 0) base_sh = b0 + tot;
      __syncthreads();
    }
  }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

struct TeLaunch {
  int threads, grid, smem;
};

// Samples of the target staged in shared memory at a time: the whole series
// when its states take at most 64 KB (10,000-20,000 samples of u16 states, any
// series up to 65,536 samples of u8 states), else tiles of 32 KB, which leave
// the histograms room for every bin count the coarsening limit allows.
static int z_tile(int N, int zbytes) {
  if ((int64_t)N * zbytes <= 65536) return N;
  return 32768 / zbytes;
}

static int plan_te_launch(const TeParams& P, const tenex_te_config* cfg, const DevAttr& A,
                          TeLaunch* L, int64_t max_slot_bytes) {
  // Default shape: 2 CTAs x 512 threads per SM. When the largest histogram needs
  // the shared memory of a whole SM (b_max ~ 32 and above) the loop below drops
  // to one CTA per SM; with both left to the library the CTA then takes 1024
  // threads, so an SM keeps 32 warps (10,000 genes x 20,000 cells, b_max 38:
  // 989 ms against 1055 ms for one 512-thread CTA).
  const bool auto_shape = !(cfg && (cfg->threads || cfg->ctas_per_sm));
  int threads = (cfg && cfg->threads) ? cfg->threads : 512;
  int cps = (cfg && cfg->ctas_per_sm) ? cfg->ctas_per_sm : 2;  // lowered below if slots do not fit
  if (threads != 128 && threads != 256 && threads != 512 && threads != 1024)
    return fail(TENEX_ERR_BADARG, "threads must be 128, 256, 512 or 1024 (got %d)", threads);
  if (cps < 1 || cps * threads > A.max_threads_per_sm)
    return fail(TENEX_ERR_BADARG, "ctas_per_sm=%d x threads=%d exceeds %d threads/SM", cps,
                threads, A.max_threads_per_sm);
  const int fixed = (cfg && cfg->smem_bytes) ? cfg->smem_bytes : 0;
  if (fixed > A.smem_optin)
    return fail(TENEX_ERR_BADARG, "smem_bytes=%d exceeds the device opt-in %d", fixed,
                A.smem_optin);
  const SmemLayout SL = smem_layout(P.ztile, P.zbytes, P.bmax, P.mbmax);
  int smem = 0;
  // With shared memory sized automatically, fewer CTAs per SM are used when the
  // largest pair's histogram would not fit (e.g. 38-bin genes need ~110 KB).
  // Pairs that still do not fit at one CTA per SM go to the global-memory
  // overflow launch (te_run).
  for (;; --cps) {
    smem = fixed ? fixed : std::min((A.smem_per_sm / cps) - 1024, A.smem_optin);
    smem = smem / 16 * 16;
    if ((int64_t)SL.slot_off + max_slot_bytes <= smem) break;
    if (fixed || cps == 1) break;
  }
  if (auto_shape && cps == 1) threads = std::min(1024, A.max_threads_per_sm);
  if ((int64_t)SL.slot_off + 1024 > smem)
    return fail(TENEX_ERR_UNSUPPORTED,
                "the target block (%d B of shared memory: marginals for b up to %d and %d "
                "staged samples) leaves no room for histograms in %d B; coarsen the bins",
                SL.slot_off, P.mbmax, P.ztile, smem);
  L->threads = threads;
  L->smem = smem;
  L->grid = A.sm_count * cps;
  return TENEX_OK;
}

// Shared memory one CTA per SM can have (the planner's largest choice).
static int smem_one_cta(const DevAttr& A) {
  return std::min(A.smem_per_sm - 1024, A.smem_optin) / 16 * 16;
}

// Largest target b whose marginal tables stay in shared memory: b_max when the
// target block with tables for b_max leaves at least 1 KB for histograms (the
// shared-memory kernel's own limit), else the largest b that leaves 64 KB. Targets
// above it (coarsening off, b in the hundreds) run all their pairs in the overflow
// launch with the tables in global memory.
static int marginal_bound(int b_max, int ztile, int zbytes, int smem_max) {
  if (smem_layout(ztile, zbytes, b_max, b_max).slot_off + 1024 <= smem_max) return b_max;
  for (int b = b_max - 1; b > 1; --b)
    if (smem_layout(ztile, zbytes, b_max, b).slot_off + 65536 <= smem_max) return b;
  return 1;
}

// Per-CTA global scratch of the overflow launch for a target's marginal tables:
// c2a (b_max^2 ints, padded to an even count) then {c1/c2a, c2a} (b_max^2 float2).
static int64_t gmarg_words(int b_max) {
  const int64_t b2 = (int64_t)b_max * b_max;
  return round_up(2 * ((b2 + 1) / 2) + 2 * b2, 4);
}

// Per-CTA c2b scratch of the overflow launch (b_max^2 counts, 16-byte rows of CTAs).
static int64_t gc2b_words(int b_max) { return round_up((int64_t)b_max * b_max, 4); }

// Whether some pair needs the overflow launch: the largest pair's histogram does
// not fit a slot, or the largest target's tables do not fit shared memory.
static bool needs_overflow(int b_max, int N, int zbytes, int mbmax, int smem) {
  const SmemLayout SL = smem_layout(z_tile(N, zbytes), zbytes, b_max, mbmax);
  return b_max > mbmax || !slot_fits(b_max, b_max, N, (int64_t)smem - SL.slot_off);
}

// Global-memory overflow slots (bytes, 0 if no pair needs the overflow launch): one
// b_max^3 32-bit slot per overflow CTA, as many CTAs as fit 4 GiB (at least one, at
// most one per SM: every SM up to b_max = 160, 64 CTAs at b_max = 254), and when
// targets exceed the marginal bound, each CTA's scratch for their tables.
static int64_t gmem_slot_count(int b_max, const DevAttr& A) {
  const int64_t words = (int64_t)b_max * b_max * b_max;
  return std::max<int64_t>(1, std::min<int64_t>(A.sm_count, ((int64_t)4 << 30) / (words * 4)));
}
static int64_t gmem_bytes(int b_max, int N, int zbytes, const DevAttr& A) {
  const int smem = smem_one_cta(A);
  const int mb = marginal_bound(b_max, z_tile(N, zbytes), zbytes, smem);
  if (!needs_overflow(b_max, N, zbytes, mb, smem)) return 0;
  const int64_t ns = gmem_slot_count(b_max, A);
  const int64_t marg = mb < b_max ? ns * gmarg_words(b_max) * 4 : 0;
  return round_up(ns * (int64_t)b_max * b_max * b_max * 4, 256) + round_up(marg, 256) +
         round_up(ns * gc2b_words(b_max) * 4, 256);
}

}  // namespace tenex

using namespace tenex;

// Launch shape the histogram kernels would use on the current device for series
// of row_len samples at this lag and b_max, with cfg as given (NULL or 0 fields:
// the defaults): threads per CTA, CTAs per SM, dynamic shared memory per CTA and
// sources per item. Computed by the same planner as the launches.
extern "C" int tenex_te_launch_shape(int64_t row_len, int64_t lag, int b_max,
                                     const tenex_te_config* cfg, int* threads, int* ctas_per_sm,
                                     int* smem_bytes, int* src_chunk) {
  if (!threads || !ctas_per_sm || !smem_bytes || !src_chunk)
    return fail(TENEX_ERR_BADARG, "output pointers must be non-NULL");
  if (lag < 1 || row_len <= lag) return fail(TENEX_ERR_BADARG, "need 1 <= lag < row_len");
  if (row_len >= ((int64_t)1 << 31))
    return fail(TENEX_ERR_UNSUPPORTED, "row_len = %lld samples (must be < 2^31)",
                (long long)row_len);
  if (b_max < 1 || b_max > 255) return fail(TENEX_ERR_BADARG, "b_max must be in 1..255");
  DevAttr A;
  int st = current_device_attr(&A);
  if (st) return st;
  TeParams P{};
  P.N = (int)(row_len - lag);
  P.bmax = b_max;
  P.zbytes = b_max <= 16 ? 1 : 2;
  P.ztile = z_tile(P.N, P.zbytes);
  P.mbmax = marginal_bound(b_max, P.ztile, P.zbytes, smem_one_cta(A));
  const int64_t hb = P.N < 65536 ? (b_max + 1) / 2 : b_max;
  const int64_t worst_slot = round_up((int64_t)b_max * b_max * hb, 4) * 4;
  TeLaunch L{};
  if ((st = plan_te_launch(P, cfg, A, &L, worst_slot))) return st;
  *threads = L.threads;
  *ctas_per_sm = L.grid / A.sm_count;
  *smem_bytes = L.smem;
  *src_chunk = (cfg && cfg->src_chunk) ? cfg->src_chunk : 512;
  return TENEX_OK;
}

extern "C" size_t tenex_te_workspace_bytes(int n_vars, int64_t row_len, int b_max) {
  if (n_vars < 1 || b_max < 1) return sizeof(WsHeader);
  size_t total = (size_t)ws_total(n_vars, b_max);
  DevAttr A;
  if (row_len > 1 && row_len < ((int64_t)1 << 31) && current_device_attr(&A) == TENEX_OK)
    total += (size_t)gmem_bytes(b_max, (int)row_len, b_max <= 16 ? 1 : 2, A);
  return total;
}

extern "C" int tenex_workspace_status(const void* workspace, void* stream) {
  if (!workspace) return fail(TENEX_ERR_BADARG, "workspace is NULL");
  WsHeader h;
  cudaError_t e = cudaMemcpyAsync(&h, workspace, sizeof(h), cudaMemcpyDeviceToHost,
                                  as_stream(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
  if (e != cudaSuccess) return check_cuda(e, "tenex_workspace_status");
  if (h.bad_data == 2)
    return fail(TENEX_ERR_BADDATA,
                "a pair-list item mixed targets or held an index outside [0, n_vars); those "
                "pairs were not computed");
  if (h.bad_data)
    return fail(TENEX_ERR_BADDATA,
                "a bin value was >= its gene's n_per_var, or n_per_var was outside [1, b_max]; "
                "no TE was computed");
  if (h.bad_item) return fail(TENEX_ERR_UNSUPPORTED,
                              "a work item's histogram did not fit shared memory");
  return TENEX_OK;
}

// Common driver of the TE entry points. pairs/item_start/n_items select the
// pair-list mode (then p0 must be 0 and n_pairs the list length).
static int te_run(const uint8_t* bins, int64_t ld, const int32_t* npv, int b_max, int n,
                  int64_t row_len, int64_t lag, int64_t p0, int64_t n_pairs, int out_mode,
                  float* out, int64_t out_ld, const float* obs, double* sum, double* sumsq,
                  int32_t* cnt, int32_t* counts, int64_t counts_stride, void* workspace,
                  size_t ws_bytes, const tenex_te_config* cfg, void* stream_,
                  const int64_t* pairs = nullptr, const int64_t* item_start = nullptr,
                  int64_t n_items_list = 0) {
  cudaStream_t stream = as_stream(stream_);
  if (!bins || !npv) return fail(TENEX_ERR_BADARG, "bins and n_per_var must be non-NULL");
  if (n < 2) return fail(TENEX_ERR_BADARG, "n_vars must be >= 2 (got %d)", n);
  if (b_max < 1 || b_max > 255)
    return fail(TENEX_ERR_UNSUPPORTED, "b_max=%d: the shared-memory kernel handles 1..255",
                b_max);
  if (lag < 1 || row_len <= lag)
    return fail(TENEX_ERR_BADARG, "need 1 <= lag < row_len (lag=%lld, row_len=%lld)",
                (long long)lag, (long long)row_len);
  if (row_len >= ((int64_t)1 << 31))
    return fail(TENEX_ERR_UNSUPPORTED, "row_len=%lld: series must be shorter than 2^31",
                (long long)row_len);
  if (ld < row_len || (ld % 16) != 0 || (reinterpret_cast<uintptr_t>(bins) % 16) != 0)
    return fail(TENEX_ERR_BADARG,
                "bins rows must be 16-byte aligned with ld %% 16 == 0 and ld >= row_len "
                "(ld=%lld, row_len=%lld)",
                (long long)ld, (long long)row_len);
  const int64_t total = (int64_t)n * (n - 1);
  if (!pairs && (p0 < 0 || n_pairs < 0 || p0 + n_pairs > total))
    return fail(TENEX_ERR_BADARG, "pair range [%lld, %lld) outside [0, %lld)", (long long)p0,
                (long long)(p0 + n_pairs), (long long)total);
  if (pairs && (!item_start || n_items_list < 0 || n_pairs < 0 || p0 != 0))
    return fail(TENEX_ERR_BADARG, "pair list needs item_start, n_items >= 0 and n_pairs >= 0");
  if (n_pairs == 0) return TENEX_OK;  // an empty range touches no output (NULL allowed)
  if (out_mode != kOutStats && !out) return fail(TENEX_ERR_BADARG, "out must be non-NULL");
  if (out_mode == kOutMatrix && out_ld < n)
    return fail(TENEX_ERR_BADARG, "out_ld (%lld) must be >= n_vars", (long long)out_ld);
  if (out_mode == kOutStats && (!obs || !sum || !sumsq || !cnt))
    return fail(TENEX_ERR_BADARG, "observed, sum, sumsq and count_ge must be non-NULL");
  if (!workspace || (int64_t)ws_bytes < ws_total(n, b_max))
    return fail(TENEX_ERR_OOM, "workspace must be >= %lld bytes (tenex_te_workspace_bytes)",
                (long long)ws_total(n, b_max));
  if (counts && counts_stride < (int64_t)b_max * b_max * b_max)
    return fail(TENEX_ERR_BADARG, "counts_stride must be >= b_max^3");
  DevAttr A;
  int st = current_device_attr(&A);
  if (st) return st;

  TeParams P{};
  P.bins = bins;
  P.ld = ld;
  P.npv = npv;
  P.n = n;
  P.N = (int)(row_len - lag);
  P.lag = (int)lag;
  P.p0 = p0;
  P.p1 = p0 + n_pairs;
  // 512 sources per item: fewer target stagings than 128 (3% faster at 10,000
  // genes), and a chunk of 512 source rows still fits L2 beside the others
  P.W = (cfg && cfg->src_chunk) ? cfg->src_chunk : 512;
  if (P.W < 1) return fail(TENEX_ERR_BADARG, "src_chunk must be >= 1");
  if (pairs) {
    P.pairs = pairs;
    P.item_start = item_start;
    P.n_items = n_items_list;
    P.t_first = 0;
    P.n_targets = 1;
    P.n_chunks = 1;
    P.tblock = 1;
  } else {
    P.t_first = (int)(p0 / (n - 1));
    const int t_last = (int)((P.p1 - 1) / (n - 1));
    P.n_targets = t_last - P.t_first + 1;
    P.n_chunks = (n + P.W - 1) / P.W;
    P.n_items = (int64_t)P.n_targets * P.n_chunks;
    // about 20% of L2 for the block's target rows: at 512 sources per item the
    // full 10,000 x 20,000 launch reads 144 GB from DRAM with it against 229 GB
    // with 40% (same time; the launch is bound by the shared-memory pipe)
    const int64_t rows = (int64_t)A.l2_bytes / 5 / std::max<int64_t>(ld, 1);
    P.tblock = (int)std::max<int64_t>(1, std::min<int64_t>(P.n_targets, rows));
  }
  if (P.n_items == 0) return TENEX_OK;
  if (P.n_items > 0x7fffffffLL - 65536)
    return fail(TENEX_ERR_UNSUPPORTED, "too many work items (%lld); raise src_chunk",
                (long long)P.n_items);
  P.bmax = b_max;
  P.zbytes = b_max <= 16 ? 1 : 2;
  P.ztile = z_tile(P.N, P.zbytes);
  P.mbmax = marginal_bound(b_max, P.ztile, P.zbytes, smem_one_cta(A));
  P.big = P.N >= (1 << 24) ? 1 : 0;
  P.out_mode = out_mode;
  P.out = out;
  P.out_ld = out_ld;
  P.obs = obs;
  P.sum = sum;
  P.sumsq = sumsq;
  P.cnt_ge = cnt;
  P.counts_dbg = counts;
  P.counts_stride = counts_stride;
  P.ws = reinterpret_cast<WsHeader*>(workspace);
  unsigned char* wsb = reinterpret_cast<unsigned char*>(workspace);
  int32_t* order = reinterpret_cast<int32_t*>(wsb + ws_order_off(n, b_max));
  P.order = order;

  // worst case the device can meet: 16-bit halves when N < 65536, else 32-bit
  const int64_t hb = P.N < 65536 ? (b_max + 1) / 2 : b_max;
  const int64_t worst_slot = round_up((int64_t)b_max * b_max * hb, 4) * 4;
  TeLaunch L{};
  st = plan_te_launch(P, cfg, A, &L, worst_slot);
  if (st) return st;
  P.smem_bytes = L.smem;
  // pairs whose histogram does not fit shared memory, and every pair of a target
  // beyond the marginal bound: global-memory overflow launch
  const bool overflow = needs_overflow(b_max, P.N, P.zbytes, P.mbmax, L.smem);
  int64_t n_gslots = 0;
  if (overflow) {
    P.gslot_words = (int64_t)b_max * b_max * b_max;
    n_gslots = gmem_slot_count(b_max, A);
    const int64_t slot_bytes = round_up(n_gslots * P.gslot_words * 4, 256);
    const int64_t marg_bytes =
        P.mbmax < b_max ? round_up(n_gslots * gmarg_words(b_max) * 4, 256) : 0;
    const int64_t c2b_bytes = round_up(n_gslots * gc2b_words(b_max) * 4, 256);
    const int64_t need = ws_total(n, b_max) + slot_bytes + marg_bytes + c2b_bytes;
    if ((int64_t)ws_bytes < need)
      return fail(TENEX_ERR_UNSUPPORTED,
                  "pairs with b up to %d do not fit shared memory and need %lld bytes of "
                  "global-memory slots in the workspace (%lld given; size it with "
                  "tenex_te_workspace_bytes)", b_max, (long long)need, (long long)ws_bytes);
    unsigned char* g = reinterpret_cast<unsigned char*>(workspace) + ws_total(n, b_max);
    P.gslots = reinterpret_cast<uint32_t*>(g);
    if (marg_bytes) {
      P.gmarg = reinterpret_cast<int32_t*>(g + slot_bytes);
      P.gmarg_words = gmarg_words(b_max);
    }
    P.gc2b = reinterpret_cast<uint32_t*>(g + slot_bytes + marg_bytes);
    P.gc2b_words = gc2b_words(b_max);
  }
  P.overflow = overflow ? 1 : 0;
  int64_t grid = L.grid;
  if (grid > P.n_items) grid = P.n_items;

  cudaError_t e = cudaMemsetAsync(workspace, 0, sizeof(WsHeader), stream);
  if (e != cudaSuccess) return check_cuda(e, "workspace reset");
  gene_prepass_kernel<<<n, 256, 0, stream>>>(bins, ld, npv, b_max, n, row_len, P.ws);
  st = check_launch("gene_prepass_kernel");
  if (st) return st;
  if (!pairs) {
    source_order_kernel<<<1, 1024, 0, stream>>>(npv, n, order);
    st = check_launch("source_order_kernel");
    if (st) return st;
  }
  e = cudaFuncSetAttribute(te_pair_tile_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           L.smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
  te_pair_tile_kernel<false><<<(int)grid, L.threads, L.smem, stream>>>(P);
  st = check_launch("te_pair_tile_kernel");
  if (st || !overflow) return st;
  e = cudaFuncSetAttribute(te_pair_tile_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           L.smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
  te_pair_tile_kernel<true><<<(int)std::min<int64_t>(n_gslots, P.n_items), L.threads, L.smem,
                        stream>>>(P);
  return check_launch("te_pair_tile_kernel (global-memory overflow)");
}

extern "C" int tenex_te_pairfree(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                                 int b_max, int n_vars, int64_t row_len, int64_t lag,
                                 int64_t pair_offset, int64_t n_pairs, float* out,
                                 int out_mode, int64_t out_ld, void* workspace,
                                 size_t workspace_bytes, const tenex_te_config* cfg,
                                 void* stream) {
  if (out_mode != TENEX_OUT_PAIRFREE && out_mode != TENEX_OUT_MATRIX)
    return fail(TENEX_ERR_BADARG, "out_mode must be TENEX_OUT_PAIRFREE or TENEX_OUT_MATRIX");
  return te_run(bins, ld, n_per_var, b_max, n_vars, row_len, lag, pair_offset, n_pairs,
                out_mode == TENEX_OUT_PAIRFREE ? kOutPairfree : kOutMatrix, out, out_ld,
                nullptr, nullptr, nullptr, nullptr, nullptr, 0, workspace, workspace_bytes,
                cfg, stream);
}

extern "C" int tenex_te_pairfree_counts(const uint8_t* bins, int64_t ld,
                                        const int32_t* n_per_var, int b_max, int n_vars,
                                        int64_t row_len, int64_t lag, int64_t pair_offset,
                                        int64_t n_pairs, float* out, int32_t* counts,
                                        int64_t counts_stride, void* workspace,
                                        size_t workspace_bytes, const tenex_te_config* cfg,
                                        void* stream) {
  if (!counts) return fail(TENEX_ERR_BADARG, "counts must be non-NULL");
  return te_run(bins, ld, n_per_var, b_max, n_vars, row_len, lag, pair_offset, n_pairs,
                kOutPairfree, out, 0, nullptr, nullptr, nullptr, nullptr, counts,
                counts_stride, workspace, workspace_bytes, cfg, stream);
}

extern "C" int tenex_surrogate_accumulate(const uint8_t* bins, int64_t ld,
                                          const int32_t* n_per_var, int b_max, int n_vars,
                                          int64_t row_len, int64_t lag, int64_t pair_offset,
                                          int64_t n_pairs, const float* observed, double* sum,
                                          double* sumsq, int32_t* count_ge, void* workspace,
                                          size_t workspace_bytes, const tenex_te_config* cfg,
                                          void* stream) {
  return te_run(bins, ld, n_per_var, b_max, n_vars, row_len, lag, pair_offset, n_pairs,
                kOutStats, nullptr, 0, observed, sum, sumsq, count_ge, nullptr, 0, workspace,
                workspace_bytes, cfg, stream);
}

extern "C" int tenex_te_pairs(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                              int b_max, int n_vars, int64_t row_len, int64_t lag,
                              const int64_t* pairs, int64_t n_pairs, const int64_t* item_start,
                              int64_t n_items, float* out, void* workspace,
                              size_t workspace_bytes, const tenex_te_config* cfg,
                              void* stream) {
  if (!pairs || !item_start) return fail(TENEX_ERR_BADARG, "pairs and item_start must be non-NULL");
  return te_run(bins, ld, n_per_var, b_max, n_vars, row_len, lag, 0, n_pairs, kOutPairfree, out,
                0, nullptr, nullptr, nullptr, nullptr, nullptr, 0, workspace, workspace_bytes,
                cfg, stream, pairs, item_start, n_items);
}

extern "C" int tenex_surrogate_accumulate_pairs(
    const uint8_t* bins, int64_t ld, const int32_t* n_per_var, int b_max, int n_vars,
    int64_t row_len, int64_t lag, const int64_t* pairs, int64_t n_pairs,
    const int64_t* item_start, int64_t n_items, const float* observed, double* sum,
    double* sumsq, int32_t* count_ge, void* workspace, size_t workspace_bytes,
    const tenex_te_config* cfg, void* stream) {
  if (!pairs || !item_start) return fail(TENEX_ERR_BADARG, "pairs and item_start must be non-NULL");
  return te_run(bins, ld, n_per_var, b_max, n_vars, row_len, lag, 0, n_pairs, kOutStats, nullptr,
                0, observed, sum, sumsq, count_ge, nullptr, 0, workspace, workspace_bytes, cfg,
                stream, pairs, item_start, n_items);
}

// ---------------------------------------------------------------------------
// Entry point for callers that must not allocate device memory.
//
// Some hosts of this library cannot call cudaMalloc once they are running:
// services that reserve their whole device-memory budget at start-up and treat
// any later allocation as a fault, processes whose device memory is owned by
// another framework's pooling allocator, and foreign-language bindings that
// have no way to own the lifetime of a device buffer. tenex_te_pairfree needs
// a caller-provided workspace; this variant instead uses the fixed scratch
// area below, which is part of the library's device image: every GPU on which
// the library is loaded keeps these 4 MiB for the life of the process.
//
// The scratch address is looked up once per device (cudaGetSymbolAddress, with
// that device current) by the first call made on that device, so that first
// call should come before any stream capture. All calls share the one area and
// each call rewrites it (work ticket and validation words are cleared, the
// source order recomputed), so calls that overlap on the GPU — on two
// streams, or from two threads — race and must not be issued.
// ---------------------------------------------------------------------------
namespace tenex {
namespace {
constexpr size_t kStaticScratchBytes = (size_t)4 << 20;
__device__ __align__(256) unsigned char g_static_scratch[kStaticScratchBytes];

int static_scratch(void** out) {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return check_cuda(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(TENEX_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess) return check_cuda(e, "cudaGetSymbolAddress(scratch)");
    addr[dev] = p;
  }
  *out = addr[dev];
  return TENEX_OK;
}
}  // namespace
}  // namespace tenex

// Status word of a static-scratch call: 0 = inputs valid and every pair
// computed; 1 = a bin value >= its gene's n_per_var or n_per_var outside
// [1, b_max] (no TE computed); 3 = a work item's histogram did not fit shared
// memory (its pairs were not computed).
__global__ void static_status_kernel(const WsHeader* h, int32_t* status) {
  const int bad = h->bad_data;
  *status = bad != 0 ? bad : (h->bad_item != 0 ? 3 : 0);
}

extern "C" int tenex_te_pairfree_static(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                                        int b_max, int n_vars, int64_t row_len, int64_t lag,
                                        int64_t pair_offset, int64_t n_pairs, float* out,
                                        int out_mode, int64_t out_ld, int32_t* status,
                                        const tenex_te_config* cfg, void* stream) {
  if (n_vars < 2 || b_max < 1 || b_max > 255)
    return fail(TENEX_ERR_BADARG, "need n_vars >= 2 and 1 <= b_max <= 255");
  const int64_t need = ws_total(n_vars, b_max);
  if (need > (int64_t)kStaticScratchBytes)
    return fail(TENEX_ERR_UNSUPPORTED,
                "n_vars=%d with b_max=%d needs %lld bytes of scratch; the built-in area holds "
                "%zu bytes (about 4*n_vars + 512 must fit). Use tenex_te_pairfree "
                "with a workspace instead.",
                n_vars, b_max, (long long)need, kStaticScratchBytes);
  if (lag >= 1 && row_len > lag && row_len < ((int64_t)1 << 31)) {
    // pairs too large for shared memory (coarsening off) need global-memory
    // histogram slots, far beyond the built-in area
    DevAttr A;
    const int st0 = current_device_attr(&A);
    if (st0) return st0;
    const int64_t ov = gmem_bytes(b_max, (int)(row_len - lag), b_max <= 16 ? 1 : 2, A);
    if (ov > 0)
      return fail(TENEX_ERR_UNSUPPORTED,
                  "b_max=%d: pairs whose histogram does not fit shared memory need %lld bytes "
                  "of global-memory histogram slots, which the built-in %zu-byte scratch area "
                  "cannot hold; coarsen the bins, or call tenex_te_pairfree with a workspace of "
                  "tenex_te_workspace_bytes() bytes",
                  b_max, (long long)(need + ov), kStaticScratchBytes);
  }
  void* ws = nullptr;
  int st = static_scratch(&ws);
  if (st) return st;
  st = tenex_te_pairfree(bins, ld, n_per_var, b_max, n_vars, row_len, lag, pair_offset, n_pairs,
                         out, out_mode, out_ld, ws, kStaticScratchBytes, cfg, stream);
  if (st || !status) return st;
  if (n_pairs == 0) {  // nothing ran: the area still holds an earlier call's words
    return check_cuda(cudaMemsetAsync(status, 0, sizeof(int32_t), as_stream(stream)),
                      "status reset");
  }
  static_status_kernel<<<1, 1, 0, as_stream(stream)>>>(reinterpret_cast<const WsHeader*>(ws),
                                                       status);
  return check_launch("static_status_kernel");
}
