// gemm_b2.cu — binary (b_max = 2) TE matrix on the 5th-generation tensor cores.
//
// Reference: tenex/kernels/gemm_b2.py:307-425 (three FP32 cuBLAS GEMMs
// C = fp.p^T, D = p.p^T, E = f.p^T, with f = x[:, tau:], p = x[:, :-tau],
// fp = f*p) and the Triton epilogue :65-187 (8 joint cells from C, D, E and
// per-gene marginals, then sum c*log2(c*c1/(c2a*c2b)) / N).
//
// B200 design:
//   * pack kernel: one pass over the bins (one warp per segment of a row)
//     writes the lag-shifted K-major int8 operand F and FP = F & P (rows padded
//     to a multiple of 128 bytes, zero filled), the per-gene counts nf, np, nfp,
//     and flags any bin other than 0/1; P is the bins themselves (a tensor map
//     with K extent L, TMA zero-fills beyond it). The 4-bit form packs P too.
//   * GEMM kernel: one CTA per tile of 128 sources x TN targets (TN from
//     {128, 112, 96, 80, 64}, picked per matrix so the tiles finish in the
//     fewest rounds on the SMs; widths of 80 and below run two CTAs per SM,
//     B2Layout). A producer warp brings, per stage, one
//     128-byte wide box of FP, P, F (TN target rows each) and P (128 source
//     rows) by TMA (cp.async.bulk.tensor.2d, no multicast), 128-byte swizzled
//     (the K-major SWIZZLE_128B layout the MMA descriptors name); a separate MMA
//     warp issues, per 32-byte K step, two tcgen05.mma with the source tile as
//     A (M = 128 lanes = sources): B = [FP; P] of the targets as one N = 2 TN
//     MMA (C^T, D^T) and B = F at N = TN (E^T), accumulators in TMEM. The source
//     tile is read twice per K step rather than three times. kind::i8 on int8
//     operands (int32 sums, exact) or kind::mxf4 on packed E2M1 operands with
//     unit block scales (float32 sums, exact below 2^24).
//   * Epilogue: every warp of the CTA (16, or 8 with two CTAs per SM); warp w
//     reads TMEM lanes 32*(w%4).. (one source per lane) and its share of the TN
//     target columns (a quarter, or half) with tcgen05.ld, forms
//     the 8 cells (target marginals and c1/c2a staged in shared memory) and
//     writes TE(src -> tgt) to out[src, tgt], four consecutive targets of a
//     source row per 16-byte store.
//   * Every mbarrier wait is bounded; on expiry the kernel records an error
//     word, drains the copies it issued (bounded), frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdint>
#include <iterator>
#include <mutex>

#include "common.cuh"
#include "tcgen05.cuh"

namespace tenex {
namespace {

constexpr int kTile = 128;     // sources per tile (M = 128 TMEM lanes); targets per tile <= 128
constexpr int kKt = 128;       // bytes of K per pipeline stage (4 MMA K-steps of 32)
// one stage: FP, P, F of TN targets and P of 128 sources, 128 bytes of K each
// (every box starts on a 1024-byte swizzle atom: TN is a multiple of 16)
__host__ __device__ constexpr int stage_bytes(int TN) { return (3 * TN + kTile) * kKt; }
constexpr int kTileN[] = {128, 112, 96, 80, 64};  // target-tile widths (MMA N = TN and 2 TN)

// Per-width layout. TN > 80: one CTA per SM (512 threads, three stages, 512 TMEM
// columns: C at 0, D at TN, E at 256, 4-bit scale factors at 384 / 392). TN <= 80:
// the three accumulators and the scale factors fit 256 columns (E at 2 TN rounded
// up to 32, scale factors at 240 / 248), so two CTAs share an SM (256 threads,
// two stages each): one CTA's epilogue and stage waits overlap the other's MMAs.
template <int TN>
struct B2Layout {
  static constexpr bool kPair = TN <= 80;
  static constexpr int kThreads = kPair ? 256 : 512;
  static constexpr int kCtasPerSm = kPair ? 2 : 1;
  static constexpr int kStages = kPair ? 2 : 3;
  static constexpr int kTmemCols = kPair ? 256 : 512;
  static constexpr uint32_t kECol = kPair ? (uint32_t)((2 * TN + 31) / 32 * 32) : 256u;
  static constexpr uint32_t kSfaCol = kPair ? 240u : 384u, kSfbCol = kPair ? 248u : 392u;
  static constexpr int kColGroups = kThreads / 128;  // epilogue warps per TMEM lane quarter
  static constexpr int kSmem = kStages * stage_bytes(TN) + 1024 + 256 + 7 * kTile * 4;
  static_assert(!kPair || kECol + TN <= kSfaCol, "accumulators overlap the scale factors");
  static_assert((TN / kColGroups) % 4 == 0, "epilogue columns per warp: a multiple of 4");
};

struct B2Params {
  int n;            // genes
  int L;            // samples per pair
  int Lpad;         // padded K (multiple of kKt)
  const int32_t* marg;  // (3, n): nf, np, nfp
  float* out;       // (n, n): out[src * ld + tgt]
  int64_t out_ld;
  int vec_out;      // out and out_ld allow 16-byte row stores
  int* err;         // device error word (1 = a wait expired, 2 = a bin was not 0/1)
};

__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[4]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
}

__device__ __forceinline__ void tmem_ld(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}

__device__ __forceinline__ void tmem_wait_ld() {
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// c * log2(c * c1 / (c2a * c2b)); exactly 0 for an empty cell and where the two
// products are equal (the reference's ratio is exactly 1 there); otherwise the
// ratio as c * (1/c2b) * (c1/c2a), with q = c1/c2a divided once per target state
// and rb = 1/c2b once per source state (approximate reciprocal, 1 ulp), and
// lg2.approx: far below the 1e-6 TE budget, and 12 MUFU operations per pair
// (4 reciprocals, 8 logarithms) instead of a division per cell.
__device__ __forceinline__ float cell_term(float c, float c1, float c2a, float c2b, float q,
                                           float rb) {
  const bool e = c == 0.f || c * c1 == c2a * c2b;
  const float r = e ? 1.f : c * rb * q;
  return c * __log2f(r);
}

// Pack: F[g, t] = x[g, t+lag] (the lag-shifted operand TMA cannot address: its
// copies start on 16-byte boundaries) and FP = F & P for t < L (0 beyond, up to
// Lpad), plus the per-gene counts nf, np, nfp. The int8 form writes F and FP
// (P is read from the bins directly); the 4-bit form writes F, FP and P as
// packed E2M1 values (1.0 = 0x2, 0.0 = 0x0; sample 2k in the low nibble of byte
// k, 2k + 1 in the high one), rows of Lpad / 2 bytes.
// One warp per segment of a gene's row (32 lanes x one chunk of kChunk samples),
// so a matrix of a few thousand genes still puts every SM's memory requests in
// flight at once: a lane issues all its loads (the chunk of P and the aligned
// window of F around it) before its first store; a scalar path covers the row
// end. The counts reduce by shuffles and go to `marg` (zeroed by the caller) by
// one atomic per count and warp.
// Every bin must be 0 or 1 (the GEMM sums the raw bytes): a larger value sets
// the error word to 2.
constexpr int kPackWarps = 4;

template <bool FP4>
struct PackChunk {
  static constexpr int kSamples = FP4 ? 32 : 16;  // samples per lane
  static constexpr int kSeg = 32 * kSamples;      // samples per warp
};

__device__ __forceinline__ uint32_t e2m1_nibbles(uint32_t w) {
  // four 0/1 bytes b0..b3 -> 16 bits: 2*b0 | 2*b1 << 4 | 2*b2 << 8 | 2*b3 << 12
  const uint32_t t = (w | (w >> 4)) & 0x00ff00ffu;
  return __byte_perm(t, 0, 0x4420) << 1;
}

template <bool FP4>
__global__ void __launch_bounds__(kPackWarps * 32)
b2_pack_kernel(const uint8_t* __restrict__ bins, int64_t ld, int n, int L, int lag, int Lpad,
               int nseg, uint8_t* __restrict__ ops, int32_t* __restrict__ marg,
               int* __restrict__ err) {
  constexpr int S = PackChunk<FP4>::kSamples;
  constexpr int NW = S / 4;  // 32-bit words of 0/1 bytes per operand and lane
  const int64_t wid = (int64_t)blockIdx.x * kPackWarps + (threadIdx.x >> 5);
  if (wid >= (int64_t)n * nseg) return;  // whole warps only: the shuffles below see full warps
  const int g = (int)(wid / nseg);
  const int seg = (int)(wid - (int64_t)g * nseg);
  const int lane = threadIdx.x & 31;
  const int t = seg * PackChunk<FP4>::kSeg + lane * S;
  const uint8_t* row = bins + (int64_t)g * ld;
  int nf = 0, np = 0, nfp = 0;
  uint32_t high = 0;  // any bit above bit 0 of a byte: a bin other than 0/1
  if (t < Lpad) {
    uint32_t f[NW], p[NW];
    const int64_t fa = (int64_t)(t + lag) & ~(int64_t)15;  // aligned start of F's window
    if (t + S <= L && fa + S + 16 <= ld) {
      uint4 pv[S / 16], av[S / 16 + 1];
#pragma unroll
      for (int u = 0; u < S / 16; ++u) pv[u] = *reinterpret_cast<const uint4*>(row + t + 16 * u);
#pragma unroll
      for (int u = 0; u < S / 16 + 1; ++u)
        av[u] = *reinterpret_cast<const uint4*>(row + fa + 16 * u);
      uint32_t w[NW + 4];
#pragma unroll
      for (int u = 0; u < S / 16 + 1; ++u) {
        w[4 * u] = av[u].x;
        w[4 * u + 1] = av[u].y;
        w[4 * u + 2] = av[u].z;
        w[4 * u + 3] = av[u].w;
      }
      // F's words start sh bytes into the window: a whole-word shift by selects
      // (registers, no local-memory indexing), then a byte funnel shift
      const int sh = (t + lag) & 15, qw = sh >> 2;
      uint32_t ws[NW + 1];
#pragma unroll
      for (int i = 0; i <= NW; ++i)
        ws[i] = qw == 0 ? w[i] : qw == 1 ? w[i + 1] : qw == 2 ? w[i + 2] : w[i + 3];
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        f[k] = __funnelshift_r(ws[k], ws[k + 1], (sh & 3) * 8);
        const uint4 q = pv[k >> 2];
        p[k] = (k & 3) == 0 ? q.x : (k & 3) == 1 ? q.y : (k & 3) == 2 ? q.z : q.w;
      }
    } else {
#pragma unroll
      for (int k = 0; k < NW; ++k) {
        uint32_t fk = 0, pk = 0;
        for (int j = 0; j < 4; ++j) {
          const int tt = t + 4 * k + j;
          if (tt < L) {
            fk |= (uint32_t)row[tt + lag] << (8 * j);
            pk |= (uint32_t)row[tt] << (8 * j);
          }
        }
        f[k] = fk;
        p[k] = pk;
      }
    }
#pragma unroll
    for (int k = 0; k < NW; ++k) {
      high |= (f[k] | p[k]) & 0xfefefefeu;
      nf += __popc(f[k]);
      np += __popc(p[k]);
      nfp += __popc(f[k] & p[k]);
    }
    if (FP4) {
      const int64_t rowb = Lpad / 2;
      uint8_t* Fr = ops + (int64_t)g * rowb;
      uint8_t* FPr = ops + ((int64_t)n + g) * rowb;
      uint8_t* Pr = ops + (2 * (int64_t)n + g) * rowb;
      uint32_t of[NW / 2], ofp[NW / 2], op[NW / 2];
#pragma unroll
      for (int k = 0; k < NW / 2; ++k) {
        of[k] = e2m1_nibbles(f[2 * k]) | (e2m1_nibbles(f[2 * k + 1]) << 16);
        ofp[k] = e2m1_nibbles(f[2 * k] & p[2 * k]) |
                 (e2m1_nibbles(f[2 * k + 1] & p[2 * k + 1]) << 16);
        op[k] = e2m1_nibbles(p[2 * k]) | (e2m1_nibbles(p[2 * k + 1]) << 16);
      }
      *reinterpret_cast<uint4*>(Fr + t / 2) = make_uint4(of[0], of[1], of[2], of[3]);
      *reinterpret_cast<uint4*>(FPr + t / 2) = make_uint4(ofp[0], ofp[1], ofp[2], ofp[3]);
      *reinterpret_cast<uint4*>(Pr + t / 2) = make_uint4(op[0], op[1], op[2], op[3]);
    } else {
      uint8_t* Fr = ops + (int64_t)g * Lpad;
      uint8_t* FPr = ops + ((int64_t)n + g) * Lpad;
      *reinterpret_cast<uint4*>(Fr + t) = make_uint4(f[0], f[1], f[2], f[3]);
      *reinterpret_cast<uint4*>(FPr + t) =
          make_uint4(f[0] & p[0], f[1] & p[1], f[2] & p[2], f[3] & p[3]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nf += __shfl_xor_sync(0xffffffffu, nf, o);
    np += __shfl_xor_sync(0xffffffffu, np, o);
    nfp += __shfl_xor_sync(0xffffffffu, nfp, o);
  }
  if (lane < 3) {
    const int v = lane == 0 ? nf : (lane == 1 ? np : nfp);
    if (v) atomicAdd(marg + (int64_t)lane * n + g, v);
  }
  if (__any_sync(0xffffffffu, high != 0) && lane == 0) atomicExch(err, 2);
}

// Tensor maps of the operands: F and FP (packed, n x Lpad) and P (the bins
// themselves, n x L with row stride ld; TMA fills columns >= L and rows >= n
// with zeros). The 4-bit form has all three packed (rows of Lpad / 2 bytes).
// Target boxes are TN rows high, source boxes 128 (two maps of P).
struct B2Maps {
  CUtensorMap F, Pt, FP, Ps;
};

// 4-bit form: TMEM columns of the UE8M0 scale factors (all 1.0) after the
// accumulators (B2Layout): A (sources, M = 128) at kSfaCol, B (targets, up to
// N = 256) at kSfbCol; 8 columns each hold every layout those take.

// TE(src -> target ti of the tile) from the three sums C, D, E of the pair, the
// target's staged marginals (tmarg: nf, np, nfp; tq: c1/c2a for the target
// states 11, 01, 10, 00) and the source's np (npj): the 8 cells and their terms.
__device__ __forceinline__ float b2_pair_te(float C, float Dv, float E, int ti, float npj,
                                            float N, const float* tmarg, const float* tq) {
  const float nf = tmarg[ti], np_ = tmarg[kTile + ti], nfp = tmarg[2 * kTile + ti];
  const float c1_1 = np_, c1_0 = N - np_;
  const float c2a11 = nfp, c2a01 = np_ - nfp, c2a10 = nf - nfp, c2a00 = N - nf - np_ + nfp;
  const float c2b11 = Dv, c2b01 = npj - Dv, c2b10 = np_ - Dv, c2b00 = N - np_ - npj + Dv;
  const float q11 = tq[ti], q01 = tq[kTile + ti], q10 = tq[2 * kTile + ti],
              q00 = tq[3 * kTile + ti];
  const float rb11 = __fdividef(1.f, c2b11), rb01 = __fdividef(1.f, c2b01),
              rb10 = __fdividef(1.f, c2b10), rb00 = __fdividef(1.f, c2b00);
  float te = 0.f;
  te += cell_term(C, c1_1, c2a11, c2b11, q11, rb11);                                // [1,1,1]
  te += cell_term(Dv - C, c1_1, c2a01, c2b11, q01, rb11);                           // [0,1,1]
  te += cell_term(E - C, c1_0, c2a10, c2b01, q10, rb01);                            // [1,0,1]
  te += cell_term(npj - Dv - E + C, c1_0, c2a00, c2b01, q00, rb01);                 // [0,0,1]
  te += cell_term(nfp - C, c1_1, c2a11, c2b10, q11, rb10);                          // [1,1,0]
  te += cell_term(np_ - Dv - nfp + C, c1_1, c2a01, c2b10, q01, rb10);               // [0,1,0]
  te += cell_term(nf - E - nfp + C, c1_0, c2a10, c2b00, q10, rb00);                 // [1,0,0]
  te += cell_term(N - nf - np_ - npj + nfp + Dv + E - C, c1_0, c2a00, c2b00, q00,
                  rb00);                                                            // [0,0,0]
  return te;
}

// Four consecutive targets ia .. ia + 3 of source row j: one 16-byte store when
// they are all inside the matrix, off the diagonal and aligned; else one by one.
__device__ __forceinline__ void b2_store4(const B2Params& prm, float* orow, int ia, int j,
                                          const float (&res)[4]) {
  if (prm.vec_out && ia + 4 <= prm.n && (j < ia || j >= ia + 4)) {
    *reinterpret_cast<float4*>(orow + ia) = make_float4(res[0], res[1], res[2], res[3]);
  } else {
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (ia + u < prm.n && ia + u != j) orow[ia + u] = res[u];
  }
}

// TE of NC consecutive targets (tile columns cb .. cb + NC - 1) for the source
// of this thread's TMEM lane: the three sums from TMEM (every lane of the warp
// loads, as tcgen05.ld requires), then b2_pair_te and b2_store4.
template <bool FP4, int NC>
__device__ __forceinline__ void b2_cells(const B2Params& prm, uint32_t lane_base, int cb, int TN,
                                         uint32_t ecol, int m0, int j, bool active, float npj,
                                         const float* tmarg, const float* tq) {
  uint32_t rc[NC], rd[NC], re[NC];
  tmem_ld(lane_base + (uint32_t)cb, rc);
  tmem_ld(lane_base + (uint32_t)(TN + cb), rd);
  tmem_ld(lane_base + ecol + (uint32_t)cb, re);
  tmem_wait_ld();
  if (!active) return;
  const float N = (float)prm.L;
  const float invL = 1.0f / N;
  float* orow = prm.out + (int64_t)j * prm.out_ld;
#pragma unroll
  for (int q0 = 0; q0 < NC; q0 += 4) {
    float res[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int q = q0 + u;
      const float C = FP4 ? __uint_as_float(rc[q]) : (float)rc[q];
      const float Dv = FP4 ? __uint_as_float(rd[q]) : (float)rd[q];
      const float E = FP4 ? __uint_as_float(re[q]) : (float)re[q];
      res[u] = b2_pair_te(C, Dv, E, cb + q, npj, N, tmarg, tq) * invL;
    }
    b2_store4(prm, orow, m0 + cb + q0, j, res);
  }
}

// FP4 = false: kind::i8 MMAs on the int8 operands (K = 32 per MMA), int32 sums.
// FP4 = true: kind::mxf4 MMAs on the packed E2M1 operands (K = 64 per MMA, two
// samples per byte: half the shared-memory bytes per multiply), unit block
// scales, float32 sums (exact integers below 2^24).
// TN: targets per tile (a multiple of 16, at most 128): [FP; P] is one MMA of
// N = 2 TN and F one of N = TN.
template <bool FP4, int TN>
__global__ void __launch_bounds__(B2Layout<TN>::kThreads, B2Layout<TN>::kCtasPerSm)
    b2_gemm_kernel(const __grid_constant__ B2Maps maps, B2Params prm) {
  using LY = B2Layout<TN>;
  constexpr int kStages = LY::kStages, kTmemCols = LY::kTmemCols, kB2Threads = LY::kThreads;
  constexpr uint32_t kSfaCol = LY::kSfaCol, kSfbCol = LY::kSfbCol, kECol = LY::kECol;
  constexpr int kStageBytes = stage_bytes(TN);
  constexpr int kTgtBytes = TN * kKt;  // one target operand box per stage
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte align the operand region
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* stage_base = smem;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accbar = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accbar + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  // the tile's target marginals nf, np, nfp as floats and c1/c2a for the target
  // states (x1, x0) = 11, 01, 10, 00 (epilogue operands)
  float* tmarg = reinterpret_cast<float*>(smem + kStages * kStageBytes + 256);
  float* tq = tmarg + 3 * kTile;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int m0 = blockIdx.y * TN;     // targets
  const int n0 = blockIdx.x * kTile;  // sources
  const int nk = (FP4 ? prm.Lpad / 2 : prm.Lpad) / kKt;  // 128-byte K stages

  if (tid == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accbar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_u32(tmem_slot)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *tmem_slot;
  if (FP4) {
    // unit scale factors (UE8M0 127 = 1.0 in every byte) for the MMAs to read
    if (warp < 4) {
      const uint32_t lanes = (uint32_t)(warp * 32) << 16;
      tmem_st8(tmem + lanes + kSfaCol, 0x7f7f7f7fu);
      tmem_st8(tmem + lanes + kSfbCol, 0x7f7f7f7fu);
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }

  // ---- producer (warp 0, lane 0): TMA loads of stage k into buffer k % kStages,
  // each once the MMAs that read the buffer's previous contents completed --------
  if (tid == 0) {
    int issued = 0;
    bool ok = true;
    for (int k = 0; k < nk; ++k) {
      const int s = k % kStages;
      if (k >= kStages &&
          (*(volatile int*)abort_flag || !mbar_wait(&empty[s], (uint32_t)(((k / kStages) - 1) & 1)))) {
        ok = false;
        break;
      }
      unsigned char* buf = stage_base + s * kStageBytes;
      mbar_expect_tx(&full[s], kStageBytes);
      const int x0 = k * kKt;
      // one 128-byte wide box per operand (TN or 128 rows), 128-byte swizzled
      tma_load_2d(buf + 0 * kTgtBytes, &maps.FP, x0, m0, &full[s]);
      tma_load_2d(buf + 1 * kTgtBytes, &maps.Pt, x0, m0, &full[s]);
      tma_load_2d(buf + 2 * kTgtBytes, &maps.F, x0, m0, &full[s]);
      tma_load_2d(buf + 3 * kTgtBytes, &maps.Ps, x0, n0, &full[s]);
      issued = k + 1;
    }
    if (!ok) {
      // no exit with copies in flight: wait (bounded) for every issued load
      atomicExch(prm.err, 1);
      *(volatile int*)abort_flag = 1;
      for (int k = issued - kStages > 0 ? issued - kStages : 0; k < issued; ++k)
        (void)mbar_wait(&full[k % kStages], (uint32_t)((k / kStages) & 1));
    }
  }

  // ---- MMA issuer (warp 1, lane 0): stage k's MMAs as soon as its operands are
  // in place; never waits on MMA completion, so the tensor pipe gets the stages
  // back to back. The source tile P_j is the A operand (M = 128 lanes = sources)
  // and the target tiles are B: [FP_i; P_i] (adjacent in the stage, one N = 256
  // MMA) and F_i (N = 128), so a K step reads P_j twice instead of three times
  // (20 KB of shared memory instead of 24 at TN = 128). TMEM columns 0..TN-1 =
  // C^T, TN..2TN-1 = D^T, 256..256+TN-1 = E^T.
  if (tid == 32) {
    const uint32_t idesc256 = FP4 ? idesc_mxf4(kTile, 2 * TN) : idesc_i8(kTile, 2 * TN);
    const uint32_t idesc128 = FP4 ? idesc_mxf4(kTile, TN) : idesc_i8(kTile, TN);
    bool ok = true;
    for (int k = 0; k < nk; ++k) {
      const int s = k % kStages;
      const uint32_t ph = (uint32_t)((k / kStages) & 1);
      if (*(volatile int*)abort_flag || !mbar_wait(&full[s], ph)) {
        ok = false;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      unsigned char* buf = stage_base + s * kStageBytes;
      const uint32_t bFPP = smem_u32(buf + 0 * kTgtBytes);  // FP_i rows, then P_i rows
      const uint32_t bF = smem_u32(buf + 2 * kTgtBytes);
      const uint32_t aPj = smem_u32(buf + 3 * kTgtBytes);
#pragma unroll
      for (int kk = 0; kk < kKt / 32; ++kk) {
        const uint32_t off = kk * 32;  // 32-byte K step inside the 128-byte swizzle row
        const uint64_t ad = smem_desc_sw128(aPj + off);
        const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
        if (FP4) {
          mma_mxf4(tmem + 0, ad, smem_desc_sw128(bFPP + off), idesc256, acc, tmem + kSfaCol,
                   tmem + kSfbCol);
          mma_mxf4(tmem + kECol, ad, smem_desc_sw128(bF + off), idesc128, acc, tmem + kSfaCol,
                   tmem + kSfbCol);
        } else {
          mma_i8(tmem + 0, ad, smem_desc_sw128(bFPP + off), idesc256, acc);
          mma_i8(tmem + kECol, ad, smem_desc_sw128(bF + off), idesc128, acc);
        }
      }
      mma_commit(&empty[s]);  // stage s free once these MMAs complete
    }
    if (!ok) {
      atomicExch(prm.err, 1);
      *(volatile int*)abort_flag = 1;
    }
    mma_commit(accbar);  // arrives after every issued MMA, so the epilogue wakes either way
  }

  // ---- epilogue: every warp; lane quarter warp % 4, column group warp / 4 -----
  // (the warps that neither load nor issue stage the target marginals first;
  // a c2a of 0 gives q = inf or NaN, never read: its cells are empty)
  if (tid >= 64) {
    for (int k = tid - 64; k < TN; k += kB2Threads - 64) {
      const int i = m0 + k;
      float nf = 0.f, np_ = 0.f, nfp = 0.f;
      if (i < prm.n) {
        nf = (float)prm.marg[i];
        np_ = (float)prm.marg[(int64_t)prm.n + i];
        nfp = (float)prm.marg[2 * (int64_t)prm.n + i];
      }
      tmarg[k] = nf;
      tmarg[kTile + k] = np_;
      tmarg[2 * kTile + k] = nfp;
      const float N = (float)prm.L, c1_1 = np_, c1_0 = N - np_;
      tq[k] = c1_1 / nfp;
      tq[kTile + k] = c1_1 / (np_ - nfp);
      tq[2 * kTile + k] = c1_0 / (nf - nfp);
      tq[3 * kTile + k] = c1_0 / (N - nf - np_ + nfp);
    }
  }
  bool ok_acc = mbar_wait_sleep(accbar, 0, 200);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok_acc && tid == 0) atomicExch(prm.err, 1);
  const bool run = ok_acc && (*(volatile int*)abort_flag == 0);
  const int lq = warp & 3, cq = warp >> 2;
  const int j = n0 + lq * 32 + (tid & 31);  // source gene of this thread's TMEM lane
  const float npj = j < prm.n ? (float)prm.marg[prm.n + j] : 0.f;
  const uint32_t lane_base = tmem + ((uint32_t)(lq * 32) << 16);
  // TN / kColGroups target columns per warp, in chunks of 16, 8 and 4 (a multiple of 4)
  constexpr int kCw = TN / LY::kColGroups;
  const bool active = run && j < prm.n;
  int cb = cq * kCw;
  const int ce = cb + kCw;
  for (; cb + 16 <= ce; cb += 16)
    b2_cells<FP4, 16>(prm, lane_base, cb, TN, kECol, m0, j, active, npj, tmarg, tq);
  if (cb + 8 <= ce) {
    b2_cells<FP4, 8>(prm, lane_base, cb, TN, kECol, m0, j, active, npj, tmarg, tq);
    cb += 8;
  }
  if (cb + 4 <= ce)
    b2_cells<FP4, 4>(prm, lane_base, cb, TN, kECol, m0, j, active, npj, tmarg, tq);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(kTmemCols)
                 : "memory");
  }
}

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link).
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                                  const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                                  const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static std::once_flag once;
  static EncodeTiledFn fn = nullptr;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(p);
  });
  return fn;
}

static int make_map(CUtensorMap* map, const uint8_t* base, int rows, int64_t cols,
                    int64_t stride, int box_rows) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(TENEX_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)stride};
  const cuuint32_t box[2] = {(cuuint32_t)kKt, (cuuint32_t)box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, (void*)base, dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                   CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(TENEX_ERR_LAUNCH, "cuTensorMapEncodeTiled failed (%d)", (int)r);
  return TENEX_OK;
}

}  // namespace
}  // namespace tenex

using namespace tenex;

// Workspace: the packed operands (the larger of the two forms: int8 F and FP,
// n x round_up(L, 128) bytes each; 4-bit F, FP and P, n x round_up(L, 256) / 2
// bytes each), then the per-gene counts (3 x n int32), then the error word.
static int64_t b2_ops_bytes(int n, int64_t L) {
  const int64_t i8 = 2 * (int64_t)n * round_up(L, kKt);
  const int64_t f4 = 3 * (int64_t)n * (round_up(L, 2 * kKt) / 2);
  return round_up(i8 > f4 ? i8 : f4, 256);
}

extern "C" size_t tenex_b2_workspace_bytes(int n_vars, int64_t row_len, int64_t lag) {
  if (n_vars < 1 || row_len <= lag) return 256;
  return (size_t)(b2_ops_bytes(n_vars, row_len - lag) + round_up(3 * (int64_t)n_vars * 4, 256) +
                  256);
}

// One GEMM launch of target-tile width TN: ceil(n / 128) x ceil(n / TN) tiles.
template <bool FP4, int TN>
static int launch_gemm(const B2Maps& maps, const B2Params& prm, cudaStream_t stream) {
  const int smem = B2Layout<TN>::kSmem;
  cudaError_t e = cudaFuncSetAttribute(b2_gemm_kernel<FP4, TN>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
  const dim3 grid((unsigned)((prm.n + kTile - 1) / kTile), (unsigned)((prm.n + TN - 1) / TN));
  b2_gemm_kernel<FP4, TN><<<grid, B2Layout<TN>::kThreads, smem, stream>>>(maps, prm);
  return check_launch("b2_gemm_kernel");
}

// Target-tile width for n genes on `sms` SMs: the one whose tiles (one CTA per
// SM at a time) finish in the fewest tile-rows, counting each tile's fixed
// pipeline fill as 16 rows; ties go to the wider tile. n = 2,000 on 148 SMs:
// TN = 112 (288 tiles, two rounds of 112 rows) against TN = 128 (256 tiles, two
// rounds of 128 rows).
static int pick_tile_n(int n, int sms) {
  const int64_t src_tiles = (n + kTile - 1) / kTile;
  int best = kTileN[0];
  int64_t best_cost = INT64_MAX;
  for (int tn : kTileN) {
    const int64_t tiles = src_tiles * ((n + tn - 1) / tn);
    const int64_t rounds = (tiles + sms - 1) / (sms > 0 ? sms : 1);
    const int64_t cost = rounds * (tn + 16);
    if (cost < best_cost) {
      best_cost = cost;
      best = tn;
    }
  }
  return best;
}

extern "C" int tenex_te_binary_matrix_ex(const uint8_t* bins, int64_t ld, int n_vars,
                                         int64_t row_len, int64_t lag, float* out,
                                         int64_t out_ld, void* workspace, size_t workspace_bytes,
                                         int kind, int tile_n, void* stream_) {
  cudaStream_t stream = as_stream(stream_);
  if (!bins || !out || !workspace) return fail(TENEX_ERR_BADARG, "bins, out, workspace non-NULL");
  if (n_vars < 2) return fail(TENEX_ERR_BADARG, "n_vars must be >= 2");
  if (lag < 1 || row_len <= lag)
    return fail(TENEX_ERR_BADARG, "need 1 <= lag < row_len");
  if (ld < row_len) return fail(TENEX_ERR_BADARG, "ld must be >= row_len");
  if ((ld & 15) || (reinterpret_cast<uintptr_t>(bins) & 15))
    return fail(TENEX_ERR_BADARG, "bins and ld must be 16-byte aligned");
  if (out_ld < n_vars) return fail(TENEX_ERR_BADARG, "out_ld must be >= n_vars");
  if (kind < 0 || kind > 2)
    return fail(TENEX_ERR_BADARG, "kind must be 0 (default), 1 (int8) or 2 (4-bit)");
  if (tile_n != 0 && std::find(std::begin(kTileN), std::end(kTileN), tile_n) == std::end(kTileN))
    return fail(TENEX_ERR_BADARG, "tile_n must be 0 (automatic) or one of 128, 112, 96, 80, 64");
  DevAttr A;
  const int ast = current_device_attr(&A);
  if (ast) return ast;
  const int tn = tile_n != 0 ? tile_n : pick_tile_n(n_vars, A.sm_count);
  const bool fp4 = kind != 1;
  const int64_t L = row_len - lag;
  if (L >= ((int64_t)1 << 24))
    return fail(TENEX_ERR_UNSUPPORTED, "L=%lld: float32 cell counts are exact only below 2^24",
                (long long)L);
  const int64_t Lpad = round_up(L, fp4 ? 2 * kKt : kKt);
  if ((int64_t)workspace_bytes < (int64_t)tenex_b2_workspace_bytes(n_vars, row_len, lag))
    return fail(TENEX_ERR_OOM, "workspace too small (tenex_b2_workspace_bytes)");
  if ((reinterpret_cast<uintptr_t>(workspace) & 255) != 0)
    return fail(TENEX_ERR_BADARG, "workspace must be 256-byte aligned");
  unsigned char* ws = reinterpret_cast<unsigned char*>(workspace);
  uint8_t* ops = ws;
  const int64_t ob = b2_ops_bytes(n_vars, L);
  int32_t* marg = reinterpret_cast<int32_t*>(ws + ob);
  int* err = reinterpret_cast<int*>(ws + ob + round_up(3 * (int64_t)n_vars * 4, 256));
  // the per-gene counts (accumulated by the pack) and the error word, in one memset
  cudaError_t e = cudaMemsetAsync(marg, 0, (size_t)((unsigned char*)err - (unsigned char*)marg) +
                                               sizeof(int), stream);
  if (e != cudaSuccess) return check_cuda(e, "memset");
  const int seg = fp4 ? PackChunk<true>::kSeg : PackChunk<false>::kSeg;
  const int nseg = (int)((Lpad + seg - 1) / seg);
  const int64_t pack_warps = (int64_t)n_vars * nseg;
  const unsigned pack_grid = (unsigned)((pack_warps + kPackWarps - 1) / kPackWarps);
  if (fp4)
    b2_pack_kernel<true><<<pack_grid, kPackWarps * 32, 0, stream>>>(
        bins, ld, n_vars, (int)L, (int)lag, (int)Lpad, nseg, ops, marg, err);
  else
    b2_pack_kernel<false><<<pack_grid, kPackWarps * 32, 0, stream>>>(
        bins, ld, n_vars, (int)L, (int)lag, (int)Lpad, nseg, ops, marg, err);
  int st = check_launch("b2_pack_kernel");
  if (st) return st;
  B2Maps maps;
  if (fp4) {
    const int64_t rb = Lpad / 2;
    if ((st = make_map(&maps.F, ops, n_vars, rb, rb, tn))) return st;
    if ((st = make_map(&maps.FP, ops + (int64_t)n_vars * rb, n_vars, rb, rb, tn))) return st;
    if ((st = make_map(&maps.Pt, ops + 2 * (int64_t)n_vars * rb, n_vars, rb, rb, tn))) return st;
    if ((st = make_map(&maps.Ps, ops + 2 * (int64_t)n_vars * rb, n_vars, rb, rb, kTile)))
      return st;
  } else {
    if ((st = make_map(&maps.F, ops, n_vars, Lpad, Lpad, tn))) return st;
    if ((st = make_map(&maps.Pt, bins, n_vars, L, ld, tn))) return st;
    if ((st = make_map(&maps.Ps, bins, n_vars, L, ld, kTile))) return st;
    if ((st = make_map(&maps.FP, ops + (int64_t)n_vars * Lpad, n_vars, Lpad, Lpad, tn))) return st;
  }
  B2Params prm;
  prm.n = n_vars;
  prm.L = (int)L;
  prm.Lpad = (int)Lpad;
  prm.marg = marg;
  prm.out = out;
  prm.out_ld = out_ld;
  prm.vec_out = (out_ld % 4 == 0 && (reinterpret_cast<uintptr_t>(out) & 15) == 0) ? 1 : 0;
  prm.err = err;
  switch (tn) {
    case 128: return fp4 ? launch_gemm<true, 128>(maps, prm, stream)
                         : launch_gemm<false, 128>(maps, prm, stream);
    case 112: return fp4 ? launch_gemm<true, 112>(maps, prm, stream)
                         : launch_gemm<false, 112>(maps, prm, stream);
    case 96: return fp4 ? launch_gemm<true, 96>(maps, prm, stream)
                        : launch_gemm<false, 96>(maps, prm, stream);
    case 80: return fp4 ? launch_gemm<true, 80>(maps, prm, stream)
                        : launch_gemm<false, 80>(maps, prm, stream);
    default: return fp4 ? launch_gemm<true, 64>(maps, prm, stream)
                        : launch_gemm<false, 64>(maps, prm, stream);
  }
}

extern "C" int tenex_b2_tile_n(int n_vars, int* tile_n) {
  if (n_vars < 2 || !tile_n) return fail(TENEX_ERR_BADARG, "n_vars >= 2, tile_n non-NULL");
  DevAttr A;
  const int st = current_device_attr(&A);
  if (st) return st;
  *tile_n = pick_tile_n(n_vars, A.sm_count);
  return TENEX_OK;
}

extern "C" int tenex_te_binary_matrix_kind(const uint8_t* bins, int64_t ld, int n_vars,
                                           int64_t row_len, int64_t lag, float* out,
                                           int64_t out_ld, void* workspace,
                                           size_t workspace_bytes, int kind, void* stream) {
  return tenex_te_binary_matrix_ex(bins, ld, n_vars, row_len, lag, out, out_ld, workspace,
                                   workspace_bytes, kind, 0, stream);
}

extern "C" int tenex_te_binary_matrix(const uint8_t* bins, int64_t ld, int n_vars, int64_t row_len,
                                      int64_t lag, float* out, int64_t out_ld, void* workspace,
                                      size_t workspace_bytes, void* stream) {
  return tenex_te_binary_matrix_kind(bins, ld, n_vars, row_len, lag, out, out_ld, workspace,
                                     workspace_bytes, 0, stream);
}

extern "C" int tenex_b2_status(const void* workspace, int n_vars, int64_t row_len, int64_t lag,
                               void* stream) {
  if (!workspace) return fail(TENEX_ERR_BADARG, "workspace is NULL");
  const int64_t L = row_len - lag;
  const unsigned char* ws = reinterpret_cast<const unsigned char*>(workspace);
  const int* err = reinterpret_cast<const int*>(ws + b2_ops_bytes(n_vars, L) +
                                                round_up(3 * (int64_t)n_vars * 4, 256));
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, as_stream(stream));
  if (e == cudaSuccess) e = cudaStreamSynchronize(as_stream(stream));
  if (e != cudaSuccess) return check_cuda(e, "tenex_b2_status");
  if (h == 2) return fail(TENEX_ERR_BADDATA, "binary bins must be 0 or 1; results invalid");
  if (h) return fail(TENEX_ERR_TIMEOUT, "a tensor-core pipeline wait expired; results invalid");
  return TENEX_OK;
}
