// gemm_b2.cu — binary (b_max = 2) TE matrix on the 5th-generation tensor cores.
//
// Reference: tenex/kernels/gemm_b2.py:307-425 (three FP32 cuBLAS GEMMs
// C = fp.p^T, D = p.p^T, E = f.p^T, with f = x[:, tau:], p = x[:, :-tau],
// fp = f*p) and the Triton epilogue :65-187 (8 joint cells from C, D, E and
// per-gene marginals, then sum c*log2(c*c1/(c2a*c2b)) / N).
//
// B200 design:
//   * pack kernel: one pass over the bins writes the lag-shifted K-major int8
//     operand F and FP = F & P (rows padded to a multiple of 128 bytes, zero
//     filled), the per-gene counts nf, np, nfp, and flags any bin other than
//     0/1; P is the bins themselves (a tensor map with K extent L, TMA zero-fills
//     beyond it).
//   * GEMM kernel: one CTA per 128 x 128 (target x source) tile of the matrix.
//     A producer warp brings, per stage, one 128-byte x 128-row box of FP, P, F
//     (targets) and P (sources) by TMA (cp.async.bulk.tensor.2d, no multicast),
//     128-byte swizzled (the K-major SWIZZLE_128B layout the MMA descriptors
//     name); a separate MMA warp issues, per 32-byte K step, two
//     tcgen05.mma.kind::i8 with the source tile as A (M = 128 lanes = sources):
//     B = [FP; P] of the targets as one N = 256 MMA (C^T, D^T) and B = F at
//     N = 128 (E^T), int32 accumulators in TMEM (384 columns). Shared-memory
//     bandwidth (operand reads plus TMA writes) bounds the main loop, hence the
//     source tile read twice per K step rather than three times. The counts are
//     exact integers (int32, N < 2^31).
//   * Epilogue: sixteen warps; warp w reads TMEM lanes 32*(w%4).. (one source
//     per lane) and a quarter of the 128 target columns with tcgen05.ld, forms
//     the 8 cells (target marginals staged in shared memory) and writes
//     TE(src -> tgt) to out[src, tgt], four consecutive targets of a source row
//     per 16-byte store.
//   * Every mbarrier wait is bounded; on expiry the kernel records an error
//     word, drains the copies it issued (bounded), frees TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "common.cuh"
#include "tcgen05.cuh"

namespace tenex {
namespace {

constexpr int kTile = 128;     // M = N = 128
constexpr int kKt = 128;       // bytes of K per pipeline stage (4 MMA K-steps of 32)
constexpr int kStages = 3;
constexpr int kOpBytes = kKt * kTile;          // one operand tile per stage (16 KB)
constexpr int kStageBytes = 4 * kOpBytes;      // FP, P, F (targets) + P (sources)
constexpr int kTmaBytes = kStageBytes;          // all four by TMA
constexpr int kTmemCols = 512;

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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
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
// ratio by approximate division (2 ulp) and lg2.approx, far below the 1e-6 TE budget.
__device__ __forceinline__ float cell_term(float c, float c1, float c2a, float c2b) {
  const float num = c * c1, den = c2a * c2b;
  const float r = (c > 0.f && num != den) ? __fdividef(num, den) : 1.f;
  return c * __log2f(r);
}

// Pack: F[g, t] = x[g, t+lag] (the lag-shifted operand TMA cannot address: its
// copies start on 16-byte boundaries) and FP = F & P for t < L (0 beyond, up to
// Lpad), plus the per-gene counts nf, np, nfp; P = x[g, t] is read from the bins
// directly. One warp per gene, kPackWarps genes per CTA, so the counts reduce
// with shuffles alone (no CTA barrier). Each lane makes 16 bytes of F and FP
// from two aligned 16-byte loads, two chunks per pass with all six loads issued
// before the first store; a scalar path covers the row end.
// Every bin must be 0 or 1 (the GEMM sums the raw bytes): a larger value sets
// the error word to 2.
constexpr int kPackWarps = 4;

__global__ void __launch_bounds__(kPackWarps * 32)
b2_pack_kernel(const uint8_t* __restrict__ bins, int64_t ld, int n, int L, int lag, int Lpad,
               uint8_t* __restrict__ ops, int32_t* __restrict__ marg, int* __restrict__ err) {
  const int g = blockIdx.x * kPackWarps + (threadIdx.x >> 5);
  if (g >= n) return;  // whole warps only: the shuffles below see full warps
  const int lane = threadIdx.x & 31;
  const uint8_t* row = bins + (int64_t)g * ld;
  uint8_t* Fr = ops + (int64_t)g * Lpad;
  uint8_t* FPr = ops + ((int64_t)n + g) * Lpad;
  int nf = 0, np = 0, nfp = 0;
  uint32_t high = 0;  // any bit above bit 0 of a byte: a bin other than 0/1
  const int sh = lag & 15;
  for (int t0 = lane * 16; t0 < Lpad; t0 += 2 * 32 * 16) {
    uint4 pv[2], av[2], bv[2];
    bool fast[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = t0 + u * 32 * 16;
      const int64_t fa = (int64_t)(t + lag) & ~(int64_t)15;  // aligned start of F's window
      fast[u] = t + 16 <= L && fa + 32 <= ld;
      if (fast[u]) {
        pv[u] = *reinterpret_cast<const uint4*>(row + t);
        av[u] = *reinterpret_cast<const uint4*>(row + fa);
        bv[u] = *reinterpret_cast<const uint4*>(row + fa + 16);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = t0 + u * 32 * 16;
      if (t >= Lpad) break;
      uint32_t f[4], p[4];
      if (fast[u]) {
        const uint32_t w[8] = {av[u].x, av[u].y, av[u].z, av[u].w,
                               bv[u].x, bv[u].y, bv[u].z, bv[u].w};
        const uint32_t pw[4] = {pv[u].x, pv[u].y, pv[u].z, pv[u].w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          // bytes sh + 4k .. sh + 4k + 3 of the 32-byte window
          const int byte = sh + 4 * k;
          const uint32_t lo = w[byte >> 2], hi = w[(byte >> 2) + 1];
          f[k] = __funnelshift_r(lo, hi, (byte & 3) * 8);
          p[k] = pw[k];
        }
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
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
      for (int k = 0; k < 4; ++k) high |= (f[k] | p[k]) & 0xfefefefeu;
      *reinterpret_cast<uint4*>(Fr + t) = make_uint4(f[0], f[1], f[2], f[3]);
      *reinterpret_cast<uint4*>(FPr + t) =
          make_uint4(f[0] & p[0], f[1] & p[1], f[2] & p[2], f[3] & p[3]);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        nf += __popc(f[k]);
        np += __popc(p[k]);
        nfp += __popc(f[k] & p[k]);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nf += __shfl_xor_sync(0xffffffffu, nf, o);
    np += __shfl_xor_sync(0xffffffffu, np, o);
    nfp += __shfl_xor_sync(0xffffffffu, nfp, o);
  }
  if (lane < 3) marg[(int64_t)lane * n + g] = lane == 0 ? nf : (lane == 1 ? np : nfp);
  if (__any_sync(0xffffffffu, high != 0) && lane == 0) atomicExch(err, 2);
}

// 4-bit form of the pack: F, FP and P as packed E2M1 values (1.0 = 0x2, 0.0 =
// 0x0; sample 2k in the low nibble of byte k, 2k + 1 in the high one), rows of
// Lpad / 2 bytes (Lpad a multiple of 256: whole 128-byte TMA boxes), the same
// per-gene counts and the same 0/1 check. Each lane makes 16 bytes of each
// operand from 32 samples (two aligned 16-byte loads of P and a 48-byte aligned
// window of F), two such chunks per pass with all their loads in flight.
__device__ __forceinline__ uint32_t e2m1_nibbles(uint32_t w) {
  // four 0/1 bytes b0..b3 -> 16 bits: 2*b0 | 2*b1 << 4 | 2*b2 << 8 | 2*b3 << 12
  const uint32_t t = (w | (w >> 4)) & 0x00ff00ffu;
  return __byte_perm(t, 0, 0x4420) << 1;
}

__global__ void __launch_bounds__(kPackWarps * 32)
b2_pack4_kernel(const uint8_t* __restrict__ bins, int64_t ld, int n, int L, int lag, int Lpad,
                uint8_t* __restrict__ ops, int32_t* __restrict__ marg, int* __restrict__ err) {
  const int g = blockIdx.x * kPackWarps + (threadIdx.x >> 5);
  if (g >= n) return;  // whole warps only: the shuffles below see full warps
  const int lane = threadIdx.x & 31;
  const int64_t rowb = Lpad / 2;
  const uint8_t* row = bins + (int64_t)g * ld;
  uint8_t* Fr = ops + (int64_t)g * rowb;
  uint8_t* FPr = ops + ((int64_t)n + g) * rowb;
  uint8_t* Pr = ops + (2 * (int64_t)n + g) * rowb;
  int nf = 0, np = 0, nfp = 0;
  uint32_t high = 0;
  for (int t0 = lane * 32; t0 < Lpad; t0 += 2 * 32 * 32) {
    // two 32-sample chunks per pass, all ten loads issued before the first store
    uint4 pv[2][2], av[2][3];
    bool fast[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = t0 + u * 32 * 32;
      const int64_t fa = (int64_t)(t + lag) & ~(int64_t)15;
      fast[u] = t + 32 <= L && fa + 48 <= ld;
      if (fast[u]) {
        pv[u][0] = *reinterpret_cast<const uint4*>(row + t);
        pv[u][1] = *reinterpret_cast<const uint4*>(row + t + 16);
        av[u][0] = *reinterpret_cast<const uint4*>(row + fa);
        av[u][1] = *reinterpret_cast<const uint4*>(row + fa + 16);
        av[u][2] = *reinterpret_cast<const uint4*>(row + fa + 32);
      }
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int t = t0 + u * 32 * 32;
      if (t >= Lpad) break;
      uint32_t f[8], p[8];
      if (fast[u]) {
        const uint32_t w[12] = {av[u][0].x, av[u][0].y, av[u][0].z, av[u][0].w,
                                av[u][1].x, av[u][1].y, av[u][1].z, av[u][1].w,
                                av[u][2].x, av[u][2].y, av[u][2].z, av[u][2].w};
        const uint32_t pw[8] = {pv[u][0].x, pv[u][0].y, pv[u][0].z, pv[u][0].w,
                                pv[u][1].x, pv[u][1].y, pv[u][1].z, pv[u][1].w};
        const int sh = (t + lag) & 15;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const int byte = sh + 4 * k;
          f[k] = __funnelshift_r(w[byte >> 2], w[(byte >> 2) + 1], (byte & 3) * 8);
          p[k] = pw[k];
        }
      } else {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
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
      uint32_t of[4], ofp[4], op[4];
#pragma unroll
      for (int k = 0; k < 8; ++k) {
        high |= (f[k] | p[k]) & 0xfefefefeu;
        nf += __popc(f[k]);
        np += __popc(p[k]);
        nfp += __popc(f[k] & p[k]);
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        of[k] = e2m1_nibbles(f[2 * k]) | (e2m1_nibbles(f[2 * k + 1]) << 16);
        ofp[k] = e2m1_nibbles(f[2 * k] & p[2 * k]) |
                 (e2m1_nibbles(f[2 * k + 1] & p[2 * k + 1]) << 16);
        op[k] = e2m1_nibbles(p[2 * k]) | (e2m1_nibbles(p[2 * k + 1]) << 16);
      }
      *reinterpret_cast<uint4*>(Fr + t / 2) = make_uint4(of[0], of[1], of[2], of[3]);
      *reinterpret_cast<uint4*>(FPr + t / 2) = make_uint4(ofp[0], ofp[1], ofp[2], ofp[3]);
      *reinterpret_cast<uint4*>(Pr + t / 2) = make_uint4(op[0], op[1], op[2], op[3]);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    nf += __shfl_xor_sync(0xffffffffu, nf, o);
    np += __shfl_xor_sync(0xffffffffu, np, o);
    nfp += __shfl_xor_sync(0xffffffffu, nfp, o);
  }
  if (lane < 3) marg[(int64_t)lane * n + g] = lane == 0 ? nf : (lane == 1 ? np : nfp);
  if (__any_sync(0xffffffffu, high != 0) && lane == 0) atomicExch(err, 2);
}

// Tensor maps of the operands: F and FP (packed, n x Lpad) and P (the bins
// themselves, n x L with row stride ld; TMA fills columns >= L and rows >= n
// with zeros). The 4-bit form has all three packed (rows of Lpad / 2 bytes).
struct B2Maps {
  CUtensorMap F, P, FP;
};

constexpr int kB2Threads = 512;
// 4-bit form: TMEM columns of the UE8M0 scale factors (all 1.0), after the
// three 128-column accumulators: A (sources, M = 128) at kSfaCol, B (targets,
// up to N = 256) at kSfbCol; 8 columns each hold every layout those take.
constexpr uint32_t kSfaCol = 384, kSfbCol = 392;

// FP4 = false: kind::i8 MMAs on the int8 operands (K = 32 per MMA), int32 sums.
// FP4 = true: kind::mxf4 MMAs on the packed E2M1 operands (K = 64 per MMA, two
// samples per byte: half the shared-memory bytes per multiply), unit block
// scales, float32 sums (exact integers below 2^24).
template <bool FP4>
__global__ void __launch_bounds__(kB2Threads, 1)
    b2_gemm_kernel(const __grid_constant__ B2Maps maps, B2Params prm) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte align the operand region
  unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
  unsigned char* stage_base = smem;
  uint64_t* full = reinterpret_cast<uint64_t*>(smem + kStages * kStageBytes);
  uint64_t* empty = full + kStages;
  uint64_t* accbar = empty + kStages;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(accbar + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  // the tile's target marginals nf, np, nfp as floats (epilogue operands)
  float* tmarg = reinterpret_cast<float*>(smem + kStages * kStageBytes + 256);

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int m0 = blockIdx.y * kTile;  // targets
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
      mbar_expect_tx(&full[s], kTmaBytes);
      const int x0 = k * kKt;
      // one 128-byte x 128-row box per operand, 128-byte swizzled
      tma_load_2d(buf + 0 * kOpBytes, &maps.FP, x0, m0, &full[s]);
      tma_load_2d(buf + 1 * kOpBytes, &maps.P, x0, m0, &full[s]);
      tma_load_2d(buf + 2 * kOpBytes, &maps.F, x0, m0, &full[s]);
      tma_load_2d(buf + 3 * kOpBytes, &maps.P, x0, n0, &full[s]);
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
  // (20 KB of shared memory instead of 24; shared-memory bandwidth bounds the
  // main loop). TMEM columns 0-127 = C^T, 128-255 = D^T, 256-383 = E^T.
  if (tid == 32) {
    const uint32_t idesc256 = FP4 ? idesc_mxf4(kTile, 2 * kTile) : idesc_i8(kTile, 2 * kTile);
    const uint32_t idesc128 = FP4 ? idesc_mxf4(kTile, kTile) : idesc_i8(kTile, kTile);
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
      const uint32_t bFPP = smem_u32(buf + 0 * kOpBytes);  // FP_i rows, then P_i rows
      const uint32_t bF = smem_u32(buf + 2 * kOpBytes);
      const uint32_t aPj = smem_u32(buf + 3 * kOpBytes);
#pragma unroll
      for (int kk = 0; kk < kKt / 32; ++kk) {
        const uint32_t off = kk * 32;  // 32-byte K step inside the 128-byte swizzle row
        const uint64_t ad = smem_desc_sw128(aPj + off);
        const uint32_t acc = (k > 0 || kk > 0) ? 1u : 0u;
        if (FP4) {
          mma_mxf4(tmem + 0, ad, smem_desc_sw128(bFPP + off), idesc256, acc, tmem + kSfaCol,
                   tmem + kSfbCol);
          mma_mxf4(tmem + 256, ad, smem_desc_sw128(bF + off), idesc128, acc, tmem + kSfaCol,
                   tmem + kSfbCol);
        } else {
          mma_i8(tmem + 0, ad, smem_desc_sw128(bFPP + off), idesc256, acc);
          mma_i8(tmem + 256, ad, smem_desc_sw128(bF + off), idesc128, acc);
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

  // ---- epilogue: 16 warps; lane quarter warp % 4, column quarter warp / 4 ---
  // (the warps that neither load nor issue stage the target marginals first)
  if (tid >= 64) {
    for (int k = tid - 64; k < 3 * kTile; k += kB2Threads - 64) {
      const int c = k / kTile, i = m0 + (k - c * kTile);
      tmarg[k] = i < prm.n ? (float)prm.marg[(int64_t)c * prm.n + i] : 0.f;
    }
  }
  bool ok_acc = mbar_wait_sleep(accbar, 0, 200);
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!ok_acc && tid == 0) atomicExch(prm.err, 1);
  const bool run = ok_acc && (*(volatile int*)abort_flag == 0);
  const int lq = warp & 3, cq = warp >> 2;
  const int j = n0 + lq * 32 + (tid & 31);  // source gene of this thread's TMEM lane
  const float N = (float)prm.L;
  const float invL = 1.0f / N;
  const float npj = j < prm.n ? (float)prm.marg[prm.n + j] : 0.f;
  const uint32_t lane_base = tmem + ((uint32_t)(lq * 32) << 16);
  for (int cb = cq * (kTile / 4); cb < (cq + 1) * (kTile / 4); cb += 16) {
    uint32_t rc[16], rd[16], re[16];
    tmem_ld16(lane_base + 0 + cb, rc);
    tmem_ld16(lane_base + 128 + cb, rd);
    tmem_ld16(lane_base + 256 + cb, re);
    tmem_wait_ld();
    if (!run || j >= prm.n) continue;
    const int i0 = m0 + cb;  // first target of the 16 (the same for every lane: broadcast loads)
    float* orow = prm.out + (int64_t)j * prm.out_ld;
#pragma unroll
    for (int q0 = 0; q0 < 16; q0 += 4) {
      float res[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int q = q0 + u;
        const int ti = cb + q;  // target within the tile (marginals 0 beyond n)
        const float nf = tmarg[ti], np_ = tmarg[kTile + ti], nfp = tmarg[2 * kTile + ti];
        const float c1_1 = np_, c1_0 = N - np_;
        const float c2a11 = nfp, c2a01 = np_ - nfp, c2a10 = nf - nfp, c2a00 = N - nf - np_ + nfp;
        const float C = FP4 ? __uint_as_float(rc[q]) : (float)rc[q];
        const float Dv = FP4 ? __uint_as_float(rd[q]) : (float)rd[q];
        const float E = FP4 ? __uint_as_float(re[q]) : (float)re[q];
        const float c2b11 = Dv, c2b01 = npj - Dv, c2b10 = np_ - Dv, c2b00 = N - np_ - npj + Dv;
        float te = 0.f;
        te += cell_term(C, c1_1, c2a11, c2b11);                                   // [1,1,1]
        te += cell_term(Dv - C, c1_1, c2a01, c2b11);                              // [0,1,1]
        te += cell_term(E - C, c1_0, c2a10, c2b01);                               // [1,0,1]
        te += cell_term(npj - Dv - E + C, c1_0, c2a00, c2b01);                    // [0,0,1]
        te += cell_term(nfp - C, c1_1, c2a11, c2b10);                             // [1,1,0]
        te += cell_term(np_ - Dv - nfp + C, c1_1, c2a01, c2b10);                  // [0,1,0]
        te += cell_term(nf - E - nfp + C, c1_0, c2a10, c2b00);                    // [1,0,0]
        te += cell_term(N - nf - np_ - npj + nfp + Dv + E - C, c1_0, c2a00, c2b00);  // [0,0,0]
        res[u] = te * invL;
      }
      // four consecutive targets of row j: one 16-byte store when they are all
      // inside the matrix, off the diagonal and aligned; else one by one
      const int ia = i0 + q0;
      if (prm.vec_out && ia + 4 <= prm.n && (j < ia || j >= ia + 4)) {
        *reinterpret_cast<float4*>(orow + ia) = make_float4(res[0], res[1], res[2], res[3]);
      } else {
#pragma unroll
        for (int u = 0; u < 4; ++u)
          if (ia + u < prm.n && ia + u != j) orow[ia + u] = res[u];
      }
    }
  }
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
                    int64_t stride) {
  EncodeTiledFn enc = encode_fn();
  if (!enc) return fail(TENEX_ERR_UNSUPPORTED, "cuTensorMapEncodeTiled is unavailable");
  const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
  const cuuint64_t strides[1] = {(cuuint64_t)stride};
  const cuuint32_t box[2] = {(cuuint32_t)kKt, (cuuint32_t)kTile};
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

extern "C" int tenex_te_binary_matrix_kind(const uint8_t* bins, int64_t ld, int n_vars,
                                           int64_t row_len, int64_t lag, float* out,
                                           int64_t out_ld, void* workspace,
                                           size_t workspace_bytes, int kind, void* stream_) {
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
  cudaError_t e = cudaMemsetAsync(err, 0, sizeof(int), stream);
  if (e != cudaSuccess) return check_cuda(e, "memset");
  const int pack_grid = (n_vars + kPackWarps - 1) / kPackWarps;
  if (fp4)
    b2_pack4_kernel<<<pack_grid, kPackWarps * 32, 0, stream>>>(bins, ld, n_vars, (int)L,
                                                                (int)lag, (int)Lpad, ops, marg,
                                                                err);
  else
    b2_pack_kernel<<<pack_grid, kPackWarps * 32, 0, stream>>>(bins, ld, n_vars, (int)L, (int)lag,
                                                               (int)Lpad, ops, marg, err);
  int st = check_launch("b2_pack_kernel");
  if (st) return st;
  B2Maps maps;
  if (fp4) {
    const int64_t rb = Lpad / 2;
    if ((st = make_map(&maps.F, ops, n_vars, rb, rb))) return st;
    if ((st = make_map(&maps.FP, ops + (int64_t)n_vars * rb, n_vars, rb, rb))) return st;
    if ((st = make_map(&maps.P, ops + 2 * (int64_t)n_vars * rb, n_vars, rb, rb))) return st;
  } else {
    if ((st = make_map(&maps.F, ops, n_vars, Lpad, Lpad))) return st;
    if ((st = make_map(&maps.P, bins, n_vars, L, ld))) return st;
    if ((st = make_map(&maps.FP, ops + (int64_t)n_vars * Lpad, n_vars, Lpad, Lpad))) return st;
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
  const int smem = kStages * kStageBytes + 1024 + 256 + 3 * kTile * 4;
  const unsigned tiles = (unsigned)((n_vars + kTile - 1) / kTile);
  if (fp4) {
    e = cudaFuncSetAttribute(b2_gemm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
    b2_gemm_kernel<true><<<dim3(tiles, tiles), kB2Threads, smem, stream>>>(maps, prm);
  } else {
    e = cudaFuncSetAttribute(b2_gemm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             smem);
    if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
    b2_gemm_kernel<false><<<dim3(tiles, tiles), kB2Threads, smem, stream>>>(maps, prm);
  }
  return check_launch("b2_gemm_kernel");
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
