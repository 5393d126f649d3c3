// tcgen05.cuh — inline-PTX helpers for the 5th-generation tensor cores (sm_100a):
// mbarriers with bounded waits, TMA 2-D tile loads (no multicast), shared-memory
// matrix descriptors, kind::i8 MMA issue and commit. Shared by the GEMM-B2 kernel
// and the tensor-pipe roofline probe.
#pragma once
#include <cuda.h>
#include <stdint.h>

namespace tenex {

constexpr uint32_t kSpinLimit = 1u << 22;  // bounded mbarrier polling (seconds at most)

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

// Polls the phase `parity` of an mbarrier at most kSpinLimit times; false on expiry.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// mbar_wait with a pause between polls, for warps that only wait (keeps them off
// the shared-memory pipe while the producer's copies land); same bound on polls.
__device__ __forceinline__ bool mbar_wait_sleep(uint64_t* bar, uint32_t parity, unsigned ns) {
  const uint32_t a = smem_u32(bar);
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
    __nanosleep(ns);
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, int x, int y,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, "
      "{%2, %3}], [%4];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(smem_u32(bar))
      : "memory");
}

// K-major SWIZZLE_NONE shared-memory descriptor (version 1 for sm_100):
// start >> 4 in [0,14), LBO >> 4 in [16,30), SBO >> 4 in [32,46), version 1 at [46,48).
__device__ __forceinline__ uint64_t smem_desc(uint32_t start, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((start >> 4) & 0x3fffu);
  d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
  d |= (uint64_t)1 << 46;
  return d;  // base_offset 0, lbo_mode 0, layout_type 0 (SWIZZLE_NONE)
}

// K-major SWIZZLE_128B shared-memory descriptor (sm_100 layout type 2 at [61,64)):
// rows of 128 bytes, 8-row groups 1024 bytes apart (SBO), LBO unused (16 bytes);
// the tile must be 1024-byte aligned. A K sub-step of 32 bytes inside the 128-byte
// swizzle row advances `start` by 32 bytes.
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t start) {
  uint64_t d = 0;
  d |= (uint64_t)((start >> 4) & 0x3fffu);
  d |= (uint64_t)1 << 16;                 // LBO = 16 bytes (ignored for this layout)
  d |= (uint64_t)(1024 >> 4) << 32;       // SBO = 1024 bytes
  d |= (uint64_t)1 << 46;                 // descriptor version for sm_100
  d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::i8: D s32 (bits 4-5 = 2), A/B unsigned 8-bit (0),
// K-major A and B, N >> 3 at bit 17, M >> 4 at bit 24.
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N) {
  return (2u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}

// Instruction descriptor, kind::mxf4 with block scales: A and B E2M1 (format 1
// at bits 7-9 and 10-12), K-major, N >> 3 at bit 17, UE8M0 scales (bit 23),
// M >> 4 at bit 24, scale-factor byte ids 0 (bits 4-5, 29-30), dense K = 64.
__host__ __device__ constexpr uint32_t idesc_mxf4(int M, int N) {
  return (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | (1u << 23) |
         ((uint32_t)(M >> 4) << 24);
}

// D += A * B with A, B packed E2M1 (two per byte, K = 64 per MMA = 32 bytes of a
// K-major row) and one UE8M0 scale per 32 elements read from TMEM at sfa / sfb;
// float32 accumulators.
__device__ __forceinline__ void mma_mxf4(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc,
                                         uint32_t idesc, uint32_t accumulate, uint32_t sfa,
                                         uint32_t sfb) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::mxf4.block_scale.block32 [%0], %1, %2, %3, [%5], [%6], "
      "p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(sfa), "r"(sfb)
      : "memory");
}

// Stores v into 8 consecutive TMEM columns starting at taddr for the 32 lanes of
// the calling warp's lane quarter (taddr's lane field = 32 * (warp % 4)).
__device__ __forceinline__ void tmem_st8(uint32_t taddr, uint32_t v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %1, %1, %1, %1, %1, %1, %1};" ::"r"(
          taddr),
      "r"(v)
      : "memory");
  asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// Plain arrival (release at CTA scope) on a shared-memory mbarrier.
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Orders this thread's earlier shared-memory stores before later reads by the
// async proxy (tcgen05.mma operand fetch, TMA stores).
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_u32(bar))
      : "memory");
}


}  // namespace tenex
