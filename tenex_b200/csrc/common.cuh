// common.cuh — shared helpers of the sm_100a TE library: status/error text,
// device attributes, small device utilities.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "../../include/tenex_sm100.h"

namespace tenex {

// Records a formatted error message for tenex_last_error() on this thread and
// returns `code`, so entry points can write `return fail(TENEX_ERR_BADARG, ...)`.
int fail(int code, const char* fmt, ...);

// Converts a pending CUDA error (after a launch) into TENEX_ERR_LAUNCH.
int check_cuda(cudaError_t e, const char* what);
int check_launch(const char* what);

// Cached per-device attributes (queried once per device).
struct DevAttr {
  int sm_count;
  int smem_optin;
  int smem_per_sm;
  int l2_bytes;
  int max_threads_per_sm;
};
int current_device_attr(DevAttr* out);

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

__host__ __device__ inline int64_t round_up(int64_t x, int64_t m) { return (x + m - 1) / m * m; }

// Workspace layout shared by the TE entry points (all offsets 256-byte aligned).
//   [0]   uint32 work ticket of the persistent kernel
//   [4]   int32  data-validation word (nonzero = bad bin / n_per_var)
//   [8]   int32  unsupported-item word (nonzero = an item's histogram did not fit)
//   [12]  uint32 work ticket of the global-memory overflow launch
struct WsHeader {
  unsigned int ticket;
  int bad_data;
  int bad_item;
  unsigned int ov_ticket;
  int pad[60];
};
static_assert(sizeof(WsHeader) == 256, "workspace header is 256 bytes");

}  // namespace tenex

// ---- device helpers -------------------------------------------------------
namespace tenex {
namespace dev {

__device__ __forceinline__ uint4 ldg_nc_v4(const uint4* p) {
  uint4 r;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(r.x), "=r"(r.y), "=r"(r.z), "=r"(r.w)
               : "l"(p));
  return r;
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ unsigned warp_max(unsigned v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    unsigned w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// Named barrier over `nthreads` threads (a multiple of 32) with id in [1, 15].
__device__ __forceinline__ void named_bar(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

}  // namespace dev
}  // namespace tenex
