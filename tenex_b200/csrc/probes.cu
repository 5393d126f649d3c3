// probes.cu — microbenchmarks that measure the roofline denominators the TE
// kernels are judged against (no vendor figure exists for them):
//   mode 0: conflict-free shared-memory atomicAdd (int32): lane l of every warp
//           updates a word in bank l; all SMs, 1024 threads per CTA.
//   mode 1: the same with 16-bit halves (increment 1 or 1<<16), the TE kernel's
//           packed-counter form.
//   mode 2: uniformly random words in a 4096-word region (bank conflicts and
//           same-address collisions as random data produces them).
//   mode 3: lane-striped but every warp of the CTA updates the same 32 words
//           each time (no bank conflict inside an instruction, same addresses
//           across consecutive instructions).
// The entry point times the kernel with CUDA events on `stream` and returns the
// number of increments and the milliseconds (synchronises the stream).
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tenex {

__global__ void __launch_bounds__(1024, 1) smem_atomic_probe(int mode, int iters,
                                                             unsigned* sink) {
  __shared__ unsigned s[4096];
  const int tid = threadIdx.x;
  for (int i = tid; i < 4096; i += blockDim.x) s[i] = 0u;
  __syncthreads();
  const int lane = tid & 31, warp = tid >> 5;
  uint32_t x = 0x9e3779b9u * (uint32_t)(blockIdx.x * blockDim.x + tid + 1);
  if (mode == 0) {
#pragma unroll 8
    for (int i = 0; i < iters; ++i) atomicAdd(&s[lane + 32 * ((i + warp) & 127)], 1u);
  } else if (mode == 1) {
#pragma unroll 8
    for (int i = 0; i < iters; ++i)
      atomicAdd(&s[lane + 32 * ((i + warp) & 127)], 1u << ((i & 1) << 4));
  } else if (mode == 3) {
#pragma unroll 8
    for (int i = 0; i < iters; ++i) atomicAdd(&s[lane], 1u);
  } else {
#pragma unroll 8
    for (int i = 0; i < iters; ++i) {
      x ^= x << 13;
      x ^= x >> 17;
      x ^= x << 5;
      atomicAdd(&s[x & 4095u], 1u);
    }
  }
  __syncthreads();
  unsigned acc = 0;
  for (int i = tid; i < 4096; i += blockDim.x) acc += s[i];
  if (acc == 0xffffffffu) sink[0] = acc;  // keeps the work observable
}

}  // namespace tenex

using namespace tenex;

extern "C" int tenex_probe_smem_atomics(int mode, int iters, int64_t* increments, float* ms,
                                        void* stream_) {
  if (mode < 0 || mode > 3 || iters < 1 || !increments || !ms)
    return fail(TENEX_ERR_BADARG, "mode in 0..3, iters >= 1, outputs non-NULL");
  DevAttr A;
  int st = current_device_attr(&A);
  if (st) return st;
  cudaStream_t s = as_stream(stream_);
  unsigned* sink = nullptr;
  cudaError_t e = cudaMallocAsync(&sink, sizeof(unsigned), s);
  if (e != cudaSuccess) return check_cuda(e, "cudaMallocAsync");
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  const int grid = A.sm_count, block = 1024;
  smem_atomic_probe<<<grid, block, 0, s>>>(mode, iters, sink);  // warm-up
  cudaEventRecord(e0, s);
  smem_atomic_probe<<<grid, block, 0, s>>>(mode, iters, sink);
  cudaEventRecord(e1, s);
  st = check_launch("smem_atomic_probe");
  e = cudaEventSynchronize(e1);
  if (!st && e != cudaSuccess) st = check_cuda(e, "cudaEventSynchronize");
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFreeAsync(sink, s);
  *ms = t;
  *increments = (int64_t)grid * block * iters;
  return st;
}
