// runtime.cu — status/error text, device attributes, and the small data-movement
// kernels of the C ABI (block shuffle).
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <mutex>

#include "common.cuh"

namespace tenex {

static thread_local char g_last_error[1024] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return code;
}

int check_cuda(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return TENEX_OK;
  return fail(TENEX_ERR_LAUNCH, "%s: %s (%s)", what, cudaGetErrorString(e),
              cudaGetErrorName(e));
}

int check_launch(const char* what) { return check_cuda(cudaGetLastError(), what); }

int current_device_attr(DevAttr* out) {
  static std::mutex mu;
  static DevAttr cache[64];
  static bool have[64] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return check_cuda(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return fail(TENEX_ERR_UNSUPPORTED, "device index %d", dev);
  std::lock_guard<std::mutex> lk(mu);
  if (!have[dev]) {
    DevAttr a{};
    e = cudaDeviceGetAttribute(&a.sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&a.smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&a.smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor,
                                 dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&a.l2_bytes, cudaDevAttrL2CacheSize, dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&a.max_threads_per_sm,
                                 cudaDevAttrMaxThreadsPerMultiProcessor, dev);
    if (e != cudaSuccess) return check_cuda(e, "cudaDeviceGetAttribute");
    cache[dev] = a;
    have[dev] = true;
  }
  *out = cache[dev];
  return TENEX_OK;
}

// out[g, t*K+k] = in[g, (perm[g, t/bl]*bl + t%bl)*K + k] for t < n_blocks*bl; tail copied.
// With blK = bl*K bytes per block, byte i < head of a row maps to
// perm[g, i / blK] * blK + i % blK. Grid: (ceil(T*K / 4096), n_vars, copies); each
// thread gathers 16 consecutive output bytes (one 32-bit division, then a running
// block offset) and writes them as one 16-byte store when the row holds all 16
// (rows start on 16-byte boundaries, checked by the launcher), bytewise at the row
// end. row < 2^31 (checked). Copy s reads perm + s * perm_stride and writes
// out + s * out_stride.
__global__ void block_shuffle_kernel(const uint8_t* __restrict__ in, int64_t in_ld, int n,
                                     uint32_t row, uint32_t blK, uint32_t head,
                                     const int32_t* __restrict__ perm, int64_t perm_stride,
                                     int n_blocks, uint8_t* __restrict__ out, int64_t out_ld,
                                     int64_t out_stride) {
  const int g = blockIdx.y;
  const uint8_t* src = in + (int64_t)g * in_ld;
  uint8_t* dst = out + (int64_t)blockIdx.z * out_stride + (int64_t)g * out_ld;
  const int32_t* pg = perm + (int64_t)blockIdx.z * perm_stride + (int64_t)g * n_blocks;
  const uint32_t i0 = (blockIdx.x * blockDim.x + threadIdx.x) * 16u;
  if (i0 >= row) return;
  uint32_t b = i0 / blK, off = i0 - b * blK;
  uint32_t w[4] = {0u, 0u, 0u, 0u};
#pragma unroll
  for (uint32_t u = 0; u < 16u; ++u) {
    const uint32_t i = i0 + u;
    if (i < row) {
      uint32_t j = i;
      if (i < head) {
        uint32_t pb = (uint32_t)pg[b];
        if (pb >= (uint32_t)n_blocks) pb = b;  // out-of-range entry: identity
        j = pb * blK + off;
      }
      w[u >> 2] |= (uint32_t)src[j] << (8u * (u & 3u));
    }
    if (++off == blK) {
      off = 0;
      ++b;
    }
  }
  if (i0 + 16u <= row) {
    *reinterpret_cast<uint4*>(dst + i0) = make_uint4(w[0], w[1], w[2], w[3]);
  } else {
    for (uint32_t u = 0; i0 + u < row; ++u) dst[i0 + u] = (uint8_t)(w[u >> 2] >> (8u * (u & 3u)));
  }
}

// sum[m] += te[m]; sumsq[m] += te[m]^2 (float32 widened); count_ge[m] += te[m] >= obs[m],
// for m off the diagonal of an (n, n) matrix (the diagonal is handled by the caller).
__global__ void stats_accumulate_kernel(const float* __restrict__ te, const float* __restrict__ obs,
                                        double* __restrict__ sum, double* __restrict__ sumsq,
                                        int32_t* __restrict__ cnt, int n) {
  const int64_t total = (int64_t)n * n;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < total;
       m += (int64_t)gridDim.x * blockDim.x) {
    if (m / n == m % n) continue;
    const float t = te[m];
    const double d = (double)t;
    sum[m] += d;
    sumsq[m] += d * d;
    cnt[m] += t >= obs[m] ? 1 : 0;
  }
}

}  // namespace tenex

using namespace tenex;

extern "C" int tenex_stats_accumulate(const float* te, const float* observed, double* sum,
                                      double* sumsq, int32_t* count_ge, int n_vars, void* stream) {
  if (!te || !observed || !sum || !sumsq || !count_ge)
    return fail(TENEX_ERR_BADARG, "all pointers must be non-NULL");
  if (n_vars < 1) return fail(TENEX_ERR_BADARG, "n_vars must be >= 1");
  const int64_t total = (int64_t)n_vars * n_vars;
  const int64_t blocks64 = (total + 255) / 256;
  const int blocks = (int)(blocks64 < 4096 ? blocks64 : 4096);
  stats_accumulate_kernel<<<blocks, 256, 0, as_stream(stream)>>>(te, observed, sum, sumsq,
                                                                 count_ge, n_vars);
  return check_launch("stats_accumulate_kernel");
}

extern "C" int tenex_abi_version(void) { return 1; }

extern "C" int tenex_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return TENEX_ERR_BADARG;
  strncpy(buf, g_last_error, len - 1);
  buf[len - 1] = '\0';
  return TENEX_OK;
}

extern "C" int tenex_device_query(int device, tenex_dev_info* info) {
  if (!info) return fail(TENEX_ERR_BADARG, "info is NULL");
  int prev = 0;
  cudaError_t e = cudaGetDevice(&prev);
  if (e != cudaSuccess) return check_cuda(e, "cudaGetDevice");
  if (device != prev) {
    e = cudaSetDevice(device);
    if (e != cudaSuccess) return check_cuda(e, "cudaSetDevice");
  }
  DevAttr a;
  int st = current_device_attr(&a);
  int major = 0, minor = 0;
  if (st == TENEX_OK) {
    e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device);
    if (e != cudaSuccess) st = check_cuda(e, "cudaDeviceGetAttribute");
  }
  if (device != prev) cudaSetDevice(prev);
  if (st) return st;
  info->sm_count = a.sm_count;
  info->smem_optin = a.smem_optin;
  info->smem_per_sm = a.smem_per_sm;
  info->l2_bytes = a.l2_bytes;
  info->cc_major = major;
  info->cc_minor = minor;
  info->max_threads_per_sm = a.max_threads_per_sm;
  return TENEX_OK;
}

extern "C" int tenex_block_shuffle_many(const uint8_t* in, int64_t in_ld, int n_vars, int64_t T,
                                        int K, const int32_t* perms, int n_copies, int n_blocks,
                                        int block_length, uint8_t* out, int64_t out_ld,
                                        int64_t out_copy_stride, void* stream) {
  if (!in || !out || !perms) return fail(TENEX_ERR_BADARG, "in, out and perms must be non-NULL");
  if (n_vars < 1 || T < 1 || K < 1) return fail(TENEX_ERR_BADARG, "empty bins");
  if (n_copies < 1) return fail(TENEX_ERR_BADARG, "n_copies must be >= 1");
  if (block_length < 1 || n_blocks < 1 || (int64_t)n_blocks * block_length > T)
    return fail(TENEX_ERR_BADARG, "need n_blocks*block_length <= T (n_blocks=%d, bl=%d, T=%lld)",
                n_blocks, block_length, (long long)T);
  if (in_ld < T * K || out_ld < T * K)
    return fail(TENEX_ERR_BADARG, "row strides must be >= T*K");
  const int64_t copy_bytes = (int64_t)(n_vars - 1) * out_ld + T * K;
  if (n_copies > 1 && out_copy_stride < copy_bytes)
    return fail(TENEX_ERR_BADARG, "copies overlap (out_copy_stride %lld < %lld)",
                (long long)out_copy_stride, (long long)copy_bytes);
  const uint8_t* in_end = in + (int64_t)(n_vars - 1) * in_ld + T * K;
  const uint8_t* out_end = out + (int64_t)(n_copies - 1) * out_copy_stride + copy_bytes;
  if (in < out_end && out < in_end) return fail(TENEX_ERR_BADARG, "block shuffle cannot run in place");
  if ((reinterpret_cast<uintptr_t>(out) & 15) || (out_ld & 15) || (n_copies > 1 && (out_copy_stride & 15)))
    return fail(TENEX_ERR_BADARG, "out, out_ld and out_copy_stride must be 16-byte aligned");
  const int64_t row = T * K;
  if (row > 0x7fffffff - 4096)
    return fail(TENEX_ERR_UNSUPPORTED, "row of %lld bytes", (long long)row);
  const int64_t gx = (row + 4095) / 4096;
  if (n_vars > 65535 || n_copies > 65535)
    return fail(TENEX_ERR_UNSUPPORTED, "grid too large (n_vars=%d, copies=%d)", n_vars, n_copies);
  dim3 grid((unsigned)gx, (unsigned)n_vars, (unsigned)n_copies);
  block_shuffle_kernel<<<grid, 256, 0, as_stream(stream)>>>(
      in, in_ld, n_vars, (uint32_t)row, (uint32_t)(block_length * K),
      (uint32_t)((int64_t)n_blocks * block_length * K), perms, (int64_t)n_vars * n_blocks,
      n_blocks, out, out_ld, out_copy_stride);
  return check_launch("block_shuffle_kernel");
}

extern "C" int tenex_block_shuffle(const uint8_t* in, int64_t in_ld, int n_vars, int64_t T, int K,
                                   const int32_t* perm, int n_blocks, int block_length,
                                   uint8_t* out, int64_t out_ld, void* stream) {
  return tenex_block_shuffle_many(in, in_ld, n_vars, T, K, perm, 1, n_blocks, block_length, out,
                                  out_ld, 0, stream);
}
