// dpi.cu — data-processing-inequality (DPI) trimming of a thresholded TE network.
//
// Replaces the row-batched torch loop of the FDR method's trimming step
// (tenex/inference/fdr.py:61-133). For the network matrix A (n x n, A[i][j] = TE
// of the kept edge i -> j, 0 elsewhere):
//   indirect[i][j] = max(0, max_{k mediator} min(A[i][k], A[k][j]))
//   out[i][j]      = keep_all[i] ? A[i][j]
//                                : (A[i][j] >= indirect[i][j] + thr ? A[i][j] : 0)
// The reference starts `indirect` at zero and takes the maximum over the
// mediators active in a row batch; a k whose column is zero in row i adds
// min(0, .) <= 0 and cannot raise the maximum, so the product over every
// mediator k gives the same values. keep_all marks the rows of batches with no
// active mediator, which the reference keeps unfiltered (fdr.py:98-104).
// min/max select one of their inputs, so the result is exact in float32.
//
// Dense form: the (max, min) product runs on the FP32 min/max pipe: 128 x 128 output tile
// per CTA, 8 x 8 per thread, K slices of 16 staged through double-buffered
// shared memory. Two k steps share one three-input max (sm_100 max.f32 with
// three sources): three min/max instructions per (i, j) and two k.
#include "common.cuh"

#include <math.h>

namespace tenex {
namespace {

constexpr int kTile = 128;
constexpr int kKc = 16;
constexpr int kThreads = 256;

struct DpiArgs {
  const float* a;
  int64_t lda;
  int n;
  const uint8_t* mediator;  // NULL: every k is a mediator
  const uint8_t* keep_all;  // NULL: no row is kept unfiltered
  float thr;
  float* out;
  int64_t ldo;
};

// Thread t stages A[i0 + t/2][k0 + (t%2)*8 + q] (q < 8) and A[k0 + t/16][j0 + (t%16)*8 + q];
// entries outside the matrix, and rows k that are no mediator, read as -inf so
// they never win the maximum.
__device__ __forceinline__ void load_slices(const DpiArgs& P, int i0, int j0, int k0, float ra[8],
                                            float rb[8]) {
  const int t = threadIdx.x;
  const int i = i0 + (t >> 1);
  const int ka = k0 + (t & 1) * 8;
  const int kb = k0 + (t >> 4);
  const int jb = j0 + (t & 15) * 8;
  const bool kb_ok = kb < P.n && (P.mediator == nullptr || P.mediator[kb] != 0);
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    ra[q] = (i < P.n && ka + q < P.n) ? __ldg(P.a + (int64_t)i * P.lda + ka + q) : -INFINITY;
    rb[q] = (kb_ok && jb + q < P.n) ? __ldg(P.a + (int64_t)kb * P.lda + jb + q) : -INFINITY;
  }
}

__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float r;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
  return r;
}

__global__ void __launch_bounds__(kThreads, 2) dpi_trim_kernel(DpiArgs P) {
  __shared__ __align__(16) float As[2][kKc][kTile];  // As[k][i] = A[i0 + i][k0 + k]
  __shared__ __align__(16) float Bs[2][kKc][kTile];  // Bs[k][j] = A[k0 + k][j0 + j]
  const int t = threadIdx.x;
  const int tx = t & 15, ty = t >> 4;
  const int i0 = blockIdx.y * kTile, j0 = blockIdx.x * kTile;

  float acc[8][8];
#pragma unroll
  for (int r = 0; r < 8; ++r)
#pragma unroll
    for (int c = 0; c < 8; ++c) acc[r][c] = 0.f;

  float ra[8] = {}, rb[8] = {};
  auto stage = [&](int buf) {
#pragma unroll
    for (int q = 0; q < 8; ++q) As[buf][(t & 1) * 8 + q][t >> 1] = ra[q];
    *reinterpret_cast<float4*>(&Bs[buf][t >> 4][(t & 15) * 8]) = make_float4(rb[0], rb[1], rb[2], rb[3]);
    *reinterpret_cast<float4*>(&Bs[buf][t >> 4][(t & 15) * 8 + 4]) =
        make_float4(rb[4], rb[5], rb[6], rb[7]);
  };

  load_slices(P, i0, j0, 0, ra, rb);
  stage(0);
  __syncthreads();
  const int nk = (P.n + kKc - 1) / kKc;
  for (int kc = 0; kc < nk; ++kc) {
    const int buf = kc & 1;
    if (kc + 1 < nk) load_slices(P, i0, j0, (kc + 1) * kKc, ra, rb);
#pragma unroll
    for (int k = 0; k < kKc; k += 2) {
      // rows ty*4..+3 and 64+ty*4..+3, columns tx*4..+3 and 64+tx*4..+3
      float bv[2][8];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const float4 b0 = *reinterpret_cast<const float4*>(&Bs[buf][k + h][tx * 4]);
        const float4 b1 = *reinterpret_cast<const float4*>(&Bs[buf][k + h][64 + tx * 4]);
        bv[h][0] = b0.x; bv[h][1] = b0.y; bv[h][2] = b0.z; bv[h][3] = b0.w;
        bv[h][4] = b1.x; bv[h][5] = b1.y; bv[h][6] = b1.z; bv[h][7] = b1.w;
      }
#pragma unroll
      for (int rh = 0; rh < 2; ++rh) {
        const float4 a0 = *reinterpret_cast<const float4*>(&As[buf][k][rh * 64 + ty * 4]);
        const float4 a1 = *reinterpret_cast<const float4*>(&As[buf][k + 1][rh * 64 + ty * 4]);
        const float av0[4] = {a0.x, a0.y, a0.z, a0.w};
        const float av1[4] = {a1.x, a1.y, a1.z, a1.w};
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
          for (int c = 0; c < 8; ++c)
            acc[rh * 4 + r][c] =
                fmax3(acc[rh * 4 + r][c], fminf(av0[r], bv[0][c]), fminf(av1[r], bv[1][c]));
      }
    }
    if (kc + 1 < nk) {
      stage(buf ^ 1);
      __syncthreads();
    }
  }

#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int i = i0 + (r < 4 ? ty * 4 + r : 64 + ty * 4 + (r - 4));
    if (i >= P.n) continue;
    const bool keep = P.keep_all != nullptr && P.keep_all[i] != 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int j = j0 + (c < 4 ? tx * 4 + c : 64 + tx * 4 + (c - 4));
      if (j >= P.n) continue;
      const float v = P.a[(int64_t)i * P.lda + j];
      const float ind = acc[r][c] + P.thr;
      P.out[(int64_t)i * P.ldo + j] = (keep || v >= ind) ? v : 0.f;
    }
  }
}

// ---- sparse form ------------------------------------------------------------
// Only positive A[i][k] and A[k][j] can raise indirect[i][j] above its starting
// zero, so the product needs, for each row i, the rows k of its positive entries
// (k a mediator) and their positive entries: sum_k indeg(k) * outdeg(k) updates
// instead of n^3. The network is given in CSR (row_ptr, col, val: the nonzero
// entries, columns ascending within a row). One CTA per row i keeps
// indirect[i][.] in shared memory as the bit patterns of non-negative floats,
// whose unsigned order is their numeric order, so atomicMax on them is the float
// maximum; each warp takes one entry (k, v) of row i at a time and its lanes walk
// row k. The result is one keep flag per CSR entry with the dense kernel's rule
// (entries whose column lies outside [0, n) are ignored and never kept).
constexpr int kSparseThreads = 256;

__global__ void __launch_bounds__(kSparseThreads) dpi_trim_sparse_kernel(
    const int64_t* __restrict__ row_ptr, const int32_t* __restrict__ col,
    const float* __restrict__ val, int n, const uint8_t* __restrict__ mediator,
    const uint8_t* __restrict__ keep_all, float thr, uint8_t* __restrict__ keep) {
  extern __shared__ uint32_t ind[];  // n words: max(0, max_k min(A[i][k], A[k][j])) as bits
  const int i = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n_warps = kSparseThreads / 32;
  for (int j = tid; j < n; j += kSparseThreads) ind[j] = 0u;
  __syncthreads();
  const int64_t e0 = row_ptr[i], e1 = row_ptr[i + 1];
  for (int64_t e = e0 + warp; e < e1; e += n_warps) {
    const int k = col[e];
    const float v = val[e];
    if ((unsigned)k >= (unsigned)n || !(v > 0.f) || (mediator != nullptr && mediator[k] == 0))
      continue;  // warp-uniform
    const int64_t f1 = row_ptr[k + 1];
    for (int64_t f = row_ptr[k] + lane; f < f1; f += 32) {
      const float w = val[f];
      const int j = col[f];
      if (w > 0.f && (unsigned)j < (unsigned)n) atomicMax(&ind[j], __float_as_uint(fminf(v, w)));
    }
  }
  __syncthreads();
  const bool all = keep_all != nullptr && keep_all[i] != 0;
  for (int64_t e = e0 + tid; e < e1; e += kSparseThreads) {
    const int j = col[e];
    if ((unsigned)j >= (unsigned)n) {  // malformed entry: never kept
      keep[e] = 0;
      continue;
    }
    const float a = val[e];
    const float t = __uint_as_float(ind[j]) + thr;
    keep[e] = (all || a >= t) ? 1 : 0;
  }
}

}  // namespace
}  // namespace tenex

using namespace tenex;

extern "C" int tenex_dpi_trim_sparse(const int64_t* row_ptr, const int32_t* col, const float* val,
                                     int n_vars, const uint8_t* mediator, const uint8_t* keep_all,
                                     float trim_threshold, uint8_t* keep, void* stream) {
  if (!row_ptr || !col || !val || !keep)
    return fail(TENEX_ERR_BADARG, "row_ptr, col, val and keep must be non-NULL");
  if (n_vars < 1) return fail(TENEX_ERR_BADARG, "n_vars must be >= 1");
  DevAttr A;
  int st = current_device_attr(&A);
  if (st) return st;
  const int64_t smem = (int64_t)n_vars * 4;
  if (smem > A.smem_optin)
    return fail(TENEX_ERR_UNSUPPORTED, "n_vars=%d: the row of %lld bytes exceeds shared memory "
                "(%d bytes); use tenex_dpi_trim", n_vars, (long long)smem, A.smem_optin);
  cudaError_t e = cudaFuncSetAttribute(dpi_trim_sparse_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
  dpi_trim_sparse_kernel<<<n_vars, kSparseThreads, (size_t)smem, as_stream(stream)>>>(
      row_ptr, col, val, n_vars, mediator, keep_all, trim_threshold, keep);
  return check_launch("dpi_trim_sparse_kernel");
}

extern "C" int tenex_dpi_trim(const float* te, int64_t ld, int n_vars, const uint8_t* mediator,
                              const uint8_t* keep_all, float trim_threshold, float* out,
                              int64_t out_ld, void* stream) {
  if (!te || !out) return fail(TENEX_ERR_BADARG, "te and out must be non-NULL");
  if (n_vars < 1) return fail(TENEX_ERR_BADARG, "n_vars must be >= 1");
  if (ld < n_vars || out_ld < n_vars) return fail(TENEX_ERR_BADARG, "row strides must be >= n_vars");
  if (out == te) return fail(TENEX_ERR_BADARG, "out must not alias te");
  const int64_t tiles = (n_vars + kTile - 1) / kTile;
  if (tiles > 65535) return fail(TENEX_ERR_UNSUPPORTED, "n_vars=%d exceeds the grid limit", n_vars);
  DpiArgs P{te, ld, n_vars, mediator, keep_all, trim_threshold, out, out_ld};
  dim3 grid((unsigned)tiles, (unsigned)tiles);
  dpi_trim_kernel<<<grid, kThreads, 0, as_stream(stream)>>>(P);
  return check_launch("dpi_trim_kernel");
}
