// preprocess.cu — GPU discretisation, dense bin remap and coarsening.
//
//   tenex_fsbwl_bins   FSBW-L binning (reference tenex/preprocess.py:61-88, the
//                      numpy path, and the clamp(min=0) of :680). Bit-identical
//                      to numpy: std(ddof=1) uses numpy's float32 pairwise
//                      summation tree (blocks of <= 128 with 8 accumulators,
//                      split at n/2 rounded down to a multiple of 8), the mean
//                      and variance divide in float64 and round to float32 as
//                      np.true_divide(float32, intp) does, and every float op is
//                      an explicit round-to-nearest intrinsic so nothing is
//                      contracted into an FMA.
//   tenex_remap_dense  per-gene dense relabelling (tenex/preprocess.py:401-459):
//                      value -> rank among the gene's distinct values.
//   tenex_coarsen      new = old * limit / n_per_var for genes above the limit
//                      (tenex/preprocess.py:462-551; coarsen_bins_cuda of
//                      tenex/csrc/adaptive_smem.cu:557-592).
//   tenex_coarsen_narrow  the same rule from uint16 bins (genes with more than
//                      256 distinct values, int16 in the reference,
//                      tenex/preprocess.py:335-354,520-536) into uint8 rows.
#include <cuda_runtime.h>
#include <stdint.h>

#include "common.cuh"

namespace tenex {
namespace {

constexpr int kMaxLeaves = 2048;      // leaves of the pairwise tree (each >= 57 samples)
constexpr int kMaxRemapValues = 8192;  // distinct raw bin values a gene may span

// numpy's pairwise_sum on one leaf (n <= 128), float32.
__device__ float leaf_sum(const float* a, int n) {
  if (n < 8) {
    float res = 0.f;
    for (int i = 0; i < n; ++i) res = __fadd_rn(res, a[i]);
    return res;
  }
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = a[k];
  int i = 8;
  for (; i < n - (n % 8); i += 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = __fadd_rn(r[k], a[i + k]);
  }
  float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                        __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
  for (; i < n; ++i) res = __fadd_rn(res, a[i]);
  return res;
}

// Same on (a[i] - mean)^2, the squared deviations np.var sums.
__device__ float leaf_sumsq(const float* a, int n, float mean) {
  auto sq = [&](int i) {
    const float d = __fsub_rn(a[i], mean);
    return __fmul_rn(d, d);
  };
  if (n < 8) {
    float res = 0.f;
    for (int i = 0; i < n; ++i) res = __fadd_rn(res, sq(i));
    return res;
  }
  float r[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) r[k] = sq(k);
  int i = 8;
  for (; i < n - (n % 8); i += 8) {
#pragma unroll
    for (int k = 0; k < 8; ++k) r[k] = __fadd_rn(r[k], sq(i + k));
  }
  float res = __fadd_rn(__fadd_rn(__fadd_rn(r[0], r[1]), __fadd_rn(r[2], r[3])),
                        __fadd_rn(__fadd_rn(r[4], r[5]), __fadd_rn(r[6], r[7])));
  for (; i < n; ++i) res = __fadd_rn(res, sq(i));
  return res;
}

// Enumerates, left to right, the nodes of the pairwise_sum(0, n) tree that hold
// at most `cap` samples and have no such ancestor (cap = 128: the leaves).
// Serial, one thread.
__device__ int enum_nodes(int n, int cap, int* starts, int* lens) {
  int so[64], sl[64];
  int sp = 0, nl = 0;
  so[sp] = 0;
  sl[sp] = n;
  ++sp;
  while (sp > 0) {
    --sp;
    const int o = so[sp], l = sl[sp];
    if (l <= cap) {
      starts[nl] = o;
      lens[nl] = l;
      ++nl;
    } else {
      int n2 = l / 2;
      n2 -= n2 % 8;
      so[sp] = o + n2;  // right, popped second
      sl[sp] = l - n2;
      ++sp;
      so[sp] = o;  // left, popped first
      sl[sp] = n2;
      ++sp;
    }
  }
  return nl;
}

// Combines the sums of those nodes in the order of
// pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2).
__device__ float combine_nodes(int n, int cap, const float* node) {
  // explicit post-order walk: frames (len, state); values on a separate stack
  int fl[64], fs[64];
  float val[64];
  int sp = 0, vp = 0, k = 0;
  fl[0] = n;
  fs[0] = 0;
  sp = 1;
  while (sp > 0) {
    const int l = fl[sp - 1];
    if (l <= cap) {
      val[vp++] = node[k++];
      --sp;
      continue;
    }
    int n2 = l / 2;
    n2 -= n2 % 8;
    if (fs[sp - 1] == 0) {  // visit left
      fs[sp - 1] = 1;
      fl[sp] = n2;
      fs[sp] = 0;
      ++sp;
    } else if (fs[sp - 1] == 1) {  // visit right
      fs[sp - 1] = 2;
      fl[sp] = l - n2;
      fs[sp] = 0;
      ++sp;
    } else {  // both done
      const float r = val[--vp];
      const float lft = val[--vp];
      val[vp++] = __fadd_rn(lft, r);
      --sp;
    }
  }
  return val[0];
}

// Rows longer than kSuperLen are summed as a tree of "super nodes" of at most
// kSuperLen samples (every subtree's sum is independent of where it sits), each
// super node leaf by leaf in shared memory.
constexpr int kSuperLen = kMaxLeaves * 56;  // leaves of a super node: >= 57 samples each
constexpr int kMaxSuper = 1024;             // super nodes hold >= kSuperLen/2 - 8 samples
constexpr int64_t kMaxPairwiseLen = (int64_t)(kMaxSuper - 1) * (kSuperLen / 2 - 8);

struct PairwiseScratch {
  int lstart[kMaxLeaves];
  int llen[kMaxLeaves];
  float lsum[kMaxLeaves];
  int sstart[kMaxSuper];
  int slen[kMaxSuper];
  float ssum[kMaxSuper];
  int nl, ns;
  float result;
};

// numpy's float32 pairwise sum of row[0, T) (SQ: of the squared deviations
// (row[i] - mean)^2 that np.var sums), bit for bit; all CTA threads call it,
// the result is returned to all of them.
template <bool SQ>
__device__ float row_pairwise_sum(const float* row, int T, float mean, PairwiseScratch& S) {
  const int tid = threadIdx.x;
  if (tid == 0) S.ns = enum_nodes(T, kSuperLen, S.sstart, S.slen);
  __syncthreads();
  const int ns = S.ns;
  for (int k = 0; k < ns; ++k) {
    const int o = S.sstart[k], l = S.slen[k];
    if (tid == 0) S.nl = enum_nodes(l, 128, S.lstart, S.llen);
    __syncthreads();
    const int nl = S.nl;
    for (int j = tid; j < nl; j += blockDim.x)
      S.lsum[j] = SQ ? leaf_sumsq(row + o + S.lstart[j], S.llen[j], mean)
                     : leaf_sum(row + o + S.lstart[j], S.llen[j]);
    __syncthreads();
    if (tid == 0) S.ssum[k] = combine_nodes(l, 128, S.lsum);
    __syncthreads();
  }
  if (tid == 0) S.result = combine_nodes(T, kSuperLen, S.ssum);
  __syncthreads();
  return S.result;
}

// One CTA (128 threads) per gene.
__global__ void fsbwl_kernel(const float* __restrict__ x, int64_t ldx, int T, float kp,
                             int32_t* __restrict__ bins, int64_t ldb,
                             int32_t* __restrict__ n_bins) {
  __shared__ PairwiseScratch S;
  __shared__ float sh_sd, sh_mn, sh_mx;
  __shared__ float wmin[32], wmax[32];
  const int g = blockIdx.x;
  const float* row = x + (int64_t)g * ldx;
  const int tid = threadIdx.x;
  // min / max
  float mn = 3.402823466e38f, mx = -3.402823466e38f;
  for (int t = tid; t < T; t += blockDim.x) {
    const float v = row[t];
    mn = fminf(mn, v);
    mx = fmaxf(mx, v);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  }
  if ((tid & 31) == 0) {
    wmin[tid >> 5] = mn;
    wmax[tid >> 5] = mx;
  }
  const float s = row_pairwise_sum<false>(row, T, 0.f, S);
  if (tid == 0) {
    float a = wmin[0], b = wmax[0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) {
      a = fminf(a, wmin[w]);
      b = fmaxf(b, wmax[w]);
    }
    sh_mn = a;
    sh_mx = b;
  }
  const float mean = __double2float_rn(__ddiv_rn((double)s, (double)T));
  const float ss = row_pairwise_sum<true>(row, T, mean, S);
  if (tid == 0) {
    const double cnt = T - 1 > 0 ? (double)(T - 1) : 0.0;
    const float var = __double2float_rn(__ddiv_rn((double)ss, cnt));
    float sd = __fsqrt_rn(var);
    if (sd == 0.f || isnan(sd)) sd = 1.0f;
    sh_sd = sd;
    n_bins[g] = (int32_t)ceilf(__fdiv_rn(__fsub_rn(sh_mx, sh_mn), sd));
  }
  __syncthreads();
  const float sd = sh_sd;
  const float shifted = __fsub_rn(sh_mn, __fmul_rn(kp, sd));
  int32_t* brow = bins + (int64_t)g * ldb;
  for (int t = tid; t < T; t += blockDim.x) {
    const float q = floorf(__fdiv_rn(__fsub_rn(row[t], shifted), sd));
    int32_t b = (int32_t)q;
    brow[t] = b < 0 ? 0 : b;  // clamp(min=0)
  }
}

template <typename In>
__device__ __forceinline__ int32_t load_raw(const void* base, int64_t i) {
  return (int32_t)reinterpret_cast<const In*>(base)[i];
}

// One CTA per gene: presence flags over [0, max], exclusive scan, relabel.
template <typename In, typename Out>
__global__ void remap_kernel(const void* __restrict__ raw, int64_t ldr, int64_t row_len,
                             Out* __restrict__ out, int64_t ldo, int32_t* __restrict__ npv,
                             int* __restrict__ err) {
  __shared__ int rank[kMaxRemapValues];
  __shared__ int wred[32];
  __shared__ int sh_hi;
  const int g = blockIdx.x;
  const int tid = threadIdx.x;
  const int64_t base = (int64_t)g * ldr;
  int hi = 0;
  for (int64_t i = tid; i < row_len; i += blockDim.x) {
    int32_t v = load_raw<In>(raw, base + i);
    v = v < 0 ? 0 : v;
    hi = v > hi ? v : hi;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  if ((tid & 31) == 0) wred[tid >> 5] = hi;
  __syncthreads();
  if (tid == 0) {
    int h = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) h = max(h, wred[w]);
    sh_hi = h;
  }
  __syncthreads();
  const int H = sh_hi;
  if (H >= kMaxRemapValues) {
    if (tid == 0) {
      atomicExch(err, 1);
      npv[g] = 0;
    }
    return;
  }
  for (int v = tid; v <= H; v += blockDim.x) rank[v] = 0;
  __syncthreads();
  for (int64_t i = tid; i < row_len; i += blockDim.x) {
    int32_t v = load_raw<In>(raw, base + i);
    rank[v < 0 ? 0 : v] = 1;
  }
  __syncthreads();
  if (tid == 0) {  // exclusive scan (H is small: bins span ~sqrt(T) values)
    int c = 0;
    for (int v = 0; v <= H; ++v) {
      const int p = rank[v];
      rank[v] = c;
      c += p;
    }
    npv[g] = c;
    const int cap = sizeof(Out) == 1 ? 256 : 65536;
    if (c > cap) atomicExch(err, 2);
  }
  __syncthreads();
  Out* orow = out + (int64_t)g * ldo;
  for (int64_t i = tid; i < row_len; i += blockDim.x) {
    int32_t v = load_raw<In>(raw, base + i);
    orow[i] = (Out)rank[v < 0 ? 0 : v];
  }
}

// In-place coarsening of uint8 rows; grid (chunks, genes).
__global__ void coarsen_kernel(uint8_t* __restrict__ bins, int64_t ld, int64_t row_len,
                               const int32_t* __restrict__ npv, int limit) {
  const int g = blockIdx.y;
  const int b = npv[g];
  if (b <= limit) return;
  uint8_t* row = bins + (int64_t)g * ld;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < row_len;
       i += (int64_t)gridDim.x * blockDim.x)
    row[i] = (uint8_t)(((int)row[i] * limit) / b);
}

// Coarsening of uint16 rows into uint8 rows (bins of genes with more than 256
// distinct values): new = old * limit / b above the limit, else a plain copy;
// grid (chunks, genes). Every output value is below min(b, limit) <= 255.
__global__ void coarsen_narrow_kernel(const uint16_t* __restrict__ in, int64_t ldi,
                                      int64_t row_len, const int32_t* __restrict__ npv,
                                      int limit, uint8_t* __restrict__ out, int64_t ldo) {
  const int g = blockIdx.y;
  const int b = npv[g];
  const uint16_t* row = in + (int64_t)g * ldi;
  uint8_t* orow = out + (int64_t)g * ldo;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < row_len;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int v = row[i];
    orow[i] = (uint8_t)(b > limit ? (v * limit) / b : v);
  }
}

// Binarisation 1[x > thr_g] into uint8 padded rows, one CTA per gene.
// mode 0: thr = 0 (nonzero); 1: thr = float32 mean with numpy's pairwise sum and
// float64 division (np.mean on float32 rows); 2: thr = thr_in[g].
// n_per_var[g] = max - min + 1 of the binary row (1 if constant, else 2).
__global__ void binarize_kernel(const float* __restrict__ x, int64_t ldx, int T, int mode,
                                const float* __restrict__ thr_in, uint8_t* __restrict__ out,
                                int64_t ldo, int32_t* __restrict__ npv) {
  __shared__ PairwiseScratch S;
  __shared__ float sh_thr;
  const int g = blockIdx.x;
  const float* row = x + (int64_t)g * ldx;
  const int tid = threadIdx.x;
  if (mode == 1) {
    const float s = row_pairwise_sum<false>(row, T, 0.f, S);
    if (tid == 0) sh_thr = __double2float_rn(__ddiv_rn((double)s, (double)T));
  } else if (tid == 0) {
    sh_thr = mode == 0 ? 0.f : thr_in[g];
  }
  __syncthreads();
  const float thr = sh_thr;
  uint8_t* orow = out + (int64_t)g * ldo;
  int any1 = 0, any0 = 0;
  // 16 samples per thread and step when both rows are 16-byte aligned: four
  // 16-byte loads, one 16-byte store of the 0/1 bytes; the same comparison as the
  // scalar tail (a NaN compares false: bin 0)
  int t0 = 0;
  if (((reinterpret_cast<uintptr_t>(row) | reinterpret_cast<uintptr_t>(orow)) & 15) == 0) {
    const int nv = T >> 4;
    const float4* r4 = reinterpret_cast<const float4*>(row);
    for (int v = tid; v < nv; v += blockDim.x) {
      uint32_t w[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const float4 a = __ldg(r4 + 4 * v + k);
        w[k] = (uint32_t)(a.x > thr) | ((uint32_t)(a.y > thr) << 8) |
               ((uint32_t)(a.z > thr) << 16) | ((uint32_t)(a.w > thr) << 24);
      }
      *reinterpret_cast<uint4*>(orow + 16 * (int64_t)v) = make_uint4(w[0], w[1], w[2], w[3]);
      any1 |= (w[0] | w[1] | w[2] | w[3]) != 0u;
      any0 |= (w[0] & w[1] & w[2] & w[3]) != 0x01010101u;
    }
    t0 = nv << 4;
  }
  for (int t = t0 + tid; t < T; t += blockDim.x) {
    const uint8_t b = row[t] > thr ? 1 : 0;
    orow[t] = b;
    any1 |= b;
    any0 |= b ^ 1;
  }
  any1 = __syncthreads_or(any1);
  any0 = __syncthreads_or(any0);
  if (tid == 0) npv[g] = (any1 && any0) ? 2 : 1;
}

__global__ void coarsen_npv_kernel(int32_t* npv, int n, int limit) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < n && npv[g] > limit) npv[g] = limit;
}

}  // namespace
}  // namespace tenex

using namespace tenex;

extern "C" int tenex_fsbwl_bins(const float* x, int64_t ldx, int n_vars, int T, float kp,
                                int32_t* bins, int64_t ldb, int32_t* n_bins, void* stream) {
  if (!x || !bins || !n_bins) return fail(TENEX_ERR_BADARG, "x, bins, n_bins must be non-NULL");
  if (n_vars < 1 || T < 1) return fail(TENEX_ERR_BADARG, "empty expression matrix");
  if (ldx < T || ldb < T) return fail(TENEX_ERR_BADARG, "row strides must be >= T");
  if ((int64_t)T > kMaxPairwiseLen)
    return fail(TENEX_ERR_UNSUPPORTED, "T=%d exceeds the discretiser's %lld-sample limit", T,
                (long long)kMaxPairwiseLen);
  fsbwl_kernel<<<n_vars, 128, 0, as_stream(stream)>>>(x, ldx, T, kp, bins, ldb, n_bins);
  return check_launch("fsbwl_kernel");
}

extern "C" int tenex_remap_dense(const void* raw, int in_bytes, int64_t ldr, int n_vars,
                                 int64_t row_len, void* out, int out_bytes, int64_t ldo,
                                 int32_t* n_per_var, int* err, void* stream) {
  if (!raw || !out || !n_per_var || !err)
    return fail(TENEX_ERR_BADARG, "raw, out, n_per_var and err must be non-NULL");
  if (n_vars < 1 || row_len < 1) return fail(TENEX_ERR_BADARG, "empty bins");
  if (ldr < row_len || ldo < row_len) return fail(TENEX_ERR_BADARG, "row strides < row_len");
  cudaStream_t s = as_stream(stream);
  const dim3 grid(n_vars), block(256);
  if (out_bytes == 1) {
    if (in_bytes == 1)
      remap_kernel<uint8_t, uint8_t><<<grid, block, 0, s>>>(raw, ldr, row_len, (uint8_t*)out, ldo,
                                                            n_per_var, err);
    else if (in_bytes == 2)
      remap_kernel<uint16_t, uint8_t><<<grid, block, 0, s>>>(raw, ldr, row_len, (uint8_t*)out,
                                                             ldo, n_per_var, err);
    else if (in_bytes == 4)
      remap_kernel<int32_t, uint8_t><<<grid, block, 0, s>>>(raw, ldr, row_len, (uint8_t*)out, ldo,
                                                            n_per_var, err);
    else
      return fail(TENEX_ERR_BADARG, "in_bytes must be 1, 2 or 4");
  } else if (out_bytes == 2) {
    if (in_bytes == 1)
      remap_kernel<uint8_t, uint16_t><<<grid, block, 0, s>>>(raw, ldr, row_len, (uint16_t*)out,
                                                             ldo, n_per_var, err);
    else if (in_bytes == 2)
      remap_kernel<uint16_t, uint16_t><<<grid, block, 0, s>>>(raw, ldr, row_len, (uint16_t*)out,
                                                              ldo, n_per_var, err);
    else if (in_bytes == 4)
      remap_kernel<int32_t, uint16_t><<<grid, block, 0, s>>>(raw, ldr, row_len, (uint16_t*)out,
                                                             ldo, n_per_var, err);
    else
      return fail(TENEX_ERR_BADARG, "in_bytes must be 1, 2 or 4");
  } else {
    return fail(TENEX_ERR_BADARG, "out_bytes must be 1 or 2");
  }
  return check_launch("remap_kernel");
}

extern "C" int tenex_coarsen(uint8_t* bins, int64_t ld, int n_vars, int64_t row_len,
                             int32_t* n_per_var, int limit, void* stream) {
  if (!bins || !n_per_var) return fail(TENEX_ERR_BADARG, "bins and n_per_var must be non-NULL");
  if (limit < 1 || limit > 255) return fail(TENEX_ERR_BADARG, "limit must be in [1, 255]");
  if (n_vars < 1 || row_len < 1) return fail(TENEX_ERR_BADARG, "empty bins");
  if (n_vars > 65535) return fail(TENEX_ERR_UNSUPPORTED, "n_vars > 65535");
  cudaStream_t s = as_stream(stream);
  const int64_t chunks64 = (row_len + 4095) / 4096;
  const unsigned chunks = (unsigned)(chunks64 < 1024 ? chunks64 : 1024);
  coarsen_kernel<<<dim3(chunks, n_vars), 256, 0, s>>>(bins, ld, row_len, n_per_var, limit);
  int st = check_launch("coarsen_kernel");
  if (st) return st;
  coarsen_npv_kernel<<<(n_vars + 255) / 256, 256, 0, s>>>(n_per_var, n_vars, limit);
  return check_launch("coarsen_npv_kernel");
}

extern "C" int tenex_coarsen_narrow(const uint16_t* in, int64_t ldi, int n_vars, int64_t row_len,
                                    int32_t* n_per_var, int limit, uint8_t* out, int64_t ldo,
                                    void* stream) {
  if (!in || !out || !n_per_var)
    return fail(TENEX_ERR_BADARG, "in, out and n_per_var must be non-NULL");
  if (limit < 1 || limit > 255) return fail(TENEX_ERR_BADARG, "limit must be in [1, 255]");
  if (n_vars < 1 || row_len < 1) return fail(TENEX_ERR_BADARG, "empty bins");
  if (ldi < row_len || ldo < row_len) return fail(TENEX_ERR_BADARG, "row strides < row_len");
  if (n_vars > 65535) return fail(TENEX_ERR_UNSUPPORTED, "n_vars > 65535");
  cudaStream_t s = as_stream(stream);
  const int64_t chunks64 = (row_len + 4095) / 4096;
  const unsigned chunks = (unsigned)(chunks64 < 1024 ? chunks64 : 1024);
  coarsen_narrow_kernel<<<dim3(chunks, n_vars), 256, 0, s>>>(in, ldi, row_len, n_per_var, limit,
                                                             out, ldo);
  int st = check_launch("coarsen_narrow_kernel");
  if (st) return st;
  coarsen_npv_kernel<<<(n_vars + 255) / 256, 256, 0, s>>>(n_per_var, n_vars, limit);
  return check_launch("coarsen_npv_kernel");
}

extern "C" int tenex_binarize(const float* x, int64_t ldx, int n_vars, int T, int mode,
                              const float* thresholds, uint8_t* out, int64_t ldo,
                              int32_t* n_per_var, void* stream) {
  if (!x || !out || !n_per_var) return fail(TENEX_ERR_BADARG, "x, out, n_per_var non-NULL");
  if (n_vars < 1 || T < 1) return fail(TENEX_ERR_BADARG, "empty expression matrix");
  if (ldx < T || ldo < T) return fail(TENEX_ERR_BADARG, "row strides must be >= T");
  if (mode < 0 || mode > 2) return fail(TENEX_ERR_BADARG, "mode must be 0, 1 or 2");
  if (mode == 2 && !thresholds) return fail(TENEX_ERR_BADARG, "mode 2 needs thresholds");
  if (mode == 1 && (int64_t)T > kMaxPairwiseLen)
    return fail(TENEX_ERR_UNSUPPORTED, "T=%d too long for the mean binariser", T);
  binarize_kernel<<<n_vars, 128, 0, as_stream(stream)>>>(x, ldx, T, mode, thresholds, out, ldo,
                                                         n_per_var);
  return check_launch("binarize_kernel");
}
