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

// 1[row[t] > thr] into orow[0, T) by all CTA threads; returns (to every thread)
// bit 0: some sample is 1, bit 1: some sample is 0. A NaN compares false (bin 0).
// NC: row is global memory read through the non-coherent path; else a generic
// pointer (a row staged in shared memory).
template <bool NC = true>
__device__ int binarize_row(const float* __restrict__ row, uint8_t* __restrict__ orow, int T,
                            float thr) {
  const int tid = threadIdx.x;
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
        const float4 a = NC ? __ldg(r4 + 4 * v + k) : r4[4 * v + k];
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
  return (any1 ? 1 : 0) | (any0 ? 2 : 0);
}

// Binarisation 1[x > thr_g] into uint8 padded rows, one CTA per gene.
// mode 0: thr = 0 (nonzero); 1: thr = float32 mean with numpy's pairwise sum and
// float64 division (np.mean on float32 rows; rows longer than one plan, see
// binarize_mean_kernel); 2: thr = thr_in[g].
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
  const int any = binarize_row(row, out + (int64_t)g * ldo, T, sh_thr);
  if (tid == 0) npv[g] = any == 3 ? 2 : 1;
}

// numpy's pairwise_sum tree of one row length (T <= kSuperLen: one level of
// leaves of <= 128 samples), laid out for a parallel evaluation: the leaves left
// to right, then the internal nodes sorted by height, so that one pass per height
// adds the two operands of every node of that height. Value ids: leaves 0..nl-1,
// internal node at sorted position p: nl + p. The root is the last id.
constexpr int kMaxPlanHeight = 32;
struct MeanPlan {
  int lstart[kMaxLeaves];
  int16_t llen[kMaxLeaves];
  uint32_t op[kMaxLeaves];          // sorted internal nodes: left | right << 16
  float val[2 * kMaxLeaves];        // leaf sums, then internal sums
  int level[kMaxPlanHeight + 2];    // internal nodes of height h: [level[h], level[h+1])
  int nl, ni, height;
};

// Builds the plan (thread 0, serial; once per CTA). val[] is scratch here.
__device__ void build_mean_plan(int T, MeanPlan& P) {
  const int nl = enum_nodes(T, 128, P.lstart, reinterpret_cast<int*>(P.val));
  for (int j = 0; j < nl; ++j) P.llen[j] = (int16_t)reinterpret_cast<int*>(P.val)[j];
  // post-order walk: internal node m (creation order) gets operands and a height
  uint32_t* tmp_op = reinterpret_cast<uint32_t*>(P.val);               // [kMaxLeaves)
  int* tmp_h = reinterpret_cast<int*>(P.val) + kMaxLeaves;              // [kMaxLeaves)
  int fl[64], fs[64], vid[64], vh[64];
  int sp = 1, vp = 0, k = 0, ni = 0, H = 0;
  fl[0] = T;
  fs[0] = 0;
  while (sp > 0) {
    const int l = fl[sp - 1];
    if (l <= 128) {
      vid[vp] = k++;
      vh[vp++] = 0;
      --sp;
      continue;
    }
    int n2 = l / 2;
    n2 -= n2 % 8;
    if (fs[sp - 1] < 2) {
      fl[sp] = fs[sp - 1] == 0 ? n2 : l - n2;
      fs[sp - 1] += 1;
      fs[sp] = 0;
      ++sp;
    } else {
      const int ir = vid[--vp], hr = vh[vp];
      const int il = vid[--vp], hl = vh[vp];
      const int h = max(hl, hr) + 1;
      tmp_op[ni] = (uint32_t)il | ((uint32_t)ir << 16);
      tmp_h[ni] = h;
      H = max(H, h);
      vid[vp] = nl + ni++;
      vh[vp++] = h;
      --sp;
    }
  }
  // counting sort by height; children precede parents in post-order, so their
  // sorted positions are known when a parent is placed
  int cur[kMaxPlanHeight + 2];
  for (int h = 0; h <= H + 1; ++h) cur[h] = 0;
  for (int m = 0; m < ni; ++m) ++cur[tmp_h[m]];
  int acc = 0;
  for (int h = 0; h <= H + 1; ++h) {
    P.level[h] = acc;
    acc += cur[h];
    cur[h] = P.level[h];
  }
  for (int m = 0; m < ni; ++m) {
    const int pos = cur[tmp_h[m]]++;
    uint32_t l = tmp_op[m] & 0xffffu, r = tmp_op[m] >> 16;
    if ((int)l >= nl) l = nl + tmp_h[l - nl];   // tmp_h[child] already holds its position
    if ((int)r >= nl) r = nl + tmp_h[r - nl];
    P.op[pos] = l | (r << 16);
    tmp_h[m] = pos;
  }
  P.nl = nl;
  P.ni = ni;
  P.height = H;
}

// The mean binariser for T <= kSuperLen: a persistent CTA builds the row
// length's plan once and then, per gene, sums the leaves eight lanes to a leaf
// (lane k holds numpy's accumulator r[k]: a stride-8 pass over the leaf, so the
// eight lanes read 32 contiguous bytes per step), folds the eight accumulators
// with xor shuffles 1, 2, 4 (((r0+r1)+(r2+r3))+((r4+r5)+(r6+r7)), numpy's order;
// float addition commutes exactly), adds the tail, then evaluates the internal
// nodes one height per pass. The row is read again for the comparison (from L2).
__global__ void __launch_bounds__(256) binarize_mean_kernel(const float* __restrict__ x,
                                                            int64_t ldx, int T, int n_vars,
                                                            uint8_t* __restrict__ out,
                                                            int64_t ldo,
                                                            int32_t* __restrict__ npv) {
  __shared__ MeanPlan P;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int n_warps = blockDim.x >> 5;
  if (tid == 0) build_mean_plan(T, P);
  __syncthreads();
  const int nl = P.nl, ni = P.ni, H = P.height;
  for (int g = blockIdx.x; g < n_vars; g += gridDim.x) {
    const float* row = x + (int64_t)g * ldx;
    // leaves: four per warp and step, eight lanes each
    for (int jb = warp * 4; jb < nl; jb += n_warps * 4) {
      const int j = jb + (lane >> 3);
      const int kk = lane & 7;
      const bool active = j < nl;
      const int s = active ? P.lstart[j] : 0;
      const int n = active ? P.llen[j] : 0;
      const int m8 = n - n % 8;
      float r = 0.f;
      if (n >= 8) {
        const float* a = row + s + kk;
        r = a[0];
        for (int i = 8; i < m8; i += 8) r = __fadd_rn(r, a[i]);
      }
      r = __fadd_rn(r, __shfl_xor_sync(0xffffffffu, r, 1));
      r = __fadd_rn(r, __shfl_xor_sync(0xffffffffu, r, 2));
      r = __fadd_rn(r, __shfl_xor_sync(0xffffffffu, r, 4));
      if (active && kk == 0) {
        float res = r;
        if (n < 8) {
          res = 0.f;
          for (int i = 0; i < n; ++i) res = __fadd_rn(res, row[s + i]);
        } else {
          for (int i = m8; i < n; ++i) res = __fadd_rn(res, row[s + i]);
        }
        P.val[j] = res;
      }
    }
    __syncthreads();
    for (int h = 1; h <= H; ++h) {
      for (int p = P.level[h] + tid; p < P.level[h + 1]; p += blockDim.x) {
        const uint32_t o = P.op[p];
        P.val[nl + p] = __fadd_rn(P.val[o & 0xffffu], P.val[o >> 16]);
      }
      __syncthreads();
    }
    const float sum = P.val[ni > 0 ? nl + ni - 1 : 0];
    const float thr = __double2float_rn(__ddiv_rn((double)sum, (double)T));
    const int any = binarize_row(row, out + (int64_t)g * ldo, T, thr);
    if (tid == 0) npv[g] = any == 3 ? 2 : 1;
    // binarize_row ends in __syncthreads_or: val[] is free for the next gene
  }
}

// float32 -> uint32 key with the same order as the values (-inf first, -0 just
// below +0); selection runs on keys, thresholds come back through select_float.
__device__ __forceinline__ uint32_t select_key(float v) {
  const uint32_t u = __float_as_uint(v);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float select_float(uint32_t k) {
  return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

constexpr int kSelectThreads = 512;
constexpr int kSelectHead = 2048;     // bytes before the staged row: histogram + misc

// Median / quantile binarisation (the reference's numpy backend: np.median and
// np.quantile "linear" per row, tenex/binarize.py:126-150). A persistent CTA per
// group of genes; a row that fits is staged in shared memory (one HBM read),
// else every pass reads it from global memory (L2). The order statistic of rank
// k0 is found by four radix passes over 8-bit digits of the order-preserving key
// (histogram counts aggregated per warp and digit with __match_any_sync, so runs
// of tied values cost one atomic), the one of rank k0 + 1, where the threshold
// needs it, is the same key if the tie run goes on, else the smallest key above
// (one min pass). Any NaN in the row makes numpy's threshold NaN: every bin 0.
// Thresholds in numpy's arithmetic: median = s[h] (T odd) or float32(
// double(s[h-1] + s[h] in float32) / 2); quantile: virtual index (T - 1) q in
// float64, a + (b - a) g for g < 0.5 else b - (b - a)(1 - g), b - a in float32 and
// the rest in float64; numpy then compares the float32 data with that float64
// value, which selects the same samples as x > t32 with t32 = the float64 value
// rounded toward -inf.
__global__ void __launch_bounds__(kSelectThreads) binarize_select_kernel(
    const float* __restrict__ x, int64_t ldx, int T, int n_vars, int median, double q,
    int stage, uint8_t* __restrict__ out, int64_t ldo, int32_t* __restrict__ npv) {
  extern __shared__ __align__(16) unsigned char sm[];
  int* hist = reinterpret_cast<int*>(sm);          // [256]
  int* misc = hist + 256;                          // [8]
  float* srow = reinterpret_cast<float*>(sm + kSelectHead);
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const int warp = tid >> 5;
  const int n_warps = blockDim.x >> 5;
  // ranks the threshold reads (same for every gene)
  int k0;
  bool need_b;
  double gam = 0.0;
  if (median) {
    k0 = (T & 1) ? T / 2 : T / 2 - 1;
    need_b = (T & 1) == 0;
  } else {
    const double vi = __dmul_rn((double)(T - 1), q);
    const double lo = floor(vi);
    gam = __dsub_rn(vi, lo);
    need_b = vi < (double)(T - 1);
    k0 = need_b ? (int)lo : T - 1;
  }
  for (int g = blockIdx.x; g < n_vars; g += gridDim.x) {
    const float* grow = x + (int64_t)g * ldx;
    const float* r = grow;
    bool nan = false;
    if (stage) {
      // 16-byte copies (the host stages only 16-byte aligned rows); the previous
      // gene's readers of srow finished in binarize_row's closing barrier
      const int nv = T >> 2;
      const float4* g4 = reinterpret_cast<const float4*>(grow);
      float4* s4 = reinterpret_cast<float4*>(srow);
      for (int v = tid; v < nv; v += blockDim.x) {
        const float4 a = __ldg(g4 + v);
        nan |= (a.x != a.x) | (a.y != a.y) | (a.z != a.z) | (a.w != a.w);
        s4[v] = a;
      }
      for (int t = (nv << 2) + tid; t < T; t += blockDim.x) {
        const float a = __ldg(grow + t);
        nan |= a != a;
        srow[t] = a;
      }
      r = srow;
    } else {
      for (int t = tid; t < T; t += blockDim.x) {
        const float a = __ldg(grow + t);
        nan |= a != a;
      }
    }
    nan = __syncthreads_or(nan);
    float thr = __uint_as_float(0x7fc00000u);    // NaN: every sample compares false
    if (!nan) {
      uint32_t prefix = 0u, pmask = 0u;
      int rank = k0, cnt = 0;
      for (int shift = 24; shift >= 0; shift -= 8) {
        if (tid < 256) hist[tid] = 0;
        __syncthreads();
        for (int base = warp * 32; base < T; base += n_warps * 32) {
          const int t = base + lane;
          int d = 256;                              // 256: not counted
          if (t < T) {
            const uint32_t k = select_key(r[t]);
            if ((k & pmask) == prefix) d = (int)((k >> shift) & 255u);
          }
          const unsigned m = __match_any_sync(0xffffffffu, d);
          if (d < 256 && lane == __ffs(m) - 1) atomicAdd(&hist[d], __popc(m));
        }
        __syncthreads();
        if (warp == 0) {
          // digit holding rank: lane l scans bins [8l, 8l + 8)
          int c[8], s = 0;
#pragma unroll
          for (int i = 0; i < 8; ++i) {
            c[i] = hist[lane * 8 + i];
            s += c[i];
          }
          int incl = s;
#pragma unroll
          for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
          }
          int before = incl - s;
          if (rank >= before && rank < incl) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
              if (rank >= before && rank < before + c[i]) {
                misc[0] = lane * 8 + i;
                misc[1] = rank - before;
                misc[2] = c[i];
              }
              before += c[i];
            }
          }
        }
        __syncthreads();
        prefix |= (uint32_t)misc[0] << shift;
        pmask |= 255u << shift;
        rank = misc[1];
        cnt = misc[2];
      }
      const float a = select_float(prefix);
      float b = a;
      if (need_b && rank + 1 >= cnt) {
        // the tie run of a ends at rank k0: b = the smallest key above a
        uint32_t mn = 0xffffffffu;
        for (int t = tid; t < T; t += blockDim.x) {
          const uint32_t k = select_key(r[t]);
          if (k > prefix) mn = min(mn, k);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        if (tid == 0) misc[3] = (int)0xffffffffu;
        __syncthreads();
        if (lane == 0) atomicMin(reinterpret_cast<unsigned*>(&misc[3]), mn);
        __syncthreads();
        b = select_float((uint32_t)misc[3]);
      }
      if (median) {
        thr = need_b ? __double2float_rn(__dmul_rn((double)__fadd_rn(a, b), 0.5)) : a;
      } else if (!need_b) {
        // index at the top: numpy interpolates s[T-1] with itself (b - (b - a)
        // (1 - gamma)), exact for a finite maximum and NaN (inf - inf) for an
        // infinite one
        thr = isinf(a) ? __uint_as_float(0x7fc00000u) : a;
      } else {
        const double diff = (double)__fsub_rn(b, a);
        const double t64 = gam >= 0.5 ? __dsub_rn((double)b, __dmul_rn(diff, __dsub_rn(1.0, gam)))
                                      : __dadd_rn((double)a, __dmul_rn(diff, gam));
        thr = __double2float_rn(t64);
        if ((double)thr > t64) thr = nextafterf(thr, -INFINITY);
      }
    }
    uint8_t* orow = out + (int64_t)g * ldo;
    const int any = stage ? binarize_row<false>(r, orow, T, thr)
                          : binarize_row<true>(grow, orow, T, thr);
    if (tid == 0) npv[g] = any == 3 ? 2 : 1;
  }
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
  if (mode == 1 && T <= kSuperLen) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, binarize_mean_kernel, 256, 0);
    const int grid = (int)std::min<int64_t>(n_vars, (int64_t)std::max(1, sms * per_sm));
    binarize_mean_kernel<<<grid, 256, 0, as_stream(stream)>>>(x, ldx, T, n_vars, out, ldo,
                                                              n_per_var);
    return check_launch("binarize_mean_kernel");
  }
  binarize_kernel<<<n_vars, 128, 0, as_stream(stream)>>>(x, ldx, T, mode, thresholds, out, ldo,
                                                         n_per_var);
  return check_launch("binarize_kernel");
}

extern "C" int tenex_binarize_select(const float* x, int64_t ldx, int n_vars, int T, int median,
                                     double q, uint8_t* out, int64_t ldo, int32_t* n_per_var,
                                     void* stream) {
  if (!x || !out || !n_per_var) return fail(TENEX_ERR_BADARG, "x, out, n_per_var non-NULL");
  if (n_vars < 1 || T < 1) return fail(TENEX_ERR_BADARG, "empty expression matrix");
  if (ldx < T || ldo < T) return fail(TENEX_ERR_BADARG, "row strides must be >= T");
  if (!median && !(q >= 0.0 && q <= 1.0))
    return fail(TENEX_ERR_BADARG, "quantile q must be in [0, 1]");
  int dev = 0, sms = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  // stage the row in shared memory when it fits and its 16-byte copies are aligned
  const int64_t staged = (int64_t)kSelectHead + 4 * (int64_t)T;
  const bool stage = staged <= optin && (reinterpret_cast<uintptr_t>(x) & 15) == 0 &&
                     (ldx & 3) == 0;
  const int smem = stage ? (int)staged : kSelectHead;
  cudaError_t e = cudaFuncSetAttribute(binarize_select_kernel,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  if (e != cudaSuccess) return fail(TENEX_ERR_LAUNCH, "binarize_select smem: %s", cudaGetErrorString(e));
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, binarize_select_kernel, kSelectThreads,
                                                smem);
  const int grid = (int)std::min<int64_t>(n_vars, (int64_t)std::max(1, sms * per_sm));
  binarize_select_kernel<<<grid, kSelectThreads, smem, as_stream(stream)>>>(
      x, ldx, T, n_vars, median ? 1 : 0, q, stage ? 1 : 0, out, ldo, n_per_var);
  return check_launch("binarize_select_kernel");
}
