// null_mlp.cu — learned null model of the surrogate test (no reference
// counterpart): per-gene features, per-pair feature assembly, and a small MLP
// (16 -> 64 -> 64 -> 2, GELU) with BF16 weights and FP32 accumulation, plus the
// kernels that train it (forward with stored pre-activations, backward deltas,
// batch-reduced weight gradients, Adam on an FP32 master copy).
//
// Parameter vector (FP32 master and BF16 copy, same order):
//   W1[64][16] b1[64] W2[64][64] b2[64] W3[2][64] b3[2]   (5378 values)
// Feature vector of a pair (src -> tgt), before standardisation:
//   0-5  target: log2 b, H(x_t), H(x_{t+lag}, x_t), 2H - H2 (lag-1 information),
//        log2 mean run length, 2^H / b
//   6-11 source: the same six
//   12 log2 of the pair's independence bias E_iid (below), 13 log2 block length,
//   14 log2 of (b_t - 1)(b_s - 1) b_t + 1, 15 log2 of 2^{H2_t} * 2^{H_s}
//
// E_iid is the expected plug-in bias of N ln2 * TE when source and target are
// independent and each joint cell count is Poisson with its independence mean:
//   E_iid = sum_{a,b} g(n_a q_b) - sum_{x,b} g(n_x q_b),
// n_a = count of target state a = (x_{t+lag}, x_t), n_x = count of x_t, q_b =
// source marginal over the same N positions, g(m) = E[C ln C] - m ln m for
// C ~ Poisson(m). (The m ln m parts cancel against the target's own entropy
// terms, so E_iid is the whole expectation under that model.) It carries the
// small-count behaviour of sparse tables that per-gene summaries miss.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <algorithm>

#include "common.cuh"

namespace tenex {
namespace {

constexpr int kIn = 16, kH = 64, kOut = 2;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kH * kIn, kOffW2 = kOffB1 + kH,
              kOffB2 = kOffW2 + kH * kH, kOffW3 = kOffB2 + kH, kOffB3 = kOffW3 + kOut * kH,
              kParams = kOffB3 + kOut;
static_assert(kOffW1 % 4 == 0 && kOffW2 % 4 == 0 && kIn % 4 == 0 && kH % 4 == 0,
              "weight rows are read as float4");
constexpr int kGeneFeat = 8;

__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.f + erff(x * 0.70710678118654752f));
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float cdf = 0.5f * (1.f + erff(x * 0.70710678118654752f));
  const float pdf = 0.3989422804014327f * expf(-0.5f * x * x);
  return cdf + x * pdf;
}

// ---- per-gene features (one CTA per gene, b <= 64 for the joint entropy) ----
__global__ void gene_features_kernel(const uint8_t* __restrict__ bins, int64_t ld,
                                     const int32_t* __restrict__ npv, int n, int N, int lag,
                                     float* __restrict__ feat) {
  __shared__ int h1[256];
  __shared__ int h2[64 * 64];
  __shared__ int changes;
  const int g = blockIdx.x;
  const int b = npv[g];
  const uint8_t* row = bins + (int64_t)g * ld;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h1[i] = 0;
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x) h2[i] = 0;
  if (threadIdx.x == 0) changes = 0;
  __syncthreads();
  const bool joint = b >= 1 && b <= 64;
  int ch = 0;
  for (int s = threadIdx.x; s < N; s += blockDim.x) {
    const int x0 = row[s], x1 = row[s + lag];
    atomicAdd(&h1[x0], 1);
    if (joint && x0 < 64 && x1 < 64) atomicAdd(&h2[x1 * 64 + x0], 1);
    ch += x1 != x0;
  }
  atomicAdd(&changes, ch);
  __syncthreads();
  __shared__ double part[2][32];
  double e1 = 0.0, e2 = 0.0;
  const double invN = 1.0 / (double)N;
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h1[i]) {
      const double p = h1[i] * invN;
      e1 -= p * log2(p);
    }
  for (int i = threadIdx.x; i < 64 * 64; i += blockDim.x)
    if (h2[i]) {
      const double p = h2[i] * invN;
      e2 -= p * log2(p);
    }
  e1 = dev::warp_sum(e1);
  e2 = dev::warp_sum(e2);
  if ((threadIdx.x & 31) == 0) {
    part[0][threadIdx.x >> 5] = e1;
    part[1][threadIdx.x >> 5] = e2;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double H1 = 0.0, H2 = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      H1 += part[0][w];
      H2 += part[1][w];
    }
    float* f = feat + (int64_t)g * kGeneFeat;
    const float nan = __int_as_float(0x7fc00000);
    f[0] = log2f((float)max(b, 1));
    f[1] = (float)H1;
    f[2] = joint ? (float)H2 : nan;
    f[3] = joint ? (float)(2.0 * H1 - H2) : nan;
    f[4] = log2f((float)N / (float)(changes + 1));
    f[5] = (float)(exp2(H1) / (double)max(b, 1));
    f[6] = 0.f;
    f[7] = 0.f;
  }
}

// ---- E_iid: g table, source marginals, per-pair double sum ------------------
constexpr int kGTable = 1024;
constexpr float kGLo = -10.f, kGHi = 8.f;  // table covers m in [2^-10, 2^8]
constexpr int kEiidMaxB = 64;

// g(m) = E[C ln C] - m ln m, C ~ Poisson(m), on a log2 grid (float64 series).
__global__ void g_table_kernel(float* __restrict__ table) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kGTable) return;
  const double m = exp2((double)kGLo + (double)(kGHi - kGLo) * i / (kGTable - 1));
  const int kmax = (int)(m + 14.0 * sqrt(m) + 60.0);
  double p = exp(-m), acc = 0.0;
  for (int k = 1; k <= kmax; ++k) {
    p *= m / k;
    acc += p * k * log((double)k);
  }
  table[i] = (float)(acc - m * log(m));
}

// g(m) from the table, with its two limits outside it: -m ln m + m^2 ln 2 for
// small m, 1/2 + 1/(12m) + 1/(12m^2) for large m.
__device__ __forceinline__ float g_poisson(float m, const float* __restrict__ tab) {
  if (m <= 0.f) return 0.f;
  if (m < 9.765625e-4f) return m * (0.69314718f * m - __logf(m));
  if (m > 256.f) {
    const float r = 1.f / m;
    return 0.5f + r * (0.083333333f + 0.083333333f * r);
  }
  const float pos = (__log2f(m) - kGLo) * ((kGTable - 1) / (kGHi - kGLo));
  const int i = max(0, min((int)pos, kGTable - 2));
  const float f = pos - (float)i;
  return fmaf(f, tab[i + 1] - tab[i], tab[i]);
}

// q[g][b] = count of y_s = b over s < N, / N, and cnt[g][b] the count itself
// (b < 64; genes with b > 64 unused).
__global__ void source_marginal_kernel(const uint8_t* __restrict__ bins, int64_t ld, int N,
                                       float* __restrict__ q, int* __restrict__ cnt) {
  __shared__ int h[256];
  const int g = blockIdx.x;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  const uint8_t* row = bins + (int64_t)g * ld;
  for (int s = threadIdx.x; s < N; s += blockDim.x) atomicAdd(&h[row[s]], 1);
  __syncthreads();
  if (threadIdx.x < kEiidMaxB) {
    q[(int64_t)g * kEiidMaxB + threadIdx.x] = (float)h[threadIdx.x] / N;
    cnt[(int64_t)g * kEiidMaxB + threadIdx.x] = h[threadIdx.x];
  }
}

// One CTA per target: its non-zero n_a and n_x in shared memory, threads over
// sources. out[src * n + tgt] = E_iid (NaN when b_t or b_s > 64).
// TABLE: the target's sum over its state counts depends on the source bin only
// through q = c / N, so the CTA first tabulates F(c) = sum_a g(n_a q) - sum_x
// g(n_x q) for every count c in [0, N] (shared memory, N + 1 floats), with the
// same operations in the same order as the per-pair loop, then each pair adds
// F(c_b) over its source bins: the same floats, bitwise, in (N + 1) instead of
// (sources x bins) evaluations of the state sum.
template <bool TABLE>
__global__ void __launch_bounds__(256) eiid_kernel(const uint8_t* __restrict__ bins, int64_t ld,
                                                   const int32_t* __restrict__ npv, int n, int N,
                                                   int lag, const float* __restrict__ q,
                                                   const int* __restrict__ cnt,
                                                   const float* __restrict__ gtab,
                                                   float* __restrict__ out) {
  extern __shared__ float Ftab[];  // TABLE: N + 1 entries
  __shared__ int hz[kEiidMaxB * kEiidMaxB];
  __shared__ int hx[kEiidMaxB];
  __shared__ float la[kEiidMaxB * kEiidMaxB + kEiidMaxB];
  __shared__ float tab[kGTable];
  __shared__ int nz, nx;
  const int t = blockIdx.x;
  const int bt = npv[t];
  const float nan = __int_as_float(0x7fc00000);
  if (bt < 1 || bt > kEiidMaxB) {
    for (int s = threadIdx.x; s < n; s += blockDim.x)
      if (s != t) out[(int64_t)s * n + t] = nan;
    return;
  }
  for (int i = threadIdx.x; i < bt * bt; i += blockDim.x) hz[i] = 0;
  for (int i = threadIdx.x; i < kEiidMaxB; i += blockDim.x) hx[i] = 0;
  for (int i = threadIdx.x; i < kGTable; i += blockDim.x) tab[i] = gtab[i];
  if (threadIdx.x == 0) nz = nx = 0;
  __syncthreads();
  const uint8_t* row = bins + (int64_t)t * ld;
  for (int s = threadIdx.x; s < N; s += blockDim.x) {
    const int x0 = row[s], x1 = row[s + lag];
    if (x0 < bt && x1 < bt) {
      atomicAdd(&hz[x1 * bt + x0], 1);
      atomicAdd(&hx[x0], 1);
    }
  }
  __syncthreads();
  // compact lists: the non-zero n_a, then the non-zero n_x after them, in index
  // order (one warp, ballot + prefix count), so every run sums the terms below
  // in the same order and E_iid is bitwise reproducible
  if (threadIdx.x < 32) {
    const unsigned lane = threadIdx.x;
    const unsigned below = (1u << lane) - 1u;
    int base = 0;
    for (int i0 = 0; i0 < bt * bt; i0 += 32) {
      const int i = i0 + (int)lane;
      const bool nzv = i < bt * bt && hz[i] != 0;
      const unsigned m = __ballot_sync(0xffffffffu, nzv);
      if (nzv) la[base + __popc(m & below)] = (float)hz[i];
      base += __popc(m);
    }
    const int kz0 = base;
    for (int i0 = 0; i0 < bt; i0 += 32) {
      const int i = i0 + (int)lane;
      const bool nzv = i < bt && hx[i] != 0;
      const unsigned m = __ballot_sync(0xffffffffu, nzv);
      if (nzv) la[base + __popc(m & below)] = (float)hx[i];
      base += __popc(m);
    }
    if (lane == 0) {
      nz = kz0;
      nx = base - kz0;
    }
  }
  __syncthreads();
  const int kz = nz;
  const int kx = nx;
  if (TABLE) {
    for (int c = threadIdx.x; c <= N; c += blockDim.x) {
      const float qb = (float)c / N;  // the source_marginal_kernel's q for count c
      float part = 0.f;
      if (qb > 0.f) {
        for (int a = 0; a < kz; ++a) part += g_poisson(la[a] * qb, tab);
        for (int a = 0; a < kx; ++a) part -= g_poisson(la[kz + a] * qb, tab);
      }
      Ftab[c] = part;
    }
    __syncthreads();
  }
  for (int s = threadIdx.x; s < n; s += blockDim.x) {
    if (s == t) continue;
    const int bs = npv[s];
    float acc = nan;
    if (bs >= 1 && bs <= kEiidMaxB) {
      acc = 0.f;
      if (TABLE) {
        const int* cs = cnt + (int64_t)s * kEiidMaxB;
        for (int b = 0; b < bs; ++b) {
          const int c = cs[b];
          if (c <= 0) continue;
          acc += Ftab[c];
        }
      } else {
        const float* qs = q + (int64_t)s * kEiidMaxB;
        for (int b = 0; b < bs; ++b) {
          const float qb = qs[b];
          if (qb <= 0.f) continue;
          float part = 0.f;
          for (int a = 0; a < kz; ++a) part += g_poisson(la[a] * qb, tab);
          for (int a = 0; a < kx; ++a) part -= g_poisson(la[kz + a] * qb, tab);
          acc += part;
        }
      }
    }
    out[(int64_t)s * n + t] = acc;
  }
}

__device__ __forceinline__ void pair_features(const float* __restrict__ gf, float eiid, int tgt,
                                              int src, float log2bl, float* x) {
  const float* t = gf + (int64_t)tgt * kGeneFeat;
  const float* s = gf + (int64_t)src * kGeneFeat;
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    x[k] = t[k];
    x[6 + k] = s[k];
  }
  x[12] = eiid != eiid ? eiid : log2f(fmaxf(eiid, 1e-6f));
  x[13] = log2bl;
  const float bt = exp2f(t[0]), bs = exp2f(s[0]);
  x[14] = log2f((bt - 1.f) * (bs - 1.f) * bt + 1.f);
  x[15] = t[2] + s[1];
}

// Forward of one sample with weights in shared memory (float, 16-byte
// aligned) and a transposed copy of W2 (w2t[i * kH + j] = W2[j][i]). Returns
// the two outputs; optionally stores z1 and z2 (pre-activations). The outer
// loop runs over the first hidden layer's units i; each g1[i] is added into all
// kH second-layer sums at once (kH independent chains, kept in registers).
// Every sum is still evaluated in the plain row order, b + w0*x0 + w1*x1 + ...
// left to right, so the outputs do not depend on this loop structure. Weights
// are read four at a time; all lanes read the same address (broadcast).
__device__ __forceinline__ void mlp_forward_one(const float* __restrict__ w,
                                                const float* __restrict__ w2t, const float* x,
                                                float* z1s, float* z2s, float& o0, float& o1) {
  const float4* w4 = reinterpret_cast<const float4*>(w);
  const float4* t4 = reinterpret_cast<const float4*>(w2t);
  float a2[kH];
#pragma unroll
  for (int j = 0; j < kH; ++j) a2[j] = w[kOffB2 + j];
#pragma unroll 1
  for (int i = 0; i < kH; ++i) {
    float a = w[kOffB1 + i];
#pragma unroll
    for (int f = 0; f < kIn / 4; ++f) {
      const float4 v = w4[(kOffW1 + i * kIn) / 4 + f];
      a = fmaf(v.x, x[4 * f], a);
      a = fmaf(v.y, x[4 * f + 1], a);
      a = fmaf(v.z, x[4 * f + 2], a);
      a = fmaf(v.w, x[4 * f + 3], a);
    }
    if (z1s) z1s[i] = a;
    const float g = gelu(a);
#pragma unroll
    for (int j = 0; j < kH / 4; ++j) {
      const float4 v = t4[(i * kH) / 4 + j];
      a2[4 * j] = fmaf(v.x, g, a2[4 * j]);
      a2[4 * j + 1] = fmaf(v.y, g, a2[4 * j + 1]);
      a2[4 * j + 2] = fmaf(v.z, g, a2[4 * j + 2]);
      a2[4 * j + 3] = fmaf(v.w, g, a2[4 * j + 3]);
    }
  }
  o0 = w[kOffB3];
  o1 = w[kOffB3 + 1];
#pragma unroll
  for (int j = 0; j < kH; ++j) {
    if (z2s) z2s[j] = a2[j];
    const float g = gelu(a2[j]);
    o0 = fmaf(w[kOffW3 + j], g, o0);
    o1 = fmaf(w[kOffW3 + kH + j], g, o1);
  }
}

__device__ __forceinline__ void load_weights(const __nv_bfloat16* __restrict__ wb, float* ws) {
  for (int i = threadIdx.x; i < kParams; i += blockDim.x) ws[i] = __bfloat162float(wb[i]);
}

// w2t[i * kH + j] = W2[j][i], the layout mlp_forward_one reads.
__device__ __forceinline__ void load_w2t(const __nv_bfloat16* __restrict__ wb, float* w2t) {
  for (int k = threadIdx.x; k < kH * kH; k += blockDim.x) {
    const int i = k / kH, j = k - i * kH;
    w2t[k] = __bfloat162float(wb[kOffW2 + j * kH + i]);
  }
}

// Inference over all pairs: mu_log/sigma_log matrices at [src, tgt] (diagonal
// untouched), features standardised by (fmean, fstd); NaN features give NaN
// outputs (the caller sends those pairs to the full surrogate test).
__global__ void __launch_bounds__(128, 4) null_predict_kernel(
    const float* __restrict__ gf, const float* __restrict__ eiid, int n, float log2bl,
    const __nv_bfloat16* __restrict__ wb, const float* __restrict__ fmean,
    const float* __restrict__ fstd, float* __restrict__ out0, float* __restrict__ out1) {
  __shared__ __align__(16) float w[kParams];
  __shared__ __align__(16) float w2t[kH * kH];
  __shared__ float mu[kIn], sd[kIn];
  load_weights(wb, w);
  load_w2t(wb, w2t);
  if (threadIdx.x < kIn) {
    mu[threadIdx.x] = fmean[threadIdx.x];
    sd[threadIdx.x] = fstd[threadIdx.x];
  }
  __syncthreads();
  const int64_t total = (int64_t)n * n;
  for (int64_t m = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; m < total;
       m += (int64_t)gridDim.x * blockDim.x) {
    const int src = (int)(m / n), tgt = (int)(m - (int64_t)src * n);
    if (src == tgt) continue;
    float x[kIn];
    pair_features(gf, eiid[m], tgt, src, log2bl, x);
#pragma unroll
    for (int f = 0; f < kIn; ++f) x[f] = (x[f] - mu[f]) / sd[f];
    float o0, o1;
    mlp_forward_one(w, w2t, x, nullptr, nullptr, o0, o1);
    out0[m] = o0;
    out1[m] = o1;
  }
}

// Raw (unstandardised) features of a pair list.
__global__ void pair_features_kernel(const float* __restrict__ gf, const float* __restrict__ eiid,
                                     int n, const int32_t* __restrict__ tgt,
                                     const int32_t* __restrict__ src, int64_t P, float log2bl,
                                     float* __restrict__ X) {
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < P;
       p += (int64_t)gridDim.x * blockDim.x) {
    float x[kIn];
    const int t = tgt[p], s = src[p];
    pair_features(gf, eiid[(int64_t)s * n + t], t, s, log2bl, x);
#pragma unroll
    for (int f = 0; f < kIn; ++f) X[p * kIn + f] = x[f];
  }
}

// Training forward: X (B x 16, standardised), stores z1 (B x 64), z2 (B x 64),
// out (B x 2) and dout = out - Y; loss[0] += sum of squared errors / 2.
__global__ void __launch_bounds__(128) mlp_train_forward_kernel(
    const float* __restrict__ X, const float* __restrict__ Y, int B,
    const __nv_bfloat16* __restrict__ wb, float* __restrict__ z1, float* __restrict__ z2,
    float* __restrict__ dout, float* __restrict__ loss) {
  __shared__ __align__(16) float w[kParams];
  __shared__ __align__(16) float w2t[kH * kH];
  load_weights(wb, w);
  load_w2t(wb, w2t);
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.f;
  if (b < B) {
    float x[kIn];
#pragma unroll
    for (int f = 0; f < kIn; ++f) x[f] = X[(int64_t)b * kIn + f];
    float o0, o1;
    mlp_forward_one(w, w2t, x, z1 + (int64_t)b * kH, z2 + (int64_t)b * kH, o0, o1);
    const float d0 = o0 - Y[2 * b], d1 = o1 - Y[2 * b + 1];
    dout[2 * b] = d0;
    dout[2 * b + 1] = d1;
    l = 0.5f * (d0 * d0 + d1 * d1);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, l);
}

// Backward deltas per sample: dz2 = (W3^T dout) * gelu'(z2), dz1 = (W2^T dz2) * gelu'(z1).
// Overwrites z2 with dz2 and z1 with dz1 (the pre-activations are not needed after).
__global__ void __launch_bounds__(128) mlp_train_deltas_kernel(
    const __nv_bfloat16* __restrict__ wb, const float* __restrict__ dout, int B,
    float* __restrict__ z1, float* __restrict__ z2) {
  __shared__ __align__(16) float w[kParams];
  load_weights(wb, w);
  __syncthreads();
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= B) return;
  const float d0 = dout[2 * b], d1 = dout[2 * b + 1];
  float* zz2 = z2 + (int64_t)b * kH;
  float* zz1 = z1 + (int64_t)b * kH;
  float dz2[kH];
#pragma unroll 8
  for (int j = 0; j < kH; ++j) {
    const float dg = w[kOffW3 + j] * d0 + w[kOffW3 + kH + j] * d1;
    dz2[j] = dg * gelu_grad(zz2[j]);
    zz2[j] = dz2[j];
  }
  for (int i = 0; i < kH; ++i) {
    float dg = 0.f;
#pragma unroll 8
    for (int j = 0; j < kH; ++j) dg = fmaf(w[kOffW2 + j * kH + i], dz2[j], dg);
    zz1[i] = dg * gelu_grad(zz1[i]);
  }
}

// Weight gradients as batch reductions, one thread per parameter, averaged over B.
// Needs the layer inputs: x (X), g1 = gelu(z1_pre) and g2 = gelu(z2_pre), recomputed
// from stored copies z1p / z2p of the pre-activations.
__global__ void mlp_weight_grads_kernel(const float* __restrict__ X, const float* __restrict__ z1p,
                                        const float* __restrict__ z2p,
                                        const float* __restrict__ dz1, const float* __restrict__ dz2,
                                        const float* __restrict__ dout, int B,
                                        float* __restrict__ grad) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  float acc = 0.f;
  if (p < kOffB1) {  // W1[i][f]
    const int i = p / kIn, f = p - i * kIn;
    for (int b = 0; b < B; ++b) acc = fmaf(dz1[(int64_t)b * kH + i], X[(int64_t)b * kIn + f], acc);
  } else if (p < kOffW2) {  // b1[i]
    const int i = p - kOffB1;
    for (int b = 0; b < B; ++b) acc += dz1[(int64_t)b * kH + i];
  } else if (p < kOffB2) {  // W2[j][i]
    const int q = p - kOffW2, j = q / kH, i = q - j * kH;
    for (int b = 0; b < B; ++b)
      acc = fmaf(dz2[(int64_t)b * kH + j], gelu(z1p[(int64_t)b * kH + i]), acc);
  } else if (p < kOffW3) {  // b2[j]
    const int j = p - kOffB2;
    for (int b = 0; b < B; ++b) acc += dz2[(int64_t)b * kH + j];
  } else if (p < kOffB3) {  // W3[k][j]
    const int q = p - kOffW3, k = q / kH, j = q - k * kH;
    for (int b = 0; b < B; ++b) acc = fmaf(dout[2 * b + k], gelu(z2p[(int64_t)b * kH + j]), acc);
  } else {  // b3[k]
    const int k = p - kOffB3;
    for (int b = 0; b < B; ++b) acc += dout[2 * b + k];
  }
  grad[p] = acc / (float)B;
}

// Adam on the FP32 master copy, then the BF16 copy used by the forward kernels.
__global__ void mlp_adam_kernel(float* __restrict__ master, const float* __restrict__ grad,
                                float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                                float b2, float eps, float bc1, float bc2, float wd,
                                __nv_bfloat16* __restrict__ wb) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const float g = grad[p] + wd * master[p];
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  const float upd = (mm / bc1) / (sqrtf(vv / bc2) + eps);
  const float w = master[p] - lr * upd;
  master[p] = w;
  wb[p] = __float2bfloat16_rn(w);
}

__global__ void to_bf16_kernel(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst,
                               int count) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < count) dst[p] = __float2bfloat16_rn(src[p]);
}

}  // namespace
}  // namespace tenex

using namespace tenex;

extern "C" int tenex_mlp_param_count(void) { return kParams; }

extern "C" int tenex_gene_features(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                                   int n_vars, int64_t row_len, int64_t lag, float* feat,
                                   void* stream) {
  if (!bins || !n_per_var || !feat) return fail(TENEX_ERR_BADARG, "null pointer");
  if (n_vars < 1 || lag < 1 || row_len <= lag) return fail(TENEX_ERR_BADARG, "bad shape");
  gene_features_kernel<<<n_vars, 256, 0, as_stream(stream)>>>(bins, ld, n_per_var, n_vars,
                                                              (int)(row_len - lag), (int)lag, feat);
  return check_launch("gene_features_kernel");
}

extern "C" size_t tenex_eiid_workspace_bytes(int n_vars) {
  return n_vars < 1 ? 0
                    : (size_t)n_vars * kEiidMaxB * (sizeof(float) + sizeof(int)) +
                          kGTable * sizeof(float);
}

extern "C" int tenex_eiid_matrix(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                                 int n_vars, int64_t row_len, int64_t lag, float* eiid,
                                 void* workspace, size_t workspace_bytes, void* stream) {
  if (!bins || !n_per_var || !eiid || !workspace) return fail(TENEX_ERR_BADARG, "null pointer");
  if (n_vars < 2 || lag < 1 || row_len <= lag) return fail(TENEX_ERR_BADARG, "bad shape");
  if (row_len - lag >= ((int64_t)1 << 31)) return fail(TENEX_ERR_UNSUPPORTED, "N >= 2^31");
  if (workspace_bytes < tenex_eiid_workspace_bytes(n_vars))
    return fail(TENEX_ERR_BADARG, "workspace of %zu bytes < %zu", workspace_bytes,
                tenex_eiid_workspace_bytes(n_vars));
  if (reinterpret_cast<uintptr_t>(workspace) % 16)
    return fail(TENEX_ERR_BADARG, "workspace must be 16-byte aligned");
  cudaStream_t s = as_stream(stream);
  float* q = static_cast<float*>(workspace);
  float* tab = q + (size_t)n_vars * kEiidMaxB;
  int* cnt = reinterpret_cast<int*>(tab + kGTable);
  const int N = (int)(row_len - lag);
  g_table_kernel<<<kGTable / 256, 256, 0, s>>>(tab);
  source_marginal_kernel<<<n_vars, 256, 0, s>>>(bins, ld, N, q, cnt);
  // the count table pays when it is smaller than the per-pair work it replaces
  // (N + 1 entries against ~n sources x a few bins) and fits shared memory
  DevAttr A;
  int st = current_device_attr(&A);
  if (st) return st;
  cudaFuncAttributes fa{};
  cudaFuncGetAttributes(&fa, eiid_kernel<true>);
  const int64_t tab_bytes = ((int64_t)N + 1) * (int64_t)sizeof(float);
  if ((int64_t)N + 1 <= 4 * (int64_t)n_vars && tab_bytes + (int64_t)fa.sharedSizeBytes <= A.smem_optin) {
    cudaError_t e = cudaFuncSetAttribute(eiid_kernel<true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)tab_bytes);
    if (e != cudaSuccess) return check_cuda(e, "cudaFuncSetAttribute");
    eiid_kernel<true><<<n_vars, 256, (size_t)tab_bytes, s>>>(bins, ld, n_per_var, n_vars, N,
                                                             (int)lag, q, cnt, tab, eiid);
  } else {
    eiid_kernel<false><<<n_vars, 256, 0, s>>>(bins, ld, n_per_var, n_vars, N, (int)lag, q, cnt,
                                              tab, eiid);
  }
  return check_launch("eiid kernels");
}

extern "C" int tenex_pair_features(const float* gene_feat, const float* eiid, int n_vars,
                                   const int32_t* tgt, const int32_t* src, int64_t n_pairs,
                                   float log2bl, float* X, void* stream) {
  if (!gene_feat || !eiid || !tgt || !src || !X) return fail(TENEX_ERR_BADARG, "null pointer");
  if (n_pairs <= 0) return TENEX_OK;
  const int blocks = (int)std::min<int64_t>((n_pairs + 255) / 256, 8192);
  pair_features_kernel<<<blocks, 256, 0, as_stream(stream)>>>(gene_feat, eiid, n_vars, tgt, src,
                                                              n_pairs, log2bl, X);
  return check_launch("pair_features_kernel");
}

extern "C" int tenex_null_predict(const float* gene_feat, const float* eiid, int n_vars,
                                  float log2bl, const void* weights_bf16, const float* feat_mean,
                                  const float* feat_std, float* out_mu, float* out_sigma,
                                  void* stream) {
  if (!gene_feat || !eiid || !weights_bf16 || !feat_mean || !feat_std || !out_mu || !out_sigma)
    return fail(TENEX_ERR_BADARG, "null pointer");
  if (n_vars < 2) return fail(TENEX_ERR_BADARG, "n_vars must be >= 2");
  DevAttr A;
  int st = current_device_attr(&A);
  if (st) return st;
  null_predict_kernel<<<A.sm_count * 8, 128, 0, as_stream(stream)>>>(
      gene_feat, eiid, n_vars, log2bl, static_cast<const __nv_bfloat16*>(weights_bf16),
      feat_mean, feat_std, out_mu, out_sigma);
  return check_launch("null_predict_kernel");
}

extern "C" int tenex_mlp_train_step(const float* X, const float* Y, int batch, void* weights_bf16,
                                    float* master, float* adam_m, float* adam_v, float* scratch,
                                    float lr, float beta1, float beta2, float eps, float wd,
                                    int step, float* loss, void* stream) {
  if (!X || !Y || !weights_bf16 || !master || !adam_m || !adam_v || !scratch || !loss)
    return fail(TENEX_ERR_BADARG, "null pointer");
  if (batch < 1 || step < 1) return fail(TENEX_ERR_BADARG, "batch and step must be >= 1");
  cudaStream_t s = as_stream(stream);
  // scratch layout: z1 | z2 | z1 copy | z2 copy | dout | grad
  float* z1 = scratch;
  float* z2 = z1 + (int64_t)batch * kH;
  float* z1p = z2 + (int64_t)batch * kH;
  float* z2p = z1p + (int64_t)batch * kH;
  float* dout = z2p + (int64_t)batch * kH;
  float* grad = dout + (int64_t)batch * kOut;
  __nv_bfloat16* wb = static_cast<__nv_bfloat16*>(weights_bf16);
  const int blocks = (batch + 127) / 128;
  mlp_train_forward_kernel<<<blocks, 128, 0, s>>>(X, Y, batch, wb, z1, z2, dout, loss);
  cudaError_t e = cudaMemcpyAsync(z1p, z1, sizeof(float) * 2 * (size_t)batch * kH,
                                  cudaMemcpyDeviceToDevice, s);  // z1|z2 -> z1p|z2p
  if (e != cudaSuccess) return check_cuda(e, "copy pre-activations");
  mlp_train_deltas_kernel<<<blocks, 128, 0, s>>>(wb, dout, batch, z1, z2);
  mlp_weight_grads_kernel<<<(kParams + 127) / 128, 128, 0, s>>>(X, z1p, z2p, z1, z2, dout, batch,
                                                                grad);
  const float bc1 = 1.f - powf(beta1, (float)step), bc2 = 1.f - powf(beta2, (float)step);
  mlp_adam_kernel<<<(kParams + 127) / 128, 128, 0, s>>>(master, grad, adam_m, adam_v, lr, beta1,
                                                        beta2, eps, bc1, bc2, wd, wb);
  return check_launch("mlp train step");
}

extern "C" size_t tenex_mlp_scratch_floats(int batch) {
  return (size_t)batch * (4 * kH + kOut) + kParams;
}

extern "C" int tenex_mlp_gradients(const float* X, const float* Y, int batch,
                                   const void* weights_bf16, float* scratch, float* grad_out,
                                   float* loss, void* stream) {
  if (!X || !Y || !weights_bf16 || !scratch || !grad_out || !loss)
    return fail(TENEX_ERR_BADARG, "null pointer");
  cudaStream_t s = as_stream(stream);
  float* z1 = scratch;
  float* z2 = z1 + (int64_t)batch * kH;
  float* z1p = z2 + (int64_t)batch * kH;
  float* z2p = z1p + (int64_t)batch * kH;
  float* dout = z2p + (int64_t)batch * kH;
  const __nv_bfloat16* wb = static_cast<const __nv_bfloat16*>(weights_bf16);
  const int blocks = (batch + 127) / 128;
  mlp_train_forward_kernel<<<blocks, 128, 0, s>>>(X, Y, batch, wb, z1, z2, dout, loss);
  cudaError_t e = cudaMemcpyAsync(z1p, z1, sizeof(float) * 2 * (size_t)batch * kH,
                                  cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return check_cuda(e, "copy pre-activations");
  mlp_train_deltas_kernel<<<blocks, 128, 0, s>>>(wb, dout, batch, z1, z2);
  mlp_weight_grads_kernel<<<(kParams + 127) / 128, 128, 0, s>>>(X, z1p, z2p, z1, z2, dout, batch,
                                                                grad_out);
  return check_launch("mlp gradients");
}

extern "C" int tenex_to_bf16(const float* src, void* dst, int count, void* stream) {
  if (!src || !dst || count < 0) return fail(TENEX_ERR_BADARG, "bad arguments");
  if (count == 0) return TENEX_OK;
  to_bf16_kernel<<<(count + 255) / 256, 256, 0, as_stream(stream)>>>(
      src, static_cast<__nv_bfloat16*>(dst), count);
  return check_launch("to_bf16_kernel");
}
