/*
 * te_oracle.c — CPU ORACLE for the TE hot path. TEST INFRASTRUCTURE ONLY.
 *
 * This file is the checker: tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline / reference arm may call it; the product path never does.
 * It restates, in plain C, the reference algorithms below (file:line relative
 * to the reference project):
 *
 *   oracle_fsbwl        tenex/preprocess.py:61-88 (bin_fsbw_l_numpy) with numpy's
 *                       float32 pairwise summation (numpy/_core/src/umath/
 *                       loops_utils.h.src, PW_BLOCKSIZE 128) and np.std's
 *                       float64 division by the integer count (_methods.py _var)
 *   oracle_remap        tenex/preprocess.py:401-459 (remap_bins: per-gene
 *                       torch.unique(return_inverse) = rank among sorted uniques)
 *   oracle_coarsen      tenex/preprocess.py:462-551 (new = old*limit // n_per_var)
 *   oracle_counts       tenex/kernels/scatter_add.py:63-90 (cnt3 via flat index
 *                       xt1*B^2 + xt*B + yt) with per-pair b_t, b_s layout of
 *                       tenex/csrc/adaptive_smem.cu:77
 *   oracle_te_*         tenex/csrc/full_smem.cu:113-141 (sum over c3>0 of
 *                       c3*log2(c3*c1/(c2a*c2b)) / N), evaluated in float64
 *
 * Bins are int32, row-major with row stride ld; sample s in [0, N) of a pair
 * reads x[s+lag], x[s] (target) and y[s] (source), N = row_len - lag.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* numpy FLOAT_pairwise_sum for a contiguous float32 array. */
static float pw_sum_f32(const float* a, int64_t n) {
  if (n < 8) {
    float res = 0.f;
    for (int64_t i = 0; i < n; i++) res += a[i];
    return res;
  } else if (n <= 128) {
    float r[8];
    for (int k = 0; k < 8; k++) r[k] = a[k];
    int64_t i;
    for (i = 8; i < n - (n % 8); i += 8) {
      for (int k = 0; k < 8; k++) r[k] += a[i + k];
    }
    float res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
    for (; i < n; i++) res += a[i];
    return res;
  } else {
    int64_t n2 = n / 2;
    n2 -= n2 % 8;
    return pw_sum_f32(a, n2) + pw_sum_f32(a + n2, n - n2);
  }
}

/* np.std(row, ddof=1) in float32, bit-for-bit as numpy computes it. */
float oracle_std_ddof1(const float* row, int T, float* scratch) {
  float s = pw_sum_f32(row, T);
  float mean = (float)((double)s / (double)T);
  for (int t = 0; t < T; t++) {
    float d = row[t] - mean;
    scratch[t] = d * d;
  }
  float ss = pw_sum_f32(scratch, T);
  int64_t cnt = T - 1 > 0 ? T - 1 : 0;
  float var = (float)((double)ss / (double)cnt);
  return sqrtf(var);
}

/* FSBW-L binning: bins (n, T) int32 before clamp/remap, n_bins (n,). */
void oracle_fsbwl(const float* x, int n, int T, float kp, int32_t* bins, int32_t* n_bins) {
#pragma omp parallel
  {
    float* scratch = (float*)malloc(sizeof(float) * (size_t)(T > 0 ? T : 1));
#pragma omp for schedule(static)
    for (int g = 0; g < n; g++) {
      const float* row = x + (int64_t)g * T;
      float sd = oracle_std_ddof1(row, T, scratch);
      if (sd == 0.f || isnan(sd)) sd = 1.0f;
      float mn = row[0], mx = row[0];
      for (int t = 1; t < T; t++) {
        if (row[t] < mn) mn = row[t];
        if (row[t] > mx) mx = row[t];
      }
      n_bins[g] = (int32_t)ceilf((mx - mn) / sd);
      float shifted = mn - kp * sd;
      for (int t = 0; t < T; t++) bins[(int64_t)g * T + t] = (int32_t)floorf((row[t] - shifted) / sd);
    }
    free(scratch);
  }
}

/* Per-gene dense remap after clamp(min=0): bin -> rank among the gene's sorted
 * distinct values. In place; writes n_per_var; returns b_max. */
int oracle_remap(int32_t* bins, int n, int64_t row, int32_t* npv) {
  int bmax = 0;
#pragma omp parallel for schedule(static) reduction(max : bmax)
  for (int g = 0; g < n; g++) {
    int32_t* r = bins + (int64_t)g * row;
    int32_t hi = 0;
    for (int64_t i = 0; i < row; i++) {
      if (r[i] < 0) r[i] = 0;
      if (r[i] > hi) hi = r[i];
    }
    int32_t* rank = (int32_t*)calloc((size_t)hi + 1, sizeof(int32_t));
    for (int64_t i = 0; i < row; i++) rank[r[i]] = 1;
    int32_t c = 0;
    for (int32_t v = 0; v <= hi; v++) {
      int32_t present = rank[v];
      rank[v] = c;
      c += present;
    }
    for (int64_t i = 0; i < row; i++) r[i] = rank[r[i]];
    npv[g] = c;
    if (c > bmax) bmax = c;
    free(rank);
  }
  return bmax;
}

/* Coarsening: genes with n_per_var > limit get new = old*limit / n_per_var. */
int oracle_coarsen(int32_t* bins, int n, int64_t row, int32_t* npv, int limit) {
  int bmax = 0;
  for (int g = 0; g < n; g++) {
    if (npv[g] > limit) {
      int32_t* r = bins + (int64_t)g * row;
      for (int64_t i = 0; i < row; i++) r[i] = (int32_t)(((int64_t)r[i] * limit) / npv[g]);
      npv[g] = limit;
    }
    if (npv[g] > bmax) bmax = npv[g];
  }
  return bmax;
}

/* Joint counts of one pair: cnt[xt1*bt*bs + xt*bs + yt] (bt*bt*bs int64). */
void oracle_counts(const int32_t* bins, int64_t ld, int64_t row_len, int64_t lag, int tgt,
                   int src, int bt, int bs, int64_t* cnt) {
  const int32_t* x = bins + (int64_t)tgt * ld;
  const int32_t* y = bins + (int64_t)src * ld;
  const int64_t N = row_len - lag;
  memset(cnt, 0, sizeof(int64_t) * (size_t)bt * bt * bs);
  for (int64_t s = 0; s < N; s++) cnt[((int64_t)x[s + lag] * bt + x[s]) * bs + y[s]]++;
}

static double te_from_counts(const int64_t* c3, int bt, int bs, int64_t N, double* c1,
                             double* c2a, double* c2b) {
  memset(c1, 0, sizeof(double) * bt);
  memset(c2a, 0, sizeof(double) * bt * bt);
  memset(c2b, 0, sizeof(double) * bt * bs);
  for (int i = 0; i < bt; i++)
    for (int j = 0; j < bt; j++)
      for (int k = 0; k < bs; k++) {
        double v = (double)c3[((int64_t)i * bt + j) * bs + k];
        c1[j] += v;
        c2a[i * bt + j] += v;
        c2b[j * bs + k] += v;
      }
  double te = 0.0;
  for (int i = 0; i < bt; i++)
    for (int j = 0; j < bt; j++)
      for (int k = 0; k < bs; k++) {
        double c = (double)c3[((int64_t)i * bt + j) * bs + k];
        double den = c2a[i * bt + j] * c2b[j * bs + k];
        if (c > 0.0 && den > 0.0) te += c * log2(c * c1[j] / den);
      }
  return te / (double)N;
}

static void te_pair_list(const int32_t* bins, int64_t ld, int64_t row_len, int64_t lag,
                         const int32_t* npv, int bmax, const int64_t* tgts, const int64_t* srcs,
                         int64_t P, double* te, int nthreads) {
  const int64_t N = row_len - lag;
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
#else
  (void)nthreads;
#endif
#pragma omp parallel
  {
    int64_t* c3 = (int64_t*)malloc(sizeof(int64_t) * (size_t)bmax * bmax * bmax);
    double* c1 = (double*)malloc(sizeof(double) * bmax);
    double* c2a = (double*)malloc(sizeof(double) * bmax * bmax);
    double* c2b = (double*)malloc(sizeof(double) * bmax * bmax);
#pragma omp for schedule(dynamic, 64)
    for (int64_t p = 0; p < P; p++) {
      int t = (int)tgts[p], s = (int)srcs[p];
      int bt = npv[t], bs = npv[s];
      oracle_counts(bins, ld, row_len, lag, t, s, bt, bs, c3);
      te[p] = te_from_counts(c3, bt, bs, N, c1, c2a, c2b);
    }
    free(c3);
    free(c1);
    free(c2a);
    free(c2b);
  }
}

/* FP64 TE for pair-free ids [p0, p0+P). */
void oracle_te_pairfree(const int32_t* bins, int64_t ld, int n, int64_t row_len, int64_t lag,
                        const int32_t* npv, int64_t p0, int64_t P, double* te, int nthreads) {
  int bmax = 1;
  for (int g = 0; g < n; g++)
    if (npv[g] > bmax) bmax = npv[g];
  int64_t* tg = (int64_t*)malloc(sizeof(int64_t) * (size_t)(P > 0 ? P : 1));
  int64_t* sr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(P > 0 ? P : 1));
  for (int64_t q = 0; q < P; q++) {
    int64_t p = p0 + q;
    int64_t t = p / (n - 1), sl = p % (n - 1);
    tg[q] = t;
    sr[q] = sl + (sl >= t);
  }
  te_pair_list(bins, ld, row_len, lag, npv, bmax, tg, sr, P, te, nthreads);
  free(tg);
  free(sr);
}

/* FP64 TE for an explicit (target, source) pair list (pairs[2p]=tgt, pairs[2p+1]=src). */
void oracle_te_pairs(const int32_t* bins, int64_t ld, int n, int64_t row_len, int64_t lag,
                     const int32_t* npv, const int64_t* pairs, int64_t P, double* te,
                     int nthreads) {
  int bmax = 1;
  for (int g = 0; g < n; g++)
    if (npv[g] > bmax) bmax = npv[g];
  int64_t* tg = (int64_t*)malloc(sizeof(int64_t) * (size_t)(P > 0 ? P : 1));
  int64_t* sr = (int64_t*)malloc(sizeof(int64_t) * (size_t)(P > 0 ? P : 1));
  for (int64_t q = 0; q < P; q++) {
    tg[q] = pairs[2 * q];
    sr[q] = pairs[2 * q + 1];
  }
  te_pair_list(bins, ld, row_len, lag, npv, bmax, tg, sr, P, te, nthreads);
  free(tg);
  free(sr);
}
