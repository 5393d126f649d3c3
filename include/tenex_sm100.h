/*
 * tenex_sm100.h — C ABI of libtenex_sm100.so, the sm_100a (B200) kernels behind
 * the pairwise transfer-entropy (TE) path of TENEX.
 *
 * Every entry point:
 *   - takes plain device pointers, sizes and an explicit cudaStream_t (passed
 *     as void*; NULL means the legacy default stream),
 *   - is asynchronous with respect to the host unless stated otherwise,
 *   - returns a tenex_status (0 = OK); tenex_last_error() gives the text of the
 *     last failure on the calling thread.
 *
 * Bin layout used by all TE entry points ("padded rows"):
 *   bins[g * ld + i], g in [0, n_vars), i in [0, row_len), uint8, with
 *   ld * 1 byte a multiple of 16 and the base pointer 16-byte aligned.
 *   A reference tensor bin_arrs of shape (n, T, K) maps to row_len = T*K and
 *   lag = tau*K: sample s in [0, N), N = row_len - lag, has
 *   x_{t+tau} = row[s + lag], x_t = row[s], y_t = src_row[s]
 *   (reference: tenex/kernels/scatter_add.py:63-79, the (t, k) samples of one
 *   pair flattened in row-major order).
 *
 * Pair-free ids (reference: tenex/csrc/full_smem.cu:190-195):
 *   p = tgt * (n_vars - 1) + src_local, src = src_local + (src_local >= tgt).
 */
#ifndef TENEX_SM100_H
#define TENEX_SM100_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
enum {
  TENEX_OK = 0,
  TENEX_ERR_BADARG = 1,      /* invalid argument (shape, alignment, pointer) */
  TENEX_ERR_UNSUPPORTED = 2, /* configuration this build cannot run */
  TENEX_ERR_OOM = 3,         /* workspace too small / allocation failed */
  TENEX_ERR_LAUNCH = 4,      /* CUDA launch or runtime error */
  TENEX_ERR_TIMEOUT = 5,     /* a bounded device-side wait expired */
  TENEX_ERR_BADDATA = 6      /* bin value >= n_per_var[g] or n_per_var out of range */
};

/* Output layouts of the TE entry points. */
enum {
  TENEX_OUT_PAIRFREE = 0, /* out[p - pair_offset], float32                         */
  TENEX_OUT_MATRIX = 1    /* out[src * out_ld + tgt] = TE(src -> tgt), float32     */
};

typedef struct {
  int sm_count;
  int smem_optin;         /* cudaDevAttrMaxSharedMemoryPerBlockOptin */
  int smem_per_sm;        /* cudaDevAttrMaxSharedMemoryPerMultiprocessor */
  int l2_bytes;
  int cc_major, cc_minor;
  int max_threads_per_sm;
} tenex_dev_info;

/* Launch shape of the persistent histogram kernels (0 fields, or a NULL config,
 * = defaults: 2 CTAs x 512 threads per SM, 512 sources per item; when the
 * largest pair's histogram does not fit two CTAs per SM, one CTA per SM, of
 * 1024 threads if neither threads nor ctas_per_sm was given). */
typedef struct {
  int threads;      /* threads per CTA: 128, 256, 512 or 1024          */
  int ctas_per_sm;  /* resident CTAs per SM (grid = sm_count * this)    */
  int src_chunk;    /* sources per work item (one target per item)     */
  int smem_bytes;   /* dynamic shared memory per CTA (0 = fill the SM)  */
} tenex_te_config;

int tenex_abi_version(void);
/* Copies the last error text of this thread into buf (NUL-terminated). */
int tenex_last_error(char* buf, size_t len);
/* Replaces get_smem_optin (tenex/csrc/full_smem.cu:150-155) and the
 * query_smem_optin helper (tenex/kernels/__init__.py:44-71). */
int tenex_device_query(int device, tenex_dev_info* info);

/* Bytes of device workspace the TE / surrogate entry points need: a 256-byte
 * header (work tickets, validation words) plus the source processing order
 * (n_vars int32, genes sorted by bin count), rounded up to 256 bytes; plus, when
 * pairs with b up to b_max would not fit a shared-memory slot on the current
 * device (coarsening off), the global-memory histogram slots of the overflow
 * launch. A workspace without them makes such a call fail with the size it
 * needs. */
size_t tenex_te_workspace_bytes(int n_vars, int64_t row_len, int b_max);

/* The launch shape the histogram kernels would use on the current device for
 * rows of row_len samples at this lag and b_max, with cfg as given (NULL or 0
 * fields: the defaults above): threads per CTA, CTAs per SM, dynamic shared
 * memory per CTA and sources per item. Same planner as the launches. */
int tenex_te_launch_shape(int64_t row_len, int64_t lag, int b_max, const tenex_te_config* cfg,
                          int* threads, int* ctas_per_sm, int* smem_bytes, int* src_chunk);

/* Reads back the data-validation word a previous TE call left in the
 * workspace (synchronises `stream`). Returns TENEX_ERR_BADDATA if any bin value
 * was >= its gene's n_per_var, else TENEX_OK. */
int tenex_workspace_status(const void* workspace, void* stream);

/* Multi-bin TE over a contiguous pair-free id range, exact integer counts in
 * shared memory, fused count -> marginal -> TE reduction.
 * Replaces te_smem_launch_pairfree (tenex/csrc/full_smem.cu:350-381) and
 * te_adaptive_smem_kernel_pairfree's launcher (tenex/kernels/adaptive_smem.py:1029-1107):
 * one kernel covers both Full-SMEM (uniform b) and Adaptive-SMEM (per-gene b).
 * b_max = max(n_per_var) (the reference's B argument), 1..255; every
 * n_per_var[g] must lie in [1, b_max] and every bin of gene g below n_per_var[g]
 * (checked on the device; see tenex_workspace_status). n_pairs == 0 returns
 * TENEX_OK without touching out or the workspace (either may then be NULL). */
int tenex_te_pairfree(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                      int b_max, int n_vars, int64_t row_len, int64_t lag,
                      int64_t pair_offset, int64_t n_pairs,
                      float* out, int out_mode, int64_t out_ld,
                      void* workspace, size_t workspace_bytes,
                      const tenex_te_config* cfg, void* stream);

/* Same kernel, additionally exporting the raw int32 joint counts of every pair
 * for parity checks: counts[(p - pair_offset) * counts_stride + xt1*bt*bs + xt*bs + yt]
 * (the index of tenex/csrc/adaptive_smem.cu:77). */
int tenex_te_pairfree_counts(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                             int b_max, int n_vars, int64_t row_len, int64_t lag,
                             int64_t pair_offset, int64_t n_pairs,
                             float* out, int32_t* counts, int64_t counts_stride,
                             void* workspace, size_t workspace_bytes,
                             const tenex_te_config* cfg, void* stream);

/* Same computation as tenex_te_pairfree, for callers that cannot allocate
 * device memory. (No counterpart in the reference.) Its scratch is a fixed
 * 4 MiB area inside the library's device image, so n_vars * 4 plus about
 * 512 bytes must fit in 4 MiB (TENEX_ERR_UNSUPPORTED otherwise; up to about
 * 1,048,000 genes). Bins whose largest histograms do not fit shared memory
 * (coarsening off) need global-memory slots the area cannot hold: such calls
 * return TENEX_ERR_UNSUPPORTED before launching anything (use tenex_te_pairfree).
 * The area's address is looked up by the first call on each device (make that
 * call before any stream capture) and kept for the life of the process, so a
 * device reset (cudaDeviceReset) after that first call is not supported; every
 * call reuses and re-initialises the same area, so calls that overlap on the
 * GPU race and must not be issued. status: optional device int32 that receives
 * the call's outcome, written on `stream`: 0 = inputs valid and every pair
 * computed (also for an empty range), 1 = a bin value >= its gene's n_per_var
 * or n_per_var outside [1, b_max] (no TE computed), 3 = a work item's histogram
 * did not fit shared memory (its pairs not computed); NULL skips it.
 * Allocates nothing: no cudaMalloc, cudaFree or allocating library call. */
int tenex_te_pairfree_static(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                             int b_max, int n_vars, int64_t row_len, int64_t lag,
                             int64_t pair_offset, int64_t n_pairs, float* out, int out_mode,
                             int64_t out_ld, int32_t* status, const tenex_te_config* cfg,
                             void* stream);

/* TE for an explicit pair list (the source-filter path of the reference:
 * te_smem_launch, tenex/csrc/full_smem.cu:319-347, and compute_single_gpu).
 * pairs: device int64 (n_pairs, 2) = [target, source], grouped so that equal
 * targets are consecutive; item_start: device int64 (n_items + 1) splitting the
 * list into runs of one target (the caller chooses the run length, e.g. <= 128).
 * out[i] = TE(pairs[i,1] -> pairs[i,0]). Malformed items (mixed targets, indices
 * out of range) are skipped and reported by tenex_workspace_status. */
int tenex_te_pairs(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                   int b_max, int n_vars, int64_t row_len, int64_t lag,
                   const int64_t* pairs, int64_t n_pairs, const int64_t* item_start,
                   int64_t n_items, float* out, void* workspace, size_t workspace_bytes,
                   const tenex_te_config* cfg, void* stream);

/* Surrogate accumulation: TE of already-shuffled bins for the pair range, then
 * sum[s*n+t] += te, sumsq[s*n+t] += te^2 (te rounded to float32 first, then
 * widened), count_ge[s*n+t] += (te >= observed[s*n+t]).
 * Replaces the per-surrogate accumulator update of
 * tenex/inference/surrogate_test.py:389-406. */
int tenex_surrogate_accumulate(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                               int b_max, int n_vars, int64_t row_len, int64_t lag,
                               int64_t pair_offset, int64_t n_pairs,
                               const float* observed, double* sum, double* sumsq,
                               int32_t* count_ge,
                               void* workspace, size_t workspace_bytes,
                               const tenex_te_config* cfg, void* stream);

/* Surrogate accumulation for an explicit pair list (same pair/item conventions as
 * tenex_te_pairs; accumulators indexed [src * n + tgt]). */
int tenex_surrogate_accumulate_pairs(const uint8_t* bins, int64_t ld, const int32_t* n_per_var,
                                     int b_max, int n_vars, int64_t row_len, int64_t lag,
                                     const int64_t* pairs, int64_t n_pairs,
                                     const int64_t* item_start, int64_t n_items,
                                     const float* observed, double* sum, double* sumsq,
                                     int32_t* count_ge, void* workspace, size_t workspace_bytes,
                                     const tenex_te_config* cfg, void* stream);

/* Surrogate accumulation from a finished TE matrix te[src*n + tgt] (the
 * matrix-kernel path, GEMM-B2): same update as tenex_surrogate_accumulate, off
 * the diagonal. */
int tenex_stats_accumulate(const float* te, const float* observed, double* sum, double* sumsq,
                           int32_t* count_ge, int n_vars, void* stream);

/* Block shuffle of every gene's time axis (tenex/inference/surrogate_test.py:107-162):
 * out[g, t*K + k] = in[g, (perm[g, t/bl]*bl + t%bl)*K + k] for t < n_blocks*bl,
 * tail t >= n_blocks*bl unchanged. bl = 1 with n_blocks = T is the random shuffle.
 * perm is int32 (n_vars, n_blocks) for one surrogate. */
int tenex_block_shuffle(const uint8_t* in, int64_t in_ld, int n_vars, int64_t T, int K,
                        const int32_t* perm, int n_blocks, int block_length,
                        uint8_t* out, int64_t out_ld, void* stream);

/* n_copies block shuffles of the same bins in one launch (the learned null's
 * verification pass): copy s uses perms + s*n_vars*n_blocks and writes the
 * (n_vars, out_ld) rows at out + s*out_copy_stride. The outputs must not
 * overlap the input or each other; T*K < 2^31. */
int tenex_block_shuffle_many(const uint8_t* in, int64_t in_ld, int n_vars, int64_t T, int K,
                             const int32_t* perms, int n_copies, int n_blocks, int block_length,
                             uint8_t* out, int64_t out_ld, int64_t out_copy_stride, void* stream);

/* FSBW-L discretisation, bit-identical to the reference's numpy path
 * (bin_fsbw_l_numpy, tenex/preprocess.py:61-88, then clamp(min=0) of :680):
 * x float32 (n_vars, T) row stride ldx; bins int32 (n_vars, T) row stride ldb;
 * n_bins[g] = ceil((max-min)/std). T <= 114688. */
int tenex_fsbwl_bins(const float* x, int64_t ldx, int n_vars, int T, float kp,
                     int32_t* bins, int64_t ldb, int32_t* n_bins, void* stream);

/* Dense per-gene relabelling, replaces remap_bins (tenex/preprocess.py:401-459):
 * out[g, i] = rank of max(raw[g, i], 0) among gene g's distinct values.
 * in_bytes 1 (uint8), 2 (uint16) or 4 (int32); out_bytes 1 (uint8) or 2 (uint16).
 * *err (device int, caller-zeroed) becomes 1 if a gene spans more than 8192 raw
 * values, 2 if a gene has more distinct values than the output type holds. */
int tenex_remap_dense(const void* raw, int in_bytes, int64_t ldr, int n_vars, int64_t row_len,
                      void* out, int out_bytes, int64_t ldo, int32_t* n_per_var, int* err,
                      void* stream);

/* In-place coarsening of uint8 padded rows, replaces coarsen_bins / coarsen_bins_cuda
 * (tenex/preprocess.py:462-551, tenex/csrc/adaptive_smem.cu:557-592):
 * genes with n_per_var > limit get bin*limit/n_per_var and n_per_var = limit. */
int tenex_coarsen(uint8_t* bins, int64_t ld, int n_vars, int64_t row_len, int32_t* n_per_var,
                  int limit, void* stream);

/* Coarsening of uint16 padded rows (genes with more than 256 distinct bins,
 * which the reference keeps as int16 until coarsened: tenex/preprocess.py:335-354
 * and the int16 branch of coarsen_bins, :520-536) into uint8 padded rows `out`:
 * genes with n_per_var > limit get bin*limit/n_per_var and n_per_var = limit,
 * the others are copied (their values are below n_per_var <= limit <= 255).
 * ldi in uint16 elements, ldo in bytes; in and out must not overlap. */
int tenex_coarsen_narrow(const uint16_t* in, int64_t ldi, int n_vars, int64_t row_len,
                         int32_t* n_per_var, int limit, uint8_t* out, int64_t ldo,
                         void* stream);

/* Binarisation 1[x > thr_g] (tenex/binarize.py:225-295; kernels of
 * tenex/csrc/binarize_cuda.cu:14-56): mode 0 nonzero (thr 0), 1 mean (numpy
 * float32 mean), 2 caller thresholds[g]. out: uint8 padded rows; n_per_var[g]
 * = 1 for a constant row, else 2 (the reference's max - min + 1). */
int tenex_binarize(const float* x, int64_t ldx, int n_vars, int T, int mode,
                   const float* thresholds, uint8_t* out, int64_t ldo, int32_t* n_per_var,
                   void* stream);

/* Median / quantile binarisation with numpy's thresholds (the reference's
 * default numpy backend, tenex/binarize.py:126-150: np.median, np.quantile
 * "linear"; replaces the chunked torch.quantile threshold of
 * tenex/kernels/binarize_kernel.py:158-183): median != 0 for np.median, else
 * quantile q in [0, 1]. A row holding a NaN gets numpy's NaN threshold (all
 * bins 0). Per-row radix selection, no sort; out and n_per_var as
 * tenex_binarize. */
int tenex_binarize_select(const float* x, int64_t ldx, int n_vars, int T, int median, double q,
                          uint8_t* out, int64_t ldo, int32_t* n_per_var, void* stream);

/* Binary (b_max = 2) TE matrix on the tensor cores; replaces compute_te_gemm_b2
 * (tenex/kernels/gemm_b2.py:307-425) and its Triton epilogue (:65-187).
 * bins: uint8 {0,1} padded rows (read in place by TMA: 16-byte aligned rows);
 * out[src * out_ld + tgt] = TE(src -> tgt) (diagonal untouched; the caller
 * zeroes it). L = row_len - lag < 2^24. workspace: tenex_b2_workspace_bytes(),
 * 256-byte aligned (the lag-shifted operand copy and per-gene counts). */
size_t tenex_b2_workspace_bytes(int n_vars, int64_t row_len, int64_t lag);
int tenex_te_binary_matrix(const uint8_t* bins, int64_t ld, int n_vars, int64_t row_len,
                           int64_t lag, float* out, int64_t out_ld, void* workspace,
                           size_t workspace_bytes, void* stream);
/* Same with the operand form chosen: kind 1 = int8 operands (tcgen05 kind::i8,
 * int32 sums), 2 = packed 4-bit operands (kind::mxf4: the 0/1 values as E2M1,
 * two per byte, unit block scales, float32 sums, exact below 2^24), 0 = the
 * default (2). Both give the same counts and TE. */
int tenex_te_binary_matrix_kind(const uint8_t* bins, int64_t ld, int n_vars, int64_t row_len,
                                int64_t lag, float* out, int64_t out_ld, void* workspace,
                                size_t workspace_bytes, int kind, void* stream);
/* Same, with the GEMM's target-tile width chosen by the caller: tile_n = 0
 * picks it from n_vars and the SM count (the width whose tiles finish in the
 * fewest rounds, tenex_b2_tile_n), else one of 128, 112, 96, 80, 64
 * (TENEX_ERR_BADARG otherwise). Every width gives bitwise the same matrix. */
int tenex_te_binary_matrix_ex(const uint8_t* bins, int64_t ld, int n_vars, int64_t row_len,
                              int64_t lag, float* out, int64_t out_ld, void* workspace,
                              size_t workspace_bytes, int kind, int tile_n, void* stream);
/* The target-tile width tenex_te_binary_matrix picks on the current device for
 * n_vars genes. */
int tenex_b2_tile_n(int n_vars, int* tile_n);
/* Error word of the last tenex_te_binary_matrix call on this workspace
 * (synchronises `stream`): TENEX_ERR_BADDATA if a bin was not 0 or 1,
 * TENEX_ERR_TIMEOUT if a pipeline wait expired. */
int tenex_b2_status(const void* workspace, int n_vars, int64_t row_len, int64_t lag,
                    void* stream);

/* DPI trimming of the FDR method's network; replaces the row-batched torch loop
 * of _trim (tenex/inference/fdr.py:61-133). te: n x n float (kept edges, 0
 * elsewhere), row stride ld. out[i*out_ld + j] = te[i][j] if keep_all[i], else
 * te[i][j] when te[i][j] >= max(0, max_{k: mediator[k]} min(te[i][k], te[k][j]))
 * + trim_threshold, else 0 (float32 sum and compare as in the reference).
 * mediator / keep_all: n bytes each, NULL = all k / no row. out must not alias te. */
int tenex_dpi_trim(const float* te, int64_t ld, int n_vars, const uint8_t* mediator,
                   const uint8_t* keep_all, float trim_threshold, float* out, int64_t out_ld,
                   void* stream);
/* Sparse form of tenex_dpi_trim (same rule, same results) for networks given in
 * CSR: row_ptr[n_vars + 1] (int64), col / val the nonzero entries (columns
 * ascending within a row). keep[e] = 1 if entry e survives, else 0. Work is
 * sum over k of (positive entries into k) x (positive entries out of k); one row
 * of n_vars floats must fit shared memory (TENEX_ERR_UNSUPPORTED otherwise). */
int tenex_dpi_trim_sparse(const int64_t* row_ptr, const int32_t* col, const float* val,
                          int n_vars, const uint8_t* mediator, const uint8_t* keep_all,
                          float trim_threshold, uint8_t* keep, void* stream);

/* ---- Learned null model of the surrogate test (no reference counterpart) ----
 * MLP 16 -> 64 -> 64 -> 2 (GELU), parameters W1[64][16] b1[64] W2[64][64] b2[64]
 * W3[2][64] b3[2] (tenex_mlp_param_count() values), BF16 for the forward,
 * FP32 master copy for training. Outputs: log(mu * N), log(sigma * N) of a
 * pair's surrogate-TE distribution. */
int tenex_mlp_param_count(void);
/* Per-gene features (n_vars x 8 float): log2 b, H(x_t), H(x_{t+lag}, x_t),
 * 2H - H2, log2 mean run length, 2^H / b (joint terms NaN when b > 64). */
int tenex_gene_features(const uint8_t* bins, int64_t ld, const int32_t* n_per_var, int n_vars,
                        int64_t row_len, int64_t lag, float* feat, void* stream);
/* Independence bias of every ordered pair, eiid[src*n + tgt] (float, NaN when
 * b_t or b_s > 64): E_iid = sum_{a,b} g(n_a q_b) - sum_{x,b} g(n_x q_b) with n_a the
 * counts of the target's (x_{t+lag}, x_t) states, n_x of x_t, q_b the source's
 * marginal over the same N = row_len - lag positions and g(m) = E[C ln C] - m ln m
 * for C ~ Poisson(m) (the expected plug-in bias of N ln2 * TE under independence).
 * Workspace: tenex_eiid_workspace_bytes(n_vars) bytes, 16-byte aligned. */
size_t tenex_eiid_workspace_bytes(int n_vars);
int tenex_eiid_matrix(const uint8_t* bins, int64_t ld, const int32_t* n_per_var, int n_vars,
                      int64_t row_len, int64_t lag, float* eiid, void* workspace,
                      size_t workspace_bytes, void* stream);
/* Raw 16 features of the pairs (tgt[i], src[i]) into X (n_pairs x 16); eiid is the
 * (n_vars x n_vars) matrix of tenex_eiid_matrix. */
int tenex_pair_features(const float* gene_feat, const float* eiid, int n_vars,
                        const int32_t* tgt, const int32_t* src, int64_t n_pairs, float log2bl,
                        float* X, void* stream);
/* Prediction for every ordered pair: out_mu[src*n + tgt], out_sigma[...] (log scale;
 * NaN where a feature is undefined); features standardised by feat_mean/feat_std. */
int tenex_null_predict(const float* gene_feat, const float* eiid, int n_vars, float log2bl,
                       const void* weights_bf16, const float* feat_mean, const float* feat_std,
                       float* out_mu, float* out_sigma, void* stream);
/* Scratch floats needed by a training step / gradient call of `batch` samples. */
size_t tenex_mlp_scratch_floats(int batch);
/* Gradients of the mean squared error / 2 over a batch (X standardised, Y targets)
 * w.r.t. all parameters (grad_out, tenex_mlp_param_count() floats); *loss += sum. */
int tenex_mlp_gradients(const float* X, const float* Y, int batch, const void* weights_bf16,
                        float* scratch, float* grad_out, float* loss, void* stream);
/* One Adam step (bias-corrected, decoupled weight decay wd) on the FP32 master
 * copy; refreshes the BF16 weights. */
int tenex_mlp_train_step(const float* X, const float* Y, int batch, void* weights_bf16,
                         float* master, float* adam_m, float* adam_v, float* scratch, float lr,
                         float beta1, float beta2, float eps, float wd, int step, float* loss,
                         void* stream);
int tenex_to_bf16(const float* src, void* dst, int count, void* stream);

/* Roofline probe (no reference counterpart): times `iters` shared-memory
 * atomicAdds per thread on every SM (mode 0 conflict-free int32, 1 conflict-free
 * 16-bit halves, 2 random words, 3 the same 32 words from every warp) and returns the increment count and the
 * milliseconds. Synchronises `stream`. */
int tenex_probe_smem_atomics(int mode, int iters, int64_t* increments, float* ms, void* stream);
/* Roofline probe (no reference counterpart): dense INT8 tensor-pipe rate. One CTA per SM
 * issues `iters` tcgen05.mma.kind::i8 (M=128, N=256, K=32) from shared-memory operands
 * into TMEM; returns the operation count (2*M*N*K per MMA) and the milliseconds.
 * Synchronises `stream`; TENEX_ERR_TIMEOUT if the bounded completion wait expired. */
int tenex_probe_tc_int8(int iters, double* ops, float* ms, void* stream);
/* Roofline probe (no reference counterpart): dense 4-bit (kind::mxf4, packed E2M1
 * with unit UE8M0 block scales) tensor-pipe rate, M=128, N=256, K=64 per MMA, the
 * denominator of the 4-bit GEMM-B2 form; same conventions as tenex_probe_tc_int8. */
int tenex_probe_tc_fp4(int iters, double* ops, float* ms, void* stream);
/* Roofline probe (no reference counterpart): the GEMM-B2 kernel's own MMA sequence
 * (per 128-byte K stage four K steps of an N = 2 tile_n and an N = tile_n MMA,
 * swizzled operands walking three stage buffers) issued back to back on every SM
 * with no copies and no waits: the rate that bounds the GEMM's main loop for
 * that instruction mix. kind: 1 = int8, 2 = 4-bit; tile_n in {128, 112, 96, 80,
 * 64}; `stages` K stages per SM; ops = 6 * 128 * tile_n * K per stage per SM. */
int tenex_probe_tc_gemm_b2(int kind, int tile_n, int stages, double* ops, float* ms,
                           void* stream);
/* Roofline probe (no reference counterpart): FP32 min/max issue rate, the bound of
 * tenex_dpi_trim. Every thread of 2 CTAs x 1024 threads per SM runs `iters` steps
 * of 8 independent chains (two min.f32 and one three-input max.f32 each); returns
 * the instruction count and the milliseconds. Synchronises `stream`. */
int tenex_probe_minmax(int iters, double* instructions, float* ms, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TENEX_SM100_H */
