"""CPU oracle for the TE hot path — TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference
arm import this module; the product path (tenex_b200) never does.

Contents (reference file:line relative to the reference project):
  fsbwl(x, kp)                 tenex/preprocess.py:61-88 + :680 clamp
  remap(bins)                  tenex/preprocess.py:401-459
  coarsen(bins, npv, limit)    tenex/preprocess.py:462-551
  binarize(x, method, q)       tenex/binarize.py:45-150 with the default numpy backend
                               (1[x > thr]; median = np.median, quantile = np.quantile
                               "linear" (Hyndman-Fan type 7), restated from a sort)
  counts(bins, lag, t, s, npv) tenex/kernels/scatter_add.py:63-90
  te_pairfree / te_pairs       tenex/csrc/full_smem.cu:113-141 in float64
  te_matrix                    pair-free output assembled as
                               tenex/transferentropy.py:1394-1410 does
  block_shuffle                tenex/inference/surrogate_test.py:107-162
  surrogate_stats              tenex/inference/surrogate_test.py:384-468, 890-933
  scatter_add_te               torch restatement of tenex/kernels/scatter_add.py:33-119
                               (the reference's own CPU algorithm, used as the
                               timed CPU baseline on machines without the reference)

The C part (te_oracle.c) is built by oracle/Makefile into oracle/_build/.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(HERE, "_build", "libte_oracle.so")
_lib = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")
_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")


def build() -> str:
    """Compiles te_oracle.c (make -C oracle)."""
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return _SO


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_SO) or os.path.getmtime(_SO) < os.path.getmtime(
                os.path.join(HERE, "te_oracle.c")):
            build()
        L = ctypes.CDLL(_SO)
        L.oracle_fsbwl.argtypes = [_f32p, ctypes.c_int, ctypes.c_int, ctypes.c_float, _i32p, _i32p]
        L.oracle_fsbwl.restype = None
        L.oracle_std_ddof1.argtypes = [_f32p, ctypes.c_int, _f32p]
        L.oracle_std_ddof1.restype = ctypes.c_float
        L.oracle_remap.argtypes = [_i32p, ctypes.c_int, ctypes.c_int64, _i32p]
        L.oracle_remap.restype = ctypes.c_int
        L.oracle_coarsen.argtypes = [_i32p, ctypes.c_int, ctypes.c_int64, _i32p, ctypes.c_int]
        L.oracle_coarsen.restype = ctypes.c_int
        L.oracle_counts.argtypes = [_i32p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int64,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _i64p]
        L.oracle_counts.restype = None
        L.oracle_te_pairfree.argtypes = [_i32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int64,
                                         ctypes.c_int64, _i32p, ctypes.c_int64, ctypes.c_int64,
                                         _f64p, ctypes.c_int]
        L.oracle_te_pairfree.restype = None
        L.oracle_te_pairs.argtypes = [_i32p, ctypes.c_int64, ctypes.c_int, ctypes.c_int64,
                                      ctypes.c_int64, _i32p, _i64p, ctypes.c_int64, _f64p,
                                      ctypes.c_int]
        L.oracle_te_pairs.restype = None
        _lib = L
    return _lib


def _flat_bins(bins) -> tuple[np.ndarray, int, int]:
    """(n, T) or (n, T, K) int array -> contiguous int32 (n, T*K), row_len, K."""
    b = np.asarray(bins)
    if b.ndim == 2:
        b = b[:, :, None]
    n, T, K = b.shape
    # int32 C-contiguous input is used as it is (no per-call copy of large bins)
    return np.ascontiguousarray(b.reshape(n, T * K), dtype=np.int32), T * K, K


# ---------------------------------------------------------------- preprocess
def std_ddof1(row: np.ndarray) -> np.float32:
    r = np.ascontiguousarray(row, dtype=np.float32)
    return np.float32(lib().oracle_std_ddof1(r, r.shape[0], np.empty_like(r)))


def fsbwl(x: np.ndarray, kp: float = 0.5) -> tuple[np.ndarray, np.ndarray]:
    """FSBW-L bins (n, T) int32 clamped at 0, and n_bins (n,) int32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, T = x.shape
    bins = np.empty((n, T), np.int32)
    nb = np.empty(n, np.int32)
    lib().oracle_fsbwl(x, n, T, float(kp), bins, nb)
    np.maximum(bins, 0, out=bins)
    return bins, nb


def remap(bins: np.ndarray) -> tuple[np.ndarray, np.ndarray, int]:
    b = np.ascontiguousarray(bins, dtype=np.int32).copy()
    n = b.shape[0]
    row = int(np.prod(b.shape[1:]))
    npv = np.empty(n, np.int32)
    bmax = lib().oracle_remap(b, n, row, npv)
    return b, npv, int(bmax)


def coarsen(bins: np.ndarray, npv: np.ndarray, limit: int) -> tuple[np.ndarray, np.ndarray, int]:
    b = np.ascontiguousarray(bins, dtype=np.int32).copy()
    p = np.ascontiguousarray(npv, dtype=np.int32).copy()
    n = b.shape[0]
    row = int(np.prod(b.shape[1:]))
    bmax = lib().oracle_coarsen(b, n, row, p, int(limit))
    return b, p, int(bmax)


def smem_bin_limit(smem_optin: int, warps: int = 32) -> int:
    """Largest B with (B^3 + 2B^2 + B + warps)*4 <= smem_optin
    (tenex/kernels/adaptive_smem.py:701-726)."""
    B = max(2, int((smem_optin / 4) ** (1.0 / 3.0)))
    while B > 2 and (B ** 3 + 2 * B ** 2 + B + warps) * 4 > smem_optin:
        B -= 1
    return B


def binarize_thresholds(x: np.ndarray, method: str, q: float = 0.5) -> np.ndarray:
    """Per-row thresholds of the reference's numpy binarizers, restated from a
    sorted copy: median -> the middle value, or (a + b) / 2 of the two middle
    values with a + b in float32 (np.median's mean); quantile -> numpy's linear
    method, virtual index (T - 1) q in float64, lerp of the neighbours a, b with
    diff = b - a in float32 and gamma in float64: a + diff * gamma, or
    b - diff * (1 - gamma) when gamma >= 0.5, in float64. mean -> float32
    pairwise mean as np.mean; nonzero -> 0."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    n, T = x.shape
    if method == "nonzero":
        return np.zeros(n, np.float32)
    if method == "mean":
        return x.mean(axis=1)
    s = np.sort(x, axis=1)
    if method == "median":
        h = T // 2
        if T % 2:
            return s[:, h].copy()
        return ((s[:, h - 1] + s[:, h]).astype(np.float64) / 2).astype(np.float32)
    vi = (T - 1) * float(q)
    if vi >= T - 1:
        return s[:, T - 1].astype(np.float64)
    lo = int(np.floor(vi))
    g = vi - lo
    a, b = s[:, lo], s[:, lo + 1]
    diff = (b - a).astype(np.float64)
    if g >= 0.5:
        return b.astype(np.float64) - diff * (1.0 - g)
    return a.astype(np.float64) + diff * g


def binarize(x: np.ndarray, method: str, q: float = 0.5) -> np.ndarray:
    """uint8 1[x > thr] per row (the comparison in the threshold's precision)."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    thr = binarize_thresholds(x, method, 0.5 if method == "median" else q)
    return (x > thr[:, None]).astype(np.uint8)


# ---------------------------------------------------------------- counts / TE
def counts(bins, tau: int, tgt: int, src: int, npv) -> np.ndarray:
    """int64 (bt, bt, bs) joint counts c3[xt1, xt, yt] of one ordered pair."""
    b, row, K = _flat_bins(bins)
    npv = np.asarray(npv, np.int32)
    bt, bs = int(npv[tgt]), int(npv[src])
    out = np.empty(bt * bt * bs, np.int64)
    lib().oracle_counts(b, row, row, tau * K, int(tgt), int(src), bt, bs, out)
    return out.reshape(bt, bt, bs)


def te_pairfree(bins, npv, tau: int = 1, pair_offset: int = 0, n_pairs: int | None = None,
                threads: int = 0) -> np.ndarray:
    """float64 TE for pair-free ids [pair_offset, pair_offset + n_pairs)."""
    b, row, K = _flat_bins(bins)
    n = b.shape[0]
    total = n * (n - 1)
    if n_pairs is None:
        n_pairs = total - pair_offset
    out = np.empty(max(n_pairs, 0), np.float64)
    if n_pairs > 0:
        lib().oracle_te_pairfree(b, row, n, row, tau * K, np.asarray(npv, np.int32),
                                 int(pair_offset), int(n_pairs), out, int(threads))
    return out


def te_pairs(bins, npv, pairs: np.ndarray, tau: int = 1, threads: int = 0) -> np.ndarray:
    """float64 TE for explicit pairs (P, 2) = [target, source]."""
    b, row, K = _flat_bins(bins)
    n = b.shape[0]
    pr = np.ascontiguousarray(pairs, dtype=np.int64)
    out = np.empty(pr.shape[0], np.float64)
    if pr.shape[0] > 0:
        lib().oracle_te_pairs(b, row, n, row, tau * K, np.asarray(npv, np.int32), pr,
                              pr.shape[0], out, int(threads))
    return out


def pairfree_to_matrix(ent: np.ndarray, n: int) -> np.ndarray:
    """matrix[i, j] = TE(i -> j) from pair-free order (tgt-major)."""
    m = np.zeros((n, n), dtype=ent.dtype)
    e2 = ent.reshape(n, n - 1)
    for t in range(n):
        m[t, :t] = e2[t, :t]
        m[t, t + 1:] = e2[t, t:]
    return m.T.copy()


def te_matrix(bins, npv, tau: int = 1, threads: int = 0) -> np.ndarray:
    n = np.asarray(bins).shape[0]
    return pairfree_to_matrix(te_pairfree(bins, npv, tau, threads=threads), n)


# ---------------------------------------------------------------- surrogate
def block_shuffle(bins: np.ndarray, perm: np.ndarray, block_length: int) -> np.ndarray:
    """Shuffles every gene's time axis by its block permutation perm[g, :]."""
    b = np.asarray(bins)
    if b.ndim == 2:
        b = b[:, :, None]
    n, T, K = b.shape
    nb = perm.shape[1]
    head = nb * block_length
    out = b.copy()
    blocks = b[:, :head].reshape(n, nb, block_length, K)
    out[:, :head] = np.take_along_axis(blocks, perm[:, :, None, None].astype(np.int64),
                                       axis=1).reshape(n, head, K)
    return out


def surrogate_stats(bins, npv, perms: np.ndarray, block_length: int, observed: np.ndarray,
                    tau: int = 1, threads: int = 0):
    """sum, sum_sq (float64) and count_ge (int32) over surrogates k of
    TE_k = TE(block_shuffle(bins, perms[k])), accumulated as the reference's
    loop path does (float32 TE widened to float64; te_k >= observed over the
    whole matrix, diagonal included)."""
    b = np.asarray(bins)
    n = b.shape[0]
    s = np.zeros((n, n), np.float64)
    ss = np.zeros((n, n), np.float64)
    c = np.zeros((n, n), np.int32)
    obs = np.asarray(observed, np.float32)
    for k in range(perms.shape[0]):
        sh = block_shuffle(b, perms[k], block_length)
        tk = te_matrix(sh, npv, tau, threads).astype(np.float32)
        s += tk
        ss += tk.astype(np.float64) ** 2
        c += (tk >= obs).astype(np.int32)
    return s, ss, c


# ---------------------------------------------------------------- CPU baseline
def scatter_add_te(bins, pairs: np.ndarray, B: int, tau: int = 1, batch: int = 2048):
    """The reference CPU algorithm (scatter_add histogram, float32 marginals and
    log2), restated with torch ops; returns float32 TE per pair."""
    import torch
    b = torch.as_tensor(np.asarray(bins))
    if b.dim() == 2:
        b = b[:, :, None]
    b = b.to(torch.int32)
    n, T, K = b.shape
    L = T - tau
    N = L * K
    B2, B3 = B * B, B * B * B
    pr = torch.as_tensor(np.asarray(pairs, np.int64))
    out = []
    for beg in range(0, pr.shape[0], batch):
        tg = pr[beg:beg + batch, 0]
        sg = pr[beg:beg + batch, 1]
        nb = tg.shape[0]
        target = b[tg]
        idx = target[:, tau:, :].to(torch.int64) * B2 + target[:, :-tau, :].to(torch.int64) * B
        idx += b[sg][:, :-tau, :].to(torch.int64)
        idx += (torch.arange(nb, dtype=torch.int64) * B3).view(-1, 1, 1)
        cnt = torch.zeros(nb * B3, dtype=torch.int32)
        cnt.scatter_add_(0, idx.reshape(-1), torch.ones(nb * N, dtype=torch.int32))
        c3 = cnt.view(nb, B, B, B).float()
        c2a = c3.sum(dim=3)
        c2b = c3.sum(dim=1)
        c1 = c3.sum(dim=(1, 3))
        num = c3 * c1[:, None, :, None]
        den = (c2a[:, :, :, None] * c2b[:, None, :, :]).clamp_(min=1)
        r = (num / den).log2_().mul_(c3).nan_to_num_(0.0)
        out.append(r.sum(dim=(1, 2, 3)) / N)
    return torch.cat(out).numpy() if out else np.zeros(0, np.float32)
