"""Oracle (test infrastructure only): numpy restatement of the FDR inference
method of the reference, used by the tests as the checker of
tenex_b200.inference.fdr, never by the product.

  fdr_threshold   tenex/inference/__init__.py:129-139 (fdr_threshold_gpu):
                  z = (te - mean) / std (ddof=1), p = erfc(z / sqrt 2) / 2,
                  Benjamini-Hochberg (:115-126), keep adjusted p < fdr
  top_links       tenex/inference/__init__.py:157-162 (links > 0)
  dpi_trim        tenex/inference/fdr.py:61-133 (_trim): row batches, mediators =
                  rows with a positive sum, indirect = max(0, max_k min(A[i,k], A[k,j]))
                  over the batch's active mediators, keep A[i,j] >= indirect + thr,
                  batches without an active mediator kept whole

Pinned against tests/golden/fdr_trim.npz (the reference's own functions run on
CPU tensors).
"""
from __future__ import annotations

import math

import numpy as np


def bh_adjust(p: np.ndarray) -> np.ndarray:
    """Benjamini-Hochberg adjusted p-values (float64)."""
    p = np.asarray(p, dtype=np.float64)
    m = p.size
    if m == 0:
        return p
    order = np.argsort(p, kind="stable")
    adj = p[order] * m / np.arange(1, m + 1)
    adj = np.minimum(adj, 1.0)
    adj = np.minimum.accumulate(adj[::-1])[::-1]
    out = np.empty_like(adj)
    out[order] = adj
    return out


def fdr_threshold(te: np.ndarray, pairs: np.ndarray, fdr: float):
    """Edges kept by the z-score / BH rule, in input order (float64 arithmetic)."""
    te = np.asarray(te, dtype=np.float64)
    std = te.std(ddof=1) if te.size > 1 else 0.0
    if std == 0 or not np.isfinite(std):
        return np.zeros(0, np.float32), pairs[:0], np.zeros(0)
    z = (te - te.mean()) / std
    p = 0.5 * np.array([math.erfc(v / math.sqrt(2.0)) for v in z])
    adj = bh_adjust(p)
    keep = adj < fdr
    return te[keep].astype(np.float32), pairs[keep], adj


def top_links(te: np.ndarray, pairs: np.ndarray, links: int):
    """The `links` largest TE values, descending."""
    k = min(links, te.size)
    idx = np.argsort(-np.asarray(te, dtype=np.float64), kind="stable")[:k]
    return np.asarray(te, np.float32)[idx], pairs[idx]


def dpi_trim(n: int, pairs: np.ndarray, te_values: np.ndarray, batch_size: int,
             trim_threshold: float):
    """(pairs, values) kept by the reference's trimming loop, row-major order."""
    arr = np.zeros((n, n), np.float32)
    arr[pairs[:, 0], pairs[:, 1]] = np.asarray(te_values, np.float32)
    mediator = arr.sum(axis=1, dtype=np.float64) > 0
    if not mediator.any():
        return pairs, np.asarray(te_values, np.float32)
    out_p, out_v = [], []
    med_idx = np.nonzero(mediator)[0]
    thr = np.float32(trim_threshold)
    for r0 in range(0, n, batch_size):
        batch = arr[r0:r0 + batch_size]
        if not (batch != 0).any():
            continue
        cols = np.unique(np.nonzero(batch)[1])
        active = cols[np.isin(cols, med_idx)]
        if active.size == 0:
            kept = batch
        else:
            indirect = np.zeros_like(batch)
            for k in active:
                np.maximum(indirect, np.minimum(batch[:, k:k + 1], arr[k][None, :]), out=indirect)
            if trim_threshold != 0.0:
                indirect = (indirect + thr).astype(np.float32)
            kept = np.where(batch >= indirect, batch, np.float32(0))
        rows, cc = np.nonzero(kept)
        out_p.append(np.stack((rows + r0, cc), axis=1))
        out_v.append(kept[rows, cc])
    if not out_p:
        return np.zeros((0, 2), np.int64), np.zeros(0, np.float32)
    return np.concatenate(out_p).astype(np.int64), np.concatenate(out_v).astype(np.float32)


def dpi_matrix(a: np.ndarray, mediator: np.ndarray | None = None,
               keep_all: np.ndarray | None = None, trim_threshold: float = 0.0,
               rows: np.ndarray | None = None) -> np.ndarray:
    """The trimmed matrix of one tenex_dpi_trim call, by its definition:
    out[i,j] = a[i,j] if keep_all[i] or a[i,j] >= max(0, max_{k mediator}
    min(a[i,k], a[k,j])) + thr, else 0 (float32 throughout; `rows` selects rows)."""
    a = np.asarray(a, np.float32)
    n = a.shape[0]
    med = np.ones(n, bool) if mediator is None else np.asarray(mediator, bool)
    keep = np.zeros(n, bool) if keep_all is None else np.asarray(keep_all, bool)
    rows = np.arange(n) if rows is None else np.asarray(rows)
    am = a[med]
    out = np.zeros((rows.size, n), np.float32)
    thr = np.float32(trim_threshold)
    for r, i in enumerate(rows):
        if am.shape[0]:
            ind = np.maximum(np.float32(0), np.minimum(a[i, med][:, None], am).max(axis=0))
        else:
            ind = np.zeros(n, np.float32)
        ind = (ind + thr).astype(np.float32)
        out[r] = a[i] if keep[i] else np.where(a[i] >= ind, a[i], np.float32(0))
    return out
