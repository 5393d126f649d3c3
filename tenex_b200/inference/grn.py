"""GRN edge container (reference: tenex/inference/grn.py:10-27) and the pair
helpers of tenex/inference/__init__.py:86-126."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch


@dataclass
class GRN:
    source: np.ndarray   # (n_edges,) names
    target: np.ndarray   # (n_edges,) names
    te: np.ndarray       # (n_edges,) float32 scores
    pairs: np.ndarray    # (n_edges, 2) (source_idx, target_idx)

    def __len__(self):
        return len(self.te)

    def to_sif(self) -> np.ndarray:
        return np.stack((self.source, self.te.astype(str), self.target), axis=1)

    def to_edge_list(self) -> list[tuple[str, str, float]]:
        return [(s, t, float(v)) for s, t, v in zip(self.source, self.target, self.te)]


def build_pairs(variable_names: np.ndarray, sources=None) -> np.ndarray:
    """Directed (source, target) index pairs, optionally source-filtered."""
    n = len(variable_names)
    if sources is not None:
        _, src_idx, _ = np.intersect1d(variable_names, sources, return_indices=True)
        src_rep = np.repeat(src_idx, n)
        tgt_rep = np.tile(np.arange(n), len(src_idx))
        mask = src_rep != tgt_rep
        return np.stack((src_rep[mask], tgt_rep[mask]), axis=1)
    idx = np.arange(n)
    src = np.repeat(idx, n - 1)
    base = np.tile(np.arange(n - 1), n)
    tgt = base + (base >= src).astype(np.int64)
    return np.stack((src, tgt), axis=1).astype(np.int32)


def make_grn(variable_names: np.ndarray, pairs: np.ndarray, te: np.ndarray) -> GRN:
    return GRN(source=variable_names[pairs[:, 0]], target=variable_names[pairs[:, 1]],
               te=te.astype(np.float32), pairs=pairs)


_SCAN_ROW = 4096


def cummin_1d(x: torch.Tensor) -> torch.Tensor:
    """Running minimum of a 1-D floating-point tensor, equal element for element
    to x.cummin(0).values (min is exact; a NaN propagates to every later
    element). A 1-D scan runs as a single row on the GPU; here the tensor is cut
    into rows of _SCAN_ROW scanned in parallel, and each row is then lowered by
    the running minimum of the rows before it (computed the same way)."""
    m = x.numel()
    if m <= _SCAN_ROW:
        return x.cummin(0).values
    rows = -(-m // _SCAN_ROW)
    pad = rows * _SCAN_ROW - m
    xp = torch.cat((x, x.new_full((pad,), float("inf")))) if pad else x
    s = xp.view(rows, _SCAN_ROW).cummin(1).values
    carry = cummin_1d(s[:, -1].contiguous())
    s[1:] = torch.minimum(s[1:], carry[:-1, None])
    return s.reshape(-1)[:m]


def bh_fdr_gpu(pval: torch.Tensor, alpha: float) -> torch.Tensor:
    """Benjamini-Hochberg adjusted p-values (sort, p*m/rank, reverse cummin)."""
    m = pval.shape[0]
    if m == 0:
        return pval
    sorted_pval, sort_idx = pval.sort()
    rank = torch.arange(1, m + 1, device=pval.device, dtype=pval.dtype)
    adjusted = (sorted_pval * m / rank).clamp(max=1.0)
    adjusted = cummin_1d(adjusted.flip(0)).flip(0)
    result = torch.empty_like(adjusted)
    result[sort_idx] = adjusted
    return result
