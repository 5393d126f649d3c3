"""Pair-list TE (source-filter path): explicit [target, source] pairs.

Replaces the reference's pair-based launch (tenex/kernels/full_smem.py:470-567,
te_smem_launch in tenex/csrc/full_smem.cu:319-347). Pairs are stably sorted by
target (the reference sorts them the same way, tenex/transferentropy.py:494-496)
and cut into runs of one target of at most `run` pairs; each run is one work
item of the persistent kernel, so a target's joint states are staged once per
run. Results are returned in the caller's pair order.
"""
from __future__ import annotations

import numpy as np
import torch

from tenex_b200 import native
from tenex_b200.kernels import device as D


def item_table(tgt_sorted: np.ndarray, run: int = 128) -> np.ndarray:
    """Start offsets of runs of equal targets, each at most `run` long (+ end)."""
    tgt_sorted = np.asarray(tgt_sorted)
    P = tgt_sorted.shape[0]
    if P == 0:
        return np.zeros(1, np.int64)
    change = np.flatnonzero(np.diff(tgt_sorted)) + 1
    starts = np.concatenate([[0], change]).astype(np.int64)
    lens = np.diff(np.concatenate([starts, [P]]))
    nchunk = (lens + run - 1) // run
    first = np.cumsum(nchunk) - nchunk                 # index of each segment's first item
    k = np.arange(int(nchunk.sum()), dtype=np.int64) - np.repeat(first, nchunk)
    items = np.repeat(starts, nchunk) + run * k
    return np.concatenate([items, [P]]).astype(np.int64)


def te_pair_list(db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int, pairs: np.ndarray,
                 cfg=None, run: int = 128, check_data: bool = True) -> torch.Tensor:
    """float32 TE per pair (device tensor), pairs (P, 2) int = [target, source]."""
    pairs = np.asarray(pairs, dtype=np.int64).reshape(-1, 2)
    P = pairs.shape[0]
    dev = db.data.device
    out = torch.empty(P, dtype=torch.float32, device=dev)
    if P == 0:
        return out
    order = np.argsort(pairs[:, 0], kind="stable")
    sp = np.ascontiguousarray(pairs[order])
    items = item_table(sp[:, 0], run)
    pairs_d = torch.from_numpy(sp).to(dev)
    items_d = torch.from_numpy(items).to(dev)
    npv = npv.to(device=dev, dtype=torch.int32).contiguous()
    ws = D.workspace(dev, db.n, db.row_len, b_max)
    s = native.stream_ptr()
    tmp = torch.empty(P, dtype=torch.float32, device=dev)
    native.call("tenex_te_pairs", db.ptr(), db.ld, npv.data_ptr(), int(b_max), db.n,
                db.row_len, tau * db.K, pairs_d.data_ptr(), P, items_d.data_ptr(),
                items.shape[0] - 1, tmp.data_ptr(), ws.data_ptr(), ws.numel(), D._cfg(cfg), s)
    if check_data:
        native.call("tenex_workspace_status", ws.data_ptr(), s)
    out[torch.from_numpy(order).to(dev)] = tmp
    return out
