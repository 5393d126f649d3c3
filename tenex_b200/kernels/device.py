"""Device-side data layout and launch wrappers shared by the TE kernel classes.

Bins live in HBM as "padded rows": a uint8 tensor (n, ld) with ld a multiple of
64 bytes, so every row starts on a 64-byte boundary and the histogram kernel can
stream sources with 16-byte vector loads. A reference tensor bin_arrs (n, T, K)
is stored as row[t*K + k] (row_len = T*K) and TE uses lag = tau*K.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from tenex_b200 import native

ROW_ALIGN = 64


@dataclass
class DeviceBins:
    data: torch.Tensor   # (n, ld) uint8, CUDA
    n: int
    T: int
    K: int

    @property
    def row_len(self) -> int:
        return self.T * self.K

    @property
    def ld(self) -> int:
        return int(self.data.shape[1])

    def unpadded(self) -> torch.Tensor:
        """(n, T, K) view-free copy of the bins (uint8)."""
        return self.data[:, :self.row_len].reshape(self.n, self.T, self.K).contiguous()


def to_host(t: torch.Tensor) -> np.ndarray:
    """numpy copy of a device tensor, made through page-locked memory from torch's
    caching host allocator: a copy into fresh pageable memory runs at a few GB/s
    (the destination's pages are first touched during the copy), a copy into
    reused page-locked memory near the link rate. The array keeps its block
    alive; once the array is released the block goes back to the allocator's
    cache and the next copy of that size reuses it."""
    if t.device.type != "cuda":
        return t.numpy()
    h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
    h.copy_(t)
    return h.numpy()


def padded_ld(row_len: int) -> int:
    return (row_len + ROW_ALIGN - 1) // ROW_ALIGN * ROW_ALIGN


def empty_bins(n: int, T: int, K: int, device) -> DeviceBins:
    data = torch.zeros((n, padded_ld(T * K)), dtype=torch.uint8, device=device)
    return DeviceBins(data, n, T, K)


def pack_bins(bin_arrs, device, b_max: int | None = None) -> DeviceBins:
    """Copies (n, T) / (n, T, K) integer bins into the padded uint8 layout.

    Bin values must fit uint8 (the shared-memory kernels handle b <= 255).
    """
    if isinstance(bin_arrs, DeviceBins):
        return bin_arrs
    t = torch.as_tensor(np.asarray(bin_arrs)) if not isinstance(bin_arrs, torch.Tensor) \
        else bin_arrs
    if t.dim() == 2:
        t = t.unsqueeze(-1)
    if t.dim() != 3:
        raise ValueError(f"bin_arrs must be (n, T) or (n, T, K); got shape {tuple(t.shape)}")
    n, T, K = (int(s) for s in t.shape)
    if b_max is not None and b_max > 255:
        raise ValueError(f"b_max={b_max} does not fit the uint8 bin layout")
    db = empty_bins(n, T, K, device)
    src = t.reshape(n, T * K).to(device=device)
    if src.dtype != torch.uint8:
        src = src.to(torch.int32).clamp_(0, 255).to(torch.uint8)
    db.data[:, :T * K].copy_(src)
    return db


def _ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else int(t.data_ptr())


def workspace(device, n: int, row_len: int, b_max: int) -> torch.Tensor:
    nb = int(native.lib().tenex_te_workspace_bytes(int(n), int(row_len), int(b_max)))
    return torch.empty(nb, dtype=torch.uint8, device=device)


def _cfg(cfg) -> ctypes.POINTER(native.TeConfig) | None:
    if cfg is None:
        return None
    if isinstance(cfg, dict):
        cfg = native.te_config(**cfg)
    return ctypes.byref(cfg)


def te_pairfree(db: DeviceBins, n_per_var: torch.Tensor, b_max: int, tau: int = 1,
                pair_offset: int = 0, n_pairs: int | None = None, out: torch.Tensor | None = None,
                matrix: bool = False, cfg=None, check_data: bool = True,
                counts: torch.Tensor | None = None, counts_stride: int = 0) -> torch.Tensor:
    """TE for pair-free ids [pair_offset, pair_offset + n_pairs) on the bins' device.

    matrix=False: returns float32 (n_pairs,) in pair-free order.
    matrix=True:  writes out[src, tgt] = TE(src -> tgt) into an (n, n) float32
                  tensor (allocated zeroed when `out` is None; diagonal untouched).
    """
    dev = db.data.device
    n = db.n
    total = n * (n - 1)
    if n_pairs is None:
        n_pairs = total - pair_offset
    npv = n_per_var.to(device=dev, dtype=torch.int32).contiguous()
    if out is None:
        out = (torch.zeros((n, n), dtype=torch.float32, device=dev) if matrix
               else torch.empty(max(n_pairs, 0), dtype=torch.float32, device=dev))
    if n_pairs == 0:
        return out                   # nothing to compute (the C entry point is a no-op too)
    ws = workspace(dev, n, db.row_len, b_max)
    s = native.stream_ptr()
    lag = tau * db.K
    if counts is not None:
        native.call("tenex_te_pairfree_counts", db.data.data_ptr(), db.ld, npv.data_ptr(),
                    int(b_max), n, db.row_len, lag, int(pair_offset), int(n_pairs),
                    out.data_ptr(), counts.data_ptr(), int(counts_stride), ws.data_ptr(),
                    ws.numel(), _cfg(cfg), s)
    else:
        native.call("tenex_te_pairfree", db.data.data_ptr(), db.ld, npv.data_ptr(), int(b_max),
                    n, db.row_len, lag, int(pair_offset), int(n_pairs), out.data_ptr(),
                    native.OUT_MATRIX if matrix else native.OUT_PAIRFREE,
                    n if matrix else 0, ws.data_ptr(), ws.numel(), _cfg(cfg), s)
    if check_data:
        native.call("tenex_workspace_status", ws.data_ptr(), s)
    return out


def surrogate_accumulate(db: DeviceBins, n_per_var: torch.Tensor, b_max: int, tau: int,
                         observed: torch.Tensor, ssum: torch.Tensor, ssq: torch.Tensor,
                         cnt: torch.Tensor, pair_offset: int = 0, n_pairs: int | None = None,
                         cfg=None, ws: torch.Tensor | None = None) -> None:
    """Adds one surrogate's TE (from already-shuffled bins) into the (n, n)
    accumulators: sum/sumsq float64, count_ge int32 (slot [src, tgt])."""
    n = db.n
    if n_pairs is None:
        n_pairs = n * (n - 1) - pair_offset
    if ws is None:
        ws = workspace(db.data.device, n, db.row_len, b_max)
    native.call("tenex_surrogate_accumulate", db.data.data_ptr(), db.ld,
                n_per_var.data_ptr(), int(b_max), n, db.row_len, tau * db.K, int(pair_offset),
                int(n_pairs), observed.data_ptr(), ssum.data_ptr(), ssq.data_ptr(),
                cnt.data_ptr(), ws.data_ptr(), ws.numel(), _cfg(cfg), native.stream_ptr())


def block_shuffle(db: DeviceBins, perm: torch.Tensor, block_length: int,
                  out: DeviceBins | None = None) -> DeviceBins:
    """Block-shuffles every gene's time axis by perm (n, n_blocks) int32."""
    if out is None:
        out = empty_bins(db.n, db.T, db.K, db.data.device)
    perm = perm.to(dtype=torch.int32).contiguous()
    native.call("tenex_block_shuffle", db.data.data_ptr(), db.ld, db.n, db.T, db.K,
                perm.data_ptr(), int(perm.shape[1]), int(block_length), out.data.data_ptr(),
                out.ld, native.stream_ptr())
    return out
