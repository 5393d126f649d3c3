"""Device-side data layout and launch wrappers shared by the TE kernel classes.

Bins live in HBM as "padded rows": a uint8 tensor (n, ld) with ld a multiple of
64 bytes, so every row starts on a 64-byte boundary and the histogram kernel can
stream sources with 16-byte vector loads. A reference tensor bin_arrs (n, T, K)
is stored as row[t*K + k] (row_len = T*K) and TE uses lag = tau*K.
"""
from __future__ import annotations

import ctypes
import os
import threading
from dataclasses import dataclass

import numpy as np
import torch

from tenex_b200 import native

ROW_ALIGN = 64


@dataclass
class DeviceBins:
    data: torch.Tensor   # (n, ld) uint8, CUDA (uint16 "wide" bins: genes with > 256 bins)
    n: int
    T: int
    K: int

    @property
    def row_len(self) -> int:
        return self.T * self.K

    @property
    def ld(self) -> int:
        """Row stride in elements (bytes for the uint8 layout)."""
        return int(self.data.shape[1])

    @property
    def wide(self) -> bool:
        """uint16 bins: some gene has more than 256 distinct values. Only the
        coarsening step reads them; it writes the uint8 layout the TE kernels use."""
        return self.data.dtype != torch.uint8

    def ptr(self) -> int:
        """Device address of the uint8 rows the TE kernels read."""
        if self.wide:
            raise ValueError("these bins hold genes with more than 256 distinct values (uint16); "
                             "the TE kernels read uint8 bins: coarsen them first "
                             "(AdaptiveSMEMKernel.prepare / preprocess.coarsen_bins)")
        return self.data.data_ptr()

    def unpadded(self) -> torch.Tensor:
        """(n, T, K) view-free copy of the bins (uint8)."""
        return self.data[:, :self.row_len].reshape(self.n, self.T, self.K).contiguous()


_copy_pool = None
_copy_workers = max(1, min(8, os.cpu_count() or 1))
_copy_pool_lock = threading.Lock()
_STAGE_BYTES = 32 << 20        # one staging chunk of the host -> device copy
_DIRECT_BYTES = 16 << 20       # smaller arrays take the plain pageable copy (to device)
_DIRECT_HOST_BYTES = 4 << 20   # and below this, the plain copy back


def _pool():
    global _copy_pool
    with _copy_pool_lock:
        if _copy_pool is None:
            from concurrent.futures import ThreadPoolExecutor
            _copy_pool = ThreadPoolExecutor(max_workers=_copy_workers,
                                            thread_name_prefix="tenex-h2d")
        return _copy_pool


def all_finite(a: np.ndarray) -> bool:
    """np.isfinite(a).all() for a large C-contiguous array, checked in 4M-element
    slabs on the host copy threads (ufuncs run without the GIL)."""
    a = np.asarray(a)
    if a.size < (1 << 23) or not a.flags.c_contiguous:
        return bool(np.isfinite(a).all())
    flat = a.reshape(-1)
    step = 1 << 22
    return all(_pool().map(lambda c: bool(np.isfinite(flat[c:c + step]).all()),
                           range(0, flat.size, step)))


def to_device(a, device) -> torch.Tensor:
    """Device copy of a host array (numpy or CPU tensor), same shape and dtype.
    A large array goes through two page-locked staging chunks: host threads fill
    chunk i + 1 (numpy copies run without the GIL) while the DMA engine moves
    chunk i, which runs several times faster than one pageable copy (the driver
    stages a pageable copy through its own buffer with one host thread). A
    page-locked tensor is copied directly. The source is no longer read once
    this returns (except a page-locked source, read by the DMA in stream order);
    the device copy is ordered on the current stream."""
    if isinstance(a, torch.Tensor):
        if a.device.type == "cuda" or (torch.cuda.is_available() and a.is_pinned()):
            return a.to(device)             # already DMA-able: one direct copy
        a = a.numpy()
    a = np.ascontiguousarray(a)
    device = torch.device(device)
    if device.type != "cuda" or a.nbytes < _DIRECT_BYTES or a.dtype == object:
        return torch.as_tensor(a).to(device)
    flat = a.reshape(-1)
    proto = torch.from_numpy(flat[:1].copy())
    out = torch.empty(flat.size, dtype=proto.dtype, device=device)
    per = max(1, _STAGE_BYTES // a.itemsize)
    bufs = [torch.empty(per, dtype=proto.dtype, pin_memory=True) for _ in range(2)]
    done = [None, None]
    pool = _pool()
    workers = _copy_workers
    with torch.cuda.device(device):
        stream = torch.cuda.current_stream()
        for i, off in enumerate(range(0, flat.size, per)):
            k = min(per, flat.size - off)
            j = i & 1
            if done[j] is not None:
                done[j].synchronize()        # the DMA that last read this chunk is over
            dst = bufs[j].numpy()
            step = -(-k // workers)
            cuts = [(c, min(c + step, k)) for c in range(0, k, step)]
            list(pool.map(lambda r: np.copyto(dst[r[0]:r[1]], flat[off + r[0]:off + r[1]]),
                          cuts))
            out[off:off + k].copy_(bufs[j][:k], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
            done[j] = ev
    return out.view(a.shape)


def to_host(t: torch.Tensor) -> np.ndarray:
    """numpy copy of a device tensor. A large tensor comes back through two
    page-locked staging chunks: the DMA engine fills chunk i + 1 while host
    threads copy chunk i out into an ordinary numpy array. One pageable copy
    runs at a few GB/s (the driver's own staging with one host thread, and the
    destination's pages first touched inside the copy); the staging chunks come
    from torch's caching host allocator and are released before this returns,
    so no page-locked memory outlives the call."""
    if t.device.type != "cuda":
        return t.numpy()
    t = t.contiguous()
    nbytes = t.numel() * t.element_size()
    if nbytes < _DIRECT_HOST_BYTES:
        return t.cpu().numpy()
    flat = t.view(-1)
    numel = flat.numel()
    out = np.empty(numel, dtype=torch.empty(0, dtype=t.dtype).numpy().dtype)
    per = max(1, _STAGE_BYTES // t.element_size())
    bufs = [torch.empty(per, dtype=t.dtype, pin_memory=True) for _ in range(2)]
    offs = list(range(0, numel, per))
    done = [None, None]
    pool = _pool()
    with torch.cuda.device(t.device):
        stream = torch.cuda.current_stream()

        def issue(i):
            off = offs[i]
            k = min(per, numel - off)
            bufs[i & 1][:k].copy_(flat[off:off + k], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
            done[i & 1] = ev

        issue(0)
        for i, off in enumerate(offs):
            if i + 1 < len(offs):
                issue(i + 1)       # its buffer's previous chunk was copied out last pass
            done[i & 1].synchronize()
            k = min(per, numel - off)
            src = bufs[i & 1].numpy()
            step = -(-k // _copy_workers)
            list(pool.map(lambda c: np.copyto(out[off + c:off + min(c + step, k)],
                                              src[c:min(c + step, k)]), range(0, k, step)))
    return out.reshape(tuple(t.shape))


def padded_ld(row_len: int) -> int:
    return (row_len + ROW_ALIGN - 1) // ROW_ALIGN * ROW_ALIGN


def empty_bins(n: int, T: int, K: int, device, wide: bool = False) -> DeviceBins:
    data = torch.zeros((n, padded_ld(T * K)), dtype=torch.uint16 if wide else torch.uint8,
                       device=device)
    return DeviceBins(data, n, T, K)


def pack_bins(bin_arrs, device, b_max: int | None = None) -> DeviceBins:
    """Copies (n, T) / (n, T, K) integer bins into the padded uint8 layout.

    Bin values must fit uint8 (the shared-memory kernels handle b <= 255): larger
    values raise ValueError (dense-remap such bins with preprocess.remap_bins,
    which keeps them as uint16 until coarsened).
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
    src = t.reshape(n, T * K)
    src = to_device(src, device) if src.device.type == "cpu" else src.to(device=device)
    if src.dtype != torch.uint8:
        src = src.to(torch.int32)
        if src.numel() and int(src.max()) > 255:
            raise ValueError("bin values above 255 do not fit the uint8 bin layout; remap them "
                             "with tenex_b200.preprocess.remap_bins and coarsen them first")
        src = src.clamp_(0, 255).to(torch.uint8)
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
        native.call("tenex_te_pairfree_counts", db.ptr(), db.ld, npv.data_ptr(),
                    int(b_max), n, db.row_len, lag, int(pair_offset), int(n_pairs),
                    out.data_ptr(), counts.data_ptr(), int(counts_stride), ws.data_ptr(),
                    ws.numel(), _cfg(cfg), s)
    else:
        native.call("tenex_te_pairfree", db.ptr(), db.ld, npv.data_ptr(), int(b_max),
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
    native.call("tenex_surrogate_accumulate", db.ptr(), db.ld,
                n_per_var.data_ptr(), int(b_max), n, db.row_len, tau * db.K, int(pair_offset),
                int(n_pairs), observed.data_ptr(), ssum.data_ptr(), ssq.data_ptr(),
                cnt.data_ptr(), ws.data_ptr(), ws.numel(), _cfg(cfg), native.stream_ptr())


def block_shuffle(db: DeviceBins, perm: torch.Tensor, block_length: int,
                  out: DeviceBins | None = None) -> DeviceBins:
    """Block-shuffles every gene's time axis by perm (n, n_blocks) int32."""
    if out is None:
        out = empty_bins(db.n, db.T, db.K, db.data.device)
    perm = perm.to(dtype=torch.int32).contiguous()
    native.call("tenex_block_shuffle", db.ptr(), db.ld, db.n, db.T, db.K,
                perm.data_ptr(), int(perm.shape[1]), int(block_length), out.data.data_ptr(),
                out.ld, native.stream_ptr())
    return out


def block_shuffle_many(db: DeviceBins, perms: torch.Tensor, block_length: int,
                       out: DeviceBins) -> DeviceBins:
    """S block shuffles in one launch: perms (S, n, n_blocks) int32; shuffled
    copy s goes to rows [s*n, (s+1)*n) of out (S*n rows)."""
    S, n, nb = (int(v) for v in perms.shape)
    if n != db.n or out.n < S * n or out.ld != db.ld or out.row_len != db.row_len:
        raise ValueError("block_shuffle_many: out must hold S copies of the bins' layout")
    perms = perms.to(dtype=torch.int32).contiguous()
    native.call("tenex_block_shuffle_many", db.ptr(), db.ld, n, db.T, db.K,
                perms.data_ptr(), S, nb, int(block_length), out.data.data_ptr(), out.ld,
                n * out.ld, native.stream_ptr())
    return out
