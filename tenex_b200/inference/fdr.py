"""FDR inference: z-score -> Benjamini-Hochberg -> optional DPI trimming.

Mirrors FDRMethod (tenex/inference/fdr.py:16-58) and the thresholding helpers
of tenex/inference/__init__.py:129-162 with the same arguments (fdr=0.01,
links=0, sources, is_trimming=True, trim_threshold=0.0, batch_size=512) and
return values (GRN, or (GRN, trimmed GRN) with trimming). Thresholding runs on
the device as the reference's GPU branch does (z-score with the unbiased std,
p = erfc(z / sqrt 2) / 2, BH, keep adjusted p < fdr; or the `links` largest);
the trimming step's (max, min) matrix product over the mediators is a CUDA
kernel, dense (tenex_dpi_trim) or over the nonzero entries
(tenex_dpi_trim_sparse), whichever does less work.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from tenex_b200 import _log, native
from tenex_b200.inference.grn import bh_fdr_gpu, build_pairs, make_grn
from tenex_b200.kernels import device as D


def fdr_threshold_gpu(te: torch.Tensor, pairs: torch.Tensor, fdr: float):
    """Edges whose BH-adjusted one-sided z-score p-value is below `fdr`
    (tenex/inference/__init__.py:129-139)."""
    std = te.std()
    if std == 0:
        return torch.empty(0, device=te.device), pairs[:0]
    z = (te - te.mean()) / std
    pval = 0.5 * torch.erfc(z / 1.4142135623730951)
    adj = bh_fdr_gpu(pval, 0.05)
    mask = adj < fdr
    return te[mask], pairs[mask]


class _LazyPairs:
    """(src, tgt) rows of the all-pairs list for pair ids, computed on indexing
    (src = id // (n-1), tgt = id % (n-1) skipping the diagonal)."""

    def __init__(self, n: int, device):
        self.n, self.device = n, device

    def __len__(self):
        return self.n * (self.n - 1)

    def __getitem__(self, idx):
        if isinstance(idx, torch.Tensor) and idx.dtype == torch.bool:
            idx = idx.nonzero(as_tuple=True)[0]
        elif isinstance(idx, slice):
            idx = torch.arange(len(self), device=self.device)[idx]
        idx = torch.as_tensor(idx, device=self.device, dtype=torch.long)
        src = idx // max(self.n - 1, 1)
        t = idx - src * (self.n - 1)
        return torch.stack((src, t + (t >= src).long()), dim=1)


def _offdiag(M: torch.Tensor):
    n = M.shape[0]
    te = M[~torch.eye(n, dtype=torch.bool, device=M.device)]
    return te, _LazyPairs(n, M.device)


def threshold_pairs_device(te: torch.Tensor, pairs, fdr: float = 0.01, links: int = 0):
    """Top-`links` or FDR thresholding (tenex/inference/__init__.py:155-170) on
    the device; returns device tensors (te_cut, pairs_cut)."""
    if links > 0:
        k = min(links, len(te))
        _, idx = te.topk(k)
        idx = idx[te[idx].argsort(descending=True)]
        return te[idx], pairs[idx]
    return fdr_threshold_gpu(te, pairs, fdr)


def threshold_pairs(te: torch.Tensor, pairs: torch.Tensor, fdr: float = 0.01, links: int = 0):
    """threshold_pairs_device with numpy results (te_cut, pairs_cut)."""
    te_c, p_c = threshold_pairs_device(te, pairs, fdr, links)
    return D.to_host(te_c), D.to_host(p_c)


def dpi_trim_matrix(arr: torch.Tensor, mediator: torch.Tensor | None = None,
                    keep_all: torch.Tensor | None = None, trim_threshold: float = 0.0,
                    out: torch.Tensor | None = None) -> torch.Tensor:
    """tenex_dpi_trim on a float32 (n, n) device matrix: entries that survive the
    DPI test (or whole rows flagged keep_all), zero elsewhere."""
    if arr.dim() != 2 or arr.shape[0] != arr.shape[1] or arr.dtype != torch.float32:
        raise ValueError("arr must be a square float32 matrix")
    if arr.device.type != "cuda":
        raise RuntimeError("DPI trimming runs on a CUDA device; got " + str(arr.device))
    arr = arr.contiguous()
    n = arr.shape[0]
    if out is None:
        out = torch.empty_like(arr)

    def _mask(m):
        if m is None:
            return None
        m = m.to(device=arr.device, dtype=torch.uint8).contiguous()
        if m.numel() != n:
            raise ValueError("mediator / keep_all must have n entries")
        return m
    med, keep = _mask(mediator), _mask(keep_all)
    native.call("tenex_dpi_trim", arr.data_ptr(), n, n,
                med.data_ptr() if med is not None else None,
                keep.data_ptr() if keep is not None else None,
                ctypes.c_float(trim_threshold), out.data_ptr(), out.stride(0), native.stream_ptr())
    return out


def dpi_trim_sparse(arr: torch.Tensor, mediator: torch.Tensor | None = None,
                    keep_all: torch.Tensor | None = None, trim_threshold: float = 0.0):
    """tenex_dpi_trim_sparse on the nonzero entries of a float32 (n, n) device
    matrix; returns (rows, cols, vals) of the surviving entries, row-major."""
    if arr.device.type != "cuda":
        raise RuntimeError("DPI trimming runs on a CUDA device; got " + str(arr.device))
    n = arr.shape[0]
    rows, cols = torch.nonzero(arr, as_tuple=True)
    if rows.numel() == 0:
        return rows, cols, arr[rows, cols]
    vals = arr[rows, cols].contiguous()
    row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=arr.device)
    row_ptr[1:] = torch.cumsum(torch.bincount(rows, minlength=n), 0)
    col32 = cols.to(torch.int32).contiguous()
    keep = torch.empty(rows.numel(), dtype=torch.uint8, device=arr.device)
    med = None if mediator is None else mediator.to(torch.uint8).contiguous()
    ka = None if keep_all is None else keep_all.to(torch.uint8).contiguous()
    native.call("tenex_dpi_trim_sparse", row_ptr.data_ptr(), col32.data_ptr(), vals.data_ptr(), n,
                med.data_ptr() if med is not None else None,
                ka.data_ptr() if ka is not None else None, ctypes.c_float(trim_threshold),
                keep.data_ptr(), native.stream_ptr())
    k = keep.bool()
    return rows[k], cols[k], vals[k]


def _sparse_pays(arr: torch.Tensor, mediator: torch.Tensor) -> bool:
    """The sparse form's updates (sum over mediators k of positive in-degree x
    positive out-degree) against 1.5 n^3 dense min/max instructions; an update
    (a gather and a shared atomicMax) costs ~10 dense instructions."""
    n = arr.shape[0]
    if n * 4 > native.device_info(arr.device.index).smem_optin:
        return False
    pos = arr > 0
    work = (pos.sum(0).double() * pos.sum(1).double() * mediator.double()).sum().item()
    return work * 10.0 < 1.5 * float(n) ** 3


def dpi_trim(n: int, variable_names, pairs: np.ndarray, te_values: np.ndarray,
             device: torch.device, batch_size: int = 512, trim_threshold: float = 0.0,
             method: str = "auto"):
    """Trimmed GRN of the kept edges (tenex/inference/fdr.py:61-133): mediators
    are rows with a positive sum; row batches of `batch_size` without an active
    mediator are kept whole; the rest keep A[i,j] >= indirect + trim_threshold.
    method: "dense" (tenex_dpi_trim), "sparse" (tenex_dpi_trim_sparse) or "auto"
    (sparse when its work is the smaller); both give the same edges."""
    if method not in ("auto", "dense", "sparse"):
        raise ValueError(f"method must be 'auto', 'dense' or 'sparse' (got {method!r})")
    arr = torch.zeros((n, n), dtype=torch.float32, device=device)
    if len(pairs):
        p = torch.as_tensor(pairs, device=device).long()
        arr[p[:, 0], p[:, 1]] = torch.as_tensor(te_values, device=device).float()
    mediator = arr.sum(dim=1) > 0
    if not bool(mediator.any()):
        host = [D.to_host(x) if isinstance(x, torch.Tensor) else np.asarray(x)
                for x in (pairs, te_values)]
        return make_grn(variable_names, host[0], host[1])
    # a batch is active when one of its nonzero columns is a mediator
    row_active = ((arr != 0) & mediator[None, :]).any(dim=1)
    nb = (n + batch_size - 1) // batch_size
    pad = nb * batch_size - n
    batch_active = torch.nn.functional.pad(row_active, (0, pad)).view(nb, batch_size).any(dim=1)
    keep_all = (~batch_active).repeat_interleave(batch_size)[:n]
    if method == "sparse" or (method == "auto" and _sparse_pays(arr, mediator)):
        rows, cols, vals = dpi_trim_sparse(arr, mediator, keep_all, trim_threshold)
    else:
        out = dpi_trim_matrix(arr, mediator, keep_all, trim_threshold)
        rows, cols = torch.nonzero(out, as_tuple=True)
        vals = out[rows, cols]
    if rows.numel() == 0:
        return make_grn(variable_names, np.empty((0, 2), dtype=np.int32),
                        np.empty(0, dtype=np.float32))
    kept = D.to_host(torch.stack((rows, cols), dim=1))
    return make_grn(variable_names, kept, D.to_host(vals))


class FDRMethod:
    """'fdr' inference method (tenex/inference/fdr.py:16-58)."""

    @property
    def name(self) -> str:
        return "fdr"

    def infer(self, te_matrix, variable_names, device, **kwargs):
        fdr = kwargs.get("fdr", 0.01)
        links = kwargs.get("links", 0)
        sources = kwargs.get("sources", None)
        is_trimming = kwargs.get("is_trimming", True)
        trim_threshold = kwargs.get("trim_threshold", 0.0)
        batch_size = kwargs.get("batch_size", 512)
        dpi_method = kwargs.get("dpi_method", "auto")
        device = torch.device(device)
        if device.type != "cuda":
            raise RuntimeError("the fdr method runs on a CUDA device in this package; got "
                               f"{device}")
        variable_names = np.asarray(variable_names)
        te_matrix = np.asarray(te_matrix, dtype=np.float32)
        M = D.to_device(te_matrix, device)
        if sources is None:
            # build_pairs' all-pairs order is the row-major off-diagonal order of
            # M[src, tgt]: select it on the device instead of materialising the
            # n(n-1) x 2 index array on the host
            te_t, pairs_t = _offdiag(M)
        else:
            pairs_np = build_pairs(variable_names, sources)
            pairs_t = torch.from_numpy(np.ascontiguousarray(pairs_np)).to(device, dtype=torch.long)
            te_t = M[pairs_t[:, 0], pairs_t[:, 1]]
        te_d, pairs_d = threshold_pairs_device(te_t, pairs_t, fdr=fdr, links=links)
        grn = make_grn(variable_names, D.to_host(pairs_d), D.to_host(te_d))
        _log.vprint(f"[TENEX] inference(fdr): {len(grn)} links after thresholding")
        if not is_trimming:
            return grn
        trimmed = dpi_trim(te_matrix.shape[0], variable_names, pairs_d, te_d, device,
                           batch_size=batch_size, trim_threshold=trim_threshold,
                           method=dpi_method)
        _log.vprint(f"[TENEX] inference(fdr): {len(trimmed)} links after trimming")
        return grn, trimmed
