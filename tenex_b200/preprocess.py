"""GPU preprocessing of the TE path: discretisation, dense remap, coarsening.

Mirrors tenex/preprocess.py of the reference:
  discretize()      :554-688  (FSBW-L; the numpy/FastTENET bins, bit-exact)
  remap_bins()      :401-459
  coarsen_bins()    :462-551
  compact_dtype()   :335-354  (the dtype the reference stores bins in; here the
                               device layout is uint8 padded rows, uint16 for
                               genes of more than 256 distinct bins until they are
                               coarsened, and this only decides the dtype handed
                               back to callers)
All work runs in libtenex_sm100.so kernels; bins stay on the device as
DeviceBins (uint8 or uint16, rows padded to 64 elements).
"""
from __future__ import annotations

import numpy as np
import torch

from tenex_b200 import native
from tenex_b200.kernels import device as D

SUPPORTED_METHODS = ("FSBW-L", "DEFAULT")


def compact_dtype(b_max: int) -> np.dtype:
    """int8 if b_max <= 127, int16 if <= 32767, else int32 (reference rule)."""
    if b_max <= 127:
        return np.dtype(np.int8)
    if b_max <= 32767:
        return np.dtype(np.int16)
    return np.dtype(np.int32)


def _device(device) -> torch.device:
    dev = torch.device(device) if device is not None else torch.device("cuda", 0)
    if dev.type != "cuda":
        raise RuntimeError("the TE preprocessing kernels run on CUDA devices only")
    return dev


def fsbwl_bins(x, kp: float = 0.5, device=None) -> tuple[torch.Tensor, torch.Tensor]:
    """FSBW-L bins (int32 (n, T), clamped at 0) and n_bins, bit-identical to
    bin_fsbw_l_numpy + clamp(min=0) of the reference."""
    dev = _device(device)
    xt = torch.as_tensor(np.ascontiguousarray(x, dtype=np.float32)) if not isinstance(
        x, torch.Tensor) else x.to(torch.float32)
    xt = (D.to_device(xt, dev) if xt.device.type == "cpu" else xt.to(dev)).contiguous()
    n, T = (int(s) for s in xt.shape)
    bins = torch.empty((n, T), dtype=torch.int32, device=dev)
    nb = torch.empty(n, dtype=torch.int32, device=dev)
    native.call("tenex_fsbwl_bins", xt.data_ptr(), T, n, T, float(kp), bins.data_ptr(), T,
                nb.data_ptr(), native.stream_ptr())
    return bins, nb


def remap_bins(raw, K: int = 1, device=None) -> tuple[D.DeviceBins, torch.Tensor, int]:
    """Dense per-gene relabelling of integer bins (n, T[, K]) into the padded
    device layout: uint8, or uint16 when a gene has more than 256 distinct
    values (coarsen_bins narrows those). Returns (DeviceBins, n_per_var int32,
    b_max)."""
    dev = _device(device)
    t = raw if isinstance(raw, torch.Tensor) else torch.as_tensor(np.asarray(raw))
    if t.dim() == 3:
        K = int(t.shape[2])
        t = t.reshape(t.shape[0], -1)
    if t.dtype.is_floating_point or t.dtype == torch.uint16:
        t = t.to(torch.int32)             # on the host: same conversion as before upload
    # integers go up in their own width (staged copy) and are widened on the device
    t = D.to_device(t, dev) if t.device.type == "cpu" else t.to(dev)
    if t.dtype == torch.uint8:
        in_bytes = 1
    else:
        t = t.to(torch.int32)
        in_bytes = 4
    t = t.contiguous()
    n, row = (int(s) for s in t.shape)
    if row % K:
        raise ValueError(f"row length {row} is not a multiple of K={K}")
    npv = torch.empty(n, dtype=torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    db = None
    for wide in (False, True):
        # uint8 rows; a gene with more than 256 distinct values keeps uint16 rows
        # (the reference's int16 bins, tenex/preprocess.py:335-354) until the
        # coarsening step narrows them
        db = D.empty_bins(n, row // K, K, dev, wide=wide)
        err.zero_()
        native.call("tenex_remap_dense", t.data_ptr(), in_bytes, row, n, row,
                    db.data.data_ptr(), 2 if wide else 1, db.ld, npv.data_ptr(), err.data_ptr(),
                    native.stream_ptr())
        # the error word and b_max come back in one copy (one wait on the stream)
        e, b_max = (int(v) for v in torch.stack((err[0], npv.max())).cpu())
        if e == 1:
            raise ValueError("a gene's raw bins span more than 8192 values; cannot remap")
        if e == 0:
            break
    return db, npv, b_max


def discretize(arr, method: str = "FSBW-L", kp: float = 0.5, device=None,
               use_numpy_bins: bool | None = True):
    """FSBW-L discretisation + dense remap on the GPU.

    Returns (bins: DeviceBins, n_bins: int32 tensor, b_max, n_per_var: int32
    tensor), the tuple of the reference's discretize() with the bins kept on the
    device. The GPU bins equal the reference's numpy (FastTENET-exact) bins for
    every value of use_numpy_bins; the reference's torch-on-CUDA std differs
    from numpy in the last float32 bit, which this build does not reproduce.
    """
    if method.upper() not in SUPPORTED_METHODS:
        raise ValueError(f"Unknown or unsupported binning method '{method}'. "
                         f"This build implements {list(SUPPORTED_METHODS)}")
    dev = _device(device)
    bins, nb = fsbwl_bins(arr, kp, dev)
    db, npv, b_max = remap_bins(bins, 1, dev)
    return db, nb, b_max, npv


def coarsen_bins(db: D.DeviceBins, n_per_var: torch.Tensor, smem_bin_limit: int):
    """Coarsening new = old * limit // n_per_var for genes above the limit, in
    place on uint8 bins; uint16 bins (genes with more than 256 distinct values)
    are coarsened into new uint8 bins. Returns (db, n_per_var, new b_max)."""
    npv = n_per_var.to(device=db.data.device, dtype=torch.int32).contiguous()
    if db.wide:
        out = D.empty_bins(db.n, db.T, db.K, db.data.device)
        native.call("tenex_coarsen_narrow", db.data.data_ptr(), db.ld, db.n, db.row_len,
                    npv.data_ptr(), int(smem_bin_limit), out.data.data_ptr(), out.ld,
                    native.stream_ptr())
        return out, npv, int(npv.max().item())
    native.call("tenex_coarsen", db.data.data_ptr(), db.ld, db.n, db.row_len, npv.data_ptr(),
                int(smem_bin_limit), native.stream_ptr())
    return db, npv, int(npv.max().item())
