"""GPU binarisation to {0, 1} (routes the compute to GEMM-B2).

Mirrors tenex/binarize.py (binarize :225-295, methods nonzero / mean / median /
quantile): 1[x > thr_g] per variable. nonzero and mean run entirely in the
binarize kernel (the mean with numpy's float32 pairwise summation); median and
quantile take their per-variable thresholds from torch.quantile on the device
and then use the same kernel. Returns the discretize() tuple with the bins in
the padded uint8 device layout.
"""
from __future__ import annotations

import numpy as np
import torch

from tenex_b200 import native
from tenex_b200.kernels import device as D

_METHODS = ("nonzero", "mean", "median", "quantile")


def available_binarizers() -> list[str]:
    return list(_METHODS)


def binarize(arr, method: str = "nonzero", device=None, q: float = 0.5, **_unused):
    key = method.lower()
    if key not in _METHODS:
        raise ValueError(f"unknown binarization '{method}'. available: {available_binarizers()}")
    dev = torch.device(device) if device is not None else torch.device("cuda", 0)
    x = torch.as_tensor(np.ascontiguousarray(arr, dtype=np.float32)) if not isinstance(
        arr, torch.Tensor) else arr.to(torch.float32)
    x = x.to(dev).contiguous()
    n, T = (int(s) for s in x.shape)
    db = D.empty_bins(n, T, 1, dev)
    npv = torch.empty(n, dtype=torch.int32, device=dev)
    thr = None
    if key in ("median", "quantile"):
        qq = 0.5 if key == "median" else float(q)
        if not 0.0 <= qq <= 1.0:
            raise ValueError(f"quantile q must be in [0, 1] (got {q})")
        thr = torch.quantile(x, qq, dim=1).contiguous()
        mode = 2
    else:
        mode = 0 if key == "nonzero" else 1
    native.call("tenex_binarize", x.data_ptr(), T, n, T, mode,
                thr.data_ptr() if thr is not None else None, db.data.data_ptr(), db.ld,
                npv.data_ptr(), native.stream_ptr())
    b_max = int(npv.max().item())
    return db, npv.clone(), b_max, npv
