"""GPU binarisation to {0, 1} (routes the compute to GEMM-B2).

Mirrors tenex/binarize.py (binarize :225-295, methods nonzero / mean / median /
quantile, default numpy backend :45-150): 1[x > thr_g] per variable. nonzero
and mean run in tenex_binarize (the mean with numpy's float32 pairwise
summation and float64 division). median and quantile run in
tenex_binarize_select: a per-row radix selection of the order statistics
np.median / np.quantile ("linear") read, with numpy's arithmetic on them
(np.median's (a + b) / 2 with a + b in float32; np.quantile's virtual index
(T - 1) q in float64, a + (b - a) gamma or b - (b - a)(1 - gamma) in float64,
compared exactly with the float32 data), and numpy's NaN rule: a row holding a
NaN has a NaN threshold, so all its bins are 0. No sort and no device memory
beyond the bins.
Returns the discretize() tuple with the bins in the padded uint8 device layout.
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
    if key in ("median", "quantile"):
        if key == "quantile" and not 0.0 <= float(q) <= 1.0:
            raise ValueError(f"quantile q must be in [0, 1] (got {q})")
        native.call("tenex_binarize_select", x.data_ptr(), T, n, T, 1 if key == "median" else 0,
                    float(q), db.data.data_ptr(), db.ld, npv.data_ptr(), native.stream_ptr())
    else:
        native.call("tenex_binarize", x.data_ptr(), T, n, T, 0 if key == "nonzero" else 1,
                    None, db.data.data_ptr(), db.ld, npv.data_ptr(), native.stream_ptr())
    b_max = int(npv.max().item())
    return db, npv.clone(), b_max, npv
