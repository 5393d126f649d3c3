"""GPU binarisation to {0, 1} (routes the compute to GEMM-B2).

Mirrors tenex/binarize.py (binarize :225-295, methods nonzero / mean / median /
quantile, default numpy backend :45-150): 1[x > thr_g] per variable. nonzero
and mean run entirely in the binarize kernel (the mean with numpy's float32
pairwise summation). median and quantile thresholds come from rows sorted on
the device in blocks of rows (the sort's memory bounded like the reference's
chunked quantile, :97-115) with numpy's arithmetic: np.median's
(a + b) / 2 with a + b in float32, and np.quantile's "linear" method (virtual
index (T - 1) q in float64, a + (b - a) gamma or b - (b - a)(1 - gamma) in
float64). numpy compares the float32 data with that float64 threshold; the
kernel compares in float32 against the threshold rounded toward -inf, which
selects the same values (x > t64 exactly when x > rd32(t64) for float32 x).
Returns the discretize() tuple with the bins in the padded uint8 device layout.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from tenex_b200 import native
from tenex_b200.kernels import device as D

_METHODS = ("nonzero", "mean", "median", "quantile")
_SORT_BYTES = 1 << 30       # device memory one block of row sorts may take


def available_binarizers() -> list[str]:
    return list(_METHODS)


def sorted_thresholds(x: torch.Tensor, median: bool, q: float) -> torch.Tensor:
    """float32 per-row thresholds (see the module comment) from device sorts of
    blocks of rows, each block's sort within _SORT_BYTES (values + int64 indices
    plus the block: ~16 bytes per element)."""
    n, T = (int(s) for s in x.shape)
    rows = max(1, min(n, _SORT_BYTES // max(1, 16 * T)))
    thr = torch.empty(n, dtype=torch.float32, device=x.device)
    vi = (T - 1) * q
    lo = int(math.floor(vi))
    g = vi - lo
    for r0 in range(0, n, rows):
        s = torch.sort(x[r0:r0 + rows], dim=1).values
        if median:
            h = T // 2
            t = s[:, h] if T % 2 else ((s[:, h - 1] + s[:, h]).double() / 2).float()
        else:
            if vi >= T - 1:
                t64 = s[:, T - 1].double()
            else:
                a, b = s[:, lo], s[:, lo + 1]
                diff = (b - a).double()
                t64 = (b.double() - diff * (1.0 - g)) if g >= 0.5 else (a.double() + diff * g)
            t = t64.float()
            t = torch.where(t.double() > t64, torch.nextafter(t, torch.full_like(t, -math.inf)),
                            t)
        thr[r0:r0 + rows] = t
    return thr


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
        if key == "quantile" and not 0.0 <= float(q) <= 1.0:
            raise ValueError(f"quantile q must be in [0, 1] (got {q})")
        thr = sorted_thresholds(x, key == "median", float(q))
        mode = 2
    else:
        mode = 0 if key == "nonzero" else 1
    native.call("tenex_binarize", x.data_ptr(), T, n, T, mode,
                thr.data_ptr() if thr is not None else None, db.data.data_ptr(), db.ld,
                npv.data_ptr(), native.stream_ptr())
    b_max = int(npv.max().item())
    return db, npv.clone(), b_max, npv
