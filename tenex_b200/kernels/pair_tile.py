"""Shared implementation of the Full-SMEM and Adaptive-SMEM kernel classes.

Both reference backends (tenex/kernels/full_smem.py, tenex/kernels/adaptive_smem.py)
map to one persistent sm_100a kernel (te_pair_tile_kernel): per-gene bin
counts are read on the device, so a uniform-b run (Full-SMEM) and an uneven
run (Adaptive-SMEM) are the same launch. The classes keep the reference's
names, supports() predicates and prepare() (coarsening) so kernel choice and
the bins the kernel sees are the reference's.
"""
from __future__ import annotations

from typing import Optional

import numpy as np
import torch

from tenex_b200 import native
from tenex_b200.kernels import TEKernel
from tenex_b200.kernels import device as D

# Launch shapes the autotuner tries: (threads, ctas_per_sm, src_chunk); 0 = the
# library's choice (2 x 512 threads, or 1 x 1024 when the largest histogram needs
# a whole SM's shared memory)
TUNE_SPACE = [(0, 0, 512), (1024, 1, 512), (512, 2, 512), (512, 2, 256), (1024, 1, 256),
              (256, 4, 128), (256, 4, 256), (512, 2, 128), (1024, 1, 128), (256, 2, 64)]
# Without autotuning the library picks the shape; 512 sources per item. Measured
# (ms per all-pairs launch): 10,000 x 20,000 (b_max 38) 989 vs 1097 for the old
# 2 x 512 / 128 default; 5,000 x 10,000 (b_max 32) 256.0 vs 258.8; 2,000 x 5,000
# (b_max 16) 11.37 vs 11.78 (11.14 for the best tuned shape).
DEFAULT_CFG = dict(threads=0, ctas_per_sm=0, src_chunk=512)
_tune_cache: dict[tuple, dict] = {}


def _npv_tensor(n_per_var, device) -> torch.Tensor:
    """int32 n_per_var on `device` (a tensor already there is used as it is: no
    round trip through the host)."""
    if isinstance(n_per_var, torch.Tensor):
        return n_per_var.to(device=device, dtype=torch.int32).contiguous()
    return torch.as_tensor(np.asarray(n_per_var), dtype=torch.int32).to(device).contiguous()


def autotune(db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int = 1,
             sample_pairs: int = 6_000_000, space=TUNE_SPACE) -> dict:
    """Times each launch shape on a contiguous slice of pair ids (whole targets
    from the middle of the range) and returns the fastest; cached per
    (device, n, T, K, b_max, tau, bin-count histogram). The slice is large
    enough (6M pairs: ~60 ms per shape at 10k genes x 20k cells, ~80 items of
    512 sources per SM) that the end of a launch, where few items remain, does
    not decide between item sizes; a 2M-pair slice picked 128 sources per item,
    3% slower than 512 on the full launch."""
    dev = db.data.device
    npv_h = npv.cpu().numpy()
    key = (torch.cuda.get_device_name(dev), db.n, db.T, db.K, int(b_max), int(tau),
           tuple(np.bincount(np.minimum(npv_h, 64), minlength=65)[::4]))
    if key in _tune_cache:
        return _tune_cache[key]
    n = db.n
    total = n * (n - 1)
    cnt = min(total, max(n - 1, (sample_pairs // (n - 1)) * (n - 1)))
    p0 = ((total - cnt) // 2) // (n - 1) * (n - 1)
    best, best_t = dict(DEFAULT_CFG), float("inf")
    for th, cps, w in space:
        cfg = dict(threads=th, ctas_per_sm=cps, src_chunk=w)
        try:
            D.te_pairfree(db, npv, b_max, tau, p0, cnt, cfg=cfg, check_data=False)
            torch.cuda.synchronize(dev)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
            D.te_pairfree(db, npv, b_max, tau, p0, cnt, cfg=cfg, check_data=False)
            e1.record()
            e1.synchronize()
            t = e0.elapsed_time(e1)
        except Exception:
            continue
        if t < best_t:
            best, best_t = cfg, t
    _tune_cache[key] = best
    return best


class PairTileKernel(TEKernel):
    """Pair-free / pair-list TE through the persistent shared-memory kernel."""

    cfg: Optional[dict] = None  # launch shape override (None: tuned or default)

    @property
    def supports_pairfree(self) -> bool:
        return True

    def launch_cfg(self, db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int,
                   autotune_shape: bool) -> dict:
        if self.cfg is not None:
            return self.cfg
        if autotune_shape:
            return autotune(db, npv, b_max, tau)
        return DEFAULT_CFG

    def compute_pairfree_device(self, db: D.DeviceBins, n_per_var, b_max: int, tau: int,
                                pair_offset: int = 0, n_pairs: Optional[int] = None,
                                matrix: bool = False, out: Optional[torch.Tensor] = None,
                                autotune_shape: bool = False) -> torch.Tensor:
        """Device-resident result: pair-free float32 vector, or the (n, n) matrix
        with [src, tgt] = TE(src -> tgt) when matrix=True."""
        npv = _npv_tensor(n_per_var, db.data.device)
        cfg = self.launch_cfg(db, npv, b_max, tau, autotune_shape)
        return D.te_pairfree(db, npv, int(b_max), tau, pair_offset, n_pairs, out=out,
                             matrix=matrix, cfg=cfg)

    def compute_pairfree(self, bin_arrs, n_vars: int, b_max: int, n_per_var, tau: int,
                         device, pair_offset: int = 0,
                         n_pairs_local: Optional[int] = None) -> np.ndarray:
        dev = torch.device(device) if not isinstance(device, torch.device) else device
        db = D.pack_bins(bin_arrs, dev, b_max)
        if db.n != n_vars:
            raise ValueError(f"bin_arrs has {db.n} variables, n_vars={n_vars}")
        te = self.compute_pairfree_device(db, n_per_var, b_max, tau, pair_offset,
                                          n_pairs_local)
        return D.to_host(te)

    def compute_pairfree_cross(self, bin_arrs, n_per_var, n_tgt: int, n_src: int, tau: int,
                               device, pair_offset: int = 0,
                               n_pairs_local: Optional[int] = None) -> np.ndarray:
        """TE between two disjoint gene blocks (tenex/kernels/adaptive_smem.py:1114-1160,
        the variable-blocking path): bin_arrs rows [0, n_tgt) are the targets and
        [n_tgt, n_tgt + n_src) the sources; pair id = tgt_local * n_src + src_local,
        value TE(source -> target). Runs as a pair list built on the device."""
        from tenex_b200.kernels.pair_list import item_table
        dev = torch.device(device) if not isinstance(device, torch.device) else device
        total = int(n_tgt) * int(n_src)
        if n_pairs_local is None:
            n_pairs_local = total - pair_offset
        if pair_offset < 0 or n_pairs_local < 0 or pair_offset + n_pairs_local > total:
            raise ValueError(f"pair range [{pair_offset}, {pair_offset + n_pairs_local}) "
                             f"outside [0, {total})")
        out = torch.empty(n_pairs_local, dtype=torch.float32, device=dev)
        if n_pairs_local == 0:
            return D.to_host(out)
        b_max = int(torch.as_tensor(n_per_var).max())
        db = D.pack_bins(bin_arrs, dev, b_max)
        npv = _npv_tensor(n_per_var, dev)
        ids = torch.arange(pair_offset, pair_offset + n_pairs_local, device=dev, dtype=torch.int64)
        tgt = ids // n_src
        pairs = torch.stack((tgt, n_tgt + ids - tgt * n_src), dim=1).contiguous()
        items = torch.from_numpy(item_table(tgt.cpu().numpy(), 128)).to(dev)
        ws = D.workspace(dev, db.n, db.row_len, b_max)
        s = native.stream_ptr()
        native.call("tenex_te_pairs", db.ptr(), db.ld, npv.data_ptr(), b_max, db.n,
                    db.row_len, tau * db.K, pairs.data_ptr(), n_pairs_local, items.data_ptr(),
                    items.numel() - 1, out.data_ptr(), ws.data_ptr(), ws.numel(),
                    D._cfg(self.cfg), s)
        native.call("tenex_workspace_status", ws.data_ptr(), s)
        return D.to_host(out)

    def compute_single_gpu(self, bin_arrs, pairs, b_max, n_per_var, tau, batch_size, device,
                           **kwargs) -> np.ndarray:
        from tenex_b200.kernels.pair_list import te_pair_list
        dev = torch.device(device) if not isinstance(device, torch.device) else device
        db = D.pack_bins(bin_arrs, dev, b_max)
        npv = _npv_tensor(n_per_var, dev)
        pr = pairs.cpu().numpy() if isinstance(pairs, torch.Tensor) else np.asarray(pairs)
        return te_pair_list(db, npv, int(b_max), tau, pr, cfg=self.cfg).cpu().numpy()
