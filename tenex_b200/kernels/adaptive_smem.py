"""Adaptive-SMEM kernel class (reference: tenex/kernels/adaptive_smem.py:1213-1330).

supports() accepts any b_max on CUDA; prepare() applies the reference's
coarsening rule (coarsen every gene above compute_smem_bin_limit(opt-in, warps))
with the GPU coarsening kernel, so the bins the TE kernel sees are the
reference's bins. Per-pair histograms of uneven size (b_t^2 * b_s cells) are
packed by the persistent kernel (slot size chosen per work item).
"""
from __future__ import annotations

import torch

from tenex_b200 import _log

from tenex_b200.kernels import _next_pow2
from tenex_b200.kernels.pair_tile import PairTileKernel


def compute_smem_bin_limit(smem_optin: int, warps: int = 32) -> int:
    """Largest B with (B^3 + 2B^2 + B + warps) * 4 <= smem_optin
    (reference rule, tenex/kernels/adaptive_smem.py:701-726): 38 on B200."""
    B = max(2, int((smem_optin / 4) ** (1.0 / 3.0)))
    while B > 2 and (B ** 3 + 2 * B ** 2 + B + warps) * 4 > smem_optin:
        B -= 1
    return B


class AdaptiveSMEMKernel(PairTileKernel):
    """Per-gene b (uneven histograms) through the shared-memory kernel."""

    @property
    def name(self) -> str:
        return "Adaptive-SMEM"

    def supports(self, b_max, on_cuda, smem_optin, smem_bytes, n_per_var,
                 source_filter) -> bool:
        return bool(on_cuda)

    def prepare(self, bin_arrs, n_per_var, b_max, **kwargs):
        """Coarsens genes above the shared-memory bin limit (in place on the
        device bins). kwargs: use_coarsening (None/True apply, False reject
        b_max above the limit), smem_optin, tau."""
        from tenex_b200.kernels import device as D
        from tenex_b200.preprocess import coarsen_bins
        use_coarsening = kwargs.get("use_coarsening")
        on_cuda = kwargs.get("on_cuda", True)
        if not on_cuda:
            return bin_arrs, n_per_var, b_max
        smem_optin = kwargs.get("smem_optin")
        if not smem_optin:
            from tenex_b200.kernels import query_smem_optin
            smem_optin = query_smem_optin(torch.cuda.current_device())
        db = bin_arrs
        N = (db.T - kwargs.get("tau", 1)) * db.K if isinstance(db, D.DeviceBins) else None
        warps = max(128, min(1024, _next_pow2(max(N or 1024, 1)))) // 32
        limit = compute_smem_bin_limit(int(smem_optin), warps=warps)
        if b_max <= limit:
            return bin_arrs, n_per_var, b_max
        if use_coarsening is False:
            # as the reference (tenex/kernels/adaptive_smem.py:1252-1262): bins stay
            # as they are and the pairs whose histogram does not fit shared memory
            # run in the kernel's global-memory overflow launch; bins are uint8 here
            if b_max >= 256:
                raise ValueError(
                    f"coarsening=False but b_max={b_max} >= 256, which the global-memory "
                    f"overflow path cannot hold in uint8 bins. Use coarsening=None (default) "
                    f"or kp<0.5 to reduce bins.")
            _log.vprint("[TENEX] bin coarsening disabled: shared-memory kernel + global-memory "
                        "overflow")
            return bin_arrs, n_per_var, b_max
        return coarsen_bins(bin_arrs, n_per_var, limit)
