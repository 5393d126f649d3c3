"""Full-SMEM kernel class (reference: tenex/kernels/full_smem.py:669-750).

Same name and supports() predicate as the reference (b_max^3 <= 65536 and the
reference's shared-memory formula within the device opt-in); the work runs in
the persistent pair-tile kernel of te_pair.cu.
"""
from __future__ import annotations

from tenex_b200.kernels.pair_tile import PairTileKernel


class FullSMEMKernel(PairTileKernel):
    """Uniform-b pairs through the shared-memory histogram kernel."""

    @property
    def name(self) -> str:
        return "Full-SMEM"

    def supports(self, b_max, on_cuda, smem_optin, smem_bytes, n_per_var,
                 source_filter) -> bool:
        if not on_cuda:
            return False
        return b_max ** 3 <= 65536 and smem_bytes <= smem_optin
