"""TE kernel plugin API and registry (the drop-in boundary of the TE path).

Mirrors tenex/kernels/__init__.py of the reference (TEKernel ABC :85-442,
register/get_kernel/auto_select/registered_kernels :447-519,
query_smem_optin :44-71, compute_smem_bytes :74-80): same names, argument
meaning, priority order and errors, so callers written against the reference
keep working. Behind it every kernel calls libtenex_sm100.so (sm_100a); there
is no CPU or library fallback.

Priority (highest first):
  1. GEMM-B2       — binary data (b_max = 2), no source filter: tcgen05 INT8 GEMM
  2. Full-SMEM     — b_max^3 <= 65536 and the reference's SMEM formula fits
  3. Adaptive-SMEM — any b_max (bins coarsened to the device's shared-memory limit)
"""
from __future__ import annotations

from abc import ABC, abstractmethod
from typing import Optional

import numpy as np
import torch


def _next_pow2(x: int) -> int:
    return 1 << max(0, (x - 1).bit_length())


def query_smem_optin(device_ids=0) -> int:
    """Opt-in shared memory per block (bytes) of a device, or the minimum over a
    list of devices. Raises if the native library or CUDA is unavailable."""
    from tenex_b200 import native
    ids = list(device_ids) if isinstance(device_ids, (list, tuple)) else [int(device_ids)]
    if not ids:
        return 48 * 1024
    return min(int(native.device_info(int(d)).smem_optin) for d in ids)


def compute_smem_bytes(b_max: int, n_time: int, n_kernels: int, tau: int) -> int:
    """The reference's Full-SMEM footprint formula, kept for kernel-selection parity."""
    b2 = b_max * b_max
    b3 = b_max ** 3
    N = (n_time - tau) * n_kernels
    bs = max(128, min(1024, _next_pow2(max(N, 2 * b2))))
    return b3 * 4 + b2 * 4 * 2 + b_max * 4 + (bs // 32) * 4


class TEKernel(ABC):
    """Strategy interface of one TE backend."""

    @property
    @abstractmethod
    def name(self) -> str:
        """Kernel name for logging and get_kernel() (e.g. 'Full-SMEM')."""

    @property
    def is_matrix_kernel(self) -> bool:
        """True for kernels that compute the full (n, n) matrix directly."""
        return False

    @property
    def supports_pairfree(self) -> bool:
        return False

    @abstractmethod
    def supports(self, b_max: int, on_cuda: bool, smem_optin: int, smem_bytes: int,
                 n_per_var: Optional[torch.Tensor], source_filter: bool) -> bool:
        """True if this kernel can handle the given data configuration."""

    def compute_single_gpu(self, bin_arrs, pairs, b_max: int, n_per_var, tau: int,
                           batch_size: Optional[int], device: torch.device,
                           **kwargs) -> np.ndarray:
        """TE for an explicit (P, 2) [target, source] pair list; float32 (P,)."""
        raise NotImplementedError(f"{self.name} has no pair-list path")

    def compute_pairfree(self, bin_arrs, n_vars: int, b_max: int, n_per_var, tau: int,
                         device: torch.device, pair_offset: int = 0,
                         n_pairs_local: Optional[int] = None) -> np.ndarray:
        """TE for pair-free ids [pair_offset, pair_offset + n_pairs_local); float32."""
        raise NotImplementedError(f"{self.name} has no pair-free path")

    def compute_matrix(self, data, n_vars: int, tau: int, device: torch.device,
                       **kwargs) -> np.ndarray:
        """Full (n, n) matrix with [i, j] = TE(j -> i). Override for matrix kernels."""
        raise NotImplementedError(f"{self.name} is a pair-based kernel")

    def compute_multi_gpu(self, bin_arrs_cpu, pairs_np, b_max: int, n_per_var_cpu, tau: int,
                          batch_size: Optional[int], device_ids: list, **kwargs) -> np.ndarray:
        """Pair list over several devices (tenex/kernels/__init__.py:148-236): contiguous
        chunks of ceil(P / n_devices) pairs, one host thread per device, each with its
        own copy of the bins calling compute_single_gpu; results in the caller's pair
        order. The devices work independently (no collectives)."""
        from concurrent.futures import ThreadPoolExecutor
        pairs_np = np.asarray(pairs_np)
        P = pairs_np.shape[0]
        ids = [int(d) for d in device_ids]
        if not ids:
            raise ValueError("device_ids must name at least one device")
        chunk = -(-P // len(ids)) if P else 0

        def run(rank: int) -> np.ndarray:
            beg, end = rank * chunk, min(P, (rank + 1) * chunk)
            if beg >= end:
                return np.empty(0, np.float32)
            torch.cuda.set_device(ids[rank])
            dev = torch.device("cuda", ids[rank])
            return self.compute_single_gpu(bin_arrs_cpu, pairs_np[beg:end], b_max, n_per_var_cpu,
                                           tau, batch_size, dev, **kwargs)

        with ThreadPoolExecutor(max_workers=len(ids)) as ex:
            parts = list(ex.map(run, range(len(ids))))
        return np.concatenate(parts) if parts else np.empty(0, np.float32)

    def compute_matrix_multi_gpu(self, data, n_vars: int, tau: int, device_ids: list,
                                 **kwargs) -> np.ndarray:
        """Full matrix over several devices. Override for matrix kernels."""
        raise NotImplementedError(f"{self.name} is a pair-based kernel")

    def peak_batch_bytes(self, b_max: int, T: int, K: int, batch_size: int, tau: int = 1) -> int:
        return batch_size * 4 + batch_size * 2 * 8

    def peak_bytes_per_pair(self, b_max: int, T: int, K: int, tau: int = 1) -> int:
        """Device bytes per pair of a pair-list launch: the float32 result and the
        (target, source) int64 pair. Histograms live in shared memory."""
        return 4 + 2 * 8

    def heuristic_batch_size(self, bin_arrs, b_max: int, tau: int = 1) -> int:
        """Pairs per pair-list launch that fit 80% of the free device memory
        (tenex/kernels/__init__.py:266-322 sizes batches the same way). The
        persistent kernels take any number of pairs in one launch, so the batch
        only bounds the pair and result buffers."""
        device = getattr(bin_arrs, "device", torch.device("cpu"))
        if device.type != "cuda":
            return 2048
        shape = tuple(bin_arrs.shape)
        T, K = int(shape[1]), int(shape[2]) if len(shape) > 2 else 1
        free = torch.cuda.mem_get_info(device)[0]
        budget = max(0, int(free * 0.8) - (256 << 20))
        return max(1024, budget // self.peak_bytes_per_pair(b_max, T, K, tau))

    def autotune_batch_size(self, bin_arrs, b_max: int, n_per_var, tau: int,
                            device: torch.device) -> int:
        """The batch size does not change the persistent kernel's speed (work is
        handed out by an atomic ticket inside one launch), so the tuned value is
        the memory heuristic's; the launch shape is tuned separately
        (tenex_b200.kernels.pair_tile.autotune)."""
        return self.heuristic_batch_size(bin_arrs, b_max, tau)

    def prepare(self, bin_arrs, n_per_var, b_max: int, **kwargs):
        """Optional preprocessing hook (e.g. bin coarsening). Default: no-op."""
        return bin_arrs, n_per_var, b_max

    def log_description(self, **kwargs) -> str:
        b_max = kwargs.get("b_max")
        return f"{self.name} (b_max={b_max})" if b_max is not None else self.name


_REGISTRY: list[TEKernel] = []
_REGISTERED = False


def register(kernel: TEKernel) -> TEKernel:
    _REGISTRY.append(kernel)
    return kernel


def get_kernel(name: str) -> TEKernel:
    """Registered kernel by name (case-insensitive); KeyError if unknown."""
    needle = name.lower()
    for k in _REGISTRY:
        if k.name.lower() == needle:
            return k
    raise KeyError(f"Kernel '{name}' not found. Available: {[k.name for k in _REGISTRY]}")


def auto_select(b_max: int, on_cuda: bool, smem_optin: int, smem_bytes: int,
                n_per_var: Optional[torch.Tensor], source_filter: bool,
                exclude: Optional[set[str]] = None) -> TEKernel:
    """First registered kernel (priority order) whose supports() accepts the data."""
    for kernel in _REGISTRY:
        if exclude and kernel.name in exclude:
            continue
        if kernel.supports(b_max, on_cuda, smem_optin, smem_bytes, n_per_var, source_filter):
            return kernel
    raise RuntimeError(f"No suitable TE kernel found for b_max={b_max}, on_cuda={on_cuda}, "
                       f"smem_optin={smem_optin}")


def registered_kernels() -> list[TEKernel]:
    return list(_REGISTRY)


def _register_all() -> None:
    global _REGISTERED
    if _REGISTERED:
        return
    _REGISTERED = True
    from tenex_b200.kernels.gemm_b2 import GEMMB2Kernel
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    from tenex_b200.kernels.adaptive_smem import AdaptiveSMEMKernel
    register(GEMMB2Kernel())
    register(FullSMEMKernel())
    register(AdaptiveSMEMKernel())


_register_all()
