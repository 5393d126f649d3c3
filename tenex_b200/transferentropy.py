"""TransferEntropyEngine — the public entry point of the TE path.

Mirrors tenex/transferentropy.py of the reference (constructor :54-106,
compute() :537-1038, result assembly :1383-1436): same arguments, validation
errors, kernel selection (explicit kernel= checked with supports(), else
auto_select) and result object. Everything from discretisation to the (n, n)
matrix runs on one CUDA device in libtenex_sm100.so kernels; the bins never
leave the device until the result is wrapped.

Differences from the reference, by design:
  * accelerator="cpu" is rejected: this build has no CPU path (the TE kernels
    are sm_100a code); "auto" requires CUDA.
  * devices= with several ids splits the pair-id range into contiguous chunks,
    one host thread and one copy of the bins per device (the reference's
    in-process split, tenex/transferentropy.py:360-440); the devices share no
    data path. Several processes (one per GPU, torchrun) use
    tenex_b200.distributed instead.
  * Bins are always the numpy/FastTENET FSBW-L bins (the reference's GPU torch
    binning differs from them in the last float32 bit of std).
"""
from __future__ import annotations

import time
from typing import Optional, Union

import numpy as np
import torch

from tenex_b200 import _log
from tenex_b200.kernels import compute_smem_bytes, query_smem_optin
from tenex_b200.kernels import device as D
from tenex_b200.preprocess import compact_dtype, discretize
from tenex_b200.result import TransferEntropyResult


class TransferEntropyEngine:
    """Pairwise transfer entropy for all (or source-filtered) variable pairs.

    data           : (n_vars, T) float32 time series (column = time step)
    variable_names : (n_vars,) unique names
    sources        : optional subset of variable_names used as TE sources
    """

    def __init__(self, data: np.ndarray, variable_names: np.ndarray,
                 sources: Optional[np.ndarray] = None):
        if data is None or variable_names is None:
            raise ValueError("data and variable_names are required.")
        self._data = np.asarray(data, dtype=np.float32)
        self._variable_names = np.asarray(variable_names)
        if self._data.ndim != 2 or self._data.size == 0:
            raise ValueError(f"data must be a non-empty 2-D array of shape (n_vars, T); "
                             f"got shape {self._data.shape}")
        if not D.all_finite(self._data):
            raise ValueError("data contains NaN or infinite values")
        if self._variable_names.ndim != 1:
            raise ValueError(f"variable_names must be 1-D; got shape "
                             f"{self._variable_names.shape}")
        n_vars = self._data.shape[0]
        if self._variable_names.shape[0] != n_vars:
            raise ValueError(f"variable_names length ({self._variable_names.shape[0]}) must "
                             f"match the number of variables ({n_vars})")
        if len(np.unique(self._variable_names)) != n_vars:
            raise ValueError("variable_names must be unique")
        if sources is not None:
            src = np.atleast_1d(np.asarray(sources))
            if src.ndim != 1:
                raise ValueError(f"sources must be 1-D; got shape {src.shape}")
            missing = np.setdiff1d(src, self._variable_names)
            if missing.size > 0:
                raise ValueError(f"source names not found in variable_names: {list(missing)}")
            if len(np.unique(src)) != src.shape[0]:
                raise ValueError("sources must not contain duplicate names")
            self._sources = src.copy()
        else:
            self._sources = None
        self._result_matrix = None
        self._bin_cache: dict = {}
        self._pairs_cache: dict = {}
        self._last_run_info: Optional[dict] = None
        self._last_bin_arrs = None
        self._last_n_per_var = None

    @property
    def variable_names(self) -> np.ndarray:
        return self._variable_names

    def clear_cache(self):
        self._bin_cache.clear()
        self._pairs_cache.clear()

    def save_result_matrix(self, spath: str):
        if self._result_matrix is None:
            raise ValueError("compute() has not been called yet")
        tmp = np.concatenate([self._variable_names[:, None],
                              self._result_matrix.astype(str)], axis=1)
        header = np.concatenate((["TE"], self._variable_names))
        np.savetxt(spath, np.concatenate([header[None, :], tmp]), delimiter="\t", fmt="%s")

    # ------------------------------------------------------------------ devices
    @staticmethod
    def _resolve_accelerator_and_devices(accelerator: str = "auto",
                                         devices: Union[int, list, str, None] = "auto"
                                         ) -> list[int]:
        accel = accelerator.lower()
        if accel == "cpu":
            raise NotImplementedError(
                "accelerator='cpu': this build runs the TE path on CUDA (sm_100a) only")
        if accel not in ("auto", "gpu"):
            raise ValueError(f"Unknown accelerator '{accelerator}'. "
                             f"Choose from: 'auto', 'cpu', 'gpu'")
        if not torch.cuda.is_available():
            raise RuntimeError(f"accelerator='{accelerator}' but no CUDA device is available")
        all_gpus = list(range(torch.cuda.device_count()))
        if devices is None or (isinstance(devices, str) and devices == "auto"):
            ids = [torch.cuda.current_device()]
        elif isinstance(devices, int):
            if devices == -1:
                ids = all_gpus
            elif devices <= 0:
                raise ValueError(f"devices as int must be >= 1 or -1 (got {devices})")
            elif devices > len(all_gpus):
                raise ValueError(f"Requested {devices} GPUs but only {len(all_gpus)} available")
            else:
                ids = all_gpus[:devices]
        elif isinstance(devices, (list, tuple)):
            for d in devices:
                if d not in all_gpus:
                    raise ValueError(f"GPU {d} not available. Available: {all_gpus}")
            ids = list(devices)
        else:
            raise TypeError(f"devices must be 'auto', int, list[int], or None "
                            f"(got {type(devices).__name__})")
        return ids

    # ------------------------------------------------------------------ bins
    def _discretize(self, binning_method: str, kp: float, device: torch.device):
        key = (binning_method.upper(), float(kp), str(device))
        if key not in self._bin_cache:
            self._bin_cache[key] = discretize(self._data, binning_method, kp, device)
        return self._bin_cache[key]

    def _binarize(self, method: str, device: torch.device, params: Optional[dict]):
        from tenex_b200.binarize import binarize
        key = ("BIN:" + method.upper(), tuple(sorted((params or {}).items())), str(device))
        if key not in self._bin_cache:
            self._bin_cache[key] = binarize(self._data, method, device, **(params or {}))
        return self._bin_cache[key]

    def _build_pairs(self, n_vars: int) -> np.ndarray:
        """[target, source] pairs for the source filter, stably sorted by target
        (reference order, tenex/transferentropy.py:456-498)."""
        key = (n_vars, None if self._sources is None else tuple(self._sources))
        if key in self._pairs_cache:
            return self._pairs_cache[key]
        _, inds, _ = np.intersect1d(self._variable_names, self._sources, return_indices=True)
        if len(inds) == 0:
            raise ValueError("No source names found in variable_names.")
        srcs = inds.astype(np.int64)
        blocks = []
        for t in range(n_vars):
            s_valid = srcs[srcs != t]
            if len(s_valid):
                b = np.empty((len(s_valid), 2), np.int64)
                b[:, 0] = t
                b[:, 1] = s_valid
                blocks.append(b)
        pairs = np.concatenate(blocks) if blocks else np.empty((0, 2), np.int64)
        pairs = pairs[np.argsort(pairs[:, 0], kind="stable")]
        self._pairs_cache[key] = pairs
        return pairs

    @staticmethod
    def _select_kernel(kernel_name, b_max, on_cuda, smem_optin, smem_bytes, n_per_var,
                       source_filter):
        from tenex_b200.kernels import auto_select, get_kernel
        if kernel_name is not None:
            k = get_kernel(kernel_name)
            if k.name == "GEMM-B2" and b_max != 2:
                raise ValueError(f"kernel='GEMM-B2' requires binary data (b_max=2), but this "
                                 f"data has b_max={b_max}. Use kernel=None for auto-selection.")
            if not k.supports(b_max, on_cuda, smem_optin, smem_bytes, n_per_var, source_filter):
                raise ValueError(f"kernel={kernel_name!r} does not support this configuration "
                                 f"(b_max={b_max}, on_cuda={on_cuda}, source_filter="
                                 f"{source_filter}). Use kernel=None for auto-selection.")
            return k
        return auto_select(b_max, on_cuda, smem_optin, smem_bytes, n_per_var, source_filter)

    # ------------------------------------------------------------------ compute
    def compute(self, accelerator: str = "auto", devices: Union[int, list, str, None] = "auto",
                binning_method: str = "FSBW-L", binarization: Optional[str] = None,
                binarization_backend: Optional[str] = None,
                binarization_kwargs: Optional[dict] = None, kp: float = 0.5, tau: int = 1,
                batch_size: Optional[int] = None, autotune: bool = False,
                kernel: Optional[str] = None, coarsening: Optional[bool] = None,
                use_numpy_bins: Optional[bool] = None, profile: bool = False,
                verbose: bool = False) -> TransferEntropyResult:
        """Pairwise TE; returns a TransferEntropyResult whose matrix[i, j] = TE(i -> j).

        Arguments are the reference's. batch_size and use_numpy_bins are accepted
        and have no effect (one persistent launch covers all pairs; bins are
        always FastTENET-exact); autotune=True times launch shapes once per data
        shape and caches the fastest.
        """
        _log.set_verbose(verbose)
        t0 = time.time()
        device_ids = self._resolve_accelerator_and_devices(accelerator, devices)
        dev = torch.device("cuda", device_ids[0])
        torch.cuda.set_device(dev)
        stream = torch.cuda.current_stream(dev)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(8)] if profile else None

        def mark(i):
            if ev is not None:
                ev[i].record(stream)

        mark(0)
        arr = self._data
        n_vars, T = arr.shape
        if isinstance(tau, bool) or not isinstance(tau, (int, np.integer)) or tau < 1:
            raise ValueError(f"tau must be an integer >= 1; got {tau!r}")
        if T <= tau:
            raise ValueError(f"Time series length T={T} must be greater than tau={tau}")
        if n_vars < 2:
            self._result_matrix = np.zeros((n_vars, n_vars), dtype=np.float32)
            self._last_run_info, self._last_bin_arrs, self._last_n_per_var = {}, None, None
            return self._wrap_result()
        mark(1)

        if binarization is not None:
            db, n_bins, b_max, npv = self._binarize(binarization, dev, binarization_kwargs)
        else:
            db, n_bins, b_max, npv = self._discretize(binning_method, kp, dev)
        K = db.K
        n_samples = (db.T - tau) * K
        if n_samples >= 2 ** 31:
            raise ValueError(f"sample count l_eff*K={n_samples} exceeds the int32 histogram "
                             f"limit (2^31); counts would overflow")
        mark(2)

        smem_bytes = compute_smem_bytes(b_max, db.T, K, tau)
        smem_optin = query_smem_optin(device_ids)
        source_filter = self._sources is not None
        kobj = self._select_kernel(kernel, b_max, True, smem_optin, smem_bytes, npv,
                                   source_filter)
        info = {"n_vars": n_vars, "T": T, "K": K, "tau": tau, "n_pairs": n_vars * (n_vars - 1),
                "device_ids": device_ids, "n_gpus": len(device_ids),
                "binning_method": binning_method if binarization is None else binarization,
                "binarization": binarization, "kp": kp, "b_max_before_coarsen": b_max,
                "b_max": b_max, "kernel": kobj.name, "smem_optin": smem_optin,
                "smem_bytes": smem_bytes, "source_filter": source_filter,
                "bin_dtype": "uint16" if db.wide else "uint8",
                "bin_bytes": db.data.numel()}
        _log.vprint(f"[TENEX] data: {n_vars} x {T}, K={K}, b_max={b_max}, kernel={kobj.name}")
        mark(3)

        if kobj.is_matrix_kernel:
            info.update(mode="matrix", pair_free=False, coarsened=False)
            mark(4)
            if len(device_ids) > 1:
                # [i, j] = TE(j -> i) from the matrix kernels' multi-device entry
                self._result_matrix = kobj.compute_matrix_multi_gpu(
                    self._host_bins(db), n_vars, tau, device_ids).T.copy()
                mark(5)
            else:
                m = kobj.compute_matrix_device(db, tau)  # [src, tgt] = TE(src -> tgt)
                mark(5)
                self._result_matrix = D.to_host(m)
            self._finish(info, db, npv, b_max, ev, stream, t0, "matrix")
            return self._wrap_result()

        # prepare (coarsening) works on a copy so the cached bins stay intact
        work = D.DeviceBins(db.data.clone(), db.n, db.T, db.K)
        npv_w = npv.clone()
        work, npv_w, b_max_w = kobj.prepare(work, npv_w, b_max, use_coarsening=coarsening,
                                            on_cuda=True, n_vars=n_vars, tau=tau,
                                            smem_optin=smem_optin)
        info.update(b_max=b_max_w, coarsened=b_max_w != b_max)
        mark(4)
        mark(5)
        if source_filter:
            info.update(mode="pair", pair_free=False)
            pairs = self._build_pairs(n_vars)
            if len(device_ids) > 1:
                te_h = kobj.compute_multi_gpu(self._host_bins(work), pairs, b_max_w,
                                              npv_w.cpu(), tau, batch_size, device_ids)
                mark(6)
            else:
                from tenex_b200.kernels.pair_list import te_pair_list
                te = te_pair_list(work, npv_w, b_max_w, tau, pairs,
                                  cfg=getattr(kobj, "cfg", None))
                mark(6)
                te_h = D.to_host(te)
            rm = np.zeros((n_vars, n_vars), dtype=np.float32)
            rm[pairs[:, 0], pairs[:, 1]] = te_h
            self._result_matrix = rm.T.copy()
        else:
            info.update(mode="pairfree", pair_free=True)
            if len(device_ids) > 1:
                self._result_matrix = self._pairfree_multi_device(
                    kobj, work, npv_w, b_max_w, tau, device_ids, autotune)
                mark(6)
            else:
                m = kobj.compute_pairfree_device(work, npv_w, b_max_w, tau, matrix=True,
                                                 autotune_shape=autotune)
                mark(6)
                self._result_matrix = D.to_host(m)
        self._finish(info, work, npv_w, b_max_w, ev, stream, t0, "pair")
        return self._wrap_result()

    @staticmethod
    def _host_bins(db: D.DeviceBins) -> np.ndarray:
        """(n, T, K) host copy of device bins (the padding dropped)."""
        return D.to_host(db.data[:, :db.row_len]).reshape(db.n, db.T, db.K)

    @staticmethod
    def _pairfree_multi_device(kobj, work: D.DeviceBins, npv: torch.Tensor, b_max: int,
                               tau: int, device_ids: list, autotune: bool) -> np.ndarray:
        """All-pairs TE split over devices: contiguous pair-id chunks of
        ceil(n(n-1) / devices), one host thread per device with its own copy of the
        prepared bins; the per-device matrices hold disjoint entries and are summed
        (exactly: every entry has one non-zero contributor)."""
        from concurrent.futures import ThreadPoolExecutor
        from tenex_b200.distributed import pair_range
        n = work.n
        total = n * (n - 1)
        host = work.data.cpu()
        npv_h = npv.cpu()

        def run(rank: int):
            p0, p1 = pair_range(total, rank, len(device_ids))
            if p1 <= p0:
                return None
            torch.cuda.set_device(device_ids[rank])
            dev = torch.device("cuda", device_ids[rank])
            db = D.DeviceBins(host.to(dev), n, work.T, work.K)
            m = kobj.compute_pairfree_device(db, npv_h.to(dev), b_max, tau, p0, p1 - p0,
                                             matrix=True, autotune_shape=autotune)
            return D.to_host(m)

        with ThreadPoolExecutor(max_workers=len(device_ids)) as ex:
            parts = [p for p in ex.map(run, range(len(device_ids))) if p is not None]
        out = parts[0].copy()
        for p in parts[1:]:
            out += p
        return out

    def _finish(self, info, db, npv, b_max, ev, stream, t0, mode):
        if ev is not None:
            ev[7].record(stream)
            ev[7].synchronize()

            def sec(a, b):
                try:
                    return ev[a].elapsed_time(ev[b]) / 1000.0
                except (RuntimeError, ValueError):
                    return 0.0
            timings = {"total": time.time() - t0, "data_align": sec(0, 1),
                       "discretize": sec(1, 2), "kernel_select": sec(2, 3),
                       "prepare": sec(3, 4)}
            if mode == "matrix":
                timings["compute"] = sec(4, 5)
            else:
                timings["compute"] = sec(5, 6)
                timings["assemble"] = sec(6, 7)
            info["timings"] = timings
        self._last_run_info = info
        # the compact dtype is applied on the device (bins are < 256, so the values
        # are unchanged), then one staged copy
        dt = torch.from_numpy(np.empty(0, dtype=compact_dtype(b_max))).dtype
        self._last_bin_arrs = D.to_host(db.unpadded().to(dt))
        self._last_n_per_var = npv.cpu().numpy()
        elapsed = time.time() - t0
        _log.vprint(f"[TENEX] done -- {elapsed:.3f}s "
                    f"({info['n_pairs'] / max(elapsed, 1e-9):,.0f} pairs/s)")

    def _wrap_result(self) -> TransferEntropyResult:
        info = self._last_run_info or {}
        return TransferEntropyResult(matrix=self._result_matrix,
                                     variable_names=self._variable_names,
                                     bin_arrs=self._last_bin_arrs,
                                     n_per_var=self._last_n_per_var,
                                     b_max=info.get("b_max", 0), tau=info.get("tau", 1),
                                     kernel=info.get("kernel", ""),
                                     timings=info.get("timings"), sources=self._sources)
