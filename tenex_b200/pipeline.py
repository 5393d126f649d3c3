"""Pipeline — cached TE matrix + surrogate test, and the multi-lag combine.

Mirrors tenex/pipeline.py (PipelineResult :44-77, Pipeline :79-420): the same
constructor, configure() / te_result / clear_cache() / infer() / run() API and
the same multi-lag combine (_infer_multi_lag :251-314,
_combine_surrogate_multi_lag :316-410), which re-runs the TE hot path and the
surrogate test once per lag and merges the per-lag results per pair ("max":
lag with the largest effective TE; "adaptive_select": smallest p; "weighted_sum":
effective TE summed with weights -log p for p < 0.05), with a Bonferroni p
(K * min p) and BH-FDR over the off-diagonal pairs. infer() dispatches to the
registered methods ('surrogate_test', 'fdr'); CLR/ND/TRACE/POINT are not part of
this package and raise NotImplementedError.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from tenex_b200 import _log
from tenex_b200.result import TransferEntropyResult
from tenex_b200.transferentropy import TransferEntropyEngine

_FUSED_METHODS = frozenset({"surrogate_test"})


@dataclass
class PipelineResult:
    te_result: TransferEntropyResult
    inference_results: dict[str, Any] = field(default_factory=dict)

    @property
    def matrix(self) -> np.ndarray:
        return self.te_result.matrix

    def get(self, method: str) -> Any:
        return self.inference_results[method]

    def __getattr__(self, name: str) -> Any:
        inf = self.__dict__.get("inference_results", {})
        if name in inf:
            return inf[name]
        raise AttributeError(f"{type(self).__name__!r} has no attribute {name!r}")


class Pipeline:
    """TE matrix (computed lazily, cached) + link inference on it."""

    def __init__(self, engine: TransferEntropyEngine | None = None, **defaults):
        self.engine = engine
        self._defaults = dict(defaults)
        self._te_result: TransferEntropyResult | None = None
        self._compute_kwargs: dict[str, Any] = {}
        self._data_fingerprint: tuple | None = None
        if engine is not None:
            self._data_fingerprint = self._fingerprint(engine._data, engine._variable_names,
                                                       engine._sources)

    @staticmethod
    def _fingerprint(data, variable_names, sources) -> tuple:
        def _key(arr):
            if arr is None:
                return None
            a = np.asarray(arr)
            return (a.ctypes.data, a.shape, str(a.dtype))
        return (_key(data), _key(variable_names), _key(sources))

    def configure(self, **kwargs) -> "Pipeline":
        """Keyword arguments for engine.compute(); a change drops the cached matrix."""
        changed = any(k not in self._compute_kwargs or self._compute_kwargs[k] != v
                      for k, v in kwargs.items())
        self._compute_kwargs.update(kwargs)
        if changed:
            self._te_result = None
        return self

    def _ensure_engine(self, data, variable_names, sources) -> None:
        if data is None:
            if self.engine is None:
                raise ValueError("Pipeline has no engine; pass data and variable_names to "
                                 "run() (or construct Pipeline with a pre-built engine).")
            return
        if variable_names is None:
            raise ValueError("variable_names is required when data is provided.")
        fp = self._fingerprint(data, variable_names, sources)
        if self.engine is not None and fp == self._data_fingerprint:
            return
        self.engine = TransferEntropyEngine(data=data, variable_names=variable_names,
                                            sources=sources)
        self._data_fingerprint = fp
        self._te_result = None

    @property
    def te_result(self) -> TransferEntropyResult:
        if self._te_result is None:
            self._te_result = self.engine.compute(**self._compute_kwargs)
        return self._te_result

    def clear_cache(self) -> None:
        self._te_result = None

    def infer(self, method: str, taus: list[int] | None = None, lag_combine: str = "max",
              **kwargs) -> Any:
        """One inference method on the cached TE matrix; with `taus`, one run per lag
        combined per pair (only the surrogate test)."""
        if taus is not None:
            return self._infer_multi_lag(taus=taus, combine=lag_combine,
                                         inference_method=method, **kwargs)
        from tenex_b200.inference import get_method
        params = {**self._defaults, **kwargs}
        method_obj = get_method(method)
        te = self.te_result
        device = params.pop("device", None)
        device = torch.device("cuda", 0) if device is None else torch.device(device)
        if method in _FUSED_METHODS:
            params.setdefault("bin_data", te.bin_arrs)
            params.setdefault("n_per_var", te.n_per_var)
            params.setdefault("b_max", te.b_max)
            params.setdefault("kernel", te.kernel)
            params.setdefault("tau", te.tau)
        sources = getattr(self.engine, "_sources", None)
        if sources is not None:
            params.setdefault("sources", sources)
        return method_obj.infer(te.matrix, te.variable_names, device, **params)

    def _infer_multi_lag(self, taus: list[int], combine: str = "max",
                         inference_method: str = "surrogate_test", **kwargs) -> Any:
        if not taus:
            raise ValueError("taus must be a non-empty list of time-lags")
        if combine not in ("adaptive_select", "weighted_sum", "max"):
            raise ValueError(f"combine must be 'adaptive_select', 'weighted_sum', or 'max' "
                             f"(got {combine!r})")
        if inference_method != "surrogate_test":
            raise NotImplementedError(f"multi_lag combine for {inference_method!r} is not "
                                      f"supported; only 'surrogate_test' is implemented")
        per_tau = []
        original_tau = self._compute_kwargs.get("tau", 1)
        for tau in taus:
            self.configure(tau=tau)
            self.clear_cache()
            _log.vprint(f"[TENEX] multi_lag: computing tau={tau}")
            per_tau.append(self.infer(inference_method, **kwargs))
        self.configure(tau=original_tau)
        device = kwargs.get("device")
        device = torch.device("cuda", 0) if device is None else torch.device(device)
        return self._combine_surrogate_multi_lag(per_tau, taus, combine,
                                                 variable_names=self.engine.variable_names,
                                                 device=device)

    @staticmethod
    def _combine_surrogate_multi_lag(results: list, taus: list[int], combine: str,
                                     variable_names, device):
        """Per-pair merge of per-lag SurrogateTestResults (the reference's rules and
        expressions, tenex/pipeline.py:316-410); BH on `device`."""
        from tenex_b200.inference.grn import bh_fdr_gpu, make_grn
        from tenex_b200.inference.surrogate_test import SurrogateTestResult
        n = results[0].observed_te.shape[0]
        variable_names = np.asarray(variable_names)
        K = len(taus)
        obs = np.stack([r.observed_te for r in results], axis=0)
        eff = np.stack([r.effective_te for r in results], axis=0)
        mean = np.stack([r.mean_surrogate_te for r in results], axis=0)
        std = np.stack([r.std_surrogate_te for r in results], axis=0)
        pv = np.stack([r.p_values for r in results], axis=0)

        def pick(idx):
            return [np.take_along_axis(a, idx, axis=0)[0] for a in (eff, obs, mean, std)]

        if combine == "max":
            effective, observed, mean_s, std_s = pick(np.argmax(eff, axis=0, keepdims=True))
        elif combine == "adaptive_select":
            effective, observed, mean_s, std_s = pick(np.argmin(pv, axis=0, keepdims=True))
        else:
            w = np.where(pv < 0.05, -np.log(pv + 1e-12), 0.0).astype(np.float32)
            if not np.any(w > 0):
                raise ValueError(f"weighted_sum: no pair passed p<0.05 at any lag in "
                                 f"taus={taus}; the combined result would be identically zero. "
                                 f"Loosen n_surrogates, add more lags, or switch to "
                                 f"combine='max'.")
            effective = np.sum(eff * w, axis=0)
            _, observed, mean_s, std_s = pick(np.argmin(pv, axis=0, keepdims=True))
        p_values = np.minimum(1.0, pv.min(axis=0) * K).astype(np.float32)
        np.fill_diagonal(p_values, 1.0)
        fdr = results[0].fdr
        off = ~np.eye(n, dtype=bool)
        adj = bh_fdr_gpu(torch.from_numpy(p_values[off]).to(device), alpha=fdr).cpu().numpy()
        sig = np.zeros((n, n), dtype=bool)
        sig[off] = adj < fdr
        sig &= effective > 0
        pairs = np.argwhere(sig).astype(np.int64)
        grn = make_grn(variable_names, pairs, effective[pairs[:, 0], pairs[:, 1]])
        _log.vprint(f"[TENEX] multi_lag ({combine}, taus={taus}): {len(grn)} significant "
                    f"edges (FDR<{fdr})")
        first = results[0]
        return SurrogateTestResult(observed_te=observed.astype(np.float32),
                                   mean_surrogate_te=mean_s.astype(np.float32),
                                   std_surrogate_te=std_s.astype(np.float32),
                                   effective_te=effective.astype(np.float32),
                                   p_values=p_values, grn=grn, n_surrogates=first.n_surrogates,
                                   shuffle_method=first.shuffle_method,
                                   block_length=first.block_length, p_method=first.p_method,
                                   fdr=fdr)

    def run(self, data=None, variable_names=None, sources=None, methods=None,
            method_kwargs=None, verbose: bool = False) -> PipelineResult:
        """TE matrix once, then each requested method on it."""
        _log.set_verbose(verbose)
        self._ensure_engine(data, variable_names, sources)
        methods = list(methods) if methods else ["surrogate_test"]
        method_kwargs = method_kwargs or {}
        out = PipelineResult(te_result=self.te_result)
        for m in methods:
            out.inference_results[m] = self.infer(m, **method_kwargs.get(m, {}))
        return out
