"""Pipeline: one TE matrix per set of compute arguments, link inference on it,
and the surrogate test across several time lags.

Public surface of the reference's tenex/pipeline.py (PipelineResult :44-77,
Pipeline :79-440): Pipeline(engine=None, **inference_defaults), configure(),
te_result, clear_cache(), infer(method, taus=None, lag_combine="max", ...) and
run(). Inference methods come from the registry ('surrogate_test', 'fdr');
CLR/ND/TRACE/POINT are not part of this package and raise NotImplementedError.

Design:
  * TE results are cached per frozen set of engine.compute() arguments, so
    configure() never has to invalidate anything and a lag sweep does not touch
    the configured run: a sweep computes each lag's matrix, runs the surrogate
    test on it and drops the matrix before the next lag (one n x n matrix alive
    at a time).
  * The per-lag results are merged per pair by merge_lag_results. Its rules and
    expressions are the reference's (tenex/pipeline.py:316-410), because the
    merged statistics must equal the reference's bit for bit: "max" keeps each
    pair's lag of largest effective TE, "adaptive_select" its lag of smallest p,
    "weighted_sum" sums effective TE with weights -ln(p + 1e-12) where p < 0.05
    (statistics of the smallest-p lag otherwise); every rule reports the
    Bonferroni p = min(1, K * min p), and edges are BH-FDR over the off-diagonal
    pairs with positive merged effective TE.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any

import numpy as np
import torch

from tenex_b200 import _log
from tenex_b200.result import TransferEntropyResult
from tenex_b200.transferentropy import TransferEntropyEngine

LAG_RULES = ("max", "adaptive_select", "weighted_sum")
# methods that read the bins of the TE run (the others use only the matrix)
_NEEDS_BINS = frozenset({"surrogate_test"})


@dataclass
class PipelineResult:
    """The TE result of a run() and each inference method's result by name."""

    te_result: TransferEntropyResult
    inference_results: dict[str, Any] = field(default_factory=dict)

    @property
    def matrix(self) -> np.ndarray:
        return self.te_result.matrix

    def get(self, method: str) -> Any:
        return self.inference_results[method]

    def __getattr__(self, name: str) -> Any:
        # pr.surrogate_test, pr.fdr, ...: the method results as attributes
        results = self.__dict__.get("inference_results", {})
        try:
            return results[name]
        except KeyError:
            raise AttributeError(f"PipelineResult has no method result or field {name!r}") \
                from None


def _as_device(device) -> torch.device:
    if device is None:
        return torch.device("cuda", 0)
    return device if isinstance(device, torch.device) else torch.device(device)


def _freeze(value) -> Any:
    """Hashable stand-in of a compute() argument (lists, dicts, arrays)."""
    if isinstance(value, dict):
        return tuple(sorted((k, _freeze(v)) for k, v in value.items()))
    if isinstance(value, (list, tuple)):
        return tuple(_freeze(v) for v in value)
    if isinstance(value, np.ndarray):
        return ("ndarray", value.shape, str(value.dtype), value.tobytes())
    return value


class Pipeline:
    """TE matrix (computed on first use and cached) plus link inference on it.

    engine   : an optional pre-built TransferEntropyEngine; without one, run()
               builds it from its data / variable_names / sources.
    defaults : inference keyword arguments used by every infer() call unless
               the call overrides them (e.g. fdr=0.05).
    """

    def __init__(self, engine: TransferEntropyEngine | None = None, **defaults):
        self.engine = engine
        self._defaults = dict(defaults)
        self._compute_args: dict[str, Any] = {}
        self._cache: dict[tuple, TransferEntropyResult] = {}

    # ---------------------------------------------------------------- TE runs
    def configure(self, **compute_args) -> "Pipeline":
        """Sets engine.compute() arguments (binning_method, tau, kernel, ...) for
        te_result and infer(); returns self so calls chain."""
        self._compute_args.update(compute_args)
        return self

    def _te(self, keep: bool = True, **override) -> TransferEntropyResult:
        if self.engine is None:
            raise ValueError("no data yet: call run(data=..., variable_names=...) or build the "
                             "Pipeline around a TransferEntropyEngine")
        args = {**self._compute_args, **override}
        key = _freeze(args)
        res = self._cache.get(key)
        if res is None:
            res = self.engine.compute(**args)
            if keep:
                self._cache[key] = res
        return res

    @property
    def te_result(self) -> TransferEntropyResult:
        """The TE result for the configured compute() arguments (cached)."""
        return self._te()

    def clear_cache(self) -> None:
        self._cache.clear()

    def _use_data(self, data, variable_names, sources) -> None:
        if data is None:
            if self.engine is None:
                raise ValueError("no data yet: call run(data=..., variable_names=...) or build "
                                 "the Pipeline around a TransferEntropyEngine")
            return
        if variable_names is None:
            raise ValueError("run(data=...) also needs variable_names (one per row of data)")
        e = self.engine
        if (e is not None and e._data is data and e._variable_names is variable_names
                and e._sources is sources):
            return                      # the engine already wraps these very arrays
        self.engine = TransferEntropyEngine(data=data, variable_names=variable_names,
                                            sources=sources)
        self._cache.clear()

    # -------------------------------------------------------------- inference
    def _run_method(self, te: TransferEntropyResult, method: str, kwargs: dict) -> Any:
        from tenex_b200.inference import get_method
        impl = get_method(method)
        params = {**self._defaults, **kwargs}
        device = _as_device(params.pop("device", None))
        if method in _NEEDS_BINS:
            for k, v in (("bin_data", te.bin_arrs), ("n_per_var", te.n_per_var),
                         ("b_max", te.b_max), ("kernel", te.kernel), ("tau", te.tau)):
                params.setdefault(k, v)
        if getattr(self.engine, "_sources", None) is not None:
            # BH and thresholds cover only the source-filtered pairs that were computed
            params.setdefault("sources", self.engine._sources)
        return impl.infer(te.matrix, te.variable_names, device, **params)

    def infer(self, method: str, taus: list[int] | None = None, lag_combine: str = "max",
              **kwargs) -> Any:
        """Runs one inference method on the TE matrix. With `taus`, the surrogate
        test runs once per lag on that lag's matrix and the results are merged per
        pair by `lag_combine` ("max", "adaptive_select" or "weighted_sum")."""
        if taus is None:
            return self._run_method(self._te(), method, kwargs)
        taus = [int(t) for t in taus]
        if not taus:
            raise ValueError("taus: give at least one lag")
        if lag_combine not in LAG_RULES:
            raise ValueError(f"lag_combine={lag_combine!r}: expected one of {LAG_RULES}")
        if method != "surrogate_test":
            raise NotImplementedError(f"lags can be merged for the surrogate test only, "
                                      f"not for {method!r}")
        per_lag = []
        for tau in taus:
            _log.vprint(f"[TENEX] lag sweep: tau={tau}")
            per_lag.append(self._run_method(self._te(keep=False, tau=tau), method, kwargs))
        return merge_lag_results(per_lag, taus, lag_combine, self.engine.variable_names,
                                 _as_device(kwargs.get("device")))

    def run(self, data=None, variable_names=None, sources=None, methods=None,
            method_kwargs=None, verbose: bool = False) -> PipelineResult:
        """TE matrix once (for the configured arguments), then every method in
        `methods` (default: the surrogate test) with its `method_kwargs` entry."""
        _log.set_verbose(verbose)
        self._use_data(data, variable_names, sources)
        per_method = method_kwargs or {}
        out = PipelineResult(te_result=self.te_result)
        for m in (list(methods) if methods else ["surrogate_test"]):
            out.inference_results[m] = self.infer(m, **per_method.get(m, {}))
        return out


def merge_lag_results(results: list, taus: list[int], rule: str, variable_names, device):
    """One SurrogateTestResult from per-lag ones (same pairs, lags `taus`).

    Each pair takes the statistics (observed, mean, std and, except for
    weighted_sum, effective TE) of one lag: its largest effective TE ("max") or
    its smallest p ("adaptive_select", "weighted_sum"); weighted_sum's effective
    TE is sum_k eff_k * w_k with w_k = -ln(p_k + 1e-12) for p_k < 0.05, else 0.
    p = min(1, K * min_k p_k) (Bonferroni over the K lags), 1 on the diagonal;
    edges: BH-FDR at the first result's fdr over the off-diagonal pairs (on
    `device`) and merged effective TE > 0. The float32 expressions are the
    reference's (tenex/pipeline.py:316-410), evaluated in numpy as there."""
    from tenex_b200.inference.grn import bh_fdr_gpu, make_grn
    from tenex_b200.inference.surrogate_test import SurrogateTestResult
    if rule not in LAG_RULES:
        raise ValueError(f"lag_combine={rule!r}: expected one of {LAG_RULES}")
    K = len(results)
    fields = ("effective_te", "observed_te", "mean_surrogate_te", "std_surrogate_te", "p_values")
    st = {f: np.stack([getattr(r, f) for r in results]) for f in fields}   # (K, n, n) each
    pv = st["p_values"]
    pick = (np.argmax(st["effective_te"], axis=0) if rule == "max"
            else np.argmin(pv, axis=0))[None]                               # (1, n, n) lag index
    merged = {f: np.take_along_axis(st[f], pick, axis=0)[0] for f in fields[:4]}
    if rule == "weighted_sum":
        w = np.where(pv < 0.05, -np.log(pv + 1e-12), 0.0).astype(np.float32)
        if not (w > 0).any():
            raise ValueError(f"weighted_sum over taus={list(taus)}: every pair has p >= 0.05 at "
                             f"every lag, so all weights are zero; use more surrogates or lags, "
                             f"or lag_combine='max'")
        merged["effective_te"] = np.sum(st["effective_te"] * w, axis=0)
    n = pv.shape[1]
    p = np.minimum(1.0, pv.min(axis=0) * K).astype(np.float32)
    np.fill_diagonal(p, 1.0)
    fdr = results[0].fdr
    off = ~np.eye(n, dtype=bool)
    adj = bh_fdr_gpu(torch.from_numpy(p[off]).to(device), alpha=fdr).cpu().numpy()
    keep = np.zeros((n, n), dtype=bool)
    keep[off] = adj < fdr
    eff = merged["effective_te"]
    edges = np.argwhere(keep & (eff > 0)).astype(np.int64)
    grn = make_grn(np.asarray(variable_names), edges, eff[edges[:, 0], edges[:, 1]])
    _log.vprint(f"[TENEX] lag merge '{rule}' over taus={list(taus)}: {len(grn)} edges at "
                f"FDR < {fdr}")
    r0 = results[0]
    return SurrogateTestResult(observed_te=merged["observed_te"].astype(np.float32),
                               mean_surrogate_te=merged["mean_surrogate_te"].astype(np.float32),
                               std_surrogate_te=merged["std_surrogate_te"].astype(np.float32),
                               effective_te=eff.astype(np.float32), p_values=p, grn=grn,
                               n_surrogates=r0.n_surrogates, shuffle_method=r0.shuffle_method,
                               block_length=r0.block_length, p_method=r0.p_method, fdr=fdr)
