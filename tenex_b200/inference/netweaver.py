"""NetWeaver (reference: tenex/inference/netweaver.py:21-165): wraps a TE result
and dispatches infer(method=...), auto-filling the surrogate test's bin_data,
n_per_var, b_max, kernel and tau from a TransferEntropyResult."""
from __future__ import annotations

import numpy as np
import torch

from tenex_b200 import _log


class NetWeaver:
    def __init__(self, result, sources=None, fdr: float = 0.01, links: int = 0,
                 is_trimming: bool = True, trim_threshold: float = 0.0):
        from tenex_b200.result import TransferEntropyResult
        if isinstance(result, TransferEntropyResult):
            self.result_matrix = result.matrix
            self.variable_names = result.variable_names
            self.bin_arrs = result.bin_arrs
            self.n_per_var = result.n_per_var
            self.b_max = result.b_max
            self.kernel = result.kernel
            self.tau = result.tau
        elif isinstance(result, tuple) and len(result) == 2:
            self.result_matrix = np.asarray(result[0], dtype=np.float32)
            self.variable_names = np.asarray(result[1])
            self.bin_arrs = self.n_per_var = self.b_max = self.kernel = None
            self.tau = 1
        else:
            raise TypeError("result must be a TransferEntropyResult or "
                            "(matrix, variable_names) tuple")
        self.sources = sources if sources is not None else getattr(result, "sources", None)
        self.fdr = fdr
        self.links = links
        self.is_trimming = is_trimming
        self.trim_threshold = trim_threshold

    def infer(self, method: str = "fdr", device=None, verbose: bool = False, **kwargs):
        """'fdr' -> GRN, or (GRN, trimmed GRN) with trimming; 'surrogate_test' ->
        SurrogateTestResult (tenex/inference/netweaver.py:77-165)."""
        from tenex_b200.inference import get_method
        _log.set_verbose(verbose)
        dev = torch.device(device) if device is not None else torch.device("cuda", 0)
        m = get_method(method)
        params = dict(fdr=self.fdr, links=self.links, sources=self.sources,
                      is_trimming=self.is_trimming, trim_threshold=self.trim_threshold)
        if method == "surrogate_test":
            for drop in ("links", "is_trimming", "trim_threshold"):
                params.pop(drop)
            if "bin_data" not in kwargs and self.bin_arrs is not None:
                params["bin_data"] = self.bin_arrs
            if "n_per_var" not in kwargs and self.n_per_var is not None:
                params["n_per_var"] = self.n_per_var
            if "b_max" not in kwargs and self.b_max is not None:
                params["b_max"] = self.b_max
            if "kernel" not in kwargs and self.kernel:
                params["kernel"] = self.kernel
            if "tau" not in kwargs:
                params["tau"] = self.tau
        params.update(kwargs)
        return m.infer(self.result_matrix, self.variable_names, dev, **params)
