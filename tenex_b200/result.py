"""TransferEntropyResult (reference: tenex/result.py:12-105), same fields and
numpy-compatibility behaviour."""
from __future__ import annotations

import numpy as np


class TransferEntropyResult:
    """(n, n) float32 TE matrix ([i, j] = TE(i -> j)) with run metadata:
    variable_names, bin_arrs (n, T, K), n_per_var, b_max, tau, kernel, timings,
    sources."""

    __slots__ = ("matrix", "variable_names", "bin_arrs", "n_per_var", "b_max", "tau", "kernel",
                 "timings", "sources")

    def __init__(self, matrix: np.ndarray, variable_names: np.ndarray,
                 bin_arrs: np.ndarray | None = None, n_per_var: np.ndarray | None = None,
                 b_max: int = 0, tau: int = 1, kernel: str = "", timings: dict | None = None,
                 sources: np.ndarray | None = None):
        self.matrix = matrix
        self.variable_names = np.asarray(variable_names)
        self.bin_arrs = bin_arrs
        self.n_per_var = n_per_var
        self.b_max = b_max
        self.tau = tau
        self.kernel = kernel
        self.timings = timings
        self.sources = sources

    def __array__(self, dtype=None, copy=None):
        arr = self.matrix if dtype is None else self.matrix.astype(dtype)
        return arr.copy() if copy else arr

    def __getitem__(self, key):
        return self.matrix[key]

    @property
    def shape(self):
        return self.matrix.shape

    @property
    def dtype(self):
        return self.matrix.dtype

    @property
    def ndim(self):
        return self.matrix.ndim

    @property
    def size(self):
        return self.matrix.size

    @property
    def T(self):
        return self.matrix.T

    def __len__(self):
        return len(self.matrix)

    @property
    def n_vars(self) -> int:
        return self.matrix.shape[0]

    def __repr__(self):
        return (f"TransferEntropyResult(n_vars={self.n_vars}, kernel='{self.kernel}', "
                f"tau={self.tau}, b_max={self.b_max})")
