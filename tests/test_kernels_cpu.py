"""Host-side contracts of the kernel plugin API (no GPU)."""
import numpy as np
import pytest
import torch

from tenex_b200.kernels import get_kernel
from tenex_b200.kernels.pair_list import item_table


def _item_table_loop(t, run):
    P = len(t)
    if P == 0:
        return np.zeros(1, np.int64)
    change = np.flatnonzero(np.diff(t)) + 1
    starts = np.concatenate([[0], change, [P]])
    out = []
    for a, b in zip(starts[:-1], starts[1:]):
        out.extend(range(int(a), int(b), run))
    out.append(P)
    return np.asarray(out, np.int64)


def test_item_table_runs():
    rng = np.random.default_rng(0)
    for _ in range(200):
        t = np.sort(rng.integers(0, rng.integers(1, 40), rng.integers(0, 600)))
        run = int(rng.integers(1, 70))
        assert np.array_equal(item_table(t, run), _item_table_loop(t, run))


def test_batch_size_hooks_and_multi_device_contracts():
    k = get_kernel("Full-SMEM")
    cpu_bins = torch.zeros((4, 100, 1), dtype=torch.uint8)
    assert k.heuristic_batch_size(cpu_bins, 4) == 2048
    assert k.peak_bytes_per_pair(4, 100, 1) == 20
    with pytest.raises(ValueError):
        k.compute_multi_gpu(cpu_bins, np.zeros((3, 2), np.int64), 4, torch.ones(4), 1, None, [])
    with pytest.raises(NotImplementedError):
        k.compute_matrix_multi_gpu(cpu_bins, 4, 1, [0])
    with pytest.raises(ValueError):
        get_kernel("GEMM-B2").compute_matrix_multi_gpu(cpu_bins, 4, 1, [])


def test_host_copy_helpers_without_cuda():
    """to_device / to_host keep shape, dtype and values on a CPU target (the
    staging path is CUDA-only and is covered by the GPU tests)."""
    from tenex_b200.kernels import device as D
    a = np.arange(24, dtype=np.int16).reshape(4, 6)
    t = D.to_device(a, "cpu")
    assert t.dtype == torch.int16 and torch.equal(t, torch.as_tensor(a))
    assert np.array_equal(D.to_host(t), a)


def test_all_finite_matches_numpy():
    from tenex_b200.kernels import device as D
    x = np.random.default_rng(3).standard_normal((700, 20_000)).astype(np.float32)
    assert D.all_finite(x)
    for bad in (np.nan, np.inf, -np.inf):
        y = x.copy()
        y[699, 19_998] = bad
        assert not D.all_finite(y) and not np.isfinite(y).all()
    assert not D.all_finite(y[:, ::2]) and D.all_finite(x[:, ::2])  # non-contiguous
