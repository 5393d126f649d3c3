"""Multi-rank host logic of tenex_b200.distributed on CPU (gloo, world size 2 and 3).

The per-rank TE of a pair chunk comes from an oracle-backed stand-in kernel
defined here (the GPU kernel cannot run without a GPU); what is under test is
the split of the pair-id range, the bins broadcast and the exact assembly of
the per-rank chunks by all-gather (bit-identical to one rank computing all)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from oracle import oracle as O
from tenex_b200 import distributed as TD


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class _OracleDB:
    """The fields te_matrix_sharded reads from DeviceBins, over host bins."""

    def __init__(self, bins: np.ndarray):
        self.bins = bins
        self.n = bins.shape[0]
        self.data = torch.from_numpy(bins.reshape(self.n, -1))


class _OracleKernel:
    calls = []

    def compute_pairfree_device(self, db, npv, b_max, tau, pair_offset, n_pairs, matrix, out):
        vals = O.te_pairfree(db.bins, npv.numpy(), tau, pair_offset, n_pairs).astype(np.float32)
        assert not matrix and out.numel() == n_pairs
        out.copy_(torch.from_numpy(vals))
        self.calls.append((pair_offset, n_pairs))
        return out


def _data(n=13, T=300, seed=4):
    rng = np.random.default_rng(seed)
    npv = rng.integers(2, 7, n).astype(np.int32)
    bins = (rng.random((n, T)) * npv[:, None]).astype(np.uint8)
    return bins, npv


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        bins, npv = _data()
        n = bins.shape[0]
        # broadcast: only rank 0 holds the data
        b, p = TD.broadcast_bins(torch.from_numpy(bins) if rank == 0 else None,
                                 torch.from_numpy(npv) if rank == 0 else None, "cpu")
        assert b.shape == (n, bins.shape[1], 1)
        assert np.array_equal(b[..., 0].numpy(), bins) and np.array_equal(p.numpy(), npv)
        # sharded TE matrix
        k = _OracleKernel()
        m = TD.te_matrix_sharded(k, _OracleDB(b[..., 0].numpy()), p, int(npv.max()), 1)
        ref = O.te_matrix(bins, npv, 1).astype(np.float32)   # [src, tgt]
        assert np.array_equal(m.numpy(), ref)
        p0, p1 = TD.pair_range(n * (n - 1), rank, world)
        assert k.calls == ([(p0, p1 - p0)] if p1 > p0 else [])
        # disjoint float64 / int32 statistics combine exactly
        rng = np.random.default_rng(rank)
        s = torch.zeros((n, n), dtype=torch.float64)
        c = torch.zeros((n, n), dtype=torch.int32)
        full_s = np.zeros((n, n))
        full_c = np.zeros((n, n), np.int32)
        for r in range(world):
            q0, q1 = TD.pair_range(n * (n - 1), r, world)
            vals = np.random.default_rng(100 + r).random(q1 - q0) * 1e-3
            mm = TD.pairfree_chunk_to_matrix(vals.astype(np.float32), n, q0).astype(np.float64)
            full_s += mm
            full_c += (mm > 5e-4).astype(np.int32)
            if r == rank:
                s += torch.from_numpy(mm)
                c += torch.from_numpy((mm > 5e-4).astype(np.int32))
        TD.assemble_matrices(s, c)
        assert np.array_equal(s.numpy(), full_s) and np.array_equal(c.numpy(), full_c)
        with open(os.path.join(out_dir, f"ok{rank}"), "w") as f:
            f.write("ok")
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_te_and_stats_gloo(tmp_path, world):
    O.build()
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    for r in range(world):
        assert (tmp_path / f"ok{r}").read_text() == "ok"


def test_pair_range_matches_reference_split():
    # chunk = ceil(n_pairs / n_gpus), offset = rank * chunk (tenex/transferentropy.py:378,424)
    for n_pairs, world in [(99_990_000, 8), (10, 3), (2, 3), (7, 7), (0, 2), (5, 1)]:
        chunk = -(-n_pairs // world)
        got = [TD.pair_range(n_pairs, r, world) for r in range(world)]
        assert got[0][0] == 0 and got[-1][1] == n_pairs
        for r, (p0, p1) in enumerate(got):
            assert p0 == min(r * chunk, n_pairs)
            assert p1 - p0 == max(0, min(chunk, n_pairs - r * chunk))
        assert all(a[1] == b[0] for a, b in zip(got, got[1:]))
    with pytest.raises(ValueError):
        TD.pair_range(10, 2, 2)


def test_chunk_to_matrix_layout():
    n = 5
    vals = np.arange(n * (n - 1), dtype=np.float32) + 1
    m = TD.pairfree_chunk_to_matrix(vals, n, 0)
    assert np.array_equal(m, O.pairfree_to_matrix(vals, n).astype(np.float32))


@pytest.mark.parametrize("n", [2, 3, 7, 40])
def test_pairfree_to_matrix_on_device_layout(n):
    vals = torch.arange(n * (n - 1), dtype=torch.float32) + 1
    m = TD.pairfree_to_matrix(vals, n)
    assert np.array_equal(m.numpy(), O.pairfree_to_matrix(vals.numpy(), n).astype(np.float32))
    src, tgt = TD.pairfree_ids_to_cells(n, 0, n * (n - 1), "cpu")
    assert torch.equal(m[src, tgt], vals)
