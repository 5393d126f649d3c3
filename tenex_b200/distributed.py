"""Several GPUs: one process per GPU, the ordered-pair range split across ranks.

Pairs are independent, so the TE matrix and the surrogate statistics shard
without any exchange on the data path. The reference splits the pair-id range
[0, n(n-1)) into contiguous chunks of ceil(n(n-1) / n_gpus)
(tenex/transferentropy.py:376-379, 424-428) and runs one thread per GPU; here
each rank is its own process (torchrun, NCCL over NVLink), computes its chunk
with the single-GPU kernels, and the chunks are combined by one collective:

  * bins + n_per_var: broadcast once from rank 0 (broadcast_bins);
  * TE matrix: each rank fills its pairs of a zeroed (n, n) float32 matrix and
    an all-reduce SUM assembles it (the supports are disjoint, and x + 0 is
    exact, so the result is bit-identical to one GPU computing every pair);
  * surrogate statistics: the same all-reduce over the float64 sum / sum of
    squares and the int32 count_ge of each rank's pairs.

No kernel here waits on another rank's memory; the only cross-GPU traffic is
the NCCL broadcast and all-reduce.
"""
from __future__ import annotations

import math

import numpy as np
import torch
import torch.distributed as dist


def world_and_rank(group=None) -> tuple[int, int]:
    if not (dist.is_available() and dist.is_initialized()):
        return 1, 0
    return dist.get_world_size(group), dist.get_rank(group)


def pair_range(n_pairs: int, rank: int, world: int) -> tuple[int, int]:
    """[p0, p1) of rank's contiguous chunk, chunk = ceil(n_pairs / world) (the
    reference's split); trailing ranks may get an empty range."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside world of {world}")
    chunk = math.ceil(n_pairs / world) if n_pairs > 0 else 0
    p0 = min(rank * chunk, n_pairs)
    return p0, min(p0 + chunk, n_pairs)


def broadcast_bins(bins: torch.Tensor | None, n_per_var: torch.Tensor | None, device,
                   src: int = 0, group=None) -> tuple[torch.Tensor, torch.Tensor]:
    """Rank `src` sends its uint8 (n, T, K) bins and int32 n_per_var; every rank
    returns its own copies on `device` (one shape broadcast + two data
    broadcasts)."""
    world, rank = world_and_rank(group)
    if rank == src:
        if bins is None or n_per_var is None:
            raise ValueError("the source rank must pass bins and n_per_var")
        b = bins.to(device=device, dtype=torch.uint8)
        if b.dim() == 2:
            b = b.unsqueeze(-1)
        b = b.contiguous()
        npv = n_per_var.to(device=device, dtype=torch.int32).contiguous()
        shape = torch.tensor(list(b.shape), dtype=torch.int64, device=device)
    else:
        shape = torch.zeros(3, dtype=torch.int64, device=device)
    if world == 1:
        return b, npv
    dist.broadcast(shape, src, group=group)
    n, T, K = (int(v) for v in shape.tolist())
    if rank != src:
        b = torch.empty((n, T, K), dtype=torch.uint8, device=device)
        npv = torch.empty(n, dtype=torch.int32, device=device)
    dist.broadcast(b, src, group=group)
    dist.broadcast(npv, src, group=group)
    return b, npv


def combine_disjoint(*tensors: torch.Tensor, group=None) -> None:
    """In-place all-reduce SUM of per-rank results whose non-zero entries are
    disjoint across ranks (exact for float and integer types)."""
    world, _ = world_and_rank(group)
    if world == 1:
        return
    for t in tensors:
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)


def te_matrix_sharded(kernel, db, n_per_var: torch.Tensor, b_max: int, tau: int,
                      group=None) -> torch.Tensor:
    """(n, n) float32 TE matrix [src, tgt] on every rank: this rank's pair chunk
    from `kernel.compute_pairfree_device`, then combine_disjoint."""
    world, rank = world_and_rank(group)
    n = int(db.n)
    p0, p1 = pair_range(n * (n - 1), rank, world)
    dev = db.data.device
    out = torch.zeros((n, n), dtype=torch.float32, device=dev)
    if p1 > p0:
        kernel.compute_pairfree_device(db, n_per_var, b_max, tau, p0, p1 - p0, matrix=True,
                                       out=out)
    combine_disjoint(out, group=group)
    return out


def surrogate_sharded(db, n_per_var: torch.Tensor, b_max: int, tau: int, observed: torch.Tensor,
                      perms: torch.Tensor, block_length: int, cfg=None, use_graph: bool = False,
                      group=None):
    """Surrogate sum / sum of squares / count_ge ((n, n) device tensors, all
    pairs) with each rank running every surrogate on its own pair chunk."""
    from tenex_b200.inference.surrogate_test import SurrogateAccumulator, run_surrogates
    world, rank = world_and_rank(group)
    n = int(db.n)
    p0, p1 = pair_range(n * (n - 1), rank, world)
    acc = SurrogateAccumulator(db, n_per_var, b_max, tau, observed, False, cfg, p0, p1 - p0)
    if p1 > p0:
        run_surrogates(acc, perms, block_length, use_graph)
    combine_disjoint(acc.sum, acc.sumsq, acc.cnt, group=group)
    return acc.sum, acc.sumsq, acc.cnt


def pairfree_chunk_to_matrix(values: np.ndarray, n: int, p0: int) -> np.ndarray:
    """Host helper: place pair-free values of ids [p0, p0 + len) into a zeroed
    (n, n) [src, tgt] matrix (pair id p = tgt * (n - 1) + src_local)."""
    m = np.zeros((n, n), dtype=np.float32)
    p = np.arange(p0, p0 + len(values), dtype=np.int64)
    tgt = p // (n - 1)
    sl = p % (n - 1)
    src = sl + (sl >= tgt)
    m[src, tgt] = values
    return m
