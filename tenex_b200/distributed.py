"""Several GPUs: one process per GPU, the ordered-pair range split across ranks.

Pairs are independent, so the TE matrix and the surrogate statistics shard
without any exchange on the data path. The reference splits the pair-id range
[0, n(n-1)) into contiguous chunks of ceil(n(n-1) / n_gpus)
(tenex/transferentropy.py:376-379, 424-428) and runs one thread per GPU; here
each rank is its own process (torchrun, NCCL over NVLink), computes its chunk
with the single-GPU kernels, and the chunks are assembled by one collective:

  * bins + n_per_var: broadcast once from rank 0 (broadcast_bins);
  * results: each rank's chunk is a contiguous run of pair-free ids (target-
    major), so its values form one contiguous vector; an all-gather of the
    equal-sized (padded) chunks gives every rank the whole pair-free vector,
    which becomes the (n, n) [src, tgt] matrix with one on-device transpose.
    Each rank receives (world - 1) / world of the n(n-1) values: ~400 MB for
    the float32 TE of 10,000 genes (an all-reduce of zero-filled n x n
    matrices would move twice that). Values are copied, not summed, so the
    result is bit-identical to one GPU computing every pair;
  * surrogate statistics: the same all-gather of each rank's chunk of the
    float64 sum / sum of squares and the int32 count_ge.

No kernel here waits on another rank's memory; the only cross-GPU traffic is
the NCCL broadcast and all-gather. Under a gloo process group (CUDA broadcast
supported, CUDA all-gather not) the all-gather goes through host memory.
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


def pairfree_ids_to_cells(n: int, p0: int, p1: int, device) -> tuple[torch.Tensor, torch.Tensor]:
    """(src, tgt) of pair-free ids [p0, p1): p = tgt * (n - 1) + src_local,
    src = src_local + (src_local >= tgt)."""
    p = torch.arange(p0, p1, dtype=torch.int64, device=device)
    tgt = torch.div(p, n - 1, rounding_mode="floor")
    sl = p - tgt * (n - 1)
    return sl + (sl >= tgt).to(torch.int64), tgt


def pairfree_to_matrix(pf: torch.Tensor, n: int) -> torch.Tensor:
    """(n, n) [src, tgt] matrix (zero diagonal) from the full pair-free vector
    (n(n-1) values in target-major order), on pf's device. Target-major, the
    off-diagonal cells of row t are its sources in increasing order, and the
    n(n-1) off-diagonal cells of a row-major (n, n) matrix are exactly the cells
    after flat position 0 cut into n - 1 rows of n + 1 (the diagonal is the last
    of each), so the vector drops into place with one strided copy; the matrix
    is its transpose."""
    mt = torch.zeros((n, n), dtype=pf.dtype, device=pf.device)
    if n > 1:
        mt.view(-1)[1:].view(n - 1, n + 1)[:, :n].copy_(pf[:n * (n - 1)].view(n - 1, n))
    return mt.t().contiguous()


def gather_pairfree(local: torch.Tensor, n_pairs: int, group=None) -> torch.Tensor:
    """Every rank's contiguous chunk (pair_range) of a per-pair vector, all-gathered
    into the full (n_pairs,) vector on every rank. `local` holds this rank's
    p1 - p0 values."""
    world, rank = world_and_rank(group)
    p0, p1 = pair_range(n_pairs, rank, world)
    if local.numel() != p1 - p0:
        raise ValueError(f"rank {rank} holds {local.numel()} values for pair ids [{p0}, {p1})")
    if world == 1:
        return local
    chunk = pair_range(n_pairs, 0, world)[1]
    # NCCL gathers device tensors in place; gloo gathers host tensors only, so
    # with gloo the chunks go through host memory and the result comes back
    stage = local.is_cuda and dist.get_backend(group) != "nccl"
    where = torch.device("cpu") if stage else local.device
    send = torch.zeros(chunk, dtype=local.dtype, device=where)
    send[:p1 - p0] = local
    full = torch.empty(chunk * world, dtype=local.dtype, device=where)
    dist.all_gather_into_tensor(full, send, group=group)
    return full[:n_pairs].to(local.device) if stage else full[:n_pairs]


def assemble_matrices(*mats: torch.Tensor, group=None) -> None:
    """In place: (n, n) [src, tgt] matrices of which each rank filled only the
    cells of its own pair chunk become the full matrices on every rank (one
    all-gather of each rank's chunk per matrix; diagonals are left as they are)."""
    world, rank = world_and_rank(group)
    if world == 1:
        return
    for m in mats:
        n = int(m.shape[0])
        total = n * (n - 1)
        src, tgt = pairfree_ids_to_cells(n, *pair_range(total, rank, world), m.device)
        full = gather_pairfree(m[src, tgt].contiguous(), total, group)
        diag = torch.diagonal(m).clone()
        m.copy_(pairfree_to_matrix(full, n))
        torch.diagonal(m).copy_(diag)


def te_matrix_sharded(kernel, db, n_per_var: torch.Tensor, b_max: int, tau: int,
                      group=None) -> torch.Tensor:
    """(n, n) float32 TE matrix [src, tgt] on every rank: this rank's pair chunk
    as a pair-free vector from `kernel.compute_pairfree_device`, then one
    all-gather and the on-device transpose."""
    world, rank = world_and_rank(group)
    n = int(db.n)
    total = n * (n - 1)
    p0, p1 = pair_range(total, rank, world)
    dev = db.data.device
    local = torch.empty(p1 - p0, dtype=torch.float32, device=dev)
    if p1 > p0:
        kernel.compute_pairfree_device(db, n_per_var, b_max, tau, p0, p1 - p0, matrix=False,
                                       out=local)
    return pairfree_to_matrix(gather_pairfree(local, total, group), n)


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
    assemble_matrices(acc.sum, acc.sumsq, acc.cnt, group=group)
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
