"""The multi-rank path of tenex_b200.distributed with the CUDA kernels: two
processes on one GPU in a gloo process group. Each rank runs the TE kernel on its
own chunk of the pair-id range (the ranks' kernels never wait on one another; the
broadcast and all-gather go through gloo). The assembled results must equal, bit
for bit, the same per-rank launches made in one process and placed by pair id,
for the TE matrix (te_matrix_sharded) and the surrogate sums, sums of squares and
counts (surrogate_sharded); and one launch over every pair within 1e-6 (TE) and
1e-5 (sums of six surrogates): a rank's share of a target can carve that target's
shared memory for a different largest source bin count, which may change the
float32 summation order of its entropy terms."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out_dir):
    import datetime

    from tenex_b200 import distributed as TD
    from tenex_b200 import workloads as W
    from tenex_b200.inference.surrogate_test import (SurrogateAccumulator, build_block_perm,
                                                     run_surrogates)
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.full_smem import FullSMEMKernel

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    status = "ok"
    try:
        dev = torch.device("cuda:0")
        torch.cuda.set_device(dev)
        x, npv, _ = W.cfg5_bins(61, 1500, seed=2201)
        b, p = TD.broadcast_bins(torch.from_numpy(x) if rank == 0 else None,
                                 torch.from_numpy(npv) if rank == 0 else None, dev)
        assert b.is_cuda and np.array_equal(b[..., 0].cpu().numpy(), x)
        db = D.pack_bins(b, dev)
        bmax = int(npv.max())
        n = x.shape[0]
        kern = FullSMEMKernel()
        total = n * (n - 1)
        ranges = [TD.pair_range(total, r, world) for r in range(world)]
        m = TD.te_matrix_sharded(kern, db, p, bmax, 1)
        # the same per-rank launches made in this process and placed by pair id
        chunks = []
        for a, e in ranges:
            out = torch.empty(e - a, dtype=torch.float32, device=dev)
            kern.compute_pairfree_device(db, p, bmax, 1, a, e - a, matrix=False, out=out)
            chunks.append(out)
        here = TD.pairfree_to_matrix(torch.cat(chunks), n)
        one = kern.compute_pairfree_device(db, p, bmax, 1, 0, total, matrix=True)
        torch.cuda.synchronize()
        assert m.is_cuda and torch.equal(m, here), "assembled TE matrix differs"
        assert float((m - one).abs().max()) <= 1e-6, "TE differs from one launch"
        perms, bl, _ = build_block_perm(n, x.shape[1], "block", 30, 0, 6, 11, dev)
        s, q, c = TD.surrogate_sharded(db, p, bmax, 1, one, perms, bl)
        accs = []
        for a, e in ranges:
            acc = SurrogateAccumulator(db, p, bmax, 1, one, False, None, a, e - a)
            run_surrogates(acc, perms, bl, False)
            accs.append(acc)
        full = SurrogateAccumulator(db, p, bmax, 1, one, False, None, 0, total)
        run_surrogates(full, perms, bl, False)
        torch.cuda.synchronize()
        off = ~torch.eye(n, dtype=torch.bool, device=dev)
        # each accumulator holds only its own range's cells (zeros elsewhere)
        assert torch.equal(s[off], (accs[0].sum + accs[1].sum)[off]), "sums differ"
        assert torch.equal(q[off], (accs[0].sumsq + accs[1].sumsq)[off]), "sums of squares differ"
        assert torch.equal(c[off], (accs[0].cnt + accs[1].cnt)[off]), "counts differ"
        assert float((s - full.sum)[off].abs().max()) <= 1e-5, "sums differ from one launch"
    except Exception as e:  # reported through the file, the parent asserts
        status = f"{type(e).__name__}: {e}"
    finally:
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(status)
        dist.destroy_process_group()


def test_two_ranks_on_one_gpu_match_one_process(cuda, tmp_path):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    for r in range(world):
        assert (tmp_path / f"rank{r}.txt").read_text() == "ok", r
