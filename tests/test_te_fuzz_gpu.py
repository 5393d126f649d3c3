"""Seeded random configurations of the TE kernels against the oracle.

Each case draws its own gene count, series length, per-gene bin counts
(constant genes included), skew, lag tau, samples per cell K, launch shape
(threads, sources per work item) and pair-id range, so the kernel's item
carving, slot sizes, 16/32-bit counters, ragged tails and output modes meet
shapes no hand-written case lists. Counts are compared cell by cell on a few
pairs per case, TE on every pair of the range (<= 1e-6 of the float64 oracle),
and the matrix output against the pair-free one. Binary cases also go through
GEMM-B2 at a random target-tile width.
"""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200.kernels import device as D
from tenex_b200.kernels.gemm_b2 import TILE_N, te_binary_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _case(seed):
    rng = np.random.default_rng(9000 + seed)
    n = int(rng.integers(2, 41))
    K = int(rng.choice([1, 1, 1, 2]))
    tau = int(rng.choice([1, 1, 2, 3]))
    T = int(rng.integers(tau + 2, 2500))
    b_hi = int(rng.choice([2, 4, 9, 16, 24, 38]))
    b = rng.integers(1, b_hi + 1, n)
    skew = bool(rng.random() < 0.5)
    rows = []
    for bb in b:
        p = rng.dirichlet(np.full(int(bb), 0.3 if skew else 3.0))
        rows.append(rng.choice(int(bb), size=T * K, p=p))
    x = np.stack(rows).astype(np.int32)
    rem, npv, bmax = O.remap(x)
    bins = rem.reshape(n, T, K)
    total = n * (n - 1)
    p0 = int(rng.integers(0, total))
    cnt = int(rng.integers(1, total - p0 + 1))
    cfg = dict(threads=int(rng.choice([128, 256, 512, 1024])),
               src_chunk=int(rng.choice([0, 1, 7, 64, 512])))
    return dict(bins=bins, npv=npv, bmax=bmax, tau=tau, p0=p0, cnt=cnt, cfg=cfg, n=n)


@pytest.mark.parametrize("seed", range(24))
def test_random_configuration(cuda, seed):
    c = _case(seed)
    bins, npv, bmax, tau, n = c["bins"], c["npv"], c["bmax"], c["tau"], c["n"]
    db = D.pack_bins(bins, cuda)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=cuda)
    te = D.te_pairfree(db, npv_t, bmax, tau=tau, pair_offset=c["p0"], n_pairs=c["cnt"],
                       cfg=c["cfg"]).cpu().numpy()
    ref = O.te_pairfree(bins, npv, tau, c["p0"], c["cnt"])
    assert np.max(np.abs(te.astype(np.float64) - ref)) <= TOL, c["cfg"]
    # raw counts of the first pairs of the range (at most 16), cell by cell
    nc = min(c["cnt"], 16)
    stride = bmax ** 3
    counts = torch.full((nc, stride), -1, dtype=torch.int32, device=cuda)
    D.te_pairfree(db, npv_t, bmax, tau=tau, pair_offset=c["p0"], n_pairs=nc, cfg=c["cfg"],
                  counts=counts, counts_stride=stride)
    cnt = counts.cpu().numpy()
    for k in range(nc):
        p = c["p0"] + k
        t, sl = divmod(p, n - 1)
        s = sl + (sl >= t)
        rc = O.counts(bins, tau, t, s, npv).reshape(-1)
        assert np.array_equal(cnt[k, :rc.size], rc), (seed, p, t, s)
    # the matrix output holds the same values at [src, tgt]
    m = D.te_pairfree(db, npv_t, bmax, tau=tau, pair_offset=c["p0"], n_pairs=c["cnt"],
                      matrix=True, cfg=c["cfg"]).cpu().numpy()
    ids = np.arange(c["p0"], c["p0"] + c["cnt"])
    t, sl = np.divmod(ids, n - 1)
    s = sl + (sl >= t)
    assert np.array_equal(m[s, t].view(np.uint32), te.view(np.uint32))


@pytest.mark.parametrize("seed", range(8))
def test_random_binary_configuration(cuda, seed):
    rng = np.random.default_rng(9500 + seed)
    n = int(rng.integers(2, 300))
    tau = int(rng.choice([1, 2, 3]))
    T = int(rng.integers(tau + 2, 3000))
    rate = rng.uniform(0.02, 0.6, n)[:, None]
    x = (rng.random((n, T)) < rate).astype(np.uint8)
    x[rng.random(n) < 0.05] = 0                       # a few constant genes
    tn = int(rng.choice(TILE_N))
    form = str(rng.choice(["fp4", "int8"]))
    m = te_binary_matrix(D.pack_bins(x, cuda), tau, operands=form, tile_n=tn).cpu().numpy()
    ref = O.te_matrix(x.astype(np.int32), np.full(n, 2, np.int32), tau=tau)
    assert np.all(np.diag(m) == 0)
    assert np.max(np.abs(m.astype(np.float64) - ref)) <= TOL, (n, T, tau, tn, form)
