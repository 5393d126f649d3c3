"""CUDA multi-bin TE kernel against the oracle: counts bit-exact, TE <= 1e-6."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200.kernels import device as D
from tenex_b200 import native

pytestmark = pytest.mark.gpu
TOL = 1e-6  # absolute TE tolerance against the float64 oracle


def _rand_bins(rng, n, T, b_lo, b_hi, K=1):
    b = rng.integers(b_lo, b_hi + 1, n)
    x = np.stack([rng.integers(0, bb, T * K) for bb in b]).astype(np.int32)
    rem, npv, bmax = O.remap(x)
    return rem.reshape(n, T, K), npv, bmax


def _gpu_te(bins, npv, bmax, cuda, tau=1, **kw):
    db = D.pack_bins(bins, cuda)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=cuda)
    out = D.te_pairfree(db, npv_t, bmax, tau=tau, **kw)
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("threads", [128, 512])
@pytest.mark.parametrize("b_lo,b_hi,T", [(1, 4, 300), (2, 12, 1000), (2, 32, 700),
                                         (17, 38, 400), (2, 16, 3000), (1, 2, 500)])
def test_counts_bitexact_and_te(cuda, b_lo, b_hi, T, threads):
    rng = np.random.default_rng(b_hi * 100 + T)
    n = 9
    bins, npv, bmax = _rand_bins(rng, n, T, b_lo, b_hi)
    P = n * (n - 1)
    stride = bmax ** 3
    counts = torch.full((P, stride), -1, dtype=torch.int32, device=cuda)
    te = _gpu_te(bins, npv, bmax, cuda, counts=counts, counts_stride=stride,
                 cfg=dict(threads=threads)).cpu().numpy()
    cnt = counts.cpu().numpy()
    for p in range(P):
        t, sl = divmod(p, n - 1)
        s = sl + (sl >= t)
        ref = O.counts(bins, 1, t, s, npv).reshape(-1)
        assert np.array_equal(cnt[p, :ref.size], ref), (p, t, s)
    ref_te = O.te_pairfree(bins, npv)
    assert np.max(np.abs(te - ref_te)) <= TOL


def _check_all_counts(cnt, bins, npv, n):
    for p in range(n * (n - 1)):
        t, sl = divmod(p, n - 1)
        s = sl + (sl >= t)
        ref = O.counts(bins, 1, t, s, npv).reshape(-1)
        assert np.array_equal(cnt[p, :ref.size], ref), (p, t, s)


@pytest.mark.parametrize("threads", [512, 1024])
def test_series_longer_than_shared_memory(cuda, threads):
    """150,000 samples with b up to 38: the target's states (300 KB as u16) are
    staged in tiles; pairs of two 38-bin genes (54,872 32-bit cells) run in the
    global-memory launch. Counts bit-exact for all 30 pairs, TE within 1e-6."""
    rng = np.random.default_rng(150_000)
    bvals = [38, 5, 17, 2, 38, 11]
    n, T = len(bvals), 150_000
    x = np.stack([rng.integers(0, b, T) for b in bvals]).astype(np.int32)
    x[2, 1:] = np.minimum(x[0, :-1] // 2, 16)       # a coupled pair
    bins, npv, bmax = O.remap(x)
    bins = bins.reshape(n, T, 1)
    stride = bmax ** 3
    counts = torch.full((n * (n - 1), stride), -1, dtype=torch.int32, device=cuda)
    te = _gpu_te(bins, npv, bmax, cuda, counts=counts, counts_stride=stride,
                 cfg=dict(threads=threads)).cpu().numpy()
    _check_all_counts(counts.cpu().numpy(), bins, npv, n)
    assert np.max(np.abs(te - O.te_pairfree(bins, npv))) <= TOL


def test_long_series_every_output_mode(cuda):
    """The sample-tiled staging (series past 65,536 u8 states) behind every output
    mode: pair-free ids with tau = 2 and K = 2, the matrix, an explicit pair list
    (the source filter) and the surrogate statistics epilogue, against the oracle."""
    from tenex_b200.kernels.pair_list import te_pair_list
    rng = np.random.default_rng(70_001)
    bins, npv, bmax = _rand_bins(rng, 7, 40_003, 2, 9, K=2)      # row_len 80,006 u8 states
    te = _gpu_te(bins, npv, bmax, cuda, tau=2).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(bins, npv, tau=2))) <= TOL
    db = D.pack_bins(bins, cuda)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=cuda)
    m = D.te_pairfree(db, npv_t, bmax, tau=1, matrix=True).cpu().numpy()
    assert np.max(np.abs(m - O.te_matrix(bins, npv))) <= TOL
    pairs = np.array([[0, 3], [0, 5], [2, 1], [6, 0], [6, 2], [6, 4]], np.int64)
    got = te_pair_list(db, npv_t, bmax, 1, pairs).cpu().numpy()
    assert np.max(np.abs(got - O.te_pairs(bins, npv, pairs))) <= TOL
    # surrogate statistics: one accumulation of the observed bins themselves adds
    # TE into the sums and counts TE >= observed (all ties)
    n = 7
    obs = torch.as_tensor(m, device=cuda)
    ssum = torch.zeros((n, n), dtype=torch.float64, device=cuda)
    ssq = torch.zeros_like(ssum)
    cnt = torch.zeros((n, n), dtype=torch.int32, device=cuda)
    D.surrogate_accumulate(db, npv_t, bmax, 1, obs, ssum, ssq, cnt)
    torch.cuda.synchronize()
    off = ~np.eye(n, dtype=bool)
    assert np.max(np.abs(ssum.cpu().numpy()[off] - m[off])) <= TOL
    assert np.all(cnt.cpu().numpy()[off] == 1)


def test_series_of_2_pow_24_samples(cuda):
    """N = 2^24 + 40 samples (beyond float32's exact integers): 32-bit counters,
    float64 entropy pass. Counts bit-exact, TE within 1e-6 of the oracle."""
    rng = np.random.default_rng(24)
    T = (1 << 24) + 41
    bvals = [2, 5, 3]
    x = np.stack([rng.integers(0, b, T, dtype=np.int32) for b in bvals])
    x[1, 1:] = np.where(rng.random(T - 1) < 0.3, x[0, :-1], x[1, 1:])  # coupling
    npv = np.array(bvals, np.int32)
    bins = x.astype(np.uint8).reshape(3, T, 1)
    stride = 5 ** 3
    counts = torch.full((6, stride), -1, dtype=torch.int32, device=cuda)
    te = _gpu_te(bins, npv, 5, cuda, counts=counts, counts_stride=stride).cpu().numpy()
    _check_all_counts(counts.cpu().numpy(), bins, npv, 3)
    ref = O.te_pairfree(bins, npv)
    assert np.max(np.abs(te - ref)) <= TOL
    assert te[1 * 2 + 0] > 0.01                      # source 0 -> target 1 is coupled


@pytest.mark.parametrize("T,b_big", [(900, 90), (70000, 41), (900, 200), (20000, 150)])
def test_global_memory_overflow_counts(cuda, T, b_big):
    # genes whose b_t^2 * b_s histogram cannot fit shared memory (no coarsening): those
    # pairs run in the global-memory overflow launch, the rest in shared memory. T=70000
    # makes N >= 65536 (32-bit counters only, so 41 bins already overflow). With b in
    # the hundreds the target's marginal tables no longer fit shared memory either:
    # every pair of such a target runs in the overflow launch with the tables in
    # global memory.
    rng = np.random.default_rng(T + b_big)
    bvals = [3, b_big, 5, b_big - 7, 2]
    n = len(bvals)
    x = np.stack([rng.integers(0, b, T) for b in bvals]).astype(np.int32)
    bins, npv, bmax = O.remap(x)
    bins = bins.reshape(n, T, 1)
    P = n * (n - 1)
    stride = bmax ** 3
    counts = torch.full((P, stride), -1, dtype=torch.int32, device=cuda)
    te = _gpu_te(bins, npv, bmax, cuda, counts=counts, counts_stride=stride).cpu().numpy()
    cnt = counts.cpu().numpy()
    for p in range(P):
        t, sl = divmod(p, n - 1)
        s = sl + (sl >= t)
        ref = O.counts(bins, 1, t, s, npv).reshape(-1)
        assert np.array_equal(cnt[p, :ref.size], ref), (p, t, s)
    assert np.max(np.abs(te - O.te_pairfree(bins, npv))) <= TOL
    # the overflow pairs' entropy from their samples is bitwise reproducible
    again = _gpu_te(bins, npv, bmax, cuda).cpu().numpy()
    assert np.array_equal(again.view(np.uint32), te.view(np.uint32))
    # pair-list mode (source filter) takes the same two launches
    pairs = np.array([[1, 0], [1, 3], [0, 1], [4, 3], [3, 1]], np.int64)
    from tenex_b200.kernels.pair_list import te_pair_list
    db = D.pack_bins(bins, cuda)
    got = te_pair_list(db, torch.as_tensor(npv, device=cuda), bmax, 1, pairs).cpu().numpy()
    assert np.max(np.abs(got - O.te_pairs(bins, npv, pairs))) <= TOL


@pytest.mark.parametrize("tau,K", [(1, 1), (2, 1), (1, 2), (3, 2)])
def test_tau_and_k(cuda, tau, K):
    rng = np.random.default_rng(tau * 10 + K)
    bins, npv, bmax = _rand_bins(rng, 11, 257, 2, 9, K=K)
    te = _gpu_te(bins, npv, bmax, cuda, tau=tau).cpu().numpy()
    ref = O.te_pairfree(bins, npv, tau=tau)
    assert np.max(np.abs(te - ref)) <= TOL


def test_matrix_mode_and_golden(cuda, golden):
    g = golden("discretize_cfg1.npz")
    bins = g["bins"]
    npv = g["n_per_var"]
    db = D.pack_bins(bins, cuda)
    m = D.te_pairfree(db, torch.as_tensor(npv, device=cuda), int(g["b_max"]),
                      matrix=True).cpu().numpy()
    assert np.max(np.abs(m - g["matrix"])) <= TOL  # reference CPU compute()
    assert np.all(np.diag(m) == 0)


def test_pair_ranges_and_launch_shapes(cuda):
    rng = np.random.default_rng(5)
    n = 40
    bins, npv, bmax = _rand_bins(rng, n, 600, 2, 16)
    ref = O.te_pairfree(bins, npv)
    db = D.pack_bins(bins, cuda)
    npv_t = torch.as_tensor(npv, device=cuda)
    for cfg in (None, dict(threads=128, src_chunk=7),
                dict(threads=1024, ctas_per_sm=2, src_chunk=3),
                dict(threads=256, smem_bytes=48 * 1024, src_chunk=64),
                dict(threads=256, ctas_per_sm=2, src_chunk=5),
                dict(smem_bytes=40 * 1024, threads=1024),
                dict(smem_bytes=24 * 1024, threads=128)):
        for p0, cnt in ((0, n * (n - 1)), (5, 77), (n * (n - 1) - 13, 13), (123, 1)):
            te = D.te_pairfree(db, npv_t, bmax, pair_offset=p0, n_pairs=cnt, cfg=cfg)
            assert np.max(np.abs(te.cpu().numpy() - ref[p0:p0 + cnt])) <= TOL, (cfg, p0)
    # an empty range is a no-op, not an error
    assert D.te_pairfree(db, npv_t, bmax, pair_offset=17, n_pairs=0).numel() == 0


@pytest.mark.parametrize("T", [2, 3, 17])
def test_shortest_series(cuda, T):
    # N = T - 1 samples, down to one: TE of a single sample is 0
    rng = np.random.default_rng(T)
    bins, npv, bmax = _rand_bins(rng, 6, T, 1, 4)
    te = _gpu_te(bins, npv, bmax, cuda).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(bins, npv))) <= TOL
    if T == 2:
        assert np.all(te == 0)


@pytest.mark.parametrize("threads", [256, 1024])
def test_long_series_u32_counters(cuda, threads):
    rng = np.random.default_rng(77)
    bins, npv, bmax = _rand_bins(rng, 5, 70001, 2, 16)  # N >= 65536: 32-bit counters
    te = _gpu_te(bins, npv, bmax, cuda, cfg=dict(threads=threads)).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(bins, npv))) <= TOL


def test_shared_slot_counts(cuda):
    """Small shared memory forces several warps per slot (named barriers); counts exact."""
    rng = np.random.default_rng(12)
    n = 6
    bins, npv, bmax = _rand_bins(rng, n, 2500, 10, 16)
    P = n * (n - 1)
    stride = bmax ** 3
    counts = torch.full((P, stride), -1, dtype=torch.int32, device=cuda)
    te = _gpu_te(bins, npv, bmax, cuda, counts=counts, counts_stride=stride,
                 cfg=dict(smem_bytes=24 * 1024, threads=1024)).cpu().numpy()
    cnt = counts.cpu().numpy()
    for p in range(P):
        t, sl = divmod(p, n - 1)
        s = sl + (sl >= t)
        ref = O.counts(bins, 1, t, s, npv).reshape(-1)
        assert np.array_equal(cnt[p, :ref.size], ref), (p, t, s)
    assert np.max(np.abs(te - O.te_pairfree(bins, npv))) <= TOL


def test_constant_source_gives_zero(cuda):
    rng = np.random.default_rng(3)
    bins, npv, bmax = _rand_bins(rng, 6, 300, 2, 5)
    bins[2] = 0
    npv = npv.copy()
    npv[2] = 1
    te = _gpu_te(bins, npv, bmax, cuda).cpu().numpy()
    for t in range(6):
        if t == 2:
            continue
        sl = 2 if 2 < t else 1  # src_local of source 2 for target t
        assert te[t * 5 + sl] == 0.0


def test_duplicate_source_gives_zero(cuda):
    # source == target's own series: y_t = x_t, so every cell has c3*c1 == c2a*c2b and
    # TE(src -> tgt) = I(x_{t+1}; x_t | x_t) = 0 exactly, as in the reference's formula
    rng = np.random.default_rng(5)
    bins, npv, bmax = _rand_bins(rng, 6, 700, 2, 9)
    bins[4] = bins[1]
    npv = npv.copy()
    npv[4] = npv[1]
    te = _gpu_te(bins, npv, bmax, cuda).cpu().numpy()
    assert te[1 * 5 + 3] == 0.0            # target 1, source 4 (src_local 3)
    assert te[4 * 5 + 1] == 0.0            # target 4, source 1


def test_bad_bins_raise_without_fault(cuda):
    rng = np.random.default_rng(4)
    bins, npv, bmax = _rand_bins(rng, 6, 300, 2, 5)
    npv = npv.copy()
    npv[3] = max(1, npv[3] - 1)  # a bin value now exceeds its gene's n_per_var
    with pytest.raises(native.TenexError, match="BADDATA"):
        _gpu_te(bins, npv, bmax, cuda)
    # the context stays usable
    bins2, npv2, bmax2 = _rand_bins(rng, 6, 300, 2, 5)
    te = _gpu_te(bins2, npv2, bmax2, cuda).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(bins2, npv2))) <= TOL


def test_determinism(cuda):
    # items are handed out by an atomic ticket, but each pair's counts and the order
    # of its entropy sum are fixed: repeated runs give identical integers and float bits
    rng = np.random.default_rng(8)
    bins, npv, bmax = _rand_bins(rng, 30, 2000, 2, 16)
    P, stride = 30 * 29, bmax ** 3
    runs = []
    for _ in range(2):
        counts = torch.zeros((P, stride), dtype=torch.int32, device=cuda)
        te = _gpu_te(bins, npv, bmax, cuda, counts=counts, counts_stride=stride)
        runs.append((te.cpu().numpy().view(np.uint32), counts.cpu().numpy()))
    assert np.array_equal(runs[0][0], runs[1][0])
    assert np.array_equal(runs[0][1], runs[1][1])


def test_skewed_bins_dominant_value_derivation(cuda):
    """Heavily skewed and constant genes exercise the derived row/column."""
    rng = np.random.default_rng(21)
    n, T = 12, 4000
    x = np.zeros((n, T), np.int32)
    for g in range(n):
        b = int(rng.integers(2, 20))
        p = np.ones(b)
        p[0] = 40.0 * (g % 3)  # g % 3 == 0: no dominant value
        p /= p.sum()
        x[g] = rng.choice(b, T, p=p)
    x[5] = 3  # constant gene
    bins, npv, bmax = O.remap(x)
    P = n * (n - 1)
    stride = bmax ** 3
    counts = torch.full((P, stride), -1, dtype=torch.int32, device=cuda)
    te = _gpu_te(bins, npv, bmax, cuda, counts=counts, counts_stride=stride).cpu().numpy()
    cnt = counts.cpu().numpy()
    for p in range(P):
        t, sl = divmod(p, n - 1)
        s = sl + (sl >= t)
        ref = O.counts(bins, 1, t, s, npv).reshape(-1)
        assert np.array_equal(cnt[p, :ref.size], ref), (p, t, s)
    assert np.max(np.abs(te - O.te_pairfree(bins, npv))) <= TOL


def test_full_size_all_pairs_sampled_parity_and_determinism(cuda, full_size_multibin):
    """The full 10,000-gene x 20,000-cell workload (95% of genes b ~ U{2..16},
    5% b ~ U{64..256} coarsened to 38 bins; all 99,990,000 ordered pairs in one
    launch, matrix output): 4,000 random pairs plus 300 pairs on each side of
    three coarsened genes against the float64 C oracle within 1e-6, and a second
    launch bitwise equal to the first."""
    fs = full_size_multibin
    cb, cnpv, m1 = fs["bins"], fs["npv"], fs["matrix"]
    n = cb.shape[0]
    rng = np.random.default_rng(44)
    src = rng.integers(0, n, 4000)
    tgt = rng.integers(0, n, 4000)
    heavy = np.flatnonzero(fs["npv_raw"] > 38)[:3]
    assert len(heavy) == 3
    for h in heavy:
        other = rng.integers(0, n, 300)
        src = np.concatenate([src, other, np.full(300, h)])
        tgt = np.concatenate([tgt, np.full(300, h), other])
    keep = src != tgt
    src, tgt = src[keep], tgt[keep]
    ref = O.te_pairs(cb, cnpv, np.stack([tgt, src], axis=1))
    got = m1[torch.as_tensor(src, device=cuda), torch.as_tensor(tgt, device=cuda)].double()
    assert np.max(np.abs(got.cpu().numpy() - ref)) <= TOL
    assert np.all(np.diag(m1[:4, :4].cpu().numpy()) == 0)
    m2 = fs["kernel"].compute_pairfree_device(fs["db"], fs["npv_t"], fs["b_max"], 1, matrix=True)
    assert torch.equal(m1.view(torch.int32), m2.view(torch.int32))


def test_full_size_multibin_b32_sampled_parity(cuda):
    """5,000 genes x 10,000 cells, b ~ U{2..32} (5% of genes AR lag-1), all
    24,995,000 ordered pairs in one launch: 4,000 random pairs within 1e-6 of
    the float64 oracle; the pair-free vector agrees with the matrix output."""
    from tenex_b200 import workloads as W
    x, npv = W.cfg3_bins()
    bins = np.ascontiguousarray(x, dtype=np.uint8)
    n = bins.shape[0]
    bmax = int(np.max(npv))
    db = D.pack_bins(bins, cuda)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=cuda)
    m = D.te_pairfree(db, npv_t, bmax, matrix=True)              # [src, tgt]
    rng = np.random.default_rng(45)
    src = rng.integers(0, n, 4000)
    tgt = rng.integers(0, n, 4000)
    keep = src != tgt
    src, tgt = src[keep], tgt[keep]
    ref = O.te_pairs(bins, npv, np.stack([tgt, src], axis=1))
    got = m[torch.as_tensor(src, device=cuda), torch.as_tensor(tgt, device=cuda)].double()
    assert np.max(np.abs(got.cpu().numpy() - ref)) <= TOL
    pf = D.te_pairfree(db, npv_t, bmax)                          # target-major pair-free ids
    pid = tgt * (n - 1) + src - (src > tgt)
    assert torch.equal(pf[torch.as_tensor(pid, device=cuda)].cpu(), got.float().cpu())


def test_launch_shape_query(cuda):
    """tenex_te_launch_shape reports the planner's choice: 2 x 512 threads with
    512 sources per item by default, 1 x 1024 when the largest histogram (38
    bins at 19,999 samples) needs a whole SM's shared memory, and an explicit
    config as given."""
    small = native.te_launch_shape(5000, 1, 16)
    assert (small["threads"], small["ctas_per_sm"], small["src_chunk"]) == (512, 2, 512)
    big = native.te_launch_shape(20000, 1, 38)
    assert (big["threads"], big["ctas_per_sm"]) == (1024, 1)
    fixed = native.te_launch_shape(20000, 1, 38, dict(threads=512, ctas_per_sm=2, src_chunk=64))
    assert (fixed["threads"], fixed["ctas_per_sm"], fixed["src_chunk"]) == (512, 1, 64)
    assert 0 < big["smem_bytes"] <= native.device_info(0).smem_optin
    with pytest.raises(native.TenexError):
        native.te_launch_shape(10, 10, 4)
