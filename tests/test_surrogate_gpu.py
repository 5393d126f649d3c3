"""Surrogate test on the GPU against the reference fixture and the oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200 import TransferEntropyEngine, workloads as W
from tenex_b200.inference import NetWeaver
from tenex_b200.inference.surrogate_test import (SurrogateAccumulator, build_block_perm,
                                                 run_surrogates, surrogate_statistics)
from tenex_b200.kernels import device as D

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _acc(bins, npv, bmax, obs, cuda, binary=False):
    db = D.pack_bins(bins, cuda)
    return SurrogateAccumulator(db, torch.as_tensor(npv, dtype=torch.int32, device=cuda), bmax,
                                1, torch.as_tensor(obs, dtype=torch.float32, device=cuda),
                                binary)


def test_reference_permutations_reproduce_reference_stats(cuda, golden):
    """The reference's own CPU run (its RNG, its kernel): our kernels given its
    block permutations reproduce its mean / std of the surrogate TE."""
    g = golden("surrogate.npz")
    perm = torch.as_tensor(g["perm"], device=cuda)
    acc = _acc(g["bins"], g["n_per_var"], int(g["n_per_var"].max()), g["observed"], cuda)
    run_surrogates(acc, perm, int(g["block_length"]), use_graph=False)
    S = perm.shape[0]
    mean, std, eff, p = surrogate_statistics(g["observed"], acc.sum.cpu().numpy(),
                                             acc.sumsq.cpu().numpy(), acc.cnt.cpu().numpy(), S,
                                             "parametric")
    assert np.max(np.abs(mean - g["mean"])) <= TOL
    assert np.max(np.abs(std - g["std"])) <= 2e-6
    assert np.max(np.abs(eff - g["effective"])) <= TOL


@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("bl", [20, 1])
def test_cuda_rng_surrogates_match_oracle(cuda, use_graph, bl):
    """Each side compares its surrogate TE with its own observed TE (as the
    method does): pairs whose shuffle leaves the joint counts unchanged tie
    exactly on both sides."""
    x, npv, _ = W.cfg5_bins(n=24, T=600, seed=3, n_planted=3)
    bmax = int(npv.max())
    obs_ref = O.te_matrix(x, npv).astype(np.float32)
    db = D.pack_bins(x, cuda)
    obs = D.te_pairfree(db, torch.as_tensor(npv, device=cuda), bmax, matrix=True).cpu().numpy()
    assert np.max(np.abs(obs - obs_ref)) <= TOL
    S = 6
    perms, eff_bl, nb = build_block_perm(24, 600, "block", bl if bl > 1 else 600, 0, S, 42, cuda)
    acc = _acc(x, npv, bmax, obs, cuda)
    run_surrogates(acc, perms, eff_bl, use_graph=use_graph)
    s, ss, c = O.surrogate_stats(x, npv, perms.cpu().numpy(), eff_bl, obs_ref)
    off = ~np.eye(24, dtype=bool)
    assert np.max(np.abs(acc.sum.cpu().numpy() - s)) <= S * TOL
    assert np.max(np.abs(acc.sumsq.cpu().numpy() - ss)) <= S * TOL
    cg = acc.cnt.cpu().numpy()
    assert np.mean(cg[off] != c[off]) <= 1e-3  # ties within 1e-6 may flip a comparison
    assert np.max(np.abs(cg[off] - c[off])) <= 1


def test_binary_surrogates_use_gemm_path(cuda):
    x, _ = W.cfg2_binary(n=40, T=700, seed=4, n_planted=3)
    npv = np.full(40, 2, np.int32)
    obs = O.te_matrix(x.astype(np.int32), npv).astype(np.float32)
    perms, bl, _ = build_block_perm(40, 700, "block", 25, 0, 4, 7, cuda)
    acc = _acc(x, npv, 2, obs, cuda, binary=True)
    run_surrogates(acc, perms, bl)
    s, ss, c = O.surrogate_stats(x.astype(np.int32), npv, perms.cpu().numpy(), bl, obs)
    assert np.max(np.abs(acc.sum.cpu().numpy() - s)) <= 4 * TOL


def test_netweaver_surrogate_end_to_end(cuda):
    x, planted = W.cfg1_expression(n=30, T=500, seed=11, n_planted=4)
    names = np.array([f"g{i}" for i in range(30)])
    res = TransferEntropyEngine(x, names).compute(accelerator="gpu")
    st = NetWeaver(res, fdr=0.05).infer("surrogate_test", device=cuda, n_surrogates=8,
                                        block_length=20, seed=5)
    perms, bl, _ = build_block_perm(30, 500, "block", 20, 0, 8, 5, cuda)
    s, ss, c = O.surrogate_stats(res.bin_arrs.astype(np.int32), res.n_per_var,
                                 perms.cpu().numpy(), bl, res.matrix)
    c[np.arange(30), np.arange(30)] += 8
    mean, std, eff, p = surrogate_statistics(res.matrix, s, ss, c, 8, "parametric")
    assert np.max(np.abs(st.mean_surrogate_te - mean)) <= TOL
    assert np.max(np.abs(st.effective_te - eff)) <= TOL
    assert st.p_values.shape == (30, 30) and np.all(np.diag(st.p_values) == 1.0)
    st_mc = NetWeaver(res, fdr=0.05).infer("surrogate_test", device=cuda, n_surrogates=8,
                                           block_length=20, seed=5, p_method="mc")
    assert np.all((st_mc.p_values > 0) & (st_mc.p_values <= 1))
    with pytest.raises(ValueError):
        NetWeaver(res).infer("surrogate_test", device=cuda, n_surrogates=1)
    with pytest.raises(NotImplementedError):
        NetWeaver(res).infer("trace", device=cuda)
    # fused=: accepted for the kernels the reference has a fused variant of (the same
    # float64 accumulation runs either way), refused for the others as the reference does
    for fused in (True, False, None):
        sf = NetWeaver(res, fdr=0.05).infer("surrogate_test", device=cuda, n_surrogates=8,
                                            block_length=20, seed=5, fused=fused)
        assert np.array_equal(sf.p_values, st.p_values)
    with pytest.raises(ValueError, match="fused"):
        NetWeaver(res).infer("surrogate_test", device=cuda, n_surrogates=8, kernel="GEMM-B2",
                             fused=True)


def test_pipeline_multi_lag_surrogate(cuda):
    # the pipeline recomputes TE and the surrogate test per lag and merges them; each
    # per-lag run must equal NetWeaver's single-lag run on the same engine output
    from tenex_b200 import TransferEntropyEngine
    from tenex_b200.inference import NetWeaver
    from tenex_b200.pipeline import Pipeline, merge_lag_results
    x, _ = W.cfg1_expression(n=30, T=400, seed=5, n_planted=3)
    names = np.array([f"g{i}" for i in range(30)])
    kw = dict(n_surrogates=8, block_length=10, fdr=0.05, seed=3)
    pipe = Pipeline(TransferEntropyEngine(x, names), fdr=0.05).configure(binning_method="FSBW-L")
    for combine in ("max", "adaptive_select"):
        multi = pipe.infer("surrogate_test", taus=[1, 2], lag_combine=combine, device=cuda, **kw)
        singles = []
        for tau in (1, 2):
            te = TransferEntropyEngine(x, names).compute(tau=tau)
            singles.append(NetWeaver(te, fdr=0.05).infer("surrogate_test", device=cuda, **kw))
        ref = merge_lag_results(singles, [1, 2], combine, names, cuda)
        assert np.array_equal(multi.p_values, ref.p_values)
        assert np.array_equal(multi.effective_te, ref.effective_te)
        assert np.array_equal(multi.grn.pairs, ref.grn.pairs)


def test_surrogate_over_several_devices(cuda):
    # devices=[0, 0]: the pair range split over two host threads (one GPU here, the
    # same code path as two); the same statistics as one device up to float rounding
    from tenex_b200 import workloads as W
    from tenex_b200.kernels import device as Dv
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    x, npv, _ = W.cfg5_bins(n=60, T=600, seed=77)
    obs = FullSMEMKernel().compute_pairfree_device(
        Dv.pack_bins(x, cuda), torch.as_tensor(npv, device=cuda), int(npv.max()), 1,
        matrix=True).cpu().numpy()
    names = np.array([f"g{i}" for i in range(60)])
    kw = dict(bin_data=x, n_per_var=npv, b_max=int(npv.max()), kernel="Full-SMEM", tau=1,
              n_surrogates=12, block_length=20, fdr=0.05, seed=5)
    one = NetWeaver((obs, names), fdr=0.05).infer("surrogate_test", device=cuda, **kw)
    two = NetWeaver((obs, names), fdr=0.05).infer("surrogate_test", device=cuda,
                                                   devices=[0, 0], **kw)
    assert np.allclose(one.mean_surrogate_te, two.mean_surrogate_te, rtol=1e-6, atol=1e-8)
    assert np.allclose(one.p_values, two.p_values, rtol=1e-4, atol=1e-6)
    assert np.array_equal(one.grn.pairs, two.grn.pairs)


def test_device_statistics_match_numpy_expressions(cuda):
    # the single-device test computes the statistics on the device with the same
    # float64 / float32 expressions as the host path; erfc is the only library call
    from tenex_b200.inference.surrogate_test import pair_statistics, pair_statistics_device
    rng = np.random.default_rng(3)
    n, S = 300, 100
    te = (rng.gamma(2.0, 0.002, (S, n, n))).astype(np.float32)
    obs = (rng.gamma(2.0, 0.002, (n, n)) + (rng.random((n, n)) < 0.02) * 0.01).astype(np.float32)
    s1 = te.astype(np.float64).sum(0)
    s2 = (te.astype(np.float64) ** 2).sum(0)
    cnt = (te >= obs).sum(0).astype(np.int32)
    for method in ("parametric", "mc"):
        ref = pair_statistics(obs, s1, s2, cnt, S, method)
        got = pair_statistics_device(*(torch.from_numpy(a).to(cuda) for a in (obs, s1, s2, cnt)),
                                     S, method)
        got = [g.cpu().numpy() for g in got]
        for r, g in zip(ref[:3], got[:3]):
            assert np.array_equal(r.view(np.uint32), g.view(np.uint32))
        ulps = np.abs(ref[3].view(np.int32).astype(np.int64) - got[3].view(np.int32).astype(np.int64))
        assert ulps.max() <= 1 and (ulps > 0).mean() < 1e-3, (method, ulps.max(), (ulps > 0).sum())


def test_full_size_surrogates_sampled_against_oracle(cuda):
    """2,000 genes x 5,000 cells (b ~ U{2..16} Markov), 100 block shuffles of
    length 50 with the reference's seeds (42 + k): the device sums, sums of
    squares and counts of 1,500 sampled pairs against the float64 oracle run on
    the same permutations (float32 TE widened to float64, as the reference's
    loop accumulates)."""
    x, npv, _ = W.cfg5_bins()
    n, T = x.shape
    bmax = int(npv.max())
    db = D.pack_bins(x, cuda)
    obs = D.te_pairfree(db, torch.as_tensor(npv, device=cuda), bmax, matrix=True).cpu().numpy()
    S, bl = 100, 50
    perms, eff_bl, _ = build_block_perm(n, T, "block", bl, 0, S, 42, cuda)
    acc = _acc(x, npv, bmax, obs, cuda)
    run_surrogates(acc, perms, eff_bl)
    rng = np.random.default_rng(46)
    src = rng.integers(0, n, 1500)
    tgt = rng.integers(0, n, 1500)
    keep = src != tgt
    src, tgt = src[keep], tgt[keep]
    pairs_ts = np.stack([tgt, src], axis=1)
    obs_ref = O.te_pairs(x, npv, pairs_ts).astype(np.float32)
    assert np.max(np.abs(obs[src, tgt] - obs_ref)) <= TOL
    s = np.zeros(len(src))
    ss = np.zeros(len(src))
    c = np.zeros(len(src), np.int64)
    ph = perms.cpu().numpy()
    for k in range(S):
        te = O.te_pairs(O.block_shuffle(x, ph[k], eff_bl), npv, pairs_ts).astype(np.float32)
        t64 = te.astype(np.float64)
        s += t64
        ss += t64 * t64
        c += te >= obs_ref
    assert np.max(np.abs(acc.sum.cpu().numpy()[src, tgt] - s)) <= S * TOL
    assert np.max(np.abs(acc.sumsq.cpu().numpy()[src, tgt] - ss)) <= S * TOL
    cg = acc.cnt.cpu().numpy()[src, tgt]
    assert np.mean(cg != c) <= 1e-2           # ties within 1e-6 may flip a comparison
    assert np.max(np.abs(cg - c)) <= 2


@pytest.mark.parametrize("T,K,bl", [(600, 1, 50), (601, 2, 7), (97, 1, 1), (1000, 3, 333)])
def test_block_shuffles_bitexact_single_and_batched(cuda, T, K, bl):
    """tenex_block_shuffle and tenex_block_shuffle_many (several copies in one
    launch) against the oracle's shuffle: every copy bit-exact, the tail after
    the last whole block unchanged."""
    rng = np.random.default_rng(T + K + bl)
    n, S = 37, 5
    x = rng.integers(0, 200, (n, T, K)).astype(np.uint8)
    nb = T // bl
    perms = np.stack([np.argsort(rng.random((n, nb)), axis=1) for _ in range(S)]).astype(np.int32)
    db = D.pack_bins(x, cuda)
    big = D.empty_bins(S * n, T, K, cuda)
    D.block_shuffle_many(db, torch.as_tensor(perms, device=cuda), bl, big)
    got = big.unpadded().cpu().numpy()
    for s in range(S):
        ref = O.block_shuffle(x, perms[s], bl)
        assert np.array_equal(got[s * n:(s + 1) * n], ref)
        one = D.block_shuffle(db, torch.as_tensor(perms[s], device=cuda), bl)
        assert np.array_equal(one.unpadded().cpu().numpy(), ref)
