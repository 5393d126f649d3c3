"""Generates tests/golden/*.npz from the reference implementation itself.

Run in a container that has the reference source tree (it is imported, never
copied):  python tests/golden/make_golden.py /path/to/reference

The fixtures are small (seconds to produce) and pin the oracle and the
product to the reference's own CPU code paths:
  discretize_cfg1.npz   tenex.preprocess.discretize(use_numpy_bins=True) and
                        TransferEntropyEngine.compute(accelerator="cpu") on a
                        cfg1-shaped expression matrix (n=40, T=300)
  scatter_multibin.npz  tenex.kernels.scatter_add.compute_te_scatter_add on
                        random multi-bin data, all ordered pairs, tau=1 and tau=2
  scatter_k2.npz        same with K=2 samples per time step
  remap.npz             tenex.preprocess.remap_bins on gapped int32 bins
  coarsen.npz           tenex.preprocess.coarsen_bins (CPU path), limit 38
  gemm_b2.npz           tenex.kernels.gemm_b2.compute_te_gemm_b2 (torch path, CPU)
  surrogate.npz         SurrogateTestMethod.infer on CPU (scatter_add kernel, block
                        shuffles) plus the block permutations its RNG schedule draws
  smem_limit.npz        compute_smem_bin_limit for a few SMEM sizes
  multilag.npz          Pipeline._combine_surrogate_multi_lag (max, adaptive_select,
                        weighted_sum) on three synthetic per-lag surrogate results
  fdr_trim.npz          the FDR method's thresholding (fdr_threshold_gpu, top-K) and
                        DPI trimming (_trim) on CPU tensors, for a synthetic TE matrix
                        with planted direct and indirect edges

  coarsen_wide.npz      tenex.preprocess.remap_bins + _compact_dtype (int16) +
                        coarsen_bins on genes with 257, 300 and 1000 distinct bins
  binarize.npz          tenex.binarize.binarize (numpy backend): median, quantile
                        q = 0.7 / 0.25, mean and nonzero at T = 400 and 401

`python tests/golden/make_golden.py /path/to/reference multilag` (or `fdr`, `wide`, `binarize`)
writes only that one.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))


def main(ref: str) -> None:
    sys.path.insert(0, ref)
    sys.path.insert(0, REPO)
    os.environ.setdefault("TENEX_CPU_ONLY", "1")
    import torch
    from tenex.preprocess import discretize, remap_bins, coarsen_bins
    from tenex.transferentropy import TransferEntropyEngine
    from tenex.kernels.scatter_add import compute_te_scatter_add
    from tenex.kernels.gemm_b2 import compute_te_gemm_b2
    from tenex.kernels.adaptive_smem import compute_smem_bin_limit
    from tenex.inference.surrogate_test import SurrogateTestMethod, _build_block_perm
    from tenex_b200 import workloads as W

    cpu = torch.device("cpu")

    # 1. discretisation + full CPU compute on cfg1-shaped expression
    x, planted = W.cfg1_expression(n=40, T=300, seed=7, n_planted=4)
    bins, n_bins, b_max, npv = discretize(x, method="FSBW-L", kp=0.5, device=cpu,
                                          use_numpy_bins=True)
    names = np.array([f"g{i}" for i in range(x.shape[0])])
    res = TransferEntropyEngine(x, names).compute(accelerator="cpu")
    np.savez_compressed(os.path.join(HERE, "discretize_cfg1.npz"), x=x,
                        bins=bins.numpy().astype(np.int32), n_bins=np.asarray(n_bins),
                        b_max=b_max, n_per_var=npv.numpy(), matrix=np.asarray(res.matrix),
                        planted=planted)

    # 2. multi-bin scatter_add, tau=1 and tau=2
    rng = np.random.default_rng(11)
    n, T = 24, 400
    b = rng.integers(1, 13, n)
    xb = np.stack([rng.integers(0, bb, T) for bb in b]).astype(np.int32)
    xb, npv_d, bmax_d = remap_bins(torch.from_numpy(xb[:, :, None].copy()))
    t_idx, s_idx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    msk = t_idx != s_idx
    pairs = np.stack([t_idx[msk], s_idx[msk]], 1).astype(np.int64)
    te1 = compute_te_scatter_add(xb, torch.from_numpy(pairs), bmax_d, tau=1)
    te2 = compute_te_scatter_add(xb, torch.from_numpy(pairs), bmax_d, tau=2)
    np.savez_compressed(os.path.join(HERE, "scatter_multibin.npz"),
                        bins=xb.numpy()[:, :, 0], n_per_var=npv_d.numpy(), b_max=bmax_d,
                        pairs=pairs, te_tau1=te1, te_tau2=te2)

    # 3. K = 2
    n, T, K = 10, 150, 2
    xk = rng.integers(0, 5, (n, T, K)).astype(np.int32)
    xk, npv_k, bmax_k = remap_bins(torch.from_numpy(xk))
    t_idx, s_idx = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    msk = t_idx != s_idx
    pk = np.stack([t_idx[msk], s_idx[msk]], 1).astype(np.int64)
    tek = compute_te_scatter_add(xk, torch.from_numpy(pk), bmax_k, tau=1)
    np.savez_compressed(os.path.join(HERE, "scatter_k2.npz"), bins=xk.numpy(),
                        n_per_var=npv_k.numpy(), b_max=bmax_k, pairs=pk, te=tek)

    # 4. remap on gapped bins
    raw = (rng.integers(0, 9, (16, 200)) * rng.integers(1, 4, (16, 1))).astype(np.int32)
    raw[3] = 5  # a constant gene
    rem, npv_r, bmax_r = remap_bins(torch.from_numpy(raw[:, :, None].copy()))
    np.savez_compressed(os.path.join(HERE, "remap.npz"), raw=raw, remapped=rem.numpy()[:, :, 0],
                        n_per_var=npv_r.numpy(), b_max=bmax_r)

    # 5. coarsening (CPU path of coarsen_bins)
    nb = rng.integers(2, 80, 20).astype(np.int32)
    cb = np.stack([rng.integers(0, v, 300) for v in nb]).astype(np.int32)
    for g in range(20):  # make every bin value present so n_per_var is exact
        cb[g, :nb[g]] = np.arange(nb[g])
    c_out, c_npv, c_bmax = coarsen_bins(torch.from_numpy(cb[:, :, None].copy()),
                                        torch.from_numpy(nb.copy()), 38)
    np.savez_compressed(os.path.join(HERE, "coarsen.npz"), bins=cb, n_per_var=nb,
                        limit=38, out=c_out.numpy()[:, :, 0].astype(np.int32),
                        out_npv=c_npv.numpy(), out_bmax=c_bmax)

    # 6. GEMM-B2 (torch path on CPU)
    xbin, _ = W.cfg2_binary(n=30, T=500, seed=5, n_planted=3)
    gm = compute_te_gemm_b2(xbin.astype(np.int32), tau=1, device=cpu, use_triton=False)
    np.savez_compressed(os.path.join(HERE, "gemm_b2.npz"), bins=xbin, te_ij_j_to_i=gm)

    # 7. surrogate test on CPU with the scatter_add kernel
    xs, npv_s, _pl = W.cfg5_bins(n=12, T=200, seed=9, n_planted=2)
    xs32 = xs.astype(np.int32)[:, :, None]
    bmax_s = int(npv_s.max())
    t_idx, s_idx = np.meshgrid(np.arange(12), np.arange(12), indexing="ij")
    msk = t_idx != s_idx
    ps = np.stack([t_idx[msk], s_idx[msk]], 1).astype(np.int64)
    te_obs = compute_te_scatter_add(torch.from_numpy(xs32), torch.from_numpy(ps), bmax_s, tau=1)
    obs = np.zeros((12, 12), np.float32)
    obs[ps[:, 0], ps[:, 1]] = te_obs
    obs = obs.T.copy()  # [i, j] = TE(i -> j)
    S, bl, seed = 6, 10, 42
    res_s = SurrogateTestMethod().infer(obs, np.array([f"g{i}" for i in range(12)]), cpu,
                                        bin_data=xs32, n_per_var=npv_s, b_max=bmax_s,
                                        kernel="scatter_add", tau=1, n_surrogates=S,
                                        block_length=bl, fdr=0.05, seed=seed)
    perm, eff_bl, n_blocks = _build_block_perm(12, 200, 199, "block", bl, 0, S, seed, cpu)
    np.savez_compressed(os.path.join(HERE, "surrogate.npz"), bins=xs, n_per_var=npv_s,
                        observed=obs, perm=perm.numpy(), block_length=bl, seed=seed,
                        mean=res_s.mean_surrogate_te, std=res_s.std_surrogate_te,
                        effective=res_s.effective_te, p_values=res_s.p_values,
                        n_edges=len(res_s.grn))

    # 8. SMEM bin limit rule
    sizes = np.array([49152, 101376, 166912, 232448], np.int64)
    lim = np.array([compute_smem_bin_limit(int(s), warps=32) for s in sizes])
    np.savez_compressed(os.path.join(HERE, "smem_limit.npz"), smem=sizes, limit=lim)
    print("golden fixtures written to", HERE)


def wide(ref: str) -> None:
    """Genes with more than 256 distinct bins: the reference remaps them into
    int32, stores them as int16 (_compact_dtype) and coarsens the int16 bins to
    the B200 shared-memory limit (38) in coarsen_bins."""
    sys.path.insert(0, ref)
    os.environ.setdefault("TENEX_CPU_ONLY", "1")
    import torch
    from tenex.preprocess import _compact_dtype, coarsen_bins, remap_bins
    rng = np.random.default_rng(256)
    n, T = 40, 4000
    nb = rng.integers(2, 30, n)
    nb[3], nb[17], nb[30] = 300, 1000, 257
    raw = np.stack([rng.choice(np.arange(0, 3 * v, 3), T) for v in nb]).astype(np.int32)
    for g in range(n):          # every value present, shuffled into the series
        raw[g, rng.permutation(T)[:nb[g]]] = np.arange(0, 3 * nb[g], 3)
    rem, npv, bmax = remap_bins(torch.from_numpy(raw[:, :, None].copy()))
    rem16 = _compact_dtype(rem, bmax)
    assert rem16.dtype == torch.int16
    remapped = rem16.numpy()[:, :, 0].copy()           # coarsen_bins works in place
    out, out_npv, out_bmax = coarsen_bins(rem16, npv.clone(), 38)
    np.savez_compressed(os.path.join(HERE, "coarsen_wide.npz"), raw=raw,
                        remapped=remapped, n_per_var=npv.numpy(), b_max=bmax,
                        limit=38, out=out.numpy()[:, :, 0].astype(np.int32),
                        out_dtype=str(out.dtype), out_npv=out_npv.numpy(), out_bmax=out_bmax)
    print("coarsen_wide.npz written to", HERE)


def binarized(ref: str) -> None:
    """tenex.binarize.binarize with its default numpy backend (np.median and
    np.quantile thresholds) on expression matrices with many ties (zeros), at an
    even and an odd number of time points."""
    sys.path.insert(0, ref)
    sys.path.insert(0, REPO)
    os.environ.setdefault("TENEX_CPU_ONLY", "1")
    import torch
    from tenex.binarize import binarize
    from tenex_b200 import workloads as W
    out = {}
    for T in (400, 401):
        x, _ = W.cfg1_expression(n=50, T=T, seed=8)
        out[f"x{T}"] = x
        for tag, method, params in (("median", "median", {}), ("q70", "quantile", {"q": 0.7}),
                                    ("q25", "quantile", {"q": 0.25}),
                                    ("mean", "mean", {}), ("nonzero", "nonzero", {})):
            b, _, _, npv = binarize(x, method=method, device=torch.device("cpu"), **params)
            out[f"{tag}{T}"] = b.numpy()[:, :, 0].astype(np.uint8)
            out[f"{tag}{T}_npv"] = npv.numpy()
    np.savez_compressed(os.path.join(HERE, "binarize.npz"), **out)
    print("binarize.npz written to", HERE)


def multilag(ref: str) -> None:
    """The reference's multi-lag combine on synthetic per-lag surrogate results."""
    sys.path.insert(0, ref)
    os.environ.setdefault("TENEX_CPU_ONLY", "1")
    import torch
    from tenex.pipeline import Pipeline
    from tenex.inference import make_grn
    from tenex.inference.surrogate_test import SurrogateTestResult

    rng = np.random.default_rng(21)
    n, taus = 15, [1, 2, 3]
    names = np.array([f"g{i}" for i in range(n)])
    stacks = {k: [] for k in ("observed", "mean", "std", "effective", "p")}
    results = []
    for _ in taus:
        obs = (rng.random((n, n)) * 0.05).astype(np.float32)
        np.fill_diagonal(obs, 0.0)
        mean = (rng.random((n, n)) * 0.03).astype(np.float32)
        std = (rng.random((n, n)) * 0.01 + 1e-3).astype(np.float32)
        eff = (obs - mean).astype(np.float32)
        p = (rng.random((n, n)) ** 4).astype(np.float32)
        np.fill_diagonal(p, 1.0)
        for k, v in zip(stacks, (obs, mean, std, eff, p)):
            stacks[k].append(v)
        results.append(SurrogateTestResult(
            observed_te=obs, mean_surrogate_te=mean, std_surrogate_te=std, effective_te=eff,
            p_values=p, grn=make_grn(names, np.zeros((0, 2), np.int64), np.zeros(0)),
            n_surrogates=10, shuffle_method="block", block_length=5, p_method="parametric",
            fdr=0.05))
    out = {k: np.stack(v) for k, v in stacks.items()}
    for combine in ("max", "adaptive_select", "weighted_sum"):
        r = Pipeline._combine_surrogate_multi_lag(results, taus, combine, names,
                                                  torch.device("cpu"))
        for f in ("observed_te", "mean_surrogate_te", "std_surrogate_te", "effective_te",
                  "p_values"):
            out[f"{combine}_{f}"] = getattr(r, f)
        out[f"{combine}_pairs"] = r.grn.pairs
    np.savez_compressed(os.path.join(HERE, "multilag.npz"), taus=np.array(taus), **out)
    print("multilag.npz written to", HERE)


def fdr_te_matrix(n: int = 150, seed: int = 31) -> tuple[np.ndarray, list]:
    """Synthetic TE matrix: small background, planted chains a -> b -> c with a
    weaker direct a -> c (an indirect edge DPI removes), a few exact ties and
    exact zeros."""
    rng = np.random.default_rng(seed)
    m = (rng.gamma(2.0, 0.002, (n, n))).astype(np.float32)
    m[rng.random((n, n)) < 0.05] = 0.0
    chains = []
    for c in range(12):
        a, b, d = rng.choice(n, 3, replace=False)
        ab, bd = np.float32(0.2 + 0.02 * c), np.float32(0.15 + 0.01 * c)
        m[a, b], m[b, d] = ab, bd
        m[a, d] = np.float32(0.1) if c % 3 else bd     # c % 3 == 0: a tie with min(ab, bd)
        chains.append((a, b, d))
    np.fill_diagonal(m, 0.0)
    return m, chains


def fdr(ref: str) -> None:
    """The reference's FDR thresholding and DPI trimming on CPU tensors."""
    sys.path.insert(0, ref)
    os.environ.setdefault("TENEX_CPU_ONLY", "1")
    import torch
    from tenex.inference import build_pairs, fdr_threshold_gpu, threshold_pairs
    from tenex.inference.fdr import _trim

    cpu = torch.device("cpu")
    m, _ = fdr_te_matrix()
    n = m.shape[0]
    names = np.array([f"g{i}" for i in range(n)])
    pairs = build_pairs(names)
    te = m[pairs[:, 0], pairs[:, 1]]
    out = {"matrix": m}
    cases = [("a", dict(fdr=0.01, links=0, thr=0.0, bs=512)),
             ("b", dict(fdr=0.05, links=0, thr=0.001, bs=7)),
             ("c", dict(fdr=0.01, links=300, thr=0.0, bs=64)),
             ("d", dict(fdr=0.2, links=0, thr=-0.01, bs=33)),
             ("e", dict(fdr=0.05, links=0, thr=0.15, bs=5))]
    for tag, c in cases:
        te_t = torch.from_numpy(te)
        pairs_t = torch.from_numpy(pairs).long()
        if c["links"]:
            te_cut, pairs_cut = threshold_pairs(te_t, pairs_t, cpu, fdr=c["fdr"], links=c["links"])
        else:
            tc, pc = fdr_threshold_gpu(te_t, pairs_t, c["fdr"])
            te_cut, pairs_cut = tc.numpy(), pc.numpy()
        grn = _trim(m, names, pairs_cut, te_cut, device=cpu, batch_size=c["bs"],
                    trim_threshold=c["thr"])
        out[f"{tag}_cfg"] = np.array([c["fdr"], c["links"], c["thr"], c["bs"]], np.float64)
        out[f"{tag}_cut_pairs"] = np.asarray(pairs_cut)
        out[f"{tag}_cut_te"] = np.asarray(te_cut, np.float32)
        out[f"{tag}_trim_pairs"] = np.asarray(grn.pairs)
        out[f"{tag}_trim_te"] = np.asarray(grn.te, np.float32)
    np.savez_compressed(os.path.join(HERE, "fdr_trim.npz"), **out)
    print("fdr_trim.npz written to", HERE)


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_golden.py REFERENCE_SOURCE_TREE [multilag|fdr|wide|binarize]")
    ref_dir = sys.argv[1]
    only = sys.argv[2] if len(sys.argv) > 2 else None
    if only == "multilag":
        multilag(ref_dir)
    elif only == "fdr":
        fdr(ref_dir)
    elif only == "wide":
        wide(ref_dir)
    elif only == "binarize":
        binarized(ref_dir)
    else:
        main(ref_dir)
        multilag(ref_dir)
        fdr(ref_dir)
        wide(ref_dir)
        binarized(ref_dir)
