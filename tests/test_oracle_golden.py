"""The oracle against the reference's own outputs (golden fixtures)."""
import numpy as np

from oracle import oracle as O


def test_fsbwl_and_remap_match_reference_discretize(golden):
    g = golden("discretize_cfg1.npz")
    bins, nb = O.fsbwl(g["x"], 0.5)
    assert np.array_equal(nb, g["n_bins"])
    rem, npv, bmax = O.remap(bins)
    assert np.array_equal(rem, g["bins"][:, :, 0])
    assert np.array_equal(npv, g["n_per_var"])
    assert bmax == int(g["b_max"])


def test_te_matrix_matches_reference_cpu_compute(golden):
    g = golden("discretize_cfg1.npz")
    m = O.te_matrix(g["bins"], g["n_per_var"], tau=1)
    # reference: float32 scatter_add; oracle: float64 of the same formula
    assert np.max(np.abs(m - g["matrix"])) < 1e-6
    assert np.all(np.diag(m) == 0)


def test_te_pairs_match_scatter_add_tau1_tau2(golden):
    g = golden("scatter_multibin.npz")
    for tau, key in ((1, "te_tau1"), (2, "te_tau2")):
        te = O.te_pairs(g["bins"], g["n_per_var"], g["pairs"], tau=tau)
        assert np.max(np.abs(te - g[key])) < 1e-6, tau


def test_te_pairs_match_scatter_add_k2(golden):
    g = golden("scatter_k2.npz")
    te = O.te_pairs(g["bins"], g["n_per_var"], g["pairs"], tau=1)
    assert np.max(np.abs(te - g["te"])) < 1e-6


def test_remap_matches_reference(golden):
    g = golden("remap.npz")
    rem, npv, bmax = O.remap(g["raw"])
    assert np.array_equal(rem, g["remapped"])
    assert np.array_equal(npv, g["n_per_var"])
    assert bmax == int(g["b_max"])


def test_coarsen_matches_reference(golden):
    g = golden("coarsen.npz")
    out, npv, bmax = O.coarsen(g["bins"], g["n_per_var"], int(g["limit"]))
    assert np.array_equal(out, g["out"])
    assert np.array_equal(npv, g["out_npv"])
    assert bmax == int(g["out_bmax"])


def test_remap_and_coarsen_of_wide_bins_match_reference(golden):
    """Genes of 257, 300 and 1000 distinct bins: the reference's int32 remap,
    int16 storage and coarsening to 38 bins."""
    g = golden("coarsen_wide.npz")
    rem, npv, bmax = O.remap(g["raw"])
    assert np.array_equal(rem, g["remapped"])
    assert np.array_equal(npv, g["n_per_var"])
    assert bmax == int(g["b_max"]) == 1000
    out, onpv, obmax = O.coarsen(rem, npv, int(g["limit"]))
    assert np.array_equal(out, g["out"])
    assert np.array_equal(onpv, g["out_npv"])
    assert obmax == int(g["out_bmax"])


def test_smem_bin_limit_rule(golden):
    g = golden("smem_limit.npz")
    for s, lim in zip(g["smem"], g["limit"]):
        assert O.smem_bin_limit(int(s)) == int(lim)
    assert O.smem_bin_limit(232448) == 38  # B200 opt-in


def test_binary_te_matches_reference_gemm_b2(golden):
    g = golden("gemm_b2.npz")
    x = g["bins"].astype(np.int32)
    npv = np.full(x.shape[0], 2, np.int32)
    m = O.te_matrix(x, npv)  # [i, j] = TE(i -> j)
    ref = g["te_ij_j_to_i"].T  # reference rows are targets
    assert np.max(np.abs(m - ref)) < 1e-6


def test_surrogate_stats_match_reference_loop(golden):
    g = golden("surrogate.npz")
    S = g["perm"].shape[0]
    s, ss, c = O.surrogate_stats(g["bins"], g["n_per_var"], g["perm"], int(g["block_length"]),
                                 g["observed"])
    mean = (s / S).astype(np.float32)
    std = np.sqrt(np.maximum(ss / S - (s / S) ** 2, 0.0)).astype(np.float32)
    assert np.max(np.abs(mean - g["mean"])) < 1e-6
    assert np.max(np.abs(std - g["std"])) < 2e-6


def test_binarize_thresholds_match_reference_numpy_backend(golden):
    g = golden("binarize.npz")
    for T in (400, 401):
        x = g[f"x{T}"]
        for tag, method, q in (("median", "median", 0.5), ("q70", "quantile", 0.7),
                               ("q25", "quantile", 0.25), ("mean", "mean", 0.5),
                               ("nonzero", "nonzero", 0.5)):
            assert np.array_equal(O.binarize(x, method, q), g[f"{tag}{T}"]), (tag, T)
