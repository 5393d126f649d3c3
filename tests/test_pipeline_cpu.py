"""Multi-lag combine of the surrogate test against the reference's own output
(tests/golden/multilag.npz, made by tenex.pipeline.Pipeline._combine_surrogate_multi_lag)."""
import numpy as np
import pytest
import torch

from tenex_b200.inference.grn import make_grn
from tenex_b200.inference.surrogate_test import SurrogateTestResult
from tenex_b200.pipeline import Pipeline


def _results(g):
    n = g["observed"].shape[1]
    names = np.array([f"g{i}" for i in range(n)])
    out = []
    for k in range(len(g["taus"])):
        out.append(SurrogateTestResult(
            observed_te=g["observed"][k], mean_surrogate_te=g["mean"][k],
            std_surrogate_te=g["std"][k], effective_te=g["effective"][k],
            p_values=g["p"][k], grn=make_grn(names, np.zeros((0, 2), np.int64), np.zeros(0)),
            n_surrogates=10, shuffle_method="block", block_length=5, p_method="parametric",
            fdr=0.05))
    return out, names


@pytest.mark.parametrize("combine", ["max", "adaptive_select", "weighted_sum"])
def test_combine_matches_reference(golden, combine):
    g = golden("multilag.npz")
    res, names = _results(g)
    r = Pipeline._combine_surrogate_multi_lag(res, list(g["taus"]), combine, names,
                                              torch.device("cpu"))
    for f in ("observed_te", "mean_surrogate_te", "std_surrogate_te", "effective_te",
              "p_values"):
        assert np.array_equal(getattr(r, f), g[f"{combine}_{f}"]), f
    assert np.array_equal(r.grn.pairs, g[f"{combine}_pairs"])


def test_combine_errors(golden):
    g = golden("multilag.npz")
    res, names = _results(g)
    for r in res:
        r.p_values = np.ones_like(r.p_values)
    with pytest.raises(ValueError, match="weighted_sum"):
        Pipeline._combine_surrogate_multi_lag(res, [1, 2, 3], "weighted_sum", names,
                                              torch.device("cpu"))
    p = Pipeline()
    with pytest.raises(ValueError, match="non-empty"):
        p._infer_multi_lag([], "max")
    with pytest.raises(ValueError, match="combine"):
        p._infer_multi_lag([1], "mean")
    with pytest.raises(NotImplementedError):
        p._infer_multi_lag([1], "max", inference_method="clr")
    with pytest.raises(ValueError, match="no engine"):
        p.run()
