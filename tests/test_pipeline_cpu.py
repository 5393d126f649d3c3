"""Multi-lag merge of the surrogate test against the reference's own output
(tests/golden/multilag.npz, made by tenex.pipeline.Pipeline._combine_surrogate_multi_lag),
and the Pipeline's argument checks."""
import numpy as np
import pytest
import torch

from tenex_b200.inference.grn import make_grn
from tenex_b200.inference.surrogate_test import SurrogateTestResult
from tenex_b200.pipeline import Pipeline, merge_lag_results


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
    r = merge_lag_results(res, list(g["taus"]), combine, names, torch.device("cpu"))
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
        merge_lag_results(res, [1, 2, 3], "weighted_sum", names, torch.device("cpu"))
    with pytest.raises(ValueError, match="lag_combine"):
        merge_lag_results(res, [1, 2, 3], "mean", names, torch.device("cpu"))
    p = Pipeline()
    with pytest.raises(ValueError, match="at least one lag"):
        p.infer("surrogate_test", taus=[])
    with pytest.raises(ValueError, match="lag_combine"):
        p.infer("surrogate_test", taus=[1], lag_combine="mean")
    with pytest.raises(NotImplementedError):
        p.infer("clr", taus=[1])
    with pytest.raises(ValueError, match="no data"):
        p.run()
    with pytest.raises(ValueError, match="variable_names"):
        p.run(data=np.zeros((3, 10), np.float32))
