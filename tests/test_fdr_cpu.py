"""FDR method (z-score, BH, DPI trimming): the oracle against the reference's own
outputs, and the host-side contract (no CUDA needed)."""
import os

import numpy as np
import pytest
import torch

from oracle import fdr_oracle as F
from tenex_b200.inference import get_method
from tenex_b200.inference.grn import build_pairs

GOLD = os.path.join(os.path.dirname(__file__), "golden", "fdr_trim.npz")
CASES = "abcde"


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


def _ranked(pairs, te):
    order = np.lexsort((pairs[:, 1], pairs[:, 0], -te.astype(np.float64)))
    return pairs[order], te[order]


@pytest.mark.parametrize("case", CASES)
def test_oracle_threshold_matches_reference(gold, case):
    m = gold["matrix"]
    names = np.array([f"g{i}" for i in range(m.shape[0])])
    pairs = build_pairs(names)
    te = m[pairs[:, 0], pairs[:, 1]]
    fdr, links, _, _ = gold[f"{case}_cfg"]
    if links:
        tc, pc = F.top_links(te, pairs, int(links))
        # ties may come back in any order: compare value-ranked lists
        a, b = _ranked(pc, tc), _ranked(gold[f"{case}_cut_pairs"], gold[f"{case}_cut_te"])
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
        assert np.all(np.diff(gold[f"{case}_cut_te"].astype(np.float64)) <= 0)
    else:
        tc, pc, _ = F.fdr_threshold(te, pairs, fdr)
        assert np.array_equal(pc, gold[f"{case}_cut_pairs"])
        assert np.array_equal(tc, gold[f"{case}_cut_te"])


@pytest.mark.parametrize("case", CASES)
def test_oracle_trim_matches_reference(gold, case):
    n = gold["matrix"].shape[0]
    _, _, thr, bs = gold[f"{case}_cfg"]
    tp, tv = F.dpi_trim(n, gold[f"{case}_cut_pairs"], gold[f"{case}_cut_te"], int(bs), thr)
    assert np.array_equal(tp, gold[f"{case}_trim_pairs"])
    assert np.array_equal(tv, gold[f"{case}_trim_te"])


def test_golden_exercises_trimming_paths(gold):
    n = gold["matrix"].shape[0]
    for case in CASES:
        assert len(gold[f"{case}_trim_te"]) < len(gold[f"{case}_cut_te"])  # DPI removed edges
    # case e: a batch without an active mediator keeps an edge below the threshold
    _, _, thr, bs = gold["e_cfg"]
    one_batch = F.dpi_trim(n, gold["e_cut_pairs"], gold["e_cut_te"], n, thr)[1]
    assert len(one_batch) != len(gold["e_trim_te"])


def test_dpi_matrix_definition_matches_batched_loop(gold):
    # a single batch with every row active: the matrix definition equals the loop
    n = gold["matrix"].shape[0]
    pairs, te = gold["a_cut_pairs"], gold["a_cut_te"]
    a = np.zeros((n, n), np.float32)
    a[pairs[:, 0], pairs[:, 1]] = te
    med = a.sum(axis=1) > 0
    out = F.dpi_matrix(a, med)
    rows, cols = np.nonzero(out)
    tp, tv = F.dpi_trim(n, pairs, te, n, 0.0)
    assert np.array_equal(np.stack((rows, cols), 1), tp)
    assert np.array_equal(out[rows, cols], tv)


def test_fdr_method_registered_and_cuda_only():
    m = get_method("fdr")
    assert m.name == "fdr"
    with pytest.raises(RuntimeError, match="CUDA"):
        m.infer(np.zeros((3, 3), np.float32), np.array(["a", "b", "c"]), torch.device("cpu"))
    with pytest.raises(NotImplementedError):
        get_method("clr")


@pytest.mark.parametrize("m", [1, 4096, 4097, 50_000, 4096 * 4096 + 17])
def test_blocked_cummin_equals_sequential(m):
    """BH's reverse running minimum is computed in rows of 4096 plus a carry pass;
    it must equal the one-row scan element for element, ties and NaN included."""
    from tenex_b200.inference.grn import bh_fdr_gpu, cummin_1d
    g = torch.Generator().manual_seed(m)
    for dt in (torch.float32, torch.float64):
        x = torch.rand(m, generator=g, dtype=dt)
        x[::5] = x[::5].round(decimals=2)
        assert torch.equal(cummin_1d(x), x.cummin(0).values)
        if m > 2:
            x[m // 3] = float("nan")
            a, b = cummin_1d(x), x.cummin(0).values
            assert torch.equal(a.isnan(), b.isnan())
            assert torch.equal(a[~a.isnan()], b[~b.isnan()])
    if m > 100_000:
        return
    p = torch.rand(m, generator=g, dtype=torch.float64) ** 4
    ref = F.bh_adjust(p.numpy())
    assert np.allclose(bh_fdr_gpu(p, 0.05).numpy(), ref, rtol=1e-12, atol=0)
