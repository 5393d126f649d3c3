"""This package against the reference's own CUDA kernels, on the same inputs and
the same GPU.

The reference (cxinsys/tenex) is not part of this repository. When it has been
installed next to it under baseline/_ref (pip install --target, its CUDA
extensions built for sm_100a), these tests import it and run its wrappers:
  * compute_te_adaptive_smem_pairfree (tenex/kernels/adaptive_smem.py:1029),
  * compute_te_smem_pairfree (tenex/kernels/full_smem.py:570),
  * compute_te_gemm_b2 (tenex/kernels/gemm_b2.py:307, cuBLAS + Triton),
  * TransferEntropyEngine.compute (tenex/transferentropy.py:537), with and
    without coarsening,
  * SurrogateTestMethod.infer (tenex/inference/surrogate_test.py:599).
Without that install every test here is skipped.

The reference's kernels evaluate c3*log2f(c3*c1/(c2a*c2b)) in float32 with
fast-math and sum in float32; this package's TE is within 1e-6 of the float64
oracle. The two float32 results are held to the same 1e-6 (measured on B200:
at most 4.8e-7 apart on these inputs, and the surrogate tests select the same
edges); tests whose oracle runs in a second or two also check this package
against the oracle.
"""
import os
import sys

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200 import TransferEntropyEngine, workloads as W
from tenex_b200.kernels import device as D
from tenex_b200.kernels.gemm_b2 import te_binary_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-6      # this package against the float64 oracle
REF_TOL = 1e-6  # this package against the reference's float32 fast-math kernels

REF_DIR = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                       "baseline", "_ref")


@pytest.fixture(scope="module")
def ref(cuda):
    if not os.path.isdir(os.path.join(REF_DIR, "tenex", "_ext")):
        pytest.skip("the reference is not installed under baseline/_ref")
    if REF_DIR not in sys.path:
        sys.path.insert(0, REF_DIR)
    import tenex
    return tenex


def _report(name, a, b):
    d = float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64))))
    print(f"{name}: max |ours - reference| = {d:.3e}")
    return d


def test_adaptive_smem_pairfree_matches_reference_kernel(cuda, ref):
    """cfg4's generator at 400 genes x 4,000 cells (5% of genes with b in the
    hundreds, coarsened to 38 by the reference's rule): all 159,600 pairs."""
    from tenex.kernels.adaptive_smem import compute_te_adaptive_smem_pairfree
    x, npv = W.cfg4_bins(400, 4000, seed=2101)
    cb, cnpv, bmax = O.coarsen(x, npv, 38)
    n = cb.shape[0]
    ours = D.te_pairfree(D.pack_bins(cb, cuda), torch.as_tensor(cnpv, device=cuda),
                         bmax).cpu().numpy()
    theirs = compute_te_adaptive_smem_pairfree(
        torch.from_numpy(cb.astype(np.int8)[:, :, None]).to(cuda),
        torch.from_numpy(cnpv.astype(np.int32)).to(cuda), n, 1)
    assert theirs.shape == ours.shape
    assert _report("Adaptive-SMEM", ours, theirs) <= REF_TOL
    ids = np.random.default_rng(0).choice(ours.size, 2000, replace=False)
    t, sl = np.divmod(ids, n - 1)
    pairs = np.stack([t, sl + (sl >= t)], axis=1)               # [target, source]
    assert np.max(np.abs(ours[ids] - O.te_pairs(cb, cnpv, pairs))) <= TOL


def test_full_smem_pairfree_matches_reference_kernel(cuda, ref):
    """b ~ U{2..32} (cfg3's generator) at 200 genes x 3,000 cells: all pairs."""
    from tenex.kernels.full_smem import compute_te_smem_pairfree
    x, npv = W.cfg3_bins(200, 3000, seed=2102)
    bmax = int(npv.max())
    n = x.shape[0]
    ours = D.te_pairfree(D.pack_bins(x, cuda), torch.as_tensor(npv, device=cuda),
                         bmax).cpu().numpy()
    theirs = compute_te_smem_pairfree(
        torch.from_numpy(np.ascontiguousarray(x, dtype=np.int32)[:, :, None]).to(cuda),
        bmax, n, 1)
    assert _report("Full-SMEM", ours, theirs) <= REF_TOL
    assert np.max(np.abs(ours - O.te_pairfree(x, npv))) <= TOL


def test_gemm_b2_matches_reference(cuda, ref):
    """Binary Markov bins (cfg2's generator) at 500 genes x 3,001 cells."""
    from tenex.kernels.gemm_b2 import compute_te_gemm_b2
    x, _ = W.cfg2_binary(500, 3001, seed=2103)
    ours = te_binary_matrix(D.pack_bins(x, cuda)).cpu().numpy()     # [src, tgt]
    theirs = compute_te_gemm_b2(x.astype(np.int32), tau=1, device=cuda)  # [tgt, src]
    assert _report("GEMM-B2", ours, theirs.T) <= REF_TOL
    assert np.all(np.diag(ours) == 0) and np.all(np.diag(theirs) == 0)


def _expression_with_heavy_genes(n, T, seed):
    """cfg1's expression generator with a tenth of the genes replaced by rows of
    45 FSBW-L bins: one sample at each of -22..22 (unit spacing, just above
    the row's standard deviation) and the rest near 0, in random order. Such
    genes pass the 38-bin limit of Adaptive-SMEM's coarsening on B200."""
    x, _ = W.cfg1_expression(n, T, seed=seed)
    rng = np.random.default_rng(seed + 1)
    for g in rng.choice(n, n // 10, replace=False):
        v = np.concatenate([np.arange(-22, 23, dtype=np.float64), np.zeros(T - 45)])
        x[g] = rng.permutation(v + rng.normal(0.0, 0.02, T)).astype(np.float32)
    return x


@pytest.mark.parametrize("coarsening", [None, False])
def test_engine_compute_matches_reference_engine(cuda, ref, coarsening):
    """TransferEntropyEngine.compute(accelerator="gpu") of both packages on the same
    expression matrix (numpy binning on both sides): same bins, same kernel,
    the same TE matrix. With coarsening=False the heavy genes' pairs take the
    global-memory kernels of both."""
    x = _expression_with_heavy_genes(80, 8000, seed=2104)
    names = np.array([f"g{i}" for i in range(x.shape[0])])
    r_ref = ref.TransferEntropyEngine(x, names).compute(
        accelerator="gpu", devices=[0], use_numpy_bins=True, coarsening=coarsening)
    r_ours = TransferEntropyEngine(x, names).compute(
        accelerator="gpu", devices=[0], use_numpy_bins=True, coarsening=coarsening)
    assert r_ours.kernel == r_ref.kernel
    assert np.array_equal(np.asarray(r_ours.n_per_var), np.asarray(r_ref.n_per_var))
    assert np.array_equal(np.asarray(r_ours.bin_arrs).astype(np.int32),
                          np.asarray(r_ref.bin_arrs).astype(np.int32))
    assert r_ours.matrix.shape == r_ref.matrix.shape
    assert _report(f"engine ({r_ours.kernel}, coarsening={coarsening})",
                   r_ours.matrix, r_ref.matrix) <= REF_TOL


def test_surrogate_test_matches_reference(cuda, ref):
    """SurrogateTestMethod.infer of both packages with the same seed: block
    shuffles drawn from the same torch generator, so the surrogate TEs differ only
    by the kernels' float32 rounding. 80 genes x 1,600 cells (the reference's
    loop path, float64 sums), 20 shuffles of blocks of 40."""
    from tenex.inference.surrogate_test import SurrogateTestMethod as RefMethod
    from tenex_b200.inference.surrogate_test import SurrogateTestMethod
    x, npv, _ = W.cfg5_bins(80, 1600, seed=2105)
    bmax = int(npv.max())
    obs = D.te_pairfree(D.pack_bins(x, cuda), torch.as_tensor(npv, device=cuda), bmax)
    obs = O.pairfree_to_matrix(obs.cpu().numpy(), x.shape[0])     # [src, tgt]
    names = np.array([f"g{i}" for i in range(x.shape[0])])
    kw = dict(bin_data=x[:, :, None].astype(np.int32), n_per_var=npv.astype(np.int32),
              b_max=bmax, kernel="Full-SMEM", tau=1, n_surrogates=20, block_length=40,
              fdr=0.05, seed=7)
    r_ref = RefMethod().infer(obs, names, cuda, **kw)
    r_ours = SurrogateTestMethod().infer(obs, names, cuda, **kw)
    off = ~np.eye(x.shape[0], dtype=bool)
    assert _report("surrogate mean", r_ours.mean_surrogate_te[off],
                   r_ref.mean_surrogate_te[off]) <= REF_TOL
    assert _report("surrogate std", r_ours.std_surrogate_te[off],
                   r_ref.std_surrogate_te[off]) <= REF_TOL
    e_ours = set(zip(r_ours.grn.source, r_ours.grn.target))
    e_ref = set(zip(r_ref.grn.source, r_ref.grn.target))
    union = e_ours | e_ref
    jac = len(e_ours & e_ref) / len(union) if union else 1.0
    print(f"surrogate edges: ours {len(e_ours)}, reference {len(e_ref)}, Jaccard {jac:.4f}")
    assert jac >= 0.99
