"""FDR method on the GPU: tenex_dpi_trim bit-exact against the oracle, and the
method end to end against the reference's own outputs."""
import os

import numpy as np
import pytest
import torch

from oracle import fdr_oracle as F
from tenex_b200.inference import NetWeaver, get_method
import ctypes

from tenex_b200 import native
from tenex_b200.inference.fdr import dpi_trim, dpi_trim_matrix, dpi_trim_sparse
from tenex_b200.inference.grn import build_pairs

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "fdr_trim.npz")


def _sparse_net(rng, n, density, neg=False):
    a = (rng.gamma(2.0, 0.05, (n, n)) * (rng.random((n, n)) < density)).astype(np.float32)
    # exact ties between direct and indirect paths
    k = max(1, n // 20)
    i, j, m = rng.integers(0, n, k), rng.integers(0, n, k), rng.integers(0, n, k)
    a[i, j] = np.minimum(a[i, m], a[m, j])
    if neg:
        a[rng.random((n, n)) < 0.01] = np.float32(-1e-3)
    np.fill_diagonal(a, 0)
    return a


@pytest.mark.parametrize("n,density,thr", [(1, 1.0, 0.0), (5, 0.6, 0.0), (130, 0.1, 0.0),
                                           (257, 0.05, 0.002), (300, 0.3, -0.01)])
def test_dpi_kernel_bitexact(cuda, n, density, thr):
    rng = np.random.default_rng(n)
    a = _sparse_net(rng, n, density, neg=(thr < 0))
    med = rng.random(n) < 0.8
    keep = rng.random(n) < 0.1
    for m_, k_ in ((None, None), (med, keep)):
        ref = F.dpi_matrix(a, m_, k_, thr)
        got = dpi_trim_matrix(torch.from_numpy(a).to(cuda),
                              None if m_ is None else torch.from_numpy(m_),
                              None if k_ is None else torch.from_numpy(k_), thr).cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("n,density,thr", [(1, 1.0, 0.0), (7, 0.6, 0.0), (200, 0.05, 0.0),
                                           (513, 0.02, 0.003), (300, 0.4, -0.01)])
def test_dpi_sparse_equals_dense(cuda, n, density, thr):
    rng = np.random.default_rng(1000 + n)
    a = _sparse_net(rng, n, density, neg=True)
    med = rng.random(n) < 0.85
    keep = rng.random(n) < 0.1
    A = torch.from_numpy(a).to(cuda)
    for m_, k_ in ((None, None), (med, keep)):
        mt = None if m_ is None else torch.from_numpy(m_).to(cuda)
        kt = None if k_ is None else torch.from_numpy(k_).to(cuda)
        dense = dpi_trim_matrix(A, mt, kt, thr)
        r, c = torch.nonzero(dense, as_tuple=True)
        rs, cs, vs = dpi_trim_sparse(A, mt, kt, thr)
        assert torch.equal(rs, r) and torch.equal(cs, c)
        assert torch.equal(vs.view(torch.int32), dense[r, c].view(torch.int32))


def test_dpi_sparse_guards(cuda):
    # an entry whose column is out of range is ignored (no fault) and never kept
    row_ptr = torch.tensor([0, 2, 3], dtype=torch.int64, device=cuda)
    col = torch.tensor([1, 5, 0], dtype=torch.int32, device=cuda)
    val = torch.tensor([0.5, 0.7, 0.25], dtype=torch.float32, device=cuda)
    keep = torch.full((3,), 7, dtype=torch.uint8, device=cuda)
    native.call("tenex_dpi_trim_sparse", row_ptr.data_ptr(), col.data_ptr(), val.data_ptr(), 2,
                None, None, ctypes.c_float(0.0), keep.data_ptr(), native.stream_ptr())
    assert keep.tolist() == [1, 0, 1]
    big = 200_000                                      # a row of 800 KB cannot fit shared memory
    rp = torch.zeros(big + 1, dtype=torch.int64, device=cuda)
    with pytest.raises(native.TenexError) as ei:
        native.call("tenex_dpi_trim_sparse", rp.data_ptr(), col.data_ptr(), val.data_ptr(), big,
                    None, None, ctypes.c_float(0.0), keep.data_ptr(), native.stream_ptr())
    assert ei.value.status == native.TENEX_ERR_UNSUPPORTED


def test_dpi_kernel_large_rows(cuda):
    n = 2000
    rng = np.random.default_rng(5)
    a = _sparse_net(rng, n, 0.02)
    got = dpi_trim_matrix(torch.from_numpy(a).to(cuda)).cpu().numpy()
    rows = rng.choice(n, 24, replace=False)
    ref = F.dpi_matrix(a, rows=rows)
    assert np.array_equal(got[rows], ref)
    # trimming only removes entries, never changes a kept one
    kept = got != 0
    assert np.array_equal(got[kept], a[kept])


def _assert_cut_close(grn, te, pairs, fdr):
    """Same kept edges as the float64 oracle, except pairs whose adjusted p lies
    within rounding of the cut (float32 mean/std on the device)."""
    tc, pc, adj = F.fdr_threshold(te, pairs, fdr)
    got = {tuple(p) for p in np.asarray(grn.pairs).tolist()}
    want = {tuple(p) for p in pc.tolist()}
    idx = {tuple(p): i for i, p in enumerate(pairs.tolist())}
    for p in got ^ want:
        assert abs(adj[idx[p]] - fdr) <= 1e-4 * fdr, p


@pytest.mark.parametrize("dpi_method", ["dense", "sparse", "auto"])
@pytest.mark.parametrize("case", "abcde")
def test_fdr_method_against_reference(cuda, case, dpi_method):
    z = np.load(GOLD)
    m = z["matrix"]
    n = m.shape[0]
    names = np.array([f"g{i}" for i in range(n)])
    fdr, links, thr, bs = z[f"{case}_cfg"]
    grn, trimmed = get_method("fdr").infer(m, names, cuda, fdr=fdr, links=int(links),
                                           trim_threshold=thr, batch_size=int(bs),
                                           dpi_method=dpi_method)
    gp, gt = z[f"{case}_cut_pairs"], z[f"{case}_cut_te"]
    if links:
        order = lambda p, t: np.lexsort((p[:, 1], p[:, 0], -t.astype(np.float64)))
        o1, o2 = order(grn.pairs, grn.te), order(gp, gt)
        assert np.array_equal(grn.pairs[o1], gp[o2]) and np.array_equal(grn.te[o1], gt[o2])
    else:
        pairs = build_pairs(names)
        _assert_cut_close(grn, m[pairs[:, 0], pairs[:, 1]], pairs, fdr)
        if not np.array_equal(grn.pairs, gp):   # a borderline flip: check the trim on our cut
            tp, tv = F.dpi_trim(n, grn.pairs, grn.te, int(bs), thr)
            assert np.array_equal(trimmed.pairs, tp) and np.array_equal(trimmed.te, tv)
            return
        assert np.array_equal(grn.te, gt)
    assert np.array_equal(trimmed.pairs, z[f"{case}_trim_pairs"])
    assert np.array_equal(trimmed.te, z[f"{case}_trim_te"])
    assert list(trimmed.source) == [names[i] for i in z[f"{case}_trim_pairs"][:, 0]]


def test_fdr_no_trimming_and_netweaver_default(cuda):
    z = np.load(GOLD)
    m = z["matrix"]
    names = np.array([f"g{i}" for i in range(m.shape[0])])
    grn = get_method("fdr").infer(m, names, cuda, fdr=0.01, is_trimming=False)
    assert np.array_equal(grn.pairs, z["a_cut_pairs"])
    out = NetWeaver((m, names)).infer(device=cuda)          # method='fdr' by default
    assert isinstance(out, tuple) and np.array_equal(out[1].pairs, z["a_trim_pairs"])
    # a constant matrix: zero std, no edges
    flat = np.full_like(m, 0.1)
    assert len(get_method("fdr").infer(flat, names, cuda)[0]) == 0


def test_fdr_source_filter_and_no_mediator(cuda):
    rng = np.random.default_rng(9)
    n = 60
    m = _sparse_net(rng, n, 0.5)
    names = np.array([f"g{i}" for i in range(n)])
    tfs = names[:7]
    grn, trimmed = get_method("fdr").infer(m, names, cuda, fdr=0.2, sources=tfs)
    pairs = build_pairs(names, tfs)
    te = m[pairs[:, 0], pairs[:, 1]]
    _assert_cut_close(grn, te, pairs, 0.2)
    tp, tv = F.dpi_trim(n, grn.pairs, grn.te, 512, 0.0)
    assert np.array_equal(trimmed.pairs, tp) and np.array_equal(trimmed.te, tv)
    # no row with a positive sum: the cut network comes back unchanged
    p = np.array([[0, 1], [2, 3]])
    g = dpi_trim(4, names[:4], p, np.array([-0.5, -0.25], np.float32), cuda)
    assert np.array_equal(g.pairs, p)


def test_fdr_full_size_threshold_and_dpi_forms_agree(cuda, full_size_multibin):
    """The FDR method's steps on the 10,000-gene TE matrix (99,990,000 pairs):
    BH-FDR 0.01 on the device keeps the pairs at the top of the TE ranking (p
    falls as TE rises), and the sparse and dense DPI kernels give the same
    trimmed network bit for bit (about 2 million kept edges)."""
    from tenex_b200.inference.fdr import _offdiag, threshold_pairs_device
    M = full_size_multibin["matrix"]
    n = M.shape[0]
    te_t, pairs_t = _offdiag(M)
    te_d, pairs_d = threshold_pairs_device(te_t, pairs_t, fdr=0.01)
    kept = te_d.numel()
    assert 0 < kept < te_t.numel()
    at_or_above = int((te_t >= te_d.min()).sum())
    assert kept <= at_or_above <= kept + 2      # ulp-level wiggles of erfc at the cut at most
    A = torch.zeros((n, n), dtype=torch.float32, device=cuda)
    A[pairs_d[:, 0], pairs_d[:, 1]] = te_d
    med = A.sum(dim=1) > 0
    dense = dpi_trim_matrix(A, med, None, 0.0)
    r, c = torch.nonzero(dense, as_tuple=True)
    rs, cs, vs = dpi_trim_sparse(A, med, None, 0.0)
    assert torch.equal(rs, r) and torch.equal(cs, c)
    assert torch.equal(vs.view(torch.int32), dense[r, c].view(torch.int32))
    assert 0 < r.numel() < kept
    assert torch.all(A[r, c] == dense[r, c])           # trimming only removes edges
