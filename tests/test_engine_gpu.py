"""End-to-end engine and preprocessing kernels against the reference goldens / oracle."""
import warnings

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200 import TransferEntropyEngine, workloads as W
from tenex_b200.kernels import device as D
from tenex_b200.kernels.adaptive_smem import AdaptiveSMEMKernel
from tenex_b200.preprocess import coarsen_bins, discretize, fsbwl_bins, remap_bins

pytestmark = pytest.mark.gpu
TOL = 1e-6


def test_engine_cfg1_golden(cuda, golden):
    g = golden("discretize_cfg1.npz")
    names = np.array([f"g{i}" for i in range(g["x"].shape[0])])
    res = TransferEntropyEngine(g["x"], names).compute(accelerator="gpu", profile=True)
    assert res.kernel == "Full-SMEM"
    assert np.array_equal(res.bin_arrs[:, :, 0].astype(np.int32), g["bins"][:, :, 0])
    assert np.array_equal(res.n_per_var, g["n_per_var"])
    assert res.b_max == int(g["b_max"])
    assert np.max(np.abs(res.matrix - g["matrix"])) <= TOL
    assert np.all(np.diag(res.matrix) == 0)
    assert set(res.timings) >= {"total", "discretize", "compute"}


@pytest.mark.parametrize("n,T", [(7, 1), (9, 7), (33, 128), (31, 129), (40, 1000), (12, 5003),
                                 (6, 20001), (3, 114689), (3, 300007)])
def test_fsbwl_bitexact_vs_numpy(cuda, n, T):
    rng = np.random.default_rng(n * T)
    x = np.log1p(rng.lognormal(0, 1, (n, T)) * (rng.random((n, T)) > 0.6)).astype(np.float32)
    x[0] = 1.5  # constant row: std 0 -> 1
    bins, nb = fsbwl_bins(x, 0.5, cuda)
    rb, rnb = O.fsbwl(x, 0.5)
    assert np.array_equal(nb.cpu().numpy(), rnb)
    assert np.array_equal(bins.cpu().numpy(), rb)


def test_compute_on_series_longer_than_shared_memory(cuda):
    """compute(accelerator="gpu") on 6 genes x 150,000 cells: FSBW-L over rows
    longer than one shared-memory pass of the pairwise sum, and TE launches whose
    target states are staged in tiles. Bins equal the oracle's, TE within 1e-6."""
    x, _ = W.cfg1_expression(n=6, T=150_000, seed=12, n_planted=2)
    names = np.array([f"g{i}" for i in range(6)])
    res = TransferEntropyEngine(x, names).compute(accelerator="gpu")
    rb, _ = O.fsbwl(x, 0.5)
    bins, npv, bmax = O.remap(rb)
    if bmax > 38:                                    # the B200 coarsening limit
        bins, npv, bmax = O.coarsen(bins, npv, 38)
    assert np.array_equal(res.bin_arrs[:, :, 0].astype(np.int32), bins)
    assert np.max(np.abs(res.matrix - O.te_matrix(bins, npv))) <= TOL


def test_remap_and_discretize_match_reference(cuda, golden):
    g = golden("remap.npz")
    db, npv, bmax = remap_bins(g["raw"], 1, cuda)
    assert np.array_equal(db.unpadded()[:, :, 0].cpu().numpy().astype(np.int32), g["remapped"])
    assert np.array_equal(npv.cpu().numpy(), g["n_per_var"])
    assert bmax == int(g["b_max"])
    c = golden("discretize_cfg1.npz")
    db2, nb2, bmax2, npv2 = discretize(c["x"], "FSBW-L", 0.5, cuda)
    assert np.array_equal(db2.unpadded()[:, :, 0].cpu().numpy().astype(np.int32),
                          c["bins"][:, :, 0])
    assert np.array_equal(nb2.cpu().numpy(), c["n_bins"])


def test_coarsen_matches_reference(cuda, golden):
    g = golden("coarsen.npz")
    db = D.pack_bins(g["bins"], cuda)
    db, npv, bmax = coarsen_bins(db, torch.as_tensor(g["n_per_var"], device=cuda), int(g["limit"]))
    assert np.array_equal(db.unpadded()[:, :, 0].cpu().numpy().astype(np.int32), g["out"])
    assert np.array_equal(npv.cpu().numpy(), g["out_npv"])
    assert bmax == int(g["out_bmax"])


def test_genes_with_more_than_256_bins(cuda, golden):
    """Genes of 257, 300 and 1000 distinct bins (the reference keeps them as int16
    until coarsened): remap_bins keeps uint16 rows, AdaptiveSMEMKernel.prepare
    coarsens them to the B200 limit (38) into uint8 rows equal to the reference's
    coarsen_bins output, and the TE of all pairs is within 1e-6 of the oracle on
    those bins. The uint16 bins themselves are refused by the TE kernels."""
    from tenex_b200.preprocess import remap_bins
    g = golden("coarsen_wide.npz")
    db, npv, bmax = remap_bins(g["raw"], 1, cuda)
    assert db.wide and bmax == int(g["b_max"]) == 1000
    assert np.array_equal(db.unpadded()[:, :, 0].cpu().numpy().astype(np.int32), g["remapped"])
    assert np.array_equal(npv.cpu().numpy(), g["n_per_var"])
    k = AdaptiveSMEMKernel()
    with pytest.raises(ValueError, match="256"):
        k.compute_pairfree_device(db, npv, bmax, 1)
    with pytest.raises(ValueError, match="256"):
        k.prepare(db, npv.clone(), bmax, tau=1, use_coarsening=False, smem_optin=232448)
    db2, npv2, bmax2 = k.prepare(db, npv.clone(), bmax, tau=1, smem_optin=232448)
    assert not db2.wide and bmax2 == int(g["out_bmax"]) == 38
    assert np.array_equal(db2.unpadded()[:, :, 0].cpu().numpy().astype(np.int32), g["out"])
    assert np.array_equal(npv2.cpu().numpy(), g["out_npv"])
    te = k.compute_pairfree_device(db2, npv2, bmax2, 1).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(g["out"], g["out_npv"]))) <= TOL
    # the plugin's host entry takes the raw int32 bins the same way once remapped
    with pytest.raises(ValueError, match="255"):
        D.pack_bins(g["raw"], cuda)


def test_adaptive_prepare_and_heavy_genes(cuda):
    x, npv = W.multibin(40, 1500, 4, 2, 16, heavy_frac=0.25, heavy_lo=64, heavy_hi=200)
    db = D.pack_bins(x, cuda)
    k = AdaptiveSMEMKernel()
    db2, npv2, bmax2 = k.prepare(db, torch.as_tensor(npv, device=cuda), int(npv.max()), tau=1,
                                 smem_optin=232448)
    assert bmax2 == 38
    cb, cnpv, cbmax = O.coarsen(x, npv, 38)
    assert np.array_equal(db2.unpadded()[:, :, 0].cpu().numpy().astype(np.int32), cb)
    te = k.compute_pairfree_device(db2, npv2, bmax2, 1).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(cb, cnpv))) <= TOL


def test_adaptive_no_coarsening_uses_overflow(cuda):
    # use_coarsening=False: heavy genes keep all their bins; their pairs run in the
    # global-memory overflow launch and TE equals the oracle on the raw bins
    x, npv = W.multibin(24, 1200, 6, 2, 12, heavy_frac=0.25, heavy_lo=60, heavy_hi=120)
    db = D.pack_bins(x, cuda)
    k = AdaptiveSMEMKernel()
    bmax = int(npv.max())
    db2, npv2, bmax2 = k.prepare(db, torch.as_tensor(npv, device=cuda), bmax, tau=1,
                                 use_coarsening=False, smem_optin=232448)
    assert bmax2 == bmax > 38
    te = k.compute_pairfree_device(db2, npv2, bmax2, 1).cpu().numpy()
    assert np.max(np.abs(te - O.te_pairfree(x, npv))) <= TOL
    with pytest.raises(ValueError, match="256"):
        k.prepare(db, torch.as_tensor(npv, device=cuda), 256, tau=1, use_coarsening=False,
                  smem_optin=232448)


@pytest.mark.parametrize("T", [400, 401])
@pytest.mark.parametrize("method,q,tag", [("nonzero", None, "nonzero"), ("mean", None, "mean"),
                                          ("median", None, "median"), ("quantile", 0.7, "q70"),
                                          ("quantile", 0.25, "q25")])
def test_binarization_routes_to_gemm_b2(cuda, golden, method, q, tag, T):
    """Bins bit-equal to the reference's binarize (numpy backend, its default) on
    expression data with many ties, at an even and an odd series length; the
    binary matrix goes through GEMM-B2 and matches the oracle."""
    g = golden("binarize.npz")
    x = g[f"x{T}"]
    names = np.array([f"g{i}" for i in range(x.shape[0])])
    res = TransferEntropyEngine(x, names).compute(
        accelerator="gpu", binarization=method,
        binarization_kwargs={"q": q} if q is not None else None)
    assert res.kernel == "GEMM-B2"
    b = res.bin_arrs[:, :, 0].astype(np.uint8)
    assert np.array_equal(b, g[f"{tag}{T}"])
    ref = O.te_matrix(b, np.full(x.shape[0], 2, np.int32))
    assert np.max(np.abs(res.matrix - ref)) <= TOL


@pytest.mark.parametrize("n,T", [(3, 1), (3, 7), (5, 8), (5, 9), (40, 128), (40, 129), (40, 1000),
                                 (2000, 4099), (2000, 20000), (64, 114688), (8, 114689),
                                 (4, 250000)])
def test_mean_binarisation_bitexact_vs_numpy(cuda, n, T):
    """The mean binariser against numpy's float32 np.mean (pairwise sum, float64
    division) at lengths that reach every leaf shape of the pairwise tree, the
    persistent plan kernel with more genes than CTAs (n = 2000) and the
    super-node kernel beyond one plan (T > 114688); NaN / inf rows included."""
    from tenex_b200.binarize import binarize
    rng = np.random.default_rng(T)
    x = (rng.standard_normal((n, T)) * 10.0 ** rng.uniform(-3, 3, (n, 1))).astype(np.float32)
    x[rng.random((n, T)) < 0.3] = 0
    x[0] = 1.5                                               # constant row
    if n > 2:
        x[1, T // 2] = np.nan
        x[2, 0] = np.inf
    db, npv, _, _ = binarize(x, "mean", device=cuda)
    with np.errstate(invalid="ignore"):
        ref = (x > np.mean(x, axis=1, keepdims=True)).astype(np.uint8)
    got = D.to_host(db.unpadded()).reshape(n, T)
    assert np.array_equal(got, ref)
    ref_npv = np.where(ref.max(axis=1) != ref.min(axis=1), 2, 1)
    assert np.array_equal(npv.cpu().numpy(), ref_npv)


@pytest.mark.parametrize("n,T", [(4, 1), (4, 2), (6, 7), (40, 400), (40, 401), (2000, 20000),
                                 (16, 57088), (8, 70000)])
@pytest.mark.parametrize("method,q", [("median", 0.5), ("quantile", 0.0), ("quantile", 0.25),
                                      ("quantile", 0.7), ("quantile", 0.999),
                                      ("quantile", 1.0)])
def test_select_binarisation_bitexact_vs_numpy(cuda, n, T, method, q):
    """Median / quantile binarisation against numpy's np.median / np.quantile
    (the reference's numpy backend): rows staged in shared memory (T a multiple
    of 4 up to the opt-in size) and read from global memory (odd T, T = 70000),
    heavy ties (zeros, a few repeated levels), a NaN row (numpy's threshold is
    NaN: all bins 0), an inf row and a constant row."""
    from tenex_b200.binarize import binarize
    rng = np.random.default_rng(T + int(q * 1000))
    x = (rng.standard_normal((n, T)) * 10.0 ** rng.uniform(-3, 3, (n, 1))).astype(np.float32)
    x[rng.random((n, T)) < 0.4] = 0
    x[rng.random((n, T)) < 0.1] = np.float32(2.5)
    x[0] = -0.0
    if n > 3:
        x[1, T // 2] = np.nan
        x[2, 0] = np.inf
        x[3, : T // 2] = -np.inf
    db, npv, _, _ = binarize(x, method, device=cuda, q=q)
    with np.errstate(invalid="ignore"), warnings.catch_warnings():
        warnings.simplefilter("ignore", RuntimeWarning)
        thr = (np.median(x, axis=1, keepdims=True) if method == "median"
               else np.quantile(x, q, axis=1, keepdims=True))
        ref = (x > thr).astype(np.uint8)
    got = D.to_host(db.unpadded()).reshape(n, T)
    assert np.array_equal(got, ref)
    ref_npv = np.where(ref.max(axis=1) != ref.min(axis=1), 2, 1)
    assert np.array_equal(npv.cpu().numpy(), ref_npv)


def test_source_filter_pair_list(cuda, golden):
    g = golden("discretize_cfg1.npz")
    n = g["x"].shape[0]
    names = np.array([f"g{i}" for i in range(n)])
    srcs = names[[3, 7, 11, 20]]
    res = TransferEntropyEngine(g["x"], names, sources=srcs).compute(accelerator="gpu")
    full = g["matrix"]
    for s in (3, 7, 11, 20):
        row = full[s].copy()
        row[s] = 0.0
        assert np.max(np.abs(res.matrix[s] - row)) <= TOL
    other = np.setdiff1d(np.arange(n), [3, 7, 11, 20])
    assert np.all(res.matrix[other] == 0)


def test_engine_contracts(cuda):
    x, _ = W.cfg1_expression(n=10, T=200, seed=1)
    names = np.array([f"g{i}" for i in range(10)])
    eng = TransferEntropyEngine(x, names)
    with pytest.raises(ValueError):
        eng.compute(accelerator="gpu", kernel="GEMM-B2")
    with pytest.raises(KeyError):
        eng.compute(accelerator="gpu", kernel="nope")
    with pytest.raises(ValueError):
        eng.compute(accelerator="gpu", tau=0)
    r = TransferEntropyEngine(x[:1], names[:1]).compute(accelerator="gpu")
    assert r.matrix.shape == (1, 1) and r.matrix[0, 0] == 0
    r2 = eng.compute(accelerator="gpu", kernel="Adaptive-SMEM", tau=2)
    ref = O.te_matrix(r2.bin_arrs, r2.n_per_var, tau=2)
    assert np.max(np.abs(r2.matrix - ref)) <= TOL


def test_multi_device_and_cross_block_entry_points(cuda):
    from oracle import oracle as O
    from tenex_b200.kernels import get_kernel
    rng = np.random.default_rng(12)
    n, T = 30, 900
    b = rng.integers(2, 12, n)
    x = np.stack([rng.integers(0, bb, T) for bb in b]).astype(np.int32)
    bins, npv, bmax = O.remap(x)
    ref = O.te_matrix(bins, npv)                      # [src, tgt]
    k = get_kernel("Adaptive-SMEM")
    pairs = np.stack(np.nonzero(~np.eye(n, dtype=bool)), axis=1)[::3][:, ::-1].copy()  # [tgt, src]
    bt = torch.from_numpy(bins.reshape(n, T, 1).astype(np.uint8))
    npv_t = torch.from_numpy(npv.astype(np.int32))
    single = k.compute_single_gpu(bt, pairs, bmax, npv_t, 1, None, cuda)
    for ids in ([0], [0, 0]):                         # two host threads may share a device
        multi = k.compute_multi_gpu(bt, pairs, bmax, npv_t, 1, None, ids)
        assert np.array_equal(multi, single)
    assert np.max(np.abs(single - ref[pairs[:, 1], pairs[:, 0]])) <= 1e-6
    # cross block: targets 0..9 against sources 20..29, pair id = tgt_local * n_src + src_local
    tg, sr = np.arange(10), np.arange(20, 30)
    sub = np.concatenate([tg, sr])
    cross = k.compute_pairfree_cross(bt[sub], npv_t[sub], 10, 10, 1, cuda)
    want = ref[np.ix_(sr, tg)].T.reshape(-1)          # [tgt_local, src_local]
    assert np.max(np.abs(cross - want)) <= 1e-6
    part = k.compute_pairfree_cross(bt[sub], npv_t[sub], 10, 10, 1, cuda, pair_offset=37,
                                    n_pairs_local=21)
    assert np.array_equal(part, cross[37:58])
    # the binary matrix kernel's multi-device entry
    xb = (rng.random((20, 400)) < 0.4).astype(np.int32)
    xb[:, :2] = [1, 0]
    g = get_kernel("GEMM-B2")
    m1 = g.compute_matrix(xb[..., None], 20, 1, cuda)
    m2 = g.compute_matrix_multi_gpu(xb[..., None], 20, 1, [0])
    assert np.array_equal(m1, m2)


def test_compute_over_several_devices(cuda):
    # devices=[0, 0]: two host threads, two pair-id chunks (one device here, the
    # same code path as two GPUs); equal to the single-device matrix
    x, _ = W.cfg1_expression(n=40, T=300, seed=3)
    names = np.array([f"g{i}" for i in range(40)])
    one = TransferEntropyEngine(x, names).compute(accelerator="gpu", devices=[0]).matrix
    two = TransferEntropyEngine(x, names).compute(accelerator="gpu", devices=[0, 0])
    assert np.max(np.abs(two.matrix - one)) <= 1e-6
    assert np.all(np.diag(two.matrix) == 0)
    tf = names[:6]
    a = TransferEntropyEngine(x, names, sources=tf).compute(accelerator="gpu", devices=[0]).matrix
    b = TransferEntropyEngine(x, names, sources=tf).compute(accelerator="gpu", devices=[0, 0]).matrix
    assert np.max(np.abs(a - b)) <= 1e-6
    xb = (np.random.default_rng(4).random((25, 300)) < 0.4).astype(np.float32)
    nb = np.array([f"b{i}" for i in range(25)])
    c = TransferEntropyEngine(xb, nb).compute(accelerator="gpu", devices=[0],
                                              binarization="nonzero").matrix
    d = TransferEntropyEngine(xb, nb).compute(accelerator="gpu", devices=[0, 0],
                                              binarization="nonzero").matrix
    assert np.array_equal(c, d)


@pytest.mark.parametrize("dtype,shape", [(np.float32, (2500, 2500)), (np.uint8, (3, 20_000_011)),
                                         (np.int16, (4097, 4099)), (np.float64, (7,)),
                                         (np.int64, (9_000_001,))])
def test_staged_host_copy_equals_plain_copy(cuda, dtype, shape):
    """to_device (page-locked staging chunks filled by host threads) gives the
    same tensor as a plain copy: sizes below, at and across chunk boundaries,
    several dtypes, and a non-contiguous source."""
    rng = np.random.default_rng(7)
    if np.issubdtype(dtype, np.integer):
        info = np.iinfo(dtype)
        a = rng.integers(info.min, info.max, size=shape, dtype=dtype, endpoint=True)
    else:
        a = (rng.standard_normal(shape) * 100).astype(dtype)
    t = D.to_device(a, cuda)
    assert t.dtype == torch.as_tensor(a).dtype and tuple(t.shape) == a.shape
    assert torch.equal(t.cpu(), torch.as_tensor(a))
    if a.ndim == 2:
        b = a.T                                           # non-contiguous view
        assert torch.equal(D.to_device(b, cuda).cpu(), torch.as_tensor(np.ascontiguousarray(b)))
    src = torch.as_tensor(a)
    assert torch.equal(D.to_device(src, cuda).cpu(), src)


@pytest.mark.parametrize("dtype,shape", [(torch.float32, (4000, 4000)), (torch.int64, (9_000_001,)),
                                         (torch.bool, (3, 30_000_001)), (torch.uint8, (5_000_000,)),
                                         (torch.float64, (1000, 3))])
def test_staged_device_copy_back_equals_plain(cuda, dtype, shape):
    """to_host (DMA into two page-locked chunks, host threads copying out) gives
    the array a plain .cpu().numpy() gives: sizes below, at and across the
    32 MB chunks, several dtypes, a non-contiguous source."""
    g = torch.Generator(device=cuda).manual_seed(11)
    if dtype == torch.bool:
        t = torch.rand(shape, generator=g, device=cuda) > 0.5
    elif dtype.is_floating_point:
        t = torch.randn(shape, generator=g, device=cuda, dtype=dtype)
    else:
        t = torch.randint(0, 200, shape, generator=g, device=cuda, dtype=dtype)
    h = D.to_host(t)
    ref = t.cpu().numpy()
    assert h.dtype == ref.dtype and h.shape == ref.shape and np.array_equal(h, ref)
    if t.dim() == 2:
        assert np.array_equal(D.to_host(t.t()), t.t().cpu().numpy())
