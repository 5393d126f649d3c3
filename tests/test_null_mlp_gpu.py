"""Learned-null kernels: features, forward and gradients against the float64 oracle."""
import numpy as np
import pytest
import torch

from oracle import mlp_oracle as M
from tenex_b200 import native, workloads as W
from tenex_b200.inference import learned_null as LN
from tenex_b200.kernels import device as D

pytestmark = pytest.mark.gpu


def test_gene_features_match_numpy(cuda):
    x, npv, _ = W.cfg5_bins(n=40, T=900, seed=8)
    db = D.pack_bins(x, cuda)
    gf = LN.gene_features(db, torch.as_tensor(npv, device=cuda), 1).cpu().numpy()
    ref = M.gene_features(x, npv, 1)
    assert np.allclose(gf[:, :6], ref, rtol=1e-5, atol=1e-5)


def test_mlp_gradients_match_float64_oracle(cuda):
    rng = np.random.default_rng(3)
    p = LN.init_params(rng)
    p[1024:1088] = rng.normal(0, 0.1, 64)  # non-zero biases exercise those terms
    B = 96
    X = rng.normal(0, 1, (B, 16)).astype(np.float32)
    Y = rng.normal(0, 1, (B, 2)).astype(np.float32)
    pt = torch.from_numpy(p).to(cuda)
    wb = torch.empty(p.size, dtype=torch.bfloat16, device=cuda)
    native.call("tenex_to_bf16", pt.data_ptr(), wb.data_ptr(), p.size, native.stream_ptr())
    scratch = torch.empty(int(native.lib().tenex_mlp_scratch_floats(B)), device=cuda)
    grad = torch.empty(p.size, device=cuda)
    loss = torch.zeros(1, device=cuda)
    Xd, Yd = torch.from_numpy(X).to(cuda), torch.from_numpy(Y).to(cuda)
    native.call("tenex_mlp_gradients", Xd.data_ptr(), Yd.data_ptr(), B, wb.data_ptr(),
                scratch.data_ptr(), grad.data_ptr(), loss.data_ptr(), native.stream_ptr())
    g_ref, l_ref = M.gradients(M.bf16_round(p), X.astype(np.float64), Y.astype(np.float64))
    g = grad.cpu().numpy()
    assert abs(float(loss.item()) - l_ref) <= 1e-4 * abs(l_ref) + 1e-5
    assert np.max(np.abs(g - g_ref)) <= 2e-4 * np.max(np.abs(g_ref)) + 1e-6


def test_eiid_matches_float64_series(cuda):
    # E_iid = sum g(n_a q_b) - sum g(n_x q_b); the kernel's g is a 1024-point table
    # with its two analytic limits, the oracle sums the Poisson series directly.
    x, npv, _ = W.cfg5_bins(n=30, T=800, seed=9)
    npv = npv.copy()
    x[3] = (np.arange(800) * 7 % 70).astype(np.uint8)   # one gene with 70 states: NaN row/col
    npv[3] = 70
    db = D.pack_bins(x, cuda)
    got = LN.eiid_matrix(db, torch.as_tensor(npv, dtype=torch.int32, device=cuda), 1).cpu().numpy()
    ref = M.eiid(x, npv, 1)
    off = ~np.eye(30, dtype=bool)
    assert np.array_equal(np.isnan(got[off]), np.isnan(ref[off]))
    ok = off & ~np.isnan(ref)
    assert np.isnan(got[3, 5]) and np.isnan(got[5, 3])
    assert np.allclose(got[ok], ref[ok], rtol=2e-4, atol=1e-3)


def test_null_predict_matches_float64_forward(cuda):
    x, npv, _ = W.cfg5_bins(n=30, T=800, seed=9)
    db = D.pack_bins(x, cuda)
    npv_t = torch.as_tensor(npv, device=cuda)
    rng = np.random.default_rng(5)
    gf_np = np.concatenate([M.gene_features(x, npv, 1), np.zeros((30, 2))], 1)
    model = LN.NullModel(LN.init_params(rng), np.zeros(16, np.float32),
                         np.full(16, 4.0, np.float32), gf_np[:, :6].min(0) - 1,
                         gf_np[:, :6].max(0) + 1, {})
    mu, sg, ok = LN.predict(model, db, npv_t, 1, 50)
    assert bool(ok.all())
    t, s = np.meshgrid(np.arange(30), np.arange(30), indexing="ij")
    m = t != s
    tt, ss = t[m], s[m]
    gf = LN.gene_features(db, npv_t, 1)
    eiid = LN.eiid_matrix(db, npv_t, 1)
    Xr = LN.pair_features(gf, eiid, torch.as_tensor(tt, dtype=torch.int32, device=cuda),
                          torch.as_tensor(ss, dtype=torch.int32, device=cuda), 50).cpu().numpy()
    # the kernel's features equal the oracle's restatement on the kernel's inputs
    Xo = M.pair_features(gf.cpu().numpy()[:, :6], eiid.cpu().numpy(), tt, ss, 50)
    assert np.allclose(Xr, Xo, rtol=1e-5, atol=1e-5)
    out = M.forward(M.bf16_round(model.params), Xr.astype(np.float64) / 4.0)
    N = 799
    ref_mu = np.exp(out[:, 0]) / N
    got_mu = mu.cpu().numpy()[ss, tt]
    assert np.allclose(got_mu, ref_mu, rtol=2e-4)


def test_training_reduces_loss(cuda):
    rng = np.random.default_rng(0)
    X = torch.from_numpy(rng.normal(0, 1, (20000, 16)).astype(np.float32)).to(cuda)
    Y = torch.stack([torch.sin(X[:, 0]) + 0.5 * X[:, 1], X[:, 2] * X[:, 3] * 0.3], 1)
    model, rep = LN.train(X, Y, torch.zeros((4, 6), device=cuda), steps=400, batch=1024,
                          lr=3e-3, Xval=X[:2000], Yval=Y[:2000])
    h = rep["loss_history"]
    assert h[-1][1] < 0.5 * h[0][1]       # mean loss of steps 251-400 vs steps 1-250
    assert max(rep["val_mse"]) < 0.05


def test_eiid_count_table_equals_pair_loop(cuda):
    # E_iid of a pair depends only on its two genes: with 200 genes the kernel
    # tabulates the target sums over counts (N + 1 <= 4 n), with 20 of the same genes
    # it sums per pair; the two must agree bit for bit
    x, npv, _ = W.cfg5_bins(n=200, T=500, seed=41)
    sub = np.arange(0, 200, 10)
    full = LN.eiid_matrix(D.pack_bins(x, cuda), torch.as_tensor(npv, dtype=torch.int32,
                                                                 device=cuda), 1).cpu().numpy()
    part = LN.eiid_matrix(D.pack_bins(x[sub], cuda),
                          torch.as_tensor(npv[sub], dtype=torch.int32, device=cuda),
                          1).cpu().numpy()
    want = full[np.ix_(sub, sub)]
    off = ~np.eye(len(sub), dtype=bool)
    assert np.array_equal(part[off].view(np.uint32), want[off].view(np.uint32))
