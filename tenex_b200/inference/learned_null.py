"""Learned null model for the surrogate test (no reference counterpart).

The block-shuffle surrogate test spends S full TE matrices to estimate, per
pair, the mean and spread of TE under the null. That distribution depends on
cheap per-gene statistics (bin counts, marginal and lag-1 joint entropies,
autocorrelation, run lengths) and on N and the block length, not on the
pair's coupling. A small MLP (16 -> 64 -> 64 -> 2, GELU, BF16 weights, FP32
accumulation; kernels in null_mlp.cu) predicts log(mu*N) and log(sigma*N) of
the null from those features and one pair-level statistic, E_iid: the
expected plug-in bias of N ln2 * TE under independence with Poisson cell
counts, sum_{a,b} g(n_a q_b) - sum_{x,b} g(n_x q_b), g(m) = E[C ln C] - m ln m
(the small-count behaviour of sparse tables; tenex_eiid_matrix).

Training: synthetic datasets from generator seeds disjoint from evaluation
(2000-2019 by default); each is run through the full surrogate test (S
shuffles, permutation seeds disjoint from evaluation too), and the per-pair
surrogate mean / std are the targets. Everything runs on the GPU through this
package's kernels (features, forward, backward, Adam).

Inference (null="learned" in SurrogateTestMethod.infer): predicted mu, sigma
give z = (TE_obs - mu) / sigma and parametric p-values; the BH-FDR threshold of
those p-values gives z_FDR. Every pair with z >= z_FDR - band (the band is
calibrated on held-out seeds and stored with the model), every pair whose genes
fall outside the features seen in training, and every pair with undefined
features goes to the full block-shuffle surrogate test (pair-list kernel, the
full test's own permutations and the same per-pair histogram counts, so those
pairs get the full test's statistics up to the float rounding of each pair's
entropy sum, whose reduction order follows the launch's warp grouping). BH is
then recomputed over the mixed p-values and the screen is
widened while z_FDR - band keeps falling. Called edges are therefore always
verified by the full test; the band only decides how many true edges could be
missed (pairs whose predicted z falls more than `band` below z_FDR). When more
than half of the pairs cannot be scored (data unlike the training set: other
series lengths, block lengths or bin statistics), the full test runs instead.
"""
from __future__ import annotations

import argparse
import os
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from tenex_b200 import _log, native
from tenex_b200.kernels import device as D

GENE_FEAT = 8
N_IN = 16
DEFAULT_MODEL = os.path.join(os.path.dirname(os.path.abspath(__file__)), "null_model_cfg5.npz")


def n_params() -> int:
    return int(native.lib().tenex_mlp_param_count())


def init_params(rng: np.random.Generator) -> np.ndarray:
    """He-style initialisation of W1, W2, W3 (biases zero), FP32."""
    H = 64
    w1 = rng.normal(0, np.sqrt(2.0 / N_IN), (H, N_IN))
    w2 = rng.normal(0, np.sqrt(2.0 / H), (H, H))
    w3 = rng.normal(0, np.sqrt(1.0 / H), (2, H))
    return np.concatenate([w1.ravel(), np.zeros(H), w2.ravel(), np.zeros(H), w3.ravel(),
                           np.zeros(2)]).astype(np.float32)


@dataclass
class NullModel:
    params: np.ndarray            # FP32 master parameters
    feat_mean: np.ndarray         # (16,)
    feat_std: np.ndarray          # (16,)
    gene_lo: np.ndarray           # (6,) per-gene feature range seen in training
    gene_hi: np.ndarray
    meta: dict = field(default_factory=dict)
    _dev_cache: dict = field(default_factory=dict, repr=False, compare=False)

    def save(self, path: str) -> None:
        np.savez(path, params=self.params, feat_mean=self.feat_mean, feat_std=self.feat_std,
                 gene_lo=self.gene_lo, gene_hi=self.gene_hi,
                 meta=np.array(repr(self.meta)))

    @staticmethod
    def load(path: str = DEFAULT_MODEL) -> "NullModel":
        if not os.path.exists(path):
            raise FileNotFoundError(
                f"{path} not found; train a model with "
                f"`python -m tenex_b200.inference.learned_null --train`")
        z = np.load(path, allow_pickle=False)
        import ast
        return NullModel(z["params"].astype(np.float32), z["feat_mean"], z["feat_std"],
                         z["gene_lo"], z["gene_hi"], ast.literal_eval(str(z["meta"])))

    def device_weights(self, dev) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """BF16 weights and the feature standardisation on `dev` (made once per device)."""
        key = str(torch.device(dev))
        if key not in self._dev_cache:
            self._dev_cache[key] = self._to_device(dev)
        return self._dev_cache[key]

    def _to_device(self, dev):
        master = torch.from_numpy(self.params).to(dev)
        wb = torch.empty(master.numel(), dtype=torch.bfloat16, device=dev)
        native.call("tenex_to_bf16", master.data_ptr(), wb.data_ptr(), master.numel(),
                    native.stream_ptr())
        return (wb, torch.from_numpy(self.feat_mean.astype(np.float32)).to(dev),
                torch.from_numpy(self.feat_std.astype(np.float32)).to(dev))


def gene_features(db: D.DeviceBins, npv: torch.Tensor, tau: int) -> torch.Tensor:
    """(n, 8) float32 per-gene features on the device."""
    feat = torch.empty((db.n, GENE_FEAT), dtype=torch.float32, device=db.data.device)
    native.call("tenex_gene_features", db.ptr(), db.ld, npv.data_ptr(), db.n,
                db.row_len, tau * db.K, feat.data_ptr(), native.stream_ptr())
    return feat


def eiid_matrix(db: D.DeviceBins, npv: torch.Tensor, tau: int) -> torch.Tensor:
    """(n, n) float32 [src, tgt] independence bias E_iid of every ordered pair."""
    dev = db.data.device
    out = torch.empty((db.n, db.n), dtype=torch.float32, device=dev)
    ws = torch.empty(int(native.lib().tenex_eiid_workspace_bytes(db.n)), dtype=torch.uint8,
                     device=dev)
    native.call("tenex_eiid_matrix", db.ptr(), db.ld, npv.data_ptr(), db.n,
                db.row_len, tau * db.K, out.data_ptr(), ws.data_ptr(), ws.numel(),
                native.stream_ptr())
    return out


def pair_features(gf: torch.Tensor, eiid: torch.Tensor, tgt: torch.Tensor, src: torch.Tensor,
                  block_length: int) -> torch.Tensor:
    """Raw (n_pairs, 16) features of the [tgt, src] pairs."""
    P = int(tgt.numel())
    X = torch.empty((P, N_IN), dtype=torch.float32, device=gf.device)
    native.call("tenex_pair_features", gf.data_ptr(), eiid.data_ptr(), int(eiid.shape[0]),
                tgt.data_ptr(), src.data_ptr(), P, float(np.log2(block_length)), X.data_ptr(),
                native.stream_ptr())
    return X


def predict(model: NullModel, db: D.DeviceBins, npv: torch.Tensor, tau: int, block_length: int,
            gf: torch.Tensor | None = None):
    """Null mean and std of TE for every ordered pair ([src, tgt], float32 device
    tensors, NaN where undefined) and a per-gene in-range flag."""
    dev = db.data.device
    n = db.n
    N = (db.T - tau) * db.K
    if gf is None:
        gf = gene_features(db, npv, tau)
    eiid = eiid_matrix(db, npv, tau)
    wb, fm, fs = model.device_weights(dev)
    lmu = torch.full((n, n), float("nan"), dtype=torch.float32, device=dev)
    lsg = torch.full((n, n), float("nan"), dtype=torch.float32, device=dev)
    native.call("tenex_null_predict", gf.data_ptr(), eiid.data_ptr(), n,
                float(np.log2(block_length)), wb.data_ptr(), fm.data_ptr(), fs.data_ptr(),
                lmu.data_ptr(), lsg.data_ptr(), native.stream_ptr())
    mu = torch.exp(lmu) / N
    sigma = torch.exp(lsg) / N
    lo = torch.from_numpy(model.gene_lo.astype(np.float32)).to(dev)
    hi = torch.from_numpy(model.gene_hi.astype(np.float32)).to(dev)
    g6 = gf[:, :6]
    in_range = ((g6 >= lo) & (g6 <= hi)).all(dim=1) & torch.isfinite(g6).all(dim=1)
    meta = model.meta
    if "N" in meta and abs(np.log2(N) - np.log2(meta["N"])) > 0.5:
        in_range[:] = False
    if "block_length" in meta and abs(np.log2(block_length) - np.log2(meta["block_length"])) > 0.5:
        in_range[:] = False
    return mu, sigma, in_range


# --------------------------------------------------------------------------- training
def surrogate_moments(db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int, S: int,
                      block_length: int, seed: int) -> tuple[torch.Tensor, torch.Tensor]:
    """Per-pair mean and population std of the surrogate TE ([src, tgt], device)."""
    from tenex_b200.inference.surrogate_test import (SurrogateAccumulator, build_block_perm,
                                                     run_surrogates)
    n = db.n
    obs = torch.zeros((n, n), dtype=torch.float32, device=db.data.device)
    acc = SurrogateAccumulator(db, npv, b_max, tau, obs, b_max == 2)
    perms, bl, _ = build_block_perm(n, db.T, "block", block_length, 0, S, seed, db.data.device)
    run_surrogates(acc, perms, bl)
    mean = acc.sum / S
    var = acc.sumsq / S - mean * mean
    return mean.float(), torch.sqrt(torch.clamp(var, min=0.0)).float()


def training_set(seeds, n: int, T: int, S: int, block_length: int, pairs_per_dataset: int,
                 dev, tau: int = 1):
    """Raw features X (P, 16) and targets Y (P, 2) = log(mu*N), log(sigma*N) on the device."""
    from tenex_b200 import workloads as W
    Xs, Ys, G = [], [], []
    N = T - tau
    rng = np.random.default_rng(12345)
    for sd in seeds:
        x, npv, _ = W.cfg5_bins(n=n, T=T, seed=int(sd))
        db = D.pack_bins(x, dev)
        npv_t = torch.as_tensor(npv, dtype=torch.int32, device=dev)
        b_max = int(npv.max())
        mean, std = surrogate_moments(db, npv_t, b_max, tau, S, block_length, 10_000 + int(sd))
        gf = gene_features(db, npv_t, tau)
        eiid = eiid_matrix(db, npv_t, tau)
        t = rng.integers(0, n, pairs_per_dataset)
        s = rng.integers(0, n - 1, pairs_per_dataset)
        s = s + (s >= t)
        tt = torch.as_tensor(t, dtype=torch.int32, device=dev)
        ss = torch.as_tensor(s, dtype=torch.int32, device=dev)
        X = pair_features(gf, eiid, tt, ss, block_length)
        mu = mean[ss.long(), tt.long()]
        sg = std[ss.long(), tt.long()]
        ok = torch.isfinite(X).all(dim=1) & (mu > 0) & (sg > 0)
        Y = torch.stack([torch.log(mu * N), torch.log(sg * N)], dim=1)
        Xs.append(X[ok])
        Ys.append(Y[ok])
        G.append(gf[:, :6])
        _log.vprint(f"[TENEX] null training data: seed {sd}, {int(ok.sum())} pairs")
    return torch.cat(Xs), torch.cat(Ys), torch.cat(G)


def train(X: torch.Tensor, Y: torch.Tensor, G: torch.Tensor, steps: int = 3000, batch: int = 8192,
          lr: float = 3e-3, wd: float = 1e-5, seed: int = 0, Xval=None, Yval=None,
          meta: dict | None = None) -> tuple[NullModel, dict]:
    """Adam on the MLP with this package's training kernels; cosine-decayed lr."""
    dev = X.device
    fm = X.mean(dim=0)
    fs = X.std(dim=0).clamp(min=1e-3)
    Xn = ((X - fm) / fs).contiguous()
    Yc = Y.contiguous()
    rng = np.random.default_rng(seed)
    master = torch.from_numpy(init_params(rng)).to(dev)
    P = master.numel()
    wb = torch.empty(P, dtype=torch.bfloat16, device=dev)
    native.call("tenex_to_bf16", master.data_ptr(), wb.data_ptr(), P, native.stream_ptr())
    m = torch.zeros(P, dtype=torch.float32, device=dev)
    v = torch.zeros(P, dtype=torch.float32, device=dev)
    scratch = torch.empty(int(native.lib().tenex_mlp_scratch_floats(batch)), dtype=torch.float32,
                          device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    n = Xn.shape[0]
    gen = torch.Generator(device=dev)
    gen.manual_seed(seed)
    hist = []
    since = 0
    t0 = time.time()
    for step in range(1, steps + 1):
        idx = torch.randint(0, n, (batch,), device=dev, generator=gen)
        xb = Xn[idx].contiguous()
        yb = Yc[idx].contiguous()
        lr_t = 0.5 * lr * (1 + np.cos(np.pi * (step - 1) / steps))
        native.call("tenex_mlp_train_step", xb.data_ptr(), yb.data_ptr(), batch, wb.data_ptr(),
                    master.data_ptr(), m.data_ptr(), v.data_ptr(), scratch.data_ptr(),
                    float(lr_t), 0.9, 0.999, 1e-8, float(wd), step, loss.data_ptr(),
                    native.stream_ptr())
        since += 1
        if step % 250 == 0 or step == steps:
            hist.append((step, float(loss.item()) / (since * batch)))
            loss.zero_()
            since = 0
    report = {"train_seconds": time.time() - t0, "loss_history": hist}
    gene_lo = G.min(dim=0).values.cpu().numpy()
    gene_hi = G.max(dim=0).values.cpu().numpy()
    model = NullModel(master.cpu().numpy(), fm.cpu().numpy(), fs.cpu().numpy(), gene_lo, gene_hi,
                      dict(meta or {}))
    if Xval is not None:
        report["val_mse"] = evaluate(model, Xval, Yval)
    return model, report


def evaluate(model: NullModel, Xraw: torch.Tensor, Y: torch.Tensor) -> list[float]:
    """Mean squared error of the two outputs on raw features (through the kernels)."""
    dev = Xraw.device
    wb, fm, fs = model.device_weights(dev)
    Xn = ((Xraw - fm) / fs).contiguous()
    B = Xn.shape[0]
    scratch = torch.empty(int(native.lib().tenex_mlp_scratch_floats(B)), dtype=torch.float32,
                          device=dev)
    grad = torch.empty(n_params(), dtype=torch.float32, device=dev)
    loss = torch.zeros(1, dtype=torch.float32, device=dev)
    native.call("tenex_mlp_gradients", Xn.data_ptr(), Y.contiguous().data_ptr(), B, wb.data_ptr(),
                scratch.data_ptr(), grad.data_ptr(), loss.data_ptr(), native.stream_ptr())
    z2off = 3 * B * 64 + B * 64  # dout lives after z1 | z2 | z1p | z2p
    dout = scratch[z2off:z2off + 2 * B].view(B, 2)
    return [float((dout[:, 0] ** 2).mean()), float((dout[:, 1] ** 2).mean())]


BANDS = tuple(np.round(np.arange(0.25, 4.01, 0.25), 2))


def analytic_null(db: D.DeviceBins, npv: torch.Tensor, tau: int):
    """The null without the network: the plug-in bias read as a scaled chi-square,
    2 N ln2 * TE ~ chi2(df) with df = 2 E_iid, so mu = E_iid / (N ln2) and
    sigma = sqrt(E_iid) / (N ln2). Same return form as predict()."""
    N = (db.T - tau) * db.K
    e = eiid_matrix(db, npv, tau)
    c = 1.0 / (N * np.log(2.0))
    mu = e * c
    sigma = torch.sqrt(torch.clamp(e, min=0.0)) * c
    ok = npv <= 64
    return mu, sigma, ok


def screen_recall(model, x: np.ndarray, npv: np.ndarray, dev, S: int, block_length: int,
                  seed: int, fdr: float = 0.05, tau: int = 1) -> dict:
    """On one dataset: the full S-shuffle test's BH-FDR edge set (parametric p) and,
    for each band in BANDS, the fraction of those edges the screen (predicted z >=
    z_FDR(predicted) - band) sends to verification, and the fraction of all pairs
    it sends. model is a NullModel, or "analytic" for analytic_null."""
    from tenex_b200.inference.grn import bh_fdr_gpu
    from tenex_b200.kernels.full_smem import FullSMEMKernel
    db = D.pack_bins(x, dev)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=dev)
    b_max = int(npv.max())
    obs = FullSMEMKernel().compute_pairfree_device(db, npv_t, b_max, tau, matrix=True)
    from tenex_b200.inference.surrogate_test import (SurrogateAccumulator, build_block_perm,
                                                     run_surrogates)
    acc = SurrogateAccumulator(db, npv_t, b_max, tau, obs, b_max == 2)
    perms, bl, _ = build_block_perm(db.n, db.T, "block", block_length, 0, S, seed, dev)
    run_surrogates(acc, perms, bl)
    mean = (acc.sum / S).float()
    std = torch.sqrt(torch.clamp(acc.sumsq / S - (acc.sum / S) ** 2, min=0.0)).float()
    off = ~torch.eye(db.n, dtype=torch.bool, device=dev)
    z_full = (obs - mean) / torch.clamp(std, min=1e-12)
    p_full = 0.5 * torch.special.erfc(z_full.double() / np.sqrt(2.0))
    sig = torch.zeros_like(off)
    sig[off] = bh_fdr_gpu(p_full[off], fdr) < fdr
    sig &= (obs - mean) > 0
    if isinstance(model, str) and model == "analytic":
        mu, sg, ok = analytic_null(db, npv_t, tau)
    else:
        mu, sg, ok = predict(model, db, npv_t, tau, block_length)
    z_pred = (obs - mu) / torch.clamp(sg, min=1e-12)
    valid = torch.isfinite(z_pred) & ok[None, :] & ok[:, None]
    p_pred = torch.where(valid, 0.5 * torch.special.erfc(z_pred.double() / np.sqrt(2.0)),
                         torch.ones_like(p_full))
    z_cut = z_of_p(bh_cut(p_pred[off], fdr), int(off.sum()), fdr)
    n_edges = int(sig.sum())
    out = {"n_edges": n_edges, "z_cut_pred": z_cut, "recall": {}, "verified": {}}
    for band in BANDS:
        screen = off & (~valid | (z_pred >= z_cut - band))
        out["recall"][band] = float((screen & sig).sum()) / max(n_edges, 1)
        out["verified"][band] = float(screen.sum()) / float(off.sum())
    return out


def calibrate_band(model: NullModel, seeds, dev, n=2000, T=5000, S=100, block_length=50,
                   target: float = 0.995) -> dict:
    """Smallest band of BANDS whose screen keeps >= target of the full test's edges
    on every held-out dataset (generator seeds `seeds`, permutation seeds 20000+)."""
    from tenex_b200 import workloads as W
    per = []
    for sd in seeds:
        x, npv, _ = W.cfg5_bins(n=n, T=T, seed=int(sd))
        per.append(screen_recall(model, x, npv, dev, S, block_length, 20_000 + int(sd)))
    band = next((b for b in BANDS if all(r["recall"][b] >= target for r in per)), BANDS[-1])
    return {"band": float(band), "target_recall": target,
            "recall": [r["recall"][band] for r in per],
            "verified_fraction": [r["verified"][band] for r in per],
            "n_edges": [r["n_edges"] for r in per]}


def train_default(device="cuda", seeds=range(2000, 2018), val_seeds=(2018, 2019), n=2000,
                  T=5000, S=100, block_length=50, pairs_per_dataset=150_000, steps=4000,
                  out=DEFAULT_MODEL) -> dict:
    """Trains on generator seeds `seeds`, reports the MSE on `val_seeds` and
    calibrates the fallback band on them (all disjoint from the evaluation seeds
    1000-1005)."""
    dev = torch.device(device)
    t0 = time.time()
    X, Y, G = training_set(list(seeds), n, T, S, block_length, pairs_per_dataset, dev)
    Xv, Yv, Gv = training_set(list(val_seeds), n, T, S, block_length, 50_000, dev)
    t_data = time.time() - t0
    meta = {"N": T - 1, "block_length": block_length, "n_surrogates": S,
            "train_seeds": [int(s) for s in seeds], "val_seeds": [int(s) for s in val_seeds],
            "generator": "cfg5_bins", "n": n, "T": T}
    model, rep = train(X, Y, torch.cat([G, Gv]), steps=steps, Xval=Xv, Yval=Yv, meta=meta)
    rep["data_seconds"] = t_data
    rep["train_pairs"] = int(X.shape[0])
    model.save(out)
    cal = calibrate_band(model, val_seeds, dev, n, T, S, block_length)
    rep["calibration"] = cal
    model.meta["band"] = cal["band"]
    model.meta["report"] = {k: rep[k] for k in ("val_mse", "train_pairs", "calibration")}
    model.save(out)
    return rep


# --------------------------------------------------------------------------- inference
def _pair_items(pairs_ts: np.ndarray, run: int = 128):
    from tenex_b200.kernels.pair_list import item_table
    order = np.argsort(pairs_ts[:, 0], kind="stable")
    sp = np.ascontiguousarray(pairs_ts[order])
    return sp, item_table(sp[:, 0], run)


def fallback_surrogates(db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int,
                        pairs_ts: np.ndarray, obs: torch.Tensor, perms: torch.Tensor, bl: int,
                        use_graph: bool = False, cfg=None):
    """Full surrogate statistics (all S = perms.shape[0] shuffles, the same
    permutations as the full test) for the listed [tgt, src] pairs only: device
    (n, n) float64 sum, sum of squares and int32 count_ge, indexed [src, tgt];
    entries of other pairs stay zero."""
    dev = db.data.device
    n = db.n
    S = perms.shape[0]
    sp, items = _pair_items(pairs_ts)
    pairs_d = torch.from_numpy(sp).to(dev)
    items_d = torch.from_numpy(items).to(dev)
    shuf = D.empty_bins(n, db.T, db.K, dev)
    ssum = torch.zeros((n, n), dtype=torch.float64, device=dev)
    ssq = torch.zeros((n, n), dtype=torch.float64, device=dev)
    cnt = torch.zeros((n, n), dtype=torch.int32, device=dev)
    ws = D.workspace(dev, n, db.row_len, b_max)

    def one(k):
        D.block_shuffle(db, perms[k], bl, out=shuf)
        native.call("tenex_surrogate_accumulate_pairs", shuf.ptr(), shuf.ld,
                    npv.data_ptr(), int(b_max), n, shuf.row_len, tau * db.K, pairs_d.data_ptr(),
                    sp.shape[0], items_d.data_ptr(), items.shape[0] - 1, obs.data_ptr(),
                    ssum.data_ptr(), ssq.data_ptr(), cnt.data_ptr(), ws.data_ptr(), ws.numel(),
                    D._cfg(cfg), native.stream_ptr())

    one(0)
    native.call("tenex_workspace_status", ws.data_ptr(), native.stream_ptr())
    if use_graph and S > 1:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for k in range(1, S):
                one(k)
        g.replay()
        torch.cuda.synchronize(dev)
        del g
    else:
        for k in range(1, S):
            one(k)
    native.call("tenex_workspace_status", ws.data_ptr(), native.stream_ptr())
    return ssum, ssq, cnt


def fallback_surrogates_batched(db: D.DeviceBins, npv: torch.Tensor, b_max: int, tau: int,
                                pairs_ts: np.ndarray, obs: torch.Tensor, perms: torch.Tensor,
                                bl: int, cfg=None, max_bytes: int | None = None):
    """fallback_surrogates with the surrogates batched into one pair-list launch:
    the shuffled copies of the bins are stacked as S_chunk * n genes (copy k of gene
    g is gene k * n + g) and every listed pair is listed once per copy, so one
    tenex_te_pairs launch covers S_chunk surrogates with full-GPU occupancy instead
    of S launches of a few thousand small work items. The per-surrogate TEs are
    then reduced over the surrogate axis in float64 (a sum of float32 values;
    the order of the additions changes the result by float64 rounding at most)."""
    dev = db.data.device
    n, S = db.n, perms.shape[0]
    sp, items = _pair_items(pairs_ts)
    P = sp.shape[0]
    ssum = torch.zeros((n, n), dtype=torch.float64, device=dev)
    ssq = torch.zeros((n, n), dtype=torch.float64, device=dev)
    cnt = torch.zeros((n, n), dtype=torch.int32, device=dev)
    if P == 0 or S == 0:
        return ssum, ssq, cnt
    sp_d = torch.from_numpy(sp).to(dev)                       # [tgt, src], sorted by target
    it_d = torch.from_numpy(items).to(dev)
    src_d, tgt_d = sp_d[:, 1], sp_d[:, 0]
    obs_p = obs[src_d, tgt_d].contiguous()
    s1 = torch.zeros(P, dtype=torch.float64, device=dev)
    s2 = torch.zeros(P, dtype=torch.float64, device=dev)
    c = torch.zeros(P, dtype=torch.int32, device=dev)
    if max_bytes is None:
        max_bytes = torch.cuda.mem_get_info(dev)[0] // 4
    chunk = int(max(1, min(S, max_bytes // max(1, n * db.ld))))
    lag = tau * db.K
    for k0 in range(0, S, chunk):
        kk = min(chunk, S - k0)
        big = D.empty_bins(kk * n, db.T, db.K, dev)
        D.block_shuffle_many(db, perms[k0:k0 + kk], bl, big)
        off = torch.arange(kk, device=dev, dtype=torch.int64)
        pairs_big = (sp_d[None, :, :] + (off * n)[:, None, None]).reshape(-1, 2).contiguous()
        items_big = torch.cat([(it_d[:-1][None, :] + (off * P)[:, None]).reshape(-1),
                               torch.tensor([kk * P], dtype=torch.int64, device=dev)])
        npv_big = npv.to(torch.int32).repeat(kk).contiguous()
        ws = D.workspace(dev, kk * n, db.row_len, b_max)
        te = torch.empty(kk * P, dtype=torch.float32, device=dev)
        native.call("tenex_te_pairs", big.ptr(), big.ld, npv_big.data_ptr(), int(b_max),
                    kk * n, big.row_len, lag, pairs_big.data_ptr(), kk * P, items_big.data_ptr(),
                    items_big.numel() - 1, te.data_ptr(), ws.data_ptr(), ws.numel(), D._cfg(cfg),
                    native.stream_ptr())
        native.call("tenex_workspace_status", ws.data_ptr(), native.stream_ptr())
        te = te.view(kk, P)
        t64 = te.double()
        s1 += t64.sum(dim=0)
        s2 += (t64 * t64).sum(dim=0)
        c += (te >= obs_p[None, :]).sum(dim=0, dtype=torch.int32)
        del big, pairs_big, items_big, ws, te
    ssum[src_d, tgt_d] = s1
    ssq[src_d, tgt_d] = s2
    cnt[src_d, tgt_d] = c
    return ssum, ssq, cnt


def bh_cut(p: torch.Tensor, fdr: float) -> float:
    """Largest p-value that BH-FDR at level fdr calls significant (adjusted
    p < fdr) among the 1-D p-values p, or 0.0 when none is. The BH-adjusted
    value of the k-th smallest p is the minimum over k' >= k of p_(k') m / k'
    (clamped at 1), so the significant set is the K smallest p-values, K the
    last rank with p_(K) m / K < fdr (the same expression as bh_fdr_gpu), and
    the cut is p_(K): one sort, no scatter back."""
    m = p.numel()
    if m == 0:
        return 0.0
    sp = p.sort().values
    rank = torch.arange(1, m + 1, device=p.device, dtype=p.dtype)
    ok = (sp * m / rank).clamp(max=1.0) < fdr
    last = int(torch.where(ok, rank, torch.zeros_like(rank)).max().item())
    return float(sp[last - 1].item()) if last > 0 else 0.0


def z_of_p(p: float, m: int, fdr: float) -> float:
    """Upper-tail normal quantile of p (of fdr / m when p is 0: nothing significant)."""
    from scipy.special import ndtri
    q = p if p > 0.0 else fdr / max(m, 1)
    return float(ndtri(1.0 - min(max(q, 1e-300), 1.0 - 1e-16)))


# launch shape of the batched verification pass (pair lists with few sources per
# target: 256-thread CTAs keep the per-item barriers short; measured on cfg5:
# 29.7 ms vs 32.6 ms for 512 threads x 2 and 39.5 ms for 1024 x 1)
VERIFY_CFG = dict(threads=256, ctas_per_sm=4, src_chunk=128)


def learned_surrogate_test(method, observed_te, variable_names, dev, bin_data, n_per_var, b_max,
                           kernel_name, tau, n_surrogates, shuffle_method, block_length, p_method,
                           fdr, seed, kwargs):
    """Surrogate test with the learned null screening the pairs (see module doc).

    Pairs whose predicted z reaches z_FDR - band (z_FDR from BH over the current
    p-values), and pairs the model cannot score, run the full S-shuffle test with
    the full test's permutations, so their statistics are the full test's (to the
    float rounding of each pair's entropy sum); the
    rest keep the predicted null. BH is recomputed on the mixed p-values and the
    screen widened until z_FDR - band stops falling (at most max_rounds times)."""
    from tenex_b200.inference.grn import build_pairs
    from tenex_b200.inference.surrogate_test import (SurrogateTestResult, bh_edges_device,
                                                     build_block_perm, pair_statistics)
    t0 = time.time()
    model = kwargs.get("null_model")
    if model is None:
        model = NullModel.load(kwargs.get("null_model_path", DEFAULT_MODEL))
    band = float(kwargs.get("fallback_band", model.meta.get("band", 1.0)))
    max_rounds = int(kwargs.get("max_rounds", 4))
    # the verification pass launches 2 x S kernels of ~0.25 ms each: eager launches
    # cost less than capturing and instantiating a graph for one replay
    use_graph = bool(kwargs.get("use_graph", False))
    n, T = bin_data.shape[0], bin_data.shape[1]
    db = D.pack_bins(bin_data, dev)
    npv = torch.as_tensor(np.asarray(n_per_var), dtype=torch.int32).to(dev)
    bl_eff = 1 if (shuffle_method == "random" or block_length <= 1
                   or block_length >= T) else block_length
    mu_d, sg_d, in_range = predict(model, db, npv, tau, max(bl_eff, 2))
    obs_d = torch.as_tensor(observed_te, dtype=torch.float32, device=dev).contiguous()
    z_d = (obs_d - mu_d) / torch.clamp(sg_d, min=1e-12)
    sources = kwargs.get("sources")
    if sources is not None:
        pb = build_pairs(np.asarray(variable_names), sources)
        tested_np = np.zeros((n, n), dtype=bool)
        tested_np[pb[:, 0], pb[:, 1]] = True
        tested = torch.from_numpy(tested_np).to(dev)
    else:
        tested = ~torch.eye(n, dtype=torch.bool, device=dev)
    valid = torch.isfinite(z_d) & in_range[None, :] & in_range[:, None]
    m_tested = int(tested.sum())
    n_unscored = int((tested & ~valid).sum())
    if n_unscored > float(kwargs.get("full_test_fraction", 0.5)) * max(m_tested, 1):
        # data unlike the training set: most pairs would go to the full test anyway,
        # so run the full test itself (its exact statistics, without the screen's
        # per-pair bookkeeping)
        full_kw = {k: v for k, v in kwargs.items() if k != "null"}
        res = method.infer(observed_te, variable_names, dev, **full_kw)
        res.null_model = "learned"
        res.info = {"n_fallback": m_tested, "fallback_fraction": 1.0, "n_invalid": n_unscored,
                    "delegated_to_full_test": True, "band": band, "rounds": 0,
                    "seconds_predict": time.time() - t0, "seconds_total": time.time() - t0,
                    "n_out_of_range_genes": int((~in_range).sum().item())}
        _log.vprint(f"[TENEX] learned null: {n_unscored} of {m_tested} pairs outside the "
                    f"model's training range; ran the full surrogate test")
        return res
    p_mix = 0.5 * torch.special.erfc(z_d.double() / np.sqrt(2.0))
    p_mix = torch.where(valid, p_mix, torch.ones_like(p_mix))
    mean_s = mu_d.clone()
    std_s = sg_d.clone()
    eff_s = obs_d - mean_s
    count = torch.zeros((n, n), dtype=torch.int32, device=dev)
    verified = torch.zeros((n, n), dtype=torch.bool, device=dev)
    t_pred = time.time() - t0
    perms = None
    rounds, z_cuts, t_verify = 0, [], 0.0
    for _ in range(max_rounds):
        z_cut = z_of_p(bh_cut(p_mix[tested], fdr), m_tested, fdr)
        z_cuts.append(z_cut)
        new = tested & ~verified & (~valid | (z_d >= z_cut - band))
        idx = torch.nonzero(new)                                   # (src, tgt)
        if idx.shape[0] == 0:
            break
        tv = time.time()
        if perms is None:
            perms, bl, _ = build_block_perm(n, T, shuffle_method, block_length, 0, n_surrogates,
                                            seed, dev)
        idx_np = idx.cpu().numpy()
        pairs_ts = np.ascontiguousarray(idx_np[:, ::-1]).astype(np.int64)
        if kwargs.get("verify_batched", True):
            ssum, ssq, cnt = fallback_surrogates_batched(
                db, npv, b_max, tau, pairs_ts, obs_d, perms, bl,
                kwargs.get("verify_cfg", VERIFY_CFG))
        else:
            ssum, ssq, cnt = fallback_surrogates(db, npv, b_max, tau, pairs_ts, obs_d, perms,
                                                 bl, use_graph,
                                                 kwargs.get("verify_cfg", VERIFY_CFG))
        si, ti = idx[:, 0], idx[:, 1]
        ms, ss_, ef, pv = pair_statistics(observed_te[idx_np[:, 0], idx_np[:, 1]],
                                          ssum[si, ti].cpu().numpy(), ssq[si, ti].cpu().numpy(),
                                          cnt[si, ti].cpu().numpy(), n_surrogates, p_method)
        mean_s[si, ti] = torch.from_numpy(ms).to(dev)
        std_s[si, ti] = torch.from_numpy(ss_).to(dev)
        eff_s[si, ti] = torch.from_numpy(ef).to(dev)
        p_mix[si, ti] = torch.from_numpy(pv).to(dev).double()
        count[si, ti] = cnt[si, ti]
        verified |= new
        rounds += 1
        t_verify += time.time() - tv
    diag = torch.arange(n, device=dev)
    p_mix[diag, diag] = 1.0
    mean_s[diag, diag] = 0.0
    std_s[diag, diag] = 0.0
    eff_s[diag, diag] = obs_d[diag, diag]
    p32 = p_mix.float()
    grn = bh_edges_device(p32, eff_s, tested, variable_names, fdr)
    host = D.to_host(torch.stack((p32, mean_s.float(), std_s.float(), eff_s.float())))
    p_values, mean_np, std_np, effective = host[0], host[1], host[2], host[3]
    n_ver = int(verified.sum())
    info = {"n_fallback": n_ver, "fallback_fraction": n_ver / max(m_tested, 1),
            "n_invalid": int((tested & ~valid).sum()), "z_cuts": z_cuts, "band": band,
            "rounds": rounds, "seconds_predict": t_pred, "seconds_verify": t_verify,
            "seconds_total": time.time() - t0,
            "n_out_of_range_genes": int((~in_range).sum().item())}
    _log.vprint(f"[TENEX] learned null: {n_ver} pairs ({100 * info['fallback_fraction']:.3f}%) "
                f"verified by the full surrogate test in {rounds} round(s); {len(grn)} edges")
    return SurrogateTestResult(observed_te=observed_te, mean_surrogate_te=mean_np,
                               std_surrogate_te=std_np, effective_te=effective, p_values=p_values,
                               grn=grn, n_surrogates=n_surrogates, shuffle_method=shuffle_method,
                               block_length=block_length if shuffle_method == "block" else None,
                               p_method=p_method, fdr=fdr, null_model="learned", info=info)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--train", action="store_true")
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--out", default=DEFAULT_MODEL)
    a = ap.parse_args()
    if a.train:
        _log.set_verbose(True)
        rep = train_default(steps=a.steps, out=a.out)
        print(rep)
