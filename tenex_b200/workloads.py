"""Seeded synthetic workloads with the shapes of the five TE benchmark configs.

No public dataset exists for these shapes (only the reference's mESC fixture),
so seeded generators stand in for the reference's mESC/skin/zebrafish/CeNGEN
runs. Each returns numpy arrays; one numpy Generator per call.

  cfg1  expression (100 x 1000 float32): zero-inflated NB counts, log1p
  cfg2  binary bins (2000 x 5000): two-state Markov chains
  cfg3  multi-bin bins (5000 x 10000): b ~ U{2..32}, Dirichlet(1) values
  cfg4  uneven bins (10000 x 20000): 95% b ~ U{2..16}, 5% b ~ U{64..256}
  cfg5  multi-bin Markov bins (2000 x 5000): b ~ U{2..16}, for the surrogate test
"""
from __future__ import annotations

import numpy as np

CONFIGS = {
    1: dict(n=100, T=1000),
    2: dict(n=2000, T=5000),
    3: dict(n=5000, T=10000),
    4: dict(n=10000, T=20000),
    5: dict(n=2000, T=5000),
}


def _planted(rng, n: int, k: int) -> np.ndarray:
    """k distinct (regulator, target) pairs with regulator != target and distinct
    targets (so k <= n)."""
    if k > n:
        raise ValueError(f"{k} planted pairs need at least {k} genes (n={n})")
    out, seen = [], set()
    while len(out) < k:
        r, t = (int(v) for v in rng.integers(0, n, 2))
        if r != t and (r, t) not in seen and t not in {p[1] for p in out}:
            seen.add((r, t))
            out.append((r, t))
    return np.array(out, dtype=np.int64)


def cfg1_expression(n: int = 100, T: int = 1000, seed: int = 1001, n_planted: int = 10):
    """float32 (n, T) log1p of zero-inflated negative-binomial counts, cells sorted
    by a uniform pseudotime; planted lag-1 regulator->target latent coupling."""
    rng = np.random.default_rng(seed)
    _pt = np.sort(rng.random(T))  # pseudotime order: cells are generated in this order
    mu = rng.lognormal(0.0, 1.0, n)
    z = np.zeros((n, T))
    eps = rng.normal(0.0, 0.3, (n, T))
    z[:, 0] = eps[:, 0]
    for t in range(1, T):
        z[:, t] = 0.9 * z[:, t - 1] + eps[:, t]
    planted = _planted(rng, n, n_planted)
    for r, t in planted:
        z[t, 1:] = 0.8 * z[r, :-1] + rng.normal(0.0, 0.3, T - 1)
    mean = mu[:, None] * np.exp(z)
    r_disp = 2.0
    lam = rng.gamma(r_disp, mean / r_disp)
    counts = rng.poisson(lam)
    counts[rng.random((n, T)) < 0.6] = 0
    return np.log1p(counts).astype(np.float32), planted


def cfg2_binary(n: int = 2000, T: int = 5000, seed: int = 1002, n_planted: int = 20):
    """uint8 {0,1} (n, T): per-gene two-state Markov chain with stationary rate
    U(0.05,0.5) and stay-probability U(0.7,0.95); planted tgt_t = src_{t-1} XOR Bern(0.1)."""
    rng = np.random.default_rng(seed)
    pi = rng.uniform(0.05, 0.5, n)
    s = rng.uniform(0.7, 0.95, n)
    p11 = s
    p01 = np.minimum((1 - s) * pi / (1 - pi), 1.0)
    x = np.zeros((n, T), np.uint8)
    x[:, 0] = rng.random(n) < pi
    u = rng.random((n, T))
    for t in range(1, T):
        prev = x[:, t - 1].astype(bool)
        x[:, t] = np.where(prev, u[:, t] < p11, u[:, t] < p01)
    planted = _planted(rng, n, n_planted)
    for r, t in planted:
        flip = rng.random(T - 1) < 0.1
        x[t, 1:] = x[r, :-1] ^ flip
    return x, planted


def _dirichlet_draws(rng, b: int, T: int, ar_frac_gene: bool, p=None) -> np.ndarray:
    if p is None:
        p = rng.dirichlet(np.ones(b))
    v = np.searchsorted(np.cumsum(p), rng.random(T) * (1 - 1e-12)).astype(np.int64)
    v = np.minimum(v, b - 1)
    if ar_frac_gene:
        keep = rng.random(T) < 0.5
        for t in range(1, T):
            if keep[t]:
                v[t] = v[t - 1]
    return v


def _dense_remap(x: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    n = x.shape[0]
    out = np.empty_like(x)
    npv = np.empty(n, np.int32)
    for g in range(n):
        u, inv = np.unique(x[g], return_inverse=True)
        out[g] = inv.reshape(x[g].shape)
        npv[g] = u.shape[0]
    return out, npv


def multibin(n: int, T: int, seed: int, b_lo: int, b_hi: int, heavy_frac: float = 0.0,
             heavy_lo: int = 64, heavy_hi: int = 256, ar_frac: float = 0.05,
             remap: bool = True):
    """Per-gene b ~ U{b_lo..b_hi} (a heavy_frac of genes U{heavy_lo..heavy_hi}),
    values i.i.d. from a per-gene Dirichlet(1) over its bins, lag-1 AR
    (x_t = x_{t-1} w.p. 0.5) on ar_frac of genes. Returns bins (uint8, or uint16
    when any b > 255... values < 256 here) dense-remapped, and n_per_var."""
    rng = np.random.default_rng(seed)
    b = rng.integers(b_lo, b_hi + 1, n)
    heavy = rng.random(n) < heavy_frac
    if heavy.any():
        b[heavy] = rng.integers(heavy_lo, heavy_hi + 1, int(heavy.sum()))
    ar = rng.random(n) < ar_frac
    dtype = np.uint8 if b.max() <= 256 else np.uint16
    x = np.empty((n, T), dtype if b.max() < 256 else np.uint16)
    # vectorised draws: inverse CDF per gene
    u = rng.random((n, T))
    for g in range(n):
        p = rng.dirichlet(np.ones(int(b[g])))
        v = np.searchsorted(np.cumsum(p), u[g] * (1 - 1e-12))
        np.minimum(v, b[g] - 1, out=v)
        if ar[g]:
            keep = rng.random(T) < 0.5
            # x_t = x_{t-1} where keep: forward-fill the kept positions
            idx = np.where(keep, 0, np.arange(T))
            np.maximum.accumulate(idx, out=idx)
            v = v[idx]
        x[g] = v
    if remap:
        x, npv = _dense_remap(x)
        return x, npv
    return x, b.astype(np.int32)


def cfg3_bins(n: int = 5000, T: int = 10000, seed: int = 1003):
    return multibin(n, T, seed, 2, 32)


def cfg4_bins(n: int = 10000, T: int = 20000, seed: int = 1004):
    return multibin(n, T, seed, 2, 16, heavy_frac=0.05, heavy_lo=64, heavy_hi=256)


def cfg5_bins(n: int = 2000, T: int = 5000, seed: int = 1005, n_planted: int = 20):
    """Per gene b ~ U{2..16} states, Markov: stay w.p. s ~ U(0.7,0.95), else a
    fresh draw from the gene's stationary Dirichlet(1); 20 planted lag-1
    copies tgt_t = src_{t-1} with 10% of samples redrawn."""
    rng = np.random.default_rng(seed)
    b = rng.integers(2, 17, n)
    s = rng.uniform(0.7, 0.95, n)
    x = np.empty((n, T), np.uint8)
    for g in range(n):
        p = rng.dirichlet(np.ones(int(b[g])))
        fresh = np.minimum(np.searchsorted(np.cumsum(p), rng.random(T) * (1 - 1e-12)), b[g] - 1)
        stay = rng.random(T) < s[g]
        stay[0] = False
        idx = np.where(stay, 0, np.arange(T))
        np.maximum.accumulate(idx, out=idx)
        x[g] = fresh[idx]
    planted = _planted(rng, n, n_planted)
    for r, t in planted:
        noise = rng.random(T - 1) < 0.1
        src = x[r, :-1].astype(np.int64) % b[t]
        redraw = rng.integers(0, b[t], T - 1)
        x[t, 1:] = np.where(noise, redraw, src)
    x, npv = _dense_remap(x)
    return x, npv, planted
