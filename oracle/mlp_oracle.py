"""CPU oracle of the learned-null MLP — TEST INFRASTRUCTURE ONLY.

float64 numpy forward / backward of the 16 -> 64 -> 64 -> 2 GELU MLP whose
kernels live in the package (null_mlp.cu), on the same BF16-rounded weights,
plus numpy restatements of the per-gene features, the pair independence bias
E_iid and the pair features. Used only by tests to check
the kernels' outputs and gradients.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

N_IN, H = 16, 64


def bf16_round(a: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even) -> float32."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(p: np.ndarray):
    o = 0
    W1 = p[o:o + H * N_IN].reshape(H, N_IN); o += H * N_IN
    b1 = p[o:o + H]; o += H
    W2 = p[o:o + H * H].reshape(H, H); o += H * H
    b2 = p[o:o + H]; o += H
    W3 = p[o:o + 2 * H].reshape(2, H); o += 2 * H
    b3 = p[o:o + 2]
    return W1, b1, W2, b2, W3, b3


def gelu(x):
    return 0.5 * x * (1 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2 * np.pi)


def forward(p: np.ndarray, X: np.ndarray) -> np.ndarray:
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, np.float64))
    z1 = X @ W1.T + b1
    z2 = gelu(z1) @ W2.T + b2
    return gelu(z2) @ W3.T + b3


def gradients(p: np.ndarray, X: np.ndarray, Y: np.ndarray):
    """Mean over the batch of d/dp of 0.5 * sum((out - Y)^2); also the summed loss."""
    W1, b1, W2, b2, W3, b3 = unpack(np.asarray(p, np.float64))
    X = np.asarray(X, np.float64)
    z1 = X @ W1.T + b1
    g1 = gelu(z1)
    z2 = g1 @ W2.T + b2
    g2 = gelu(z2)
    out = g2 @ W3.T + b3
    d = out - Y
    B = X.shape[0]
    dW3 = d.T @ g2 / B
    db3 = d.mean(0)
    dz2 = (d @ W3) * gelu_grad(z2)
    dW2 = dz2.T @ g1 / B
    db2 = dz2.mean(0)
    dz1 = (dz2 @ W2) * gelu_grad(z1)
    dW1 = dz1.T @ X / B
    db1 = dz1.mean(0)
    g = np.concatenate([dW1.ravel(), db1, dW2.ravel(), db2, dW3.ravel(), db3])
    return g, 0.5 * float((d ** 2).sum())


def gene_features(bins: np.ndarray, npv: np.ndarray, lag: int = 1) -> np.ndarray:
    """(n, 6): log2 b, H(x_t), H(x_{t+lag}, x_t), 2H - H2, log2 mean run length, 2^H / b."""
    n, T = bins.shape
    N = T - lag
    out = np.zeros((n, 6))
    for g in range(n):
        x0 = bins[g, :N].astype(np.int64)
        x1 = bins[g, lag:lag + N].astype(np.int64)
        c1 = np.bincount(x0) / N
        c1 = c1[c1 > 0]
        H1 = -(c1 * np.log2(c1)).sum()
        c2 = np.bincount(x1 * 64 + x0) / N
        c2 = c2[c2 > 0]
        H2 = -(c2 * np.log2(c2)).sum()
        ch = int((x1 != x0).sum())
        b = max(int(npv[g]), 1)
        out[g] = [np.log2(b), H1, H2, 2 * H1 - H2, np.log2(N / (ch + 1)), 2 ** H1 / b]
    return out


def g_poisson(m: np.ndarray) -> np.ndarray:
    """g(m) = E[C ln C] - m ln m for C ~ Poisson(m), by direct summation of the
    Poisson series (float64, log-space probabilities)."""
    from scipy.special import gammaln
    m = np.atleast_1d(np.asarray(m, np.float64)).ravel()
    out = np.zeros_like(m)
    pos = m > 0
    if not pos.any():
        return out
    mp = m[pos]
    kmax = int(mp.max() + 14 * np.sqrt(mp.max()) + 60)
    k = np.arange(1, kmax + 1, dtype=np.float64)
    klk = k * np.log(k)
    lg = gammaln(k + 1)
    for i0 in range(0, mp.size, 512):
        mm = mp[i0:i0 + 512, None]
        pmf = np.exp(k[None, :] * np.log(mm) - mm - lg[None, :])
        out_i = (pmf * klk[None, :]).sum(1) - mm[:, 0] * np.log(mm[:, 0])
        idx = np.flatnonzero(pos)[i0:i0 + 512]
        out[idx] = out_i
    return out


def eiid(bins: np.ndarray, npv: np.ndarray, lag: int = 1) -> np.ndarray:
    """(n, n) [src, tgt] independence bias sum_{a,b} g(n_a q_b) - sum_{x,b} g(n_x q_b)
    (NaN when either gene has more than 64 states; diagonal NaN)."""
    n, T = bins.shape
    N = T - lag
    out = np.full((n, n), np.nan)
    for t in range(n):
        bt = int(npv[t])
        if bt > 64:
            continue
        x0 = bins[t, :N].astype(np.int64)
        x1 = bins[t, lag:lag + N].astype(np.int64)
        na = np.bincount(x1 * bt + x0, minlength=bt * bt).astype(np.float64)
        nx = np.bincount(x0, minlength=bt).astype(np.float64)
        na, nx = na[na > 0], nx[nx > 0]
        for s in range(n):
            if s == t or int(npv[s]) > 64:
                continue
            q = np.bincount(bins[s, :N].astype(np.int64)) / N
            q = q[q > 0]
            out[s, t] = g_poisson(np.outer(na, q).ravel()).sum() - \
                g_poisson(np.outer(nx, q).ravel()).sum()
    return out


def pair_features(gf6: np.ndarray, eiid_m: np.ndarray, tgt, src, block_length: int) -> np.ndarray:
    """Raw (P, 16) pair features from the (n, 6) gene features and the E_iid matrix."""
    tgt = np.asarray(tgt)
    src = np.asarray(src)
    a, b = gf6[tgt], gf6[src]
    bt, bs = 2.0 ** a[:, 0], 2.0 ** b[:, 0]
    e = eiid_m[src, tgt]
    return np.concatenate([a, b, np.log2(np.maximum(e, 1e-6))[:, None],
                           np.full((tgt.size, 1), np.log2(block_length)),
                           np.log2((bt - 1) * (bs - 1) * bt + 1)[:, None],
                           (a[:, 2] + b[:, 1])[:, None]], axis=1)
