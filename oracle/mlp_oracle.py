"""CPU oracle of the learned-null MLP — TEST INFRASTRUCTURE ONLY.

float64 numpy forward / backward of the 16 -> 64 -> 64 -> 2 GELU MLP whose
kernels live in the package (null_mlp.cu), on the same BF16-rounded weights,
plus a numpy restatement of the per-gene features. Used only by tests to check
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
