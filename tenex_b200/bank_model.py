"""Bank-conflict model of the TE kernel's histogram scatter (csrc/te_pair.cu).

A warp-wide `red.shared.add` is served in one shared-memory wavefront per
distinct 32-bit word of its most loaded bank (32 banks of 4 bytes; lanes that add
to the same word are merged). The kernel issues a pair's samples in a fixed
pattern: lane l of a warp holds samples 16 l .. 16 l + 15 of each 512-sample
chunk (one 16-byte load of source bins) and step j of the 16 steps counts sample
16 l + j in every lane. Given the target's joint states z = x_t[s + lag] * b_t +
x_t[s] and the source bins y of one pair, this module replays that pattern for a
table whose cell (z, y) is word z * stride + y and returns the mean wavefronts per
reduction.

On cfg4-like bins it reproduces what the kernel's layout choices were based on
(ncu measured 3.10 wavefronts per reduction on a cfg4 slice with stride b_s, and
2.88 with the odd stride):
  * stride b_s even: lanes sharing a popular source bin but not the target state
    land in one or two banks;
  * stride b_s | 1: rows start in different banks;
  * sort_groups: each lane's 16 samples ordered by target state (the kernel's
    sorted sample groups), so a step's lanes hold states of similar rank.
"""
from __future__ import annotations

import numpy as np

LANES, PER_LANE, BANKS = 32, 16, 32


def reduction_wavefronts(words: np.ndarray) -> int:
    """Wavefronts of one warp-wide reduction into the given 32-bit word indices."""
    u = np.unique(words)
    return int(np.bincount(u % BANKS, minlength=BANKS).max())


def pair_wavefronts(z: np.ndarray, y: np.ndarray, stride: int, sort_groups: bool = False,
                    max_chunks: int | None = None) -> float:
    """Mean wavefronts per reduction of one pair's histogram pass (full 512-sample
    chunks only; `max_chunks` limits how many are replayed)."""
    z = np.asarray(z, np.int64)
    y = np.asarray(y, np.int64)
    chunk = LANES * PER_LANE
    n_chunks = min(z.size, y.size) // chunk
    if max_chunks is not None:
        n_chunks = min(n_chunks, max_chunks)
    if n_chunks == 0:
        raise ValueError("the pair needs at least one full chunk of 512 samples")
    total, count = 0, 0
    for c in range(n_chunks):
        zc = z[c * chunk:(c + 1) * chunk].reshape(LANES, PER_LANE)
        yc = y[c * chunk:(c + 1) * chunk].reshape(LANES, PER_LANE)
        if sort_groups:
            order = np.argsort(zc, axis=1, kind="stable")
            zc = np.take_along_axis(zc, order, axis=1)
            yc = np.take_along_axis(yc, order, axis=1)
        cells = zc * stride + yc
        for j in range(PER_LANE):
            total += reduction_wavefronts(cells[:, j])
            count += 1
    return total / count


def joint_states(target_bins: np.ndarray, b_t: int, lag: int = 1) -> np.ndarray:
    """z[s] = x[s + lag] * b_t + x[s] for s in [0, T - lag)."""
    x = np.asarray(target_bins, np.int64)
    return x[lag:] * b_t + x[:-lag]
