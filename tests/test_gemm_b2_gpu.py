"""tcgen05 binary TE kernel against the oracle and the reference GEMM-B2 fixture."""
import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200 import native, workloads as W
from tenex_b200.kernels import device as D
from tenex_b200.kernels.gemm_b2 import TILE_N, te_binary_matrix

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _run(x, cuda, tau=1, operands="default", tile_n=0):
    db = D.pack_bins(x, cuda)
    m = te_binary_matrix(db, tau, operands=operands, tile_n=tile_n).cpu().numpy()
    torch.cuda.synchronize()
    return m


@pytest.mark.parametrize("operands", ["int8", "fp4"])
@pytest.mark.parametrize("n,T", [(5, 40), (130, 300), (257, 1100), (129, 257), (200, 513)])
def test_binary_matrix_matches_oracle(cuda, n, T, operands):
    x, _ = W.cfg2_binary(n=n, T=T, seed=n + T, n_planted=min(3, n // 2))
    m = _run(x, cuda, operands=operands)
    ref = O.te_matrix(x.astype(np.int32), np.full(n, 2, np.int32))
    assert np.all(np.diag(m) == 0)
    assert np.max(np.abs(m - ref)) <= TOL


@pytest.mark.parametrize("operands", ["int8", "fp4"])
@pytest.mark.parametrize("tile_n", TILE_N)
@pytest.mark.parametrize("n,T", [(130, 300), (257, 1100)])
def test_every_tile_width_matches_oracle(cuda, n, T, tile_n, operands):
    # each target-tile width (MMA N = tile_n and 2 tile_n; ragged last tiles at
    # these n) against the oracle, bitwise equal to the automatic choice
    x, _ = W.cfg2_binary(n=n, T=T, seed=3 * n + T, n_planted=3)
    m = _run(x, cuda, operands=operands, tile_n=tile_n)
    ref = O.te_matrix(x.astype(np.int32), np.full(n, 2, np.int32))
    assert np.all(np.diag(m) == 0)
    assert np.max(np.abs(m - ref)) <= TOL
    assert np.array_equal(m.view(np.uint32), _run(x, cuda, operands=operands).view(np.uint32))


def test_long_series(cuda):
    # 70,000 samples per pair (int32 / float32 sums, both forms)
    x, _ = W.cfg2_binary(n=70, T=70_001, seed=77, n_planted=2)
    ref = O.te_matrix(x.astype(np.int32), np.full(70, 2, np.int32))
    m = _run(x, cuda)
    assert np.max(np.abs(m - ref)) <= TOL
    assert np.array_equal(m.view(np.uint32), _run(x, cuda, operands="int8").view(np.uint32))


@pytest.mark.parametrize("operands", ["int8", "fp4"])
def test_binary_matches_reference_fixture(cuda, golden, operands):
    g = golden("gemm_b2.npz")
    m = _run(g["bins"], cuda, operands=operands)
    assert np.max(np.abs(m - g["te_ij_j_to_i"].T)) <= TOL


@pytest.mark.parametrize("operands", ["int8", "fp4"])
def test_binary_tau2_constant_rows(cuda, operands):
    rng = np.random.default_rng(2)
    x = (rng.random((70, 500)) < 0.3).astype(np.uint8)
    x[3] = 0
    x[4] = 1
    m = _run(x, cuda, tau=2, operands=operands)
    ref = O.te_matrix(x.astype(np.int32), np.full(70, 2, np.int32), tau=2)
    assert np.max(np.abs(m - ref)) <= TOL


@pytest.mark.parametrize("operands", ["int8", "fp4"])
def test_non_binary_bins_report_bad_data(cuda, operands):
    # the GEMM sums raw bytes, so a bin other than 0/1 must be reported by the status
    # call, not silently counted; the context stays usable afterwards
    rng = np.random.default_rng(2)
    x = (rng.random((20, 300)) < 0.4).astype(np.int32)
    x[7, 123] = 2
    with pytest.raises(native.TenexError) as ei:
        te_binary_matrix(D.pack_bins(x, cuda), 1, operands=operands)
    assert ei.value.status == native.TENEX_ERR_BADDATA
    x[7, 123] = 1
    m = te_binary_matrix(D.pack_bins(x, cuda), 1, operands=operands).cpu().numpy()
    assert np.max(np.abs(m - O.te_matrix(x, np.full(20, 2, np.int32)))) <= 1e-6


def test_binary_full_size_sampled_and_deterministic(cuda):
    """2,000 genes x 5,000 cells of binary Markov bins with 20 planted lag-1
    pairs, the whole matrix in one pack + GEMM launch pair: 50,000 random pairs
    and every planted pair within 1e-6 of the float64 oracle, zero diagonal, a
    second run bitwise equal."""
    x, planted = W.cfg2_binary()
    n = x.shape[0]
    m = _run(x, cuda)                                   # [src, tgt]
    rng = np.random.default_rng(21)
    src = rng.integers(0, n, 50_000)
    tgt = rng.integers(0, n, 50_000)
    pl = np.asarray(planted, dtype=np.int64).reshape(-1, 2)
    src = np.concatenate([src, pl[:, 0]])
    tgt = np.concatenate([tgt, pl[:, 1]])
    keep = src != tgt
    src, tgt = src[keep], tgt[keep]
    ref = O.te_pairs(x.astype(np.int32), np.full(n, 2, np.int32), np.stack([tgt, src], axis=1))
    assert np.max(np.abs(m[src, tgt].astype(np.float64) - ref)) <= TOL
    assert np.all(np.diag(m) == 0)
    assert np.array_equal(m.view(np.uint32), _run(x, cuda).view(np.uint32))
    # the int8 and 4-bit operand forms give the same exact counts, so the same bits
    assert np.array_equal(m.view(np.uint32), _run(x, cuda, operands="int8").view(np.uint32))
    assert np.array_equal(m.view(np.uint32), _run(x, cuda, operands="fp4").view(np.uint32))
    # and every target-tile width the same bits
    for tn in TILE_N:
        assert np.array_equal(m.view(np.uint32), _run(x, cuda, tile_n=tn).view(np.uint32)), tn
