"""Argument checks of the C ABI that run before any CUDA call, so they are
exercised on a machine without a GPU: each bad argument returns its status
(TENEX_ERR_BADARG / TENEX_ERR_UNSUPPORTED), and the Python layer raises
TenexError naming the entry point. The buffers are host memory and are never
dereferenced: every call fails its checks first."""
import ctypes

import numpy as np
import pytest
import torch

from tenex_b200 import native

# host pointers must never reach a kernel: run only where no CUDA device exists
pytestmark = pytest.mark.skipif(torch.cuda.is_available(),
                                reason="host-pointer argument checks run without a GPU only")


def _status(name, *args):
    with pytest.raises(native.TenexError) as ei:
        native.call(name, *args)
    assert name in str(ei.value)
    return ei.value.status


def _addr(a: np.ndarray) -> int:
    return a.ctypes.data


def test_block_shuffle_many_argument_checks():
    n, T, nb, bl, S = 4, 64, 8, 8, 3
    ld = 64
    bins = np.zeros(n * ld + 64, np.uint8)
    perms = np.zeros(S * n * nb, np.int32)
    out = np.zeros(S * n * ld + 64, np.uint8)
    base = _addr(out) + (-_addr(out)) % 16                 # 16-byte aligned start
    good = (_addr(bins), ld, n, T, 1, _addr(perms), S, nb, bl, base, ld, n * ld, 0)

    def call(**kw):
        names = ["in", "in_ld", "n", "T", "K", "perms", "S", "nb", "bl", "out", "out_ld",
                 "stride", "stream"]
        args = dict(zip(names, good))
        args.update(kw)
        return _status("tenex_block_shuffle_many", *[args[k] for k in names])

    bad = native.TENEX_ERR_BADARG
    assert call(**{"in": None}) == bad                       # NULL input
    assert call(perms=None) == bad                           # NULL permutations
    assert call(S=0) == bad                                  # no copies
    assert call(bl=0) == bad                                 # empty blocks
    assert call(nb=T // bl + 1) == bad                       # blocks past the series
    assert call(out_ld=T - 1) == bad                         # row stride shorter than a row
    assert call(stride=n * ld - 16) == bad                   # copies overlap each other
    assert call(out=_addr(bins)) == bad                      # output over the input
    assert call(out=base + 1) == bad                         # output not 16-byte aligned
    assert call(out_ld=ld + 4, stride=n * (ld + 16)) == bad  # row stride not 16-byte aligned


def test_single_block_shuffle_shares_the_checks():
    n, T, ld = 2, 32, 64
    bins = np.zeros(n * ld, np.uint8)
    perm = np.zeros(n * 4, np.int32)
    assert _status("tenex_block_shuffle", _addr(bins), ld, n, T, 1, _addr(perm), 4, 8,
                   _addr(bins), ld, 0) == native.TENEX_ERR_BADARG   # in place


def test_launch_shape_argument_checks():
    out = [ctypes.c_int() for _ in range(4)]
    refs = [ctypes.byref(v) for v in out]
    bad, unsup = native.TENEX_ERR_BADARG, native.TENEX_ERR_UNSUPPORTED
    assert _status("tenex_te_launch_shape", 100, 1, 8, None, None, *refs[1:]) == bad
    assert _status("tenex_te_launch_shape", 100, 0, 8, None, *refs) == bad       # lag 0
    assert _status("tenex_te_launch_shape", 5, 5, 8, None, *refs) == bad         # lag >= row
    assert _status("tenex_te_launch_shape", 100, 1, 0, None, *refs) == bad       # b_max 0
    assert _status("tenex_te_launch_shape", 100, 1, 256, None, *refs) == bad     # b_max 256
    assert _status("tenex_te_launch_shape", 1 << 31, 1, 8, None, *refs) == unsup  # >= 2^31


def test_binary_matrix_tile_width_checks():
    n, T, ld = 4, 64, 64
    bins = np.zeros(n * ld + 64, np.uint8)
    out = np.zeros(n * n + 16, np.float32)
    ws = np.zeros(4096 + 256, np.uint8)
    bb = _addr(bins) + (-_addr(bins)) % 16
    wb = _addr(ws) + (-_addr(ws)) % 256
    bad = native.TENEX_ERR_BADARG
    def call(kind=0, tn=0):
        return _status("tenex_te_binary_matrix_ex", bb, ld, n, T, 1, _addr(out), n, wb, 4096,
                       kind, tn, 0)

    for tn in (7, 48, 256, -1):
        assert call(tn=tn) == bad
    assert call(kind=3, tn=128) == bad                    # unknown operand form
    from tenex_b200.kernels.gemm_b2 import te_binary_matrix
    with pytest.raises(ValueError, match="tile_n"):
        te_binary_matrix(None, 1, tile_n=100)
