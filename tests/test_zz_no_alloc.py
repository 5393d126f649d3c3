"""The no-allocation TE entry point against the regular one.

tenex_te_pairfree_static serves callers that cannot allocate device memory
after start-up (fixed device-memory budgets, memory owned by another
framework's pool, bindings that cannot own device buffers): it takes no
workspace and uses a fixed scratch area compiled into the library. These tests
call both entry points through the C ABI on the same inputs, twice in a row
with different data (the shared scratch must not carry state from one call to
the next), and require the same TE within the suite's 1e-6 tolerance. This
file is collected last so a failure here leaves the rest of the suite's
results intact.
"""

import numpy as np
import pytest
import torch

from oracle import oracle as O
from tenex_b200 import native
from tenex_b200.kernels import device as D

pytestmark = pytest.mark.gpu
TOL = 1e-6


def _case(seed, n, T, b_hi):
    rng = np.random.default_rng(seed)
    b = rng.integers(2, b_hi + 1, n)
    x = np.stack([rng.integers(0, bb, T) for bb in b]).astype(np.int32)
    return O.remap(x)


def _regular(db, npv_t, bmax, dev):
    n = db.n
    out = torch.zeros((n, n), dtype=torch.float32, device=dev)
    ws = D.workspace(dev, n, db.row_len, bmax)
    native.call("tenex_te_pairfree", db.data.data_ptr(), db.ld, npv_t.data_ptr(), bmax, n,
                db.row_len, 1, 0, n * (n - 1), out.data_ptr(), native.OUT_MATRIX, n,
                ws.data_ptr(), ws.numel(), None, native.stream_ptr())
    native.call("tenex_workspace_status", ws.data_ptr(), native.stream_ptr())
    return out


def _static(db, npv_t, bmax, dev, n_pairs=None, expect=0):
    n = db.n
    out = torch.zeros((n, n), dtype=torch.float32, device=dev)
    status = torch.full((1,), -1, dtype=torch.int32, device=dev)
    native.call("tenex_te_pairfree_static", db.data.data_ptr(), db.ld, npv_t.data_ptr(), bmax, n,
                db.row_len, 1, 0, n * (n - 1) if n_pairs is None else n_pairs, out.data_ptr(),
                native.OUT_MATRIX, n, status.data_ptr(), None, native.stream_ptr())
    torch.cuda.synchronize(dev)
    assert int(status.item()) == expect
    return out


def test_static_scratch_matches_workspace_entry_twice(cuda):
    cases = [_case(1, 48, 3001, 16), _case(2, 37, 1200, 38)]
    for bins, npv, bmax in cases:  # two calls in a row, different shapes and data
        db = D.pack_bins(bins, cuda)
        npv_t = torch.as_tensor(npv, dtype=torch.int32, device=cuda)
        a = _static(db, npv_t, bmax, cuda).cpu().numpy()
        b = _regular(db, npv_t, bmax, cuda).cpu().numpy()
        assert np.max(np.abs(a - b)) <= TOL
        assert np.max(np.abs(a - O.te_matrix(bins, npv))) <= TOL


def test_static_scratch_rejects_oversized_problem(cuda):
    # 1,500,000 genes need ~6 MB of scratch (4 bytes each): refused before any launch
    st = native.lib().tenex_te_pairfree_static(None, 64, None, 38, 1_500_000, 100, 1, 0, 10,
                                               None, 0, 0, None, None, None)
    assert st == native.TENEX_ERR_UNSUPPORTED
    assert "scratch" in native.last_error()


def test_static_status_after_invalid_and_empty_calls(cuda):
    """The status word reports each call's own outcome: invalid bins (a bin value
    >= its gene's n_per_var, caught by the device-side check without a fault)
    give 1 and leave the output untouched; an empty pair range right after gives
    0, not the previous call's word; a valid call after both matches the
    oracle with status 0 (no flag of the failed call survives in the shared area)."""
    bins, npv, bmax = _case(3, 20, 700, 9)
    db = D.pack_bins(bins, cuda)
    bad = np.asarray(npv, np.int32).copy()
    bad[4] = max(1, int(bad[4]) - 1)
    bad_t = torch.as_tensor(bad, dtype=torch.int32, device=cuda)
    out = _static(db, bad_t, bmax, cuda, expect=1)
    assert not bool(out.any())
    _static(db, bad_t, bmax, cuda, n_pairs=0, expect=0)
    npv_t = torch.as_tensor(npv, dtype=torch.int32, device=cuda)
    good = _static(db, npv_t, bmax, cuda).cpu().numpy()
    assert np.max(np.abs(good - O.te_matrix(bins, npv))) <= TOL


def test_static_scratch_refuses_global_memory_overflow(cuda):
    """Bins whose largest histograms need global-memory slots (coarsening off:
    120 bins at 70,000 samples) are refused before any launch, with a message
    that names the workspace entry point."""
    st = native.lib().tenex_te_pairfree_static(None, 70016, None, 120, 4, 70000, 1, 0, 12,
                                               None, 0, 0, None, None, None)
    assert st == native.TENEX_ERR_UNSUPPORTED
    assert "tenex_te_pairfree" in native.last_error()
