"""Error paths without a GPU fault: host-side fault injection (TENEX_FAULT) makes
C-ABI calls fail with a chosen status, and the Python layers turn it into
TenexError (a RuntimeError) naming the entry point."""
import numpy as np
import pytest
import torch

from tenex_b200 import native
from tenex_b200.kernels import device as D


@pytest.mark.parametrize("kind,status", [("oom", native.TENEX_ERR_OOM),
                                         ("launch_fail", native.TENEX_ERR_LAUNCH),
                                         ("bad_shape", native.TENEX_ERR_BADARG),
                                         ("timeout", native.TENEX_ERR_TIMEOUT)])
def test_injected_status_reaches_caller(monkeypatch, kind, status):
    monkeypatch.setenv("TENEX_FAULT", f"{kind}:tenex_te_pairfree")
    x = np.random.default_rng(0).integers(0, 3, (4, 50)).astype(np.uint8)
    db = D.pack_bins(x, torch.device("cpu"))
    with pytest.raises(native.TenexError) as ei:
        D.te_pairfree(db, torch.full((4,), 3, dtype=torch.int32), 3, 1)
    assert ei.value.status == status
    assert "tenex_te_pairfree" in str(ei.value) and "TENEX_FAULT" in str(ei.value)
    assert isinstance(ei.value, RuntimeError)


def test_fault_targets_one_symbol_only(monkeypatch):
    monkeypatch.setenv("TENEX_FAULT", "oom:tenex_te_pairfree")
    buf = __import__("ctypes").create_string_buffer(64)
    native.call("tenex_last_error", buf, 64)   # another entry point still runs
    monkeypatch.setenv("TENEX_FAULT", "nonsense")
    with pytest.raises(ValueError):
        native.call("tenex_last_error", buf, 64)
