"""Engine argument contracts that need no GPU."""
import numpy as np
import pytest

from tenex_b200 import TransferEntropyEngine
from tenex_b200.kernels import auto_select, compute_smem_bytes, get_kernel, registered_kernels


def test_constructor_validation():
    x = np.zeros((3, 10), np.float32)
    names = np.array(["a", "b", "c"])
    with pytest.raises(ValueError):
        TransferEntropyEngine(None, names)
    with pytest.raises(ValueError):
        TransferEntropyEngine(np.zeros(5, np.float32), names)
    with pytest.raises(ValueError):
        TransferEntropyEngine(np.full((3, 10), np.nan, np.float32), names)
    with pytest.raises(ValueError):
        TransferEntropyEngine(x, np.array(["a", "a", "c"]))
    with pytest.raises(ValueError):
        TransferEntropyEngine(x, names, sources=np.array(["zz"]))
    with pytest.raises(ValueError):
        TransferEntropyEngine(x, names, sources=np.array(["a", "a"]))


def test_cpu_accelerator_is_rejected():
    x = np.random.default_rng(0).random((3, 10)).astype(np.float32)
    eng = TransferEntropyEngine(x, np.array(["a", "b", "c"]))
    with pytest.raises(NotImplementedError):
        eng.compute(accelerator="cpu")
    with pytest.raises(ValueError):
        eng.compute(accelerator="tpu")


def test_registry_priority_matches_reference():
    assert [k.name for k in registered_kernels()] == ["GEMM-B2", "Full-SMEM", "Adaptive-SMEM"]
    optin = 232448
    assert auto_select(2, True, optin, compute_smem_bytes(2, 5000, 1, 1), None,
                       False).name == "GEMM-B2"
    assert auto_select(2, True, optin, compute_smem_bytes(2, 5000, 1, 1), None,
                       True).name == "Full-SMEM"
    assert auto_select(32, True, optin, compute_smem_bytes(32, 10000, 1, 1), None,
                       False).name == "Full-SMEM"
    assert auto_select(39, True, optin, compute_smem_bytes(39, 20000, 1, 1), None,
                       False).name == "Adaptive-SMEM"
    assert get_kernel("full-smem").name == "Full-SMEM"
    with pytest.raises(KeyError):
        get_kernel("scatter_add")
    with pytest.raises(RuntimeError):
        auto_select(4, False, 0, 0, None, False)


@pytest.mark.skipif(__import__("torch").cuda.is_available(), reason="needs a CUDA-less host")
def test_device_contract_without_cuda():
    # the reference's device contract (tests/test_device_contract.py): an explicitly
    # requested GPU must raise instead of computing elsewhere; this package has no
    # CPU path, so accelerator='auto' raises too rather than falling back
    x = np.random.RandomState(0).randn(12, 80).astype(np.float32)
    eng = TransferEntropyEngine(x, np.array([f"g{i}" for i in range(12)]))
    for kw in (dict(accelerator="gpu"), dict(accelerator="gpu", devices=[0]),
               dict(accelerator="auto")):
        with pytest.raises((RuntimeError, ValueError)):
            eng.compute(binning_method="FSBW-L", kp=0.5, tau=1, **kw)
    with pytest.raises((ValueError, RuntimeError)):
        eng.compute(accelerator="npu", binning_method="FSBW-L", kp=0.5, tau=1)
