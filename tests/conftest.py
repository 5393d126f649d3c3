import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    import numpy as np

    def load(name):
        return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))
    return load


@pytest.fixture(scope="session")
def cuda():
    """The CUDA device for gpu-marked tests; the native library must load."""
    import torch
    from tenex_b200 import native
    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    native.lib()
    return torch.device("cuda:0")


@pytest.fixture(scope="session")
def full_size_multibin(cuda):
    """The 10,000-gene x 20,000-cell workload (95% of genes b ~ U{2..16}, 5% b ~
    U{64..256} coarsened to 38 bins by the oracle) and its all-pairs TE matrix
    [src, tgt] on the device, built once per session for the full-size tests."""
    import numpy as np
    import torch
    from oracle import oracle as O
    from tenex_b200 import workloads as W
    from tenex_b200.kernels import device as D
    from tenex_b200.kernels.adaptive_smem import AdaptiveSMEMKernel
    x, npv = W.cfg4_bins(10000, 20000, seed=1004)
    cb, cnpv, bmax = O.coarsen(x, npv, 38)
    cb = np.ascontiguousarray(cb, dtype=np.uint8)
    db = D.pack_bins(cb, cuda)
    npv_t = torch.as_tensor(cnpv, dtype=torch.int32, device=cuda)
    k = AdaptiveSMEMKernel()
    m = k.compute_pairfree_device(db, npv_t, int(bmax), 1, matrix=True)
    return dict(bins=cb, npv=np.asarray(cnpv), npv_raw=np.asarray(npv), b_max=int(bmax),
                db=db, npv_t=npv_t, kernel=k, matrix=m)
