"""tenex_b200 — the pairwise transfer-entropy path of TENEX on B200 (sm_100a).

Public API (same names as the reference package `tenex`):
    TransferEntropyEngine, TransferEntropyResult
    NetWeaver, SurrogateTestResult (inference.surrogate_test)
    Pipeline, PipelineResult (cached TE + surrogate test, multi-lag combine)
    discretize, remap_bins, coarsen_bins, binarize
    kernels: TEKernel, register, get_kernel, auto_select, registered_kernels
The compute runs in libtenex_sm100.so (tenex_b200/_lib), built by
`python -m tenex_b200.build`; there is no CPU path.
"""
__version__ = "0.1.0"

from tenex_b200.result import TransferEntropyResult  # noqa: E402
from tenex_b200.transferentropy import TransferEntropyEngine  # noqa: E402
from tenex_b200.preprocess import discretize, remap_bins, coarsen_bins  # noqa: E402
from tenex_b200.binarize import binarize  # noqa: E402

__all__ = ["TransferEntropyEngine", "TransferEntropyResult", "discretize", "remap_bins",
           "coarsen_bins", "binarize", "NetWeaver", "SurrogateTestResult", "Pipeline",
           "PipelineResult"]


def __getattr__(name):
    if name in ("NetWeaver", "SurrogateTestResult"):
        from tenex_b200 import inference
        return getattr(inference, name)
    if name in ("Pipeline", "PipelineResult"):
        from tenex_b200 import pipeline
        return getattr(pipeline, name)
    raise AttributeError(name)
