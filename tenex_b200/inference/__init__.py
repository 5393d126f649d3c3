"""Link inference on top of the TE matrix through NetWeaver: the surrogate test
(and its learned null) and the FDR method (z-score, BH, DPI trimming). Mirrors
the registry of tenex/inference/__init__.py:32-81; CLR, ND, TRACE and POINT are
not part of this package."""
from tenex_b200.inference.grn import GRN, bh_fdr_gpu, build_pairs, make_grn  # noqa: F401
from tenex_b200.inference.surrogate_test import (SurrogateTestMethod,  # noqa: F401
                                                 SurrogateTestResult)
from tenex_b200.inference.fdr import FDRMethod  # noqa: F401
from tenex_b200.inference.netweaver import NetWeaver  # noqa: F401

_REGISTRY = {"surrogate_test": SurrogateTestMethod(), "fdr": FDRMethod()}
_OUT_OF_SCOPE = ("clr", "nd", "trace", "point")


def register(method) -> None:
    _REGISTRY[method.name] = method


def get_method(name: str):
    if name in _REGISTRY:
        return _REGISTRY[name]
    if name in _OUT_OF_SCOPE:
        raise NotImplementedError(f"inference method '{name}' is outside the TE hot path "
                                  f"this package implements; available: {available_methods()}")
    raise KeyError(f"Unknown method '{name}'. Available: {available_methods()}")


def available_methods() -> list[str]:
    return sorted(_REGISTRY)
