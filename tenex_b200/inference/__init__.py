"""Link inference on top of the TE matrix: the surrogate test (and its learned
null) through NetWeaver. Mirrors the registry of tenex/inference/__init__.py:32-81;
only 'surrogate_test' is part of the TE hot path built here."""
from tenex_b200.inference.grn import GRN, bh_fdr_gpu, build_pairs, make_grn  # noqa: F401
from tenex_b200.inference.surrogate_test import (SurrogateTestMethod,  # noqa: F401
                                                 SurrogateTestResult)
from tenex_b200.inference.netweaver import NetWeaver  # noqa: F401

_REGISTRY = {"surrogate_test": SurrogateTestMethod()}
_OUT_OF_SCOPE = ("fdr", "clr", "nd", "trace", "point")


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
