"""Verbose logging switch (reference: tenex/_log.py)."""
_VERBOSE = False


def set_verbose(flag: bool) -> None:
    global _VERBOSE
    _VERBOSE = bool(flag)


def vprint(*args, **kwargs) -> None:
    if _VERBOSE:
        print(*args, **kwargs)
