"""The C-ABI library loads and exports every symbol include/*.h declares."""
import ctypes
import glob
import os
import re

from tenex_b200 import native

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names |= set(re.findall(r"\b(tenex_[a-z0-9_]+)\s*\(", src))
    return names


def test_library_exports_declared_symbols():
    lib = native.lib()
    declared = _declared()
    assert declared, "no declarations found"
    missing = [n for n in sorted(declared) if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_declarations():
    assert set(native.declared_symbols()) >= _declared()


def test_abi_version_and_error_text_without_gpu():
    lib = native.lib()
    assert lib.tenex_abi_version() >= 1
    buf = ctypes.create_string_buffer(64)
    assert lib.tenex_last_error(buf, 64) == 0
    # argument checks run before any CUDA call
    st = lib.tenex_te_pairfree(None, 64, None, 4, 8, 100, 1, 0, 10, None, 0, 0, None, 0, None,
                               None)
    assert st == native.TENEX_ERR_BADARG
    assert "non-NULL" in native.last_error()
