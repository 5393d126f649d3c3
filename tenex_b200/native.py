"""ctypes binding of libtenex_sm100.so (the C ABI declared in include/tenex_sm100.h).

The library is built in-tree by tenex_b200.build. There is no fallback: if the
library is missing or fails to load, every GPU entry point raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libtenex_sm100.so")

TENEX_OK = 0
TENEX_ERR_BADARG = 1
TENEX_ERR_UNSUPPORTED = 2
TENEX_ERR_OOM = 3
TENEX_ERR_LAUNCH = 4
TENEX_ERR_TIMEOUT = 5
TENEX_ERR_BADDATA = 6

OUT_PAIRFREE = 0
OUT_MATRIX = 1

_STATUS_NAMES = {1: "BADARG", 2: "UNSUPPORTED", 3: "OOM", 4: "LAUNCH", 5: "TIMEOUT",
                 6: "BADDATA"}


class TenexError(RuntimeError):
    """A C-ABI call returned a non-zero tenex_status."""

    def __init__(self, status: int, where: str, msg: str):
        self.status = status
        super().__init__(f"{where}: TENEX_ERR_{_STATUS_NAMES.get(status, status)}: {msg}")


class DevInfo(ctypes.Structure):
    _fields_ = [("sm_count", ctypes.c_int), ("smem_optin", ctypes.c_int),
                ("smem_per_sm", ctypes.c_int), ("l2_bytes", ctypes.c_int),
                ("cc_major", ctypes.c_int), ("cc_minor", ctypes.c_int),
                ("max_threads_per_sm", ctypes.c_int)]


class TeConfig(ctypes.Structure):
    _fields_ = [("threads", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("src_chunk", ctypes.c_int), ("smem_bytes", ctypes.c_int)]


_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_S = ctypes.c_size_t

# name -> argtypes (restype int unless noted)
_SIGS = {
    "tenex_abi_version": [],
    "tenex_last_error": [ctypes.c_char_p, _S],
    "tenex_device_query": [_I, ctypes.POINTER(DevInfo)],
    "tenex_te_workspace_bytes": [_I, _L, _I],
    "tenex_te_launch_shape": [_L, _L, _I, _P, _P, _P, _P, _P],
    "tenex_workspace_status": [_P, _P],
    "tenex_te_pairfree": [_P, _L, _P, _I, _I, _L, _L, _L, _L, _P, _I, _L, _P, _S,
                          ctypes.POINTER(TeConfig), _P],
    "tenex_te_pairfree_counts": [_P, _L, _P, _I, _I, _L, _L, _L, _L, _P, _P, _L, _P, _S,
                                 ctypes.POINTER(TeConfig), _P],
    "tenex_te_pairfree_static": [_P, _L, _P, _I, _I, _L, _L, _L, _L, _P, _I, _L, _P,
                                 ctypes.POINTER(TeConfig), _P],
    "tenex_te_pairs": [_P, _L, _P, _I, _I, _L, _L, _P, _L, _P, _L, _P, _P, _S,
                       ctypes.POINTER(TeConfig), _P],
    "tenex_surrogate_accumulate": [_P, _L, _P, _I, _I, _L, _L, _L, _L, _P, _P, _P, _P, _P, _S,
                                   ctypes.POINTER(TeConfig), _P],
    "tenex_block_shuffle": [_P, _L, _I, _L, _I, _P, _I, _I, _P, _L, _P],
    "tenex_block_shuffle_many": [_P, _L, _I, _L, _I, _P, _I, _I, _I, _P, _L, _L, _P],
    "tenex_stats_accumulate": [_P, _P, _P, _P, _P, _I, _P],
    "tenex_surrogate_accumulate_pairs": [_P, _L, _P, _I, _I, _L, _L, _P, _L, _P, _L, _P, _P, _P,
                                         _P, _P, _S, ctypes.POINTER(TeConfig), _P],
    "tenex_fsbwl_bins": [_P, _L, _I, _I, ctypes.c_float, _P, _L, _P, _P],
    "tenex_remap_dense": [_P, _I, _L, _I, _L, _P, _I, _L, _P, _P, _P],
    "tenex_coarsen": [_P, _L, _I, _L, _P, _I, _P],
    "tenex_coarsen_narrow": [_P, _L, _I, _L, _P, _I, _P, _L, _P],
    "tenex_binarize": [_P, _L, _I, _I, _I, _P, _P, _L, _P, _P],
    "tenex_binarize_select": [_P, _L, _I, _I, _I, ctypes.c_double, _P, _L, _P, _P],
    "tenex_b2_workspace_bytes": [_I, _L, _L],
    "tenex_te_binary_matrix": [_P, _L, _I, _L, _L, _P, _L, _P, _S, _P],
    "tenex_te_binary_matrix_kind": [_P, _L, _I, _L, _L, _P, _L, _P, _S, _I, _P],
    "tenex_te_binary_matrix_ex": [_P, _L, _I, _L, _L, _P, _L, _P, _S, _I, _I, _P],
    "tenex_b2_tile_n": [_I, ctypes.POINTER(ctypes.c_int)],
    "tenex_b2_status": [_P, _I, _L, _L, _P],
    "tenex_dpi_trim": [_P, _L, _I, _P, _P, ctypes.c_float, _P, _L, _P],
    "tenex_dpi_trim_sparse": [_P, _P, _P, _I, _P, _P, ctypes.c_float, _P, _P],
    "tenex_mlp_param_count": [],
    "tenex_gene_features": [_P, _L, _P, _I, _L, _L, _P, _P],
    "tenex_eiid_workspace_bytes": [_I],
    "tenex_eiid_matrix": [_P, _L, _P, _I, _L, _L, _P, _P, _S, _P],
    "tenex_pair_features": [_P, _P, _I, _P, _P, _L, ctypes.c_float, _P, _P],
    "tenex_null_predict": [_P, _P, _I, ctypes.c_float, _P, _P, _P, _P, _P, _P],
    "tenex_mlp_scratch_floats": [_I],
    "tenex_mlp_gradients": [_P, _P, _I, _P, _P, _P, _P, _P],
    "tenex_mlp_train_step": [_P, _P, _I, _P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_float,
                             ctypes.c_float, ctypes.c_float, ctypes.c_float, _I, _P, _P],
    "tenex_to_bf16": [_P, _P, _I, _P],
    "tenex_probe_smem_atomics": [_I, _I, ctypes.POINTER(ctypes.c_int64),
                                 ctypes.POINTER(ctypes.c_float), _P],
    "tenex_probe_tc_int8": [_I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float),
                            _P],
    "tenex_probe_tc_fp4": [_I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float),
                           _P],
    "tenex_probe_tc_gemm_b2": [_I, _I, _I, ctypes.POINTER(ctypes.c_double),
                               ctypes.POINTER(ctypes.c_float), _P],
    "tenex_probe_minmax": [_I, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float),
                           _P],
}
_RESTYPES = {"tenex_te_workspace_bytes": ctypes.c_size_t,
             "tenex_b2_workspace_bytes": ctypes.c_size_t,
             "tenex_mlp_scratch_floats": ctypes.c_size_t,
             "tenex_eiid_workspace_bytes": ctypes.c_size_t}

_lib = None
_lock = threading.Lock()


def declared_symbols() -> list[str]:
    return list(_SIGS)


def lib() -> ctypes.CDLL:
    """Loads the library once (raises if it is missing: no CPU fallback exists)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise RuntimeError(
                    f"{LIB_PATH} is missing; build it with `python -m tenex_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, args in _SIGS.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = _RESTYPES.get(name, ctypes.c_int)
            _lib = L
    return _lib


def last_error() -> str:
    buf = ctypes.create_string_buffer(1024)
    lib().tenex_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(status: int, where: str) -> None:
    if status != TENEX_OK:
        raise TenexError(status, where, last_error())


_FAULT_CODES = {"bad_arg": TENEX_ERR_BADARG, "bad_shape": TENEX_ERR_BADARG,
                "unsupported": TENEX_ERR_UNSUPPORTED, "oom": TENEX_ERR_OOM,
                "launch_fail": TENEX_ERR_LAUNCH, "timeout": TENEX_ERR_TIMEOUT,
                "bad_data": TENEX_ERR_BADDATA}


def _injected_fault(name: str) -> int:
    """Host-side fault injection: TENEX_FAULT="kind[:symbol]" (kind in _FAULT_CODES)
    makes call() raise that status for `symbol` (every status-returning entry
    point if omitted) without running it, so the error paths can be exercised
    with no GPU fault."""
    spec = os.environ.get("TENEX_FAULT")
    if not spec:
        return TENEX_OK
    kind, _, sym = spec.partition(":")
    if sym and sym != name:
        return TENEX_OK
    if kind not in _FAULT_CODES:
        raise ValueError(f"TENEX_FAULT kind {kind!r} not in {sorted(_FAULT_CODES)}")
    return _FAULT_CODES[kind]


def call(name: str, *args) -> None:
    fault = _injected_fault(name)
    if fault:
        raise TenexError(fault, name, f"injected by TENEX_FAULT={os.environ['TENEX_FAULT']}")
    check(getattr(lib(), name)(*args), name)


_cuda_seen: bool | None = None   # whether this process sees a CUDA device (fixed per process)


def stream_ptr(stream: torch.cuda.Stream | None = None) -> int:
    """The stream handle for the C ABI (the current stream of the current device;
    0, the legacy default stream, when this process sees no CUDA device, in which
    case every entry point fails with its own status). The device check runs once
    per process and the handle comes straight from torch's current-stream table:
    torch.cuda.current_stream() re-checks device availability on every call
    (~20 us, a tenth of a small compute() call)."""
    global _cuda_seen
    if stream is not None:
        return int(stream.cuda_stream)
    if _cuda_seen is None:
        _cuda_seen = torch.cuda.is_available()
        if _cuda_seen:
            torch.cuda.init()
    if not _cuda_seen:
        return 0
    return int(torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice()))


def device_info(device: int | None = None) -> DevInfo:
    if device is None:
        device = torch.cuda.current_device()
    info = DevInfo()
    call("tenex_device_query", int(device), ctypes.byref(info))
    return info


def te_config(threads=0, ctas_per_sm=0, src_chunk=0, smem_bytes=0) -> TeConfig:
    return TeConfig(int(threads), int(ctas_per_sm), int(src_chunk), int(smem_bytes))


def probe_smem_atomics(mode: int = 0, iters: int = 4096) -> float:
    """Measured shared-memory atomic increments per second over all SMs."""
    inc = ctypes.c_int64()
    ms = ctypes.c_float()
    call("tenex_probe_smem_atomics", int(mode), int(iters), ctypes.byref(inc), ctypes.byref(ms),
         stream_ptr())
    return inc.value / (ms.value * 1e-3)


def probe_tc_int8(iters: int = 100_000) -> float:
    """Measured dense INT8 tensor-pipe operations per second over all SMs."""
    ops = ctypes.c_double()
    ms = ctypes.c_float()
    call("tenex_probe_tc_int8", int(iters), ctypes.byref(ops), ctypes.byref(ms), stream_ptr())
    return ops.value / (ms.value * 1e-3)


def te_launch_shape(row_len: int, lag: int, b_max: int, cfg: dict | None = None) -> dict:
    """The launch shape the histogram kernels resolve on the current device for
    this series length, lag, b_max and requested config (0 / None = defaults)."""
    c = cfg or {}
    tc = te_config(c.get("threads", 0), c.get("ctas_per_sm", 0), c.get("src_chunk", 0),
                   c.get("smem_bytes", 0))
    out = [ctypes.c_int() for _ in range(4)]
    call("tenex_te_launch_shape", int(row_len), int(lag), int(b_max), ctypes.byref(tc),
         *[ctypes.byref(v) for v in out])
    return dict(threads=out[0].value, ctas_per_sm=out[1].value, smem_bytes=out[2].value,
                src_chunk=out[3].value)


def probe_tc_fp4(iters: int = 100_000) -> float:
    """Measured dense 4-bit (kind::mxf4) tensor-pipe operations per second over all SMs."""
    ops = ctypes.c_double()
    ms = ctypes.c_float()
    call("tenex_probe_tc_fp4", int(iters), ctypes.byref(ops), ctypes.byref(ms), stream_ptr())
    return ops.value / (ms.value * 1e-3)


def probe_tc_gemm_b2(operands: str = "fp4", tile_n: int = 128, stages: int = 2000) -> float:
    """Measured operations per second of the GEMM-B2 kernel's own MMA sequence
    (operands "fp4" or "int8", tile_n targets per tile) issued back to back on
    every SM: the instruction-mix bound of the GEMM's main loop."""
    ops = ctypes.c_double()
    ms = ctypes.c_float()
    call("tenex_probe_tc_gemm_b2", 2 if operands == "fp4" else 1, int(tile_n), int(stages),
         ctypes.byref(ops), ctypes.byref(ms), stream_ptr())
    return ops.value / (ms.value * 1e-3)


def probe_minmax(iters: int = 20_000) -> float:
    """Measured FP32 min/max instructions per second over all SMs."""
    ins = ctypes.c_double()
    ms = ctypes.c_float()
    call("tenex_probe_minmax", int(iters), ctypes.byref(ins), ctypes.byref(ms), stream_ptr())
    return ins.value / (ms.value * 1e-3)
