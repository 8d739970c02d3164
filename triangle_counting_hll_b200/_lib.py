"""ctypes binding of libtchll.so (C ABI in include/tchll.h).

The shared library is built in-tree by ``triangle_counting_hll_b200/csrc/build.py``
(``__graft_entry__.build()``).  There is no CPU fallback: if the library or a
CUDA device is missing, every entry point raises.

Device buffers are torch CUDA tensors; objects exposing
``__cuda_array_interface__`` (Numba device arrays, CuPy arrays) are accepted at
the public boundary and wrapped without copies.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from typing import Optional

import numpy as np
import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtchll.so")

TCHLL_OK = 0
TCHLL_EINVAL = 1
TCHLL_ECUDA = 2
TCHLL_EWORKSPACE = 3

STATUS_BAD_EDGE = 1
STATUS_BAD_ROW = 2
STATUS_BAD_SLOT = 4
STATUS_BAD_KEY = 8


class TchllError(RuntimeError):
    """A CUDA or workspace failure inside libtchll."""


class CountResult(C.Structure):
    """Mirror of ``tchll_count_result`` (include/tchll.h)."""

    _fields_ = [("exact", C.c_uint64), ("hll_fx_lo", C.c_uint64), ("hll_fx_hi", C.c_uint64),
                ("n_approx", C.c_int64), ("n_exact", C.c_int64), ("n_fallback", C.c_int64),
                ("n_clamped", C.c_int64), ("status", C.c_uint32), ("reserved", C.c_uint32)]


RESULT_BYTES = C.sizeof(CountResult)
assert RESULT_BYTES == 64

_P = C.c_void_p
_I64 = C.c_int64
_I32 = C.c_int32
_U32 = C.c_uint32
_U64 = C.c_uint64
_SZ = C.c_size_t

# name -> (restype, argtypes); every symbol include/tchll.h declares.
SIGNATURES = {
    "tchll_last_error": (C.c_char_p, []),
    "tchll_version": (C.c_int, []),
    "tchll_launch_count": (_U64, []),
    "tchll_count_workspace_bytes": (C.c_int, [_I64, _I64, C.POINTER(_SZ)]),
    "tchll_hybrid_workspace_bytes": (C.c_int, [_I64, _I64, _I64, C.c_int32, C.POINTER(_SZ)]),
    "tchll_exact_count": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _P, _SZ, _P]),
    "tchll_exact_count_staged": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _SZ, _P, _P]),
    "tchll_hybrid_count_dense": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _P, _I32, _I64, _I32,
                                           _P, _P, _SZ, _P]),
    "tchll_hybrid_count_compact": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _I64, _P, _I32, _I64,
                                             _I32, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "tchll_set_count_tuning": (C.c_int, [_I32, _I32, _I32, _I32]),
    "tchll_set_count_shape": (C.c_int, [_I32, _I32]),
    "tchll_set_count_table": (C.c_int, [_I32]),
    "tchll_get_count_tuning": (C.c_int, [_P]),
    "tchll_set_count_hub": (C.c_int, [_I32, _I32, _I32, _I32]),
    "tchll_get_count_hub": (C.c_int, [_P]),
    "tchll_set_count_core": (C.c_int, [_I32, _I32, _I32, _I32]),
    "tchll_get_count_core": (C.c_int, [_P]),
    "tchll_set_hll_pass": (C.c_int, [_I32, _I32]),
    "tchll_get_hll_pass": (C.c_int, [_P]),
    "tchll_exact_count_noalloc": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P]),
    "tchll_set_phase_timing": (C.c_int, [_I32]),
    "tchll_phase_times": (C.c_int, [_P]),
    "tchll_phase_hub_ms": (C.c_int, [_P]),
    "tchll_sketch_workspace_bytes": (C.c_int, [_I64, C.POINTER(_SZ)]),
    "tchll_build_sketches_dense": (C.c_int, [_P, _I64, _P, _I64, _I64, _I32, _P, _P, _P]),
    "tchll_sketch_slots": (C.c_int, [_P, _I64, _I64, _P, _P, _P, _SZ, _P]),
    "tchll_build_sketches_compact": (C.c_int, [_P, _I64, _P, _P, _I64, _P, _I64, _I32, _P, _P]),
    "tchll_hll_add": (C.c_int, [_P, _I32, _P, _I64, _P]),
    "tchll_hll_estimate_pairs": (C.c_int, [_P, _I64, _I32, _P, _P, _I64, _P, _P]),
    "tchll_hash64": (C.c_int, [_P, _I64, _P, _P]),
    "tchll_cx_build_registers": (C.c_int, [_P, _I64, _P, _I64, _I32, _U64, _P, _P, _P]),
    "tchll_cx_hybrid_count": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _P, _I32, _I64, _P, _P, _SZ, _P]),
    "tchll_csr_workspace_bytes": (C.c_int, [_I64, C.POINTER(_SZ)]),
    "tchll_csr_build_phase1": (C.c_int, [_P, _P, _I64, _P, _P, _SZ, _P]),
    "tchll_csr_build_phase2": (C.c_int, [_I64, _I64, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _SZ, _P]),
    "tchll_adj_workspace_bytes": (C.c_int, [_I64, _I64, C.POINTER(_SZ)]),
    "tchll_csr_from_adjacency": (C.c_int, [_P, _P, _I64, _P, _I64, _P, _P, _P, _P, _P, _P, _P, _P, _P, _SZ,
                                           _P]),
    "tchll_batch_workspace_bytes": (C.c_int, [_I64, _I64, _I64, C.POINTER(_SZ)]),
    "tchll_batch_exact_count": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _I64, _P, _P, _SZ, _P]),
    "tchll_batch_hybrid_count": (C.c_int, [_P, _I64, _P, _I64, _P, _P, _I64, _P, _P, _I64, _P, _I32, _I64, _P, _I64,
                                           _P, _P, _SZ, _P]),
    "tchll_batch_local_ids": (C.c_int, [_P, _I64, _I64, _P, _P]),
    "tchll_degree_stats": (C.c_int, [_P, _P, _I64, _P, _P, _P, _P]),
    "tchll_ingest_workspace_bytes": (C.c_int, [_I64, C.POINTER(_SZ)]),
    "tchll_parse_edges": (C.c_int, [_P, _I64, C.c_char_p, _P, _P, _P, _P, _P, _SZ, _P]),
    "tchll_gen_rmat": (C.c_int, [_I32, _I64, _U32, _U32, _U32, _U64, _P, _P, _P]),
    "tchll_gen_er": (C.c_int, [_I64, _I64, _U64, _P, _P, _P]),
    "tchll_gen_lattice_count": (_I64, [_I64, _I64]),
    "tchll_gen_lattice": (C.c_int, [_I64, _I64, _U32, _U32, _U64, _P, _P, _P]),
    "tchll_gen_chung_lu": (C.c_int, [_P, _I64, _I64, _U64, _P, _P, _P]),
}

_lib = None
_lock = threading.Lock()


def load() -> C.CDLL:
    """Load libtchll.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"libtchll.so not found at {LIB_PATH}; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or "
                "`python triangle_counting_hll_b200/csrc/build.py`")
        lib = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
    return _lib


def last_error() -> str:
    msg = load().tchll_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str = "") -> None:
    """Raise for a non-zero libtchll status (ValueError for invalid arguments,
    mirroring the reference's ValueError conventions)."""
    if rc == TCHLL_OK:
        return
    msg = last_error()
    if rc == TCHLL_EINVAL:
        raise ValueError(msg)
    raise TchllError(f"{what}: {msg}" if what else msg)


def launch_count() -> int:
    return int(load().tchll_launch_count())


def require_cuda() -> None:
    if not torch.cuda.is_available():
        raise RuntimeError("triangle_counting_hll_b200 needs a CUDA device (no CPU fallback)")


# ------------------------------------------------------------ tensor plumbing
_TORCH_FROM_STR = {
    "<i4": torch.int32, "<i8": torch.int64, "|u1": torch.uint8, "<u1": torch.uint8,
    "|i1": torch.int8, "<f8": torch.float64, "<f4": torch.float32, "<u8": torch.uint64,
    "<u4": torch.uint32,
}


class _CAIWrapper:
    """Re-exports a foreign __cuda_array_interface__ so torch can alias it."""

    def __init__(self, obj):
        cai = dict(obj.__cuda_array_interface__)
        self.__cuda_array_interface__ = cai
        self._keep = obj


def as_device_tensor(x, dtype: torch.dtype, name: str = "array", device=None) -> torch.Tensor:
    """Return a contiguous CUDA tensor of ``dtype`` viewing (or, when the dtype or
    memory location differs, copying) ``x``.

    Accepts torch tensors, objects with ``__cuda_array_interface__`` (aliased,
    no copy) and host arrays (copied to the device)."""
    if isinstance(x, torch.Tensor):
        t = x
    elif hasattr(x, "__cuda_array_interface__"):
        t = torch.as_tensor(_CAIWrapper(x), device="cuda")
    else:
        t = torch.as_tensor(np.asarray(x))
    dev = device if device is not None else (t.device if t.is_cuda else torch.device("cuda", torch.cuda.current_device()))
    if t.device != dev or t.dtype != dtype:
        t = t.to(device=dev, dtype=dtype)
    if not t.is_contiguous():
        t = t.contiguous()
    return t


def ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    if t is None:
        return None
    return t.data_ptr() if t.numel() > 0 else None


def stream_handle(device=None) -> int:
    return torch.cuda.current_stream(device).cuda_stream


class Workspace:
    """Grow-only device scratch buffers owned by the caller side (the library
    never allocates), one per (device, current stream): a buffer is only ever
    used by work on the stream it was allocated on, so the caching allocator
    never hands its memory to another stream while a kernel still reads it."""

    def __init__(self):
        self._buf = {}

    def get(self, nbytes: int, device) -> torch.Tensor:
        dev = torch.device(device)
        idx = dev.index if dev.index is not None else torch.cuda.current_device()
        key = (idx, torch.cuda.current_stream(idx).cuda_stream)
        b = self._buf.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
            self._buf[key] = b
        return b

    def clear(self) -> None:
        self._buf.clear()


workspace = Workspace()


def count_result_tensor(device) -> torch.Tensor:
    return torch.empty(RESULT_BYTES, dtype=torch.uint8, device=device)


def read_count_result(t: torch.Tensor) -> CountResult:
    """Copy a device count result to the host (synchronises the stream)."""
    host = t.cpu().numpy().tobytes()
    return CountResult.from_buffer_copy(host)


def raise_on_status(res: CountResult) -> None:
    if res.status:
        parts = []
        if res.status & STATUS_BAD_EDGE:
            parts.append("edge endpoint outside [0, n_nodes)")
        if res.status & STATUS_BAD_ROW:
            parts.append("row_ptr extent outside [0, nnz] or decreasing")
        if res.status & STATUS_BAD_SLOT:
            parts.append("sketch slot outside the register rows")
        if res.status & STATUS_BAD_KEY:
            parts.append("neighbour id outside [0, n_nodes)")
        raise ValueError("malformed graph input: " + "; ".join(parts))


def hll_total(res: CountResult) -> float:
    """HLL fixed-point sum (units of 2^-32, 128-bit) as a float."""
    return (res.hll_fx_hi * 18446744073709551616.0 + res.hll_fx_lo) / 4294967296.0
