"""GPU exact and selective hybrid-HLL triangle counting (drop-in for the
reference's ``src/gpu_hybrid.py``).

Same entry points, arguments and return values as the reference
(``gpu_exact_triangle_count`` src/gpu_hybrid.py:332-354,
``gpu_hybrid_triangle_count`` :357-431); the work runs in libtchll's sm_100a
kernels (``tchll_exact_count`` / ``tchll_hybrid_count_dense``).  Device inputs
may be torch CUDA tensors or any ``__cuda_array_interface__`` object (Numba
device arrays, CuPy arrays); host arrays are copied to the current device.

Differences from the reference, by design:
  * the hybrid total is accumulated exactly in fixed point (each clamped
    per-edge estimate rounded to 2^-32), so it does not depend on launch
    order, and the union estimate sums 2^-r exactly before the FP64
    corrections (the reference GPU path uses FP32, src/gpu_hll.py:98-121);
  * malformed inputs (edge ids outside the CSR, decreasing row_ptr) raise
    ValueError instead of reading out of bounds.
"""
from __future__ import annotations

import time
import warnings

import torch

from . import _lib, core
from ._lib import as_device_tensor

# Every counting kernel here runs 256-thread CTAs; the constant and its check
# keep the reference's module surface (src/gpu_hybrid.py:13-24).
_THREADS = 256
_FLOAT64_ATOMIC_WARNED = False


def _require_supported_block_size() -> None:
    if _THREADS != 256:
        raise ValueError(
            "gpu_hybrid kernels require _THREADS == 256 (the CTA size libtchll's "
            "counting kernels are compiled for).")


def _warn_if_float64_atomic_slow(cuda_module=None) -> None:
    """Reference surface (src/gpu_hybrid.py:27-39).  This build adds HLL
    estimates with integer atomics, so only a pre-Pascal device would warn."""
    global _FLOAT64_ATOMIC_WARNED
    if _FLOAT64_ATOMIC_WARNED:
        return
    major, _ = torch.cuda.get_device_capability()
    if major < 6:
        warnings.warn("compute capability < 6.0 is not supported by libtchll", RuntimeWarning, stacklevel=2)
    _FLOAT64_ATOMIC_WARNED = True


def _inputs(row_ptr_d, col_idx_d, edge_u_d, edge_v_d):
    _lib.require_cuda()
    dev = None
    for x in (row_ptr_d, col_idx_d, edge_u_d, edge_v_d):
        if isinstance(x, torch.Tensor) and x.is_cuda:
            dev = x.device
            break
    rp = as_device_tensor(row_ptr_d, torch.int32, "row_ptr", dev)
    dev = rp.device
    ci = as_device_tensor(col_idx_d, torch.int32, "col_idx", dev)
    eu = as_device_tensor(edge_u_d, torch.int32, "edge_u", dev)
    ev = as_device_tensor(edge_v_d, torch.int32, "edge_v", dev)
    return rp, ci, eu, ev


def _is_host(x) -> bool:
    if isinstance(x, torch.Tensor):
        return not x.is_cuda
    return not hasattr(x, "__cuda_array_interface__")


def gpu_exact_triangle_count(row_ptr_d, col_idx_d, edge_u_d, edge_v_d):
    """Exact count over the given oriented edges; returns ``(count, elapsed_s)``
    where elapsed is the wall-clock time of the synchronised launch, as in the
    reference (src/gpu_hybrid.py:346-354).  Host arrays (all four) are copied
    in stages that overlap the count (``core.exact_count_host``), and elapsed
    then runs from the first copy to the result."""
    _require_supported_block_size()
    if all(_is_host(x) for x in (row_ptr_d, col_idx_d, edge_u_d, edge_v_d)):
        _lib.require_cuda()
        host = [x if isinstance(x, torch.Tensor) else torch.as_tensor(x)
                for x in (row_ptr_d, col_idx_d, edge_u_d, edge_v_d)]
        dev = torch.device("cuda", torch.cuda.current_device())
        with torch.cuda.device(dev):
            res = _lib.count_result_tensor(dev)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            core.exact_count_host(*host, device=dev, result=res)
            torch.cuda.synchronize()
            elapsed = time.perf_counter() - t0
            count = core.exact_from_result(res)
        return count, elapsed
    rp, ci, eu, ev = _inputs(row_ptr_d, col_idx_d, edge_u_d, edge_v_d)
    with torch.cuda.device(rp.device):
        res = _lib.count_result_tensor(rp.device)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        core.exact_count_tensors(rp, ci, eu, ev, result=res)
        torch.cuda.synchronize()
        elapsed = time.perf_counter() - t0
        count = core.exact_from_result(res)
    return count, elapsed


def gpu_hybrid_triangle_count(row_ptr_d, col_idx_d, edge_u_d, edge_v_d, degrees_d, sketch_regs_d, has_sketch_d,
                              gamma: int, p: int, split_kernels: bool = True):
    """Hybrid exact/HLL count over dense sketches (row v at v * 2^p, present iff
    has_sketch[v] == 1).  Returns ``(estimate, elapsed_s, stats)`` with the
    reference's stats keys (src/gpu_hybrid.py:415-430)."""
    _require_supported_block_size()
    _warn_if_float64_atomic_slow()
    rp, ci, eu, ev = _inputs(row_ptr_d, col_idx_d, edge_u_d, edge_v_d)
    dev = rp.device
    deg = as_device_tensor(degrees_d, torch.int32, "degrees", dev)
    regs = as_device_tensor(sketch_regs_d, torch.uint8, "sketch_regs", dev)
    has = as_device_tensor(has_sketch_d, torch.uint8, "has_sketch", dev)
    n_edges = int(eu.numel())
    with torch.cuda.device(dev):
        res = _lib.count_result_tensor(dev)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        core.hybrid_count_dense_tensors(rp, ci, eu, ev, deg, regs, has, int(gamma), int(p),
                                        split_kernels=bool(split_kernels), result=res)
        torch.cuda.synchronize()
        elapsed = time.perf_counter() - t0
        estimate, r = core.hybrid_from_result(res)
    n_approx, n_exact, n_clamped = int(r.n_approx), int(r.n_exact), int(r.n_clamped)
    stats = {
        "n_approx": n_approx,
        "n_exact": n_exact,
        "n_clamped": n_clamped,
        "approx_coverage": n_approx / n_edges if n_edges > 0 else 0.0,
        "clamp_ratio": n_clamped / n_approx if n_approx > 0 else 0.0,
        "kernel_mode": "split_block_reduction" if split_kernels else "fused_block_reduction",
    }
    return estimate, elapsed, stats
