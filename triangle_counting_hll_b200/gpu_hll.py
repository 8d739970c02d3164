"""GPU HLL sketch building and union estimation (drop-in for the reference's
``src/gpu_hll.py``).

``build_sketches_kernel[grid, block](row_ptr, col_idx, n_nodes, theta, p,
sketch_regs, has_sketch)`` keeps the reference's launch form
(src/gpu_hll.py:47-81, launched by experiment/exp_gpu.py:552-557) and runs
libtchll's CTA-per-vertex sketch kernel; like the reference it covers vertices
``u < min(n_nodes, grid * block)`` and max-merges into the rows it is given.
``sketch_regs`` / ``has_sketch`` are written in place, so they must already be
uint8 device buffers (torch CUDA tensors or ``__cuda_array_interface__``
objects).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, core
from ._lib import as_device_tensor


def _alpha(m: int) -> float:
    """HLL bias constant (src/gpu_hll.py:20-28, src/hll.py:26-34)."""
    if m == 16:
        return 0.673
    if m == 32:
        return 0.697
    if m == 64:
        return 0.709
    return 0.7213 / (1.0 + 1.079 / m)


def _inplace_u8(x, name: str, device) -> torch.Tensor:
    t = as_device_tensor(x, torch.uint8, name, device)
    if isinstance(x, torch.Tensor):
        if x.data_ptr() != t.data_ptr():
            raise TypeError(f"{name} must be a contiguous uint8 CUDA buffer (it is written in place)")
    elif hasattr(x, "__cuda_array_interface__"):
        if x.__cuda_array_interface__["data"][0] != t.data_ptr():
            raise TypeError(f"{name} must be a contiguous uint8 CUDA buffer (it is written in place)")
    else:
        raise TypeError(f"{name} must be a device buffer (it is written in place)")
    return t


class _SketchLauncher:
    def __init__(self, n_threads: int):
        self.n_threads = n_threads

    def __call__(self, row_ptr, col_idx, n_nodes, theta, p, sketch_regs, has_sketch):
        _lib.require_cuda()
        dev = None
        for x in (row_ptr, col_idx, sketch_regs):
            if isinstance(x, torch.Tensor) and x.is_cuda:
                dev = x.device
                break
        rp = as_device_tensor(row_ptr, torch.int32, "row_ptr", dev)
        dev = rp.device
        ci = as_device_tensor(col_idx, torch.int32, "col_idx", dev)
        regs = _inplace_u8(sketch_regs, "sketch_regs", dev)
        has = _inplace_u8(has_sketch, "has_sketch", dev)
        p = int(p)
        if not 4 <= p <= 16:
            raise ValueError(f"p must be in [4, 16], got {p}")
        n = min(int(n_nodes), int(self.n_threads), int(rp.numel()) - 1)
        if n <= 0:
            return
        if int(regs.numel()) < n * (1 << p) or int(has.numel()) < n:
            raise ValueError("sketch_regs / has_sketch too small for n_nodes * 2^p")
        with torch.cuda.device(dev):
            core.build_sketches_dense_tensors(rp, ci, n, int(theta), p, regs, has)


class _SketchKernel:
    """``build_sketches_kernel[grid, block](...)``; grid and block set the
    number of vertices covered (grid * block), as in the reference."""

    def __getitem__(self, cfg):
        grid, block = cfg[0], cfg[1]
        g = int(np.prod(grid)) if isinstance(grid, (tuple, list)) else int(grid)
        b = int(np.prod(block)) if isinstance(block, (tuple, list)) else int(block)
        if g < 0 or b <= 0:
            raise ValueError("invalid launch configuration")
        return _SketchLauncher(g * b)

    def __call__(self, *args, **kwargs):
        raise TypeError("build_sketches_kernel must be launched as build_sketches_kernel[grid, block](...)")


build_sketches_kernel = _SketchKernel()


def alloc_sketch_arrays(n_nodes: int, p: int):
    """Zeroed host arrays for sketch_regs (n_nodes * 2^p) and has_sketch
    (src/gpu_hll.py:128-133)."""
    m = 1 << p
    return np.zeros(n_nodes * m, dtype=np.uint8), np.zeros(n_nodes, dtype=np.uint8)


def alloc_sketch_arrays_device(n_nodes: int, p: int, device=None):
    """Zeroed device arrays of the same shapes, allocated on the GPU directly
    (no host zeros to copy, unlike alloc_sketch_arrays + to_device)."""
    _lib.require_cuda()
    dev = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    m = 1 << p
    return (torch.zeros(n_nodes * m, dtype=torch.uint8, device=dev),
            torch.zeros(n_nodes, dtype=torch.uint8, device=dev))


def union_estimate_rows(sketch_regs, u, v, p: int) -> float:
    """Union estimate of dense rows u and v (the device helper
    _union_estimate_device, src/gpu_hll.py:88-121, here in FP64)."""
    regs = as_device_tensor(sketch_regs, torch.uint8, "sketch_regs")
    out = core.estimate_pairs(regs, p, [int(u)], [int(v)])
    return float(out.item())
