"""The reference's other estimators, on the GPU, for comparison runs.

The main estimator is src/hll.py + src/hybrid.py (modules ``hll`` and
``hybrid``).  The reference's CPU experiment (cpu_exp/triangle_hll_
experiment.py) uses a different HLL variant, and its published CPU numbers
are quoted with it: splitmix64 with the +0x9E3779B97F4A7C15 increment and a
seed, register index from the LOW p bits, rank from h >> p, the 2^32
large-range correction, registers for every vertex, and the route "exact iff
min(d+u, d+v) <= threshold" (threshold < 0: pure HLL, ``--run pure-hll``).

``cx_hybrid_count`` returns the same tuple as the reference's hybrid_count
(:480-498): (total, exact_edges, hll_edges, exact_sum, hll_sum, clamp_count).
Sums are exact integers / 2^-32 fixed point here, so they do not depend on
thread order the way the reference's parallel Numba sums do.
"""
from __future__ import annotations

import ctypes as C
from typing import Tuple

import torch

from . import _lib, core
from ._lib import check, load, ptr, stream_handle


def cx_build_registers(g: core.DeviceCSR, p: int, seed: int = 1) -> Tuple[torch.Tensor, torch.Tensor]:
    """Dense n x 2^p registers of the cpu_exp variant (and an all-ones
    has-sketch vector)."""
    if not 4 <= p <= 16:
        raise ValueError(f"p must be in [4, 16], got {p}")
    dev = g.device
    regs = torch.empty(max(g.n_nodes, 1) << p, dtype=torch.uint8, device=dev)
    has = torch.empty(max(g.n_nodes, 1), dtype=torch.uint8, device=dev)
    check(load().tchll_cx_build_registers(ptr(g.row_ptr), g.n_nodes, ptr(g.col_idx), g.n_edges, int(p),
                                          int(seed) & 0xFFFFFFFFFFFFFFFF, ptr(regs), ptr(has),
                                          stream_handle(dev)), "cx registers")
    return regs, has


def cx_hybrid_count(g: core.DeviceCSR, regs: torch.Tensor, has: torch.Tensor, p: int, threshold: int):
    """(total, exact_edges, hll_edges, exact_sum, hll_sum, clamp_count), the
    reference's hybrid_count tuple; threshold < 0 gives the pure-HLL count."""
    dev = g.device
    res = _lib.count_result_tensor(dev)
    nb = C.c_size_t(0)
    check(load().tchll_hybrid_workspace_bytes(g.n_nodes, g.n_edges, g.n_nodes, int(p), C.byref(nb)))
    ws = _lib.workspace.get(nb.value, dev)
    check(load().tchll_cx_hybrid_count(ptr(g.row_ptr), g.n_nodes, ptr(g.col_idx), g.n_edges, ptr(g.edge_u),
                                       ptr(g.edge_v), g.n_edges, ptr(g.degrees), ptr(regs), ptr(has), int(p),
                                       int(threshold), ptr(res), ptr(ws), ws.numel(), stream_handle(dev)),
          "cx hybrid count")
    total, r = core.hybrid_from_result(res)
    hll_sum = ((int(r.hll_fx_hi) << 64) | int(r.hll_fx_lo)) / 4294967296
    return total, int(r.n_exact), int(r.n_approx), float(r.exact), hll_sum, int(r.n_clamped)


def pure_hll_count(g: core.DeviceCSR, regs: torch.Tensor, has: torch.Tensor, p: int):
    """(total, clamp_count) of the pure-HLL count (pure_hll_count,
    cpu_exp/triangle_hll_experiment.py:466-476)."""
    t = cx_hybrid_count(g, regs, has, p, -1)
    return t[0], t[5]
