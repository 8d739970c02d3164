"""Multi-GPU counting: one process per GPU, edges sharded across ranks.

The count is a sum over oriented edges, and every edge's term depends only
on the (replicated) CSR, so the edges split into independent shards.  Each
rank counts a contiguous edge range whose cost (sum over its edges of
min(d+u, d+v) + 1, the probe work of the counting kernel) is about 1/world of
the total, then the ranks exchange their 64-byte result blocks once
(all_gather) and every rank combines them exactly with Python integers --
counts and the 2^-32 fixed-point HLL sums add without rounding, so the total
does not depend on the rank order.  ``torch.distributed`` (NCCL over NVLink
between GPUs, gloo in the CPU tests) carries the gather.

Graphs too many for one GPU's batch split the same way by graph (``shard_graphs``).
"""
from __future__ import annotations

import datetime
from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np
import torch
import torch.distributed as dist

from . import _lib


def edge_costs(degrees_u: np.ndarray, degrees_v: np.ndarray) -> np.ndarray:
    """Per-edge cost estimate: min(d+u, d+v) + 1."""
    return np.minimum(degrees_u, degrees_v).astype(np.int64) + 1


def shard_bounds(costs, world: int) -> List[Tuple[int, int]]:
    """Contiguous [lo, hi) edge ranges, one per rank, of about equal total cost."""
    c = np.asarray(costs, dtype=np.int64)
    n = len(c)
    if world <= 0:
        raise ValueError("world must be positive")
    if n == 0:
        return [(0, 0)] * world
    cum = np.cumsum(c)
    total = int(cum[-1])
    cuts = [0]
    for r in range(1, world):
        cuts.append(int(np.searchsorted(cum, total * r / world, side="left")) + 1)
    cuts.append(n)
    cuts = np.maximum.accumulate(np.minimum(np.array(cuts), n))
    return [(int(cuts[r]), int(cuts[r + 1])) for r in range(world)]


def shard_graphs(sizes: Sequence[int], world: int) -> List[List[int]]:
    """Graphs of a batch dealt to ranks greedily by size (largest first)."""
    order = np.argsort(-np.asarray(sizes, dtype=np.int64), kind="stable")
    load = np.zeros(world, dtype=np.int64)
    out: List[List[int]] = [[] for _ in range(world)]
    for i in order:
        r = int(np.argmin(load))
        out[r].append(int(i))
        load[r] += int(sizes[i])
    return [sorted(x) for x in out]


RESULT_FIELDS = ("exact", "hll_fx_lo", "hll_fx_hi", "n_approx", "n_exact", "n_fallback", "n_clamped", "status")


def result_to_tuple(r) -> Tuple[int, ...]:
    return tuple(int(getattr(r, f)) for f in RESULT_FIELDS)


def combine(parts: Sequence[Tuple[int, ...]]) -> dict:
    """Exact combination of per-rank result blocks: integer sums (128-bit HLL
    sums as Python ints), status OR-ed."""
    exact = sum(p[0] for p in parts)
    fx = sum((p[2] << 64) | p[1] for p in parts)
    out = {"exact": exact, "hll_fx": fx, "total": ((exact << 32) + fx) / 4294967296}
    for i, f in enumerate(RESULT_FIELDS[3:7], start=3):
        out[f] = sum(p[i] for p in parts)
    st = 0
    for p in parts:
        st |= p[7]
    out["status"] = st
    return out


def gather_results(local: Tuple[int, ...], group=None) -> List[Tuple[int, ...]]:
    """All-gather of the 8 result fields (as int64 bit patterns)."""
    world = dist.get_world_size(group)
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    vals = [v - (1 << 64) if v >= (1 << 63) else v for v in local]
    t = torch.tensor(vals, dtype=torch.int64, device=dev)
    out = [torch.empty_like(t) for _ in range(world)]
    dist.all_gather(out, t, group=group)
    res = []
    for o in out:
        res.append(tuple(int(x) & 0xFFFFFFFFFFFFFFFF for x in o.cpu().tolist()))
    return res


def sharded_count(n_edges: int, costs: np.ndarray, count_range: Callable[[int, int], Tuple[int, ...]],
                  group=None) -> dict:
    """Count this rank's shard with count_range(lo, hi) -> result fields, then
    combine every rank's partial.  Collective: every rank must call it."""
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    lo, hi = shard_bounds(costs, world)[rank]
    local = count_range(lo, hi)
    return combine(gather_results(local, group))


class ShardedExact:
    """One rank's part of an exact count split by edges: the rank's
    contiguous, cost-balanced edge range, counted with ``count_range(lo, hi)``
    (the libtchll kernels on a GPU, any counter of the same shape in a test),
    then one all_gather of the 64-byte result blocks and the exact integer
    combination.  ``step()`` returns the whole graph's count on every rank.
    Collective: every rank calls step() the same number of times."""

    def __init__(self, costs, count_range: Callable[[int, int], Tuple[int, ...]], group=None):
        self.group = group
        rank = dist.get_rank(group)
        world = dist.get_world_size(group)
        self.lo, self.hi = shard_bounds(costs, world)[rank]
        self.count_range = count_range

    def step(self) -> dict:
        local = self.count_range(self.lo, self.hi)
        return combine(gather_results(local, self.group))


def gpu_exact_range(g) -> Callable[[int, int], Tuple[int, ...]]:
    """count_range for the exact count on a device CSR (libtchll kernels)."""
    from . import core

    def run(lo: int, hi: int):
        res, _ = core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u[lo:hi].contiguous(),
                                          g.edge_v[lo:hi].contiguous())
        return result_to_tuple(_lib.read_count_result(res))
    return run


def gpu_hybrid_range(g, rows, slot, p: int, gamma: int) -> Callable[[int, int], Tuple[int, ...]]:
    from . import core

    def run(lo: int, hi: int):
        res, _ = core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u[lo:hi].contiguous(),
                                                   g.edge_v[lo:hi].contiguous(), g.degrees, rows, slot, p, gamma,
                                                   split_kernels=True)
        return result_to_tuple(_lib.read_count_result(res))
    return run


def device_costs(g) -> np.ndarray:
    deg = g.degrees.long()
    return (torch.minimum(deg[g.edge_u.long()], deg[g.edge_v.long()]) + 1).cpu().numpy()


def init(backend: str = "nccl", timeout_s: float = 60.0):
    """Process group for one-process-per-GPU runs (env:// rendezvous)."""
    kw = {}
    if backend == "nccl":
        import os
        dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", "0")))
        torch.cuda.set_device(dev)
        kw["device_id"] = dev
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s), **kw)
