"""Exact triangle counting, forward orientation (drop-in for the reference's
``src/exact.py``).

``exact_triangle_count(forward_adj, r, per_edge_timing)`` keeps the reference's
signature and return tuple (src/exact.py:48-98): the dict is marshalled once
into a device CSR and counted by libtchll's exact kernel.  ``r`` (the
merge/binary-search ratio) is accepted for parity; the device kernel picks its
intersection method per edge group on its own, with identical counts.

With ``per_edge_timing=True`` the per-edge records ``(u, v, deg_u, deg_v,
support, time_s)`` come in the reference's order (dict order, skipping edges
whose lists are empty, src/exact.py:79-91); ``support`` is exact.  ``time_s``
differs from the reference's: the reference clocks each intersection on the
host (src/exact.py:86-90), while here all edges are counted by one device
launch, which has no per-edge clock.  Each edge's ``time_s`` is the call's
measured time apportioned by the edge's probe count, min(deg_u, deg_v) + 1
(the kernel probes the shorter list into a table of the longer one), so the
records sum to ``elapsed`` and rank edges by their real cost.
"""
from __future__ import annotations

import time
from typing import Dict, List, Tuple

import numpy as np
import torch

from . import _lib, core


def _pair_csr(a: np.ndarray, b: np.ndarray):
    a = np.asarray(a).reshape(-1)
    b = np.asarray(b).reshape(-1)
    for x in (a, b):
        if x.size and (x.min() < np.iinfo(np.int32).min or x.max() > np.iinfo(np.int32).max):
            raise ValueError("ids outside int32 are not supported")
    dev = torch.device("cuda", torch.cuda.current_device())
    col = torch.from_numpy(np.concatenate([a, b]).astype(np.int32)).to(dev)
    row_ptr = torch.tensor([0, a.size, a.size + b.size], dtype=torch.int32, device=dev)
    eu = torch.zeros(1, dtype=torch.int32, device=dev)
    ev = torch.ones(1, dtype=torch.int32, device=dev)
    return row_ptr, col, eu, ev


def _intersect_count(a, b) -> int:
    _lib.require_cuda()
    row_ptr, col, eu, ev = _pair_csr(a, b)
    res, _ = core.exact_count_tensors(row_ptr, col, eu, ev)
    return core.exact_from_result(res)


def intersect_merge(a: np.ndarray, b: np.ndarray) -> int:
    """|a cap b| of two sorted duplicate-free arrays (src/exact.py:12-14)."""
    return _intersect_count(a, b)


def intersect_bsearch(small: np.ndarray, large: np.ndarray) -> int:
    """|small cap large| (src/exact.py:17-26); same count as the merge."""
    if len(small) == 0:
        return 0
    return _intersect_count(small, large)


def intersect_adaptive(a: np.ndarray, b: np.ndarray, r: float = 8.0) -> int:
    """src/exact.py:29-41: zero for an empty side, else the intersection count."""
    if len(a) == 0 or len(b) == 0:
        return 0
    return _intersect_count(a, b)


def exact_triangle_count(forward_adj: Dict[int, np.ndarray], r: float = 8.0,
                         per_edge_timing: bool = False) -> Tuple[int, float, List]:
    """T = sum over oriented edges (u, v) of |N+(u) cap N+(v)|.

    Returns ``(count, elapsed_s, edge_data)`` (src/exact.py:48-98).  With
    per_edge_timing, edge_data holds ``(u, v, deg_u, deg_v, support, time_s)``
    per edge; time_s is modelled, not clocked: the call's elapsed time split
    in proportion to min(deg_u, deg_v) + 1, the edge's probe count."""
    _lib.require_cuda()
    adj = core.adjacency_with_missing_nodes(forward_adj)
    g = adj.csr
    edge_data: List = []
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res, pe = core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, per_edge=per_edge_timing)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    total = core.exact_from_result(res)
    if per_edge_timing:
        edge_data = _edge_records(forward_adj, adj, pe.cpu().numpy(), elapsed)
    return total, elapsed, edge_data


def _edge_records(forward_adj, adj: core.AdjacencyCSR, support_csr: np.ndarray, elapsed: float) -> List:
    """Per-edge tuples in the reference's iteration order."""
    keys = adj.keys.cpu().numpy()
    row_ptr = adj.csr.row_ptr.cpu().numpy().astype(np.int64)
    pos = {int(k): i for i, k in enumerate(keys)}
    lens = np.diff(row_ptr)
    recs = []
    for u, nbrs_u in forward_adj.items():
        if len(nbrs_u) == 0:
            continue
        i = pos[int(u)]
        base = int(row_ptr[i])
        for k, v in enumerate(nbrs_u):
            j = pos[int(v)]
            if lens[j] == 0:
                continue
            recs.append([u, int(v), len(nbrs_u), int(lens[j]), int(support_csr[base + k])])
    # the launch's time apportioned by each edge's probe count
    w = np.array([min(x[2], x[3]) + 1 for x in recs], dtype=np.float64)
    share = (elapsed * w / w.sum()) if recs else w
    return [tuple(x + [float(t)]) for x, t in zip(recs, share)]
