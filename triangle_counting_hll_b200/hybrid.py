"""Selective hybrid HLL triangle counting (drop-in for the reference's
``src/hybrid.py``).

``build_sketches`` builds every sketch of a forward adjacency dict in one
device launch (rows in one compact buffer; each returned ``HLL`` is a view of
its row) and hashes the ids the dict holds, as src/hybrid.py:36-40 does.
``hybrid_triangle_count`` routes each oriented edge exactly like
src/hybrid.py:95-148 (HLL iff min(d+u, d+v) >= gamma and both endpoints are in
``sketches``) in libtchll's fused exact/HLL kernel and returns the reference's
``(total, elapsed, stats, details)``.
"""
from __future__ import annotations

import time
from typing import Dict, List, Optional, Tuple

import numpy as np
import torch

from . import _lib, core
from .hll import HLL


def build_sketches(forward_adj: Dict[int, np.ndarray], theta: int, p: int = 8) -> Dict[int, HLL]:
    """One HLL per node whose forward degree >= theta (src/hybrid.py:15-41)."""
    if not (4 <= p <= 16):
        raise ValueError(f"p must be in [4, 16], got {p}")
    _lib.require_cuda()
    sk, _ = _build_compact(forward_adj, theta, p)
    return sk


def _build_compact(forward_adj, theta: int, p: int):
    adj = core.adjacency_with_missing_nodes(forward_adj)
    g = adj.csr
    slot, n_rows = core.sketch_slots(g.row_ptr, theta)
    rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, p, keys=adj.keys)
    m = 1 << p
    slot_h = slot.cpu().numpy()
    keys_h = adj.keys.cpu().numpy()
    order_h = adj.order.cpu().numpy()
    n_dict = len(forward_adj)
    # dict order: rows of the CSR are in ascending key order; order[i] is the
    # dict position of CSR row i (extra rows for non-key neighbours excluded).
    sketches: Dict[int, HLL] = {}
    by_dict = np.argsort(order_h, kind="stable")
    for i in by_dict:
        if order_h[i] >= n_dict:
            continue
        s = int(slot_h[i])
        if s >= 0:
            h = HLL._from_row(rows[s * m:(s + 1) * m], p)
            h._tchll_rows = rows
            h._tchll_slot = s
            sketches[int(keys_h[i])] = h
    return sketches, (adj, slot, rows)


def _sketch_table(sketches: Dict[int, HLL], keys_h: np.ndarray, device) -> Tuple[torch.Tensor, torch.Tensor, int]:
    """Compact (rows, slot) for the CSR whose ascending keys are keys_h.  Reuses
    the rows buffer when every sketch is a view of the same one."""
    n = len(keys_h)
    slot = np.full(n, -1, dtype=np.int64)
    if not sketches:
        return torch.zeros(16, dtype=torch.uint8, device=device), torch.from_numpy(slot).to(device), 4
    ps = {h.p for h in sketches.values()}
    if len(ps) != 1:
        raise ValueError("Both HLLs must have the same precision p")
    p = ps.pop()
    m = 1 << p
    ids = np.fromiter(sketches.keys(), dtype=np.int64, count=len(sketches))
    idx = np.searchsorted(keys_h, ids)
    ok = (idx < n) & (keys_h[np.minimum(idx, n - 1)] == ids) if n else np.zeros(len(ids), dtype=bool)
    hs = list(sketches.values())
    bufs = {id(getattr(h, "_tchll_rows", None)) for h in hs}
    shared = len(bufs) == 1 and getattr(hs[0], "_tchll_rows", None) is not None and all(
        not h._pending and not h._pending_scalars for h in hs)
    if shared:
        rows = hs[0]._tchll_rows
        for j, h in enumerate(hs):
            if ok[j]:
                slot[idx[j]] = h._tchll_slot
    else:
        rows = torch.empty(len(hs) * m, dtype=torch.uint8, device=device)
        for j, h in enumerate(hs):
            rows[j * m:(j + 1) * m].copy_(h.registers_device.to(device))
            if ok[j]:
                slot[idx[j]] = j
    return rows, torch.from_numpy(slot).to(device), p


def hybrid_triangle_count(forward_adj: Dict[int, np.ndarray], sketches: Dict[int, HLL], gamma: int,
                          r: float = 8.0, record_details: bool = False
                          ) -> Tuple[float, float, dict, Optional[List[dict]]]:
    """Selective hybrid global triangle estimate (src/hybrid.py:48-166).

    Returns ``(total_estimate, elapsed_s, stats, edge_details)``."""
    _lib.require_cuda()
    adj = core.adjacency_with_missing_nodes(forward_adj)
    g = adj.csr
    dev = g.device
    keys_h = adj.keys.cpu().numpy()
    rows, slot, p = _sketch_table(sketches, keys_h, dev)
    n_edges = g.n_edges
    res = _lib.count_result_tensor(dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _, pe = core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot,
                                              p, int(gamma), details=record_details, result=res)
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    total, rr = core.hybrid_from_result(res)
    n_approx, n_fallback, n_clamped = int(rr.n_approx), int(rr.n_fallback), int(rr.n_clamped)
    stats = {
        "n_edges": n_edges,
        "n_approx": n_approx,
        "n_exact": n_edges - n_approx,
        "n_fallback": n_fallback,
        "n_clamped": n_clamped,
        "approx_coverage": n_approx / n_edges if n_edges > 0 else 0.0,
        "fallback_ratio": n_fallback / (n_approx + n_fallback) if (n_approx + n_fallback) > 0 else 0.0,
        "clamp_ratio": n_clamped / n_approx if n_approx > 0 else 0.0,
    }
    details = None
    if record_details:
        details = _details(forward_adj, adj, [t.cpu().numpy() for t in pe])
    return total, elapsed, stats, details


def _details(forward_adj, adj: core.AdjacencyCSR, pe) -> List[dict]:
    support, s_hat, s_cl, method = pe
    keys = adj.keys.cpu().numpy()
    row_ptr = adj.csr.row_ptr.cpu().numpy().astype(np.int64)
    lens = np.diff(row_ptr)
    pos = {int(k): i for i, k in enumerate(keys)}
    out: List[dict] = []
    for u, nbrs_u in forward_adj.items():
        deg_u = len(nbrs_u)
        if deg_u == 0:
            continue
        base = int(row_ptr[pos[int(u)]])
        for k, v in enumerate(nbrs_u):
            e = base + k
            v_int = int(v)
            deg_v = int(lens[pos[v_int]])
            if method[e] == 1:
                out.append({"u": u, "v": v_int, "deg_u": deg_u, "deg_v": deg_v, "proxy": min(deg_u, deg_v),
                            "method": "hll", "s_hat": float(s_hat[e]), "s_clamped": float(s_cl[e])})
            else:
                s = float(support[e])
                out.append({"u": u, "v": v_int, "deg_u": deg_u, "deg_v": deg_v, "proxy": min(deg_u, deg_v),
                            "method": "exact", "s_hat": s, "s_clamped": s})
    return out
