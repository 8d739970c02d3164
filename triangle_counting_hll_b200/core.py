"""Tensor-level operations over libtchll: every call here launches CUDA kernels
through the C ABI (include/tchll.h).  The reference-compatible modules
(``graph``, ``gpu_graph``, ``exact``, ``hll``, ``hybrid``, ``gpu_hll``,
``gpu_hybrid``) are thin shims over these functions.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from . import _lib
from ._lib import as_device_tensor, check, load, ptr, stream_handle


@dataclass
class DeviceCSR:
    """Oriented forward CSR on one device (all int32, as the reference's
    ``to_csr_numpy`` returns, src/gpu_graph.py:6-41)."""

    row_ptr: torch.Tensor   # [n_nodes + 1]
    col_idx: torch.Tensor   # [n_edges]
    degrees: torch.Tensor   # [n_nodes] forward degree
    node_ids: torch.Tensor  # [n_nodes] original id of each compacted node
    edge_u: torch.Tensor    # [n_edges]
    edge_v: torch.Tensor    # [n_edges]

    @property
    def n_nodes(self) -> int:
        return int(self.row_ptr.numel() - 1)

    @property
    def n_edges(self) -> int:
        return int(self.col_idx.numel())

    @property
    def device(self) -> torch.device:
        return self.row_ptr.device

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in
                   (self.row_ptr, self.col_idx, self.degrees, self.node_ids, self.edge_u, self.edge_v))


def _device(device=None) -> torch.device:
    _lib.require_cuda()
    if device is None:
        return torch.device("cuda", torch.cuda.current_device())
    d = torch.device(device)
    if d.type != "cuda":
        raise ValueError("device must be a CUDA device")
    return d


def _ws(nbytes: int, device) -> torch.Tensor:
    return _lib.workspace.get(nbytes, device)


# ------------------------------------------------------------------ CSR (a1)
def csr_from_edges(raw_u, raw_v, device=None, undirected: bool = False):
    """Raw endpoint arrays -> oriented CSR (experiment/exp_gpu.py:288-365,
    src/graph.py:29-61 + src/gpu_graph.py:6-41): dedup, drop self-loops,
    compact ids, orient by (degree, id), sort rows.  With undirected=True
    returns (csr, undirected degree per node)."""
    dev = _device(device if device is not None else (raw_u.device if isinstance(raw_u, torch.Tensor) and raw_u.is_cuda else None))
    u = as_device_tensor(raw_u, torch.int32, "raw_u", dev)
    v = as_device_tensor(raw_v, torch.int32, "raw_v", dev)
    if u.numel() != v.numel():
        raise ValueError("raw_u and raw_v differ in length")
    L = load()
    n_raw = int(u.numel())
    nb = C.c_size_t(0)
    check(L.tchll_csr_workspace_bytes(n_raw, C.byref(nb)))
    with torch.cuda.device(dev):
        ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
        sizes = torch.empty(2, dtype=torch.int64, device=dev)
        st = stream_handle(dev)
        check(L.tchll_csr_build_phase1(ptr(u), ptr(v), n_raw, ptr(sizes), ptr(ws), nb.value, st), "csr phase 1")
        n_nodes, n_edges = (int(x) for x in sizes.cpu().tolist())
        if n_nodes < 0:
            raise ValueError("negative vertex id in edge list")
        row_ptr = torch.empty(n_nodes + 1, dtype=torch.int32, device=dev)
        col_idx = torch.empty(n_edges, dtype=torch.int32, device=dev)
        degrees = torch.empty(n_nodes, dtype=torch.int32, device=dev)
        node_ids = torch.empty(n_nodes, dtype=torch.int32, device=dev)
        edge_u = torch.empty(n_edges, dtype=torch.int32, device=dev)
        edge_v = torch.empty(n_edges, dtype=torch.int32, device=dev)
        und = torch.empty(n_nodes, dtype=torch.int32, device=dev) if undirected else None
        check(L.tchll_csr_build_phase2(n_raw, n_nodes, n_edges, ptr(row_ptr), ptr(col_idx), ptr(degrees),
                                       ptr(node_ids), ptr(edge_u), ptr(edge_v), ptr(und), ptr(ws), nb.value, st),
              "csr phase 2")
        del ws
    g = DeviceCSR(row_ptr, col_idx, degrees, node_ids, edge_u, edge_v)
    return (g, und) if undirected else g


@dataclass
class AdjacencyCSR:
    csr: DeviceCSR
    keys: torch.Tensor      # int64 [n] original ids in ascending order (node_ids)
    order: torch.Tensor     # int64 [n] dict position of each row
    missing: int            # neighbour values that were not keys


def flatten_adjacency(forward_adj: dict) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """dict node -> neighbour array  ->  (keys, lens, concatenated values),
    all int64, in dict iteration order (host marshalling only)."""
    n = len(forward_adj)
    keys = np.fromiter(forward_adj.keys(), dtype=np.int64, count=n)
    lens = np.fromiter((len(a) for a in forward_adj.values()), dtype=np.int64, count=n)
    if n and lens.sum() > 0:
        values = np.concatenate([np.asarray(a, dtype=np.int64).reshape(-1) for a in forward_adj.values()])
    else:
        values = np.zeros(0, dtype=np.int64)
    return keys, lens, values


def csr_from_adjacency(keys, lens, values, device=None) -> AdjacencyCSR:
    """forward_adj (flattened) -> CSR with rows in ascending key order, values
    replaced by key ranks (src/gpu_graph.py:19-37).  Values that are not keys
    get col -1 and are counted in ``missing``."""
    dev = _device(device)
    k = as_device_tensor(keys, torch.int64, "keys", dev)
    ln = as_device_tensor(lens, torch.int64, "lens", dev)
    vals = as_device_tensor(values, torch.int64, "values", dev)
    n = int(k.numel())
    nnz = int(vals.numel())
    if nnz > np.iinfo(np.int32).max:
        raise ValueError("more than 2^31-1 neighbour entries")
    L = load()
    nb = C.c_size_t(0)
    check(L.tchll_adj_workspace_bytes(n, nnz, C.byref(nb)))
    with torch.cuda.device(dev):
        ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
        node_ids = torch.empty(max(n, 1), dtype=torch.int64, device=dev)[:n]
        row_ptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
        degrees = torch.empty(n, dtype=torch.int32, device=dev)
        col_idx = torch.empty(nnz, dtype=torch.int32, device=dev)
        edge_u = torch.empty(nnz, dtype=torch.int32, device=dev)
        edge_v = torch.empty(nnz, dtype=torch.int32, device=dev)
        order = torch.empty(n, dtype=torch.int64, device=dev)
        missing = torch.zeros(1, dtype=torch.int64, device=dev)
        check(L.tchll_csr_from_adjacency(ptr(k), ptr(ln), n, ptr(vals), nnz, ptr(node_ids), ptr(row_ptr),
                                         ptr(degrees), ptr(col_idx), ptr(edge_u), ptr(edge_v), ptr(order),
                                         ptr(missing), ptr(ws), nb.value, stream_handle(dev)),
              "csr from adjacency")
        miss = int(missing.item())
    csr = DeviceCSR(row_ptr, col_idx, degrees, node_ids, edge_u, edge_v)
    return AdjacencyCSR(csr, node_ids, order, miss)


def adjacency_with_missing_nodes(forward_adj: dict, device=None) -> AdjacencyCSR:
    """csr_from_adjacency, adding an empty row for every neighbour id that is
    not a key (the reference treats such a v as having no forward list,
    src/exact.py:83-85, src/hybrid.py:103)."""
    keys, lens, values = flatten_adjacency(forward_adj)
    adj = csr_from_adjacency(keys, lens, values, device)
    if adj.missing:
        extra = np.setdiff1d(np.unique(values), keys)
        keys2 = np.concatenate([keys, extra])
        lens2 = np.concatenate([lens, np.zeros(len(extra), dtype=np.int64)])
        adj = csr_from_adjacency(keys2, lens2, values, device)
        assert adj.missing == 0
    return adj


# ------------------------------------------------------------- counting (a3)
def _count_ws(n_nodes: int, n_edges: int, device) -> torch.Tensor:
    nb = C.c_size_t(0)
    check(load().tchll_count_workspace_bytes(int(n_nodes), int(n_edges), C.byref(nb)))
    return _ws(nb.value, device)


def _hybrid_ws(n_nodes: int, n_edges: int, n_rows: int, p: int, device) -> torch.Tensor:
    nb = C.c_size_t(0)
    check(load().tchll_hybrid_workspace_bytes(int(n_nodes), int(n_edges), int(n_rows), int(p), C.byref(nb)))
    return _ws(nb.value, device)


def exact_count_tensors(row_ptr: torch.Tensor, col_idx: torch.Tensor, edge_u: torch.Tensor,
                        edge_v: torch.Tensor, per_edge: bool = False,
                        result: Optional[torch.Tensor] = None) -> Tuple[torch.Tensor, Optional[torch.Tensor]]:
    """Launch the exact count; returns (device result block, per-edge supports
    or None).  Stream-ordered: nothing is synchronised."""
    dev = row_ptr.device
    n_nodes = int(row_ptr.numel()) - 1
    n_edges = int(edge_u.numel())
    if int(edge_v.numel()) != n_edges:
        raise ValueError("edge_u and edge_v differ in length")
    res = result if result is not None else _lib.count_result_tensor(dev)
    pe = torch.empty(n_edges, dtype=torch.int64, device=dev) if per_edge else None
    ws = _count_ws(n_nodes, n_edges, dev)
    check(load().tchll_exact_count(ptr(row_ptr), n_nodes, ptr(col_idx), int(col_idx.numel()), ptr(edge_u),
                                   ptr(edge_v), n_edges, ptr(pe), ptr(res), ptr(ws), ws.numel(),
                                   stream_handle(dev)), "exact count")
    return res, pe


_COPY_STREAMS: Dict[int, torch.cuda.Stream] = {}


def _copy_stream(dev: torch.device) -> torch.cuda.Stream:
    i = dev.index if dev.index is not None else torch.cuda.current_device()
    if i not in _COPY_STREAMS:
        _COPY_STREAMS[i] = torch.cuda.Stream(device=i)
    return _COPY_STREAMS[i]


def exact_count_host(row_ptr: torch.Tensor, col_idx: torch.Tensor, edge_u: torch.Tensor, edge_v: torch.Tensor,
                     device=None, result: Optional[torch.Tensor] = None) -> torch.Tensor:
    """Exact count of a CSR held in host memory (pinned for asynchronous
    copies).  The arrays are copied on a copy stream in the order row_ptr,
    edge_u, edge_v, col_idx, and the count (tchll_exact_count_staged) starts
    once the first three have arrived: the pair regrouping, which reads only
    those, runs while col_idx is still crossing the host link.  Returns the
    device result block; stream-ordered on the current stream."""
    dev = _device(device)
    cs = _copy_stream(dev)
    cur = torch.cuda.current_stream(dev)
    cs.wait_stream(cur)  # the copies may overwrite nothing the caller still uses
    with torch.cuda.stream(cs):
        d = [t.to(device=dev, dtype=torch.int32, non_blocking=True).contiguous()
             for t in (row_ptr, edge_u, edge_v)]
        head = torch.cuda.Event()
        head.record(cs)
        ci = col_idx.to(device=dev, dtype=torch.int32, non_blocking=True).contiguous()
        col_ready = torch.cuda.Event()
        col_ready.record(cs)
    for t in (*d, ci):  # allocated on the copy stream, used on the current one
        t.record_stream(cur)
    cur.wait_event(head)
    rp, eu, ev = d
    n_nodes = int(rp.numel()) - 1
    n_edges = int(eu.numel())
    if int(ev.numel()) != n_edges:
        raise ValueError("edge_u and edge_v differ in length")
    res = result if result is not None else _lib.count_result_tensor(dev)
    ws = _count_ws(n_nodes, n_edges, dev)
    check(load().tchll_exact_count_staged(ptr(rp), n_nodes, ptr(ci), int(ci.numel()), ptr(eu), ptr(ev), n_edges,
                                          ptr(res), ptr(ws), ws.numel(), col_ready.cuda_event,
                                          stream_handle(dev)), "exact count")
    cur.wait_event(col_ready)  # col_idx is in use until the count ends
    return res


def hybrid_count_dense_tensors(row_ptr, col_idx, edge_u, edge_v, degrees, sketch_regs, has_sketch, gamma: int,
                               p: int, split_kernels: bool = True,
                               result: Optional[torch.Tensor] = None) -> torch.Tensor:
    dev = row_ptr.device
    n_nodes = int(row_ptr.numel()) - 1
    n_edges = int(edge_u.numel())
    m = 1 << int(p) if 4 <= int(p) <= 16 else 0
    if m and int(sketch_regs.numel()) < n_nodes * m:
        raise ValueError(f"sketch_regs holds {int(sketch_regs.numel())} bytes, need n_nodes * 2^p = {n_nodes * m}")
    if int(has_sketch.numel()) < n_nodes or int(degrees.numel()) < n_nodes:
        raise ValueError("has_sketch / degrees shorter than n_nodes")
    res = result if result is not None else _lib.count_result_tensor(dev)
    ws = _hybrid_ws(n_nodes, n_edges, n_nodes, p, dev) if m else _count_ws(n_nodes, n_edges, dev)
    check(load().tchll_hybrid_count_dense(ptr(row_ptr), n_nodes, ptr(col_idx), int(col_idx.numel()),
                                          ptr(edge_u), ptr(edge_v), n_edges, ptr(degrees), ptr(sketch_regs),
                                          ptr(has_sketch), int(p), int(gamma), 1 if split_kernels else 0,
                                          ptr(res), ptr(ws), ws.numel(), stream_handle(dev)), "hybrid count")
    return res


def hybrid_count_compact_tensors(row_ptr, col_idx, edge_u, edge_v, degrees, rows, slot, p: int, gamma: int,
                                 split_kernels: bool = False, details: bool = False,
                                 result: Optional[torch.Tensor] = None):
    """Returns (result block, (support, s_hat, s_clamped, method) or None)."""
    dev = row_ptr.device
    n_nodes = int(row_ptr.numel()) - 1
    n_edges = int(edge_u.numel())
    m = 1 << int(p) if 4 <= int(p) <= 16 else 1
    n_rows = int(rows.numel()) // m
    res = result if result is not None else _lib.count_result_tensor(dev)
    pe = None
    if details:
        pe = (torch.empty(n_edges, dtype=torch.int64, device=dev),
              torch.empty(n_edges, dtype=torch.float64, device=dev),
              torch.empty(n_edges, dtype=torch.float64, device=dev),
              torch.empty(n_edges, dtype=torch.uint8, device=dev))
    ws = _hybrid_ws(n_nodes, n_edges, n_rows, p, dev) if 4 <= int(p) <= 16 else _count_ws(n_nodes, n_edges, dev)
    pp = [ptr(t) for t in pe] if pe else [None, None, None, None]
    check(load().tchll_hybrid_count_compact(ptr(row_ptr), n_nodes, ptr(col_idx), int(col_idx.numel()),
                                            ptr(edge_u), ptr(edge_v), n_edges, ptr(degrees), ptr(rows), n_rows,
                                            ptr(slot), int(p), int(gamma), 1 if split_kernels else 0, *pp,
                                            ptr(res), ptr(ws), ws.numel(), stream_handle(dev)),
          "hybrid count")
    return res, pe


def set_count_tuning(chunk: int = 256, slots_log2: int = 10, tiny: int = 16, blocks_per_sm: int = 0,
                     warps: Optional[int] = None, pairs: Optional[bool] = None,
                     sparse: Optional[bool] = None, hub: Optional[int] = None, hub_seg: Optional[int] = None,
                     hub_lg: Optional[int] = None, hub_unroll: Optional[int] = None,
                     bitmap_lg: Optional[int] = None, overlap: Optional[int] = None,
                     packed: Optional[bool] = None, bank_sort: Optional[bool] = None,
                     hll_row_cache_p: Optional[int] = None, hll_lanes: Optional[int] = None) -> None:
    """Launch shape of the counting kernels (results do not depend on it).
    hub / hub_seg / hub_lg / hub_unroll: threshold on d+(x) above which a pair
    goes to the CTA-shared table kernels (0: off), pairs per work unit, log2
    hash-table slots, probe loads in flight per lane.  bitmap_lg: log2 bytes
    of the 32-bit hub bitmap buffer (0: off); overlap: 0 one stream, 1 the
    hub core pass (and a hybrid's HLL pass) on a second stream beside the
    exact pairs, 2 also the short-list pair kernel there, beside the hub
    kernel; packed: 16-bit hub probe lists when
    the core has at most 131,070 vertices; bank_sort: packed lists ordered by
    bitmap bank.  hll_row_cache_p / hll_lanes:
    the HLL pass's one-pass threshold on p and lanes per edge (0: by p)."""
    L = load()
    cur = get_count_tuning()
    check(L.tchll_set_hll_pass(int(cur["hll_row_cache_p"] if hll_row_cache_p is None else hll_row_cache_p),
                               int(cur["hll_lanes"] if hll_lanes is None else hll_lanes)))
    check(L.tchll_set_count_core(int(cur["bitmap_lg"] if bitmap_lg is None else bitmap_lg),
                                 int(cur["overlap"] if overlap is None else int(overlap)),
                                 int(cur["packed"] if packed is None else bool(packed)),
                                 int(cur["bank_sort"] if bank_sort is None else bool(bank_sort))))
    check(L.tchll_set_count_hub(int(cur["hub"] if hub is None else hub),
                                int(cur["hub_seg"] if hub_seg is None else hub_seg),
                                int(cur["hub_lg"] if hub_lg is None else hub_lg),
                                int(cur["hub_unroll"] if hub_unroll is None else hub_unroll)))
    check(L.tchll_set_count_table(int(cur["sparse"] if sparse is None else bool(sparse))))
    w = cur["warps"] if warps is None else int(warps)
    pr = cur["pairs"] if pairs is None else int(bool(pairs))
    # one warp fits every table size, so go through it to reach any valid shape
    check(L.tchll_set_count_shape(1, pr))
    check(L.tchll_set_count_tuning(int(chunk), int(slots_log2), int(tiny), int(blocks_per_sm)))
    check(L.tchll_set_count_shape(w, pr))


def get_count_tuning() -> dict:
    out = (C.c_int32 * 8)()
    check(load().tchll_get_count_tuning(C.cast(out, C.c_void_p)))
    hub = (C.c_int32 * 4)()
    check(load().tchll_get_count_hub(C.cast(hub, C.c_void_p)))
    co = (C.c_int32 * 4)()
    check(load().tchll_get_count_core(C.cast(co, C.c_void_p)))
    hp = (C.c_int32 * 2)()
    check(load().tchll_get_hll_pass(C.cast(hp, C.c_void_p)))
    return {"chunk": out[0], "slots_log2": out[1], "tiny": out[2], "blocks_per_sm": out[3], "warps": out[4],
            "pairs": out[5], "sparse": out[6], "hub": hub[0], "hub_seg": hub[1], "hub_lg": hub[2],
            "hub_unroll": hub[3], "bitmap_lg": co[0], "overlap": co[1], "packed": co[2], "bank_sort": co[3],
            "hll_row_cache_p": hp[0],
            "hll_lanes": hp[1]}


def set_phase_timing(enable: bool) -> None:
    check(load().tchll_set_phase_timing(1 if enable else 0))


def phase_times() -> dict:
    """Milliseconds of the last counting call's phases (needs
    set_phase_timing(True) before the call); None for phases not run."""
    out = (C.c_float * 3)()
    check(load().tchll_phase_times(C.cast(out, C.c_void_p)))
    names = ("pairs", "count", "hll")
    res = {n: (float(v) if v >= 0 else None) for n, v in zip(names, out)}
    hub = (C.c_float * 2)()
    check(load().tchll_phase_hub_ms(C.cast(hub, C.c_void_p)))
    res["hub"] = float(hub[0]) if hub[0] >= 0 else None        # hub kernels, part of "count"
    res["hub_core"] = float(hub[1]) if hub[1] >= 0 else None   # core pass before them, part of "count"
    return res


# ----------------------------------------------------------- sketches (a4)
def build_sketches_dense_tensors(row_ptr, col_idx, n_nodes: int, theta: int, p: int, sketch_regs,
                                 has_sketch) -> None:
    dev = row_ptr.device
    check(load().tchll_build_sketches_dense(ptr(row_ptr), int(n_nodes), ptr(col_idx), int(col_idx.numel()),
                                            int(theta), int(p), ptr(sketch_regs), ptr(has_sketch),
                                            stream_handle(dev)), "build sketches")


def sketch_slots(row_ptr: torch.Tensor, theta: int) -> Tuple[torch.Tensor, int]:
    """slot[u] = rank among rows of length >= theta, else -1; returns (slot, n)."""
    dev = row_ptr.device
    n = int(row_ptr.numel()) - 1
    nb = C.c_size_t(0)
    L = load()
    check(L.tchll_sketch_workspace_bytes(n, C.byref(nb)))
    ws = _ws(nb.value, dev)
    slot = torch.empty(n, dtype=torch.int64, device=dev)
    ns = torch.empty(1, dtype=torch.int64, device=dev)
    check(L.tchll_sketch_slots(ptr(row_ptr), n, int(theta), ptr(slot), ptr(ns), ptr(ws), ws.numel(),
                               stream_handle(dev)), "sketch slots")
    return slot, int(ns.item())


def build_sketches_compact_tensors(row_ptr, col_idx, slot, n_rows: int, p: int,
                                   keys: Optional[torch.Tensor] = None) -> torch.Tensor:
    """rows[n_rows, 2^p] for every u with slot[u] >= 0, hashing keys[col] (a
    per-node int64 table, e.g. original ids) when given, else the col values."""
    dev = row_ptr.device
    m = 1 << int(p)
    rows = torch.empty(max(n_rows, 1) * m, dtype=torch.uint8, device=dev)
    check(load().tchll_build_sketches_compact(ptr(row_ptr), int(row_ptr.numel()) - 1, ptr(col_idx), ptr(keys),
                                              int(col_idx.numel()), ptr(slot), int(n_rows), int(p), ptr(rows),
                                              stream_handle(dev)), "build sketches")
    return rows[: n_rows * m]


def hll_add_tensor(regs: torch.Tensor, p: int, values) -> None:
    dev = regs.device
    vals = as_device_tensor(values, torch.int64, "values", dev)
    check(load().tchll_hll_add(ptr(regs), int(p), ptr(vals), int(vals.numel()), stream_handle(dev)), "hll add")


def estimate_pairs(rows: torch.Tensor, p: int, a, b=None) -> torch.Tensor:
    """FP64 estimates (device tensor) of union(rows[a[i]], rows[b[i]]) or of
    rows[a[i]] alone."""
    dev = rows.device
    m = 1 << int(p)
    ta = as_device_tensor(a, torch.int64, "a", dev)
    tb = as_device_tensor(b, torch.int64, "b", dev) if b is not None else None
    out = torch.empty(int(ta.numel()), dtype=torch.float64, device=dev)
    check(load().tchll_hll_estimate_pairs(ptr(rows), int(rows.numel()) // m, int(p), ptr(ta), ptr(tb),
                                          int(ta.numel()), ptr(out), stream_handle(dev)), "hll estimate")
    return out


def hash64(values, device=None) -> torch.Tensor:
    dev = _device(device)
    v = as_device_tensor(values, torch.int64, "values", dev)
    out = torch.empty(int(v.numel()), dtype=torch.uint64, device=dev)
    check(load().tchll_hash64(ptr(v), int(v.numel()), ptr(out), stream_handle(dev)), "hash64")
    return out


# ---------------------------------------------------------- result reading
def exact_from_result(res_t: torch.Tensor) -> int:
    r = _lib.read_count_result(res_t)
    _lib.raise_on_status(r)
    return int(r.exact)


def hybrid_from_result(res_t: torch.Tensor) -> Tuple[float, _lib.CountResult]:
    """(total, raw result): total = exact part + HLL fixed-point part, rounded
    once to FP64."""
    r = _lib.read_count_result(res_t)
    _lib.raise_on_status(r)
    fx = (int(r.hll_fx_hi) << 64) | int(r.hll_fx_lo)
    total = ((int(r.exact) << 32) + fx) / 4294967296
    return float(total), r


# ------------------------------------------------------------- generators
def prob_threshold(p: float) -> int:
    return min(int(math.floor(p * 4294967296.0)), 0xFFFFFFFF)


def gen_rmat(scale: int, edge_factor: int = 16, a: float = 0.57, b: float = 0.19, c: float = 0.19,
             seed: int = 1, device=None) -> Tuple[torch.Tensor, torch.Tensor]:
    dev = _device(device)
    n_raw = int(edge_factor) << int(scale)
    u = torch.empty(n_raw, dtype=torch.int32, device=dev)
    v = torch.empty(n_raw, dtype=torch.int32, device=dev)
    check(load().tchll_gen_rmat(int(scale), n_raw, prob_threshold(a), prob_threshold(a + b),
                                prob_threshold(a + b + c), int(seed), ptr(u), ptr(v), stream_handle(dev)), "rmat")
    return u, v


def gen_er(n: int, n_raw: int, seed: int = 0, device=None):
    dev = _device(device)
    u = torch.empty(int(n_raw), dtype=torch.int32, device=dev)
    v = torch.empty(int(n_raw), dtype=torch.int32, device=dev)
    check(load().tchll_gen_er(int(n), int(n_raw), int(seed), ptr(u), ptr(v), stream_handle(dev)), "er")
    return u, v


def gen_lattice(rows: int, cols: int, p_diag: float = 0.3, p_del: float = 0.05, seed: int = 0, device=None):
    dev = _device(device)
    L = load()
    total = int(L.tchll_gen_lattice_count(int(rows), int(cols)))
    u = torch.empty(total, dtype=torch.int32, device=dev)
    v = torch.empty(total, dtype=torch.int32, device=dev)
    check(L.tchll_gen_lattice(int(rows), int(cols), prob_threshold(p_diag), prob_threshold(p_del), int(seed),
                              ptr(u), ptr(v), stream_handle(dev)), "lattice")
    return u, v


def chung_lu_table(n: int, beta: float) -> np.ndarray:
    """Cumulative integer weights: w_i = (i+1)^(-1/(beta-1)) scaled by 2^24,
    rounded, at least 1 (host; the table is an input of the generator)."""
    i = np.arange(1, n + 1, dtype=np.float64)
    w = np.maximum(np.rint(np.power(i, -1.0 / (beta - 1.0)) * 16777216.0), 1.0).astype(np.uint64)
    return np.cumsum(w, dtype=np.uint64)


def gen_chung_lu(n: int, avg_degree: float, beta: float, seed: int, device=None, cum: Optional[np.ndarray] = None):
    dev = _device(device)
    if cum is None:
        cum = chung_lu_table(n, beta)
    cum_t = torch.from_numpy(cum.view(np.int64)).to(dev)
    n_raw = int(round(n * avg_degree / 2.0))
    u = torch.empty(n_raw, dtype=torch.int32, device=dev)
    v = torch.empty(n_raw, dtype=torch.int32, device=dev)
    check(load().tchll_gen_chung_lu(ptr(cum_t), int(n), n_raw, int(seed), ptr(u), ptr(v), stream_handle(dev)),
          "chung-lu")
    return u, v
