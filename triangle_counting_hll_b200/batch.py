"""Batched counting: many graphs in one persistent launch.

The reference counts one graph per call (src/gpu_hybrid.py:332-431).  Here a
batch of graphs shares one concatenated CSR: each graph's raw ids are shifted
by the running sum of the previous graphs' id spaces, one device CSR build
dedups, compacts and orients everything (orientation and compaction are per
vertex, so every graph's part equals its own CSR shifted by ``vbase[g]``),
and ``tchll_batch_exact_count`` / ``tchll_batch_hybrid_count`` walk a device
chunk list whose chunks never cross a graph, adding integer totals into one
result block per graph.  Per-graph results are therefore bit-identical to
counting each graph alone (checked in tests/test_batch_serve.py).

Batched sketches hash each vertex's id within its own graph
(``tchll_batch_local_ids``), so HLL registers, and with them the hybrid
estimates, equal the one-graph-at-a-time ones exactly.

``CapturedBatch`` records the whole batched launch sequence in a CUDA graph
and replays it for repeat queries on resident graphs.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, autotune, core
from ._lib import check, load, ptr, stream_handle

# --------------------------------------------------------------- workloads


@dataclass
class GraphSpec:
    kind: str        # "er" or "chung_lu"
    n: int           # vertex id space
    seed: int


def c4_specs(n_graphs: int = 2048, median: float = 5000.0, sigma: float = 1.0, lo: int = 500, hi: int = 500000,
             seed_base: int = 0) -> List[GraphSpec]:
    """The batched workload: vertex counts lognormal(median, sigma) clipped to
    [lo, hi]; even graphs Erdos-Renyi, odd graphs Chung-Lu (exponent 2.1),
    both with average degree 12; graph i uses seed seed_base + i."""
    rng = np.random.default_rng(seed_base)
    ns = np.clip(np.round(rng.lognormal(math.log(median), sigma, n_graphs)), lo, hi).astype(np.int64)
    return [GraphSpec("er" if i % 2 == 0 else "chung_lu", int(ns[i]), seed_base + i) for i in range(n_graphs)]


def generate(spec: GraphSpec, device=None, avg_degree: float = 12.0, beta: float = 2.1):
    """Raw endpoint arrays (device int32) of one workload graph."""
    if spec.kind == "er":
        return core.gen_er(spec.n, int(round(spec.n * avg_degree / 2.0)), seed=spec.seed, device=device)
    if spec.kind == "chung_lu":
        return core.gen_chung_lu(spec.n, avg_degree, beta, seed=spec.seed, device=device)
    raise ValueError(f"unknown graph kind {spec.kind}")


# ------------------------------------------------------------------ batch


class GraphBatch:
    """Concatenated oriented CSR of several graphs plus their vertex ranges."""

    def __init__(self, csr: core.DeviceCSR, vbase: torch.Tensor, id_base: np.ndarray):
        self.csr = csr
        self.vbase = vbase          # int32 [n_graphs + 1], compacted vertex ranges
        self.id_base = id_base      # int64 [n_graphs + 1], raw id offsets used
        self._ws: Optional[torch.Tensor] = None
        self._local: Optional[torch.Tensor] = None

    @property
    def n_graphs(self) -> int:
        return int(self.vbase.numel()) - 1

    @classmethod
    def from_edge_lists(cls, graphs: Sequence[Tuple[torch.Tensor, torch.Tensor, int]], device=None) -> "GraphBatch":
        """graphs: (raw_u, raw_v, id_space) per graph; ids of graph g must lie
        in [0, id_space)."""
        dev = core._device(device)
        sizes = [int(n) for _, _, n in graphs]
        id_base = np.zeros(len(graphs) + 1, dtype=np.int64)
        id_base[1:] = np.cumsum(sizes)
        if id_base[-1] > np.iinfo(np.int32).max:
            raise ValueError("batch id space exceeds int32")
        us, vs = [], []
        for (u, v, _), b in zip(graphs, id_base[:-1]):
            u = _lib.as_device_tensor(u, torch.int32, "u", dev)
            v = _lib.as_device_tensor(v, torch.int32, "v", dev)
            us.append(u + int(b))
            vs.append(v + int(b))
        u = torch.cat(us) if us else torch.zeros(0, dtype=torch.int32, device=dev)
        v = torch.cat(vs) if vs else torch.zeros(0, dtype=torch.int32, device=dev)
        csr = core.csr_from_edges(u, v, device=dev)
        base_t = torch.from_numpy(id_base).to(dev)
        # first compacted vertex of each graph: rank of its first raw id
        vbase = torch.searchsorted(csr.node_ids.to(torch.int64), base_t).to(torch.int32)
        return cls(csr, vbase.contiguous(), id_base)

    def _workspace(self) -> torch.Tensor:
        g = self.csr
        nb = C.c_size_t(0)
        check(load().tchll_batch_workspace_bytes(g.n_nodes, g.n_edges, self.n_graphs, C.byref(nb)))
        if self._ws is None or self._ws.numel() < nb.value:
            self._ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=g.device)
        return self._ws

    def local_ids(self) -> torch.Tensor:
        """Per-vertex id within its own graph (int64)."""
        if self._local is None:
            g = self.csr
            out = torch.empty(g.n_nodes, dtype=torch.int64, device=g.device)
            check(load().tchll_batch_local_ids(ptr(self.vbase), self.n_graphs, g.n_nodes, ptr(out),
                                               stream_handle(g.device)), "local ids")
            self._local = out
        return self._local

    def exact_launch(self, results: torch.Tensor) -> None:
        """Stream-ordered batched exact count into results (n_graphs x 64 B)."""
        g = self.csr
        ws = self._workspace()
        check(load().tchll_batch_exact_count(ptr(g.row_ptr), g.n_nodes, ptr(g.col_idx), g.n_edges, ptr(g.edge_u),
                                             ptr(g.edge_v), g.n_edges, ptr(self.vbase), self.n_graphs, ptr(results),
                                             ptr(ws), ws.numel(), stream_handle(g.device)), "batch exact count")

    def exact_counts(self) -> np.ndarray:
        res = torch.empty(max(self.n_graphs, 1) * _lib.RESULT_BYTES, dtype=torch.uint8, device=self.csr.device)
        self.exact_launch(res)
        return exact_from_results(res, self.n_graphs)

    def sketches(self, theta: int, p: int) -> Tuple[torch.Tensor, torch.Tensor]:
        g = self.csr
        slot, n_rows = core.sketch_slots(g.row_ptr, theta)
        rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, p, keys=self.local_ids())
        return rows, slot

    def hybrid_launch(self, results: torch.Tensor, rows: torch.Tensor, slot: torch.Tensor, p: int,
                      gamma: int) -> None:
        g = self.csr
        ws = self._workspace()
        m = 1 << p
        check(load().tchll_batch_hybrid_count(ptr(g.row_ptr), g.n_nodes, ptr(g.col_idx), g.n_edges,
                                              ptr(g.edge_u), ptr(g.edge_v), g.n_edges, ptr(g.degrees), ptr(rows),
                                              int(rows.numel()) // m, ptr(slot), int(p), int(gamma),
                                              ptr(self.vbase), self.n_graphs, ptr(results), ptr(ws), ws.numel(),
                                              stream_handle(g.device)), "batch hybrid count")

    def hybrid_counts(self, theta: int, gamma: int, p: int):
        rows, slot = self.sketches(theta, p)
        res = torch.empty(max(self.n_graphs, 1) * _lib.RESULT_BYTES, dtype=torch.uint8, device=self.csr.device)
        self.hybrid_launch(res, rows, slot, p, gamma)
        return hybrid_from_results(res, self.n_graphs)


def _results(res: torch.Tensor, n: int) -> np.ndarray:
    raw = res[: n * _lib.RESULT_BYTES].cpu().numpy()
    dt = np.dtype([("exact", "<u8"), ("lo", "<u8"), ("hi", "<u8"), ("n_approx", "<i8"), ("n_exact", "<i8"),
                   ("n_fallback", "<i8"), ("n_clamped", "<i8"), ("status", "<u4"), ("reserved", "<u4")])
    return raw.view(dt)


def exact_from_results(res: torch.Tensor, n: int) -> np.ndarray:
    r = _results(res, n)
    if (r["status"] != 0).any():
        raise ValueError(f"malformed input in {(r['status'] != 0).sum()} graph(s) of the batch")
    return r["exact"].astype(np.int64)


def hybrid_from_results(res: torch.Tensor, n: int):
    """(totals float64[n], stats dict of int64 arrays); totals are the exact
    part plus the 2^-32 fixed-point HLL part, each rounded once."""
    r = _results(res, n)
    if (r["status"] != 0).any():
        raise ValueError(f"malformed input in {(r['status'] != 0).sum()} graph(s) of the batch")
    totals = np.array([((int(e) << 32) + ((int(h) << 64) | int(lo))) / 4294967296
                       for e, lo, h in zip(r["exact"], r["lo"], r["hi"])], dtype=np.float64)
    stats = {k: r[k].astype(np.int64) for k in ("n_approx", "n_exact", "n_fallback", "n_clamped")}
    return totals, stats


# ------------------------------------------------------------ CUDA graphs


class CapturedBatch:
    """A batched exact (or hybrid) count recorded once as a CUDA graph and
    replayed for repeat queries; the batch, workspace and sketches stay
    resident, so a replay is one graph launch plus the 64 B/graph read."""

    def __init__(self, batch: GraphBatch, hybrid: Optional[Tuple[int, int, int]] = None):
        self.batch = batch
        dev = batch.csr.device
        self.results = torch.empty(max(batch.n_graphs, 1) * _lib.RESULT_BYTES, dtype=torch.uint8, device=dev)
        self.hybrid = hybrid
        if hybrid is not None:
            theta, gamma, p = hybrid
            self.rows, self.slot = batch.sketches(theta, p)
        batch._workspace()
        self._launch()  # warm up outside capture (kernel attributes, caches)
        torch.cuda.synchronize(dev)
        self.stream = torch.cuda.Stream(device=dev)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph, stream=self.stream):
            self._launch()

    def _launch(self) -> None:
        if self.hybrid is None:
            self.batch.exact_launch(self.results)
        else:
            _, gamma, p = self.hybrid
            self.batch.hybrid_launch(self.results, self.rows, self.slot, p, gamma)

    def replay(self) -> None:
        self.graph.replay()

    def exact_counts(self) -> np.ndarray:
        self.replay()
        return exact_from_results(self.results, self.batch.n_graphs)

    def hybrid_counts(self):
        self.replay()
        return hybrid_from_results(self.results, self.batch.n_graphs)


# ------------------------------------------------- one graph at a time


def plain_exact_counts(csrs: Sequence[core.DeviceCSR]) -> np.ndarray:
    """One launch sequence and one result read per graph (the reference's
    calling pattern, src/gpu_hybrid.py:332-354)."""
    out = np.zeros(len(csrs), dtype=np.int64)
    for i, g in enumerate(csrs):
        res, _ = core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v)
        out[i] = core.exact_from_result(res)
    return out


def plain_sketches(csrs: Sequence[core.DeviceCSR], theta: int, p: int):
    """Per-graph compact sketches (each graph hashes its own compacted ids)."""
    out = []
    for g in csrs:
        slot, n_rows = core.sketch_slots(g.row_ptr, theta)
        out.append((core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, p), slot))
    return out


def plain_hybrid_counts(csrs: Sequence[core.DeviceCSR], sketches, gamma: int, p: int):
    totals = np.zeros(len(csrs), dtype=np.float64)
    stats = {k: np.zeros(len(csrs), dtype=np.int64) for k in ("n_approx", "n_exact", "n_fallback", "n_clamped")}
    for i, (g, (rows, slot)) in enumerate(zip(csrs, sketches)):
        res, _ = core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot,
                                                   p, gamma, split_kernels=True)
        t, r = core.hybrid_from_result(res)
        totals[i] = t
        for k in stats:
            stats[k][i] = int(getattr(r, k))
    return totals, stats


# ------------------------------------------------------------- benchmark


def bench_entry(dev, quick: bool = True, n_graphs: int = 2048, theta: int = 64, p: int = 10) -> Dict:
    """Graphs/s of the batched workload (2,048 graphs, lognormal sizes, half
    Erdos-Renyi / half Chung-Lu, average degree 12; hybrid p=10, theta=gamma=64),
    batched (one CUDA-graph replay) versus one graph per call, with the
    per-graph results checked bit-exact between the two."""
    specs = c4_specs(n_graphs)
    raw = [generate(s, dev) for s in specs]
    batch = GraphBatch.from_edge_lists([(u, v, s.n) for (u, v), s in zip(raw, specs)], device=dev)
    csrs = [core.csr_from_edges(u, v, device=dev) for u, v in raw]
    del raw
    out: Dict = {"n_graphs": n_graphs, "n_edges": batch.csr.n_edges, "theta": theta, "gamma": theta, "p": p,
                 "sizes": "lognormal median 5000 sigma 1.0 clipped [500, 500000]; even ER, odd Chung-Lu 2.1; deg 12"}
    reps = 3 if quick else 10
    base = core.get_count_tuning()
    try:
        return _bench_modes(dev, batch, csrs, out, reps, theta, p)
    finally:  # the tuning is process-wide: leave it as it was
        core.set_count_tuning(**base)


def _bench_modes(dev, batch, csrs, out: Dict, reps: int, theta: int, p: int) -> Dict:
    n_graphs = batch.n_graphs
    tuned = autotune.tune_batch(batch)
    out["tuning"] = tuned
    plain_sk = plain_sketches(csrs, theta, p)
    for mode in ("exact", "hybrid"):
        cap = CapturedBatch(batch, None if mode == "exact" else (theta, theta, p))
        cap.replay()
        torch.cuda.synchronize(dev)
        s = torch.cuda.Event(enable_timing=True)
        e = torch.cuda.Event(enable_timing=True)
        s.record()
        for _ in range(reps):
            got = cap.exact_counts() if mode == "exact" else cap.hybrid_counts()
        e.record()
        torch.cuda.synchronize(dev)
        ms_b = s.elapsed_time(e) / reps
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ref = plain_exact_counts(csrs) if mode == "exact" else plain_hybrid_counts(csrs, plain_sk, theta, p)
        torch.cuda.synchronize(dev)
        ms_p = (time.perf_counter() - t0) * 1e3
        if mode == "exact":
            same = bool(np.array_equal(got, ref))
        else:
            same = bool(np.array_equal(got[0], ref[0])) and all(np.array_equal(got[1][k], ref[1][k])
                                                                  for k in got[1])
        out[mode] = {"batched_ms": ms_b, "batched_graphs_per_s": n_graphs / (ms_b / 1e3),
                     "plain_ms": ms_p, "plain_graphs_per_s": n_graphs / (ms_p / 1e3),
                     "speedup": ms_p / ms_b, "bit_exact_vs_plain": same}
        del cap
    return out
