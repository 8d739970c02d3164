"""Continuous-batching serving loop for triangle-count queries.

The reference answers one query per call, synchronously (src/gpu_hybrid.py:
332-431).  ``Server`` runs a request loop on one GPU:

* requests arrive in real time (Poisson arrivals in the benchmark); each asks
  for the exact count or the hybrid estimate (p, theta, gamma) of a graph;
* admission is by device bytes: a request is admitted when its graph's CSR
  (and, for hybrid queries, its sketches) fit the budget next to what is
  resident; least-recently-used resident graphs are evicted to make room, and
  a request that could never fit is completed with an error;
* graphs stay resident after their query, so repeat queries skip the build;
* every tick, the newly admitted graphs are built together (one concatenated
  device CSR build, split into per-graph residents) on a build stream while
  the previous tick's counts run on a count stream, so arrivals overlap with
  work already on the device; then all admitted queries of the tick are
  folded into one batched count launch per mode (exact, hybrid), whose
  per-graph results are bit-identical to answering each query alone;
* latency is completion time minus arrival time; the report gives p50 / p99
  and graphs/s next to the same requests served one at a time.
"""
from __future__ import annotations

import collections
import math
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib, batch as B, core

RMAT_ABC = (0.57, 0.19, 0.19)


@dataclass
class Request:
    rid: int
    arrival: float          # seconds after the start of the run
    scale: int
    edge_factor: int
    seed: int
    mode: str               # "exact" or "hybrid"
    p: int = 12
    theta: int = 128
    gamma: int = 128

    @property
    def key(self) -> Tuple[int, int, int]:
        return (self.scale, self.edge_factor, self.seed)

    def raw_edges(self) -> int:
        return self.edge_factor << self.scale


@dataclass
class Completion:
    rid: int
    mode: str
    value: Optional[float]           # exact count (int) or hybrid estimate
    stats: Optional[Dict] = None
    latency: float = float("nan")
    error: Optional[str] = None


def c5_requests(n: int, rate_per_s: float, seed: int = 0, scale_range=(12, 20), ef_range=(8, 32),
                hybrid_frac: float = 0.5, repeat_frac: float = 0.0, p: int = 12, theta: int = 128) -> List[Request]:
    """Serving workload: Poisson arrivals at rate_per_s; R-MAT graphs with
    scale ~ U[scale_range] and edge factor ~ U[ef_range] (integers), the
    (0.57, 0.19, 0.19, 0.05) quadrant split; half exact-only, half hybrid
    (p, theta = gamma); repeat_frac of the requests re-ask an earlier graph."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate_per_s, n))
    out: List[Request] = []
    for i in range(n):
        if out and rng.random() < repeat_frac:
            prev = out[int(rng.integers(0, len(out)))]
            sc, ef, sd = prev.scale, prev.edge_factor, prev.seed
        else:
            sc = int(rng.integers(scale_range[0], scale_range[1] + 1))
            ef = int(rng.integers(ef_range[0], ef_range[1] + 1))
            sd = seed * 1000003 + i
        mode = "hybrid" if rng.random() < hybrid_frac else "exact"
        out.append(Request(i, float(t[i]), sc, ef, sd, mode, p, theta, theta))
    return out


def generate_edges(req: Request, device):
    return core.gen_rmat(req.scale, req.edge_factor, *RMAT_ABC, seed=req.seed, device=device)


def estimate_bytes(req: Request) -> int:
    """Admission estimate before the build: raw edges (8 B), CSR with edge
    arrays (16 B / edge), pair workspace (8 B / edge) and, for hybrid
    queries, at most 2m/theta sketch rows of 2^p bytes."""
    m = req.raw_edges()
    b = 40 * m + 16 * (1 << req.scale)
    if req.mode == "hybrid":
        b += (2 * m // max(req.theta, 1) + 1) << req.p
    return b


@dataclass
class Resident:
    csr: core.DeviceCSR
    nbytes: int
    last_use: float = 0.0


def split_batch(bt: B.GraphBatch) -> List[core.DeviceCSR]:
    """Per-graph CSRs (each with its own 0-based ids) out of a concatenated
    batch build."""
    g = bt.csr
    vb = bt.vbase.cpu().numpy().astype(np.int64)
    eb_all = g.row_ptr[bt.vbase.long()].cpu().numpy().astype(np.int64)  # edge range of each graph
    out = []
    for i in range(bt.n_graphs):
        a, b = int(vb[i]), int(vb[i + 1])
        ea, eb = int(eb_all[i]), int(eb_all[i + 1])
        row_ptr = (g.row_ptr[a:b + 1] - ea).contiguous()
        col = (g.col_idx[ea:eb] - a).contiguous()
        eu = (g.edge_u[ea:eb] - a).contiguous()
        ids = (g.node_ids[a:b] - int(bt.id_base[i])).contiguous()
        out.append(core.DeviceCSR(row_ptr, col, g.degrees[a:b].contiguous(), ids, eu, col.clone()))
    return out


def concat_csrs(csrs: Sequence[core.DeviceCSR], device) -> B.GraphBatch:
    """One batch CSR over resident graphs (ids shifted by running vertex
    counts; each graph's CSR is already sorted and oriented, so no rebuild)."""
    nn = np.array([c.n_nodes for c in csrs], dtype=np.int64)
    ne = np.array([c.n_edges for c in csrs], dtype=np.int64)
    voff = np.zeros(len(csrs) + 1, dtype=np.int64)
    voff[1:] = np.cumsum(nn)
    eoff = np.zeros(len(csrs) + 1, dtype=np.int64)
    eoff[1:] = np.cumsum(ne)
    if voff[-1] >= np.iinfo(np.int32).max or eoff[-1] > np.iinfo(np.int32).max:
        raise ValueError("batch exceeds int32 CSR limits")
    rps = [c.row_ptr[:-1] + int(e) for c, e in zip(csrs, eoff[:-1])]
    rps.append(torch.tensor([int(eoff[-1])], dtype=torch.int32, device=device))
    row_ptr = torch.cat(rps)
    col = torch.cat([c.col_idx + int(v) for c, v in zip(csrs, voff[:-1])])
    eu = torch.cat([c.edge_u + int(v) for c, v in zip(csrs, voff[:-1])])
    deg = torch.cat([c.degrees for c in csrs])
    ids = torch.cat([c.node_ids.to(torch.int32) for c in csrs])
    csr = core.DeviceCSR(row_ptr, col, deg, ids, eu, col)
    vbase = torch.from_numpy(voff.astype(np.int32)).to(device)
    return B.GraphBatch(csr, vbase, voff)


class Server:
    def __init__(self, device=None, budget_bytes: float = 120e9, max_batch: int = 256,
                 max_batch_edges: float = 4e8):
        self.dev = core._device(device)
        self.budget = int(budget_bytes)
        self.max_batch = max_batch
        self.max_batch_edges = int(max_batch_edges)
        self.resident: "collections.OrderedDict[Tuple, Resident]" = collections.OrderedDict()
        self.resident_bytes = 0
        self.build_stream = torch.cuda.Stream(device=self.dev)
        self.count_stream = torch.cuda.Stream(device=self.dev)
        self.stats = {"ticks": 0, "built": 0, "cache_hits": 0, "evicted": 0, "rejected": 0, "batch_sizes": []}
        self.busy: set = set()  # keys whose graphs the in-flight launch reads

    # ----------------------------------------------------------- memory
    def _evict_for(self, need: int, pinned: set) -> bool:
        while self.resident_bytes + need > self.budget:
            victim = next((k for k in self.resident if k not in pinned and k not in self.busy), None)
            if victim is None:
                return False
            r = self.resident.pop(victim)
            self.resident_bytes -= r.nbytes
            self.stats["evicted"] += 1
        return True

    # ------------------------------------------------------------ stages
    def _admit(self, queue: "collections.deque[Request]", done: List[Completion], now: float) -> List[Request]:
        """FIFO admission under the byte budget and batch limits."""
        taken: List[Request] = []
        pinned: set = set()
        reserve = 0
        edges = 0
        while queue and len(taken) < self.max_batch:
            r = queue[0]
            need = 0 if r.key in self.resident else estimate_bytes(r)
            if need > self.budget:
                queue.popleft()
                self.stats["rejected"] += 1
                done.append(Completion(r.rid, r.mode, None, latency=now - r.arrival,
                                       error=f"needs ~{need / 1e9:.1f} GB, over the {self.budget / 1e9:.1f} GB budget"))
                continue
            if taken and (edges + r.raw_edges() > self.max_batch_edges):
                break
            if not self._evict_for(reserve + need, pinned | {q.key for q in taken}):
                break
            queue.popleft()
            taken.append(r)
            pinned.add(r.key)
            reserve += need
            edges += r.raw_edges()
        return taken

    def _build(self, reqs: List[Request]) -> None:
        """Build the graphs of reqs that are not resident (one concatenated
        device build on the build stream), and make them resident."""
        todo: Dict[Tuple, Request] = {}
        for r in reqs:
            if r.key in self.resident:
                self.stats["cache_hits"] += 1
            else:
                todo.setdefault(r.key, r)
        if not todo:
            return
        with torch.cuda.stream(self.build_stream):
            items = []
            for r in todo.values():
                u, v = generate_edges(r, self.dev)
                items.append((u, v, 1 << r.scale))
            bt = B.GraphBatch.from_edge_lists(items, device=self.dev)
            parts = split_batch(bt)
        for (key, r), csr in zip(todo.items(), parts):
            nb = csr.nbytes()
            self.resident[key] = Resident(csr, nb)
            self.resident_bytes += nb
            self.stats["built"] += 1

    def _launch(self, reqs: List[Request]):
        """Fold the tick's queries into one batched launch per mode on the
        count stream; returns what is needed to finish them."""
        pending = []
        self.count_stream.wait_stream(self.build_stream)
        with torch.cuda.stream(self.count_stream):
            for mode in ("exact", "hybrid"):
                group = [r for r in reqs if r.mode == mode]
                if not group:
                    continue
                csrs = [self.resident[r.key].csr for r in group]
                for c in csrs:  # built on the build stream, read here
                    for t in (c.row_ptr, c.col_idx, c.degrees, c.node_ids, c.edge_u, c.edge_v):
                        t.record_stream(self.count_stream)
                res = torch.empty(len(group) * _lib.RESULT_BYTES, dtype=torch.uint8, device=self.dev)
                r0 = group[0]  # one (p, theta, gamma) per launch; the workload uses one setting
                if len(group) == 1:
                    # a lone query runs the single-graph path directly (same
                    # kernels and integer totals, no concatenation)
                    bt = None
                    g = csrs[0]
                    if mode == "exact":
                        core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, result=res)
                    else:
                        slot, n_rows = core.sketch_slots(g.row_ptr, r0.theta)
                        rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, r0.p)
                        core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees,
                                                          rows, slot, r0.p, r0.gamma, split_kernels=True,
                                                          result=res)
                        bt = (rows, slot)
                else:
                    bt = concat_csrs(csrs, self.dev)
                    if mode == "exact":
                        bt.exact_launch(res)
                    else:
                        rows, slot = bt.sketches(r0.theta, r0.p)
                        bt.hybrid_launch(res, rows, slot, r0.p, r0.gamma)
                ev = torch.cuda.Event()
                ev.record(self.count_stream)
                pending.append((mode, group, res, ev, bt))
        for r in reqs:
            if r.key in self.resident:
                self.resident.move_to_end(r.key)
        self.busy = {r.key for r in reqs}
        return pending

    def _finish(self, pending, done: List[Completion], t0: float) -> None:
        for mode, group, res, ev, bt in pending:
            ev.synchronize()
            now = time.perf_counter() - t0
            try:
                if mode == "exact":
                    vals = B.exact_from_results(res, len(group))
                    for r, v in zip(group, vals):
                        done.append(Completion(r.rid, mode, int(v), latency=now - r.arrival))
                else:
                    tot, st = B.hybrid_from_results(res, len(group))
                    for i, r in enumerate(group):
                        done.append(Completion(r.rid, mode, float(tot[i]), {k: int(st[k][i]) for k in st},
                                               latency=now - r.arrival))
            except ValueError as exc:  # malformed input: fail this group's queries only
                for r in group:
                    done.append(Completion(r.rid, mode, None, latency=now - r.arrival, error=str(exc)))

    # -------------------------------------------------------------- loop
    def serve(self, requests: Sequence[Request]) -> List[Completion]:
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue: "collections.deque[Request]" = collections.deque()
        done: List[Completion] = []
        t0 = time.perf_counter()
        i = 0
        inflight = None
        while len(done) < len(reqs):
            now = time.perf_counter() - t0
            while i < len(reqs) and reqs[i].arrival <= now:
                queue.append(reqs[i])
                i += 1
            nxt = self._admit(queue, done, now) if queue else []
            if nxt:
                self._build(nxt)              # overlaps with the in-flight counts
            if inflight is not None:
                self._finish(inflight, done, t0)
                inflight = None
                self.busy = set()
            if nxt:
                self.stats["ticks"] += 1
                self.stats["batch_sizes"].append(len(nxt))
                inflight = self._launch(nxt)
            elif not queue and i < len(reqs):
                time.sleep(max(0.0, min(reqs[i].arrival - (time.perf_counter() - t0), 0.002)))
        if inflight is not None:
            self._finish(inflight, done, t0)
        return sorted(done, key=lambda c: c.rid)


def serve_sequential(requests: Sequence[Request], device=None) -> List[Completion]:
    """The same requests answered one at a time, in arrival order (build,
    sketch, count, read the result), with the same real-time arrivals."""
    dev = core._device(device)
    reqs = sorted(requests, key=lambda r: r.arrival)
    out: List[Completion] = []
    t0 = time.perf_counter()
    for r in reqs:
        wait = r.arrival - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        out.append(answer_alone(r, dev, t0))
    return sorted(out, key=lambda c: c.rid)


def answer_alone(r: Request, dev, t0: Optional[float] = None) -> Completion:
    """One query on its own: the plain per-graph path."""
    u, v = generate_edges(r, dev)
    g = core.csr_from_edges(u, v, device=dev)
    del u, v
    if r.mode == "exact":
        res, _ = core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v)
        val = core.exact_from_result(res)
        st = None
    else:
        slot, n_rows = core.sketch_slots(g.row_ptr, r.theta)
        rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, r.p)
        res, _ = core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot,
                                                   r.p, r.gamma, split_kernels=True)
        val, rr = core.hybrid_from_result(res)
        st = {k: int(getattr(rr, k)) for k in ("n_approx", "n_exact", "n_fallback", "n_clamped")}
    lat = (time.perf_counter() - t0 - r.arrival) if t0 is not None else float("nan")
    return Completion(r.rid, r.mode, val, st, latency=lat)


def latency_summary(done: Sequence[Completion], wall_s: float) -> Dict:
    ok = [c for c in done if c.error is None]
    lat = np.array([c.latency for c in ok]) * 1e3
    return {"completed": len(ok), "errors": len(done) - len(ok),
            "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
            "graphs_per_s": len(ok) / wall_s if wall_s > 0 else None}


def bench_entry(dev, quick: bool = True) -> Dict:
    """Serving workload at several Poisson rates: p50/p99 latency and
    graphs/s of the continuous-batching server versus answering the same
    requests one at a time; results checked identical between the two."""
    n = 300 if quick else 20000
    out: Dict = {"requests_per_rate": n, "workload": "R-MAT scale U[12,20], ef U[8,32], 50/50 exact / hybrid "
                 "(p=12, theta=gamma=128), Poisson arrivals, 120 GB admission budget"}
    for rate in (50.0, 200.0, 1000.0):
        reqs = c5_requests(n, rate, seed=int(rate))
        srv = Server(dev, budget_bytes=120e9)
        t0 = time.perf_counter()
        got = srv.serve(reqs)
        wall = time.perf_counter() - t0
        s = latency_summary(got, wall)
        s["mean_batch"] = float(np.mean(srv.stats["batch_sizes"])) if srv.stats["batch_sizes"] else 0.0
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        ref = serve_sequential(reqs, dev)
        wall_p = time.perf_counter() - t0
        sp = latency_summary(ref, wall_p)
        same = all(a.value == b.value and a.stats == b.stats for a, b in zip(got, ref))
        out[f"rate_{int(rate)}"] = {"server": s, "sequential": sp, "identical_results": same,
                                    "throughput_ratio": (s["graphs_per_s"] or 0) / max(sp["graphs_per_s"] or 1e-9,
                                                                                       1e-9)}
    return out
