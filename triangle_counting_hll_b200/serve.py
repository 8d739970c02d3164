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
  a query for a graph still being built waits for that build;
* admitted graphs are built by a worker thread on a build stream while
  earlier counts run on a count stream, so arrivals overlap with work
  already on the device and the serving loop itself never waits for the
  GPU (the CSR build's size read-back blocks the worker only): small graphs
  are built and counted together (one batched count launch per mode, exact
  and hybrid, over their concatenated CSRs), large graphs (at least
  ``big_edges`` raw edges, which fill the GPU on their own) one at a time,
  each count launched as soon as its build is seen finished; finished
  counts are polled and answered as the host sees them.
  Per-graph results are bit-identical to answering each query alone;
* latency is completion time minus arrival time; the report gives p50 / p99
  and graphs/s next to the same requests served one at a time.
"""
from __future__ import annotations

import collections
import math
import queue
import sys
import threading
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
    device_ms: float = float("nan")  # answer_alone: device time from generation to the result


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
        b += sketch_bytes(req)
    return b


def sketch_bytes(req: Request) -> int:
    """At most 2m/theta rows of 2^p registers plus the per-vertex slots."""
    return ((2 * req.raw_edges() // max(req.theta, 1) + 1) << req.p) + 8 * (1 << req.scale)


@dataclass
class Resident:
    csr: core.DeviceCSR
    nbytes: int
    last_use: float = 0.0
    # compact sketches per (p, theta), built with the graph for hybrid queries
    sketches: Dict[Tuple[int, int], Tuple[torch.Tensor, torch.Tensor]] = field(default_factory=dict)


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


_STREAMS: Dict[int, Tuple[torch.cuda.Stream, torch.cuda.Stream]] = {}


def _server_streams(dev: torch.device) -> Tuple[torch.cuda.Stream, torch.cuda.Stream]:
    """The (build, count) stream pair of a device, shared by every Server on
    it: torch's caching allocator keeps a block pool per stream, so fresh
    streams per server would pay device allocations again.  Both have the
    default priority: a higher-priority count stream starves the builds,
    whose worker waits on each build's size read-back, and throughput at
    400 requests/s fell below the arrival rate when that was tried."""
    idx = dev.index if dev.index is not None else torch.cuda.current_device()
    if idx not in _STREAMS:
        _STREAMS[idx] = (torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev))
    return _STREAMS[idx]


class _BuildWorker(threading.Thread):
    """Builds graphs (device generator, CSR build, compact sketches of large
    hybrid queries) on the server's build stream, off the serving loop: the
    CSR build reads its vertex and edge counts back to size its outputs, and
    those waits block this thread only.  Each finished job comes back with
    an event recorded on the build stream after it."""

    def __init__(self, dev, build_stream, big_edges: int):
        super().__init__(daemon=True)
        self.dev = dev
        self.stream = build_stream
        self.big_edges = big_edges
        self.inbox: "queue.Queue" = queue.Queue()
        self.outbox: "queue.Queue" = queue.Queue()

    def run(self):
        torch.cuda.set_device(self.dev)
        while True:
            job = self.inbox.get()
            if job is None:
                return
            self.outbox.put(self.build(job))

    def build(self, job):
        """One build job on the build stream -> (job, built, event, error)."""
        out, exc = [], None
        try:
            with torch.cuda.stream(self.stream):
                for key, req, csr in job:
                    if csr is None:  # a new graph
                        u, v = generate_edges(req, self.dev)
                        csr = core.csr_from_edges(u, v, device=self.dev)
                        del u, v
                        sk = None
                        if req.mode == "hybrid" and csr.n_edges >= self.big_edges:
                            sk = _compact_sketches(csr, req)
                        out.append((key, csr, sk))
                    else:  # sketches of a resident large graph
                        out.append((key, None, _compact_sketches(csr, req)))
                ev = torch.cuda.Event()
                ev.record(self.stream)
        except Exception as e:  # reported with the job's queries
            exc, ev = e, None
        return job, out, ev, exc

    def submit(self, job) -> None:
        """Queue a job for the thread, or, when the thread is not running
        (inline serving), build it now on the calling thread."""
        if self.is_alive():
            self.inbox.put(job)
        else:
            self.outbox.put(self.build(job))


def _compact_sketches(csr: core.DeviceCSR, req: Request):
    slot, n_rows = core.sketch_slots(csr.row_ptr, req.theta)
    rows = core.build_sketches_compact_tensors(csr.row_ptr, csr.col_idx, slot, n_rows, req.p)
    return (req.p, req.theta), (rows, slot)


class Server:
    """Continuous-batching server on one GPU: a serving loop (admission,
    count launches, answers) plus a build worker thread.  See the module
    docstring."""

    def __init__(self, device=None, budget_bytes: float = 120e9, max_batch: int = 256,
                 max_batch_edges: float = 4e8, big_edges: int = 1 << 20, threaded: bool = True,
                 reserve_pools: bool = False):
        self.dev = core._device(device)
        self.threaded = threaded  # builds on a worker thread (True) or on the serving loop (False)
        self.big_edges = int(big_edges)
        self.budget = int(budget_bytes)
        self.max_batch = max_batch
        self.max_batch_edges = int(max_batch_edges)
        self.resident: "collections.OrderedDict[Tuple, Resident]" = collections.OrderedDict()
        self.resident_bytes = 0
        self.inflight_bytes = 0  # admission estimates of the jobs in the build worker
        self.build_stream, self.count_stream = _server_streams(self.dev)
        if reserve_pools:  # a process that serves and does little else on this device
            self._reserve_pools()
        self.stats = {"ticks": 0, "built": 0, "cache_hits": 0, "evicted": 0, "rejected": 0, "batch_sizes": [],
                      "single_launches": 0, "batched_launches": 0}
        self.busy: set = set()  # keys whose graphs the in-flight launches read
        self.building: Dict[Tuple, List[Request]] = {}  # keys in the build worker -> queries waiting on them
        self.pending: list = []  # launched, unanswered: (mode, requests, results, event, buffers)
        self._done: List[Completion] = []
        self._t0 = 0.0

    # ----------------------------------------------------------- memory
    def _reserve_pools(self) -> None:
        """Grow torch's cached pools of the build stream (graph arrays) to the
        budget and of the count stream (batch CSRs) to a share of it, once,
        before serving: the allocator keeps one block pool per stream, and
        filling the budget graph by graph would call cudaMalloc for every new
        graph while requests wait (measured at 400 requests/s: p99 340 ms
        with the pools growing on demand, 24 ms with them warm)."""
        free, _ = torch.cuda.mem_get_info(self.dev)
        margin = 8 << 30
        for stream, want in ((self.build_stream, int(self.budget * 1.05)), (self.count_stream, int(self.budget / 16))):
            cached = torch.cuda.memory_reserved(self.dev) - torch.cuda.memory_allocated(self.dev)
            want = min(want, free - margin) - cached
            if want < (1 << 30):
                continue
            with torch.cuda.stream(stream):
                block = torch.empty(want, dtype=torch.uint8, device=self.dev)
                del block
            free, _ = torch.cuda.mem_get_info(self.dev)

    def _evict_for(self, need: int, pinned: set) -> bool:
        while self.resident_bytes + self.inflight_bytes + need > self.budget:
            victim = next((k for k in self.resident
                           if k not in pinned and k not in self.busy and k not in self.building), None)
            if victim is None:
                return False
            r = self.resident.pop(victim)
            self.resident_bytes -= r.nbytes
            self.stats["evicted"] += 1
        return True

    # ------------------------------------------------------------ stages
    def _admit(self, queue_: "collections.deque[Request]", done: List[Completion], now: float):
        """FIFO admission under the byte budget and batch limits.  Returns
        (queries whose graphs are resident, build jobs for the worker)."""
        ready: List[Request] = []
        small_job: list = []
        jobs: list = []
        pinned: set = set()
        edges = 0
        taken = 0
        while queue_ and taken < self.max_batch:
            r = queue_[0]
            if r.key in self.building:  # its graph is being built: answer it with that build
                queue_.popleft()
                self.building[r.key].append(r)
                self.stats["cache_hits"] += 1  # one build serves both queries
                taken += 1
                continue
            res = self.resident.get(r.key)
            if res is not None:
                if r.mode == "hybrid" and res.csr.n_edges >= self.big_edges and (r.p, r.theta) not in res.sketches:
                    need = sketch_bytes(r)
                    if not self._evict_for(need, pinned | {r.key}):
                        break
                    queue_.popleft()
                    self.building[r.key] = [r]
                    self.inflight_bytes += need
                    jobs.append([(r.key, r, res.csr)])
                else:
                    queue_.popleft()
                    ready.append(r)
                    self.stats["cache_hits"] += 1
                pinned.add(r.key)
                taken += 1
                continue
            need = estimate_bytes(r)
            if need > self.budget:
                queue_.popleft()
                self.stats["rejected"] += 1
                done.append(Completion(r.rid, r.mode, None, latency=now - r.arrival,
                                       error=f"needs ~{need / 1e9:.1f} GB, over the {self.budget / 1e9:.1f} GB budget"))
                continue
            if taken and edges + r.raw_edges() > self.max_batch_edges:
                break
            if not self._evict_for(need, pinned):
                break
            queue_.popleft()
            self.building[r.key] = [r]
            self.inflight_bytes += need
            self._est[r.key] = need
            if r.raw_edges() < self.big_edges:
                small_job.append((r.key, r, None))
            else:
                jobs.append([(r.key, r, None)])
            edges += r.raw_edges()
            taken += 1
        if small_job:  # small graphs: one job, then one batched launch
            jobs.insert(0, small_job)
        for job in jobs:
            for key, r, csr in job:
                if csr is not None:
                    self._est[key] = sketch_bytes(r)
            self._worker.submit(job)
        if taken:
            self.stats["ticks"] += 1
            self.stats["batch_sizes"].append(taken)
        return ready

    def _collect(self) -> bool:
        """Make the worker's finished builds resident and launch the queries
        waiting on them; returns whether anything finished."""
        got = False
        while True:
            try:
                job, out, ev, exc = self._worker.outbox.get_nowait()
            except queue.Empty:
                return got
            got = True
            now = time.perf_counter() - self._t0
            for key, _, _ in job:
                self.inflight_bytes -= self._est.pop(key, 0)
            if exc is not None:
                for key, _, _ in job:
                    for r in self.building.pop(key, []):
                        self._done.append(Completion(r.rid, r.mode, None, latency=now - r.arrival,
                                                     error=f"build failed: {exc}"))
                continue
            self.count_stream.wait_event(ev)
            waiting: List[Request] = []
            for key, csr, sk in out:
                if csr is not None:
                    self.resident[key] = Resident(csr, csr.nbytes())
                    self.resident_bytes += self.resident[key].nbytes
                    self.stats["built"] += 1
                res = self.resident[key]
                if sk is not None:
                    (pt, (rows, slot)) = sk
                    res.sketches[pt] = (rows, slot)
                    nb = rows.numel() + slot.numel() * slot.element_size()
                    res.nbytes += nb
                    self.resident_bytes += nb
                waiting += self.building.pop(key, [])
            self._launch_all(waiting)

    def _launch_all(self, reqs: List[Request]) -> None:
        if not reqs:
            return
        self.pending += self._launch(reqs)
        self.busy = {r.key for it in self.pending for r in it[1]}

    def _launch(self, reqs: List[Request]):
        """Fold queries on resident graphs into one batched launch per mode on
        the count stream (large graphs, and a lone query, one launch each);
        returns what is needed to finish them."""
        pending = []
        with torch.cuda.stream(self.count_stream):
            for mode in ("exact", "hybrid"):
                group = [r for r in reqs if r.mode == mode]
                if not group:
                    continue
                csrs = [self.resident[r.key].csr for r in group]
                for c in csrs:  # built on the build stream, read here
                    for t in (c.row_ptr, c.col_idx, c.degrees, c.node_ids, c.edge_u, c.edge_v):
                        t.record_stream(self.count_stream)
                r0 = group[0]  # one (p, theta, gamma) per launch; the workload uses one setting
                lone = [i for i, g in enumerate(csrs) if len(group) == 1 or g.n_edges >= self.big_edges]
                lone_set = set(lone)
                rest = [i for i in range(len(group)) if i not in lone_set]
                for i in lone:
                    g = csrs[i]
                    keep = []
                    res = torch.empty(_lib.RESULT_BYTES, dtype=torch.uint8, device=self.dev)
                    if mode == "exact":
                        core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, result=res)
                    else:
                        sk = self.resident[group[i].key].sketches.get((r0.p, r0.theta))
                        if sk is None:  # a lone query on a small graph
                            slot, n_rows = core.sketch_slots(g.row_ptr, r0.theta)
                            rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, r0.p)
                        else:
                            rows, slot = sk
                            rows.record_stream(self.count_stream)
                            slot.record_stream(self.count_stream)
                        core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees,
                                                          rows, slot, r0.p, r0.gamma, split_kernels=True,
                                                          result=res)
                        keep.append((rows, slot))
                    ev = torch.cuda.Event()
                    ev.record(self.count_stream)
                    pending.append((mode, [group[i]], res, ev, keep))
                    self.stats["single_launches"] += 1
                if rest:
                    sub = [group[i] for i in rest]
                    res = torch.empty(len(sub) * _lib.RESULT_BYTES, dtype=torch.uint8, device=self.dev)
                    bt = concat_csrs([csrs[i] for i in rest], self.dev)
                    if mode == "exact":
                        bt.exact_launch(res)
                    else:
                        rows, slot = bt.sketches(r0.theta, r0.p)
                        bt.hybrid_launch(res, rows, slot, r0.p, r0.gamma)
                    ev = torch.cuda.Event()
                    ev.record(self.count_stream)
                    pending.append((mode, sub, res, ev, bt))
                    self.stats["batched_launches"] += 1
        for r in reqs:
            if r.key in self.resident:
                self.resident.move_to_end(r.key)
        return pending

    def _complete(self, item, done: List[Completion], t0: float) -> None:
        mode, group, res, ev, _ = item
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

    def _reap(self) -> bool:
        """Answer every launched query whose count has finished, never
        waiting; a query's latency ends when the host sees its result.
        Returns whether anything was answered."""
        keep = []
        got = False
        for item in self.pending:
            if not keep and item[3].query():  # the count stream finishes launches in order
                self._complete(item, self._done, self._t0)
                got = True
            else:
                keep.append(item)
        self.pending = keep
        self.busy = {r.key for it in self.pending for r in it[1]}
        return got

    # -------------------------------------------------------------- loop
    def serve(self, requests: Sequence[Request]) -> List[Completion]:
        """Serve requests in real time (arrival = seconds after the call);
        returns one Completion per request, ordered by request id.  The loop
        never waits for the GPU: builds run in the worker thread, counts of
        several ticks may be in flight on the count stream, and finished
        counts are polled."""
        reqs = sorted(requests, key=lambda r: r.arrival)
        queue_: "collections.deque[Request]" = collections.deque()
        self._done = []
        self._est: Dict[Tuple, int] = {}
        self.pending = []
        self._worker = _BuildWorker(self.dev, self.build_stream, self.big_edges)
        switch = sys.getswitchinterval()
        if self.threaded:
            # the worker needs the interpreter lock back after each CUDA call
            # it waits in: hand it over within 0.5 ms instead of 5 ms
            sys.setswitchinterval(min(switch, 5e-4))
            self._worker.start()
        self._t0 = t0 = time.perf_counter()
        i = 0
        try:
            while len(self._done) < len(reqs):
                now = time.perf_counter() - t0
                while i < len(reqs) and reqs[i].arrival <= now:
                    queue_.append(reqs[i])
                    i += 1
                busy = self._reap()
                busy |= self._collect()
                ready = self._admit(queue_, self._done, now) if queue_ else []
                if ready:
                    self._launch_all(ready)
                    busy = True
                if not busy:  # nothing to do until an arrival, a build or a count finishes
                    nxt = reqs[i].arrival - (time.perf_counter() - t0) if i < len(reqs) else 1.0
                    time.sleep(max(0.0, min(nxt, 0.0002)))
                elif self.threaded:
                    time.sleep(0)  # let the build worker take the interpreter lock
        finally:
            if self.threaded:
                self._worker.inbox.put(None)
                self._worker.join(timeout=60)
                sys.setswitchinterval(switch)
        return sorted(self._done, key=lambda c: c.rid)


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
    """One query on its own: the plain per-graph path.  ``device_ms`` is the
    CUDA-event time from the graph's generation to its result (the device
    work of one query, with the build's one size read-back inside)."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
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
    e1.record()
    lat = (time.perf_counter() - t0 - r.arrival) if t0 is not None else float("nan")
    e1.synchronize()
    return Completion(r.rid, r.mode, val, st, latency=lat, device_ms=e0.elapsed_time(e1))


def latency_summary(done: Sequence[Completion], wall_s: float) -> Dict:
    ok = [c for c in done if c.error is None]
    lat = np.array([c.latency for c in ok]) * 1e3
    out = {"completed": len(ok), "errors": len(done) - len(ok),
           "p50_ms": float(np.percentile(lat, 50)) if len(lat) else None,
           "p99_ms": float(np.percentile(lat, 99)) if len(lat) else None,
           "graphs_per_s": len(ok) / wall_s if wall_s > 0 else None}
    dms = np.array([c.device_ms for c in ok if c.device_ms == c.device_ms])
    if len(dms):  # one query at a time: the device work behind each answer
        out["device_ms_total"] = float(dms.sum())
        out["device_ms_mean"] = float(dms.mean())
        out["device_bound_graphs_per_s"] = float(len(dms) / (dms.sum() / 1e3)) if dms.sum() > 0 else None
        out["device_busy_frac"] = float(dms.sum() / 1e3 / wall_s) if wall_s > 0 else None
    return out


def _warm(dev) -> None:
    """Warm both paths (allocator pools of the server streams and the default
    stream, lazy kernel loading) on requests outside the timed sets, then one
    paced run like the timed ones, so the server's streams have served
    requests arriving one at a time too."""
    warm = [Request(i, 0.0, 20, 32, 777 + i, m) for i, m in enumerate(("exact", "hybrid", "exact", "hybrid"))]
    warm += c5_requests(40, 1e6, seed=12345)
    for _ in range(2):
        Server(dev, budget_bytes=120e9, reserve_pools=True).serve(warm)
        serve_sequential(warm, dev)
    Server(dev, budget_bytes=120e9, reserve_pools=True).serve(c5_requests(60, 50.0, seed=4242))
    # a burst of the timed mix, so the cached block pools reach the sizes
    # the timed runs ask for (their cudaMalloc calls otherwise land in them)
    Server(dev, budget_bytes=120e9, reserve_pools=True).serve(c5_requests(600, 1e4, seed=999))
    torch.cuda.synchronize(dev)


def _compare(dev, reqs, threaded: bool = True) -> Dict:
    srv = Server(dev, budget_bytes=120e9, threaded=threaded, reserve_pools=True)
    a0 = torch.cuda.memory_stats(dev).get("num_device_alloc", 0)
    t0 = time.perf_counter()
    got = srv.serve(reqs)
    wall = time.perf_counter() - t0
    s = latency_summary(got, wall)
    s["device_mallocs"] = torch.cuda.memory_stats(dev).get("num_device_alloc", 0) - a0  # cudaMalloc calls inside
    s["mean_batch"] = float(np.mean(srv.stats["batch_sizes"])) if srv.stats["batch_sizes"] else 0.0
    s["builds"] = srv.stats["built"]
    s["batched_launches"] = srv.stats["batched_launches"]
    s["single_launches"] = srv.stats["single_launches"]
    del srv
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    ref = serve_sequential(reqs, dev)
    wall_p = time.perf_counter() - t0
    sp = latency_summary(ref, wall_p)
    same = all(a.value == b.value and a.stats == b.stats for a, b in zip(got, ref))
    return {"requests": len(reqs), "server": s, "sequential": sp, "identical_results": same,
            "throughput_ratio": (s["graphs_per_s"] or 0) / max(sp["graphs_per_s"] or 1e-9, 1e-9),
            "p99_ratio": (s["p99_ms"] or 0) / max(sp["p99_ms"] or 1e-9, 1e-9)}


def bench_entry(dev, quick: bool = True) -> Dict:
    """Serving workload at several Poisson rates: p50/p99 latency and
    graphs/s of the continuous-batching server versus answering the same
    requests one at a time; results checked identical between the two.
    (The quick form, 300 requests per rate, for the headline line; bench_c5
    runs the full 20,000.)"""
    n = 300 if quick else 20000
    out: Dict = {"requests_per_rate": n, "workload": "R-MAT scale U[12,20], ef U[8,32], 50/50 exact / hybrid "
                 "(p=12, theta=gamma=128), Poisson arrivals, 120 GB admission budget"}
    _warm(dev)
    for rate in (50.0, 200.0, 1000.0):
        out[f"rate_{int(rate)}"] = _compare(dev, c5_requests(n, rate, seed=int(rate)))
        if quick:  # builds on the serving loop instead of the worker thread, for comparison
            out[f"rate_{int(rate)}_inline"] = _compare(dev, c5_requests(n, rate, seed=int(rate)), threaded=False)
    return out


def bench_c5(dev, n_saturating: int = 20000, rates=((2000.0, 20000), (400.0, 4000), (100.0, 1500))) -> Dict:
    """The serving configuration at full size: 20,000 requests arriving
    faster than either path can serve them (2,000/s), plus lower Poisson
    rates with the request counts given (about 10-15 s of arrivals each),
    each against the same requests served one at a time."""
    out: Dict = {"workload": "R-MAT scale U[12,20], ef U[8,32], 50/50 exact / hybrid (p=12, theta=gamma=128), "
                             "Poisson arrivals, 120 GB admission budget"}
    _warm(dev)
    for rate, n in rates:
        if rate == rates[0][0]:
            n = n_saturating
        out[f"rate_{int(rate)}"] = _compare(dev, c5_requests(n, rate, seed=int(rate)))
    return out
