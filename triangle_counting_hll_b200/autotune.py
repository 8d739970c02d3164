"""Launch-shape autotuner for the counting kernels, keyed on the degree
histogram.

The counting kernels take a process-wide launch shape (edges per work chunk,
per-warp hash-table capacity, lane-local merge threshold, table load); the
result never depends on it, only the speed does.  The best shape depends on
the forward-degree distribution, so the tuner summarises a graph by the
log2 histogram of its forward degrees (``tchll_degree_stats``, the statistics
experiment/gpu_graph_stats.py:100-140 computes), times a handful of
candidate shapes on the first graph of a new signature, and reuses the winner
for every later graph with the same signature.  The cache can persist to a
JSON file.
"""
from __future__ import annotations

import ctypes as C
import json
import os
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib, core
from ._lib import check, load, ptr, stream_handle

CANDIDATES: List[Dict] = [
    {"chunk": 256, "slots_log2": 11, "tiny": 16, "sparse": 0, "hub": 128},
    {"chunk": 128, "slots_log2": 11, "tiny": 16, "sparse": 0, "hub": 128},
    {"chunk": 512, "slots_log2": 11, "tiny": 16, "sparse": 0, "hub": 128},
    {"chunk": 256, "slots_log2": 11, "tiny": 48, "sparse": 1, "hub": 128},
    {"chunk": 256, "slots_log2": 10, "tiny": 24, "sparse": 0, "hub": 128},
    {"chunk": 64, "slots_log2": 9, "tiny": 32, "sparse": 0, "hub": 128},
    {"chunk": 256, "slots_log2": 11, "tiny": 16, "sparse": 0, "hub": 256},
    {"chunk": 256, "slots_log2": 10, "tiny": 24, "sparse": 0, "hub": 256},
    {"chunk": 256, "slots_log2": 11, "tiny": 16, "sparse": 0, "hub": 0},
    {"chunk": 256, "slots_log2": 10, "tiny": 24, "sparse": 0, "hub": 0},
]


def degree_stats(row_ptr: torch.Tensor = None, degrees: torch.Tensor = None) -> Dict:
    """Forward-degree statistics on the device: count of vertices with d > 0,
    sum, sum of squares, max, min, and the floor(log2 d) histogram."""
    t = row_ptr if row_ptr is not None else degrees
    dev = t.device
    n = int(row_ptr.numel()) - 1 if row_ptr is not None else int(degrees.numel())
    hist = torch.zeros(32, dtype=torch.uint64, device=dev)
    sums = torch.zeros(3, dtype=torch.uint64, device=dev)
    mm = torch.zeros(2, dtype=torch.int32, device=dev)
    check(load().tchll_degree_stats(ptr(degrees) if degrees is not None else None,
                                    ptr(row_ptr) if row_ptr is not None else None, n, ptr(hist), ptr(sums), ptr(mm),
                                    stream_handle(dev)), "degree stats")
    h = hist.cpu().view(torch.int64).numpy()
    sm = sums.cpu().view(torch.int64).numpy()
    mmh = mm.cpu().numpy()
    return {"log_hist": h, "active": int(sm[0]), "sum": int(sm[1]), "sumsq": int(sm[2]),
            "max": int(mmh[0]), "min": int(mmh[1]) if sm[0] else 0}


def signature(stats: Dict) -> str:
    """Coarse key: top log2 bucket and the degree-weighted log2 histogram in
    eighths (the work a bucket contributes grows with d, so weight by d)."""
    h = stats["log_hist"].astype(np.float64)
    if h.sum() == 0:
        return "empty"
    w = h * (2.0 ** np.arange(32))
    w = np.round(8 * w / w.sum()).astype(int)
    top = int(np.nonzero(h)[0].max())
    return f"top{top}:" + ",".join(str(x) for x in w[: top + 1])


class Autotuner:
    def __init__(self, cache_path: Optional[str] = None, candidates: Sequence[Dict] = CANDIDATES):
        self.cache_path = cache_path
        self.candidates = list(candidates)
        self.cache: Dict[str, Dict] = {}
        if cache_path and os.path.exists(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def _save(self) -> None:
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1, sort_keys=True)
            os.replace(tmp, self.cache_path)

    @staticmethod
    def apply(cfg: Dict) -> None:
        core.set_count_tuning(chunk=cfg["chunk"], slots_log2=cfg["slots_log2"], tiny=cfg["tiny"],
                              sparse=bool(cfg.get("sparse", 0)), hub=int(cfg.get("hub", 128)))

    def tune(self, key_row_ptr: torch.Tensor, run: Callable[[], None], reps: int = 2) -> Dict:
        """Pick (or recall) the fastest candidate for graphs shaped like the one
        whose CSR row_ptr is given; ``run`` performs one full count."""
        key = signature(degree_stats(key_row_ptr))
        if key in self.cache:
            self.apply(self.cache[key])
            return dict(self.cache[key], key=key, cached=True)
        dev = key_row_ptr.device
        best, best_ms = None, float("inf")
        for cfg in self.candidates:
            self.apply(cfg)
            run()  # warm-up
            torch.cuda.synchronize(dev)
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            for _ in range(reps):
                run()
            e.record()
            torch.cuda.synchronize(dev)
            ms = s.elapsed_time(e) / reps
            if ms < best_ms:
                best, best_ms = cfg, ms
        self.cache[key] = dict(best, ms=best_ms)
        self._save()
        self.apply(best)
        return dict(best, ms=best_ms, key=key, cached=False)


_default = Autotuner()


def tune_exact(g: core.DeviceCSR, tuner: Optional[Autotuner] = None) -> Dict:
    """Tune the single-graph exact count for a graph like g."""
    t = tuner or _default
    res = _lib.count_result_tensor(g.device)
    return t.tune(g.row_ptr, lambda: core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v,
                                                                result=res))


def tune_batch(batch, tuner: Optional[Autotuner] = None) -> Dict:
    """Tune the batched exact count on a GraphBatch."""
    t = tuner or _default
    res = torch.empty(max(batch.n_graphs, 1) * _lib.RESULT_BYTES, dtype=torch.uint8, device=batch.csr.device)
    return t.tune(batch.csr.row_ptr, lambda: batch.exact_launch(res))
