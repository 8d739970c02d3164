#!/usr/bin/env python
"""Headline benchmark: exact triangle count of the R-MAT scale-22 graph.

One step = one exact count (``tchll_exact_count``) over the oriented CSR of
an R-MAT graph (scale 22, edge factor 16, (a,b,c,d) = (.57,.19,.19,.05),
seed 1; symmetrised, deduplicated, self-loops dropped: 64.15 M oriented
edges), inputs resident in HBM, plus the 64-byte result read back.  The same
metric end to end (``e2e``) goes through the public API
``gpu_exact_triangle_count`` with the CSR in pinned host memory, so every step
includes the host-to-device copies.  Extra keys report the hybrid sweep
(p in {8,10,12,14}, theta = gamma = 256), the batched and serving workloads
when their modules are present, the roofline of the counting kernel and a CPU
baseline (the oracle, a C port of the reference's counting loop, on a strided
sample of the same edges).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one rank per GPU, each counting its own copy of
the graph (weak scaling); times are the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SCALE = 22
EDGE_FACTOR = 16
ABC = (0.57, 0.19, 0.19)
SEED = 1
HYB_THETA = 256
HYB_PS = (8, 10, 12, 14)
METRIC = "edges/s"
WORKLOAD = "rmat22_ef16_exact_count"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--no-extras", action="store_true", help="skip the hybrid / batched / serving extras")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU-baseline sample budget")
    ap.add_argument("--mode", choices=("exact", "hybrid"), default="exact",
                    help="exact (the headline line) or hybrid: one hybrid count per step with prebuilt compact "
                         "sketches (theta = gamma)")
    ap.add_argument("--p", type=int, default=12, help="HLL precision for --mode hybrid")
    ap.add_argument("--theta", type=int, default=HYB_THETA, help="sketch / route threshold for --mode hybrid")
    ap.add_argument("--sharded", action="store_true",
                    help="N>1: split one graph's edges across ranks (strong scaling) instead of one graph per rank")
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:  # pragma: no cover
        return os.cpu_count() or 1


def load_peaks() -> dict:
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def load_traffic(workload: str):
    path = os.path.join(ROOT, "profiles", "traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        d = json.load(f)
    return d.get(workload)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 100 ms while active."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="tchll_clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower() in ("active", "1"):
                        reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm_sorted = sorted(sm)
        return {"sm_mhz": sm_sorted[len(sm_sorted) // 2], "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm)}


# --------------------------------------------------------------------- ours
def run_ours(args):
    import numpy as np
    import torch
    import torch.distributed as dist

    from triangle_counting_hll_b200 import _lib, core
    from triangle_counting_hll_b200.gpu_hybrid import gpu_exact_triangle_count

    rank, world, local = dist_env()
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(x: float) -> float:
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    # ---- graph (weak scaling: every rank counts its own copy)
    u, v = core.gen_rmat(args.scale, EDGE_FACTOR, *ABC, seed=SEED, device=dev)
    g = core.csr_from_edges(u, v)
    del u, v
    torch.cuda.synchronize()
    deg = (g.row_ptr[1:] - g.row_ptr[:-1]).long()
    du, dv = deg[g.edge_u.long()], deg[g.edge_v.long()]
    algo_bytes = 16 * g.n_edges + 4 * int((du + dv).sum().item())
    # pairs whose longer list exceeds the hub threshold go to the hub kernel
    hub_thr = core.get_count_tuning()["hub"]
    is_hub = torch.maximum(du, dv) > hub_thr if hub_thr > 0 else torch.zeros_like(du, dtype=torch.bool)
    hub_bytes = 16 * int(is_hub.sum().item()) + 4 * int(torch.where(is_hub, du + dv, 0).sum().item())
    del du, dv, is_hub
    res = _lib.count_result_tensor(dev)
    if args.mode == "hybrid":
        return run_hybrid_line(args, g, dev, rank, world, barrier, max_over_ranks)

    if args.sharded and world > 1:
        from triangle_counting_hll_b200 import dist as D
        lo, hi = D.shard_bounds(D.device_costs(g), world)[rank]
        my_u, my_v = g.edge_u[lo:hi].contiguous(), g.edge_v[lo:hi].contiguous()

        def step():
            core.exact_count_tensors(g.row_ptr, g.col_idx, my_u, my_v, result=res)
            parts = D.gather_results(D.result_to_tuple(_lib.read_count_result(res)))
            return D.combine(parts)["exact"]
    else:
        def step():
            core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, result=res)
            return core.exact_from_result(res)  # 64-byte D2H read of the result

    for _ in range(max(args.warmup, 0)):
        count = step()
    core.set_phase_timing(True)
    launches0 = _lib.launch_count()
    clocks = ClockSampler(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kernel_ms, pair_ms, hub_ms = [], [], []
    ev0.record()
    for _ in range(args.steps):
        count = step()
        ph = core.phase_times()
        kernel_ms.append(ph["count"])
        if ph["pairs"] is not None:
            pair_ms.append(ph["pairs"])
        if ph["hub"] is not None:
            hub_ms.append(ph["hub"])
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = (_lib.launch_count() - launches0) / max(args.steps, 1)
    core.set_phase_timing(False)
    ms_total = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = ms_total / args.steps
    sharded = bool(args.sharded and world > 1)
    value = (1 if sharded else world) * g.n_edges / (ms_step / 1e3)
    kernel_avg = sum(kernel_ms) / len(kernel_ms)
    hub_avg = sum(hub_ms) / len(hub_ms) if hub_ms else None

    # ---- end to end through the public API, CSR in pinned host memory
    host = [t.cpu().pin_memory() for t in (g.row_ptr, g.col_idx, g.edge_u, g.edge_v)]
    h2d = sum(t.numel() * t.element_size() for t in host)
    for _ in range(max(1, min(args.warmup, 2))):
        gpu_exact_triangle_count(*host)
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        c_e2e, _ = gpu_exact_triangle_count(*host)
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    assert c_e2e == count
    del host

    peaks = load_peaks()
    if hub_avg:  # the dominant kernel: the hub pairs
        kname, kms, kbytes = "hub_count_kernel", hub_avg, hub_bytes
    else:
        kname, kms, kbytes = "count_kernel<exact>", kernel_avg, algo_bytes
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = load_traffic(f"{WORKLOAD}:{kname}")
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "edges/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_step,
        "higher_is_better": True,
        "scaling": "strong" if sharded else "weak",
        "vs_baseline": None,
        "dtype": "int32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "graph": f"R-MAT scale {args.scale} ef {EDGE_FACTOR} "
                   f"(a,b,c)=({ABC[0]},{ABC[1]},{ABC[2]}) seed {SEED}", "n_nodes": g.n_nodes,
                   "n_edges": g.n_edges, "triangles": count,
                   "l2": "inputs larger than L2 (CSR + edge arrays %.0f MB > 126 MB)" % (g.nbytes() / 1e6),
                   "parallelism": (f"edge shards x{world}" if sharded else f"replicas x{world}"),
                   "tuning": core.get_count_tuning()},
        "triangles_per_s": (1 if sharded else world) * count / (ms_step / 1e3),
        "hbm_frac_whole_call": (algo_bytes / (ms_step / 1e3) / 1e9) / peaks["hbm_gbs"],
        "e2e": {"value": (1 if sharded else world) * g.n_edges / (e2e_ms / 1e3), "unit": "edges/s",
                "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": _lib.RESULT_BYTES},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "peak_source": peaks["source"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "kernel_ms": kms, "algorithmic_bytes": kbytes,
                     "traffic": traffic["bytes_per_launch"] if traffic else None,
                     "traffic_source": traffic["source"] if traffic else None,
                     "count_phase": {"ms": kernel_avg, "algorithmic_bytes": algo_bytes,
                                     "frac": algo_bytes / (kernel_avg / 1e3) / 1e9 / peaks["hbm_gbs"],
                                     "hub_ms": hub_avg,
                                     "pair_kernel_ms": (kernel_avg - hub_avg) if hub_avg else kernel_avg},
                     "pair_regroup_ms": (sum(pair_ms) / len(pair_ms)) if pair_ms else None},
        "gpu_launches": launches,
        "clocks": clk,
    }

    # the extras (hybrid sweep, batched and serving workloads) are one-GPU
    # measurements: a multi-GPU run reports the headline line only
    if not args.no_extras and world == 1:
        line["hybrid"] = hybrid_sweep(g, count, dev)
        for name, mod in (("batched", "triangle_counting_hll_b200.batch"),
                          ("serving", "triangle_counting_hll_b200.serve")):
            try:
                m = __import__(mod, fromlist=["bench_entry"])
            except ImportError:
                continue
            if hasattr(m, "bench_entry"):
                line[name] = m.bench_entry(dev, quick=True)

    if rank == 0 and world == 1:
        line["cpu_baseline"] = cpu_baseline(g, count, args.cpu_seconds)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def run_hybrid_line(args, g, dev, rank, world, barrier, max_over_ranks):
    """--mode hybrid: one hybrid count (compact sketches built once, before
    timing; theta = gamma) per step.  Roofline of the dominant phase: the
    exact-pair count over exact-routed edges (16 + 4 (d+u + d+v) bytes each)
    or the HLL pass (16 + 2 * 2^p bytes per HLL edge)."""
    import torch
    import torch.distributed as dist

    from triangle_counting_hll_b200 import _lib, core
    p, theta = args.p, args.theta
    slot, n_rows = core.sketch_slots(g.row_ptr, theta)
    rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, p)
    deg = g.degrees.long()
    du, dv = deg[g.edge_u.long()], deg[g.edge_v.long()]
    hll = torch.minimum(du, dv) >= theta
    n_hll = int(hll.sum().item())
    exact_bytes = 16 * (g.n_edges - n_hll) + 4 * int(torch.where(hll, 0, du + dv).sum().item())
    hub_thr = core.get_count_tuning()["hub"]
    hub = (~hll) & (torch.maximum(du, dv) > hub_thr) if hub_thr > 0 else torch.zeros_like(hll)
    hub_bytes = 16 * int(hub.sum().item()) + 4 * int(torch.where(hub, du + dv, 0).sum().item())
    hll_bytes = n_hll * (16 + 2 * (1 << p))
    del du, dv, hll, hub
    res = _lib.count_result_tensor(dev)
    ex_res, _ = core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v)
    exact = core.exact_from_result(ex_res)

    def step():
        core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot, p, theta,
                                          split_kernels=True, result=res)
        return core.hybrid_from_result(res)

    for _ in range(max(args.warmup, 0)):
        step()
    core.set_phase_timing(True)
    launches0 = _lib.launch_count()
    clocks = ClockSampler(torch.cuda.current_device())
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    phases = []
    ev0.record()
    for _ in range(args.steps):
        total, r = step()
        phases.append(core.phase_times())
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = (_lib.launch_count() - launches0) / max(args.steps, 1)
    core.set_phase_timing(False)
    ms_step = max_over_ranks(ev0.elapsed_time(ev1)) / args.steps
    avg = {k: sum((ph[k] or 0.0) for ph in phases) / len(phases) for k in phases[0]}

    # end to end: CSR + compact sketches from pinned host memory each step
    host = [t.cpu().pin_memory() for t in (g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot)]
    h2d = sum(t.numel() * t.element_size() for t in host)

    def e2e_step():
        d = [t.to(dev, non_blocking=True) for t in host]
        core.hybrid_count_compact_tensors(*d[:7], p, theta, split_kernels=True, result=res)
        return core.hybrid_from_result(res)

    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        t2, _ = e2e_step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    assert t2 == total
    del host

    peaks = load_peaks()
    # the dominant kernel of the three: HLL pass, hub pairs, other exact pairs
    hub_ms = avg.get("hub") or 0.0
    cands = [("hll_edges_kernel", avg["hll"], hll_bytes), ("hub_count_kernel", hub_ms, hub_bytes),
             ("count_kernel", avg["count"] - hub_ms, exact_bytes - hub_bytes)]
    kname, kms, kbytes = max(cands, key=lambda c: c[1])
    achieved = kbytes / (kms / 1e3) / 1e9
    traffic = load_traffic(f"rmat{args.scale}_ef16_hybrid_p{p}_theta{theta}:{kname}")
    line = {
        "metric": METRIC, "value": world * g.n_edges / (ms_step / 1e3), "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32+u8", "data": "synthetic",
        "config": {"workload": f"rmat{args.scale}_ef16_hybrid_p{p}_theta{theta}",
                   "graph": f"R-MAT scale {args.scale} ef {EDGE_FACTOR} (a,b,c)=({ABC[0]},{ABC[1]},{ABC[2]}) "
                            f"seed {SEED}", "n_edges": g.n_edges, "p": p, "theta": theta, "gamma": theta,
                   "n_sketched": n_rows, "n_hll_edges": n_hll, "exact_triangles": exact,
                   "l2": "inputs larger than L2", "parallelism": f"replicas x{world}"},
        "estimate": total, "rel_err": abs(total - exact) / exact if exact else 0.0,
        "stats": {"n_approx": int(r.n_approx), "n_exact": int(r.n_exact), "n_clamped": int(r.n_clamped)},
        "phases_ms": avg,
        "e2e": {"value": world * g.n_edges / (e2e_ms / 1e3), "unit": "edges/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": _lib.RESULT_BYTES},
        "roofline": {"bound": "hbm", "kernel": kname, "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "peak_source": peaks["source"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "kernel_ms": kms, "algorithmic_bytes": kbytes,
                     "traffic": traffic["bytes_per_launch"] if traffic else None,
                     "traffic_source": traffic["source"] if traffic else None,
                     "kernels": {c[0]: {"ms": c[1], "algorithmic_bytes": c[2]} for c in cands}},
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def hybrid_sweep(g, exact_count: int, dev) -> dict:
    import torch

    from triangle_counting_hll_b200 import _lib, core
    out = {}
    res = _lib.count_result_tensor(dev)
    for p in HYB_PS:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        slot, n_rows = core.sketch_slots(g.row_ptr, HYB_THETA)
        rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, p)
        torch.cuda.synchronize()
        build_ms = (time.perf_counter() - t0) * 1e3
        best = None
        for _ in range(3):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot, p,
                                              HYB_THETA, split_kernels=True, result=res)
            e.record()
            torch.cuda.synchronize()
            ms = s.elapsed_time(e)
            best = ms if best is None else min(best, ms)
        total, r = core.hybrid_from_result(res)
        out[f"p{p}"] = {"theta": HYB_THETA, "gamma": HYB_THETA, "ms": best, "edges_per_s": g.n_edges / (best / 1e3),
                        "sketch_build_ms": build_ms, "n_sketched": n_rows, "estimate": total,
                        "rel_err": abs(total - exact_count) / exact_count, "n_approx": int(r.n_approx),
                        "clamp_ratio": int(r.n_clamped) / max(int(r.n_approx), 1)}
        del rows, slot
    return out


def calibrate_rate(O, rp, ci, eu, ev, cores: int, min_s: float = 1.0) -> float:
    """Edges/s of the oracle's exact count on strided samples of the oriented
    edges, grown 4x at a time until one sample runs for at least min_s (thread
    start-up and tiny samples understate the rate)."""
    import numpy as np
    E = len(eu)
    n = min(E, 4096)
    while True:
        sel = np.arange(0, E, max(E // n, 1))
        t0 = time.perf_counter()
        O.exact_count(rp, ci, eu[sel], ev[sel], nthreads=cores)
        dt = time.perf_counter() - t0
        if dt >= min_s or len(sel) >= E:
            return len(sel) / max(dt, 1e-9)
        n = min(E, n * 4 if dt <= 0 else max(n * 2, int(n * min(8.0, 1.5 * min_s / dt))))


def cpu_baseline(g, exact_count: int, budget_s: float) -> dict:
    """The oracle (C restatement of the reference's counting loop) timed on a
    strided sample of the same oriented edges, all host threads."""
    import numpy as np

    from oracle import build_oracle
    build_oracle.build()
    from oracle import oracle as O
    rp = g.row_ptr.cpu().numpy()
    ci = g.col_idx.cpu().numpy()
    eu = g.edge_u.cpu().numpy()
    ev = g.edge_v.cpu().numpy()
    cores = host_cores()
    E = len(eu)
    rate = calibrate_rate(O, rp, ci, eu, ev, cores)
    n = int(min(E, max(1, rate * budget_s)))
    stride = max(E // n, 1)
    sel = np.arange(0, E, stride)
    t0 = time.perf_counter()
    O.exact_count(rp, ci, eu[sel], ev[sel], nthreads=cores)
    dt = time.perf_counter() - t0
    return {"value": len(sel) / dt, "unit": "edges/s", "cores": cores, "kind": "port",
            "sample": f"every {stride}-th of {E} oriented edges ({len(sel)} edges, {dt:.1f} s), "
                      f"oracle exact count (merge / binary search per edge, OpenMP)"}


# ---------------------------------------------------------------- reference
def run_reference(args):
    """The reference's CPU counting loop (its C port in oracle/, all host
    threads) on this arm's workload; rank 0 only."""
    rank, world, _ = dist_env()
    if rank != 0:
        return
    import numpy as np

    from oracle import build_oracle
    build_oracle.build()
    from oracle import oracle as O
    cores = host_cores()
    u, v = O.gen_rmat(args.scale, EDGE_FACTOR, *ABC, SEED)
    g = O.csr_build(u, v)
    del u, v
    rp, ci, eu, ev = g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"]
    E = len(eu)
    rate = calibrate_rate(O, rp, ci, eu, ev, cores)
    # about 3 s of CPU work per step, less when many steps are asked for, so
    # the whole run stays near a minute of CPU time
    per_step = min(3.0, max(0.5, 60.0 / max(args.steps + args.warmup, 1)))
    stride = max(int(E // max(rate * per_step, 1.0)), 1)
    sel = np.arange(0, E, stride)
    su, sv = eu[sel], ev[sel]
    for _ in range(max(args.warmup, 0)):
        O.exact_count(rp, ci, su, sv, nthreads=cores)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        O.exact_count(rp, ci, su, sv, nthreads=cores)
    dt = (time.perf_counter() - t0) / max(args.steps, 1)
    val = len(sel) / dt
    sample = (f"every {stride}-th of {E} oriented edges ({len(sel)} edges) per step; oracle exact count "
              f"(C port of src/exact.py's loop, OpenMP)")
    line = {
        "impl": "reference", "metric": METRIC, "value": val, "unit": "edges/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "graph": f"R-MAT scale {args.scale} ef {EDGE_FACTOR} "
                   f"(a,b,c)=({ABC[0]},{ABC[1]},{ABC[2]}) seed {SEED}", "n_edges": E},
        "cpu_baseline": {"value": val, "unit": "edges/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": val, "unit": "edges/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
