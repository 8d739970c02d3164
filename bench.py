#!/usr/bin/env python
"""Headline benchmark: exact triangle count of the R-MAT scale-22 graph.

One step = one exact count (``tchll_exact_count``) over the oriented CSR of
an R-MAT graph (scale 22, edge factor 16, (a,b,c,d) = (.57,.19,.19,.05),
seed 1; symmetrised, deduplicated, self-loops dropped: 64.15 M oriented
edges), inputs resident in HBM, plus the 64-byte result read back.  The same
metric end to end (``e2e``) goes through the public API
``gpu_exact_triangle_count`` with the CSR in pinned host memory, so every step
includes the host-to-device copies.  Extra keys: the device CSR build
(``csr_build``), the hybrid sweep (p in {8,10,12,14} at theta = gamma = 256,
and theta = gamma in {64, 128}), the batched and serving workloads, the
roofline of the dominant kernel on its measured DRAM traffic, the CPU
baseline (the oracle, a C port of the reference's counting loop, over all
edges of the same graph) and ``parity``: the oracle's count must equal the
GPU's and its FP64 hybrid estimate (p = 12) must agree within 1e-6, else the
run fails.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun, one rank per GPU; by default the ranks split the
graph's oriented edges into contiguous shards of equal probe cost and
combine their result blocks with one all_gather (strong scaling), and with
--replicas every rank counts its own copy (weak scaling).  Times are CUDA
event times, the max over ranks.
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
    ap.add_argument("--mode", choices=("exact", "hybrid", "serve"), default="exact",
                    help="exact (the headline line); hybrid: one hybrid count per step with prebuilt compact "
                         "sketches (theta = gamma); serve: the serving workload at full size (20,000 requests at "
                         "the saturating rate plus two lower rates, against the sequential path)")
    ap.add_argument("--p", type=int, default=12, help="HLL precision for --mode hybrid")
    ap.add_argument("--theta", type=int, default=HYB_THETA, help="sketch / route threshold for --mode hybrid")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="launch-shape tuning for this run (core.set_count_tuning keys, e.g. bank_sort=1, hub=256); "
                         "results do not depend on it")
    ap.add_argument("--replicas", action="store_true",
                    help="N>1: every rank counts its own copy of the graph (weak scaling) instead of the default "
                         "split of one graph's edges across the ranks (strong scaling)")
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
def hub_work(g, hub_thr: int) -> dict:
    """Work of the hub pairs (table side x with d+(x) > hub_thr) of an exact
    count: pairs, probes of the raw lists (sum of d+(y)), the core (every
    vertex in some hub table side's list) and the probes left after the core
    filter (sum of plen(y)), with the byte models of the hub kernel."""
    import torch
    deg = (g.row_ptr[1:] - g.row_ptr[:-1]).long()
    eu, ev = g.edge_u.long(), g.edge_v.long()
    du, dv = deg[eu], deg[ev]
    ux = du >= dv
    x = torch.where(ux, eu, ev)
    y = torch.where(ux, ev, eu)
    lx = torch.where(ux, du, dv)
    ly = torch.where(ux, dv, du)
    hub = lx > hub_thr if hub_thr > 0 else torch.zeros_like(lx, dtype=torch.bool)
    is_hx = torch.zeros(g.n_nodes, dtype=torch.bool, device=deg.device)
    is_hx[x[hub]] = True
    core = torch.zeros(g.n_nodes, dtype=torch.bool, device=deg.device)
    core[ev[is_hx[eu]]] = True  # N+(a) = {b : (a, b) oriented}
    plen = torch.zeros(g.n_nodes, dtype=torch.int64, device=deg.device)
    plen.scatter_add_(0, eu, core[ev].long())
    n_pairs = int(hub.sum().item())
    probes = int(ly[hub].sum().item())
    fprobes = int(plen[y[hub]].sum().item())
    fquads = int(((plen[y[hub]] + 3) // 4).sum().item())
    tables = int(deg[is_hx].sum().item())
    contract = 16 * n_pairs + 4 * int((lx[hub] + ly[hub]).sum().item())
    return {"pairs": n_pairs, "probes_raw": probes, "probes_core": fprobes, "core_vertices": int(core.sum().item()),
            "hub_x": int(is_hx.sum().item()),
            # the reference's per-edge figure 16 + 4 (d+u + d+v) over the hub pairs
            "contract_bytes": contract,
            # what the kernel reads from L2 / HBM: each pair's filtered probe
            # list (16-byte quads) plus y, its row start and length (12 B),
            # each table side's list and its core indices once per segment
            "model_bytes": 16 * fquads + 12 * n_pairs + 8 * tables}


CORE16_MAX = 131070  # largest core of the packed (16-bit) hub probe lists


def hub_kernel_name(tuning: dict, core_vertices: int) -> str:
    """The hub kernel that counts with this tuning and core size (the library
    picks it on the device from the same core size)."""
    if tuning.get("packed") and core_vertices <= CORE16_MAX:
        return "hub_bitmap16_kernel"
    if tuning.get("bitmap_lg") and core_vertices + 32 <= 8 << tuning["bitmap_lg"]:
        return "hub_bitmap_kernel"
    return "hub_count_kernel"


def phase_report(pair_ms, count_ms, hub_ms, core_ms, tuning: dict) -> dict:
    """Phase times of one exact count.  With the overlap on, the hub core pass
    runs on the second stream beside the pair scatter and the short-list
    pair kernel, so it is reported apart from the serial phases."""
    out = {"pair_regroup": pair_ms, "count": count_ms, "hub_kernels": hub_ms}
    if not hub_ms:
        out["pair_kernel"] = count_ms
    elif tuning.get("overlap", 0) >= 2:  # the short-list pairs run on the second stream too
        out["hub_core_pass_beside"] = core_ms
        out["core_wait"] = count_ms - hub_ms
    elif tuning.get("overlap"):
        out["hub_core_pass_beside"] = core_ms
        out["pair_kernel_and_core_wait"] = count_ms - hub_ms
    else:
        out["hub_core_pass"] = core_ms
        out["pair_kernel"] = count_ms - hub_ms - (core_ms or 0.0)
    return out


def time_csr_build(dev, scale: int, reps: int = 3) -> dict:
    """The device CSR build (raw R-MAT endpoints in HBM -> dedup, compaction,
    orientation, sorted rows), timed with CUDA events; the reference's
    counterpart is its host loader (t_load, experiment/exp_gpu.py:264-389)."""
    import torch

    from triangle_counting_hll_b200 import core
    u, v = core.gen_rmat(scale, EDGE_FACTOR, *ABC, seed=SEED, device=dev)
    g = core.csr_from_edges(u, v)  # warm-up (workspace, lazy loading)
    ms = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        g = core.csr_from_edges(u, v)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    n_raw = int(u.numel())
    # bytes the build must move at least: the raw endpoints in, the CSR out
    io = 8 * n_raw + g.nbytes()
    best = min(ms)
    return {"ms": best, "ms_all": ms, "raw_edges": n_raw, "n_nodes": g.n_nodes, "n_edges": g.n_edges,
            "raw_edges_per_s": n_raw / (best / 1e3), "io_bytes": io, "io_gbs": io / (best / 1e3) / 1e9,
            "note": "one host sync inside (the vertex and edge counts size the outputs)"}


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
    if args.set:
        core.set_count_tuning(**{**core.get_count_tuning(),
                                 **{k: int(v) for k, v in (kv.split("=", 1) for kv in args.set)}})
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

    # ---- graph: every rank builds the same CSR
    csr_build = time_csr_build(dev, args.scale) if (world == 1 and not args.no_extras) else None
    u, v = core.gen_rmat(args.scale, EDGE_FACTOR, *ABC, seed=SEED, device=dev)
    g = core.csr_from_edges(u, v)
    del u, v
    torch.cuda.synchronize()
    deg = (g.row_ptr[1:] - g.row_ptr[:-1]).long()
    du, dv = deg[g.edge_u.long()], deg[g.edge_v.long()]
    algo_bytes = 16 * g.n_edges + 4 * int((du + dv).sum().item())
    del du, dv
    tuning = core.get_count_tuning()
    hw = hub_work(g, tuning["hub"])
    res = _lib.count_result_tensor(dev)
    if args.mode == "hybrid":
        return run_hybrid_line(args, g, dev, rank, world, barrier, max_over_ranks)

    # N > 1: the ranks split the oriented edges into contiguous ranges of
    # equal probe cost (strong scaling) unless --replicas asks for one copy
    # of the whole count per rank (weak scaling)
    sharded = world > 1 and not args.replicas
    if sharded:
        from triangle_counting_hll_b200 import dist as D
        costs = D.device_costs(g)
        lo, hi = D.shard_bounds(costs, world)[rank]
        my_u, my_v = g.edge_u[lo:hi].contiguous(), g.edge_v[lo:hi].contiguous()

        def count_mine(_lo, _hi):
            core.exact_count_tensors(g.row_ptr, g.col_idx, my_u, my_v, result=res)
            return D.result_to_tuple(_lib.read_count_result(res))
        shard = D.ShardedExact(costs, count_mine)

        def step():
            return shard.step()["exact"]
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
    kernel_ms, pair_ms, hub_ms, core_ms = [], [], [], []
    ev0.record()
    for _ in range(args.steps):
        count = step()
        ph = core.phase_times()
        kernel_ms.append(ph["count"])
        if ph["pairs"] is not None:
            pair_ms.append(ph["pairs"])
        if ph["hub"] is not None:
            hub_ms.append(ph["hub"])
            core_ms.append(ph["hub_core"])
    ev1.record()
    torch.cuda.synchronize()
    barrier()
    clk = clocks.stop()
    launches = (_lib.launch_count() - launches0) / max(args.steps, 1)
    core.set_phase_timing(False)
    ms_total = max_over_ranks(ev0.elapsed_time(ev1))
    ms_step = ms_total / args.steps
    value = (1 if sharded else world) * g.n_edges / (ms_step / 1e3)
    avg = lambda xs: (sum(xs) / len(xs)) if xs else None
    kernel_avg, hub_avg, core_avg, pair_avg = avg(kernel_ms), avg(hub_ms), avg(core_ms), avg(pair_ms)

    # ---- end to end, CSR in pinned host memory, copied to the device every
    # step: one GPU (or replicas) through the public API
    # gpu_exact_triangle_count; shards copy the CSR rows and their own edge
    # range, count it and gather the result blocks
    if sharded:
        host = [t.cpu().pin_memory() for t in (g.row_ptr, g.col_idx, my_u, my_v)]

        def e2e_count(_lo, _hi):
            d = [t.to(dev, non_blocking=True) for t in host]
            core.exact_count_tensors(*d, result=res)
            return D.result_to_tuple(_lib.read_count_result(res))
        e2e_shard = D.ShardedExact(costs, e2e_count)

        def e2e_step():
            return e2e_shard.step()["exact"]
    else:
        host = [t.cpu().pin_memory() for t in (g.row_ptr, g.col_idx, g.edge_u, g.edge_v)]

        def e2e_step():
            return gpu_exact_triangle_count(*host)[0]
    h2d = sum(t.numel() * t.element_size() for t in host)
    for _ in range(max(1, min(args.warmup, 2))):
        e2e_step()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        c_e2e = e2e_step()
    e1.record()
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1)) / args.steps
    full_count = c_e2e
    assert c_e2e == count
    del host

    peaks = load_peaks()
    kname = hub_kernel_name(tuning, hw["core_vertices"]) if hub_avg else "count_kernel<exact>"
    kms = hub_avg if hub_avg else kernel_avg
    traffic = load_traffic(f"{WORKLOAD}:{kname}") if args.scale == SCALE else None
    roof = {"bound": "hbm", "kernel": kname, "unit": "GB/s", "peak": peaks["hbm_gbs"],
            "peak_source": peaks["source"], "kernel_ms": kms}
    if traffic:
        tb = traffic["bytes_per_launch"]
        roof.update({"achieved": tb / (kms / 1e3) / 1e9, "frac": tb / (kms / 1e3) / 1e9 / peaks["hbm_gbs"],
                     "traffic": tb, "basis": "measured DRAM bytes of one launch (ncu dram__bytes_read.sum + "
                     "dram__bytes_write.sum) / CUDA-event time of the kernel", "traffic_source": traffic["source"]})
    else:
        roof.update({"achieved": None, "frac": None, "traffic": None,
                     "basis": "no ncu DRAM capture of this kernel on this workload"})
    if hub_avg:
        roof["work"] = hw
        roof["model"] = {"bytes": hw["model_bytes"], "gbs": hw["model_bytes"] / (kms / 1e3) / 1e9,
                         "note": "bytes read from L2 or HBM; most probe lists hit in L2, so this may exceed HBM"}
        roof["contract"] = {"bytes": hw["contract_bytes"],
                            "algorithmic_intensity_ratio": hw["contract_bytes"] / (kms / 1e3) / 1e9 / peaks["hbm_gbs"],
                            "note": "16 + 4 (d+u + d+v) per hub pair over peak; > 1 means the kernel reads far "
                                    "fewer bytes than both full lists per edge"}
        roof["probes_per_s"] = hw["probes_core"] / (kms / 1e3)
    issue = load_traffic(f"{WORKLOAD}:{kname}:issue") if args.scale == SCALE else None
    if issue:
        roof["issue"] = issue
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
                   "n_edges": g.n_edges, "triangles": full_count,
                   "l2": "inputs larger than L2 (CSR + edge arrays %.0f MB > 126 MB)" % (g.nbytes() / 1e6),
                   "parallelism": (f"edge shards x{world}" if sharded else f"replicas x{world}"),
                   "tuning": tuning},
        "triangles_per_s": (1 if sharded else world) * full_count / (ms_step / 1e3),
        "e2e": {"value": (1 if sharded else world) * g.n_edges / (e2e_ms / 1e3), "unit": "edges/s",
                "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": _lib.RESULT_BYTES,
                "path": ("per rank: CSR rows + own edge range H2D, shard count, 64 B D2H, all_gather" if sharded
                         else "gpu_exact_triangle_count on pinned host arrays")},
        "roofline": roof,
        "phases_ms": phase_report(pair_avg, kernel_avg, hub_avg, core_avg, tuning),
        "gpu_launches": launches,
        "clocks": clk,
    }
    if csr_build:
        line["csr_build"] = csr_build

    # the extras (hybrid sweep, batched and serving workloads) are one-GPU
    # measurements: a multi-GPU run reports the headline line only
    if not args.no_extras and world == 1:
        line["hybrid"] = hybrid_sweep(g, count, dev, exact_ms=ms_step)
        for name, mod in (("batched", "triangle_counting_hll_b200.batch"),
                          ("serving", "triangle_counting_hll_b200.serve")):
            try:
                m = __import__(mod, fromlist=["bench_entry"])
            except ImportError:
                continue
            if hasattr(m, "bench_entry"):
                line[name] = m.bench_entry(dev, quick=True)

    if rank == 0 and world == 1:
        cb, parity = cpu_baseline_and_parity(g, full_count, line.get("hybrid"), args.cpu_seconds)
        line["cpu_baseline"] = cb
        line["parity"] = parity
        if not parity["match"]:
            print(json.dumps(line), flush=True)
            raise SystemExit("parity check against the oracle failed: " + json.dumps(parity))
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
    # the dominant kernel of the three: HLL pass (on the side stream, beside
    # the others), hub pairs, other exact pairs
    hub_ms = avg.get("hub") or 0.0
    core_ms = avg.get("hub_core") or 0.0
    tuning = core.get_count_tuning()
    hname = hub_kernel_name(tuning, hub_work(g, tuning["hub"])["core_vertices"])
    cands = [("hll_edges_kernel", avg["hll"], hll_bytes), (hname, hub_ms, hub_bytes),
             ("count_kernel", avg["count"] - hub_ms - core_ms, exact_bytes - hub_bytes)]
    kname, kms, kbytes = max(cands, key=lambda c: c[1])
    traffic = load_traffic(f"rmat{args.scale}_ef16_hybrid_p{p}_theta{theta}:{kname}")
    roof = {"bound": "hbm", "kernel": kname, "peak": peaks["hbm_gbs"], "peak_source": peaks["source"],
            "unit": "GB/s", "kernel_ms": kms,
            "contract": {"bytes": kbytes, "algorithmic_intensity_ratio": kbytes / (kms / 1e3) / 1e9 / peaks["hbm_gbs"]},
            "kernels": {c[0]: {"ms": c[1], "contract_bytes": c[2]} for c in cands}}
    if traffic:
        tb = traffic["bytes_per_launch"]
        roof.update({"achieved": tb / (kms / 1e3) / 1e9, "frac": tb / (kms / 1e3) / 1e9 / peaks["hbm_gbs"],
                     "traffic": tb, "traffic_source": traffic["source"],
                     "basis": "measured DRAM bytes of one launch / CUDA-event time"})
    else:
        roof.update({"achieved": None, "frac": None, "traffic": None,
                     "basis": "no ncu DRAM capture of this kernel on this workload"})
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
        "roofline": roof,
        "gpu_launches": launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


def hybrid_sweep(g, exact_count: int, dev, exact_ms: float = None) -> dict:
    """Hybrid counts on the benched graph: the configured sweep p in
    {8, 10, 12, 14} at theta = gamma = 256 (keys p8 .. p14), plus theta =
    gamma in {64, 128} for p in {10, 12, 14} (keys g64_p10 ...), each the best
    of 3 timed calls with its relative error against the exact count; and
    the fastest point at <= 2% error with its speed-up over the exact step."""
    import torch

    from triangle_counting_hll_b200 import _lib, core
    out = {}
    res = _lib.count_result_tensor(dev)
    points = [(p, HYB_THETA, f"p{p}") for p in HYB_PS] + \
             [(p, t, f"g{t}_p{p}") for t in (64, 128) for p in (10, 12, 14)]
    for p, theta, key in points:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        slot, n_rows = core.sketch_slots(g.row_ptr, theta)
        rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, n_rows, p)
        torch.cuda.synchronize()
        build_ms = (time.perf_counter() - t0) * 1e3
        best = None
        for _ in range(3):
            s = torch.cuda.Event(enable_timing=True)
            e = torch.cuda.Event(enable_timing=True)
            s.record()
            core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot, p,
                                              theta, split_kernels=True, result=res)
            e.record()
            torch.cuda.synchronize()
            ms = s.elapsed_time(e)
            best = ms if best is None else min(best, ms)
        total, r = core.hybrid_from_result(res)
        # one more call with phase events: the HLL pass (zero masks + edge
        # estimates, on the second stream) and the exact-routed part
        core.set_phase_timing(True)
        core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot, p,
                                          theta, split_kernels=True, result=res)
        torch.cuda.synchronize()
        ph = core.phase_times()
        core.set_phase_timing(False)
        out[key] = {"theta": theta, "gamma": theta, "p": p, "ms": best, "edges_per_s": g.n_edges / (best / 1e3),
                    "sketch_build_ms": build_ms, "n_sketched": n_rows, "estimate": total,
                    "rel_err": abs(total - exact_count) / exact_count, "n_approx": int(r.n_approx),
                    "clamp_ratio": int(r.n_clamped) / max(int(r.n_approx), 1),
                    "hll_pass_ms": ph.get("hll"),
                    "exact_part_ms": (ph.get("pairs") or 0.0) + (ph.get("count") or 0.0)}
        if exact_ms:
            out[key]["speedup_vs_exact"] = exact_ms / best
        del rows, slot
    ok = [(v["ms"], k) for k, v in out.items() if isinstance(v, dict) and v["rel_err"] <= 0.02]
    if ok:
        ms, k = min(ok)
        out["best_le_2pct"] = {"key": k, "ms": ms, "rel_err": out[k]["rel_err"],
                               "speedup_vs_exact": (exact_ms / ms) if exact_ms else None}
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


HYB_RTOL = 1e-6  # hybrid estimates vs the FP64 oracle (relative)


def cpu_baseline_and_parity(g, exact_count: int, sweep, budget_s: float):
    """The oracle (C restatement of the reference's counting loop, all host
    threads) over ALL oriented edges of the benched graph: its time is the CPU
    baseline and its count must equal the GPU's.  With the hybrid sweep, the
    p = 12 estimate (theta = gamma = 256) is also checked against the oracle's
    FP64 evaluation of the reference estimator within 1e-6 relative, and so
    are its routing stats.  budget_s only caps the extra hybrid check."""
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
    t0 = time.perf_counter()
    want = int(O.exact_count(rp, ci, eu, ev, nthreads=cores))
    dt = time.perf_counter() - t0
    cb = {"value": E / dt, "unit": "edges/s", "cores": cores, "kind": "port",
          "sample": f"all {E} oriented edges of the benched graph ({dt:.1f} s), oracle exact count (C port of "
                    f"src/exact.py's merge / binary-search loop, OpenMP)"}
    parity = {"oracle_exact": want, "gpu_exact": int(exact_count), "exact_match": want == int(exact_count)}
    ok = parity["exact_match"]
    p12 = (sweep or {}).get("p12")
    if p12 is not None:
        t1 = time.perf_counter()
        slot, rows = O.build_sketches_compact(rp.astype(np.int64), ci.astype(np.int64), HYB_THETA, 12)
        otot, ost, _ = O.hybrid_count(rp, ci, eu, ev, g.degrees.cpu().numpy(), slot, rows, 12, HYB_THETA,
                                      nthreads=cores)
        rel = abs(p12["estimate"] - otot) / max(abs(otot), 1.0)
        parity["hybrid_p12"] = {"oracle": otot, "gpu": p12["estimate"], "rel_diff": rel, "rtol": HYB_RTOL,
                                "oracle_n_approx": ost["n_approx"], "gpu_n_approx": p12["n_approx"],
                                "oracle_s": time.perf_counter() - t1}
        ok = ok and rel <= HYB_RTOL and ost["n_approx"] == p12["n_approx"]
    parity["match"] = bool(ok)
    return cb, parity


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


def run_serve_line(args):
    """--mode serve: one GPU, the full serving workload; metric graphs/s of
    the server at the saturating rate, with every rate's p50 / p99 beside the
    sequential path's."""
    import torch

    from triangle_counting_hll_b200 import serve
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    clocks = ClockSampler(0)
    clocks.start()
    out = serve.bench_c5(dev)
    clk = clocks.stop()
    sat = out["rate_2000"]
    line = {"metric": "graphs/s", "value": sat["server"]["graphs_per_s"], "unit": "graphs/s", "n_gpus": 1,
            "steps": sat["requests"], "warmup": 0, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "int32+u8", "data": "synthetic",
            "config": {"workload": "serving_c5", "detail": out["workload"]},
            "serving": out, "clocks": clk}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.mode == "serve":
        run_serve_line(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
