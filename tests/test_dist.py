"""Multi-process (world size 2, gloo, CPU) tests of the sharded count: the
edge partition, the exact combination of per-rank partials, and a failing
rank surfacing as an error on the others instead of a hang.  The per-rank
counter here is the CPU oracle (test infrastructure); on GPUs the same code
runs with the libtchll counters (dist.gpu_exact_range / gpu_hybrid_range)."""
from __future__ import annotations

import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_shard_bounds_cover_and_balance():
    from triangle_counting_hll_b200.dist import shard_bounds, shard_graphs
    rng = np.random.default_rng(0)
    c = rng.integers(1, 1000, 10000)
    for world in (1, 2, 3, 8):
        b = shard_bounds(c, world)
        assert b[0][0] == 0 and b[-1][1] == len(c)
        assert all(b[i][1] == b[i + 1][0] for i in range(world - 1))
        loads = [c[lo:hi].sum() for lo, hi in b]
        assert max(loads) - min(loads) <= 2 * c.max()
    assert shard_bounds([], 3) == [(0, 0)] * 3
    assert shard_bounds([5], 4)[-1] == (1, 1) or sum(hi - lo for lo, hi in shard_bounds([5], 4)) == 1
    parts = shard_graphs([10, 1, 7, 7, 3], 2)
    assert sorted(parts[0] + parts[1]) == [0, 1, 2, 3, 4]


def test_combine_is_exact():
    from triangle_counting_hll_b200.dist import combine
    big = (1 << 64) - 5
    parts = [(3, big, 0, 1, 2, 0, 0, 0), (4, 10, 1, 1, 2, 1, 1, 2)]
    out = combine(parts)
    fx = big + 10 + (1 << 64)
    assert out["exact"] == 7 and out["hll_fx"] == fx
    assert out["total"] == ((7 << 32) + fx) / 4294967296
    assert out["n_approx"] == 2 and out["n_exact"] == 4 and out["status"] == 2


def _worker(rank, world, port, q, fail_rank):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist

    from oracle import oracle as O
    from triangle_counting_hll_b200 import dist as D
    try:
        dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=8))
        u, v = O.gen_rmat(11, 16, 0.57, 0.19, 0.19, 3)
        g = O.csr_build(u, v)
        d = g["degrees"]
        costs = D.edge_costs(d[g["edge_u"]], d[g["edge_v"]])

        def count_range(lo, hi):
            if rank == fail_rank:
                raise RuntimeError("planted failure on this rank")
            c = O.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"][lo:hi], g["edge_v"][lo:hi], nthreads=1)
            return (c, 0, 0, 0, hi - lo, 0, 0, 0)

        out = D.sharded_count(len(g["edge_u"]), costs, count_range)
        full = O.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], nthreads=1)
        ok = out["exact"] == full and out["n_exact"] == len(g["edge_u"])
        # the per-step helper bench.py's multi-GPU line uses (strong scaling:
        # one graph's edges split across the ranks), stepped twice
        shard = D.ShardedExact(costs, count_range)
        for _ in range(2):
            st = shard.step()
            ok = ok and st["exact"] == full and st["n_exact"] == len(g["edge_u"])
        bounds = D.shard_bounds(costs, world)
        ok = ok and (shard.lo, shard.hi) == bounds[rank] and bounds[0][0] == 0 and bounds[-1][1] == len(costs)
        q.put((rank, "ok", ok))
    except Exception as exc:  # reported to the parent, never hangs
        q.put((rank, "error", type(exc).__name__))
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def _run(world, fail_rank=-1, timeout=60):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q, fail_rank)) for r in range(world)]
    for p in procs:
        p.start()
    out = {}
    for _ in range(world):
        r, status, val = q.get(timeout=timeout)
        out[r] = (status, val)
    for p in procs:
        p.join(timeout=30)
        if p.is_alive():
            p.kill()
    return out


def test_two_rank_sharded_exact_count_gloo():
    out = _run(2)
    assert out == {0: ("ok", True), 1: ("ok", True)}


def test_failing_rank_raises_on_peers_not_hang():
    out = _run(2, fail_rank=1)
    assert out[1] == ("error", "RuntimeError")
    assert out[0][0] == "error"  # the gather fails (peer gone / timeout) instead of hanging


@pytest.mark.gpu
def test_gpu_shards_combine_to_the_full_count(tchll, oracle):
    """The per-rank GPU counters of each shard, combined, equal the full
    count (ranks emulated one after another on one GPU; no rank waits on
    another)."""
    import torch
    from triangle_counting_hll_b200 import core, dist as D
    dev = torch.device("cuda", 0)
    u, v = core.gen_rmat(16, 16, 0.57, 0.19, 0.19, seed=4, device=dev)
    g = core.csr_from_edges(u, v)
    costs = D.device_costs(g)
    full_res, _ = core.exact_count_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v)
    full = core.exact_from_result(full_res)
    slot, nr = core.sketch_slots(g.row_ptr, 32)
    rows = core.build_sketches_compact_tensors(g.row_ptr, g.col_idx, slot, nr, 10)
    hres, _ = core.hybrid_count_compact_tensors(g.row_ptr, g.col_idx, g.edge_u, g.edge_v, g.degrees, rows, slot,
                                                10, 32)
    htot, hr = core.hybrid_from_result(hres)
    for world in (2, 3, 8):
        bounds = D.shard_bounds(costs, world)
        ex = D.gpu_exact_range(g)
        out = D.combine([ex(lo, hi) for lo, hi in bounds])
        assert out["exact"] == full and out["n_exact"] == g.n_edges
        hy = D.gpu_hybrid_range(g, rows, slot, 10, 32)
        out = D.combine([hy(lo, hi) for lo, hi in bounds])
        assert out["total"] == htot  # fixed-point partials add exactly
        assert out["n_approx"] == int(hr.n_approx) and out["n_clamped"] == int(hr.n_clamped)
