"""Batched counting (many graphs in one launch) and the degree-keyed autotuner.

GPU tests check that per-graph results of the batched launch are bit-identical
to counting each graph alone (exact counts, hybrid fixed-point totals and
stats) and to the oracle; CPU tests cover the host-side workload generator
and the autotuner's signature.
"""
from __future__ import annotations

import numpy as np
import pytest


def test_c4_specs_distribution():
    from triangle_counting_hll_b200.batch import c4_specs
    specs = c4_specs(2048)
    ns = np.array([s.n for s in specs])
    assert len(specs) == 2048 and ns.min() >= 500 and ns.max() <= 500000
    assert 4000 < np.median(ns) < 6000
    assert [s.kind for s in specs[:4]] == ["er", "chung_lu", "er", "chung_lu"]
    assert [s.seed for s in specs[:3]] == [0, 1, 2]
    assert c4_specs(16) == c4_specs(16)  # deterministic


def test_autotune_signature_is_shape_key():
    from triangle_counting_hll_b200.autotune import signature
    h = np.zeros(32, dtype=np.int64)
    h[:4] = [100, 50, 20, 5]
    s1 = signature({"log_hist": h})
    s2 = signature({"log_hist": h * 10})  # same shape, 10x the vertices
    assert s1 == s2 and s1.startswith("top3:")
    h2 = h.copy()
    h2[10] = 3
    assert signature({"log_hist": h2}) != s1
    assert signature({"log_hist": np.zeros(32)}) == "empty"


def _small_batch(dev, n_graphs=40):
    import torch
    from triangle_counting_hll_b200 import batch as B
    specs = B.c4_specs(n_graphs, median=800, sigma=0.8, lo=50, hi=5000, seed_base=11)
    graphs = [B.generate(s, dev) for s in specs]
    items = [(u, v, s.n) for (u, v), s in zip(graphs, specs)]
    # edge cases: an empty graph, a single edge, a triangle, a dense clique
    z = torch.zeros(0, dtype=torch.int32, device=dev)
    items.insert(3, (z, z, 10))
    items.insert(7, (torch.tensor([4], dtype=torch.int32, device=dev), torch.tensor([2], dtype=torch.int32,
                                                                                    device=dev), 5))
    items.append((torch.tensor([0, 1, 2], dtype=torch.int32, device=dev),
                  torch.tensor([1, 2, 0], dtype=torch.int32, device=dev), 3))
    iu, iv = np.triu_indices(60, 1)
    items.append((torch.from_numpy(iu.astype(np.int32)).to(dev), torch.from_numpy(iv.astype(np.int32)).to(dev), 60))
    return items


@pytest.mark.gpu
def test_batched_exact_bit_exact_vs_one_at_a_time(tchll, oracle):
    import torch
    from triangle_counting_hll_b200 import batch as B
    from triangle_counting_hll_b200 import core
    dev = torch.device("cuda", 0)
    items = _small_batch(dev)
    bt = B.GraphBatch.from_edge_lists(items, device=dev)
    got = bt.exact_counts()
    csrs = [core.csr_from_edges(u, v, device=dev) for u, v, _ in items]
    ref = B.plain_exact_counts(csrs)
    assert np.array_equal(got, ref)
    # and against the oracle, graph by graph
    for (u, v, _), c in zip(items, got):
        og = oracle.csr_build(u.cpu().numpy(), v.cpu().numpy())
        assert c == oracle.exact_count(og["row_ptr"], og["col_idx"], og["edge_u"], og["edge_v"])
    assert got[-1] == 60 * 59 * 58 // 6 and got[-2] == 1 and got[3] == 0


@pytest.mark.gpu
def test_batched_hub_segments_go_to_their_graph(tchll, oracle):
    """Graphs with long forward lists (cliques of 300 and 400 vertices, and
    an R-MAT graph) between small ones: the hub kernel's segments publish
    into the right graph's result (exact and hybrid), equal to one graph at a
    time and to the oracle."""
    import torch
    from triangle_counting_hll_b200 import batch as B
    from triangle_counting_hll_b200 import core
    dev = torch.device("cuda", 0)
    items = _small_batch(dev, 12)
    for k, pos in ((300, 2), (400, 9)):
        iu, iv = np.triu_indices(k, 1)
        items.insert(pos, (torch.from_numpy((iu * 7).astype(np.int32)).to(dev),
                           torch.from_numpy((iv * 7).astype(np.int32)).to(dev), 7 * k))
    u, v = core.gen_rmat(14, 32, 0.57, 0.19, 0.19, seed=9, device=dev)
    items.insert(5, (u, v, 1 << 14))
    bt = B.GraphBatch.from_edge_lists(items, device=dev)
    csrs = [core.csr_from_edges(a, b, device=dev) for a, b, _ in items]
    assert max(int(c.degrees.max()) for c in csrs if c.n_nodes) > core.get_count_tuning()["hub"]
    got = bt.exact_counts()
    assert np.array_equal(got, B.plain_exact_counts(csrs))
    assert got[2] == 300 * 299 * 298 // 6 and got[10] == 400 * 399 * 398 // 6
    og = oracle.csr_build(u.cpu().numpy(), v.cpu().numpy())
    assert got[5] == oracle.exact_count(og["row_ptr"], og["col_idx"], og["edge_u"], og["edge_v"])
    tot, st = bt.hybrid_counts(64, 64, 10)
    rtot, rst = B.plain_hybrid_counts(csrs, B.plain_sketches(csrs, 64, 10), 64, 10)
    assert np.array_equal(tot, rtot)
    for k in rst:
        assert np.array_equal(st[k], rst[k]), k
    for i in (2, 5, 10):  # the 300-clique, the R-MAT graph, the 400-clique
        a, b, _ = items[i]
        otot, ost = _oracle_hybrid(oracle, a.cpu().numpy(), b.cpu().numpy(), 64, 64, 10)
        assert tot[i] == pytest.approx(otot, rel=1e-9) and st["n_approx"][i] == ost["n_approx"], i


def _oracle_hybrid(oracle, u, v, theta, gamma, p):
    """The oracle's hybrid total and stats of one graph given by its raw
    endpoint arrays (CSR build, compact sketches of rows >= theta, route by
    gamma)."""
    og = oracle.csr_build(u, v)
    if og["n_edges"] == 0:
        return 0.0, {"n_approx": 0, "n_exact": 0, "n_fallback": 0, "n_clamped": 0}
    oslot, orows = oracle.build_sketches_compact(og["row_ptr"].astype(np.int64), og["col_idx"].astype(np.int64),
                                                 theta, p)
    otot, ost, _ = oracle.hybrid_count(og["row_ptr"], og["col_idx"], og["edge_u"], og["edge_v"], og["degrees"],
                                       oslot, orows, p, gamma)
    return otot, ost


@pytest.mark.gpu
@pytest.mark.parametrize("theta,p", [(8, 10), (16, 8), (4, 12)])
def test_batched_hybrid_bit_exact_vs_one_at_a_time(tchll, oracle, theta, p):
    import torch
    from triangle_counting_hll_b200 import batch as B
    from triangle_counting_hll_b200 import core
    dev = torch.device("cuda", 0)
    items = _small_batch(dev)
    bt = B.GraphBatch.from_edge_lists(items, device=dev)
    tot, st = bt.hybrid_counts(theta, theta, p)
    csrs = [core.csr_from_edges(u, v, device=dev) for u, v, _ in items]
    rtot, rst = B.plain_hybrid_counts(csrs, B.plain_sketches(csrs, theta, p), theta, p)
    assert np.array_equal(tot, rtot)  # fixed-point sums: bit-identical
    for k in rst:
        assert np.array_equal(st[k], rst[k]), k
    assert st["n_approx"].sum() > 0  # the HLL path ran
    # and each graph's total and stats against the oracle's FP64 evaluation of
    # the reference estimator on that graph alone
    for i, (u, v, _) in enumerate(items):
        otot, ost = _oracle_hybrid(oracle, u.cpu().numpy(), v.cpu().numpy(), theta, theta, p)
        assert tot[i] == pytest.approx(otot, rel=1e-9, abs=1e-9), i
        assert (st["n_approx"][i], st["n_exact"][i], st["n_clamped"][i]) == \
            (ost["n_approx"], ost["n_exact"], ost["n_clamped"]), i
    ex = bt.exact_counts()
    assert np.array_equal(st["n_approx"] + st["n_exact"], np.array([c.n_edges for c in csrs]))
    assert (tot[st["n_approx"] == 0] == ex[st["n_approx"] == 0]).all()


@pytest.mark.gpu
def test_captured_batch_replays_and_tuning(tchll):
    import torch
    from triangle_counting_hll_b200 import autotune, batch as B, core
    dev = torch.device("cuda", 0)
    items = _small_batch(dev, 24)
    bt = B.GraphBatch.from_edge_lists(items, device=dev)
    ref = bt.exact_counts()
    base = core.get_count_tuning()
    try:
        cfg = autotune.tune_batch(bt, autotune.Autotuner())
        assert cfg["key"].startswith("top")
        cap = B.CapturedBatch(bt)
        a = cap.exact_counts()
        b = cap.exact_counts()
        assert np.array_equal(a, ref) and np.array_equal(b, ref)
        caph = B.CapturedBatch(bt, hybrid=(8, 8, 10))
        t1, s1 = caph.hybrid_counts()
        t2, s2 = caph.hybrid_counts()
        t3, s3 = bt.hybrid_counts(8, 8, 10)
        assert np.array_equal(t1, t2) and np.array_equal(t1, t3)
    finally:
        core.set_count_tuning(**base)


@pytest.mark.gpu
def test_degree_stats_match_numpy(tchll):
    import torch
    from triangle_counting_hll_b200 import autotune, core
    dev = torch.device("cuda", 0)
    u, v = core.gen_rmat(14, 16, 0.57, 0.19, 0.19, seed=3, device=dev)
    g = core.csr_from_edges(u, v)
    st = autotune.degree_stats(g.row_ptr)
    d = np.diff(g.row_ptr.cpu().numpy().astype(np.int64))
    dp = d[d > 0]
    assert st["active"] == len(dp) and st["sum"] == dp.sum() and st["sumsq"] == (dp * dp).sum()
    assert st["max"] == dp.max() and st["min"] == dp.min()
    ref = np.bincount(np.floor(np.log2(dp)).astype(int), minlength=32)[:32]
    assert np.array_equal(st["log_hist"], ref)


# ------------------------------------------------------------------ serving
def test_c5_requests_shape():
    from triangle_counting_hll_b200.serve import c5_requests, estimate_bytes
    reqs = c5_requests(2000, 100.0, seed=1, repeat_frac=0.2)
    arr = np.array([r.arrival for r in reqs])
    assert (np.diff(arr) >= 0).all() and 15 < arr[-1] < 25  # ~2000 / 100 s
    sc = np.array([r.scale for r in reqs])
    ef = np.array([r.edge_factor for r in reqs])
    assert sc.min() >= 12 and sc.max() <= 20 and ef.min() >= 8 and ef.max() <= 32
    frac = np.mean([r.mode == "hybrid" for r in reqs])
    assert 0.45 < frac < 0.55
    keys = [r.key for r in reqs]
    assert len(set(keys)) < len(keys)  # repeats present
    assert estimate_bytes(reqs[0]) > 40 * reqs[0].raw_edges()


def _serve_mix(dev, n=60, rate=400.0, budget=120e9, scale_range=(8, 12), repeat=0.3, big_edges=1 << 20):
    from triangle_counting_hll_b200 import serve as S
    reqs = S.c5_requests(n, rate, seed=5, scale_range=scale_range, ef_range=(4, 16), repeat_frac=repeat,
                         p=10, theta=16)
    srv = S.Server(dev, budget_bytes=budget, max_batch=32, big_edges=big_edges)
    return reqs, srv, srv.serve(reqs)


@pytest.mark.gpu
def test_server_results_same_alone_and_in_the_mix(tchll, oracle):
    import torch
    from triangle_counting_hll_b200 import serve as S
    dev = torch.device("cuda", 0)
    # graphs of >= 2^14 raw edges take the single-graph path, smaller ones are
    # batched (a burst of arrivals, so that ticks hold several small graphs)
    reqs, srv, got = _serve_mix(dev, rate=1e5, big_edges=1 << 14)
    assert len(got) == len(reqs) and all(c.error is None for c in got)
    assert srv.stats["single_launches"] > 0 and srv.stats["batched_launches"] > 0
    assert srv.stats["ticks"] < len(reqs)          # queries were batched
    assert max(srv.stats["batch_sizes"]) > 1
    assert srv.stats["cache_hits"] > 0             # repeat queries reused resident graphs
    for r, c in zip(sorted(reqs, key=lambda r: r.rid), got):
        alone = S.answer_alone(r, dev)
        assert c.value == alone.value and c.stats == alone.stats, r  # bit-identical, exact and hybrid
        # and against the oracle on the same request graph (the oracle's
        # generator draws the same edges as the device one)
        ou, ov = oracle.gen_rmat(r.scale, r.edge_factor, *S.RMAT_ABC, r.seed)
        if r.mode == "exact":
            og = oracle.csr_build(ou, ov)
            assert c.value == oracle.exact_count(og["row_ptr"], og["col_idx"], og["edge_u"], og["edge_v"]), r
        else:
            otot, ost = _oracle_hybrid(oracle, ou, ov, r.theta, r.gamma, r.p)
            assert c.value == pytest.approx(otot, rel=1e-9, abs=1e-9), r
            assert (c.stats["n_approx"], c.stats["n_clamped"]) == (ost["n_approx"], ost["n_clamped"]), r


@pytest.mark.gpu
def test_server_admission_budget_and_rejection(tchll):
    import torch
    from triangle_counting_hll_b200 import serve as S
    dev = torch.device("cuda", 0)
    small = S.Request(0, 0.0, 8, 4, 1, "exact")
    huge = S.Request(1, 0.0, 20, 32, 2, "hybrid")
    budget = 2 * S.estimate_bytes(small)
    srv = S.Server(dev, budget_bytes=budget)
    got = srv.serve([small, huge, S.Request(2, 0.01, 8, 4, 3, "exact")])
    assert got[0].error is None and got[2].error is None
    assert got[1].error is not None and "budget" in got[1].error   # host-side admission failure
    assert srv.stats["rejected"] == 1 and srv.resident_bytes <= budget
    assert got[0].value == S.answer_alone(small, dev).value
