"""Pin the CPU oracle against outputs recorded from the reference itself
(tests/golden/make_golden.py ran src/hll.py, src/exact.py, src/hybrid.py,
src/graph.py, src/gpu_graph.py and cpu_exp/triangle_hll_experiment.py)."""
from __future__ import annotations

import hashlib

import numpy as np
import pytest

GRAPHS = ["k4_tail", "er_2000", "rmat10", "rmat12", "lattice_40"]


def regen(O, name):
    if name == "k4_tail":
        return (np.array([0, 0, 0, 1, 1, 2, 3, 4], np.int32), np.array([1, 2, 3, 2, 3, 3, 4, 5], np.int32))
    if name == "er_2000":
        return O.gen_er(2000, 12000, 7)
    if name == "rmat10":
        return O.gen_rmat(10, 16, 0.57, 0.19, 0.19, 3)
    if name == "rmat12":
        return O.gen_rmat(12, 16, 0.57, 0.19, 0.19, 1)
    if name == "lattice_40":
        return O.gen_lattice(40, 40, 0.3, 0.05, 0)
    raise KeyError(name)


def test_hash64_matches_reference(golden, oracle):
    arrays, _ = golden
    out = oracle.hash64(arrays["hash_in"])
    assert np.array_equal(out, arrays["hash_out"])
    assert int(out[0]) == 0  # _hash64(0) == 0 (id 0 lands in register 0 with rank 65-p)


@pytest.mark.parametrize("p", list(range(4, 17)))
def test_registers_and_estimates(golden, oracle, p):
    arrays, meta = golden
    for name in ("ids_0_100", "ids_0_5000", "rand_300", "rand_20000", "single_0"):
        regs = oracle.sketch(p, arrays[f"set_{name}"])
        assert np.array_equal(regs, arrays[f"regs_{name}_p{p}"]), (name, p)
        e = oracle.estimate(regs)
        ref = meta["estimates"][f"{name}_p{p}"]
        # Z keeps numpy's pairwise summation order; the linear-counting log is
        # libm's where the reference used numpy's: equal to within 2 ulp
        assert e == pytest.approx(ref, rel=5e-16, abs=0), (name, p, e, ref)


def test_union_estimates(golden, oracle):
    arrays, meta = golden
    for key, ref in meta["unions"].items():
        p = int(key.split("_")[0][1:])
        e = oracle.union_estimate(arrays[f"ua_{key}"], arrays[f"ub_{key}"], p)
        assert e == pytest.approx(ref, rel=5e-16, abs=0), (key, e, ref)
    assert meta["union_p_mismatch_raises"] is True


@pytest.mark.parametrize("gname", GRAPHS)
def test_csr_and_exact(golden, oracle, gname):
    arrays, meta = golden
    case = meta["graphs"][gname]
    u, v = regen(oracle, gname)
    if gname == "k4_tail":
        assert np.array_equal(u, arrays["g_k4_tail_raw_u"]) and np.array_equal(v, arrays["g_k4_tail_raw_v"])
    g = oracle.csr_build(u, v)
    assert g["n_nodes"] == case["n_nodes"] and g["n_edges"] == case["n_edges"]
    for nm in ("row_ptr", "col_idx", "degrees", "node_ids", "edge_u", "edge_v"):
        a = np.ascontiguousarray(g[nm], dtype=np.int32)
        assert hashlib.sha256(a.tobytes()).hexdigest() == case["sha256"][nm], nm
    cnt = oracle.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], nthreads=2)
    assert cnt == case["exact"]
    cnt1 = oracle.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], nthreads=1, r=1e9)
    assert cnt1 == case["exact"]


@pytest.mark.parametrize("gname", GRAPHS)
def test_hybrid_matches_reference(golden, oracle, gname):
    arrays, meta = golden
    case = meta["graphs"][gname]
    u, v = regen(oracle, gname)
    g = oracle.csr_build(u, v)
    rp64 = g["row_ptr"].astype(np.int64)
    comp_keys = np.arange(g["n_nodes"], dtype=np.int64)  # compacted ids (Q2)
    for theta, p in ((8, 8), (16, 10), (32, 12), (4, 4)):
        key = f"t{theta}_p{p}"
        for suffix, th in (("", theta), ("_fallback", 2 * theta)):
            slot, rows = oracle.build_sketches_compact(rp64, comp_keys[g["col_idx"]], th, p)
            tot, st, det = oracle.hybrid_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], g["degrees"],
                                               slot, rows, p, theta, nthreads=1, details=True)
            ref = case["hybrid"][key + suffix]
            # sequential FP64 in the reference's edge order (per-edge logs may
            # differ from numpy's by an ulp)
            assert tot == pytest.approx(ref["total"], rel=1e-13), (key + suffix, tot, ref["total"])
            for k in ("n_edges", "n_approx", "n_exact", "n_fallback", "n_clamped"):
                assert st[k] == ref["stats"][k], (key + suffix, k)
            if suffix == "" and f"g_{gname}_{key}_s_hat" in arrays:
                np.testing.assert_allclose(det[0], arrays[f"g_{gname}_{key}_s_hat"], rtol=1e-13, atol=1e-11)
                assert np.array_equal(det[2], arrays[f"g_{gname}_{key}_method"])
    # sketches over the original ids (src/hybrid.py:39)
    ids = g["node_ids"].astype(np.int64)
    slot, rows = oracle.build_sketches_compact(rp64, ids[g["col_idx"]], 8, 8)
    if f"g_{gname}_origsk_keys" in arrays:
        keys = arrays[f"g_{gname}_origsk_keys"]
        ref_regs = arrays[f"g_{gname}_origsk_regs"]
        pos = np.searchsorted(ids, keys)
        got = rows.reshape(-1, 256)[slot[pos]]
        assert np.array_equal(got, ref_regs)
    tot, st, _ = oracle.hybrid_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], g["degrees"], slot, rows,
                                     8, 8, nthreads=1)
    ref = case["hybrid"]["orig_ids_t8_p8"]
    assert tot == pytest.approx(ref["total"], rel=1e-12)
    assert st["n_approx"] == ref["stats"]["n_approx"] and st["n_clamped"] == ref["stats"]["n_clamped"]


def test_hybrid_threads_agree(golden, oracle):
    """Multi-threaded oracle: same stats, total within FP64 reordering."""
    u, v = regen(oracle, "rmat12")
    g = oracle.csr_build(u, v)
    slot, rows = oracle.build_sketches_compact(g["row_ptr"].astype(np.int64),
                                               np.arange(g["n_nodes"], dtype=np.int64)[g["col_idx"]], 16, 10)
    t1, s1, _ = oracle.hybrid_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], g["degrees"], slot, rows,
                                    10, 16, nthreads=1)
    t4, s4, _ = oracle.hybrid_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"], g["degrees"], slot, rows,
                                    10, 16, nthreads=4)
    assert s1 == s4
    assert t4 == pytest.approx(t1, rel=1e-12)


def test_cpu_exp_variant(golden, oracle):
    arrays, meta = golden
    for key, ref in meta["cpu_exp"].items():
        p = int(key.rsplit("_p", 1)[1])
        off = arrays[f"cx_{key}_offsets"]
        adj = arrays[f"cx_{key}_adj"]
        n = len(off) - 1
        regs = oracle.cx_build_registers(off, adj, n, p, 1)
        assert np.array_equal(regs, arrays[f"cx_{key}_regs"]), key
        e = arrays[f"cx_{key}_edges"].reshape(-1, 2)
        od = arrays[f"cx_{key}_outdeg"]
        for thr in ("0", "4", "16", "1000000000"):
            out = oracle.cx_hybrid(off, adj, e[:, 0], e[:, 1], od, regs, p, int(thr))
            exp = ref[thr]
            assert out[1:3] == (int(exp[1]), int(exp[2])) and out[5] == int(exp[5]), (key, thr)
            assert out[0] == pytest.approx(exp[0], rel=1e-12, abs=1e-9), (key, thr)
        pure = oracle.cx_hybrid(off, adj, e[:, 0], e[:, 1], od, regs, p, -1)
        assert pure[0] == pytest.approx(ref["pure"][0], rel=1e-12) and pure[5] == ref["pure"][1]


def test_generators_deterministic(oracle):
    a = oracle.gen_rmat(8, 4, 0.57, 0.19, 0.19, 5)
    b = oracle.gen_rmat(8, 4, 0.57, 0.19, 0.19, 5)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    u, v = oracle.gen_lattice(30, 20, 0.3, 0.05, 1)
    keep = u != v
    # permutation is a bijection: ids stay within [0, R*C)
    assert u[keep].max() < 600 and v[keep].min() >= 0
    perm = [oracle.gen_perm(x, 600, 1) for x in range(600)]
    assert sorted(perm) == list(range(600))


def test_known_answers(oracle):
    """K_n has C(n,3) triangles; a bipartite graph and a star have none."""
    for n in (3, 4, 7, 20):
        iu, iv = np.triu_indices(n, 1)
        g = oracle.csr_build(iu.astype(np.int32), iv.astype(np.int32))
        assert oracle.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"]) == n * (n - 1) * (n - 2) // 6
    a, b = np.meshgrid(np.arange(10), np.arange(10, 25))
    g = oracle.csr_build(a.ravel().astype(np.int32), b.ravel().astype(np.int32))
    assert oracle.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"]) == 0
    g = oracle.csr_build(np.zeros(50, np.int32), np.arange(1, 51, dtype=np.int32))
    assert oracle.exact_count(g["row_ptr"], g["col_idx"], g["edge_u"], g["edge_v"]) == 0
