"""Generate golden fixtures by running the reference implementation itself.

Run in a container where the reference checkout is present (read-only):

    python tests/golden/make_golden.py /path/to/triangle_counting_hll

It imports the reference's pure-Python modules (src/hll.py, src/exact.py,
src/hybrid.py, src/graph.py, src/gpu_graph.py) and its cpu_exp script (from
a temporary copy, since Numba caching writes next to the source), feeds them
inputs made by the oracle's seeded generators, and records their outputs in
``tests/golden/golden.npz`` + ``tests/golden/golden.json``.  The tests never
import the reference; they compare the oracle and the CUDA path with these
recorded outputs.
"""
from __future__ import annotations

import hashlib
import importlib.util
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.dont_write_bytecode = True

from oracle import oracle as O  # noqa: E402


def _import_reference(ref_root: str):
    sys.path.insert(0, ref_root)
    import src.exact as exact  # noqa: F401
    import src.gpu_graph as gpu_graph
    import src.graph as graph
    import src.hll as hll
    import src.hybrid as hybrid
    return exact, graph, gpu_graph, hll, hybrid


def _import_cpu_exp(ref_root: str):
    tmp = tempfile.mkdtemp(prefix="tchll_cpuexp_")
    dst = os.path.join(tmp, "triangle_hll_experiment.py")
    shutil.copy(os.path.join(ref_root, "cpu_exp", "triangle_hll_experiment.py"), dst)
    spec = importlib.util.spec_from_file_location("triangle_hll_experiment", dst)
    mod = importlib.util.module_from_spec(spec)
    sys.modules["triangle_hll_experiment"] = mod
    spec.loader.exec_module(mod)
    return mod


def edges_from_raw(u, v):
    """Canonical undirected edge set, as src/graph.py:load_edgelist builds."""
    s = set()
    for a, b in zip(u.tolist(), v.tolist()):
        if a != b:
            s.add((min(a, b), max(a, b)))
    return s


def compacted_forward_adj(fwd):
    """Q2 convention: re-key forward_adj by the rank of each id (what the GPU
    path hashes, experiment/exp_gpu.py:371-377)."""
    ids = sorted(fwd.keys())
    idx = {x: i for i, x in enumerate(ids)}
    return {idx[k]: np.array([idx[int(x)] for x in fwd[k]], dtype=np.int64) for k in ids}


def main(ref_root: str) -> None:
    exact, graph, gpu_graph, hll, hybrid = _import_reference(ref_root)
    arrays = {}
    meta = {"reference_root_basename": os.path.basename(os.path.abspath(ref_root))}

    # ---- hash (src/hll.py:13-19), including id 0 (Q1) and wide values
    ids = np.concatenate([np.arange(0, 2048, dtype=np.int64),
                          np.array([2**31 - 1, 2**32, 2**40 + 17, 2**62, -1, -2**63], dtype=np.int64)])
    arrays["hash_in"] = ids
    arrays["hash_out"] = np.array([hll._hash64(int(x)) for x in ids], dtype=np.uint64)

    # ---- registers + estimates for every p, several set sizes
    rng = np.random.default_rng(12345)
    sets = {
        "ids_0_100": np.arange(0, 100, dtype=np.int64),
        "ids_0_5000": np.arange(0, 5000, dtype=np.int64),
        "rand_300": rng.integers(0, 2**40, 300, dtype=np.int64),
        "rand_20000": rng.integers(0, 2**31, 20000, dtype=np.int64),
        "single_0": np.array([0], dtype=np.int64),
    }
    est = {}
    for name, arr in sets.items():
        arrays[f"set_{name}"] = arr
        for p in range(4, 17):
            h = hll.HLL(p=p)
            h.add_array(arr)
            arrays[f"regs_{name}_p{p}"] = h.registers.copy()
            est[f"{name}_p{p}"] = h.estimate()
    meta["estimates"] = est

    # ---- union estimates, including LC-boundary sizes (E ~ 2.5 m)
    unions = {}
    for p in (4, 6, 8, 10, 12, 14, 16):
        m = 1 << p
        for frac in (0.5, 2.2, 2.5, 2.8, 6.0):
            k = max(1, int(frac * m))
            a = rng.integers(0, 2**31, k, dtype=np.int64)
            b = np.concatenate([a[: k // 2], rng.integers(0, 2**31, k - k // 2, dtype=np.int64)])
            ha, hb = hll.HLL(p=p), hll.HLL(p=p)
            ha.add_array(a)
            hb.add_array(b)
            key = f"p{p}_f{frac}"
            arrays[f"ua_{key}"] = ha.registers.copy()
            arrays[f"ub_{key}"] = hb.registers.copy()
            unions[key] = hll.union_estimate(ha, hb)
    meta["unions"] = unions
    try:
        hll.union_estimate(hll.HLL(p=8), hll.HLL(p=10))
        meta["union_p_mismatch_raises"] = False
    except ValueError:
        meta["union_p_mismatch_raises"] = True

    # ---- graphs: exact, CSR, hybrid (CPU reference path)
    graphs = {
        "k4_tail": (np.array([0, 0, 0, 1, 1, 2, 3, 4], dtype=np.int32),
                    np.array([1, 2, 3, 2, 3, 3, 4, 5], dtype=np.int32)),
        "er_2000": O.gen_er(2000, 12000, 7),
        "rmat10": O.gen_rmat(10, 16, 0.57, 0.19, 0.19, 3),
        "rmat12": O.gen_rmat(12, 16, 0.57, 0.19, 0.19, 1),
        "lattice_40": O.gen_lattice(40, 40, 0.3, 0.05, 0),
    }
    cases = {}
    for gname, (u, v) in graphs.items():
        edges = edges_from_raw(u, v)
        fwd, degree = graph.orient_graph(edges)
        fwd_c = compacted_forward_adj(fwd)
        row_ptr, col_idx, degrees, node_ids, eu, ev = gpu_graph.to_csr_numpy(fwd)
        if gname == "k4_tail":
            arrays[f"g_{gname}_raw_u"] = np.asarray(u, dtype=np.int32)
            arrays[f"g_{gname}_raw_v"] = np.asarray(v, dtype=np.int32)
        big = len(col_idx) > 20000
        digests = {}
        for nm, a in (("row_ptr", row_ptr), ("col_idx", col_idx), ("degrees", degrees), ("node_ids", node_ids),
                      ("edge_u", eu), ("edge_v", ev)):
            a = np.ascontiguousarray(a, dtype=np.int32)
            digests[nm] = hashlib.sha256(a.tobytes()).hexdigest()
            if not big:
                arrays[f"g_{gname}_{nm}"] = a
        deg_keys = np.array(sorted(degree), dtype=np.int64)
        arrays[f"g_{gname}_undeg"] = np.array([degree[k] for k in deg_keys], dtype=np.int64)
        cnt, _, _ = exact.exact_triangle_count(fwd)
        c = {"exact": int(cnt), "n_nodes": int(len(node_ids)), "n_edges": int(len(col_idx)), "sha256": digests}
        hyb = {}
        for theta, p in ((8, 8), (16, 10), (32, 12), (4, 4)):
            sk = hybrid.build_sketches(fwd_c, theta, p)
            tot, _, st, det = hybrid.hybrid_triangle_count(fwd_c, sk, theta, record_details=True)
            key = f"t{theta}_p{p}"
            hyb[key] = {"total": tot, "stats": st}
            if det and not big:
                arrays[f"g_{gname}_{key}_s_hat"] = np.array([d["s_hat"] for d in det], dtype=np.float64)
                arrays[f"g_{gname}_{key}_method"] = np.array([d["method"] == "hll" for d in det], dtype=np.uint8)
            # theta != gamma: fallback edges (src/hybrid.py:114-115)
            sk2 = hybrid.build_sketches(fwd_c, theta * 2, p)
            tot2, _, st2, _ = hybrid.hybrid_triangle_count(fwd_c, sk2, theta)
            hyb[key + "_fallback"] = {"total": tot2, "stats": st2}
        # original-id sketches (src/hybrid.py:39 hashes forward_adj's ids)
        sk = hybrid.build_sketches(fwd, 8, 8)
        tot, _, st, _ = hybrid.hybrid_triangle_count(fwd, sk, 8)
        hyb["orig_ids_t8_p8"] = {"total": tot, "stats": st}
        sk_keys = sorted(sk)
        if sk_keys:
            arrays[f"g_{gname}_origsk_keys"] = np.array(sk_keys, dtype=np.int64)
            arrays[f"g_{gname}_origsk_regs"] = np.stack([sk[k].registers for k in sk_keys])
        c["hybrid"] = hyb
        cases[gname] = c
    meta["graphs"] = cases

    # ---- cpu_exp HLL variant (cpu_exp/triangle_hll_experiment.py:357-498)
    cx = _import_cpu_exp(ref_root)
    assert cx.make_self_test_graph  # self-test graph exists
    cxg = {}
    for gname in ("k4_tail", "er_2000"):
        u, v = graphs[gname]
        e = np.array(sorted(edges_from_raw(u, v)), dtype=np.int64)
        ids = np.unique(e)
        e = np.searchsorted(ids, e)
        csr = cx.build_csr(len(ids), e)
        fg = cx.build_forward_graph(csr)
        for p in (4, 8):
            regs = cx.build_hll_registers_py(fg, p, seed=1)
            key = f"{gname}_p{p}"
            arrays[f"cx_{key}_regs"] = regs.reshape(-1)
            arrays[f"cx_{key}_offsets"] = fg.offsets
            arrays[f"cx_{key}_adj"] = fg.adj
            arrays[f"cx_{key}_edges"] = fg.edges.reshape(-1)
            arrays[f"cx_{key}_outdeg"] = fg.out_degree
            res = {}
            for thr in (0, 4, 16, 10**9):
                out = cx.hybrid_count_py(fg, regs, thr)
                res[str(thr)] = [float(x) for x in out]
            pure = cx.pure_hll_count_py(fg, regs)
            res["pure"] = [float(pure[0]), int(pure[1])]
            res["exact"] = int(cx.exact_forward_count_py(fg))
            cxg[key] = res
    meta["cpu_exp"] = cxg

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **arrays)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(meta, f, indent=1, sort_keys=True)
    print("wrote", len(arrays), "arrays;", os.path.getsize(os.path.join(HERE, "golden.npz")), "bytes")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the reference checkout>")
    main(sys.argv[1])
