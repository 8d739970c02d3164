"""ctypes front end of the CPU oracle (``tchll_oracle.c``).

TEST INFRASTRUCTURE ONLY: this module is the checker.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline legs import it; the
product package never does.  Each function names the reference lines it
restates (ChitandaEruQ/triangle_counting_hll).
"""
from __future__ import annotations

import ctypes as C
import math
import os
from typing import Dict, Optional, Tuple

import numpy as np

from . import build_oracle

_lib = None

_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(dtype=np.int64, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(dtype=np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(dtype=np.uint8, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class _Nullable:
    """ndpointer that also accepts None (NULL)."""

    def __init__(self, base):
        self.base = base

    def from_param(self, obj):
        if obj is None:
            return None
        return self.base.from_param(obj)


def lib():
    global _lib
    if _lib is not None:
        return _lib
    path = build_oracle.LIB
    if not os.path.exists(path):
        path = build_oracle.build()
    L = C.CDLL(path)
    L.orc_hash64.restype = C.c_uint64
    L.orc_hash64.argtypes = [C.c_uint64]
    L.orc_hash64_array.argtypes = [_i64p, C.c_int64, _u64p]
    L.orc_alpha.restype = C.c_double
    L.orc_alpha.argtypes = [C.c_int64]
    L.orc_pairwise_sum.restype = C.c_double
    L.orc_pairwise_sum.argtypes = [_f64p, C.c_int64]
    L.orc_estimate.restype = C.c_double
    L.orc_estimate.argtypes = [_u8p, C.c_int64, C.c_double]
    L.orc_hll_add.argtypes = [_u8p, C.c_int, _i64p, C.c_int64]
    L.orc_union_estimate.restype = C.c_double
    L.orc_union_estimate.argtypes = [_u8p, _u8p, C.c_int]
    L.orc_build_sketches_dense.argtypes = [_i32p, _i32p, C.c_int64, C.c_int64, C.c_int, _u8p, _u8p]
    L.orc_build_sketches_compact.restype = C.c_int64
    L.orc_build_sketches_compact.argtypes = [_i64p, _i64p, C.c_int64, C.c_int64, C.c_int,
                                             _Nullable(_i64p), _Nullable(_u8p)]
    L.orc_intersect.restype = C.c_int64
    L.orc_intersect.argtypes = [_i32p, C.c_int64, _i32p, C.c_int64, C.c_double]
    L.orc_max_threads.restype = C.c_int
    L.orc_exact_count.restype = C.c_uint64
    L.orc_exact_count.argtypes = [_i32p, _i32p, _i32p, _i32p, C.c_int64, C.c_double, C.c_int,
                                  _Nullable(_i64p)]
    L.orc_hybrid_count.restype = C.c_double
    L.orc_hybrid_count.argtypes = [_i32p, _i32p, _i32p, _i32p, C.c_int64, _i32p, _i64p, _u8p,
                                   C.c_int, C.c_int64, C.c_double, C.c_int, _i64p,
                                   _Nullable(_f64p), _Nullable(_f64p), _Nullable(_u8p)]
    L.orc_csr_build.restype = C.c_int
    L.orc_csr_build.argtypes = [_i32p, _i32p, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                _i32p, _i32p, _i32p, _i64p, _i32p, _i32p]
    L.orc_gen_draw.restype = C.c_uint64
    L.orc_gen_draw.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
    L.orc_gen_rmat.argtypes = [C.c_int, C.c_int64, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint64,
                               _i32p, _i32p]
    L.orc_gen_er.argtypes = [C.c_int64, C.c_int64, C.c_uint64, _i32p, _i32p]
    L.orc_gen_perm.restype = C.c_uint64
    L.orc_gen_perm.argtypes = [C.c_uint64, C.c_uint64, C.c_uint64]
    L.orc_gen_lattice.restype = C.c_int64
    L.orc_gen_lattice.argtypes = [C.c_int64, C.c_int64, C.c_uint32, C.c_uint32, C.c_uint64,
                                  _Nullable(_i32p), _Nullable(_i32p)]
    L.orc_gen_chung_lu.argtypes = [_u64p, C.c_int64, C.c_int64, C.c_uint64, _i32p, _i32p]
    L.orc_chung_lu_table.restype = C.c_uint64
    L.orc_chung_lu_table.argtypes = [C.c_int64, C.c_double, _u64p]
    L.orc_cx_build_registers.argtypes = [_i64p, _i64p, C.c_int64, C.c_int, C.c_uint64, _u8p]
    L.orc_cx_hybrid.argtypes = [_i64p, _i64p, _i64p, _i64p, C.c_int64, _i64p, _u8p, C.c_int,
                                C.c_int64, _f64p]
    _lib = L
    return L


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


def max_threads() -> int:
    return int(lib().orc_max_threads())


# --------------------------------------------------------------------------- HLL
def hash64(x) -> np.ndarray:
    """src/hll.py:13-19 on an int64 array."""
    x = _c(np.atleast_1d(x), np.int64)
    out = np.empty(len(x), dtype=np.uint64)
    lib().orc_hash64_array(x, len(x), out)
    return out


def alpha(m: int) -> float:
    """src/hll.py:26-34."""
    return float(lib().orc_alpha(int(m)))


def estimate(regs, alpha_: Optional[float] = None) -> float:
    """src/hll.py:37-54."""
    regs = _c(regs, np.uint8)
    a = alpha(len(regs)) if alpha_ is None else alpha_
    return float(lib().orc_estimate(regs, len(regs), a))


def hll_add(regs: np.ndarray, p: int, x) -> None:
    """src/hll.py:81-96 (in place on a uint8 register row)."""
    assert regs.dtype == np.uint8 and regs.flags.c_contiguous
    x = _c(np.atleast_1d(x), np.int64)
    lib().orc_hll_add(regs, int(p), x, len(x))


def sketch(p: int, x) -> np.ndarray:
    regs = np.zeros(1 << p, dtype=np.uint8)
    hll_add(regs, p, x)
    return regs


def union_estimate(a, b, p: int) -> float:
    """src/hll.py:112-120."""
    return float(lib().orc_union_estimate(_c(a, np.uint8), _c(b, np.uint8), int(p)))


def build_sketches_dense(row_ptr, col_idx, n_nodes, theta, p, regs=None, has=None):
    """src/gpu_hll.py:47-81 (max-merges into the given rows)."""
    m = 1 << p
    if regs is None:
        regs = np.zeros(n_nodes * m, dtype=np.uint8)
    if has is None:
        has = np.zeros(n_nodes, dtype=np.uint8)
    lib().orc_build_sketches_dense(_c(row_ptr, np.int32), _c(col_idx, np.int32), int(n_nodes),
                                   int(theta), int(p), regs, has)
    return regs, has


def build_sketches_compact(row_ptr, keys, theta, p) -> Tuple[np.ndarray, np.ndarray]:
    """src/hybrid.py:15-41: (slot[n], rows[n_sketched * 2^p])."""
    rp = _c(row_ptr, np.int64)
    ks = _c(keys, np.int64)
    n = len(rp) - 1
    L = lib()
    ns = L.orc_build_sketches_compact(rp, ks, n, int(theta), int(p), None, None)
    slot = np.empty(n, dtype=np.int64)
    rows = np.zeros(max(ns, 0) * (1 << p) + 1, dtype=np.uint8)
    L.orc_build_sketches_compact(rp, ks, n, int(theta), int(p), slot, rows)
    return slot, rows[: ns * (1 << p)]


# --------------------------------------------------------------------- counting
def intersect(a, b, r: float = 8.0) -> int:
    """src/exact.py:29-41."""
    a = _c(a, np.int32)
    b = _c(b, np.int32)
    return int(lib().orc_intersect(a, len(a), b, len(b), float(r)))


def exact_count(row_ptr, col_idx, edge_u, edge_v, r: float = 8.0, nthreads: int = 0,
                per_edge: bool = False):
    """src/exact.py:48-98 / src/gpu_hybrid.py:96-130 over the given edges."""
    eu = _c(edge_u, np.int32)
    ev = _c(edge_v, np.int32)
    pe = np.empty(len(eu), dtype=np.int64) if per_edge else None
    t = int(lib().orc_exact_count(_c(row_ptr, np.int32), _c(col_idx, np.int32), eu, ev, len(eu),
                                  float(r), int(nthreads), pe))
    return (t, pe) if per_edge else t


def hybrid_count(row_ptr, col_idx, edge_u, edge_v, degrees, slot, rows, p, gamma,
                 r: float = 8.0, nthreads: int = 1, details: bool = False):
    """src/hybrid.py:95-164 with GPU routing src/gpu_hybrid.py:80-89.

    Returns (total, stats{n_edges,n_approx,n_exact,n_fallback,n_clamped}, details|None).
    """
    eu = _c(edge_u, np.int32)
    ev = _c(edge_v, np.int32)
    n = len(eu)
    stats = np.zeros(4, dtype=np.int64)
    sh = sc = me = None
    if details:
        sh = np.empty(n, dtype=np.float64)
        sc = np.empty(n, dtype=np.float64)
        me = np.empty(n, dtype=np.uint8)
    rows = _c(rows, np.uint8)
    if rows.size == 0:
        rows = np.zeros(1, dtype=np.uint8)
    total = float(lib().orc_hybrid_count(_c(row_ptr, np.int32), _c(col_idx, np.int32), eu, ev, n,
                                         _c(degrees, np.int32), _c(slot, np.int64), rows, int(p),
                                         int(gamma), float(r), int(nthreads), stats, sh, sc, me))
    st = {"n_edges": n, "n_approx": int(stats[0]), "n_exact": int(stats[1]),
          "n_fallback": int(stats[2]), "n_clamped": int(stats[3])}
    return total, st, ((sh, sc, me) if details else None)


def dense_slots(has_sketch) -> np.ndarray:
    """Dense register layout (row u at u*m) expressed as slots."""
    h = np.asarray(has_sketch)
    idx = np.arange(len(h), dtype=np.int64)
    return np.where(h == 1, idx, -1).astype(np.int64)


# -------------------------------------------------------------------- CSR build
def csr_build(raw_u, raw_v) -> Dict[str, np.ndarray]:
    """experiment/exp_gpu.py:317-365 on in-memory endpoint arrays."""
    ru = _c(raw_u, np.int32)
    rv = _c(raw_v, np.int32)
    n_raw = len(ru)
    cap_n = 2 * n_raw + 1
    row_ptr = np.zeros(cap_n + 1, dtype=np.int32)
    col_idx = np.empty(max(n_raw, 1), dtype=np.int32)
    fdeg = np.empty(cap_n, dtype=np.int32)
    node_ids = np.empty(cap_n, dtype=np.int64)
    eu = np.empty(max(n_raw, 1), dtype=np.int32)
    ev = np.empty(max(n_raw, 1), dtype=np.int32)
    nn = C.c_int64(0)
    ne = C.c_int64(0)
    rc = lib().orc_csr_build(ru, rv, n_raw, C.byref(nn), C.byref(ne), row_ptr, col_idx, fdeg,
                             node_ids, eu, ev)
    if rc != 0:
        raise ValueError("negative vertex id in edge list")
    n, e = nn.value, ne.value
    return {"row_ptr": row_ptr[: n + 1].copy(), "col_idx": col_idx[:e].copy(),
            "degrees": fdeg[:n].copy(), "node_ids": node_ids[:n].copy(),
            "edge_u": eu[:e].copy(), "edge_v": ev[:e].copy(),
            "n_nodes": n, "n_edges": e}


# ---------------------------------------------- forward_adj (dict) restatements
def orient_graph(edges) -> Tuple[dict, dict]:
    """src/graph.py:29-61 (vectorised; same dict contents and key order rules
    are not needed by the callers, which sort keys)."""
    arr = np.array(sorted(edges), dtype=np.int64).reshape(-1, 2)
    degree: Dict[int, int] = {}
    if len(arr) == 0:
        return {}, {}
    ids, cnt = np.unique(arr.reshape(-1), return_counts=True)
    deg = dict(zip(ids.tolist(), cnt.tolist()))
    du = np.array([deg[x] for x in arr[:, 0]])
    dv = np.array([deg[x] for x in arr[:, 1]])
    first = (du < dv) | ((du == dv) & (arr[:, 0] < arr[:, 1]))
    src = np.where(first, arr[:, 0], arr[:, 1])
    dst = np.where(first, arr[:, 1], arr[:, 0])
    fwd = {int(x): [] for x in ids}
    for s, d in zip(src.tolist(), dst.tolist()):
        fwd[s].append(d)
    fwd = {k: np.array(sorted(v), dtype=np.int64) for k, v in fwd.items()}
    degree = {int(k): int(v) for k, v in deg.items()}
    return fwd, degree


def to_csr_numpy(forward_adj: dict):
    """src/gpu_graph.py:6-41."""
    node_ids = np.array(sorted(forward_adj.keys()), dtype=np.int32)
    index = {int(nid): i for i, nid in enumerate(node_ids)}
    degrees = np.array([len(forward_adj[int(nid)]) for nid in node_ids], dtype=np.int32)
    row_ptr = np.zeros(len(node_ids) + 1, dtype=np.int32)
    row_ptr[1:] = np.cumsum(degrees)
    col = np.array([index[int(v)] for nid in node_ids for v in forward_adj[int(nid)]],
                   dtype=np.int32)
    eu = np.repeat(np.arange(len(node_ids), dtype=np.int32), degrees)
    return row_ptr, col, degrees, node_ids, eu, col.copy()


# ------------------------------------------------------------------ generators
def prob_threshold(p: float) -> int:
    """Probability -> 32-bit threshold (floor(p * 2^32), capped)."""
    return min(int(math.floor(p * 4294967296.0)), 0xFFFFFFFF)


def gen_draw(seed: int, stream: int, i: int) -> int:
    return int(lib().orc_gen_draw(seed, stream, i))


def gen_rmat(scale: int, edge_factor: int, a: float, b: float, c: float, seed: int):
    n_raw = edge_factor << scale
    u = np.empty(n_raw, dtype=np.int32)
    v = np.empty(n_raw, dtype=np.int32)
    lib().orc_gen_rmat(scale, n_raw, prob_threshold(a), prob_threshold(a + b),
                       prob_threshold(a + b + c), seed, u, v)
    return u, v


def gen_er(n: int, n_raw: int, seed: int):
    u = np.empty(n_raw, dtype=np.int32)
    v = np.empty(n_raw, dtype=np.int32)
    lib().orc_gen_er(n, n_raw, seed, u, v)
    return u, v


def gen_perm(x: int, n: int, seed: int) -> int:
    return int(lib().orc_gen_perm(x, n, seed))


def gen_lattice(rows: int, cols: int, p_diag: float, p_del: float, seed: int):
    L = lib()
    td, tx = prob_threshold(p_diag), prob_threshold(p_del)
    total = L.orc_gen_lattice(rows, cols, td, tx, seed, None, None)
    u = np.empty(total, dtype=np.int32)
    v = np.empty(total, dtype=np.int32)
    L.orc_gen_lattice(rows, cols, td, tx, seed, u, v)
    return u, v


def chung_lu_table(n: int, beta: float) -> np.ndarray:
    cum = np.empty(n, dtype=np.uint64)
    lib().orc_chung_lu_table(n, float(beta), cum)
    return cum


def gen_chung_lu(n: int, avg_degree: float, beta: float, seed: int):
    cum = chung_lu_table(n, beta)
    n_raw = int(round(n * avg_degree / 2.0))
    u = np.empty(n_raw, dtype=np.int32)
    v = np.empty(n_raw, dtype=np.int32)
    lib().orc_gen_chung_lu(cum, n, n_raw, seed, u, v)
    return u, v


# ------------------------------------------------------------ cpu_exp variant
def cx_build_registers(offsets, adj, n, p, seed) -> np.ndarray:
    """cpu_exp/triangle_hll_experiment.py:386-401 (dense n x 2^p)."""
    regs = np.zeros(n * (1 << p), dtype=np.uint8)
    lib().orc_cx_build_registers(_c(offsets, np.int64), _c(adj, np.int64), int(n), int(p),
                                 int(seed) & 0xFFFFFFFFFFFFFFFF, regs)
    return regs


def cx_hybrid(offsets, adj, edge_u, edge_v, outdeg, regs, p, threshold):
    """cpu_exp/triangle_hll_experiment.py:480-498 (threshold < 0: pure HLL,
    :466-476).  Returns (total, exact_edges, hll_edges, exact_sum, hll_sum, clamp)."""
    out = np.zeros(6, dtype=np.float64)
    eu = _c(edge_u, np.int64)
    lib().orc_cx_hybrid(_c(offsets, np.int64), _c(adj, np.int64), eu, _c(edge_v, np.int64),
                        len(eu), _c(outdeg, np.int64), _c(regs, np.uint8), int(p),
                        int(threshold), out)
    return (float(out[0]), int(out[1]), int(out[2]), float(out[3]), float(out[4]), int(out[5]))
