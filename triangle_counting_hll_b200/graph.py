"""Graph loading and orientation (drop-in for the reference's ``src/graph.py``).

``orient_graph`` returns the reference's ``(forward_adj, degree)`` dicts
(src/graph.py:29-61); the dedup, degree count, (degree, id) orientation and row
sort run on the GPU through libtchll's CSR builder, with ids kept as given.
``load_edgelist`` keeps the reference's text format and set result
(src/graph.py:8-26); ``ingest.load_edge_arrays`` is the array-returning form
for large files.
"""
from __future__ import annotations

from typing import Dict, Set, Tuple

import numpy as np

from . import _lib, core


def load_edgelist(filepath: str, comment_chars: str = "#%") -> Set[Tuple[int, int]]:
    """Undirected edge set with canonical (min, max) pairs; comment lines,
    short lines and self-loops skipped (src/graph.py:8-26)."""
    from .ingest import parse_edge_text
    with open(filepath, "rb") as f:
        data = f.read()
    u, v = parse_edge_text(data, comment_chars)
    u = u.cpu().numpy().astype(np.int64)
    v = v.cpu().numpy().astype(np.int64)
    keep = u != v
    a = np.minimum(u[keep], v[keep])
    b = np.maximum(u[keep], v[keep])
    return set(zip(a.tolist(), b.tolist()))


def orient_graph(edges: Set[Tuple[int, int]]) -> Tuple[Dict[int, np.ndarray], Dict[int, int]]:
    """Orient edges by the (degree, node id) total order (src/graph.py:29-61).

    Returns ``forward_adj`` (node -> sorted int64 array of forward neighbours,
    every endpoint present, ascending node order) and ``degree`` (node ->
    undirected degree)."""
    _lib.require_cuda()
    if not edges:
        return {}, {}
    arr = np.fromiter((x for e in edges for x in e), dtype=np.int64, count=2 * len(edges)).reshape(-1, 2)
    if arr.min() < 0 or arr.max() > np.iinfo(np.int32).max:
        raise ValueError("node ids must lie in [0, 2^31) for the device path")
    g, und = core.csr_from_edges(arr[:, 0].astype(np.int32), arr[:, 1].astype(np.int32), undirected=True)
    ids = g.node_ids.cpu().numpy().astype(np.int64)
    row_ptr = g.row_ptr.cpu().numpy().astype(np.int64)
    col = ids[g.col_idx.cpu().numpy()]
    deg = und.cpu().numpy()
    forward_adj = {int(ids[i]): col[row_ptr[i]:row_ptr[i + 1]] for i in range(len(ids))}
    degree = {int(ids[i]): int(deg[i]) for i in range(len(ids))}
    return forward_adj, degree


def make_small_graph(triangles: list) -> Set[Tuple[int, int]]:
    """Edge set of the given triangles (src/graph.py:64-74)."""
    edges: Set[Tuple[int, int]] = set()
    for a, b, c in triangles:
        for x, y in ((a, b), (b, c), (a, c)):
            edges.add((min(x, y), max(x, y)))
    return edges
