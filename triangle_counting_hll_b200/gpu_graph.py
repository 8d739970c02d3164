"""Forward adjacency / edge list -> CSR on the GPU (drop-in for the reference's
``src/gpu_graph.py``, plus the device edge-list ingest the reference performs
with numpy in experiment/exp_gpu.py:264-389).

``to_csr_numpy`` / ``to_csr_gpu`` return the reference's six arrays
``(row_ptr, col_idx, degrees, node_ids, edge_u, edge_v)`` (src/gpu_graph.py:6-52)
computed by libtchll's ``tchll_csr_from_adjacency`` (device sort + remap);
``to_csr_gpu`` returns torch CUDA tensors where the reference returned CuPy
arrays.  ``csr_from_edge_list`` builds the oriented CSR straight from raw
endpoint arrays (dedup, self-loops, id compaction, (degree, id) orientation)
with ``tchll_csr_build_phase1/2``.
"""
from __future__ import annotations

import numpy as np
import torch

from . import _lib, core


def _to_csr_device(forward_adj: dict):
    _lib.require_cuda()
    keys, lens, values = core.flatten_adjacency(forward_adj)
    adj = core.csr_from_adjacency(keys, lens, values)
    if adj.missing:
        missing = np.setdiff1d(values, keys)
        raise KeyError(int(missing[0]))
    g = adj.csr
    if len(keys) and (keys.min() < np.iinfo(np.int32).min or keys.max() > np.iinfo(np.int32).max):
        raise OverflowError("node ids do not fit the reference's int32 node_ids")
    node_ids = adj.keys.to(torch.int32)
    return g.row_ptr, g.col_idx, g.degrees, node_ids, g.edge_u, g.edge_v


def to_csr_numpy(forward_adj: dict):
    """forward_adj -> int32 CSR arrays on the host (src/gpu_graph.py:6-41)."""
    return tuple(t.cpu().numpy() for t in _to_csr_device(forward_adj))


def to_csr_gpu(forward_adj: dict):
    """Same arrays as to_csr_numpy, as torch CUDA tensors (src/gpu_graph.py:44-52)."""
    return _to_csr_device(forward_adj)


def csr_from_edge_list(u, v, device=None):
    """Raw undirected endpoint arrays -> oriented CSR, returned as the
    reference loader's arrays ``(row_ptr, col_idx, degrees, node_ids, edge_u,
    edge_v)`` (experiment/exp_gpu.py:288-365), all int32 device tensors."""
    g = core.csr_from_edges(u, v, device)
    return g.row_ptr, g.col_idx, g.degrees, g.node_ids, g.edge_u, g.edge_v
