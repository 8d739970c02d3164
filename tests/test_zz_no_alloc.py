"""The allocation-free exact count, called through the C ABI.

tchll_exact_count_noalloc exists for callers that hold device pointers to a
graph but cannot allocate device memory themselves -- a foreign-language
binding without a CUDA allocator of its own, or a service that reserves all
device memory up front and allows no allocation while serving.  It must give
the same count as tchll_exact_count (which takes a caller workspace) on two
calls in a row, since every call reuses the same fixed scratch array, and it
must refuse graphs whose scratch would not fit that array.

This file is collected last on purpose, and it also passes when run alone.
"""
from __future__ import annotations

import ctypes as C

import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return t.data_ptr() if t.numel() else None


def _workspace_count(L, g, torch, dev, stream):
    nb = C.c_size_t(0)
    assert L.tchll_count_workspace_bytes(g.n_nodes, g.n_edges, C.byref(nb)) == 0
    ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
    res = torch.zeros(64, dtype=torch.uint8, device=dev)
    rc = L.tchll_exact_count(_ptr(g.row_ptr), g.n_nodes, _ptr(g.col_idx), g.n_edges, _ptr(g.edge_u),
                             _ptr(g.edge_v), g.n_edges, None, _ptr(res), _ptr(ws), nb.value, stream)
    assert rc == 0
    return res


def _noalloc_count(L, g, torch, dev, stream):
    res = torch.full((64,), 0xAB, dtype=torch.uint8, device=dev)  # stale bytes must not leak through
    rc = L.tchll_exact_count_noalloc(_ptr(g.row_ptr), g.n_nodes, _ptr(g.col_idx), g.n_edges, _ptr(g.edge_u),
                                     _ptr(g.edge_v), g.n_edges, _ptr(res), stream)
    return rc, res


def test_noalloc_matches_workspace_entry_point(tchll, oracle):
    import torch

    from triangle_counting_hll_b200 import _lib, core

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    for scale, seed in ((15, 1), (16, 7)):
        u, v = core.gen_rmat(scale, 16, 0.57, 0.19, 0.19, seed=seed, device=dev)
        g = core.csr_from_edges(u, v)
        ref = _lib.read_count_result(_workspace_count(L, g, torch, dev, stream))
        assert ref.status == 0 and ref.exact > 0
        # and independently of the shared counting code: the CPU oracle on
        # its own CSR of the same edge list
        og = oracle.csr_build(u.cpu().numpy(), v.cpu().numpy())
        assert ref.exact == oracle.exact_count(og["row_ptr"], og["col_idx"], og["edge_u"], og["edge_v"], nthreads=0)
        for _ in range(2):  # two calls in a row share the fixed scratch
            rc, res = _noalloc_count(L, g, torch, dev, stream)
            assert rc == 0, _lib.last_error()
            got = _lib.read_count_result(res)
            assert got.status == 0
            assert got.exact == ref.exact  # exact counts: bit-exact
            assert got.n_exact == ref.n_exact == g.n_edges


def test_noalloc_rejects_graphs_beyond_its_scratch(tchll):
    import torch

    from triangle_counting_hll_b200 import _lib, core

    L = _lib.load()
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev).cuda_stream
    u, v = core.gen_rmat(19, 16, 0.57, 0.19, 0.19, seed=1, device=dev)
    g = core.csr_from_edges(u, v)
    assert 8 * (g.n_edges + g.n_nodes) > (32 << 20)
    rc, _ = _noalloc_count(L, g, torch, dev, stream)
    assert rc == _lib.TCHLL_EINVAL
    assert "too large" in _lib.last_error()
