"""Device edge-list ingest: text bytes -> endpoint arrays -> oriented CSR.

The reference parses SNAP text on the host, line by line
(src/graph.py:8-26, experiment/exp_gpu.py:131-144,264-389 -- 519 s of
``t_load`` on com-Orkut).  Here the file's bytes are copied to the GPU once
and ``tchll_parse_edges`` splits lines and parses the first two integer
tokens of each in parallel, with the same skipping rules; ``load_graph`` then
hands the arrays to the device CSR builder (dedup, self-loops, id compaction,
orientation).
"""
from __future__ import annotations

import ctypes as C
from typing import Tuple, Union

import numpy as np
import torch

from . import _lib, core
from ._lib import check, load, ptr, stream_handle


def parse_edge_text(data: Union[bytes, bytearray, memoryview, np.ndarray, torch.Tensor],
                    comment_chars: str = "#%", device=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Parse edge-list text; returns int32 device tensors (u, v), self-loops
    included.  Raises ValueError on a token that is not an int32 integer
    (the reference's int() raises ValueError there)."""
    _lib.require_cuda()
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    if isinstance(data, torch.Tensor):
        text = data.to(device=dev, dtype=torch.uint8).contiguous()
    else:
        arr = np.frombuffer(bytearray(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
        text = torch.from_numpy(np.array(arr, dtype=np.uint8, copy=True)).to(dev)
    n = int(text.numel())
    L = load()
    nb = C.c_size_t(0)
    check(L.tchll_ingest_workspace_bytes(n, C.byref(nb)))
    cap = n // 4 + 2
    with torch.cuda.device(dev):
        ws = torch.empty(max(nb.value, 256), dtype=torch.uint8, device=dev)
        u = torch.empty(cap, dtype=torch.int32, device=dev)
        v = torch.empty(cap, dtype=torch.int32, device=dev)
        cnt = torch.zeros(2, dtype=torch.int64, device=dev)
        check(L.tchll_parse_edges(ptr(text), n, comment_chars.encode(), ptr(u), ptr(v), ptr(cnt[0:1]),
                                  ptr(cnt[1:2]), ptr(ws), nb.value, stream_handle(dev)), "parse edges")
        n_out, n_bad = (int(x) for x in cnt.cpu().tolist())
    if n_bad:
        raise ValueError(f"{n_bad} edge-list line(s) hold tokens that are not int32 integers")
    return u[:n_out], v[:n_out]


def load_edge_arrays(filepath: str, comment_chars: str = "#%", device=None) -> Tuple[torch.Tensor, torch.Tensor]:
    """Read a text edge list and parse it on the GPU."""
    with open(filepath, "rb") as f:
        data = f.read()
    return parse_edge_text(data, comment_chars, device)


def load_graph(filepath: str, comment_chars: str = "#%", device=None) -> core.DeviceCSR:
    """Text edge list -> oriented device CSR (the array outputs of the
    reference's _load_graph, experiment/exp_gpu.py:264-389)."""
    u, v = load_edge_arrays(filepath, comment_chars, device)
    return core.csr_from_edges(u, v, device=u.device)
