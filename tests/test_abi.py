"""C-ABI checks that need no GPU: libtchll.so loads and exports every entry
point include/tchll.h declares; the Python binding covers each of them; the
result block layout matches the header."""
from __future__ import annotations

import ctypes as C
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "tchll.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(tchll_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "tchll_exact_count" in names and "tchll_hybrid_count_dense" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from triangle_counting_hll_b200 import _lib
    lib = C.CDLL(_lib.LIB_PATH)
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    from triangle_counting_hll_b200 import _lib
    assert set(declared_functions()) == set(_lib.SIGNATURES)
    _lib.load()  # sets argtypes for every symbol


def test_host_only_entry_points():
    from triangle_counting_hll_b200 import _lib
    L = _lib.load()
    assert L.tchll_version() >= 10000
    nb = C.c_size_t(0)
    assert L.tchll_count_workspace_bytes(100, 1000, C.byref(nb)) == 0 and nb.value > 8000
    assert L.tchll_gen_lattice_count(1000, 1000) == 1000 * 999 * 2 + 999 * 999
    out = (C.c_int32 * 8)()
    assert L.tchll_get_count_tuning(C.cast(out, C.c_void_p)) == 0
    # invalid arguments are rejected on the host with TCHLL_EINVAL
    assert L.tchll_set_count_tuning(33, 11, 16, 0) == _lib.TCHLL_EINVAL
    assert "multiple of 32" in _lib.last_error()
    with pytest.raises(ValueError):
        _lib.check(L.tchll_set_count_tuning(64, 99, 16, 0))
    assert L.tchll_exact_count(None, -1, None, 0, None, None, 0, None, None, None, 0, None) == _lib.TCHLL_EINVAL


def test_result_layout_matches_header():
    from triangle_counting_hll_b200 import _lib
    text = open(HEADER).read()
    body = text[text.index("typedef struct tchll_count_result"):]
    body = body[: body.index("}")]
    fields = re.findall(r"(u?int\d+_t)\s+(\w+);", body)
    assert [f for _, f in fields] == [f for f, _ in _lib.CountResult._fields_]
    assert C.sizeof(_lib.CountResult) == 64
