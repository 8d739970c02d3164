"""Shared pytest setup: the ``gpu`` marker, repo-root imports and the golden
fixtures recorded from the reference implementation (tests/golden/)."""
from __future__ import annotations

import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN_DIR = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built libtchll.so")


@pytest.fixture(scope="session")
def golden():
    arrays = np.load(os.path.join(GOLDEN_DIR, "golden.npz"))
    with open(os.path.join(GOLDEN_DIR, "golden.json")) as f:
        meta = json.load(f)
    return arrays, meta


@pytest.fixture(scope="session")
def oracle():
    from oracle import build_oracle
    build_oracle.build()
    from oracle import oracle as O
    return O


@pytest.fixture(scope="session")
def tchll():
    """The CUDA package.  Fails (does not skip) without a CUDA device: the
    gpu-marked tests are the parity tests proper and must not pass vacuously."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("gpu test run without a CUDA device")
    import triangle_counting_hll_b200 as T
    from triangle_counting_hll_b200 import _lib
    _lib.load()
    return T
