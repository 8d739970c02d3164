"""Timing, memory and metric helpers (the reference's ``src/utils.py``
surface: relative_error, bias, proxy_label, Timer, peak_rss_mb)."""
from __future__ import annotations

import sys
import time

try:
    import resource
except ImportError:  # pragma: no cover - non-POSIX
    resource = None


def peak_rss_mb() -> float:
    """Peak resident set size of this process in MB (0.0 where unavailable)."""
    if resource is None:
        return 0.0
    peak = resource.getrusage(resource.RUSAGE_SELF).ru_maxrss
    # Linux reports kilobytes, macOS bytes.
    return peak / (1024.0 * 1024.0) if sys.platform == "darwin" else peak / 1024.0


def relative_error(estimate: float, truth: int) -> float:
    """|estimate - truth| / truth; inf for truth 0 with a non-zero estimate,
    0 when both are 0 (src/utils.py:36-43)."""
    if truth == 0:
        return 0.0 if estimate == 0 else float("inf")
    return abs(estimate - truth) / truth


def bias(estimate: float, truth: int) -> float:
    """Signed error estimate - truth."""
    return estimate - truth


_EDGES = (32, 64, 128, 256, 512)
_NAMES = ("[1,31]", "[32,63]", "[64,127]", "[128,255]", "[256,511]", "[512+]")


def proxy_label(proxy: int) -> str:
    """Bucket name of a routing proxy value (src/utils.py:55-64)."""
    for edge, name in zip(_EDGES, _NAMES):
        if proxy < edge:
            return name
    return _NAMES[-1]


class Timer:
    """``with Timer() as t: ...`` then ``t.elapsed`` (seconds)."""

    def __init__(self) -> None:
        self.elapsed: float = 0.0

    def __enter__(self) -> "Timer":
        self._t0 = time.perf_counter()
        return self

    def __exit__(self, *exc) -> None:
        self.elapsed = time.perf_counter() - self._t0
