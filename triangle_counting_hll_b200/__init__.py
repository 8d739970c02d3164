"""B200-native (sm_100a) hybrid exact / HyperLogLog triangle counting.

Drop-in for the hot path of ChitandaEruQ/triangle_counting_hll: the modules
``graph``, ``gpu_graph``, ``exact``, ``hll``, ``hybrid``, ``gpu_hll`` and
``gpu_hybrid`` keep the reference's entry points (same names, arguments,
return values and ValueError conventions) and run on libtchll, the CUDA
library built from ``csrc/`` with a C ABI declared in ``include/tchll.h``.
There is no CPU fallback: without the library or a CUDA device the entry
points raise.
"""
from .exact import exact_triangle_count, intersect_adaptive, intersect_bsearch, intersect_merge
from .gpu_graph import csr_from_edge_list, to_csr_gpu, to_csr_numpy
from .gpu_hll import alloc_sketch_arrays, alloc_sketch_arrays_device, build_sketches_kernel
from .gpu_hybrid import gpu_exact_triangle_count, gpu_hybrid_triangle_count
from .graph import load_edgelist, make_small_graph, orient_graph
from .hll import HLL, union_estimate
from .hybrid import build_sketches, hybrid_triangle_count
from .utils import Timer, bias, peak_rss_mb, proxy_label, relative_error

__all__ = [
    "exact_triangle_count", "intersect_adaptive", "intersect_bsearch", "intersect_merge",
    "csr_from_edge_list", "to_csr_gpu", "to_csr_numpy",
    "alloc_sketch_arrays", "alloc_sketch_arrays_device", "build_sketches_kernel",
    "gpu_exact_triangle_count", "gpu_hybrid_triangle_count",
    "load_edgelist", "make_small_graph", "orient_graph",
    "HLL", "union_estimate", "build_sketches", "hybrid_triangle_count",
    "Timer", "bias", "peak_rss_mb", "proxy_label", "relative_error",
]
