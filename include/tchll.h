/*
 * tchll.h -- C ABI of libtchll, the B200 (sm_100a) implementation of the
 * hybrid exact / HyperLogLog triangle-counting path of
 * ChitandaEruQ/triangle_counting_hll.
 *
 * Conventions
 *   - Every pointer argument is DEVICE memory unless its comment says "host".
 *   - Nothing here allocates device memory.  Scratch comes from a caller
 *     buffer ("workspace") whose size the matching *_workspace_bytes query
 *     returns; a NULL workspace is never dereferenced by the query.
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).  All work is
 *     stream-ordered; results written to device memory are valid once the
 *     stream has been synchronised.  No call synchronises except where noted.
 *   - Every function returns TCHLL_OK (0) or an error code; the message of the
 *     last error on the calling thread is tchll_last_error().
 *   - Ids and CSR offsets are int32, as in the reference (src/gpu_graph.py:6-41).
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the reference project).
 */
#ifndef TCHLL_H
#define TCHLL_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCHLL_OK 0
#define TCHLL_EINVAL 1     /* invalid argument (the reference raises ValueError) */
#define TCHLL_ECUDA 2      /* CUDA runtime error */
#define TCHLL_EWORKSPACE 3 /* workspace smaller than the query returned */

/* Malformed-input flags a kernel reports in tchll_count_result.status. */
#define TCHLL_STATUS_BAD_EDGE 1u /* edge endpoint outside [0, n_nodes) */
#define TCHLL_STATUS_BAD_ROW 2u  /* row_ptr extent outside [0, nnz] or decreasing */
#define TCHLL_STATUS_BAD_SLOT 4u /* sketch slot outside [0, n_rows) */
#define TCHLL_STATUS_BAD_KEY 8u  /* neighbour id (col_idx value) outside [0, n_nodes) */

/*
 * Totals written by the counting entry points (64 bytes, device memory).
 * exact      sum of exact supports over exact-routed edges (uint64, exact)
 * hll_fx     sum of clamped HLL supports in fixed point, units of 2^-32,
 *            as a 128-bit integer (hll_fx_hi:hll_fx_lo); each edge's clamped
 *            FP64 estimate is rounded to the nearest 2^-32 before summing, so
 *            the total is independent of summation order
 * n_*        the reference's stats (src/hybrid.py:152-164,
 *            src/gpu_hybrid.py:415-430); n_fallback counts edges that wanted
 *            HLL but lacked a sketch on one side
 * status     TCHLL_STATUS_* flags; non-zero means the input was malformed and
 *            the offending edges were skipped
 */
typedef struct tchll_count_result {
    uint64_t exact;
    uint64_t hll_fx_lo;
    uint64_t hll_fx_hi;
    int64_t n_approx;
    int64_t n_exact;
    int64_t n_fallback;
    int64_t n_clamped;
    uint32_t status;
    uint32_t reserved;
} tchll_count_result;

/* ------------------------------------------------------------- library --- */
const char* tchll_last_error(void);
int tchll_version(void);
/* Number of kernels this library has launched in this process (host). */
uint64_t tchll_launch_count(void);

/* --------------------------------------------- exact / hybrid counting --- */
/* Workspace for tchll_exact_count / tchll_hybrid_count_* on a CSR of n_nodes
 * rows and n_edges edges: the regrouped pair lists, per-vertex histograms and
 * offsets, the long-list work units, 16-byte-aligned copies of the probe
 * lists and, for hybrid counts, the HLL edge list -- about 20 bytes per edge
 * + 110 per vertex.  The aligned copies are optional: a workspace too small
 * for them but large enough otherwise runs without them (same results). */
int tchll_count_workspace_bytes(int64_t n_nodes, int64_t n_edges, size_t* bytes);

/* Workspace for a hybrid count whose sketches are n_rows register rows of
 * 2^p bytes (compact: the rows of tchll_build_sketches_compact; dense: n_nodes).
 * Adds the rows' zero-register masks (max(2^p / 8, 16) bytes per row) to the
 * tchll_count_workspace_bytes size: with them the HLL pass tests the
 * linear-counting branch from 2^p / 8 bytes per sketch instead of 2^p.  A
 * hybrid call given only tchll_count_workspace_bytes still runs, reading the
 * registers; the results are the same either way. */
int tchll_hybrid_workspace_bytes(int64_t n_nodes, int64_t n_edges, int64_t n_rows, int32_t p, size_t* bytes);

/*
 * Exact count: T = sum over the n_edges edges (edge_u[i], edge_v[i]) of
 * |N+(u) cap N+(v)| with N+(x) = col_idx[row_ptr[x] .. row_ptr[x+1]) (sorted,
 * duplicate-free).  Replaces gpu_exact_triangle_count
 * (src/gpu_hybrid.py:332-354) and the loop of exact_triangle_count
 * (src/exact.py:48-98).  per_edge_support (nullable, n_edges int64) receives
 * each edge's support.
 */
int tchll_exact_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                      const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                      int64_t* per_edge_support, tchll_count_result* result, void* workspace,
                      size_t workspace_bytes, void* stream);

/* tchll_exact_count (no per-edge output) for a col_idx still being copied:
 * the kernels that read col_idx first wait for col_ready_event (a
 * cudaEvent_t recorded after the copy that fills col_idx; NULL: ready), so
 * the pair regrouping, which reads only row_ptr and the edges, overlaps that
 * copy.  row_ptr, edge_u and edge_v must be ready in stream order.  Same
 * result as tchll_exact_count. */
int tchll_exact_count_staged(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                             const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                             tchll_count_result* result, void* workspace, size_t workspace_bytes,
                             void* col_ready_event, void* stream);

/*
 * Hybrid count over DENSE sketches (row v at sketch_regs + v * 2^p, present
 * iff has_sketch[v] == 1).  An edge goes to HLL iff
 * min(degrees[u], degrees[v]) >= gamma and both endpoints have a sketch.
 * split_kernels != 0 runs the exact-routed and HLL-routed edges as two
 * launches, otherwise one.  Replaces gpu_hybrid_triangle_count
 * (src/gpu_hybrid.py:357-431).  p outside [4, 16] is TCHLL_EINVAL.
 */
int tchll_hybrid_count_dense(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                             const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                             const int32_t* degrees, const uint8_t* sketch_regs, const uint8_t* has_sketch,
                             int32_t p, int64_t gamma, int32_t split_kernels, tchll_count_result* result,
                             void* workspace, size_t workspace_bytes, void* stream);

/*
 * Hybrid count over COMPACT sketches: slot[v] >= 0 selects row
 * rows + slot[v] * 2^p (n_rows rows), -1 means no sketch.  Replaces the loop
 * of hybrid_triangle_count (src/hybrid.py:48-166).  The four per-edge outputs
 * (support int64, s_hat f64, s_clamped f64, method u8: 0 exact / 1 HLL) are
 * all NULL or all set; support is written for exact edges, s_hat/s_clamped
 * for HLL edges.
 */
int tchll_hybrid_count_compact(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                               const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                               const int32_t* degrees, const uint8_t* rows, int64_t n_rows, const int64_t* slot,
                               int32_t p, int64_t gamma, int32_t split_kernels, int64_t* per_edge_support,
                               double* per_edge_s_hat, double* per_edge_s_clamped, uint8_t* per_edge_method,
                               tchll_count_result* result, void* workspace, size_t workspace_bytes,
                               void* stream);

/* Launch shape of the counting kernels (process-wide host state; no
 * counterpart in the reference, whose block size is fixed at 256,
 * src/gpu_hybrid.py:13).  chunk: edges claimed per warp (multiple of 32);
 * slots_log2: per-warp hash table capacity; tiny: lane-local merge threshold
 * on |N+u|+|N+v|; blocks_per_sm: 0 = occupancy maximum; warps_per_cta: 1-8;
 * pairs: 1 = probe the shorter list into a table of the longer one (edges
 * regrouped by a device counting sort), 0 = edges as given; sparse: 1 = hash
 * tables at load <= 1/4 where they fit (else <= 1/2).  out8 receives chunk,
 * slots_log2, tiny, blocks_per_sm, warps_per_cta, pairs, sparse and a
 * reserved 0.  Results are identical for every setting. */
int tchll_set_count_tuning(int32_t chunk, int32_t slots_log2, int32_t tiny, int32_t blocks_per_sm);
int tchll_set_count_shape(int32_t warps_per_cta, int32_t pairs);
int tchll_set_count_table(int32_t sparse);
int tchll_get_count_tuning(int32_t* out8 /* host */);

/* Hub pairs (pairs layout only, col_idx 16-byte aligned): pairs whose table
 * side x has d+(x) > threshold are counted by a kernel in which a whole CTA
 * shares one hash table of N+(x) (load <= 1/16 where 2^table_log2 slots of
 * shared memory allow), seg_pairs of x's pairs per work unit, unroll 16-byte
 * probe loads in flight per lane.  threshold 0 turns it off; otherwise
 * threshold >= 64, seg_pairs in [256, 2^20], table_log2 in [10, 15], unroll 2
 * or 4.  out4 receives the four values.  Results are identical for every
 * setting. */
int tchll_set_count_hub(int32_t threshold, int32_t seg_pairs, int32_t table_log2, int32_t unroll);
int tchll_get_count_hub(int32_t* out4 /* host */);

/* Hub core (pairs layout, with the padded lists in the workspace): the hub
 * kernels work in the coordinates of the core, the vertices that appear in
 * some hub table side's forward list; a probe list member outside the core
 * cannot match.  A table side's list becomes a bitmap in shared memory:
 * with packed != 0 and a core of at most 131,070 vertices the probe lists
 * hold 16-bit core indices (two planes) and the bitmap takes 16 KB; else,
 * when the core fits 8 * 2^bitmap_log2 bits (minus 32), 32-bit lists and a
 * bitmap of that size; else hash tables.  bitmap_log2 0 turns the 32-bit
 * bitmap off; otherwise in [10, 17].  overlap 1 runs the hub core pass
 * and a hybrid count's HLL pass on a second stream beside the exact pairs;
 * overlap 2 also moves an exact count's short-list pair kernel there, after
 * the core pass, beside the hub kernel; 0 runs everything on the caller's
 * stream (the second stream is joined before the call returns).  bank_sort != 0 orders each packed
 * list's keys by the shared-memory bank of their bitmap word (fewer bank
 * conflicts in the hub kernel, a slower core pass).  out4 receives the four
 * values.  Results are identical for every setting.  These kernels read
 * col_idx values as vertex indices: a value outside [0, n_nodes) is
 * reported as TCHLL_STATUS_BAD_KEY. */
int tchll_set_count_core(int32_t bitmap_log2, int32_t overlap, int32_t packed, int32_t bank_sort);
int tchll_get_count_core(int32_t* out4 /* host */);

/* HLL pass of the hybrid counts (with the zero masks in the workspace):
 * for p <= row_cache_max_p each group of lanes takes a contiguous run of the
 * HLL edges (CSR order, so mostly one u) and keeps u's zero mask and
 * register row in registers, reading only v's per edge.  lanes: lanes per
 * HLL edge (0: chosen by p, else a power of two in [1, 32]).  out2 receives
 * both values.  Results are identical for every setting. */
int tchll_set_hll_pass(int32_t row_cache_max_p, int32_t lanes);
int tchll_get_hll_pass(int32_t* out2 /* host */);

/*
 * Allocation-free exact count, for callers that cannot allocate device memory
 * (a binding with no CUDA allocator of its own, or a service whose device
 * memory is all reserved up front).  No counterpart in the reference.  Same
 * result as tchll_exact_count without per-edge output, but the scratch comes
 * from a fixed array of TCHLL_NOALLOC_SCRATCH_BYTES inside the library that
 * every GPU loading the library reserves until the process exits; graphs
 * needing more scratch (about 8 bytes per edge + 32 per vertex: the pair
 * lists, four per-vertex histograms / offsets and the work-unit list, so for
 * example 3 M edges on 200 K vertices fit) are rejected with TCHLL_EINVAL.
 * The first
 * call in each CUDA context looks up the array's device address (cached per
 * context id, so a context made current by the caller, or one re-created
 * after cudaDeviceReset, gets its own lookup); make that first call before
 * any stream capture.  All calls share the one array: calls that
 * overlap on the GPU (different streams or devices sharing a context) race;
 * serialize them.  Nothing here calls cudaMalloc or cudaFree.
 */
#define TCHLL_NOALLOC_SCRATCH_BYTES (32u << 20)
int tchll_exact_count_noalloc(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                              const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                              tchll_count_result* result, void* stream);

/* Phase timing for measurement (process-wide host state, off by default).
 * When enabled, the counting entry points record CUDA events on the
 * caller's stream around their phases; tchll_phase_times then waits for the
 * last call's events and writes milliseconds: ms3[0] pair regrouping,
 * ms3[1] exact-count kernels (pair kernel and hub kernels), ms3[2] HLL pass
 * (-1 for a phase the call did not run; with the overlap on, the HLL pass
 * runs beside ms3[1] on the second stream).  tchll_phase_hub_ms writes the
 * hub pairs' share of ms3[1]: ms2[0] the hub kernels, ms2[1] the core pass
 * before them (-1 when they did not run).  While timing is on, counting
 * calls serialize their enqueues. */
int tchll_set_phase_timing(int32_t enable);
int tchll_phase_times(float* ms3 /* host */);
int tchll_phase_hub_ms(float* ms2 /* host */);

/* ------------------------------------------------------------ sketches --- */
/*
 * Dense sketch build, launch-compatible with build_sketches_kernel
 * (src/gpu_hll.py:47-81): for every u, has_sketch[u] = (row length >= theta);
 * for those u, the registers of N+(u) (hashing the col_idx values) are
 * max-merged into sketch_regs[u * 2^p ..] (pass zeroed rows for fresh
 * sketches, as alloc_sketch_arrays does, src/gpu_hll.py:128-133).  Needs no
 * workspace.
 */
int tchll_build_sketches_dense(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                               int64_t theta, int32_t p, uint8_t* sketch_regs, uint8_t* has_sketch, void* stream);

/*
 * Compact sketches (src/hybrid.py:15-41): tchll_sketch_slots (workspace from
 * tchll_sketch_workspace_bytes) writes
 * slot[u] = rank of u among vertices with row length >= theta (ascending u),
 * or -1, and the number of sketches to *n_sketched (device int64).
 * tchll_build_sketches_compact then writes rows[slot[u] * 2^p ..] for every
 * sketched u (rows are overwritten, not merged).  keys (nullable, int64,
 * n_nodes) maps a column to the value hashed in its place: keys[col_idx[k]]
 * -- the original vertex ids when the CSR holds compacted ones
 * (src/hybrid.py:39 hashes forward_adj's ids); NULL hashes col_idx[k].
 */
int tchll_sketch_workspace_bytes(int64_t n_nodes, size_t* bytes);
int tchll_sketch_slots(const int32_t* row_ptr, int64_t n_nodes, int64_t theta, int64_t* slot, int64_t* n_sketched,
                       void* workspace, size_t workspace_bytes, void* stream);
int tchll_build_sketches_compact(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                 const int64_t* keys, int64_t nnz, const int64_t* slot, int64_t n_rows, int32_t p,
                                 uint8_t* rows, void* stream);

/*
 * The cpu_exp estimator variant (cpu_exp/triangle_hll_experiment.py), for
 * comparison with the reference's published CPU numbers:
 * tchll_cx_build_registers fills dense rows for EVERY vertex with the seeded
 * hash h = splitmix64(x + seed + 0x9E3779B97F4A7C15), index = low p bits,
 * rank from h >> p (:386-401), and sets has_all[u] = 1; tchll_cx_hybrid_count
 * routes an edge to exact iff min(d+u, d+v) <= threshold (threshold < 0: all
 * edges HLL, the pure-HLL count) and estimates with estimate_hll_cardinality
 * (linear counting, else the 2^32 correction; :357-366).  regs must be zeroed
 * by the caller only for tchll_cx_hybrid_count inputs not made here.
 */
int tchll_cx_build_registers(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz, int32_t p,
                             uint64_t seed, uint8_t* regs, uint8_t* has_all, void* stream);
int tchll_cx_hybrid_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                          const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges, const int32_t* degrees,
                          const uint8_t* regs, const uint8_t* has_all, int32_t p, int64_t threshold,
                          tchll_count_result* result, void* workspace, size_t workspace_bytes, void* stream);

/* HLL.add_array (src/hll.py:93-96): max-merge the registers of n int64 values
 * into one row of 2^p registers. */
int tchll_hll_add(uint8_t* regs, int32_t p, const int64_t* values, int64_t n, void* stream);

/*
 * Estimates for n_pairs pairs of rows: out[i] = estimate of the register-wise
 * max of rows[a[i]] and rows[b[i]] (union_estimate, src/hll.py:112-120), or of
 * rows[a[i]] alone when b is NULL or b[i] < 0 (HLL.estimate, src/hll.py:98-100).
 */
int tchll_hll_estimate_pairs(const uint8_t* rows, int64_t n_rows, int32_t p, const int64_t* a, const int64_t* b,
                             int64_t n_pairs, double* out, void* stream);

/* _hash64 (src/hll.py:13-19) of n int64 values. */
int tchll_hash64(const int64_t* values, int64_t n, uint64_t* out, void* stream);

/* ------------------------------------------------------------ batched --- */
/*
 * Many graphs in one launch (no counterpart in the reference, which counts
 * one graph per call).  The graphs share one CSR with disjoint vertex ranges
 * [graph_vbase[g], graph_vbase[g+1]) -- offset each graph's ids before
 * tchll_csr_build_phase1 and take the ranges from the compacted node table --
 * and edge_u/edge_v must be the CSR's own edge list (graph g's edges are
 * positions [row_ptr[vbase[g]], row_ptr[vbase[g+1]])).  results[n_graphs]
 * receives one tchll_count_result per graph, bit-identical to counting that
 * graph alone (an edge outside its graph's range sets status on that graph).
 * Work is a device-built list of chunks that never cross a graph, claimed by
 * one persistent launch.
 */
int tchll_batch_workspace_bytes(int64_t n_nodes, int64_t n_edges, int64_t n_graphs, size_t* bytes);
int tchll_batch_exact_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                            const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                            const int32_t* graph_vbase, int64_t n_graphs, tchll_count_result* results,
                            void* workspace, size_t workspace_bytes, void* stream);
/* Hybrid per graph (split exact / HLL launches, compact sketches). */
int tchll_batch_hybrid_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                             const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges, const int32_t* degrees,
                             const uint8_t* rows, int64_t n_rows, const int64_t* slot, int32_t p, int64_t gamma,
                             const int32_t* graph_vbase, int64_t n_graphs, tchll_count_result* results,
                             void* workspace, size_t workspace_bytes, void* stream);
/* local_ids[v] = v - graph_vbase[g] for v in graph g (v outside every range
 * keeps v): the key table for tchll_build_sketches_compact that makes batched
 * sketches hash the same ids as each graph's own CSR. */
int tchll_batch_local_ids(const int32_t* graph_vbase, int64_t n_graphs, int64_t n_nodes, int64_t* local_ids,
                          void* stream);

/*
 * Degree statistics (experiment/gpu_graph_stats.py:100-140): over vertices of
 * positive degree (degrees[v], or row_ptr[v+1]-row_ptr[v] when degrees is
 * NULL), sums3 = {count, sum d, sum d^2}, minmax2 = {max, min}, and
 * log_hist32[b] = number with floor(log2 d) == b (b capped at 31).
 */
int tchll_degree_stats(const int32_t* degrees, const int32_t* row_ptr, int64_t n, uint64_t* log_hist32,
                       uint64_t* sums3, int32_t* minmax2, void* stream);

/* -------------------------------------------------- CSR construction --- */
/*
 * Edge list -> oriented CSR, the array form of orient_graph + to_csr_numpy
 * (src/graph.py:29-61, src/gpu_graph.py:6-41) as vectorised in
 * experiment/exp_gpu.py:317-365: canonical (min,max) pairs, self-loops and
 * duplicates dropped, ids compacted to the rank among all endpoint ids,
 * undirected degree, orientation u->v iff (deg u, id u) < (deg v, id v),
 * rows sorted.  Two phases sharing one workspace:
 *   phase 1 writes sizes[0] = n_nodes, sizes[1] = n_edges (device int64[2]);
 *   phase 2 (after the caller has read the sizes and allocated the outputs)
 *   writes row_ptr[n_nodes+1], col_idx/edge_u/edge_v[n_edges],
 *   degrees (forward)[n_nodes], node_ids (original id)[n_nodes] and, when
 *   undirected_degrees is not NULL, the undirected degree[n_nodes]
 *   (orient_graph's degree dict, src/graph.py:41-44).
 * Negative ids are TCHLL_EINVAL via sizes[0] = -1.  Phase 1 waits for the
 * stream once, early, to read the largest id (16 bytes): it sets the width of
 * the sort keys and, when ids 0 .. max fit twice n_raw entries, lets a direct
 * rank table replace the sort of all endpoints.
 */
int tchll_csr_workspace_bytes(int64_t n_raw, size_t* bytes);
int tchll_csr_build_phase1(const int32_t* raw_u, const int32_t* raw_v, int64_t n_raw, int64_t* sizes,
                           void* workspace, size_t workspace_bytes, void* stream);
int tchll_csr_build_phase2(int64_t n_raw, int64_t n_nodes, int64_t n_edges, int32_t* row_ptr, int32_t* col_idx,
                           int32_t* degrees, int32_t* node_ids, int32_t* edge_u, int32_t* edge_v,
                           int32_t* undirected_degrees, void* workspace, size_t workspace_bytes, void* stream);

/*
 * forward_adj -> CSR, the device form of to_csr_numpy (src/gpu_graph.py:6-41):
 * keys[n] (dict order), row lengths lens[n] and the concatenated neighbour
 * values[nnz] (dict order).  Rows are emitted in ascending key order, each
 * value replaced by the rank of its key; sizes: node_ids[n], row_ptr[n+1],
 * degrees[n], col_idx/edge_u/edge_v[nnz], order[n] = dict position of each
 * emitted row.  *missing (device int64) counts values that are not keys (the
 * reference raises KeyError).
 */
int tchll_adj_workspace_bytes(int64_t n, int64_t nnz, size_t* bytes);
int tchll_csr_from_adjacency(const int64_t* keys, const int64_t* lens, int64_t n, const int64_t* values,
                             int64_t nnz, int64_t* node_ids, int32_t* row_ptr, int32_t* degrees, int32_t* col_idx,
                             int32_t* edge_u, int32_t* edge_v, int64_t* order, int64_t* missing, void* workspace,
                             size_t workspace_bytes, void* stream);

/* ------------------------------------------------------ text ingest --- */
/*
 * Parse whitespace-separated edge-list text (text: device bytes) the way
 * load_edgelist / the experiment loader read files (src/graph.py:8-26,
 * experiment/exp_gpu.py:131-144): stripped lines, empty lines and lines whose
 * first character is in comment_chars (host C string) skipped, lines with
 * fewer than two tokens skipped, first two tokens parsed as integers.  Pairs
 * go to out_u/out_v (capacity n_bytes / 4 + 2 suffices: every kept line takes
 * at least four bytes, the last three); *n_out (device int64) receives their
 * number and *n_bad the lines whose tokens are not int32 integers (the
 * reference raises ValueError on those).  Self-loops are kept (the CSR
 * builder drops them).  Synchronises `stream` once.
 */
int tchll_ingest_workspace_bytes(int64_t n_bytes, size_t* bytes);
int tchll_parse_edges(const uint8_t* text, int64_t n_bytes, const char* comment_chars, int32_t* out_u, int32_t* out_v,
                      int64_t* n_out, int64_t* n_bad, void* workspace, size_t workspace_bytes, void* stream);

/* ------------------------------------------------ synthetic generators --- */
/* Seeded generators (no counterpart in the reference, which reads SNAP
 * files); key(seed,s) = mix((seed+1)*G ^ s*C), draw(key,i) = mix(key+(i+1)*G),
 * mix = splitmix64 finaliser.  Thresholds are probabilities * 2^32. */
int tchll_gen_rmat(int32_t scale, int64_t n_raw, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t seed,
                   int32_t* u, int32_t* v, void* stream);
int tchll_gen_er(int64_t n, int64_t n_raw, uint64_t seed, int32_t* u, int32_t* v, void* stream);
int64_t tchll_gen_lattice_count(int64_t rows, int64_t cols);
int tchll_gen_lattice(int64_t rows, int64_t cols, uint32_t tdiag, uint32_t tdel, uint64_t seed, int32_t* u,
                      int32_t* v, void* stream);
int tchll_gen_chung_lu(const uint64_t* cum, int64_t n, int64_t n_raw, uint64_t seed, int32_t* u, int32_t* v,
                       void* stream);

#ifdef __cplusplus
}
#endif
#endif /* TCHLL_H */
