// count.cu -- exact and hybrid (exact / HyperLogLog) triangle counting.
//
// Reference semantics (ChitandaEruQ/triangle_counting_hll):
//   exact:   T = sum over oriented edges (u,v) of |N+(u) cap N+(v)|
//            src/exact.py:48-98, src/gpu_hybrid.py:96-130,332-354
//   hybrid:  edge -> HLL iff min(d+u, d+v) >= gamma and both endpoints carry a
//            sketch (src/hybrid.py:107-115, src/gpu_hybrid.py:80-89); HLL edges
//            add clamp(d+u + d+v - |N+(u) cup N+(v)|^, 0, min(d+u, d+v))
//            (src/hybrid.py:117-126, src/gpu_hybrid.py:288-302), the union
//            estimated from the register-wise max of the two sketches with the
//            reference's bias and range corrections (src/hll.py:37-54,112-120).
//
// Design
//   * Table side / probe side.  |N+(u) cap N+(v)| is symmetric, so each exact
//     edge becomes a pair (x, y) with x the endpoint of the LONGER list: a
//     device counting sort (histogram, scan, scatter) groups the pairs by x.
//     A warp then keeps N+(x) in a private shared-memory hash table while it
//     streams the shorter N+(y) lists through it: the probe count drops from
//     sum d+(v) to sum min(d+u, d+v) (43.4 G list elements -> 11.8 G probes on
//     R-MAT scale 22).  Per-edge outputs (details) use the edges as given.
//   * One persistent launch, work stealing: a warp claims CHUNK consecutive
//     pairs with one atomicAdd and walks them 32 at a time; pairs sharing x
//     form a group and reuse the warp's table (built once per group per chunk).
//   * The table keeps one 4-byte word per slot at load <= 1/8: a key sits in
//     its home slot or, flagged there, on a second-hash walk, so a lookup is
//     one 4-byte shared load with a rare walk (the warp seldom diverges).
//   * Pairs whose x has a long list (d+(x) > hub threshold; 90% of the probes
//     on R-MAT scale 22) are counted by a CTA-wide kernel: all warps of a CTA
//     share one table of N+(x) of up to 32 KB, so long lists also get the
//     low load factor.
//   * The group's probe lists are flattened into one stream of 16-byte quads
//     dealt to the 32 lanes by a warp scan, so short and long lists keep
//     every lane busy.
//   * Tiny pairs are merged lane-locally; tables too large for a warp fall
//     back to a warp binary search.
//   * HLL edges: the warp reads both 2^p-byte register rows with 16-byte
//     loads, merges them with __vmaxu4 and accumulates sum 2^-r EXACTLY as a
//     128-bit fixed-point integer; one lane applies the FP64 corrections,
//     clamps and adds the result in 2^-32 fixed point.
//   * Every total is an integer (uint64 exact count, 128-bit fixed-point HLL
//     sum, int64 stats) added with integer atomics, so results do not depend
//     on scheduling or partitioning: they are bit-identical run to run.
#include <cub/cub.cuh>

#include <atomic>
#include <mutex>

#include "common.cuh"
#include "hll_device.cuh"

namespace tchll {

enum : int { MODE_EXACT = 0, MODE_HYBRID = 1, MODE_HYB_EXACT = 2, MODE_HYB_HLL = 3 };

enum : uint32_t {
    ST_BAD_EDGE = 1u,  // edge endpoint outside [0, n_nodes)
    ST_BAD_ROW = 2u,   // row_ptr extent outside [0, nnz] or decreasing
    ST_BAD_SLOT = 4u,  // sketch slot outside [0, n_rows)
    ST_BAD_KEY = 8u,   // neighbour id (col_idx value) outside [0, n_nodes)
};

struct CountParams {
    const int32_t* row_ptr;
    int64_t n_nodes;
    const int32_t* col_idx;
    int64_t nnz;
    const int32_t* edge_u;
    const int32_t* edge_v;
    int64_t n_edges;
    const int32_t* n_edges_dev;  // when set, the edge count is read here (pairs)
    const int32_t* degrees;      // forward degree for routing (hybrid modes)
    const uint8_t* regs;         // register rows
    int64_t n_rows;              // rows available in regs
    const int64_t* slot;         // compact layout: row of v, or -1; null -> dense
    const uint8_t* has;          // dense layout: has_sketch[v] == 1 -> row v
    int p;
    int64_t gamma;
    int variant;          // HLL estimator: 0 the reference's src/hll.py, 1 cpu_exp's
    int64_t* pe_support;  // per-edge exact support (details), zeroed by host
    double* pe_s_hat;     // per-edge HLL s_hat (details)
    double* pe_s_cl;      // per-edge HLL clamped support (details)
    uint8_t* pe_method;   // per-edge 0 exact / 1 hll (details)
    tchll_count_result* result;
    unsigned long long* work;
    int chunk;
    int slots_log2;  // per-warp table capacity (log2 slots)
    int tiny;        // lane-local merge when |N+x| + |N+y| <= tiny
    int sparse;      // 1: table load <= 1/4 where it fits (else <= 1/2)
    // Batched mode: work units are chunks [chunk_start[i], +chunk_len[i]) of
    // one graph each (never crossing a graph), claimed one at a time; each
    // chunk's totals go to results[chunk_graph[i]].
    const int64_t* chunk_start;
    const int32_t* chunk_len;
    const int32_t* chunk_graph;
    const int64_t* n_chunks_dev;
    const int32_t* graph_vbase;  // vertex range of graph g: [vbase[g], vbase[g+1])
    int64_t n_graphs;            // batched calls: graphs in graph_vbase (else 0)
    // Hybrid with pairs: the routing pass appends HLL edges here
    int32_t* hll_u;
    int32_t* hll_v;
    unsigned long long* hll_n;
};

// Hash table of one 4-byte word per slot (per-warp tables of the pair kernel
// and the CTA tables of the hub kernel): bits 0-30 the key (0x7FFFFFFF =
// empty; vertex ids stay below INT32_MAX) and bit 31 an overflow flag.  A
// key lives in its home slot h1(k) when that was free at insertion; otherwise
// it sets the flag on h1(k) and takes the first free slot of a linear walk
// from h2(k).  A lookup reads the home slot: match -> hit; flag clear ->
// miss; flag set (about load^2 of the slots) -> walk from h2(k) to the key or
// a free slot.  At load <= 1/8 almost every lookup is ONE 4-byte shared load
// and the warp rarely diverges.
constexpr uint32_t OV_KEY = 0x7FFFFFFFu;   // key bits; this value marks an empty slot
constexpr uint32_t OV_FLAG = 0x80000000u;  // some key of this home slot lives on its h2 walk
constexpr uint32_t OV_NONE = 0x7FFFFFFEu;  // probe that matches no slot (vertex ids are below it)

__device__ __forceinline__ uint32_t ov_h1(int32_t x, int sh) { return ((uint32_t)x * 0x9E3779B1u) >> sh; }
__device__ __forceinline__ uint32_t ov_h2(int32_t x, int sh) { return ((uint32_t)x * 0x85EBCA77u) >> sh; }

// Claims slot h for key x if its key bits are empty (keeps the flag bit).
// Returns 1 placed, 0 occupied by another key, 2 already holds x.
__device__ __forceinline__ int ov_claim(uint32_t* T, uint32_t h, uint32_t x) {
    uint32_t old = *(volatile uint32_t*)(T + h);
    while ((old & OV_KEY) == OV_KEY) {
        const uint32_t prev = atomicCAS(T + h, old, (old & OV_FLAG) | x);
        if (prev == old) return 1;
        old = prev;
    }
    return (old & OV_KEY) == x ? 2 : 0;
}

// Inserts x; false only if the h2 walk finds no free slot (full table).
__device__ __forceinline__ bool ov_insert(uint32_t* T, int32_t x, int sh, uint32_t mask) {
    const uint32_t h = ov_h1(x, sh);
    if (ov_claim(T, h, (uint32_t)x)) return true;
    atomicOr(T + h, OV_FLAG);
    uint32_t g = ov_h2(x, sh);
    for (uint32_t i = 0; i <= mask; ++i) {
        if (ov_claim(T, g, (uint32_t)x)) return true;
        g = (g + 1u) & mask;
    }
    return false;
}

// The h2 walk of a lookup whose home slot was flagged: 1 at x, 0 at a free
// slot; at most mask + 1 steps.
__device__ __forceinline__ uint32_t ov_walk(const uint32_t* T, int32_t x, int sh, uint32_t mask) {
    uint32_t g = ov_h2(x, sh);
    for (uint32_t i = 0; i <= mask; ++i) {
        const uint32_t k = T[g] & OV_KEY;
        if (k == (uint32_t)x) return 1u;
        if (k == OV_KEY) return 0u;
        g = (g + 1u) & mask;
    }
    return 0u;
}

__device__ __forceinline__ int ceil_log2_i(int x) { return x <= 1 ? 0 : 32 - __clz(x - 1); }

// Loads and validates edge e; returns false (and flags status) when malformed.
__device__ __forceinline__ bool load_edge(const CountParams& P, int64_t e, int32_t& u, int32_t& v, int32_t& us,
                                          int32_t& ue, int32_t& vs, int32_t& ve, uint32_t& status) {
    // the edge arrays stream through once per pass: evict-first loads keep
    // L1 for the row_ptr entries of the high-degree endpoints, which recur
    u = __ldcs(P.edge_u + e);
    v = __ldcs(P.edge_v + e);
    if (u < 0 || v < 0 || (int64_t)u >= P.n_nodes || (int64_t)v >= P.n_nodes) {
        status |= ST_BAD_EDGE;
        return false;
    }
    us = __ldg(P.row_ptr + u);
    ue = __ldg(P.row_ptr + u + 1);
    vs = __ldg(P.row_ptr + v);
    ve = __ldg(P.row_ptr + v + 1);
    if (us < 0 || ue < us || (int64_t)ue > P.nnz || vs < 0 || ve < vs || (int64_t)ve > P.nnz) {
        status |= ST_BAD_ROW;
        return false;
    }
    return true;
}

// Hybrid routing (src/hybrid.py:107-115): wants = min(deg) >= gamma,
// both = both endpoints have a sketch.  Returns false on a bad slot.
__device__ __forceinline__ bool route(const CountParams& P, int32_t u, int32_t v, int32_t& du, int32_t& dv,
                                      int64_t& su, int64_t& sv, bool& wants, bool& both, uint32_t& status) {
    du = __ldg(P.degrees + u);
    dv = __ldg(P.degrees + v);
    const int64_t proxy = du < dv ? du : dv;
    wants = proxy >= P.gamma;
    if (P.slot) {
        su = __ldg(P.slot + u);
        sv = __ldg(P.slot + v);
    } else {
        su = __ldg(P.has + u) == 1 ? (int64_t)u : -1;
        sv = __ldg(P.has + v) == 1 ? (int64_t)v : -1;
    }
    if (su >= P.n_rows || sv >= P.n_rows) {
        status |= ST_BAD_SLOT;
        return false;
    }
    both = su >= 0 && sv >= 0;
    return true;
}

// ------------------------------------------------------------ pair build ----
// Exact edges (all edges, or in hybrid mode the exact-routed ones) become
// pairs (x, y), x the endpoint with the longer forward list (ties: u).
template <bool HYB>
__device__ __forceinline__ bool pair_of(const CountParams& P, int64_t e, int32_t& x, int32_t& y, int32_t& xl,
                                        uint32_t& status) {
    int32_t u, v, us, ue, vs, ve;
    if (!load_edge(P, e, u, v, us, ue, vs, ve, status)) return false;
    if (HYB) {
        int32_t du, dv;
        int64_t su, sv;
        bool wants, both;
        if (!route(P, u, v, du, dv, su, sv, wants, both, status)) return false;
        if (wants && both) return false;  // HLL-routed
    }
    const bool ux = (ue - us) >= (ve - vs);
    x = ux ? u : v;
    y = ux ? v : u;
    xl = ux ? (ue - us) : (ve - vs);
    return true;
}

// Batched calls: the graph of vertex v, the last g with vbase[g] <= v.
__device__ __forceinline__ int64_t graph_of(const int32_t* vbase, int64_t n_graphs, int32_t v) {
    int64_t lo = 0, hi = n_graphs - 1;
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(vbase + mid) <= v) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// Lanes whose pairs share x in a run of consecutive lanes (edges in CSR
// order share u, so the pairs with x = u come in runs): the run's first lane
// (head) and its length.  key must differ between lanes that may not merge.
// Whole warps call it (the grid-stride loops below are warp-uniform).
__device__ __forceinline__ void lane_runs(int32_t key, int lane, int& head_lane, int& run_len) {
    const int32_t prev = __shfl_up_sync(FULL, key, 1);
    const unsigned heads = __ballot_sync(FULL, lane == 0 || prev != key);
    const unsigned le = (2u << lane) - 1u;
    head_lane = 31 - __clz(heads & le);
    const unsigned after = heads & ~((2u << head_lane) - 1u);  // heads after this run's head
    run_len = (after ? __ffs(after) - 1 : 32) - head_lane;
}

// Grid-stride loop that whole warps enter and leave together: e may reach
// past n in the last pass; the body tests it.
#define WARP_EDGE_LOOP(e, n)                                                                   \
    for (int64_t _wb = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u),                \
                 e = _wb + (threadIdx.x & 31u);                                                \
         _wb < (n); _wb += (int64_t)gridDim.x * blockDim.x, e = _wb + (threadIdx.x & 31u))

template <bool HYB>
__global__ void pair_hist_kernel(const CountParams P, int32_t* cnt) {
    uint32_t status = 0;
    unsigned long long fallback = 0;
    const int lane = threadIdx.x & 31;
    WARP_EDGE_LOOP(e, P.n_edges) {
        int32_t u = 0, v = 0, us = 0, ue = 0, vs = 0, ve = 0;
        bool ok = e < P.n_edges && load_edge(P, e, u, v, us, ue, vs, ve, status);
        bool hll = false;
        if (HYB && ok) {
            int32_t du, dv;
            int64_t su, sv;
            bool wants, both;
            ok = route(P, u, v, du, dv, su, sv, wants, both, status);
            hll = ok && wants && both;
            if (ok && wants && !both) {
                if (P.graph_vbase && P.hll_u)  // batched: this edge's graph
                    atomicAdd((unsigned long long*)&P.result[graph_of(P.graph_vbase, P.n_graphs, u)].n_fallback, 1ull);
                else
                    ++fallback;
            }
        }
        {
            // a run of lanes with the same table side adds with one atomic
            const bool counted = ok && !hll;
            const int32_t x = counted ? (((ue - us) >= (ve - vs)) ? u : v) : -1 - lane;
            int head, len;
            lane_runs(x, lane, head, len);
            if (counted && lane == head) atomicAdd(cnt + x, len);
        }
        if (HYB && P.hll_u) {
            // warp-aggregated append of the HLL-routed edges
            const unsigned bal = __ballot_sync(FULL, hll);
            if (bal) {
                unsigned long long base = 0;
                if (lane == 0) base = atomicAdd(P.hll_n, (unsigned long long)__popc(bal));
                base = __shfl_sync(FULL, base, 0);
                if (hll) {
                    const unsigned long long pos = base + __popc(bal & ((1u << lane) - 1u));
                    P.hll_u[pos] = u;
                    P.hll_v[pos] = v;
                }
            }
        }
    }
    if (status) atomicOr(&P.result->status, status);
    if (HYB && P.hll_u && fallback) atomicAdd((unsigned long long*)&P.result->n_fallback, fallback);
}

// Small pairs go to [cursor[x]...) of px / py; with hub > 0, pairs whose x
// has d+(x) > hub go to the hub list, py[*n_small + cursorh[x]...] (y only).
template <bool HYB>
__global__ void pair_scatter_kernel(const CountParams P, int32_t* cursor, int32_t* cursorh, int hub,
                                    const int32_t* n_small, int32_t* px, int32_t* py) {
    uint32_t status = 0;
    const int lane = threadIdx.x & 31;
    const int64_t hbase = hub > 0 ? (int64_t)*n_small : 0;
    WARP_EDGE_LOOP(e, P.n_edges) {
        int32_t x = 0, y = 0, xl = 0;
        const bool ok = e < P.n_edges && pair_of<HYB>(P, e, x, y, xl, status);
        // a run of lanes with the same x claims its positions with one
        // atomic (x's list length, hence its list, is the same for all)
        int head, len;
        lane_runs(ok ? x : -1 - lane, lane, head, len);
        const bool to_hub = hub > 0 && xl > hub;
        int32_t base = 0;
        if (ok && lane == head) base = atomicAdd((to_hub ? cursorh : cursor) + x, len);
        base = __shfl_sync(FULL, base, head);
        if (ok) {
            const int32_t pos = base + (lane - head);
            if (to_hub) {
                py[hbase + pos] = y;
            } else {
                px[pos] = x;
                py[pos] = y;
            }
        }
    }
    (void)status;
}

// Warp-cooperative binary-search intersection count of two sorted lists in
// global memory (tables too large for a warp).  Per-lane partial counts.
__device__ __forceinline__ uint32_t warp_bsearch_count(const int32_t* a, int la, const int32_t* b, int lb, int lane) {
    if (la > lb) {
        const int32_t* t = a;
        a = b;
        b = t;
        const int tl = la;
        la = lb;
        lb = tl;
    }
    uint32_t c = 0;
    for (int i = lane; i < la; i += 32) {
        const int32_t x = __ldg(a + i);
        int lo = 0, hi = lb;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (__ldg(b + mid) < x) lo = mid + 1; else hi = mid;
        }
        c += (lo < lb && __ldg(b + lo) == x);
    }
    return c;
}

__device__ __forceinline__ uint32_t lane_merge_count(const int32_t* a, int la, const int32_t* b, int lb) {
    int i = 0, j = 0;
    uint32_t c = 0;
    while (i < la && j < lb) {
        const int32_t x = __ldg(a + i), y = __ldg(b + j);
        c += (x == y);
        i += (x <= y);
        j += (y <= x);
    }
    return c;
}

// Warp-reduces the per-lane totals and adds them to *R (lane 0, integer
// atomics; order-independent).
__device__ __forceinline__ void publish(tchll_count_result* R, uint64_t acc, U128 hacc, int64_t n_approx,
                                        int64_t n_exact, int64_t n_fallback, int64_t n_clamped, uint32_t status,
                                        int lane) {
    acc = warp_sum_u64(acc);
    hacc = warp_sum_u128(hacc);  // sub-warp HLL groups each hold their own sum
    n_approx = warp_sum_i64(n_approx);
    n_exact = warp_sum_i64(n_exact);
    n_fallback = warp_sum_i64(n_fallback);
    n_clamped = warp_sum_i64(n_clamped);
    status = __reduce_or_sync(FULL, status);
    if (lane == 0) {
        if (acc) atomicAdd((unsigned long long*)&R->exact, (unsigned long long)acc);
        atomic_add_u128((unsigned long long*)&R->hll_fx_lo, hacc);
        if (n_approx) atomicAdd((unsigned long long*)&R->n_approx, (unsigned long long)n_approx);
        if (n_exact) atomicAdd((unsigned long long*)&R->n_exact, (unsigned long long)n_exact);
        if (n_fallback) atomicAdd((unsigned long long*)&R->n_fallback, (unsigned long long)n_fallback);
        if (n_clamped) atomicAdd((unsigned long long*)&R->n_clamped, (unsigned long long)n_clamped);
        if (status) atomicOr(&R->status, status);
    }
}

template <int MODE, bool VEC, bool DETAILS>
__global__ void __launch_bounds__(256, 4) count_kernel(const CountParams P) {
    extern __shared__ __align__(16) int32_t smem[];
    const int lane = threadIdx.x & 31;
    const int wid = threadIdx.x >> 5;
    const int cap_lg = P.slots_log2;
    const int cap_keys = 1 << (cap_lg - 1);  // load <= 1/2 in 2^cap_lg slots
    uint32_t* table = reinterpret_cast<uint32_t*>(smem) + ((size_t)wid << cap_lg);

    const int32_t* __restrict__ col_idx = P.col_idx;
    const int64_t n_edges = P.n_edges_dev ? (int64_t)*P.n_edges_dev : P.n_edges;

    uint64_t acc = 0;
    U128 hacc;
    int64_t n_approx = 0, n_exact = 0, n_fallback = 0, n_clamped = 0;
    uint32_t status = 0;
    int cur_u = -1;
    int cur_lg = 5;  // log2 slots of the current table
    const int m = 1 << P.p;

    while (true) {
        unsigned long long e0 = 0;
        int64_t e1;
        int32_t gcur = -1;
        if (P.chunk_start) {
            unsigned long long ci = 0;
            if (lane == 0) ci = atomicAdd(P.work, 1ull);
            ci = __shfl_sync(FULL, ci, 0);
            if ((int64_t)ci >= *P.n_chunks_dev) break;
            e0 = (unsigned long long)__ldg(P.chunk_start + ci);
            e1 = (int64_t)e0 + __ldg(P.chunk_len + ci);
            gcur = __ldg(P.chunk_graph + ci);
        } else {
            if (lane == 0) e0 = atomicAdd(P.work, (unsigned long long)P.chunk);
            e0 = __shfl_sync(FULL, e0, 0);
            if (e0 >= (unsigned long long)n_edges) break;
            e1 = min((int64_t)e0 + P.chunk, n_edges);
        }
        for (int64_t eb = (int64_t)e0; eb < e1; eb += 32) {
            const int64_t e = eb + lane;
            int32_t u = 0, v = 0, us = 0, ue = 0, vs = 0, ve = 0;
            bool valid = e < e1 && load_edge(P, e, u, v, us, ue, vs, ve, status);
            if (valid && gcur >= 0) {
                // an edge of another graph inside this graph's chunk
                const int32_t lo_v = __ldg(P.graph_vbase + gcur), hi_v = __ldg(P.graph_vbase + gcur + 1);
                if (u < lo_v || u >= hi_v || v < lo_v || v >= hi_v) {
                    status |= ST_BAD_EDGE;
                    valid = false;
                }
            }
            bool is_hll = false;
            int64_t slot_u = -1, slot_v = -1;
            int32_t du = 0, dv = 0;
            if (MODE != MODE_EXACT && valid) {
                bool wants, both;
                valid = route(P, u, v, du, dv, slot_u, slot_v, wants, both, status);
                is_hll = valid && wants && both;
                // n_fallback: counted by the fused launch and, in split mode,
                // by the HLL launch (which sees every edge in both variants)
                if (MODE != MODE_HYB_EXACT && valid && wants && !both) ++n_fallback;
            }
            const bool do_exact = valid && !is_hll && MODE != MODE_HYB_HLL;
            const bool do_hll = valid && is_hll && MODE != MODE_HYB_EXACT;
            n_exact += do_exact;

            // ---------------------------------------------------- exact part
            const int lu = ue - us, lv = ve - vs;
            const bool tiny = do_exact && (lu + lv <= P.tiny || lu == 0 || lv == 0);
            if (tiny) {
                const uint32_t c = (lu && lv) ? lane_merge_count(col_idx + us, lu, col_idx + vs, lv) : 0u;
                acc += c;
                if (DETAILS) P.pe_support[e] = c;
            }
            unsigned pend = __ballot_sync(FULL, do_exact && !tiny);
            while (pend) {
                const int lead = __ffs(pend) - 1;
                const int32_t ucur = __shfl_sync(FULL, u, lead);
                const unsigned grp = __ballot_sync(FULL, ((pend >> lane) & 1u) && u == ucur);
                pend &= ~grp;
                const int32_t gus = __shfl_sync(FULL, us, lead);
                const int32_t gdu = __shfl_sync(FULL, lu, lead);
                const bool in = (grp >> lane) & 1u;
                if (gdu > cap_keys) {
                    // table side too long for a warp table: binary search per edge
                    unsigned g = grp;
                    while (g) {
                        const int j = __ffs(g) - 1;
                        g &= g - 1;
                        const int32_t jvs = __shfl_sync(FULL, vs, j);
                        const int32_t jlv = __shfl_sync(FULL, lv, j);
                        const uint32_t c = warp_bsearch_count(col_idx + gus, gdu, col_idx + jvs, jlv, lane);
                        acc += c;
                        if (DETAILS) {
                            const uint32_t tot = (uint32_t)warp_sum_u64(c);
                            const int64_t ej = __shfl_sync(FULL, e, j);
                            if (lane == 0) P.pe_support[ej] = tot;
                        }
                    }
                    continue;
                }
                if (ucur != cur_u) {
                    // (re)build the warp's table for N+(ucur): 2^lgs slots,
                    // load <= 1/8 (1/16 sparse) when the capacity allows,
                    // <= 1/2 always
                    int lgs = ceil_log2_i(gdu) + (P.sparse ? 4 : 3);
                    lgs = lgs < 5 ? 5 : (lgs > cap_lg ? cap_lg : lgs);
                    const int nslots = 1 << lgs;
                    __syncwarp();
                    for (int i = lane; i < (nslots >> 2); i += 32)
                        reinterpret_cast<uint4*>(table)[i] = make_uint4(OV_KEY, OV_KEY, OV_KEY, OV_KEY);
                    __syncwarp();
                    bool ok = true;
                    for (int i = lane; i < gdu; i += 32)
                        ok &= ov_insert(table, __ldg(col_idx + gus + i), 32 - lgs, (uint32_t)nslots - 1u);
                    __syncwarp();
                    if (!__all_sync(FULL, ok)) {
                        // no free slot (cannot happen at load <= 1/2): binary search for this group
                        cur_u = -1;
                        unsigned g = grp;
                        while (g) {
                            const int j = __ffs(g) - 1;
                            g &= g - 1;
                            const int32_t jvs = __shfl_sync(FULL, vs, j);
                            const int32_t jlv = __shfl_sync(FULL, lv, j);
                            const uint32_t c = warp_bsearch_count(col_idx + gus, gdu, col_idx + jvs, jlv, lane);
                            acc += c;
                            if (DETAILS) {
                                const uint32_t tot = (uint32_t)warp_sum_u64(c);
                                const int64_t ej = __shfl_sync(FULL, e, j);
                                if (lane == 0) P.pe_support[ej] = tot;
                            }
                        }
                        continue;
                    }
                    cur_u = ucur;
                    cur_lg = lgs;
                }
                const int sh = 32 - cur_lg;
                const uint32_t tmask = (1u << cur_lg) - 1u;
                // flatten the group's probe lists into quads
                int q0, nq;
                if (VEC) {
                    q0 = vs >> 2;
                    nq = (in && ve > vs) ? ((ve - 1) >> 2) - q0 + 1 : 0;
                } else {
                    q0 = vs;
                    nq = in ? (ve - vs) : 0;
                }
                const unsigned ne = __ballot_sync(FULL, nq > 0);
                const int k = __popc(ne);
                const int src = lane < k ? (int)__fns(ne, 0, lane + 1) : lane;
                const int c_q0 = __shfl_sync(FULL, q0, src);
                int c_nq = __shfl_sync(FULL, nq, src);
                const int32_t c_vs = __shfl_sync(FULL, vs, src);
                const int32_t c_ve = __shfl_sync(FULL, ve, src);
                int64_t c_e = 0;
                if (DETAILS) c_e = __shfl_sync(FULL, e, src);
                if (lane >= k) c_nq = 0;
                int incl = c_nq;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int t = __shfl_up_sync(FULL, incl, o);
                    if (lane >= o) incl += t;
                }
                const int excl = incl - c_nq;
                const int W = __shfl_sync(FULL, incl, 31);
                const int qb = c_q0 - excl;
                // Windows of 32 quads; UNR windows are mapped, loaded and then
                // probed together so each lane has UNR 16-byte loads in flight.
                constexpr int UNR = VEC ? 4 : 2;
                for (int T0 = 0; T0 < W; T0 += 32 * UNR) {
                    int qd[UNR], lo[UNR], hi[UNR];
                    int64_t my_e[UNR];
#pragma unroll
                    for (int i = 0; i < UNR; ++i) {
                        const int Ti = T0 + 32 * i;
                        qd[i] = -1;
                        lo[i] = hi[i] = 0;
                        my_e[i] = 0;
                        if (Ti < W) {  // warp-uniform
                            const unsigned cover = __ballot_sync(FULL, lane < k && excl <= Ti && Ti < incl);
                            const int b = __ffs(cover) - 1;
                            const unsigned bit =
                                (lane < k && excl > Ti && excl < Ti + 32) ? (1u << (excl - Ti)) : 0u;
                            const unsigned B = __reduce_or_sync(FULL, bit);
                            const int j = (b + __popc(B & ((2u << lane) - 1u))) & 31;
                            const int my_qb = __shfl_sync(FULL, qb, j);
                            const int32_t my_vs = __shfl_sync(FULL, c_vs, j);
                            const int32_t my_ve = __shfl_sync(FULL, c_ve, j);
                            if (DETAILS) my_e[i] = __shfl_sync(FULL, c_e, j);
                            if (Ti + lane < W) {
                                qd[i] = my_qb + Ti + lane;
                                const int base = VEC ? qd[i] * 4 : qd[i];
                                lo[i] = my_vs - base;  // valid elements of the quad: [lo, hi)
                                hi[i] = my_ve - base;
                            }
                        }
                    }
                    int4 val[UNR];
#pragma unroll
                    for (int i = 0; i < UNR; ++i) {
                        val[i] = make_int4(-1, -1, -1, -1);
                        if (qd[i] >= 0) {
                            if (VEC) {
                                const int base = qd[i] * 4;
                                if ((int64_t)base + 3 < P.nnz) {
                                    val[i] = __ldg(reinterpret_cast<const int4*>(col_idx) + qd[i]);
                                } else {
                                    val[i].x = base + 0 < P.nnz ? __ldg(col_idx + base + 0) : -1;
                                    val[i].y = base + 1 < P.nnz ? __ldg(col_idx + base + 1) : -1;
                                    val[i].z = base + 2 < P.nnz ? __ldg(col_idx + base + 2) : -1;
                                    val[i].w = base + 3 < P.nnz ? __ldg(col_idx + base + 3) : -1;
                                }
                            } else {
                                val[i].x = __ldg(col_idx + qd[i]);
                            }
                        }
                    }
                    // home slots of every key first (branch-free; elements
                    // outside the pair's list probe as OV_NONE), then the
                    // rare walks of flagged homes
                    constexpr int KPQ = VEC ? 4 : 1;  // keys per quad
                    uint32_t key[KPQ * UNR];
#pragma unroll
                    for (int i = 0; i < UNR; ++i) {
                        // mapped quads have lo <= KPQ - 1 and hi >= 1; unmapped: lo = hi = 0
                        key[KPQ * i + 0] = (lo[i] <= 0 && hi[i] > 0) ? (uint32_t)val[i].x : OV_NONE;
                        if (VEC) {
                            key[KPQ * i + 1] = (lo[i] <= 1 && hi[i] > 1) ? (uint32_t)val[i].y : OV_NONE;
                            key[KPQ * i + 2] = (lo[i] <= 2 && hi[i] > 2) ? (uint32_t)val[i].z : OV_NONE;
                            key[KPQ * i + 3] = (lo[i] <= 3 && hi[i] > 3) ? (uint32_t)val[i].w : OV_NONE;
                        }
                    }
                    const uint32_t* T = table;
                    uint32_t cq[UNR], pend = 0;
#pragma unroll
                    for (int i = 0; i < UNR; ++i) {
                        cq[i] = 0;
#pragma unroll
                        for (int j = 0; j < KPQ; ++j) {
                            const int t = KPQ * i + j;
                            const uint32_t d = T[ov_h1((int32_t)key[t], sh)] ^ key[t];
                            cq[i] += (d << 1) == 0u;
                            pend |= (d > OV_FLAG ? 1u : 0u) << t;
                        }
                    }
                    if (pend) {
#pragma unroll
                        for (int i = 0; i < UNR; ++i)
#pragma unroll
                            for (int j = 0; j < KPQ; ++j)
                                if ((pend >> (KPQ * i + j)) & 1u)
                                    cq[i] += ov_walk(T, (int32_t)key[KPQ * i + j], sh, tmask);
                    }
#pragma unroll
                    for (int i = 0; i < UNR; ++i) {
                        acc += cq[i];
                        if (DETAILS && cq[i])
                            atomicAdd((unsigned long long*)(P.pe_support + my_e[i]), (unsigned long long)cq[i]);
                    }
                }
            }

            // ------------------------------------------------------ HLL part
            if (MODE != MODE_EXACT && MODE != MODE_HYB_EXACT) {
                unsigned hm = __ballot_sync(FULL, do_hll);
                while (hm) {
                    const int j = __ffs(hm) - 1;
                    hm &= hm - 1;
                    const int64_t su = __shfl_sync(FULL, slot_u, j);
                    const int64_t sv = __shfl_sync(FULL, slot_v, j);
                    const int32_t jdu = __shfl_sync(FULL, du, j);
                    const int32_t jdv = __shfl_sync(FULL, dv, j);
                    const uint8_t* ra = P.regs + su * (int64_t)m;
                    const uint8_t* rb = P.regs + sv * (int64_t)m;
                    const double E = warp_union_estimate<VEC>(ra, rb, P.p, lane, P.variant);
                    if (lane == 0) {
                        const double s_hat = (double)((int64_t)jdu + (int64_t)jdv) - E;
                        const double upper = (double)(jdu < jdv ? jdu : jdv);
                        // max(0.0, min(s_hat, upper)) with Python's min/max
                        // argument order (src/hybrid.py:122)
                        double s_cl = (upper < s_hat) ? upper : s_hat;
                        s_cl = (s_cl > 0.0) ? s_cl : 0.0;
                        if (s_hat < 0.0 || s_hat > upper) ++n_clamped;
                        ++n_approx;
                        hacc.add((uint64_t)__double2ull_rn(s_cl * 4294967296.0));
                        if (DETAILS) {
                            const int64_t ej = eb + j;
                            P.pe_s_hat[ej] = s_hat;
                            P.pe_s_cl[ej] = s_cl;
                            P.pe_method[ej] = 1;
                        }
                    }
                }
            }
        }
        if (gcur >= 0) {  // batched: this chunk's totals belong to graph gcur
            publish(P.result + gcur, acc, hacc, n_approx, n_exact, n_fallback, n_clamped, status, lane);
            acc = 0;
            hacc = U128();
            n_approx = n_exact = n_fallback = n_clamped = 0;
            status = 0;
        }
    }

    // ---------------------------------------------------------- publish ----
    if (!P.chunk_start) publish(P.result, acc, hacc, n_approx, n_exact, n_fallback, n_clamped, status, lane);
}

// ------------------------------------------------------------ hub pairs ----
// Pairs whose table side x has a long forward list (d+(x) > hub threshold)
// carry most of the probe work on skewed graphs (R-MAT scale 22: 90% of the
// sum of min(d+u, d+v) has d+(x) > 256).  They are counted one x at a time
// by a whole CTA: the CTA builds ONE table of N+(x) in shared memory at load
// <= 1/8 (up to 2^hub_lg slots) and its warps stream the probe lists of x's
// pairs through it (a per-warp table of 8 KB would hold N+(x) only at load
// up to 1/2, where the overflow walks of the one-load table grow).
struct HubSeg {
    int32_t start;  // first pair in the hub list (pair lists hold < 2^31 entries)
    int32_t x;
    int32_t len;
    int32_t graph;  // batched counts: the graph of x (its result block); else 0
};

struct HubParams {
    const int32_t* row_ptr;
    int64_t n_nodes;
    const int32_t* col_idx;
    int64_t nnz;
    const int32_t* hy;  // y of each hub pair, grouped by x
    const int32_t* pcol;  // padded lists in core coordinates (core_pad_kernel) or null: raw lists
    const int32_t* cidx;  // core index of each vertex, -1 outside the core (with pcol)
    const int32_t* n_core;  // device: core size C, vertex of core index kPlane (with pcol)
    const int4* pl;         // packed lists per row: {first 16-byte unit, plane-0 units, all units, 0}
    int packed;             // packed 16-bit lists when C <= kCore16Max
    const HubSeg* segs;
    const unsigned long long* n_segs;
    int64_t max_segs;
    unsigned long long* seg_ctr;
    int hub_lg;    // log2 of the largest hash table (slots)
    int cap_bits;  // bitmap kernel: bits its shared buffer holds
    bool batched;  // publish per segment into result[segment graph]
    tchll_count_result* result;
};

// The hub core.  Every key that can match a hub table lies in the forward
// list of some table side x that has hub pairs; call the union of those
// lists the core (R-MAT scale 22: 108 K of 2.4 M vertices, because
// orientation by (degree, id) puts every long list's members among the
// highest-degree vertices).  The hub kernels work in core coordinates:
//   * cidx[w] = rank of w among the core vertices (ascending id), else -1;
//   * each probe list is rewritten in core indices, a member outside the
//     core becoming the sentinel C (the core size), which can never hit;
//   * a table side's list becomes a C-bit bitmap in shared memory (13.5 KB
//     on R-MAT scale 22), so a probe is one shift, one 4-byte shared load
//     and one funnel shift.
// Counts are unchanged: |N+(x) cap N+(y)| = |cidx(N+(x)) cap cidx(N+(y) cap
// core)| because N+(x) lies inside the core and cidx is one-to-one there.
//
// Padded probe lists: row y's list starts at element pad_start(y), a
// multiple of 4, and is followed by the sentinel up to the next multiple of
// 4, so every 16-byte quad holds only the list's keys or the sentinel and no
// probe needs a mask.  pad_start(y) = roundup4(row_ptr[y]) + 8 y leaves room
// for the padding of every row before y (at most 3 per row) without a scan.
__device__ __forceinline__ int64_t pad_start(int32_t rs, int32_t y) {
    return (((int64_t)rs + 3) & ~(int64_t)3) + 8 * (int64_t)y;
}

// flag[w] = 1 for every w in N+(x) of every x with hub pairs: one warp per
// hub segment (a segment names its x; the segments of one x are consecutive,
// and only the first marks x's list).  Going by segments rather than by
// vertex id keeps the warps balanced: hub vertices cluster at low ids in
// R-MAT graphs.  Each lane has four list members in flight (the loop is
// bound by the latency of the dependent flag reads, not by bandwidth).
// Values outside [0, n_nodes) are reported, not stored.
__global__ void core_mark_kernel(const int32_t* __restrict__ row_ptr, int64_t n_nodes, int64_t nnz,
                                 const int32_t* __restrict__ col, const HubSeg* __restrict__ segs,
                                 const unsigned long long* __restrict__ n_segs, int64_t max_segs, int32_t* flag,
                                 tchll_count_result* result) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t nseg = min((int64_t)*n_segs, max_segs);
    uint32_t status = 0;
    for (int64_t sg = warp; sg < nseg; sg += nwarps) {
        const int32_t x = segs[sg].x;
        if (sg > 0 && segs[sg - 1].x == x) continue;  // x's first segment marks its list
        if (x < 0 || (int64_t)x >= n_nodes) {  // warp-uniform; cannot happen
            status |= ST_BAD_EDGE;
            continue;
        }
        const int32_t s = __ldg(row_ptr + x), e = __ldg(row_ptr + x + 1);
        if (s < 0 || e < s || (int64_t)e > nnz) {
            status |= ST_BAD_ROW;
            continue;
        }
        for (int32_t i0 = s; i0 < e; i0 += 128) {
            int32_t w[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int32_t i = i0 + 32 * k + lane;
                w[k] = i < e ? __ldg(col + i) : -1;
                if (i < e && (uint64_t)(uint32_t)w[k] >= (uint64_t)n_nodes) {
                    status |= ST_BAD_KEY;
                    w[k] = -1;
                }
            }
            // the core's members recur in many hub lists: read first, and
            // store only a flag not yet seen set (a stale 0 read just
            // repeats an idempotent store)
            int32_t f[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) f[k] = w[k] >= 0 ? flag[w[k]] : 1;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (f[k] == 0) flag[w[k]] = 1;
        }
    }
    status = __reduce_or_sync(FULL, status);
    if (lane == 0 && status) atomicOr(&result->status, status);
}

// Packed probe lists hold a core index in 16 bits plus a plane: plane 0 the
// indices below kPlane, plane 1 the others minus kPlane, each plane padded
// with 0xFFFF.  In the bitmap, core index c sits at bit c (plane 0) or c + 1
// (plane 1), so bit 65535 (plane 0's padding) and bit 131071 (plane 1's) are
// never set; that works while C <= kCore16Max.
constexpr int32_t kPlane = 65535;
constexpr int32_t kCore16Max = 131070;

// n_core[1] (set to -1 before) receives the vertex of core index kPlane.
__global__ void core_index_kernel(int32_t* flag_cidx, const int32_t* __restrict__ pos, int64_t n_nodes,
                                  int32_t* n_core) {
    for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w <= n_nodes;
         w += (int64_t)gridDim.x * blockDim.x) {
        if (w == n_nodes) {
            n_core[0] = __ldg(pos + n_nodes);
        } else {
            const bool f = flag_cidx[w] != 0;
            const int32_t c = __ldg(pos + w);
            flag_cidx[w] = f ? c : -1;
            if (f && c == kPlane) n_core[1] = (int32_t)w;
        }
    }
}

// Packed probe lists (used when C <= kCore16Max; core_pad_kernel writes the
// 32-bit ones otherwise): row y starts at uint16 index pad16_start(y), a
// multiple of 8 (16 bytes); plane 0 (members below the vertex of core index
// kPlane) takes lo_units 16-byte units, plane 1 the next ones; pl[y] =
// {pad16_start(y) / 8, lo_units, all units, 0}, one 16-byte record so that
// the hub kernel finds a pair's list with one load.  roundup8(row_ptr[y]) +
// 24 y leaves room for both planes' padding (at most 7 each) of every row
// before y.  Rows are sorted (as every CSR of the reference is), so the
// planes split the row at one position P, found by an 8-way search down to
// 64 members and a count of those; a member on the wrong side of P (an
// unsorted row) or outside the core becomes padding and cannot match.
__device__ __forceinline__ int64_t pad16_start(int32_t rs, int32_t y) {
    return (((int64_t)rs + 7) & ~(int64_t)7) + 24 * (int64_t)y;
}

__device__ __forceinline__ uint32_t plane_key(const int32_t* __restrict__ col, const int32_t* __restrict__ cidx,
                                              int64_t n_nodes, int32_t i, int plane, uint32_t& status) {
    const int32_t w = __ldg(col + i);
    if ((uint64_t)(uint32_t)w >= (uint64_t)n_nodes) {
        status |= ST_BAD_KEY;
        return 0xFFFFu;
    }
    const int32_t c = __ldg(cidx + w);
    if (plane == 0) return (c >= 0 && c < kPlane) ? (uint32_t)c : 0xFFFFu;
    return c >= kPlane ? (uint32_t)(c - kPlane) : 0xFFFFu;
}

// By default the keys keep the row's order.  With bank_sort, within each
// plane the keys are ordered by the shared-memory bank of their bitmap word
// ((key >> 5) & 31; a list is a set, so order is free): the hub kernel deals
// consecutive 8-key units to consecutive lanes, so one load instruction then
// mostly touches distinct banks (R-MAT 21: 3.3 instead of 3.8 shared-memory
// wavefronts per load, but the sort costs this pass more than the hub
// kernel saves).  A counting sort per row and plane: 8 lanes count the 32
// banks in shared memory, scan them and scatter the keys; the order inside a
// bank is arbitrary; a plane of at most 8 keys is one unit and is not sorted.
__global__ void __launch_bounds__(256) core_pad16_kernel(const int32_t* __restrict__ row_ptr, int64_t n_nodes,
                                                         int64_t nnz, const int32_t* __restrict__ col,
                                                         const int32_t* __restrict__ cidx,
                                                         const int32_t* __restrict__ n_core, int packed,
                                                         int bank_sort, uint16_t* __restrict__ pcol16,
                                                         int4* __restrict__ pl, tchll_count_result* result) {
    __shared__ int s_cnt[32][32];  // per 8-lane group: bank counters, then cursors
    const int32_t C = n_core[0];
    if (!packed || C > kCore16Max) return;  // grid-uniform: the 32-bit lists apply
    const int32_t wsplit = n_core[1];       // -1: no plane 1
    const int lane = threadIdx.x & 31;
    const int sub = threadIdx.x & 7;        // 8 lanes per row
    const unsigned gmask = 0xFFu << (lane & 24);
    int* cnt = s_cnt[threadIdx.x >> 3];
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 3;
    const int64_t ng = ((int64_t)gridDim.x * blockDim.x) >> 3;
    uint32_t status = 0;
    for (int64_t y = g; y < n_nodes; y += ng) {
        const int32_t rs = __ldg(row_ptr + y), re = __ldg(row_ptr + y + 1);
        if (rs < 0 || re < rs || (int64_t)re > nnz) {
            status |= ST_BAD_ROW;
            if (sub == 0) pl[y] = make_int4(0, 0, 0, 0);
            continue;
        }
        const int32_t d = re - rs;
        int32_t P = d;
        if (wsplit >= 0) {  // P = first member >= wsplit, in [lo, hi]
            int32_t lo = 0, hi = d;
            while (hi - lo > 64) {  // group-uniform: 8 probes cut [lo, hi) into 9 parts
                const int64_t len = hi - lo;
                const bool lt = __ldg(col + rs + lo + (int32_t)(((sub + 1) * len) / 9)) < wsplit;
                const int t = __popc((__ballot_sync(gmask, lt) >> (lane & 24)) & 0xFFu);
                const int32_t nlo = t > 0 ? lo + (int32_t)((t * len) / 9) + 1 : lo;
                hi = t < 8 ? lo + (int32_t)(((t + 1) * len) / 9) : hi;
                lo = nlo;
            }
            int c = 0;  // hi - lo <= 64: eight independent loads per lane
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const int32_t m = lo + sub + 8 * t;
                if (m < hi) c += __ldg(col + rs + m) < wsplit;
            }
            c += __shfl_xor_sync(gmask, c, 1);
            c += __shfl_xor_sync(gmask, c, 2);
            c += __shfl_xor_sync(gmask, c, 4);
            P = lo + c;
        }
        const int32_t lo_units = (P + 7) >> 3, units = lo_units + ((d - P + 7) >> 3);
        const int64_t ps = pad16_start(rs, (int32_t)y);
        const int4 rec = make_int4((int32_t)(ps >> 3), lo_units, units, 0);
        if (!bank_sort) {  // list order: one 16-byte unit per lane
            for (int32_t u = sub; u < units; u += 8) {
                const int plane = u < lo_units ? 0 : 1;
                const int32_t m0 = plane == 0 ? 8 * u : P + 8 * (u - lo_units);
                const int32_t end = plane == 0 ? P : d;
                uint32_t k[8];
#pragma unroll
                for (int t = 0; t < 8; ++t)
                    k[t] = (m0 + t < end) ? plane_key(col, cidx, n_nodes, rs + m0 + t, plane, status) : 0xFFFFu;
                *reinterpret_cast<uint4*>(pcol16 + ps + 8 * u) =
                    make_uint4(k[0] | (k[1] << 16), k[2] | (k[3] << 16), k[4] | (k[5] << 16), k[6] | (k[7] << 16));
            }
            if (sub == 0) pl[y] = rec;
            continue;
        }
        for (int plane = 0; plane < 2; ++plane) {
            const int32_t m0 = plane ? P : 0, m1 = plane ? d : P;
            if (m1 <= m0) continue;  // group-uniform
            uint16_t* out = pcol16 + ps + (plane ? 8 * (int64_t)lo_units : 0);
            if (m1 - m0 <= 8) {  // one unit: one lane probes all its keys, order is moot
                out[sub] = m0 + sub < m1 ? (uint16_t)plane_key(col, cidx, n_nodes, rs + m0 + sub, plane, status)
                                         : (uint16_t)0xFFFFu;
                continue;
            }
            for (int b = sub; b < 32; b += 8) cnt[b] = 0;
            __syncwarp(gmask);
            for (int32_t m = m0 + sub; m < m1; m += 8)
                atomicAdd(cnt + ((plane_key(col, cidx, n_nodes, rs + m, plane, status) >> 5) & 31u), 1);
            __syncwarp(gmask);
            // exclusive scan of the 32 counters, 4 per lane
            const int c0 = cnt[4 * sub], c1 = cnt[4 * sub + 1], c2 = cnt[4 * sub + 2], c3 = cnt[4 * sub + 3];
            int incl = c0 + c1 + c2 + c3;
#pragma unroll
            for (int o = 1; o < 8; o <<= 1) {
                const int t = __shfl_up_sync(gmask, incl, o, 8);
                if (sub >= o) incl += t;
            }
            const int ex = incl - (c0 + c1 + c2 + c3);
            __syncwarp(gmask);
            cnt[4 * sub] = ex;
            cnt[4 * sub + 1] = ex + c0;
            cnt[4 * sub + 2] = ex + c0 + c1;
            cnt[4 * sub + 3] = ex + c0 + c1 + c2;
            __syncwarp(gmask);
            for (int32_t m = m0 + sub; m < m1; m += 8) {
                const uint32_t k = plane_key(col, cidx, n_nodes, rs + m, plane, status);
                out[atomicAdd(cnt + ((k >> 5) & 31u), 1)] = (uint16_t)k;
            }
            const int32_t nk = m1 - m0;
            for (int32_t t = nk + sub; t < ((nk + 7) & ~7); t += 8) out[t] = 0xFFFFu;
            __syncwarp(gmask);  // the counters are reused by the next plane / row
        }
        if (sub == 0) pl[y] = rec;
    }
    status = __reduce_or_sync(FULL, status);
    if (lane == 0 && status) atomicOr(&result->status, status);
}

// Probe lists in core coordinates, padded: 8 lanes per row, one 16-byte
// quad each; a member outside the core becomes the sentinel C (a bit that is
// never set: it cannot match), and so does the padding.  Rows keep their
// lengths, so a pair's probe list is [pad_start(y), + roundup4(d+(y))).
// Malformed rows are skipped with a status flag (the counting kernels flag
// them too when an edge uses them).
__global__ void core_pad_kernel(const int32_t* __restrict__ row_ptr, int64_t n_nodes, int64_t nnz,
                                const int32_t* __restrict__ col, const int32_t* __restrict__ cidx,
                                const int32_t* __restrict__ n_core, int packed, int32_t* __restrict__ pcol,
                                tchll_count_result* result) {
    const int32_t C = n_core[0];
    if (packed && C <= kCore16Max) return;  // grid-uniform: core_pad16_kernel writes the lists
    const int sub = threadIdx.x & 7;
    const int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 3;
    const int64_t ng = ((int64_t)gridDim.x * blockDim.x) >> 3;
    uint32_t status = 0;
    for (int64_t y = g; y < n_nodes; y += ng) {
        const int32_t rs = __ldg(row_ptr + y), re = __ldg(row_ptr + y + 1);
        if (rs < 0 || re < rs || (int64_t)re > nnz) {
            status |= ST_BAD_ROW;
            continue;
        }
        const int32_t d = re - rs;
        const int64_t ps = pad_start(rs, (int32_t)y);  // a multiple of 4: 16-byte aligned stores
        for (int32_t i = 4 * sub; i < d; i += 32) {
            int32_t c[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                c[k] = C;
                if (i + k < d) {
                    const int32_t w = __ldg(col + rs + i + k);
                    if ((uint64_t)(uint32_t)w < (uint64_t)n_nodes) {
                        const int32_t x = __ldg(cidx + w);
                        c[k] = x >= 0 ? x : C;
                    } else {
                        status |= ST_BAD_KEY;
                    }
                }
            }
            *reinterpret_cast<int4*>(pcol + ps + i) = make_int4(c[0], c[1], c[2], c[3]);
        }
    }
    status = __reduce_or_sync(FULL, status);
    if ((threadIdx.x & 31) == 0 && status) atomicOr(&result->status, status);
}

template <int UNR, bool PAD>
__global__ void __launch_bounds__(256, 5) hub_count_kernel(const HubParams H) {
    extern __shared__ __align__(16) uint32_t tbl[];
    __shared__ HubSeg s_seg;
    __shared__ int s_round;
    __shared__ int s_fail;
    if (PAD && ((H.packed && *H.n_core <= kCore16Max) || (H.cap_bits > 0 && *H.n_core + 32 <= H.cap_bits)))
        return;  // a bitmap kernel counted every segment
    const int tid = threadIdx.x, lane = tid & 31;
    const int32_t* __restrict__ col = H.col_idx;
    const int64_t nseg = min((int64_t)*H.n_segs, H.max_segs);
    uint64_t acc = 0;
    int64_t n_pairs = 0;
    while (true) {
        if (tid == 0) {
            const unsigned long long s = atomicAdd(H.seg_ctr, 1ull);
            if ((int64_t)s < nseg) {
                s_seg = H.segs[s];
            } else {
                s_seg.x = -1;
                s_seg.len = 0;
                s_seg.start = 0;
            }
            s_round = 0;
            s_fail = 0;
        }
        __syncthreads();
        const HubSeg sg = s_seg;
        if (sg.x < 0) break;
        if (tid == 0) n_pairs += sg.len;
        const int32_t xs = __ldg(H.row_ptr + sg.x);
        const int xl = __ldg(H.row_ptr + sg.x + 1) - xs;
        int lgs = ceil_log2_i(xl) + 4;  // load <= 1/16 where the cap allows
        lgs = lgs < 7 ? 7 : (lgs > H.hub_lg ? H.hub_lg : lgs);
        const uint32_t mask = (1u << lgs) - 1u;
        const int sh = 32 - lgs;
        const bool fits = 2 * (int64_t)xl <= (int64_t)(1 << lgs);  // load <= 1/2
        if (fits) {
            for (int i = tid; i < (1 << lgs) / 4; i += blockDim.x)
                reinterpret_cast<uint4*>(tbl)[i] = make_uint4(OV_KEY, OV_KEY, OV_KEY, OV_KEY);
            __syncthreads();
            for (int i = tid; i < xl; i += blockDim.x) {
                int32_t key = __ldg(col + xs + i);
                if (PAD) {  // core coordinates: every member of a hub list is in the core
                    key = (uint64_t)(uint32_t)key < (uint64_t)H.n_nodes ? __ldg(H.cidx + key) : -1;
                    if (key < 0) {
                        s_fail = 1;
                        continue;
                    }
                }
                if (!ov_insert(tbl, key, sh, mask)) s_fail = 1;
            }
            __syncthreads();
        }
        const bool table = fits && !s_fail;  // CTA-uniform
        // pairs per round: up to 32, fewer for short segments so that every
        // warp of the CTA gets about two rounds
        int rsz = (sg.len + 15) >> 4;
        rsz = rsz < 4 ? 4 : (rsz > 32 ? 32 : rsz);
        while (true) {
            int r = 0;
            if (lane == 0) r = atomicAdd(&s_round, rsz);
            r = __shfl_sync(FULL, r, 0);
            if (r >= sg.len) break;
            const int np = min(rsz, sg.len - r);
            int32_t rs = 0, re = 0, vs = 0, ve = 0;
            if (lane < np) {
                const int32_t y = __ldg(H.hy + sg.start + r + lane);
                rs = __ldg(H.row_ptr + y);
                re = __ldg(H.row_ptr + y + 1);
                if (PAD) {
                    vs = (int32_t)pad_start(rs, y);
                    ve = vs + ((re - rs + 3) & ~3);
                } else {
                    vs = rs;
                    ve = re;
                }
            }
            if (!table) {  // x's list too long for the table: binary search per pair
                for (int j = 0; j < np; ++j) {
                    const int32_t jrs = __shfl_sync(FULL, rs, j);
                    const int32_t jre = __shfl_sync(FULL, re, j);
                    acc += warp_bsearch_count(col + xs, xl, col + jrs, jre - jrs, lane);
                }
                continue;
            }
            // flatten the 32 probe lists into one stream of 16-byte quads
            const int q0 = vs >> 2;
            const int nq = (lane < np && ve > vs) ? ((ve - 1) >> 2) - q0 + 1 : 0;
            const unsigned ne = __ballot_sync(FULL, nq > 0);
            const int k = __popc(ne);
            const int src = lane < k ? (int)__fns(ne, 0, lane + 1) : lane;
            const int c_q0 = __shfl_sync(FULL, q0, src);
            int c_nq = __shfl_sync(FULL, nq, src);
            const int32_t c_vs = __shfl_sync(FULL, vs, src);
            const int32_t c_ve = __shfl_sync(FULL, ve, src);
            if (lane >= k) c_nq = 0;
            int incl = c_nq;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            const int excl = incl - c_nq;
            const int W = __shfl_sync(FULL, incl, 31);
            const int qb = c_q0 - excl;
            // a lane's list: starts before its window + starts in the window
            // up to the lane - 1 (B: the window's list starts)
            const unsigned lane_le = (2u << lane) - 1u;
            int S = 0;
            for (int T0 = 0; T0 < W; T0 += 32 * UNR) {
                int qd[UNR], lo[UNR], hi[UNR];
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    const int Ti = T0 + 32 * i;
                    qd[i] = -1;
                    lo[i] = hi[i] = 0;
                    if (Ti < W) {  // warp-uniform
                        const unsigned d = (unsigned)(excl - Ti);
                        const unsigned B = __reduce_or_sync(FULL, (lane < k && d < 32u) ? (1u << d) : 0u);
                        const int j = (S + __popc(B & lane_le) - 1) & 31;
                        S += __popc(B);
                        const int my_qb = __shfl_sync(FULL, qb, j);
                        const int32_t my_vs = __shfl_sync(FULL, c_vs, j);
                        const int32_t my_ve = __shfl_sync(FULL, c_ve, j);
                        if (Ti + lane < W) {
                            qd[i] = my_qb + Ti + lane;
                            if (!PAD) {
                                lo[i] = my_vs - qd[i] * 4;  // valid elements of the quad: [lo, hi)
                                hi[i] = my_ve - qd[i] * 4;
                            }
                        }
                    }
                }
                // Keys of all 4 * UNR quad elements.  Elements outside the
                // pair's list (quad edges, idle lanes) probe as OV_NONE,
                // which matches no slot; padded lists need no masking.
                uint32_t key[4 * UNR];
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    if (PAD) {
                        uint4 q = make_uint4(OV_NONE, OV_NONE, OV_NONE, OV_NONE);
                        if (qd[i] >= 0) q = __ldg(reinterpret_cast<const uint4*>(H.pcol) + qd[i]);
                        key[4 * i + 0] = q.x;
                        key[4 * i + 1] = q.y;
                        key[4 * i + 2] = q.z;
                        key[4 * i + 3] = q.w;
                    } else {
                        int4 val = make_int4(-1, -1, -1, -1);
                        if (qd[i] >= 0) {
                            const int64_t base = (int64_t)qd[i] * 4;
                            if (base + 3 < H.nnz) {
                                val = __ldg(reinterpret_cast<const int4*>(col) + qd[i]);
                            } else {
                                val.x = base + 0 < H.nnz ? __ldg(col + base + 0) : -1;
                                val.y = base + 1 < H.nnz ? __ldg(col + base + 1) : -1;
                                val.z = base + 2 < H.nnz ? __ldg(col + base + 2) : -1;
                                val.w = base + 3 < H.nnz ? __ldg(col + base + 3) : -1;
                            }
                        }
                        // lo <= 3 and hi >= 1 for every mapped quad; unmapped: lo = hi = 0
                        key[4 * i + 0] = (lo[i] <= 0 && hi[i] > 0) ? (uint32_t)val.x : OV_NONE;
                        key[4 * i + 1] = (lo[i] <= 1 && hi[i] > 1) ? (uint32_t)val.y : OV_NONE;
                        key[4 * i + 2] = (lo[i] <= 2 && hi[i] > 2) ? (uint32_t)val.z : OV_NONE;
                        key[4 * i + 3] = (lo[i] <= 3 && hi[i] > 3) ? (uint32_t)val.w : OV_NONE;
                    }
                }
                // home slots first (independent loads), then the rare walks
                // of flagged homes
                uint32_t c = 0, pend = 0, pk = 0;
#pragma unroll
                for (int t = 0; t < 4 * UNR; ++t) {
                    const uint32_t d = tbl[ov_h1((int32_t)key[t], sh)] ^ key[t];
                    c += (d << 1) == 0u;                       // key bits equal
                    const bool f = d > OV_FLAG;                // flagged home, other key
                    pend |= (f ? 1u : 0u) << t;
                    pk = f ? key[t] : pk;                      // the last such key
                }
                // each lane walks its own flagged homes: usually none, else
                // one (pk); several take the general loop
                if (pend) {
                    if ((pend & (pend - 1u)) == 0u) {
                        c += ov_walk(tbl, (int32_t)pk, sh, mask);
                    } else {
                        while (pend) {
                            const int t = __ffs(pend) - 1;
                            pend &= pend - 1u;
                            uint32_t k = key[0];
#pragma unroll
                            for (int j = 1; j < 4 * UNR; ++j) k = (t == j) ? key[j] : k;
                            c += ov_walk(tbl, (int32_t)k, sh, mask);
                        }
                    }
                }
                acc += c;
            }
        }
        if (H.batched) {  // this segment's totals belong to its graph
            acc = warp_sum_u64(acc);
            if (lane == 0 && acc) atomicAdd((unsigned long long*)&H.result[sg.graph].exact, (unsigned long long)acc);
            if (tid == 0) atomicAdd((unsigned long long*)&H.result[sg.graph].n_exact, (unsigned long long)sg.len);
            acc = 0;
            n_pairs = 0;
        }
        __syncthreads();  // every warp is done with this table
    }
    if (H.batched) return;
    acc = warp_sum_u64(acc);
    n_pairs = warp_sum_i64(n_pairs);
    if (lane == 0) {
        if (acc) atomicAdd((unsigned long long*)&H.result->exact, (unsigned long long)acc);
        if (n_pairs) atomicAdd((unsigned long long*)&H.result->n_exact, (unsigned long long)n_pairs);
    }
}

// Hub pairs over a shared-memory bitmap of N+(x) in core coordinates (see
// the hub core above).  Runs only when the core fits the shared buffer
// (C + 32 <= cap_bits, decided on the device: the host never reads C);
// otherwise it returns at once and hub_count_kernel<*, true> takes the
// segments from the same counter.
//
// A CTA claims a segment, clears ceil((C + 32) / 128) uint4 words, sets the
// bits of x's list and its warps stream the segment's probe lists through
// it, up to 32 lists per round.  The round's lists are flattened into one
// stream of 16-byte quads, 32 consecutive quads per window dealt to the 32
// lanes (coalesced loads).  A lane finds its quad's list from the bitmap B
// of list starts inside its window (one OR-reduction per window): list index
// = starts before the window + starts up to the lane - 1.  Since the probe
// lists are in core coordinates and padded with the never-set bit C, a key needs no
// mask and no bound: hit = bit key of the bitmap.
template <int UNR>
__global__ void __launch_bounds__(256, 6) hub_bitmap_kernel(const HubParams H) {
    extern __shared__ __align__(16) uint32_t bm[];
    __shared__ HubSeg s_seg;
    __shared__ int s_round;
    __shared__ int s_fail;
    const int C = *H.n_core;
    if ((H.packed && C <= kCore16Max) || C + 32 > H.cap_bits) return;  // grid-uniform: another kernel counts
    const int tid = threadIdx.x, lane = tid & 31;
    const unsigned lane_le = (2u << lane) - 1u;  // lane 31: 0 - 1 = all bits
    const uint32_t sentinel = (uint32_t)C;
    const int nw4 = (C + 32 + 127) >> 7;  // uint4 words covering bits [0, C + 32)
    const int32_t* __restrict__ col = H.col_idx;
    const uint4* __restrict__ pq = reinterpret_cast<const uint4*>(H.pcol);
    const int64_t nseg = min((int64_t)*H.n_segs, H.max_segs);
    uint64_t acc = 0;
    int64_t n_pairs = 0;
    while (true) {
        if (tid == 0) {
            const unsigned long long s = atomicAdd(H.seg_ctr, 1ull);
            if ((int64_t)s < nseg) {
                s_seg = H.segs[s];
            } else {
                s_seg.x = -1;
                s_seg.len = 0;
                s_seg.start = 0;
            }
            s_round = 0;
            s_fail = 0;
        }
        for (int i = tid; i < nw4; i += blockDim.x) reinterpret_cast<uint4*>(bm)[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        const HubSeg sg = s_seg;
        if (sg.x < 0) break;
        if (tid == 0) n_pairs += sg.len;
        const int32_t xs = __ldg(H.row_ptr + sg.x);
        const int xl = __ldg(H.row_ptr + sg.x + 1) - xs;
        for (int i = tid; i < xl; i += blockDim.x) {
            const int32_t w = __ldg(col + xs + i);
            const int32_t c = (uint64_t)(uint32_t)w < (uint64_t)H.n_nodes ? __ldg(H.cidx + w) : -1;
            if (c >= 0) atomicOr(bm + (c >> 5), 1u << (c & 31));
            else s_fail = 1;  // not in the core (cannot happen for well-formed input)
        }
        __syncthreads();
        const bool table = !s_fail;  // CTA-uniform
        // pairs per round: up to 32, fewer for short segments so that every
        // warp of the CTA gets about two rounds
        int rsz = (sg.len + 15) >> 4;
        rsz = rsz < 4 ? 4 : (rsz > 32 ? 32 : rsz);
        while (true) {
            int r = 0;
            if (lane == 0) r = atomicAdd(&s_round, rsz);
            r = __shfl_sync(FULL, r, 0);
            if (r >= sg.len) break;
            const int np = min(rsz, sg.len - r);
            int32_t vs = 0, nq = 0, rs = 0, re = 0;
            if (lane < np) {
                const int32_t y = __ldg(H.hy + sg.start + r + lane);
                rs = __ldg(H.row_ptr + y);
                re = __ldg(H.row_ptr + y + 1);
                vs = (int32_t)pad_start(rs, y);
                nq = (re - rs + 3) >> 2;
            }
            if (!table) {  // binary search per pair over the raw lists
                for (int j = 0; j < np; ++j) {
                    const int32_t jrs = __shfl_sync(FULL, rs, j);
                    const int32_t jre = __shfl_sync(FULL, re, j);
                    acc += warp_bsearch_count(col + xs, xl, col + jrs, jre - jrs, lane);
                }
                continue;
            }
            // the round's non-empty lists, compacted to lanes 0..k-1, and the
            // exclusive scan of their quad counts
            const unsigned ne = __ballot_sync(FULL, nq > 0);
            const int k = __popc(ne);
            const int src = lane < k ? (int)__fns(ne, 0, lane + 1) : lane;
            const int c_q0 = __shfl_sync(FULL, vs >> 2, src);
            int c_nq = __shfl_sync(FULL, nq, src);
            if (lane >= k) c_nq = 0;
            int incl = c_nq;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            const int excl = incl - c_nq;
            const int W = __shfl_sync(FULL, incl, 31);
            const int qb = c_q0 - excl;  // quad of stream position t in list j: qb[j] + t
            const bool starts = lane < k;
            int S = 0;  // list starts before the current window
            for (int T0 = 0; T0 < W; T0 += 32 * UNR) {
                int qd[UNR];
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    const int Ti = T0 + 32 * i;
                    qd[i] = -1;
                    if (Ti < W) {  // warp-uniform
                        const unsigned d = (unsigned)(excl - Ti);
                        const unsigned B = __reduce_or_sync(FULL, (starts && d < 32u) ? (1u << d) : 0u);
                        const int j = S + __popc(B & lane_le) - 1;
                        S += __popc(B);
                        const int my_qb = __shfl_sync(FULL, qb, j & 31);
                        if (Ti + lane < W) qd[i] = my_qb + Ti + lane;
                    }
                }
                uint32_t key[4 * UNR];
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    uint4 q = make_uint4(sentinel, sentinel, sentinel, sentinel);
                    if (qd[i] >= 0) q = __ldg(pq + qd[i]);
                    key[4 * i + 0] = q.x;
                    key[4 * i + 1] = q.y;
                    key[4 * i + 2] = q.z;
                    key[4 * i + 3] = q.w;
                }
                uint32_t c = 0;
#pragma unroll
                for (int t = 0; t < 4 * UNR; ++t) c += __funnelshift_r(bm[key[t] >> 5], 0u, key[t]) & 1u;
                acc += c;
            }
        }
        if (H.batched) {  // this segment's totals belong to its graph
            acc = warp_sum_u64(acc);
            if (lane == 0 && acc) atomicAdd((unsigned long long*)&H.result[sg.graph].exact, (unsigned long long)acc);
            if (tid == 0) atomicAdd((unsigned long long*)&H.result[sg.graph].n_exact, (unsigned long long)sg.len);
            acc = 0;
            n_pairs = 0;
        }
        __syncthreads();  // every warp is done with this bitmap
    }
    if (H.batched) return;
    acc = warp_sum_u64(acc);
    n_pairs = warp_sum_i64(n_pairs);
    if (lane == 0) {
        if (acc) atomicAdd((unsigned long long*)&H.result->exact, (unsigned long long)acc);
        if (n_pairs) atomicAdd((unsigned long long*)&H.result->n_exact, (unsigned long long)n_pairs);
    }
}

// hub_bitmap_kernel over packed probe lists (C <= kCore16Max): 8 keys per
// 16-byte unit, so the probe lists, which all pairs read from L2 or HBM, take
// half the bytes.  The bitmap has 65,536 bits (C <= 65535) or 131,072 bits
// (16 KB of shared memory); a unit's plane (the bitmap's half) follows from
// its position in the list: units at or past the list's plane-0 units are
// plane 1.  The bitmap is built from x's own packed list (16-byte loads of 8
// keys; x's members are the core's by construction, so no member can miss
// and there is no binary-search fallback).  Otherwise as hub_bitmap_kernel.
template <int UNR>
__global__ void __launch_bounds__(256, 8) hub_bitmap16_kernel(const HubParams H) {
    extern __shared__ __align__(16) uint32_t bm[];  // 4096 words
    __shared__ HubSeg s_seg;
    __shared__ int s_round;
    const int C = H.n_core[0];
    if (!H.packed || C > kCore16Max) return;  // grid-uniform: a 32-bit kernel counts
    const int tid = threadIdx.x, lane = tid & 31;
    const unsigned lane_le = (2u << lane) - 1u;
    const int nw4 = C > kPlane ? 1024 : 512;  // uint4 words: 131,072 or 65,536 bits
    const uint4* __restrict__ pq = reinterpret_cast<const uint4*>(H.pcol);
    const int64_t nseg = min((int64_t)*H.n_segs, H.max_segs);
    uint64_t acc = 0;
    int64_t n_pairs = 0;
    while (true) {
        if (tid == 0) {
            const unsigned long long s = atomicAdd(H.seg_ctr, 1ull);
            if ((int64_t)s < nseg) {
                s_seg = H.segs[s];
            } else {
                s_seg.x = -1;
                s_seg.len = 0;
                s_seg.start = 0;
            }
            s_round = 0;
        }
        for (int i = tid; i < nw4; i += blockDim.x) reinterpret_cast<uint4*>(bm)[i] = make_uint4(0u, 0u, 0u, 0u);
        __syncthreads();
        const HubSeg sg = s_seg;
        if (sg.x < 0) break;
        if (tid == 0) n_pairs += sg.len;
        {
            // N+(x) from x's own packed list (x's members are the core's by
            // construction): 8 keys per 16-byte load, padding skipped;
            // plane-1 key k is core index k + kPlane, bit k + kPlane + 1
            const int4 xr = H.pl[sg.x];
            for (int i = tid; i < xr.z; i += blockDim.x) {
                const uint4 q = __ldg(pq + xr.x + i);
                const uint32_t hb = i >= xr.y ? 65536u : 0u;
                const uint32_t w4[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
                for (int t = 0; t < 8; ++t) {
                    const uint32_t k = (w4[t >> 1] >> (16 * (t & 1))) & 0xFFFFu;
                    if (k != 0xFFFFu) atomicOr(bm + ((k + hb) >> 5), 1u << (k & 31));
                }
            }
        }
        __syncthreads();
        int rsz = (sg.len + 15) >> 4;
        rsz = rsz < 4 ? 4 : (rsz > 32 ? 32 : rsz);
        while (true) {
            int r = 0;
            if (lane == 0) r = atomicAdd(&s_round, rsz);
            r = __shfl_sync(FULL, r, 0);
            if (r >= sg.len) break;
            const int np = min(rsz, sg.len - r);
            int32_t q0 = 0, nq = 0, lo = 0;
            if (lane < np) {
                const int4 u = H.pl[__ldg(H.hy + sg.start + r + lane)];
                q0 = u.x;
                lo = u.y;
                nq = u.z;
            }
            const unsigned ne = __ballot_sync(FULL, nq > 0);
            const int k = __popc(ne);
            const int src = lane < k ? (int)__fns(ne, 0, lane + 1) : lane;
            const int c_q0 = __shfl_sync(FULL, q0, src);
            int c_nq = __shfl_sync(FULL, nq, src);
            const int c_lo = __shfl_sync(FULL, lo, src);
            if (lane >= k) c_nq = 0;
            int incl = c_nq;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int t = __shfl_up_sync(FULL, incl, o);
                if (lane >= o) incl += t;
            }
            const int excl = incl - c_nq;
            const int W = __shfl_sync(FULL, incl, 31);
            const int qb = c_q0 - excl;   // unit of stream position t in list j: qb[j] + t
            const int thr = excl + c_lo;  // stream positions >= thr[j] are list j's plane 1
            const bool starts = lane < k;
            int S = 0;
            for (int T0 = 0; T0 < W; T0 += 32 * UNR) {
                int qd[UNR], hw[UNR];
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    const int Ti = T0 + 32 * i;
                    qd[i] = -1;
                    hw[i] = 0;
                    if (Ti < W) {  // warp-uniform
                        const unsigned d = (unsigned)(excl - Ti);
                        const unsigned B = __reduce_or_sync(FULL, (starts && d < 32u) ? (1u << d) : 0u);
                        const int j = (S + __popc(B & lane_le) - 1) & 31;
                        S += __popc(B);
                        const int my_qb = __shfl_sync(FULL, qb, j);
                        const int my_thr = __shfl_sync(FULL, thr, j);
                        const int t = Ti + lane;
                        if (t < W) {
                            qd[i] = my_qb + t;
                            hw[i] = t >= my_thr ? 2048 : 0;  // plane 1: the bitmap's upper half
                        }
                    }
                }
                uint4 q[UNR];
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    q[i] = make_uint4(~0u, ~0u, ~0u, ~0u);  // padding keys: bit 65535, never set
                    if (qd[i] >= 0) q[i] = __ldg(pq + qd[i]);
                }
                uint32_t c = 0;
#pragma unroll
                for (int i = 0; i < UNR; ++i) {
                    const uint32_t* b = bm + hw[i];
                    const uint32_t w4[4] = {q[i].x, q[i].y, q[i].z, q[i].w};
#pragma unroll
                    for (int t = 0; t < 4; ++t) {
                        const uint32_t w = w4[t];
                        c += __funnelshift_r(b[(w >> 5) & 0x7FFu], 0u, w) & 1u;
                        c += __funnelshift_r(b[w >> 21], 0u, w >> 16) & 1u;
                    }
                }
                acc += c;
            }
        }
        if (H.batched) {  // this segment's totals belong to its graph
            acc = warp_sum_u64(acc);
            if (lane == 0 && acc) atomicAdd((unsigned long long*)&H.result[sg.graph].exact, (unsigned long long)acc);
            if (tid == 0) atomicAdd((unsigned long long*)&H.result[sg.graph].n_exact, (unsigned long long)sg.len);
            acc = 0;
            n_pairs = 0;
        }
        __syncthreads();  // every warp is done with this bitmap
    }
    if (H.batched) return;
    acc = warp_sum_u64(acc);
    n_pairs = warp_sum_i64(n_pairs);
    if (lane == 0) {
        if (acc) atomicAdd((unsigned long long*)&H.result->exact, (unsigned long long)acc);
        if (n_pairs) atomicAdd((unsigned long long*)&H.result->n_exact, (unsigned long long)n_pairs);
    }
}

// Hub segments: x's hub pairs [offh[x], offh[x] + cnth[x]) (shifted by the
// small-pair total *n_small) cut into pieces of at most seg pairs.
// Batched counts (vbase != null) record the graph of x, found by binary
// search in the ascending vertex offsets vbase[0..n_graphs].
__global__ void hub_segments_kernel(const int32_t* __restrict__ cnth, const int32_t* __restrict__ offh,
                                    const int32_t* __restrict__ n_small, int64_t n_nodes, int seg, HubSeg* segs,
                                    unsigned long long* n_segs, int64_t max_segs, const int32_t* __restrict__ vbase,
                                    int64_t n_graphs) {
    const int32_t base_pairs = *n_small;
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n_nodes;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = __ldg(cnth + x);
        if (c <= 0) continue;
        int32_t g = 0;
        if (vbase) {  // last g with vbase[g] <= x
            int64_t lo = 0, hi = n_graphs - 1;
            while (lo < hi) {
                const int64_t mid = (lo + hi + 1) >> 1;
                if (__ldg(vbase + mid) <= x) lo = mid; else hi = mid - 1;
            }
            g = (int32_t)lo;
        }
        const int k = (c + seg - 1) / seg;
        const unsigned long long b = atomicAdd(n_segs, (unsigned long long)k);
        for (int j = 0; j < k; ++j) {
            if ((int64_t)(b + j) >= max_segs) break;  // cannot happen: sized for the worst case
            HubSeg s;
            s.start = base_pairs + __ldg(offh + x) + j * seg;
            s.x = (int32_t)x;
            s.len = min(seg, c - j * seg);
            s.graph = g;
            segs[b + j] = s;
        }
    }
}

// Splits the pair histogram: cnt[x] keeps x's small pairs, cnth[x] gets its
// hub pairs (all of x's pairs go one way: hub-ness depends on d+(x) only).
__global__ void hub_split_kernel(const int32_t* __restrict__ row_ptr, int64_t n_nodes, int hub, int32_t* cnt,
                                 int32_t* cnth) {
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x <= n_nodes;
         x += (int64_t)gridDim.x * blockDim.x) {
        int32_t c = cnt[x];
        bool is_hub = false;
        if (x < n_nodes && c > 0) is_hub = (__ldg(row_ptr + x + 1) - __ldg(row_ptr + x)) > hub;
        cnth[x] = is_hub ? c : 0;
        if (is_hub) cnt[x] = 0;
    }
}

// ------------------------------------------------------ HLL edge list ------
// One group of L lanes per HLL edge (L = min(32, 2^p / 16): p = 8 runs two
// edges per warp, p >= 9 a warp per edge), the group's lanes striding over
// the two 2^p-byte rows with 16-byte loads.  Pass 1 counts the zero
// registers V of the merged row (zero bytes of row_u | row_v).  Every zero
// register adds exactly 1 to Z = sum 2^-r, so V >= lc_min (the smallest V
// with alpha*m^2/V <= 2.5m, with a 1e-9 margin for the FP64 comparison) proves
// the estimator takes its linear-counting branch: E = m * ln(m / V), the same
// expression the full estimator evaluates, and Z is not needed.  Otherwise
// pass 2 forms Z exactly (128-bit fixed point) and applies the full
// estimator.
struct HllParams {
    const int32_t* hu;
    const int32_t* hv;
    const unsigned long long* n_dev;
    const int32_t* degrees;
    const uint8_t* regs;
    const int64_t* slot;  // null: dense rows (row v at v * 2^p)
    const uint32_t* zm;   // zero masks, zst words per row (null: count zeros from the registers)
    int zst;
    const int32_t* vbase;  // batched: per-edge results go to result[graph of u]
    int64_t n_graphs;
    int p;
    int variant;
    uint32_t lc_min;
    int zsh;  // contiguous runs: u's mask kept in shared memory (one slot per group) when registers cannot hold it
    tchll_count_result* result;
};

// Zero-register masks: bit j of word w of row r is set iff register 32w + j
// of the row is 0.  Rows are zst >= 4 words (16-byte aligned); bits past 2^p
// stay clear.  One warp per row; dense layouts skip rows without a sketch
// (no HLL edge reads them).
__global__ void __launch_bounds__(256) zmask_kernel(const uint8_t* __restrict__ regs, int64_t n_rows,
                                                    const uint8_t* __restrict__ has, int p, int zst,
                                                    uint32_t* __restrict__ zm) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int m = 1 << p;
    for (int64_t r = warp; r < n_rows; r += nwarps) {
        if (has && !__ldg(has + r)) continue;
        const uint4* row = reinterpret_cast<const uint4*>(regs + r * (int64_t)m);
        for (int w = lane; w < zst; w += 32) {
            uint32_t bits = 0;
            if (32 * w < m) {
                const uint4 a = __ldg(row + 2 * w);
                bits = (__vcmpeq4(a.x, 0u) & 0x01010101u) | ((__vcmpeq4(a.y, 0u) & 0x01010101u) << 1) |
                       ((__vcmpeq4(a.z, 0u) & 0x01010101u) << 2) | ((__vcmpeq4(a.w, 0u) & 0x01010101u) << 3);
                if (32 * w + 16 < m) {
                    const uint4 b = __ldg(row + 2 * w + 1);
                    bits |= ((__vcmpeq4(b.x, 0u) & 0x01010101u) << 4) | ((__vcmpeq4(b.y, 0u) & 0x01010101u) << 5) |
                            ((__vcmpeq4(b.z, 0u) & 0x01010101u) << 6) | ((__vcmpeq4(b.w, 0u) & 0x01010101u) << 7);
                }
            }
            zm[r * (int64_t)zst + w] = bits;  // bit order is a permutation of the registers: only popc is used
        }
    }
}

__device__ __forceinline__ uint32_t zero_bytes(uint32_t w) { return __popc(__vcmpeq4(w, 0u)) >> 3; }

template <int L>
__device__ __forceinline__ uint32_t group_sum_u32(uint32_t x, unsigned gmask) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) x += __shfl_xor_sync(gmask, x, o);
    return x;
}

template <int L>
__device__ __forceinline__ U128 group_sum_u128(U128 v, unsigned gmask) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) {
        U128 t;
        t.lo = __shfl_xor_sync(gmask, v.lo, o);
        t.hi = __shfl_xor_sync(gmask, v.hi, o);
        v.add(t);
    }
    return v;
}

// Sum of 2^-r over the merged registers, exactly, in units of 2^-S
// (S = 65 - p, so 2^-r for every valid rank r <= S is an integer there).
// Most registers hold r <= 7: for a word w of four such registers,
//   t    = bytes 2^(7 - r_i)   (one byte permute of the table 128, 64 .. 1,
//                               selected by the four ranks packed as nibbles)
//   fast += bytes of t          (dp4a with 1,1,1,1)
//   zeros += [r_i == 0]         (a second permute of the table 1,0,..,0)
// so fast * 2^(S-7) is the words' share of the sum.  A word with a register
// >= 8 goes byte by byte: r <= 7 into fast, 8 <= r <= S into fine (units of
// 2^-S, 64 bits), r > S (only in malformed rows) into extra (FP64).
__device__ __forceinline__ void hll_word_lut(uint32_t w, int S, uint32_t& fast, uint64_t& fine, uint32_t& zeros,
                                             double& extra) {
    if ((w & 0xF8F8F8F8u) == 0u) {
        const uint32_t x = w | (w >> 4);                 // byte 0: r0 | r1 << 4, byte 2: r2 | r3 << 4
        const uint32_t sel = __byte_perm(x, 0u, 0x4420u);  // nibbles r0 r1 r2 r3
        fast = __dp4a(__byte_perm(0x10204080u, 0x01020408u, sel), 0x01010101u, fast);
        zeros = __dp4a(__byte_perm(0x00000001u, 0u, sel), 0x01010101u, zeros);
        return;
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = (int)((w >> (8 * k)) & 0xFFu);
        if (r <= 7) {
            fast += 128u >> r;
            zeros += (r == 0);
        } else if (r <= S) {
            fine += 1ull << (S - r);
        } else {
            extra += ldexp(1.0, S - r);
        }
    }
}

template <int L>
__device__ __forceinline__ uint64_t group_sum_u64(uint64_t x, unsigned gmask) {
#pragma unroll
    for (int o = L / 2; o > 0; o >>= 1) x += __shfl_xor_sync(gmask, x, o);
    return x;
}

// E = the reference's estimate of the merged row from Z = ldexp(zsum, -S)
// (zsum exact, plus extra) and the zero count V (src/hll.py:37-54; variant 1:
// cpu_exp's 2^32 correction, cpu_exp/triangle_hll_experiment.py:357-366).
__device__ __forceinline__ double hll_estimate_from(U128 zsum, double extra, uint32_t zeros, int p, int S,
                                                    int variant) {
    const int m = 1 << p;
    const double Z = ldexp(u128_to_double(zsum.lo, zsum.hi) + extra, -S);
    double alpha;
    if (m == 16) alpha = 0.673;
    else if (m == 32) alpha = 0.697;
    else if (m == 64) alpha = 0.709;
    else alpha = 0.7213 / (1.0 + 1.079 / (double)m);
    double E = alpha * (double)m * (double)m / Z;
    if (variant == 1) {
        if (E <= 2.5 * (double)m && zeros > 0) E = (double)m * log((double)m / (double)zeros);
        else if (E > 4294967296.0 / 30.0) E = -4294967296.0 * log(1.0 - E / 4294967296.0);
    } else {
        if (E <= 2.5 * (double)m) {
            if (zeros > 0) E = (double)m * log((double)m / (double)zeros);
        }
        const double two64 = 18446744073709551616.0;
        if (E > two64 / 30.0) E = -two64 * log(1.0 - E / two64);
    }
    return E;
}

// One group of L lanes per HLL edge, the group's lanes striding over the two
// 2^p-byte rows with 16-byte loads.  Pass 1 counts the zero registers V of
// the merged row from the AND of the two rows' zero masks (ZM; else from the
// registers).  Every zero register adds exactly 1 to Z = sum 2^-r, so V >=
// lc_min (the smallest V with alpha*m^2/V <= 2.5m, with a 1e-9 margin for
// the FP64 comparison) proves the estimator takes its linear-counting
// branch: E = m * ln(m / V), the same expression the full estimator
// evaluates, and Z is not needed.  Otherwise pass 2 forms Z exactly and
// applies the full estimator.  For rows of at least 32 16-byte words
// (p >= 9) the whole warp runs pass 2 for one such edge at a time
// (coalesced loads, no lane idling while one group reads two whole rows),
// so narrow groups cost nothing when a few of their edges need the
// registers; smaller rows are read by the edge's own group.
// CACHE: each group takes a contiguous run of the edge list.  The routing
// pass appends edges in CSR order, so consecutive HLL edges mostly share u,
// and the group keeps u's zero mask in registers across them (up to four
// 16-byte words per lane) and, with CROW (rows of at most 8 16-byte words
// per lane), u's register row too: an edge then reads only v's mask and
// row.  Otherwise the groups stride over the list.
template <int L, bool ZM, bool CACHE, bool CROW>
__global__ void __launch_bounds__(256, CROW ? 2 : (CACHE ? 3 : 4)) hll_edges_kernel(const HllParams H) {
    extern __shared__ __align__(16) uint4 zsm[];  // with H.zsh: 256 / L slots of one zero mask each
    const int lane = threadIdx.x & 31;
    const int sub = lane & (L - 1);
    const unsigned gmask = (L == 32) ? FULL : (((1u << L) - 1u) << (lane & ~(L - 1)));
    const int64_t gid = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / L;
    const int64_t ngroups = ((int64_t)gridDim.x * blockDim.x) / L;
    const int64_t n = (int64_t)*H.n_dev;
    const int m = 1 << H.p;
    const int nvec = m >> 4;
    const int S = 65 - H.p;
    U128 hacc;
    int64_t n_approx = 0, n_clamped = 0;
    const int64_t per = CACHE ? (n + ngroups - 1) / ngroups : 1;
    const int64_t e_lo = CACHE ? gid * per : gid;
    const int64_t e_hi = CACHE ? min(n, e_lo + per) : n;
    const int64_t e_step = CACHE ? 1 : ngroups;
    const int64_t w_first = gid - (lane / L);  // the warp's first group
    const int nq = H.zst >> 2;
    constexpr int KA = CROW ? 1 : 4;  // mask words cached per lane (p <= 10 with a cached row: one)
    const bool cache_a = CACHE && ZM && nq <= KA * L;
    int64_t cached = -1, cached_row = -1;
    uint4 ca[KA];
    uint4 ra[CROW ? 8 : 1];
    // warp-uniform trip count (pass 2 is warp-wide): CACHE runs `per` steps,
    // else while the warp's first group still has an edge
    for (int64_t k = 0; CACHE ? k < per : w_first + k * ngroups < n; ++k) {
        const int64_t e = e_lo + k * e_step;
        const bool act = e < e_hi;  // group-uniform
        int32_t u = 0, v = 0;
        int64_t su = 0, sv = 0;
        uint32_t zeros = 0;
        if (act) {
            u = __ldg(H.hu + e);
            v = __ldg(H.hv + e);
            su = H.slot ? __ldg(H.slot + u) : (int64_t)u;
            sv = H.slot ? __ldg(H.slot + v) : (int64_t)v;
            if (ZM) {  // registers zero in both rows: AND of the two zero masks
                const uint4* za = reinterpret_cast<const uint4*>(H.zm + su * (int64_t)H.zst);
                const uint4* zb = reinterpret_cast<const uint4*>(H.zm + sv * (int64_t)H.zst);
                if (cache_a) {
                    if (su != cached) {  // group-uniform
#pragma unroll
                        for (int kk = 0; kk < KA; ++kk) {
                            const int i = sub + kk * L;
                            ca[kk] = i < nq ? __ldg(za + i) : make_uint4(0u, 0u, 0u, 0u);
                        }
                        cached = su;
                    }
#pragma unroll
                    for (int kk = 0; kk < KA; ++kk) {
                        const int i = sub + kk * L;
                        if (i < nq) {
                            const uint4 b = __ldg(zb + i);
                            zeros += __popc(ca[kk].x & b.x) + __popc(ca[kk].y & b.y) + __popc(ca[kk].z & b.z) +
                                     __popc(ca[kk].w & b.w);
                        }
                    }
                } else if (CACHE && H.zsh) {
                    // u's mask in the group's shared-memory slot while
                    // consecutive edges share u: each edge reads v's only
                    uint4* zs = zsm + (size_t)(threadIdx.x / L) * nq;
                    if (su != cached) {  // group-uniform
                        __syncwarp(gmask);  // the group is done with the previous row
                        for (int i = sub; i < nq; i += L) zs[i] = __ldg(za + i);
                        __syncwarp(gmask);
                        cached = su;
                    }
#pragma unroll 4
                    for (int i = sub; i < nq; i += L) {
                        const uint4 a = zs[i], b = __ldg(zb + i);
                        zeros += __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
                    }
                } else {
#pragma unroll 4
                    for (int i = sub; i < nq; i += L) {
                        const uint4 a = __ldg(za + i), b = __ldg(zb + i);
                        zeros += __popc(a.x & b.x) + __popc(a.y & b.y) + __popc(a.z & b.z) + __popc(a.w & b.w);
                    }
                }
            } else {
                const uint4* a4 = reinterpret_cast<const uint4*>(H.regs + su * (int64_t)m);
                const uint4* b4 = reinterpret_cast<const uint4*>(H.regs + sv * (int64_t)m);
#pragma unroll 4
                for (int i = sub; i < nvec; i += L) {
                    const uint4 a = __ldg(a4 + i), b = __ldg(b4 + i);
                    zeros += zero_bytes(a.x | b.x) + zero_bytes(a.y | b.y) + zero_bytes(a.z | b.z) +
                             zero_bytes(a.w | b.w);
                }
            }
        }
        zeros = group_sum_u32<L>(zeros, gmask);
        const bool need = act && zeros < H.lc_min;  // group-uniform
        double E = 0.0;
        if (act && !need) E = (double)m * log((double)m / (double)zeros);
        // rows of fewer than 32 16-byte words (p <= 8) would leave most of
        // the warp idle in a warp-wide pass 2: there each group forms Z
        if (CROW || nvec < 32) {
            if (need) {  // the group forms Z itself (CROW: u's row kept in registers)
                uint32_t fast = 0, zz = 0;
                uint64_t fine = 0;
                double extra = 0.0;
                const uint4* a4 = reinterpret_cast<const uint4*>(H.regs + su * (int64_t)m);
                const uint4* b4 = reinterpret_cast<const uint4*>(H.regs + sv * (int64_t)m);
                if (CROW) {
                    if (su != cached_row) {  // group-uniform
#pragma unroll
                        for (int kk = 0; kk < 8; ++kk) {
                            const int i = sub + kk * L;
                            ra[kk] = i < nvec ? __ldg(a4 + i) : make_uint4(0u, 0u, 0u, 0u);
                        }
                        cached_row = su;
                    }
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk) {
                        const int i = sub + kk * L;
                        if (i < nvec) {
                            const uint4 b = __ldg(b4 + i);
                            hll_word_lut(__vmaxu4(ra[kk].x, b.x), S, fast, fine, zz, extra);
                            hll_word_lut(__vmaxu4(ra[kk].y, b.y), S, fast, fine, zz, extra);
                            hll_word_lut(__vmaxu4(ra[kk].z, b.z), S, fast, fine, zz, extra);
                            hll_word_lut(__vmaxu4(ra[kk].w, b.w), S, fast, fine, zz, extra);
                        }
                    }
                } else {
#pragma unroll 2
                    for (int i = sub; i < nvec; i += L) {
                        const uint4 a = __ldg(a4 + i), b = __ldg(b4 + i);
                        hll_word_lut(__vmaxu4(a.x, b.x), S, fast, fine, zz, extra);
                        hll_word_lut(__vmaxu4(a.y, b.y), S, fast, fine, zz, extra);
                        hll_word_lut(__vmaxu4(a.z, b.z), S, fast, fine, zz, extra);
                        hll_word_lut(__vmaxu4(a.w, b.w), S, fast, fine, zz, extra);
                    }
                }
                fast = group_sum_u32<L>(fast, gmask);
                fine = group_sum_u64<L>(fine, gmask);
#pragma unroll
                for (int o = L / 2; o > 0; o >>= 1) extra += __shfl_xor_sync(gmask, extra, o);
                U128 z;  // fast * 2^(S-7) + fine; fast <= 2^(p+7)
                z.lo = (uint64_t)fast << (S - 7);
                z.hi = (uint64_t)fast >> (71 - S);
                z.add(fine);
                E = hll_estimate_from(z, extra, zeros, H.p, S, H.variant);
            }
        } else {
            // pass 2, warp-wide: the whole warp forms Z for one edge at a
            // time (coalesced 16-byte loads over both rows), for each group
            // whose zero count left the linear-counting branch open
            unsigned pend = __ballot_sync(FULL, need && sub == 0);
            while (pend) {
                const int f = __ffs(pend) - 1;  // the group's first lane
                pend &= pend - 1;
                const int64_t fsu = __shfl_sync(FULL, su, f), fsv = __shfl_sync(FULL, sv, f);
                const uint32_t fz = __shfl_sync(FULL, zeros, f);
                const uint4* a4 = reinterpret_cast<const uint4*>(H.regs + fsu * (int64_t)m);
                const uint4* b4 = reinterpret_cast<const uint4*>(H.regs + fsv * (int64_t)m);
                uint32_t fast = 0, zz = 0;
                uint64_t fine = 0;
                double extra = 0.0;
#pragma unroll 2
                for (int i = lane; i < nvec; i += 32) {
                    const uint4 a = __ldg(a4 + i), b = __ldg(b4 + i);
                    hll_word_lut(__vmaxu4(a.x, b.x), S, fast, fine, zz, extra);
                    hll_word_lut(__vmaxu4(a.y, b.y), S, fast, fine, zz, extra);
                    hll_word_lut(__vmaxu4(a.z, b.z), S, fast, fine, zz, extra);
                    hll_word_lut(__vmaxu4(a.w, b.w), S, fast, fine, zz, extra);
                }
                fast = group_sum_u32<32>(fast, FULL);
                // registers of rank >= 8 (fine) and > S (extra, malformed rows) are rare
                if (__any_sync(FULL, fine != 0)) fine = group_sum_u64<32>(fine, FULL);
                if (__any_sync(FULL, extra != 0.0)) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) extra += __shfl_xor_sync(FULL, extra, o);
                }
                U128 z;  // fast * 2^(S-7) + fine; fast <= 2^(p+7)
                z.lo = (uint64_t)fast << (S - 7);
                z.hi = (uint64_t)fast >> (71 - S);
                z.add(fine);
                const double Ef = hll_estimate_from(z, extra, fz, H.p, S, H.variant);
                if ((lane & ~(L - 1)) == f) E = Ef;
            }
        }
        if (act && sub == 0) {
            const int32_t du = __ldg(H.degrees + u), dv = __ldg(H.degrees + v);
            const double s_hat = (double)((int64_t)du + (int64_t)dv) - E;
            const double upper = (double)(du < dv ? du : dv);
            // max(0.0, min(s_hat, upper)) with Python's min/max argument order
            double s_cl = (upper < s_hat) ? upper : s_hat;
            s_cl = (s_cl > 0.0) ? s_cl : 0.0;
            const bool clamped = s_hat < 0.0 || s_hat > upper;
            const uint64_t fx = (uint64_t)__double2ull_rn(s_cl * 4294967296.0);
            if (H.vbase) {  // batched: straight into this edge's graph
                tchll_count_result* R = H.result + graph_of(H.vbase, H.n_graphs, u);
                U128 one;
                one.lo = fx;
                atomic_add_u128((unsigned long long*)&R->hll_fx_lo, one);
                atomicAdd((unsigned long long*)&R->n_approx, 1ull);
                if (clamped) atomicAdd((unsigned long long*)&R->n_clamped, 1ull);
            } else {
                n_clamped += clamped;
                ++n_approx;
                hacc.add(fx);
            }
        }
    }
    publish(H.result, 0, hacc, n_approx, 0, 0, n_clamped, 0u, lane);
}

// ---------------------------------------------------------------- host ------
struct Tuning {
    int chunk = 256;
    int slots_log2 = 10;    // 1024 slots = 4 KB per warp: a table side of up to 128 keys at load <= 1/8
    int tiny = 16;
    int blocks_per_sm = 0;  // 0: occupancy maximum
    int warps = 8;          // warps per CTA
    int pairs = 1;          // table-side / probe-side reorientation
    int sparse = 0;         // table load <= 1/4 where it fits
    int hub = 128;          // pairs with d+(x) > hub go to the CTA-table kernels (0: off)
    int hub_seg = 2048;     // hub pairs per CTA work unit
    int hub_lg = 13;        // largest CTA hash table: 2^13 slots = 32 KB
    int hub_unroll = 2;     // quads per lane in flight (2 or 4)
    int bitmap_lg = 15;     // hub bitmap buffer: 2^15 bytes = 262,144 core vertices (0: hash tables only)
    int overlap = 1;        // side stream: 1 the hub core pass (+ the hybrid HLL pass); 2 also the short-list pairs
    int packed = 1;         // hub probe lists as 16-bit core indices when the core allows
    int bank_sort = 0;      // packed lists ordered by bitmap bank within each plane
    int hll_row_cache_p = 0;   // HLL pass: keep u's register row in registers for p <= this (0: never)
    int hll_lanes = 0;      // HLL pass: lanes per edge (0: chosen by p)
};
constexpr int HUB_MIN = 64;       // smallest hub threshold (bounds the segment count)
constexpr int HUB_SEG_MIN = 256;  // smallest segment

// The launch shape is process-wide state set through tchll_set_count_*.
// Every counting call copies it once, under the lock, and uses only its
// copy, so a concurrent setter can never change a shape half-way through a
// launch sequence (e.g. a table size versus its shared-memory allocation).
static std::mutex g_tuning_mu;
static Tuning g_tuning;
static Tuning tuning_snapshot() {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    return g_tuning;
}

// Opts a kernel into `smem` bytes of dynamic shared memory once per device
// (the attribute is per device and function); `done` is that kernel's
// per-device high-water mark, guarded by its own lock.
static std::mutex g_attr_mu;
static int ensure_smem(const void* kern, size_t smem, size_t* done, const char* what, bool carveout = false) {
    const int dev = current_device();
    if (dev < 0) return cuda_status(cudaErrorInvalidDevice, "cudaGetDevice");
    std::lock_guard<std::mutex> lock(g_attr_mu);
    if (smem > done[dev]) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return cuda_status(e, what);
        if (carveout) {
            e = cudaFuncSetAttribute(kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
            if (e != cudaSuccess) return cuda_status(e, what);
        }
        done[dev] = smem;
    }
    return TCHLL_OK;
}

// Optional phase timing: CUDA events recorded on the caller's stream around
// the pair regrouping, the exact-count launch and the HLL launch.  While
// timing is on, counting calls hold g_phase_mu for their whole enqueue, so
// the events and flags belong to one call at a time.
struct PhaseTimer {
    std::atomic<bool> on{false};
    bool made = false;
    cudaEvent_t ev[4];
    cudaEvent_t hub_ev[4];  // core pass start / end, hub kernels start / end (inside phase 1)
    cudaEvent_t hll_ev[2];  // around the HLL pass when it runs on the side stream
    bool used[3] = {false, false, false};
    bool hub_used = false;
    bool core_used = false;
    bool hll_split = false;  // phase 2 (HLL) is timed by hll_ev, not ev[2..3]
};
static PhaseTimer g_phase;
static std::mutex g_phase_mu;

// Lock held by a counting call while it records phase events.
struct PhaseScope {
    std::unique_lock<std::mutex> lock;
    PhaseScope() : lock(g_phase_mu, std::defer_lock) {
        if (g_phase.on.load()) lock.lock();
    }
    bool active() const { return lock.owns_lock() && g_phase.made; }
};

static void phase_mark(const PhaseScope& ps, int i, cudaStream_t st) {
    if (ps.active()) cudaEventRecord(g_phase.ev[i], st);
}
static void phase_used(const PhaseScope& ps, int a, int b = -1, int c = -1) {
    if (!ps.active()) return;
    for (int i : {a, b, c})
        if (i >= 0) g_phase.used[i] = true;
}
static void phase_reset(const PhaseScope& ps) {
    if (!ps.active()) return;
    for (int i = 0; i < 3; ++i) g_phase.used[i] = false;
    g_phase.hub_used = false;
    g_phase.core_used = false;
    g_phase.hll_split = false;
}

template <int MODE, bool VEC, bool DETAILS>
static int launch_mode(const CountParams& P, const Tuning& T, cudaStream_t st) {
    auto kern = count_kernel<MODE, VEC, DETAILS>;
    const int threads = T.warps * 32;
    const size_t smem = (size_t)T.warps * ((size_t)1 << P.slots_log2) * sizeof(int32_t);
    static size_t smem_set[kMaxDevices] = {};
    int rc = ensure_smem((const void*)kern, smem, smem_set, "cudaFuncSetAttribute(count_kernel)");
    if (rc) return rc;
    int bps = T.blocks_per_sm;
    if (bps <= 0) {
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, threads, smem);
        if (e != cudaSuccess) return cuda_status(e, "occupancy(count_kernel)");
        if (bps < 1) bps = 1;
    }
    const int grid = sm_count() * bps;
    kern<<<grid, threads, smem, st>>>(P);
    TCHLL_CHECK_LAUNCH("count_kernel");
    return TCHLL_OK;
}

template <int MODE>
static int launch_count(const CountParams& P, const Tuning& T, bool details, cudaStream_t st) {
    const bool vec = ((uintptr_t)P.col_idx % 16 == 0) && (P.regs == nullptr || (uintptr_t)P.regs % 16 == 0);
    if (details) return vec ? launch_mode<MODE, true, true>(P, T, st) : launch_mode<MODE, false, true>(P, T, st);
    return vec ? launch_mode<MODE, true, false>(P, T, st) : launch_mode<MODE, false, false>(P, T, st);
}

struct CountWs {
    unsigned long long* ctr;  // work counters: [0] [1] chunks, [2] hub segments made, [3] hub segments claimed
    int32_t* cnt;             // n_nodes + 1 (histogram of small pairs)
    int32_t* off;             // n_nodes + 1 (scan, then scatter cursor)
    int32_t* cnth;            // n_nodes + 1 (histogram of hub pairs)
    int32_t* offh;            // n_nodes + 1
    int32_t* px;              // n_edges
    int32_t* py;              // n_edges (small pairs, then the hub list)
    HubSeg* segs;             // max_segs
    int64_t max_segs;
    int32_t* pcol;            // padded lists in core coordinates for the hub kernels, pcap entries (null: not carved)
    int64_t pcap;
    int32_t* cflag;           // n_nodes + 1: core flags, then core indices (with pcol)
    int32_t* cpos;            // n_nodes + 1: scan of the flags (with pcol)
    int32_t* ncore;           // core size, vertex of core index kPlane (with pcol)
    int4* pl;                 // n_nodes: packed lists' {first unit, plane-0 units, all units, 0} (with pcol)
    void* tmp;
    size_t tmp_bytes;
};

// Padded lists need nnz + 8 (n_nodes + 1) entries; the workspace holds them
// for nnz <= n_edges (every oriented edge listed once).
// int32 entries of the padded-list region: the 32-bit lists (pad_start)
// or the packed ones (pad16_start, 2 bytes a key), whichever is larger.
static int64_t pad_capacity(int64_t n_nodes, int64_t nnz) {
    const int64_t w32 = nnz + 8 * (n_nodes + 1) + 8;
    const int64_t w16 = (nnz + 24 * (n_nodes + 1) + 24 + 1) / 2 + 4;
    return w32 > w16 ? w32 : w16;
}

static bool carve_count(void* ws, size_t bytes, int64_t n_nodes, int64_t n_edges, CountWs& W, size_t* need,
                        bool pad = true) {
    const size_t N = (size_t)(n_nodes > 0 ? n_nodes : 0) + 1;
    const size_t E = (size_t)(n_edges > 0 ? n_edges : 1);
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (int32_t*)nullptr, (int32_t*)nullptr, (int)N);
    Carve cv(ws, bytes);
    W.ctr = cv.take<unsigned long long>(4);
    W.cnt = cv.take<int32_t>(N);
    W.off = cv.take<int32_t>(N);
    W.cnth = cv.take<int32_t>(N);
    W.offh = cv.take<int32_t>(N);
    W.px = cv.take<int32_t>(E);
    W.py = cv.take<int32_t>(E);
    // every hub x with pairs opens one segment, every HUB_SEG_MIN pairs at most one more
    W.max_segs = (int64_t)(N < E ? N : E) + (int64_t)(E / HUB_SEG_MIN) + 1;
    W.segs = cv.take<HubSeg>((size_t)W.max_segs);
    W.pcap = pad ? pad_capacity(n_nodes, (int64_t)E) : 0;
    W.pcol = pad ? cv.take<int32_t>((size_t)W.pcap) : nullptr;
    W.cflag = pad ? cv.take<int32_t>(N) : nullptr;
    W.cpos = pad ? cv.take<int32_t>(N) : nullptr;
    W.ncore = pad ? cv.take<int32_t>(4) : nullptr;
    W.pl = pad ? cv.take<int4>(N) : nullptr;
    W.tmp_bytes = tb;
    W.tmp = cv.take<char>(tb);
    if (need) *need = cv.off;
    return cv.ok();
}

// Hybrid calls also hold the HLL edge list (8 bytes per edge) after the
// exact-count layout, then optionally the zero masks of the register rows
// (zmask_words(p) words per row); exact-only calls use the prefix.
struct HybridWs {
    int32_t* hll_u;
    int32_t* hll_v;
    unsigned long long* hll_n;
    uint32_t* zm;  // null when the workspace was sized without masks
    int zst;
};

static int zmask_words(int p) {
    const int w = (1 << p) >> 5;
    return w < 4 ? 4 : w;
}

static bool carve_count_hybrid(void* ws, size_t bytes, int64_t n_nodes, int64_t n_edges, int64_t zm_rows, int p,
                               CountWs& W, HybridWs& H, size_t* need, bool pad = true) {
    size_t base = 0;
    carve_count(nullptr, 0, n_nodes, n_edges, W, &base, pad);
    const size_t E = (size_t)(n_edges > 0 ? n_edges : 1);
    Carve cv(ws, bytes);
    char* b = cv.take<char>(base);
    H.hll_u = cv.take<int32_t>(E);
    H.hll_v = cv.take<int32_t>(E);
    H.hll_n = cv.take<unsigned long long>(1);
    H.zm = nullptr;
    H.zst = 0;
    if (zm_rows > 0) {
        H.zst = zmask_words(p);
        H.zm = cv.take<uint32_t>((size_t)zm_rows * (size_t)H.zst);
    }
    if (need) *need = cv.off;
    if (!cv.ok()) return false;
    if (!cv.dry) carve_count(b, base, n_nodes, n_edges, W, nullptr, pad);
    return true;
}

static uint32_t lc_min_for(int p) {
    const double m = (double)(1 << p);
    double alpha;
    if (p == 4) alpha = 0.673;
    else if (p == 5) alpha = 0.697;
    else if (p == 6) alpha = 0.709;
    else alpha = 0.7213 / (1.0 + 1.079 / m);
    return (uint32_t)ceil(alpha * m / 2.5 * (1.0 + 1e-9));
}

template <int L>
static int launch_hll_edges_L(HllParams H, bool crow, cudaStream_t st) {
    const int grid = sm_count() * 8;
    H.zsh = 0;
    if (H.zm && crow && L * 8 >= ((1 << H.p) >> 4)) hll_edges_kernel<L, true, true, true><<<grid, 256, 0, st>>>(H);
    else if (H.zm && H.p >= 11) {
        // masks too large for the 4 register words per lane go to shared
        // memory, one slot per group, while that fits 96 KB per CTA
        const int nq = H.zst >> 2;
        const size_t smem = nq > 4 * L ? (size_t)(256 / L) * nq * sizeof(uint4) : 0;
        size_t bytes = 0;
        if (smem > 0 && smem <= (96u << 10)) {
            static size_t set[kMaxDevices] = {0};
            const int rc = ensure_smem((const void*)hll_edges_kernel<L, true, true, false>, smem, set,
                                       "cudaFuncSetAttribute(hll_edges_kernel)");
            if (rc) return rc;
            H.zsh = 1;
            bytes = smem;
        }
        hll_edges_kernel<L, true, true, false><<<grid, 256, bytes, st>>>(H);
    }
    else if (H.zm) hll_edges_kernel<L, true, false, false><<<grid, 256, 0, st>>>(H);
    else hll_edges_kernel<L, false, false, false><<<grid, 256, 0, st>>>(H);
    TCHLL_CHECK_LAUNCH("hll_edges_kernel");
    return TCHLL_OK;
}

static int launch_hll_edges(const CountParams& P, const HybridWs& HW, const Tuning& T, cudaStream_t st) {
    HllParams H;
    H.vbase = P.graph_vbase;
    H.n_graphs = P.n_graphs;
    H.hu = HW.hll_u;
    H.hv = HW.hll_v;
    H.n_dev = HW.hll_n;
    H.degrees = P.degrees;
    H.regs = P.regs;
    H.slot = P.slot;
    H.p = P.p;
    H.variant = P.variant;
    H.lc_min = lc_min_for(P.p);
    H.result = P.result;
    H.zm = HW.zm;
    H.zst = HW.zst;
    // p <= row_cache_p (with zero masks): contiguous runs per group with u's
    // register row kept in registers, m / 128 lanes per edge (8 16-byte
    // words of the row per lane; off by default: at 128 registers per
    // thread too few warps hide the loads).  With zero masks the pass is
    // bound by the latency of its dependent loads, so narrow groups (more
    // edges in flight per warp) win: one lane per edge for p <= 10, 4 for
    // p = 11, 12, 8 above (R-MAT scale 22, theta = 256, beside the exact
    // pairs: p = 10 14.2 ms per hybrid step with 1 lane against 15.5 with 8;
    // p = 12 10.7 with 4 against 11.1 with 8; p = 14 14.0 with 8 against
    // 17.8 with 32).  Without masks one 16-byte register load per lane per
    // row.  T.hll_lanes > 0 overrides the width.
    const bool crow = H.zm != nullptr && P.p <= T.hll_row_cache_p;
    int width = (1 << P.p) >> 4;
    if (crow) width = (1 << P.p) >> 7;
    else if (H.zm) width = P.p <= 10 ? 1 : (P.p <= 12 ? 4 : 8);
    if (T.hll_lanes > 0) width = T.hll_lanes;
    if (H.zm) {
        const int64_t rows = P.slot ? P.n_rows : P.n_nodes;
        const int64_t wgrid = (rows + 7) / 8;
        const int grid = (int)(wgrid < 1 ? 1 : (wgrid > (int64_t)sm_count() * 16 ? (int64_t)sm_count() * 16 : wgrid));
        zmask_kernel<<<grid, 256, 0, st>>>(P.regs, rows, P.slot ? nullptr : P.has, P.p, H.zst, HW.zm);
        TCHLL_CHECK_LAUNCH("zmask_kernel");
    }
    switch (width >= 32 ? 32 : (width < 1 ? 1 : width)) {
        case 1: return launch_hll_edges_L<1>(H, crow, st);
        case 2: return launch_hll_edges_L<2>(H, crow, st);
        case 4: return launch_hll_edges_L<4>(H, crow, st);
        case 8: return launch_hll_edges_L<8>(H, crow, st);
        case 16: return launch_hll_edges_L<16>(H, crow, st);
        default: return launch_hll_edges_L<32>(H, crow, st);
    }
}

static int grid_edges(int64_t n) {
    int64_t g = (n + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 16;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

// Pair regrouping, part 1: histogram of table sides and its exclusive scan
// (W.off[x] = first pair of x, W.off[n_nodes] = number of pairs).
// With hub > 0 the histogram is split into small and hub pairs, both are
// scanned, and the hub segments are listed (before the scatter moves offh).
template <bool HYB>
static int pairs_hist_scan(const CountParams& P, const CountWs& W, int hub, int hub_seg, cudaStream_t st,
                           const int32_t* vbase = nullptr, int64_t n_graphs = 0) {
    const int64_t N = P.n_nodes + 1;
    TCHLL_CUDA(cudaMemsetAsync(W.cnt, 0, sizeof(int32_t) * N, st));
    pair_hist_kernel<HYB><<<grid_edges(P.n_edges), 256, 0, st>>>(P, W.cnt);
    TCHLL_CHECK_LAUNCH("pair_hist_kernel");
    if (hub > 0) {
        hub_split_kernel<<<grid_edges(N), 256, 0, st>>>(P.row_ptr, P.n_nodes, hub, W.cnt, W.cnth);
        TCHLL_CHECK_LAUNCH("hub_split_kernel");
    }
    size_t tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(W.tmp, tb, W.cnt, W.off, (int)N, st));
    count_launch();
    if (hub > 0) {
        tb = W.tmp_bytes;
        TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(W.tmp, tb, W.cnth, W.offh, (int)N, st));
        count_launch();
        hub_segments_kernel<<<grid_edges(P.n_nodes), 256, 0, st>>>(W.cnth, W.offh, W.off + P.n_nodes, P.n_nodes,
                                                                   hub_seg, W.segs, W.ctr + 2,
                                                                   W.max_segs, vbase, n_graphs);
        TCHLL_CHECK_LAUNCH("hub_segments_kernel");
    }
    return TCHLL_OK;
}

// Part 2: scatter the pairs (advances W.off[x] / W.offh[x] for x < n_nodes
// only, so the totals in [n_nodes] survive) and point Q at the small-pair list.
template <bool HYB>
static int pairs_scatter(const CountParams& P, const CountWs& W, int hub, CountParams& Q, cudaStream_t st) {
    pair_scatter_kernel<HYB><<<grid_edges(P.n_edges), 256, 0, st>>>(P, W.off, W.offh, hub, W.off + P.n_nodes,
                                                                   W.px, W.py);
    TCHLL_CHECK_LAUNCH("pair_scatter_kernel");
    Q = P;
    Q.edge_u = W.px;
    Q.edge_v = W.py;
    Q.n_edges_dev = W.off + P.n_nodes;
    return TCHLL_OK;
}

static int grid_rows(int64_t n, int per_cta) {  // one unit of work per 256 / per_cta threads
    int64_t g = (n + per_cta - 1) / per_cta;
    const int64_t cap = (int64_t)sm_count() * 16;
    return (int)(g < 1 ? 1 : (g > cap ? cap : g));
}

// The hub core pass and kernels use the padded lists when the workspace
// holds them and 16-byte unit indices fit int.
static bool hub_pad_usable(const CountParams& P, const CountWs& W) {
    const int64_t need_pad = pad_capacity(P.n_nodes, P.nnz);
    return W.pcol != nullptr && need_pad <= W.pcap && need_pad <= (int64_t)INT32_MAX;
}

// The hub core pass (needs the hub histogram W.cnth only, so it may run on a
// second stream beside the pair scatter and the short-list pairs): core
// flags, their scan, core indices, then the padded lists, packed 16-bit when
// the core allows it, else 32-bit (each pad kernel checks the core size on
// the device).
static int launch_core_pass(const CountParams& P, const CountWs& W, const Tuning& T, const PhaseScope& ps,
                            cudaStream_t st) {
    if (!hub_pad_usable(P, W)) return TCHLL_OK;
    if (ps.active()) {
        cudaEventRecord(g_phase.hub_ev[0], st);
        g_phase.core_used = true;
    }
    const int64_t N = P.n_nodes + 1;
    TCHLL_CUDA(cudaMemsetAsync(W.cflag, 0, sizeof(int32_t) * N, st));
    core_mark_kernel<<<sm_count() * 8, 256, 0, st>>>(P.row_ptr, P.n_nodes, P.nnz, P.col_idx, W.segs, W.ctr + 2,
                                                      W.max_segs, W.cflag, P.result);
    TCHLL_CHECK_LAUNCH("core_mark_kernel");
    size_t tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(W.tmp, tb, W.cflag, W.cpos, (int)N, st));
    count_launch();
    TCHLL_CUDA(cudaMemsetAsync(W.ncore + 1, 0xFF, sizeof(int32_t), st));
    core_index_kernel<<<grid_rows(N, 256), 256, 0, st>>>(W.cflag, W.cpos, P.n_nodes, W.ncore);
    TCHLL_CHECK_LAUNCH("core_index_kernel");
    core_pad16_kernel<<<grid_rows(P.n_nodes, 32), 256, 0, st>>>(P.row_ptr, P.n_nodes, P.nnz, P.col_idx, W.cflag,
                                                                W.ncore, T.packed, T.bank_sort,
                                                                reinterpret_cast<uint16_t*>(W.pcol), W.pl, P.result);
    TCHLL_CHECK_LAUNCH("core_pad16_kernel");
    core_pad_kernel<<<grid_rows(P.n_nodes, 32), 256, 0, st>>>(P.row_ptr, P.n_nodes, P.nnz, P.col_idx, W.cflag,
                                                              W.ncore, T.packed, W.pcol, P.result);
    TCHLL_CHECK_LAUNCH("core_pad_kernel");
    if (ps.active()) cudaEventRecord(g_phase.hub_ev[1], st);
    return TCHLL_OK;
}

// The hub pairs: one CTA per segment at a time, persistent grid.  With the
// padded lists (the core pass done before, on this stream or waited for):
// the packed bitmap kernel, the 32-bit bitmap kernel, then the hash kernel;
// each but the one the core size selects returns at once.  Without them (a
// small workspace): the hash kernel over the raw lists.
static int launch_hub(const CountParams& P, const CountWs& W, const Tuning& T, const PhaseScope& ps, cudaStream_t st,
                      bool batched = false) {
    HubParams H{};
    H.batched = batched;
    H.row_ptr = P.row_ptr;
    H.n_nodes = P.n_nodes;
    H.col_idx = P.col_idx;
    H.nnz = P.nnz;
    H.hy = W.py;
    H.segs = W.segs;
    H.n_segs = W.ctr + 2;
    H.max_segs = W.max_segs;
    H.seg_ctr = W.ctr + 3;
    H.hub_lg = T.hub_lg;
    H.result = P.result;
    const bool pad = hub_pad_usable(P, W);
    if (pad) {
        H.pcol = W.pcol;
        H.cidx = W.cflag;
        H.n_core = W.ncore;
        H.pl = W.pl;
        H.packed = T.packed;
    }
    if (ps.active()) cudaEventRecord(g_phase.hub_ev[2], st);
    if (pad && T.packed) {
        const size_t smem = 16384;
        auto kern = T.hub_unroll == 4 ? hub_bitmap16_kernel<4> : hub_bitmap16_kernel<2>;
        static size_t smem_set[2][kMaxDevices] = {};
        int rc = ensure_smem((const void*)kern, smem, smem_set[T.hub_unroll == 4 ? 1 : 0],
                             "cudaFuncSetAttribute(hub_bitmap16_kernel)", true);
        if (rc) return rc;
        int bps = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 256, smem);
        if (e != cudaSuccess) return cuda_status(e, "occupancy(hub_bitmap16_kernel)");
        if (bps < 1) bps = 1;
        kern<<<sm_count() * bps, 256, smem, st>>>(H);
        TCHLL_CHECK_LAUNCH("hub_bitmap16_kernel");
    }
    if (pad && T.bitmap_lg > 0) {
        const size_t smem = (size_t)1 << T.bitmap_lg;
        H.cap_bits = (int)(8 * smem);
        auto kern = T.hub_unroll == 4 ? hub_bitmap_kernel<4> : hub_bitmap_kernel<2>;
        static size_t smem_set[2][kMaxDevices] = {};
        int rc = ensure_smem((const void*)kern, smem, smem_set[T.hub_unroll == 4 ? 1 : 0],
                             "cudaFuncSetAttribute(hub_bitmap_kernel)", true);
        if (rc) return rc;
        int bps = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 256, smem);
        if (e != cudaSuccess) return cuda_status(e, "occupancy(hub_bitmap_kernel)");
        if (bps < 1) bps = 1;
        kern<<<sm_count() * bps, 256, smem, st>>>(H);
        TCHLL_CHECK_LAUNCH("hub_bitmap_kernel");
    }
    const int vi = (T.hub_unroll == 4 ? 2 : 0) + (pad ? 1 : 0);
    auto kern = vi == 3 ? hub_count_kernel<4, true>
                        : vi == 2 ? hub_count_kernel<4, false> : vi == 1 ? hub_count_kernel<2, true> : hub_count_kernel<2, false>;
    const size_t smem = sizeof(int32_t) << T.hub_lg;
    static size_t hsmem_set[4][kMaxDevices] = {};
    int rc = ensure_smem((const void*)kern, smem, hsmem_set[vi], "cudaFuncSetAttribute(hub_count_kernel)", true);
    if (rc) return rc;
    int bps = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, 256, smem);
    if (e != cudaSuccess) return cuda_status(e, "occupancy(hub_count_kernel)");
    if (bps < 1) bps = 1;
    kern<<<sm_count() * bps, 256, smem, st>>>(H);
    TCHLL_CHECK_LAUNCH("hub_count_kernel");
    if (ps.active()) {
        cudaEventRecord(g_phase.hub_ev[3], st);
        g_phase.hub_used = true;
    }
    return TCHLL_OK;
}

// Hub path in use: pairs on, and 16-byte aligned col_idx (quad loads).
static int hub_threshold(const CountParams& P, const Tuning& T) {
    return (T.hub > 0 && (uintptr_t)P.col_idx % 16 == 0) ? T.hub : 0;
}

// A second stream per device for work that overlaps the caller's stream: the
// HLL pass of a hybrid count runs there beside the exact pairs.  Fork = an
// event recorded on the caller's stream that the side stream waits for;
// join = an event recorded on the side stream that the caller's stream
// waits for before the call returns.  Both are recorded under the device's
// lock, held from fork to join, so concurrent calls never wait on each
// other's events; under stream capture this is the usual fork/join of a
// captured graph.  Stream and events are created on first use (outside any
// capture: the first call of a process is never captured by this package).
struct SideStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, mid = nullptr, join = nullptr, back = nullptr;
    std::mutex mu;
};
static SideStream g_side[kMaxDevices];
static std::mutex g_side_make_mu;

class SideFork {
  public:
    // Starts the fork (returns an error status, or TCHLL_OK with stream()
    // ready for work that may run once the caller's stream got here).
    int begin(cudaStream_t caller) {
        const int dev = current_device();
        if (dev < 0) return cuda_status(cudaErrorInvalidDevice, "cudaGetDevice");
        SideStream& S = g_side[dev];
        {
            std::lock_guard<std::mutex> mk(g_side_make_mu);
            if (S.s == nullptr) {
                TCHLL_CUDA(cudaStreamCreateWithFlags(&S.s, cudaStreamNonBlocking));
                TCHLL_CUDA(cudaEventCreateWithFlags(&S.fork, cudaEventDisableTiming));
                TCHLL_CUDA(cudaEventCreateWithFlags(&S.mid, cudaEventDisableTiming));
                TCHLL_CUDA(cudaEventCreateWithFlags(&S.join, cudaEventDisableTiming));
                TCHLL_CUDA(cudaEventCreateWithFlags(&S.back, cudaEventDisableTiming));
            }
        }
        lock_ = std::unique_lock<std::mutex>(S.mu);
        side_ = &S;
        caller_ = caller;
        TCHLL_CUDA(cudaEventRecord(S.fork, caller));
        TCHLL_CUDA(cudaStreamWaitEvent(S.s, S.fork, 0));
        return TCHLL_OK;
    }
    cudaStream_t stream() const { return side_->s; }
    // Marks the side stream's work so far; wait_mark makes the caller's
    // stream wait for it (once per fork).
    int mark() {
        TCHLL_CUDA(cudaEventRecord(side_->mid, side_->s));
        return TCHLL_OK;
    }
    int wait_mark() {
        TCHLL_CUDA(cudaStreamWaitEvent(caller_, side_->mid, 0));
        return TCHLL_OK;
    }
    // The side stream waits for the caller's work so far (once per fork).
    int side_waits_caller() {
        TCHLL_CUDA(cudaEventRecord(side_->back, caller_));
        TCHLL_CUDA(cudaStreamWaitEvent(side_->s, side_->back, 0));
        return TCHLL_OK;
    }
    // Joins: the caller's stream waits for everything enqueued on the side
    // stream so far.  Safe to call more than once.
    int end() {
        if (side_ == nullptr) return TCHLL_OK;
        SideStream* S = side_;
        side_ = nullptr;
        cudaError_t e = cudaEventRecord(S->join, S->s);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(caller_, S->join, 0);
        lock_.unlock();
        return e == cudaSuccess ? TCHLL_OK : cuda_status(e, "side stream join");
    }
    ~SideFork() { end(); }

  private:
    SideStream* side_ = nullptr;
    cudaStream_t caller_ = nullptr;
    std::unique_lock<std::mutex> lock_;
};

// col_ready (exact counts only; null = ready): an event the kernels that
// read col_idx wait for, so the pair regrouping (row_ptr and the edges only)
// overlaps a copy of col_idx still in flight.
static int run_count(CountParams P, int mode, bool details, void* ws, size_t ws_bytes, cudaStream_t st,
                     cudaEvent_t col_ready = nullptr) {
    const Tuning T = tuning_snapshot();
    CountWs W;
    HybridWs HW{};
    size_t need = 0;
    bool ok;
    // Optional parts, used when the workspace has room (same results): the
    // core-coordinate lists of the hub kernels and, for hybrid calls, the zero
    // masks that let the HLL pass test linear counting without the registers.
    if (mode == MODE_EXACT) {
        ok = carve_count(ws, ws_bytes, P.n_nodes, P.n_edges, W, &need, true);
        if (!ok) ok = carve_count(ws, ws_bytes, P.n_nodes, P.n_edges, W, &need, false);
    } else {
        const int64_t zm_rows = P.slot ? P.n_rows : P.n_nodes;
        ok = zm_rows > 0 && carve_count_hybrid(ws, ws_bytes, P.n_nodes, P.n_edges, zm_rows, P.p, W, HW, &need);
        if (!ok) ok = carve_count_hybrid(ws, ws_bytes, P.n_nodes, P.n_edges, 0, P.p, W, HW, &need, true);
        if (!ok) ok = carve_count_hybrid(ws, ws_bytes, P.n_nodes, P.n_edges, 0, P.p, W, HW, &need, false);
    }
    if (!ok || ws == nullptr) {
        set_error("workspace too small: need %zu bytes, have %zu", need, ws_bytes);
        return TCHLL_EWORKSPACE;
    }
    TCHLL_CUDA(cudaMemsetAsync(W.ctr, 0, 4 * sizeof(unsigned long long), st));
    TCHLL_CUDA(cudaMemsetAsync(P.result, 0, sizeof(tchll_count_result), st));
    if (details && P.pe_support) TCHLL_CUDA(cudaMemsetAsync(P.pe_support, 0, sizeof(int64_t) * P.n_edges, st));
    if (details && P.pe_method) TCHLL_CUDA(cudaMemsetAsync(P.pe_method, 0, P.n_edges, st));
    P.chunk = T.chunk;
    P.slots_log2 = T.slots_log2;
    P.tiny = T.tiny;
    P.sparse = T.sparse;
    P.n_edges_dev = nullptr;
    P.hll_u = nullptr;
    P.hll_v = nullptr;
    P.hll_n = nullptr;
    if (P.n_edges == 0) return TCHLL_OK;
    const bool pairs = T.pairs && !details;
    if (col_ready && !(mode == MODE_EXACT && pairs)) {
        TCHLL_CUDA(cudaStreamWaitEvent(st, col_ready, 0));
        col_ready = nullptr;
    }
    int rc;
    CountParams Q;
    PhaseScope ps;
    phase_reset(ps);
    switch (mode) {
        case MODE_EXACT:
            P.work = W.ctr;
            if (pairs) {
                // after the histogram, the hub core pass runs on the side
                // stream beside the pair scatter and the short-list pairs;
                // the hub kernels wait for it
                const int hub = hub_threshold(P, T);
                phase_mark(ps, 0, st);
                rc = pairs_hist_scan<false>(P, W, hub, T.hub_seg, st);
                if (rc) return rc;
                SideFork fork;
                const bool side = hub > 0 && T.overlap && hub_pad_usable(P, W);
                if (side) {
                    rc = fork.begin(st);
                    if (rc == TCHLL_OK && col_ready) {
                        const cudaError_t e = cudaStreamWaitEvent(fork.stream(), col_ready, 0);
                        if (e != cudaSuccess) rc = cuda_status(e, "cudaStreamWaitEvent(col_ready)");
                    }
                    if (rc == TCHLL_OK) rc = launch_core_pass(P, W, T, ps, fork.stream());
                    if (rc == TCHLL_OK) rc = fork.mark();
                    if (rc) return rc;
                }
                rc = pairs_scatter<false>(P, W, hub, Q, st);
                if (rc) return rc;
                if (col_ready) TCHLL_CUDA(cudaStreamWaitEvent(st, col_ready, 0));
                phase_mark(ps, 1, st);
                if (side && T.overlap >= 2) {
                    // the short-list pairs follow the core pass on the side
                    // stream (once scattered) and run beside the hub kernel
                    rc = fork.side_waits_caller();
                    if (rc == TCHLL_OK) rc = launch_count<MODE_EXACT>(Q, T, false, fork.stream());
                    if (rc == TCHLL_OK) rc = fork.wait_mark();
                    if (rc == TCHLL_OK) rc = launch_hub(P, W, T, ps, st);
                } else {
                    rc = launch_count<MODE_EXACT>(Q, T, false, st);
                    if (rc == TCHLL_OK && hub > 0) {
                        rc = side ? fork.wait_mark() : launch_core_pass(P, W, T, ps, st);
                        if (rc == TCHLL_OK) rc = launch_hub(P, W, T, ps, st);
                    }
                }
                phase_mark(ps, 2, st);
                const int rj = fork.end();
                phase_used(ps, 0, 1);
                return rc ? rc : rj;
            }
            phase_mark(ps, 1, st);
            rc = launch_count<MODE_EXACT>(P, T, details, st);
            phase_mark(ps, 2, st);
            phase_used(ps, 1);
            return rc;
        case MODE_HYBRID:  // one fused launch over the edges as given
            P.work = W.ctr;
            phase_mark(ps, 1, st);
            rc = launch_count<MODE_HYBRID>(P, T, details, st);
            phase_mark(ps, 2, st);
            phase_used(ps, 1);
            return rc;
        case 2:  // split: exact-routed edges, then HLL-routed edges
            if (pairs && ((uintptr_t)P.regs % 16 == 0)) {
                // One routing pass builds both work lists: the exact pairs
                // (counted by the pair launches, which also count n_exact)
                // and the HLL edge list (estimated by hll_edges_kernel, which
                // counts n_approx / n_clamped); the routing pass counts
                // n_fallback.  The HLL pass needs only the routing pass, so
                // it forks onto the side stream there and overlaps the
                // scatter and the pair launches (all add integers into the
                // same result block).
                P.work = W.ctr;
                P.hll_u = HW.hll_u;
                P.hll_v = HW.hll_v;
                P.hll_n = HW.hll_n;
                TCHLL_CUDA(cudaMemsetAsync(HW.hll_n, 0, sizeof(unsigned long long), st));
                const int hub = hub_threshold(P, T);
                phase_mark(ps, 0, st);
                rc = pairs_hist_scan<true>(P, W, hub, T.hub_seg, st);
                if (rc) return rc;
                // side stream: the hub core pass first (the hub kernels wait
                // for it), then the HLL pass
                SideFork fork;
                cudaStream_t hst = st;
                const bool core_side = hub > 0 && T.overlap && hub_pad_usable(P, W);
                if (T.overlap) {
                    rc = fork.begin(st);
                    if (rc) return rc;
                    hst = fork.stream();
                    if (core_side) {
                        rc = launch_core_pass(P, W, T, ps, hst);
                        if (rc == TCHLL_OK) rc = fork.mark();
                        if (rc) return rc;
                    }
                }
                if (ps.active()) cudaEventRecord(g_phase.hll_ev[0], hst);
                rc = launch_hll_edges(P, HW, T, hst);
                if (ps.active()) cudaEventRecord(g_phase.hll_ev[1], hst);
                if (rc) return rc;
                rc = pairs_scatter<true>(P, W, hub, Q, st);
                if (rc) return rc;
                phase_mark(ps, 1, st);
                Q.hll_u = nullptr;
                rc = launch_count<MODE_EXACT>(Q, T, false, st);
                if (rc) return rc;
                if (hub > 0) {
                    rc = core_side ? fork.wait_mark() : launch_core_pass(P, W, T, ps, st);
                    if (rc == TCHLL_OK) rc = launch_hub(P, W, T, ps, st);
                    if (rc) return rc;
                }
                phase_mark(ps, 2, st);
                rc = fork.end();
                phase_used(ps, 0, 1, 2);
                if (ps.active()) g_phase.hll_split = true;
                return rc;
            }
            P.work = W.ctr;
            phase_mark(ps, 1, st);
            rc = launch_count<MODE_HYB_EXACT>(P, T, details, st);
            if (rc) return rc;
            phase_mark(ps, 2, st);
            P.work = W.ctr + 1;
            rc = launch_count<MODE_HYB_HLL>(P, T, details, st);
            phase_mark(ps, 3, st);
            phase_used(ps, 1, 2);
            return rc;
        default:
            set_error("unknown count mode %d", mode);
            return TCHLL_EINVAL;
    }
}

static int check_common(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                        const int32_t* eu, const int32_t* ev, int64_t n_edges, tchll_count_result* result) {
    TCHLL_ARG(n_nodes >= 0 && nnz >= 0 && n_edges >= 0, "negative size");
    TCHLL_ARG(n_nodes < (int64_t)INT32_MAX && nnz <= (int64_t)INT32_MAX && n_edges <= (int64_t)INT32_MAX,
              "int32 CSR limits exceeded");
    TCHLL_ARG(result != nullptr, "result pointer is null");
    TCHLL_ARG(n_edges == 0 || (eu && ev && row_ptr), "null edge or row_ptr pointer");
    TCHLL_ARG(nnz == 0 || col_idx, "null col_idx");
    return TCHLL_OK;
}

}  // namespace tchll

using namespace tchll;

TCHLL_EXPORT int tchll_count_workspace_bytes(int64_t n_nodes, int64_t n_edges, size_t* bytes) {
    TCHLL_ARG(bytes != nullptr && n_nodes >= 0 && n_edges >= 0, "bad arguments");
    CountWs W;
    HybridWs H;
    carve_count_hybrid(nullptr, 0, n_nodes, n_edges, 0, 4, W, H, bytes);  // covers the exact-only layout too
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_hybrid_workspace_bytes(int64_t n_nodes, int64_t n_edges, int64_t n_rows, int32_t p,
                                              size_t* bytes) {
    TCHLL_ARG(bytes != nullptr && n_nodes >= 0 && n_edges >= 0 && n_rows >= 0, "bad arguments");
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    CountWs W;
    HybridWs H;
    carve_count_hybrid(nullptr, 0, n_nodes, n_edges, n_rows, p, W, H, bytes);
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_exact_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                                   const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                                   int64_t* per_edge_support, tchll_count_result* result, void* workspace,
                                   size_t workspace_bytes, void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, result);
    if (rc) return rc;
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.pe_support = per_edge_support;
    P.result = result;
    P.p = 4;
    return run_count(P, MODE_EXACT, per_edge_support != nullptr, workspace, workspace_bytes, (cudaStream_t)stream);
}

TCHLL_EXPORT int tchll_exact_count_staged(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                          int64_t nnz, const int32_t* edge_u, const int32_t* edge_v,
                                          int64_t n_edges, tchll_count_result* result, void* workspace,
                                          size_t workspace_bytes, void* col_ready_event, void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, result);
    if (rc) return rc;
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.result = result;
    P.p = 4;
    return run_count(P, MODE_EXACT, false, workspace, workspace_bytes, (cudaStream_t)stream,
                     (cudaEvent_t)col_ready_event);
}

static int hybrid_common(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                         const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges, const int32_t* degrees,
                         const uint8_t* regs, int64_t n_rows, const int64_t* slot, const uint8_t* has, int32_t p,
                         int64_t gamma, int32_t mode, int64_t* pe_support, double* pe_s_hat, double* pe_s_cl,
                         uint8_t* pe_method, tchll_count_result* result, void* ws, size_t wsb, void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, result);
    if (rc) return rc;
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_edges == 0 || degrees, "degrees is null");
    TCHLL_ARG(n_rows == 0 || regs, "register rows are null");
    TCHLL_ARG(slot || has || n_edges == 0, "need slot (compact) or has_sketch (dense)");
    const bool details = pe_support || pe_s_hat || pe_s_cl || pe_method;
    TCHLL_ARG(!details || (pe_support && pe_s_hat && pe_s_cl && pe_method),
              "per-edge outputs must be all set or all null");
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.degrees = degrees;
    P.regs = regs;
    P.n_rows = n_rows;
    P.slot = slot;
    P.has = has;
    P.p = p;
    P.gamma = gamma;
    P.pe_support = pe_support;
    P.pe_s_hat = pe_s_hat;
    P.pe_s_cl = pe_s_cl;
    P.pe_method = pe_method;
    P.result = result;
    return run_count(P, mode, details, ws, wsb, (cudaStream_t)stream);
}

TCHLL_EXPORT int tchll_hybrid_count_dense(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                          int64_t nnz, const int32_t* edge_u, const int32_t* edge_v,
                                          int64_t n_edges, const int32_t* degrees, const uint8_t* sketch_regs,
                                          const uint8_t* has_sketch, int32_t p, int64_t gamma,
                                          int32_t split_kernels, tchll_count_result* result, void* workspace,
                                          size_t workspace_bytes, void* stream) {
    return hybrid_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, degrees, sketch_regs, n_nodes,
                         nullptr, has_sketch, p, gamma, split_kernels ? 2 : MODE_HYBRID, nullptr, nullptr, nullptr,
                         nullptr, result, workspace, workspace_bytes, stream);
}

TCHLL_EXPORT int tchll_hybrid_count_compact(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                            int64_t nnz, const int32_t* edge_u, const int32_t* edge_v,
                                            int64_t n_edges, const int32_t* degrees, const uint8_t* rows,
                                            int64_t n_rows, const int64_t* slot, int32_t p, int64_t gamma,
                                            int32_t split_kernels, int64_t* per_edge_support,
                                            double* per_edge_s_hat, double* per_edge_s_clamped,
                                            uint8_t* per_edge_method, tchll_count_result* result,
                                            void* workspace, size_t workspace_bytes, void* stream) {
    TCHLL_ARG(slot != nullptr || n_edges == 0, "slot is null");
    return hybrid_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, degrees, rows, n_rows, slot,
                         nullptr, p, gamma, split_kernels ? 2 : MODE_HYBRID, per_edge_support, per_edge_s_hat,
                         per_edge_s_clamped, per_edge_method, result, workspace, workspace_bytes, stream);
}

TCHLL_EXPORT int tchll_set_count_tuning(int32_t chunk, int32_t slots_log2, int32_t tiny, int32_t blocks_per_sm) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    TCHLL_ARG(chunk >= 32 && chunk % 32 == 0 && chunk <= (1 << 20), "chunk must be a multiple of 32 in [32, 2^20]");
    TCHLL_ARG(tiny >= 0 && tiny <= 4096, "tiny must be in [0, 4096]");
    TCHLL_ARG(blocks_per_sm >= 0 && blocks_per_sm <= 32, "blocks_per_sm must be in [0, 32]");
    TCHLL_ARG(slots_log2 >= 6 && slots_log2 <= 15 && (size_t)g_tuning.warps * ((size_t)4 << slots_log2) <= 227 * 1024,
              "slots_log2 must be in [6, 15] with warps x 2^slots_log2 x 4 bytes within 227 KB of shared memory");
    g_tuning.chunk = chunk;
    g_tuning.slots_log2 = slots_log2;
    g_tuning.tiny = tiny;
    g_tuning.blocks_per_sm = blocks_per_sm;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_set_count_shape(int32_t warps_per_cta, int32_t pairs) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    TCHLL_ARG(warps_per_cta >= 1 && warps_per_cta <= 8, "warps_per_cta must be in [1, 8]");
    TCHLL_ARG((size_t)warps_per_cta * ((size_t)4 << g_tuning.slots_log2) <= 227 * 1024,
              "warps x 2^slots_log2 x 4 bytes must fit 227 KB of shared memory");
    g_tuning.warps = warps_per_cta;
    g_tuning.pairs = pairs ? 1 : 0;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_set_count_table(int32_t sparse) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    g_tuning.sparse = sparse ? 1 : 0;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_set_count_hub(int32_t threshold, int32_t seg_pairs, int32_t table_log2, int32_t unroll) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    TCHLL_ARG(threshold == 0 || threshold >= HUB_MIN, "hub threshold must be 0 (off) or >= %d", HUB_MIN);
    TCHLL_ARG(seg_pairs >= HUB_SEG_MIN && seg_pairs <= (1 << 20), "seg_pairs must be in [%d, 2^20]", HUB_SEG_MIN);
    TCHLL_ARG(table_log2 >= 10 && table_log2 <= 15, "table_log2 must be in [10, 15]");
    TCHLL_ARG(unroll == 2 || unroll == 4, "unroll must be 2 or 4");
    g_tuning.hub = threshold;
    g_tuning.hub_seg = seg_pairs;
    g_tuning.hub_lg = table_log2;
    g_tuning.hub_unroll = unroll;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_get_count_hub(int32_t* out4) {
    TCHLL_ARG(out4 != nullptr, "null output");
    const Tuning T = tuning_snapshot();
    out4[0] = T.hub;
    out4[1] = T.hub_seg;
    out4[2] = T.hub_lg;
    out4[3] = T.hub_unroll;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_set_count_core(int32_t bitmap_log2, int32_t overlap, int32_t packed, int32_t bank_sort) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    TCHLL_ARG(bitmap_log2 == 0 || (bitmap_log2 >= 10 && bitmap_log2 <= 17),
              "bitmap_log2 must be 0 (hash tables only) or in [10, 17] (1 KB .. 128 KB of shared memory)");
    g_tuning.bitmap_lg = bitmap_log2;
    TCHLL_ARG(overlap >= 0 && overlap <= 2, "overlap must be 0, 1 or 2");
    g_tuning.overlap = overlap;
    g_tuning.packed = packed ? 1 : 0;
    g_tuning.bank_sort = bank_sort ? 1 : 0;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_get_count_core(int32_t* out4) {
    TCHLL_ARG(out4 != nullptr, "null output");
    const Tuning T = tuning_snapshot();
    out4[0] = T.bitmap_lg;
    out4[1] = T.overlap;
    out4[2] = T.packed;
    out4[3] = T.bank_sort;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_set_hll_pass(int32_t row_cache_max_p, int32_t lanes) {
    std::lock_guard<std::mutex> lock(g_tuning_mu);
    TCHLL_ARG(row_cache_max_p >= 0 && row_cache_max_p <= 16, "row_cache_max_p must be in [0, 16]");
    TCHLL_ARG(lanes == 0 || (lanes >= 1 && lanes <= 32 && (lanes & (lanes - 1)) == 0),
              "lanes must be 0 (automatic) or a power of two in [1, 32]");
    g_tuning.hll_row_cache_p = row_cache_max_p;
    g_tuning.hll_lanes = lanes;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_get_hll_pass(int32_t* out2) {
    TCHLL_ARG(out2 != nullptr, "null output");
    const Tuning T = tuning_snapshot();
    out2[0] = T.hll_row_cache_p;
    out2[1] = T.hll_lanes;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_get_count_tuning(int32_t* out8) {
    TCHLL_ARG(out8 != nullptr, "out is null");
    const Tuning T = tuning_snapshot();
    out8[0] = T.chunk;
    out8[1] = T.slots_log2;
    out8[2] = T.tiny;
    out8[3] = T.blocks_per_sm;
    out8[4] = T.warps;
    out8[5] = T.pairs;
    out8[6] = T.sparse;
    out8[7] = 0;  // reserved
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_set_phase_timing(int32_t enable) {
    std::lock_guard<std::mutex> lock(g_phase_mu);
    if (enable && !g_phase.made) {
        for (int i = 0; i < 4; ++i) TCHLL_CUDA(cudaEventCreate(&g_phase.ev[i]));
        for (int i = 0; i < 4; ++i) TCHLL_CUDA(cudaEventCreate(&g_phase.hub_ev[i]));
        for (int i = 0; i < 2; ++i) TCHLL_CUDA(cudaEventCreate(&g_phase.hll_ev[i]));
        g_phase.made = true;
    }
    g_phase.on = enable != 0;
    for (int i = 0; i < 3; ++i) g_phase.used[i] = false;
    g_phase.hub_used = false;
    g_phase.core_used = false;
    g_phase.hll_split = false;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_phase_times(float* ms3) {
    TCHLL_ARG(ms3 != nullptr, "out is null");
    std::lock_guard<std::mutex> lock(g_phase_mu);
    for (int i = 0; i < 3; ++i) ms3[i] = -1.0f;
    if (!g_phase.on || !g_phase.made) return TCHLL_OK;
    for (int i = 0; i < 3; ++i) {
        if (!g_phase.used[i]) continue;
        if (i == 2 && g_phase.hll_split) {  // the HLL pass ran beside phase 1
            TCHLL_CUDA(cudaEventSynchronize(g_phase.hll_ev[1]));
            TCHLL_CUDA(cudaEventElapsedTime(&ms3[i], g_phase.hll_ev[0], g_phase.hll_ev[1]));
            continue;
        }
        TCHLL_CUDA(cudaEventSynchronize(g_phase.ev[i + 1]));
        TCHLL_CUDA(cudaEventElapsedTime(&ms3[i], g_phase.ev[i], g_phase.ev[i + 1]));
    }
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_phase_hub_ms(float* ms2) {
    TCHLL_ARG(ms2 != nullptr, "out is null");
    std::lock_guard<std::mutex> lock(g_phase_mu);
    ms2[0] = ms2[1] = -1.0f;
    if (!g_phase.on || !g_phase.made || !g_phase.hub_used) return TCHLL_OK;
    TCHLL_CUDA(cudaEventSynchronize(g_phase.hub_ev[3]));
    TCHLL_CUDA(cudaEventElapsedTime(&ms2[0], g_phase.hub_ev[2], g_phase.hub_ev[3]));
    if (g_phase.core_used) TCHLL_CUDA(cudaEventElapsedTime(&ms2[1], g_phase.hub_ev[0], g_phase.hub_ev[1]));
    return TCHLL_OK;
}

// ------------------------------------------------ allocation-free variant ---
// Some callers hold device pointers to a graph but cannot allocate device
// memory themselves: a language binding without its own CUDA allocator, or a
// service that hands all device memory to one arena up front and forbids
// allocation on the request path.  tchll_exact_count_noalloc serves them with
// the same exact count, taking its scratch (the pair list, histogram and work
// counters) from this fixed array instead of a caller workspace.  Every GPU
// that loads the library reserves the array until the process exits.
static __device__ __align__(256) unsigned char g_noalloc_scratch[TCHLL_NOALLOC_SCRATCH_BYTES];

// Host code must not pass g_noalloc_scratch itself to a kernel (on the host
// the name stands for a host-side shadow, not the device array): the device
// address comes from cudaGetSymbolAddress, with the device current.  The
// address belongs to the module as loaded in one CUDA context, so it is
// cached per context, keyed by the context's process-unique id (cuCtxGetId,
// reached through the runtime's driver entry-point query, so the library
// needs no driver link): a non-primary context made current by a caller, or
// a primary context re-created after cudaDeviceReset, gets its own lookup.
// Where the id cannot be read, every call looks the address up again.
static std::mutex g_noalloc_mu;
struct NoallocEntry {
    unsigned long long ctx_id;
    void* ptr;
};
static NoallocEntry g_noalloc_cache[64];
static int g_noalloc_used = 0;

typedef int (*CtxGetCurrentFn)(void** ctx);
typedef int (*CtxGetIdFn)(void* ctx, unsigned long long* id);

// Id of the calling thread's current context; false when unavailable.
static bool current_ctx_id(unsigned long long* id) {
    static CtxGetCurrentFn get_cur = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_cur = (CtxGetCurrentFn)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (CtxGetIdFn)f;
    });
    if (get_cur == nullptr || get_id == nullptr) return false;
    void* ctx = nullptr;
    if (get_cur(&ctx) != 0 || ctx == nullptr) return false;
    return get_id(ctx, id) == 0;
}

static int noalloc_scratch_ptr(void** out) {
    int dev = -1;
    TCHLL_CUDA(cudaGetDevice(&dev));  // also makes the runtime's context current
    unsigned long long id = 0;
    const bool have_id = current_ctx_id(&id);
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (have_id) {
        for (int i = 0; i < g_noalloc_used; ++i)
            if (g_noalloc_cache[i].ctx_id == id) {
                *out = g_noalloc_cache[i].ptr;
                return TCHLL_OK;
            }
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(noalloc scratch)");
    if (have_id) {  // a full table gives up the entry the id hashes to
        const int slot = g_noalloc_used < 64 ? g_noalloc_used++ : (int)(id % 64);
        g_noalloc_cache[slot] = NoallocEntry{id, p};
    }
    *out = p;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_exact_count_noalloc(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                           int64_t nnz, const int32_t* edge_u, const int32_t* edge_v,
                                           int64_t n_edges, tchll_count_result* result, void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, result);
    if (rc) return rc;
    CountWs W;
    size_t need = 0;
    carve_count(nullptr, 0, n_nodes, n_edges, W, &need, false);  // padded lists only when they fit too
    if (need > (size_t)TCHLL_NOALLOC_SCRATCH_BYTES) {
        set_error("graph too large for tchll_exact_count_noalloc: needs %zu bytes of scratch (about 8 per edge + "
                  "32 per vertex), the fixed limit is %u bytes; use tchll_exact_count with a workspace",
                  need, (unsigned)TCHLL_NOALLOC_SCRATCH_BYTES);
        return TCHLL_EINVAL;
    }
    void* scratch = nullptr;
    rc = noalloc_scratch_ptr(&scratch);
    if (rc) return rc;
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.result = result;
    P.p = 4;
    // run_count clears the work counters, histogram and result on the stream
    // before any kernel reads them, so leftovers of the previous call are
    // harmless; calls that overlap on the GPU would share the array and race.
    return run_count(P, MODE_EXACT, false, scratch, TCHLL_NOALLOC_SCRATCH_BYTES, (cudaStream_t)stream);
}

// ------------------------------------------------------------- batched ------
// Many graphs in one launch.  The graphs share one CSR with disjoint vertex
// ranges [vbase[g], vbase[g+1]) (ids offset per graph before the CSR build:
// orientation and compaction are per vertex, so each graph's part of the CSR
// equals its own CSR shifted).  Work is a list of chunks that never cross a
// graph; each chunk adds its integer totals to results[g], so per-graph
// results are bit-identical to one graph at a time.

// A graph whose vertex range is malformed gets no chunks (and a status flag
// from check_vbase_kernel); no vbase entry is used as an index unchecked.
__device__ __forceinline__ bool graph_range(const int32_t* base, const int32_t* vbase, int64_t g, int64_t n_nodes,
                                            int64_t& s0, int64_t& s1) {
    const int32_t a = vbase[g], b = vbase[g + 1];
    if (a < 0 || b < a || (int64_t)b > n_nodes) return false;
    s0 = base[a];
    s1 = base[b];
    return s1 >= s0;
}

__global__ void chunk_count_kernel(const int32_t* __restrict__ base, const int32_t* __restrict__ vbase,
                                   int64_t n_graphs, int64_t n_nodes, int chunk, int64_t* cnt) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g <= n_graphs;
         g += (int64_t)gridDim.x * blockDim.x) {
        if (g == n_graphs) {
            cnt[g] = 0;
            continue;
        }
        int64_t s0, s1;
        cnt[g] = graph_range(base, vbase, g, n_nodes, s0, s1) ? (s1 - s0 + chunk - 1) / chunk : 0;
    }
}

__global__ void chunk_fill_kernel(const int32_t* __restrict__ base, const int32_t* __restrict__ vbase,
                                  int64_t n_graphs, int64_t n_nodes, int chunk, const int64_t* __restrict__ coff,
                                  int64_t* cstart, int32_t* clen, int32_t* cgraph) {
    // one warp per graph
    const int lane = threadIdx.x & 31;
    for (int64_t g = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; g < n_graphs;
         g += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int64_t s0 = 0, s1 = 0;
        if (!graph_range(base, vbase, g, n_nodes, s0, s1)) continue;
        const int64_t n = coff[g + 1] - coff[g];
        for (int64_t k = lane; k < n; k += 32) {
            const int64_t st = s0 + k * chunk;
            cstart[coff[g] + k] = st;
            clen[coff[g] + k] = (int32_t)min((int64_t)chunk, s1 - st);
            cgraph[coff[g] + k] = (int32_t)g;
        }
    }
}

__global__ void check_vbase_kernel(const int32_t* __restrict__ vbase, int64_t n_graphs, int64_t n_nodes,
                                   tchll_count_result* results) {
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < n_graphs;
         g += (int64_t)gridDim.x * blockDim.x) {
        const int32_t a = vbase[g], b = vbase[g + 1];
        if (a < 0 || b < a || (int64_t)b > n_nodes) results[g].status |= ST_BAD_ROW;
    }
}

struct BatchWs {
    CountWs cw;
    HybridWs hw;      // HLL edge list (no zero masks)
    int64_t* cnt;     // n_graphs + 1
    int64_t* coff;    // n_graphs + 1 (last entry: number of chunks)
    int64_t* cstart;  // max chunks
    int32_t* clen;
    int32_t* cgraph;
    void* tmp;
    size_t tmp_bytes;
};

static int64_t max_chunks(int64_t n_edges, int64_t n_graphs, int chunk) {
    return n_edges / chunk + n_graphs + 1;
}

static bool carve_batch(void* ws, size_t bytes, int64_t n_nodes, int64_t n_edges, int64_t n_graphs, BatchWs& B,
                        size_t* need) {
    size_t cneed = 0;
    carve_count(nullptr, 0, n_nodes, n_edges, B.cw, &cneed);
    const size_t G = (size_t)n_graphs + 1;
    const size_t MC = (size_t)max_chunks(n_edges, n_graphs, 32);  // any chunk size >= 32 fits
    size_t tb = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, tb, (int64_t*)nullptr, (int64_t*)nullptr, (int)G);
    Carve cv(ws, bytes);
    char* cbase = cv.take<char>(cneed);
    B.cnt = cv.take<int64_t>(G);
    B.coff = cv.take<int64_t>(G);
    B.cstart = cv.take<int64_t>(MC);
    B.clen = cv.take<int32_t>(MC);
    B.cgraph = cv.take<int32_t>(MC);
    B.tmp_bytes = tb;
    B.tmp = cv.take<char>(tb);
    const size_t E = (size_t)(n_edges > 0 ? n_edges : 1);
    B.hw.hll_u = cv.take<int32_t>(E);
    B.hw.hll_v = cv.take<int32_t>(E);
    B.hw.hll_n = cv.take<unsigned long long>(1);
    B.hw.zm = nullptr;
    B.hw.zst = 0;
    if (need) *need = cv.off;
    if (!cv.ok() || cv.dry) return cv.ok();
    carve_count(cbase, cneed, n_nodes, n_edges, B.cw, nullptr);
    return true;
}

// Chunk list over per-graph ranges [base[vbase[g]], base[vbase[g+1]]).
static int build_chunks(const int32_t* base, const int32_t* vbase, int64_t n_graphs, int64_t n_nodes,
                        const BatchWs& B, int chunk, cudaStream_t st) {
    int64_t g = (n_graphs + 256) / 256;
    if (g > (int64_t)sm_count() * 8) g = (int64_t)sm_count() * 8;
    chunk_count_kernel<<<(int)g, 256, 0, st>>>(base, vbase, n_graphs, n_nodes, chunk, B.cnt);
    TCHLL_CHECK_LAUNCH("chunk_count_kernel");
    size_t tb = B.tmp_bytes;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(B.tmp, tb, B.cnt, B.coff, (int)(n_graphs + 1), st));
    count_launch();
    int64_t gw = (n_graphs * 32 + 255) / 256;
    if (gw > (int64_t)sm_count() * 8) gw = (int64_t)sm_count() * 8;
    if (gw < 1) gw = 1;
    chunk_fill_kernel<<<(int)gw, 256, 0, st>>>(base, vbase, n_graphs, n_nodes, chunk, B.coff, B.cstart, B.clen,
                                               B.cgraph);
    TCHLL_CHECK_LAUNCH("chunk_fill_kernel");
    return TCHLL_OK;
}

static int run_batch(CountParams P, bool hybrid, const int32_t* vbase, int64_t n_graphs, void* ws, size_t wsb,
                     cudaStream_t st) {
    const Tuning T = tuning_snapshot();
    BatchWs B;
    size_t need = 0;
    if (!carve_batch(ws, wsb, P.n_nodes, P.n_edges, n_graphs, B, &need) || ws == nullptr) {
        set_error("workspace too small: need %zu bytes, have %zu", need, wsb);
        return TCHLL_EWORKSPACE;
    }
    TCHLL_CUDA(cudaMemsetAsync(P.result, 0, sizeof(tchll_count_result) * n_graphs, st));
    TCHLL_CUDA(cudaMemsetAsync(B.cw.ctr, 0, 4 * sizeof(unsigned long long), st));
    if (n_graphs == 0) return TCHLL_OK;
    {
        int64_t g = (n_graphs + 255) / 256;
        if (g > 1024) g = 1024;
        check_vbase_kernel<<<(int)g, 256, 0, st>>>(vbase, n_graphs, P.n_nodes, P.result);
        TCHLL_CHECK_LAUNCH("check_vbase_kernel");
    }
    P.chunk = T.chunk;
    P.slots_log2 = T.slots_log2;
    P.tiny = T.tiny;
    P.sparse = T.sparse;
    P.n_edges_dev = nullptr;
    P.graph_vbase = vbase;
    P.n_graphs = n_graphs;
    P.n_chunks_dev = B.coff + n_graphs;
    P.chunk_start = B.cstart;
    P.chunk_len = B.clen;
    P.chunk_graph = B.cgraph;
    if (P.n_edges == 0) return TCHLL_OK;
    int rc;
    CountParams Q;
    PhaseScope ps;
    phase_reset(ps);
    P.work = B.cw.ctr;
    // Hybrid: the routing pass also appends the HLL-routed edges to a list
    // (16-byte aligned register rows; else the HLL edges take a second pass
    // over each graph's edges below).
    const bool hll_list = hybrid && ((uintptr_t)P.regs % 16 == 0);
    P.hll_u = hll_list ? B.hw.hll_u : nullptr;
    P.hll_v = hll_list ? B.hw.hll_v : nullptr;
    P.hll_n = hll_list ? B.hw.hll_n : nullptr;
    if (hll_list) TCHLL_CUDA(cudaMemsetAsync(B.hw.hll_n, 0, sizeof(unsigned long long), st));
    phase_mark(ps, 0, st);
    // pairs with a long table side go to the hub kernels, which publish per
    // segment into the graph of x
    const int hub = hub_threshold(P, T);
    if (hybrid) rc = pairs_hist_scan<true>(P, B.cw, hub, T.hub_seg, st, vbase, n_graphs);
    else rc = pairs_hist_scan<false>(P, B.cw, hub, T.hub_seg, st, vbase, n_graphs);
    if (rc) return rc;
    rc = build_chunks(B.cw.off, vbase, n_graphs, P.n_nodes, B, T.chunk, st);  // pair ranges (before the scatter)
    if (rc) return rc;
    if (hybrid) rc = pairs_scatter<true>(P, B.cw, hub, Q, st);
    else rc = pairs_scatter<false>(P, B.cw, hub, Q, st);
    if (rc) return rc;
    phase_mark(ps, 1, st);
    Q.n_edges_dev = nullptr;
    Q.hll_u = nullptr;
    rc = launch_count<MODE_EXACT>(Q, T, false, st);
    if (rc) return rc;
    if (hub > 0) {
        rc = launch_core_pass(P, B.cw, T, ps, st);
        if (rc == TCHLL_OK) rc = launch_hub(P, B.cw, T, ps, st, true);
        if (rc) return rc;
    }
    phase_mark(ps, 2, st);
    phase_used(ps, 0, 1);
    if (!hybrid) return TCHLL_OK;
    if (hll_list) {  // per-edge estimates into each edge's graph
        rc = launch_hll_edges(P, B.hw, T, st);
        phase_mark(ps, 3, st);
        phase_used(ps, 2);
        return rc;
    }
    // HLL-routed edges: chunks over each graph's CSR edge range
    TCHLL_CUDA(cudaMemsetAsync(B.cw.ctr + 1, 0, sizeof(unsigned long long), st));
    rc = build_chunks(P.row_ptr, vbase, n_graphs, P.n_nodes, B, T.chunk, st);
    if (rc) return rc;
    P.work = B.cw.ctr + 1;
    rc = launch_count<MODE_HYB_HLL>(P, T, false, st);
    phase_mark(ps, 3, st);
    phase_used(ps, 2);
    return rc;
}

TCHLL_EXPORT int tchll_batch_workspace_bytes(int64_t n_nodes, int64_t n_edges, int64_t n_graphs, size_t* bytes) {
    TCHLL_ARG(bytes && n_nodes >= 0 && n_edges >= 0 && n_graphs >= 0, "bad arguments");
    BatchWs B;
    carve_batch(nullptr, 0, n_nodes, n_edges, n_graphs, B, bytes);
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_batch_exact_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                                         const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                                         const int32_t* graph_vbase, int64_t n_graphs, tchll_count_result* results,
                                         void* workspace, size_t workspace_bytes, void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, results);
    if (rc) return rc;
    TCHLL_ARG(n_graphs >= 0 && (n_graphs == 0 || graph_vbase), "bad graph table");
    TCHLL_ARG(n_graphs < (int64_t)INT32_MAX, "too many graphs");
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.result = results;
    P.p = 4;
    return run_batch(P, false, graph_vbase, n_graphs, workspace, workspace_bytes, (cudaStream_t)stream);
}

TCHLL_EXPORT int tchll_batch_hybrid_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                          int64_t nnz, const int32_t* edge_u, const int32_t* edge_v,
                                          int64_t n_edges, const int32_t* degrees, const uint8_t* rows,
                                          int64_t n_rows, const int64_t* slot, int32_t p, int64_t gamma,
                                          const int32_t* graph_vbase, int64_t n_graphs,
                                          tchll_count_result* results, void* workspace, size_t workspace_bytes,
                                          void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, results);
    if (rc) return rc;
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_edges == 0 || (degrees && slot), "degrees / slot are null");
    TCHLL_ARG(n_rows == 0 || rows, "register rows are null");
    TCHLL_ARG(n_graphs >= 0 && (n_graphs == 0 || graph_vbase), "bad graph table");
    TCHLL_ARG(n_graphs < (int64_t)INT32_MAX, "too many graphs");
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.degrees = degrees;
    P.regs = rows;
    P.n_rows = n_rows;
    P.slot = slot;
    P.p = p;
    P.gamma = gamma;
    P.result = results;
    return run_batch(P, true, graph_vbase, n_graphs, workspace, workspace_bytes, (cudaStream_t)stream);
}

// cpu_exp estimator variant (cpu_exp/triangle_hll_experiment.py:466-498,
// 652-710): dense registers for every vertex; an edge is exact iff
// min(d+u, d+v) <= threshold (threshold < 0: every edge HLL, the pure-HLL
// count).  Same kernels as the hybrid with gamma = threshold + 1.
TCHLL_EXPORT int tchll_cx_hybrid_count(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx, int64_t nnz,
                                       const int32_t* edge_u, const int32_t* edge_v, int64_t n_edges,
                                       const int32_t* degrees, const uint8_t* regs, const uint8_t* has_all,
                                       int32_t p, int64_t threshold, tchll_count_result* result, void* workspace,
                                       size_t workspace_bytes, void* stream) {
    int rc = check_common(row_ptr, n_nodes, col_idx, nnz, edge_u, edge_v, n_edges, result);
    if (rc) return rc;
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_edges == 0 || (degrees && regs && has_all), "null degrees / registers");
    CountParams P{};
    P.row_ptr = row_ptr;
    P.n_nodes = n_nodes;
    P.col_idx = col_idx;
    P.nnz = nnz;
    P.edge_u = edge_u;
    P.edge_v = edge_v;
    P.n_edges = n_edges;
    P.degrees = degrees;
    P.regs = regs;
    P.n_rows = n_nodes;
    P.has = has_all;
    P.p = p;
    P.gamma = threshold < 0 ? 0 : threshold + 1;
    P.variant = 1;
    P.result = result;
    return run_count(P, 2, false, workspace, workspace_bytes, (cudaStream_t)stream);
}
