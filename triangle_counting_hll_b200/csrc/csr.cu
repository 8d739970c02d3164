// csr.cu -- device construction of the oriented CSR.
//
// Reference semantics (ChitandaEruQ/triangle_counting_hll):
//   load + dedup   src/graph.py:8-26 (canonical (min,max), self-loops dropped,
//                  set semantics), experiment/exp_gpu.py:288-303 (np.unique)
//   compaction     experiment/exp_gpu.py:317-323 (np.union1d of endpoints;
//                  ids become ranks) == src/gpu_graph.py:19-37 node_index
//   degree/orient  src/graph.py:41-54, experiment/exp_gpu.py:325-339:
//                  u -> v iff (deg u, id u) < (deg v, id v); compaction is
//                  monotone, so comparing compacted ids gives the same order
//   CSR            experiment/exp_gpu.py:350-362 (np.lexsort by (src, dst))
//
// Pipeline: largest id (one 16-byte read-back) -> pack canonical pairs into
// 2k-bit keys, k = bits of the largest id -> radix sort -> unique -> node
// table and remap -> degree histogram -> orient -> stable radix sort of the
// (src, dst) pairs by src alone -> row pointers from the sorted sources.
// The node table (compacted id = rank of the raw id among the endpoints)
// comes from a direct table when the id space fits the workspace (flag every
// endpoint id, scan the flags: rank[id] is the scan, one gather per
// endpoint), else from sorting and deduplicating all endpoints and a binary
// search per endpoint.
//
// One sort by src is enough for rows sorted by dst: the pairs reach it in
// canonical (a, b) order, a < b, and compaction keeps that order.  For a
// source s, the edges it gained by flipping (b = s, dst a < s) come before
// the edges it kept (a = s, dst b > s), each group in ascending dst, so a
// stable sort by src leaves every row ascending.
//
// Sorting, unique and scans use CUB (header templates compiled into this
// library); the other passes are kernels written here.
#include <cub/cub.cuh>

#include "common.cuh"

namespace tchll {

// Canonical keys are (a << k) | b with a < b < 2^k.  The all-ones key of 2k
// bits is never a canonical pair (it needs a == b), so it marks dropped
// self-loops and sorts after every real key.
__host__ __device__ __forceinline__ uint64_t key_sentinel(int k) { return (k >= 32) ? ~0ull : ((1ull << (2 * k)) - 1ull); }
constexpr uint32_t kEndSentinel = 0xFFFFFFFFu;

struct CsrWs {
    uint64_t* k0;
    uint64_t* k1;
    uint32_t* e0;
    uint32_t* e1;
    int32_t* deg;
    int32_t* fdeg;
    int32_t* ca;
    int32_t* cb;
    int64_t* cnt;  // [0] unique keys, [1] unique endpoints, [2] negative-id flag, [3] largest id
    void* tmp;
    size_t tmp_bytes;
};

static size_t csr_cub_tmp(int64_t n_raw) {
    const int R = (int)(n_raw > 0 ? n_raw : 1);
    size_t a = 0, b = 0, c = 0, d = 0, e = 0, f = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, a, (uint64_t*)nullptr, (uint64_t*)nullptr, R, 0, 63);
    cub::DeviceSelect::Unique(nullptr, b, (uint64_t*)nullptr, (uint64_t*)nullptr, (int64_t*)nullptr, R);
    cub::DeviceRadixSort::SortKeys(nullptr, c, (uint32_t*)nullptr, (uint32_t*)nullptr, 2 * R, 0, 32);
    cub::DeviceSelect::Unique(nullptr, d, (uint32_t*)nullptr, (uint32_t*)nullptr, (int64_t*)nullptr, 2 * R);
    cub::DeviceScan::ExclusiveSum(nullptr, e, (int32_t*)nullptr, (int32_t*)nullptr, 2 * R + 1);
    cub::DeviceRadixSort::SortPairs(nullptr, f, (uint32_t*)nullptr, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (uint32_t*)nullptr, R, 0, 32);
    size_t m = a;
    if (b > m) m = b;
    if (c > m) m = c;
    if (d > m) m = d;
    if (e > m) m = e;
    if (f > m) m = f;
    return m;
}

static bool carve_csr(void* ws, size_t bytes, int64_t n_raw, CsrWs& W, size_t* need) {
    const size_t R = (size_t)(n_raw > 0 ? n_raw : 1);
    Carve cv(ws, bytes);
    W.k0 = cv.take<uint64_t>(R);
    W.k1 = cv.take<uint64_t>(R);
    W.e0 = cv.take<uint32_t>(2 * R);
    W.e1 = cv.take<uint32_t>(2 * R);
    W.deg = cv.take<int32_t>(2 * R + 1);
    W.fdeg = cv.take<int32_t>(2 * R + 2);
    W.ca = cv.take<int32_t>(R);
    W.cb = cv.take<int32_t>(R);
    W.cnt = cv.take<int64_t>(4);
    W.tmp_bytes = csr_cub_tmp(n_raw);
    W.tmp = cv.take<char>(W.tmp_bytes);
    if (need) *need = cv.off;
    return cv.ok();
}

static int grid_n(int64_t n, int threads = 256) {
    int64_t g = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 32;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// Grid-stride loop that whole warps enter and leave together (bodies with
// warp shuffles): i may reach past n in the last pass; test it in the body.
#define WARP_GRID_STRIDE(i, n)                                                               \
    for (int64_t _wb = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u),              \
                 i = _wb + (threadIdx.x & 31u);                                              \
         _wb < (n); _wb += (int64_t)gridDim.x * blockDim.x, i = _wb + (threadIdx.x & 31u))

// Largest endpoint id (atomicMax, one per warp) and the negative-id flag.
__global__ void max_id_kernel(const int32_t* __restrict__ ru, const int32_t* __restrict__ rv, int64_t n,
                              int64_t* cnt) {
    int32_t mx = 0;
    bool neg = false;
    GRID_STRIDE(i, n) {
        const int32_t u = ru[i], v = rv[i];
        neg |= (u < 0) | (v < 0);
        mx = max(mx, max(u, v));
    }
    mx = __reduce_max_sync(0xFFFFFFFFu, mx);
    neg = __any_sync(0xFFFFFFFFu, neg);
    if ((threadIdx.x & 31) == 0) {
        atomicMax((unsigned long long*)(cnt + 3), (unsigned long long)mx);
        if (neg) cnt[2] = 1;
    }
}

__global__ void canon_kernel(const int32_t* __restrict__ ru, const int32_t* __restrict__ rv, int64_t n, int k,
                             uint64_t* keys) {
    const uint64_t sent = key_sentinel(k);
    GRID_STRIDE(i, n) {
        const int32_t u = ru[i], v = rv[i];
        const uint32_t a = (uint32_t)(u < v ? u : v), b = (uint32_t)(u < v ? v : u);
        keys[i] = (u == v || u < 0 || v < 0) ? sent : (((uint64_t)a << k) | b);
    }
}

// Endpoints of the unique keys (sentinels become kEndSentinel).
__global__ void ends_kernel(const uint64_t* __restrict__ keys, int64_t cap, const int64_t* cnt, int kb,
                            uint32_t* ends) {
    const int64_t nk = cnt[0];
    const uint64_t sent = key_sentinel(kb), lo = (1ull << kb) - 1ull;
    GRID_STRIDE(i, cap) {
        uint64_t k = i < nk ? keys[i] : sent;
        if (k == sent) {
            ends[2 * i] = kEndSentinel;
            ends[2 * i + 1] = kEndSentinel;
        } else {
            ends[2 * i] = (uint32_t)(k >> kb);
            ends[2 * i + 1] = (uint32_t)(k & lo);
        }
    }
}

__device__ __forceinline__ int64_t lower_bound_u32(const uint32_t* a, int64_t n, uint32_t x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

// Number of real edges / nodes: drop the trailing sentinel when present.
__device__ __forceinline__ int64_t n_real_edges(const uint64_t* keys, const int64_t* cnt, int kb) {
    const int64_t nk = cnt[0];
    return (nk > 0 && keys[nk - 1] == key_sentinel(kb)) ? nk - 1 : nk;
}
__device__ __forceinline__ int64_t n_real_nodes(const uint32_t* nodes, const int64_t* cnt) {
    const int64_t nn = cnt[1];
    return (nn > 0 && nodes[nn - 1] == kEndSentinel) ? nn - 1 : nn;
}

// deg[a] += (number of lanes with this a) from the last lane of each run of
// equal a (the keys are sorted by a, so runs are contiguous lanes); lanes
// past the end pass a = -1.
__device__ __forceinline__ void add_runs(int32_t* deg, int32_t a, int lane) {
    const unsigned FULLM = 0xFFFFFFFFu;
    const int32_t na = __shfl_down_sync(FULLM, a, 1);
    const bool tail = lane == 31 || na != a;  // the run's last lane
    const unsigned tails = __ballot_sync(FULLM, tail);
    if (a >= 0 && tail) {
        // the run starts after the previous tail
        const unsigned below = tails & ((1u << lane) - 1u);
        const int start = below ? 32 - __clz(below) : 0;
        atomicAdd(deg + a, lane - start + 1);
    }
}

// Sort path: binary search of both endpoints in the sorted node table.
__global__ void remap_kernel(const uint64_t* __restrict__ keys, int64_t cap, const uint32_t* __restrict__ nodes,
                             const int64_t* cnt, int kb, int32_t* ca, int32_t* cb, int32_t* deg) {
    const int64_t ne = n_real_edges(keys, cnt, kb);
    const int64_t nn = n_real_nodes(nodes, cnt);
    const uint64_t lo = (1ull << kb) - 1ull;
    const int lane = threadIdx.x & 31;
    WARP_GRID_STRIDE(i, cap) {
        const bool in = i < ne;
        int32_t a = -1;
        if (in) {
            const uint64_t k = keys[i];
            a = (int32_t)lower_bound_u32(nodes, nn, (uint32_t)(k >> kb));
            const int32_t b = (int32_t)lower_bound_u32(nodes, nn, (uint32_t)(k & lo));
            ca[i] = a;
            cb[i] = b;
            atomicAdd(deg + b, 1);
        }
        add_runs(deg, a, lane);
    }
}

// Direct path: flag[id] = 1 for both endpoints of every unique edge (flag
// zeroed over [0, max id + 1] before).  The keys are sorted, so neighbouring
// lanes mostly share a: only the first lane of each run stores it.
__global__ void flag_ends_kernel(const uint64_t* __restrict__ keys, int64_t cap, const int64_t* cnt, int kb,
                                 int32_t* flag) {
    const int64_t ne = n_real_edges(keys, cnt, kb);
    const uint64_t lo = (1ull << kb) - 1ull;
    const int lane = threadIdx.x & 31;
    WARP_GRID_STRIDE(i, cap) {
        const bool in = i < ne;
        const uint64_t k = in ? keys[i] : 0;
        const uint32_t a = (uint32_t)(k >> kb);
        const uint32_t pa = __shfl_up_sync(0xFFFFFFFFu, a, 1);
        const bool pin = __shfl_up_sync(0xFFFFFFFFu, (int)in, 1) != 0;
        if (in) {
            if (lane == 0 || !pin || pa != a) flag[a] = 1;
            flag[k & lo] = 1;
        }
    }
}

// Direct path, after rank = exclusive scan of flag over [0, ids] (ids = max
// id + 2 entries): the node table nodes[rank[id]] = id for flagged ids, and
// the number of nodes in cnt[1] (its sort-path meaning).
__global__ void rank_nodes_kernel(const int32_t* __restrict__ flag, const int32_t* __restrict__ rank, int64_t ids,
                                  uint32_t* nodes, int64_t* cnt) {
    GRID_STRIDE(i, ids) {
        if (i == ids - 1) cnt[1] = rank[i];  // flag[ids - 1] = 0: the total
        else if (flag[i]) nodes[rank[i]] = (uint32_t)i;
    }
}

// Direct path: both endpoints of every unique edge through the rank table.
__global__ void remap_direct_kernel(const uint64_t* __restrict__ keys, int64_t cap, const int32_t* __restrict__ rank,
                                    const int64_t* cnt, int kb, int32_t* ca, int32_t* cb, int32_t* deg) {
    const int64_t ne = n_real_edges(keys, cnt, kb);
    const uint64_t lo = (1ull << kb) - 1ull;
    const int lane = threadIdx.x & 31;
    WARP_GRID_STRIDE(i, cap) {
        const bool in = i < ne;
        int32_t a = -1;
        if (in) {
            const uint64_t k = keys[i];
            a = __ldg(rank + (k >> kb));
            const int32_t b = __ldg(rank + (k & lo));
            ca[i] = a;
            cb[i] = b;
            atomicAdd(deg + b, 1);
        }
        add_runs(deg, a, lane);
    }
}

__global__ void sizes_kernel(const uint64_t* keys, const uint32_t* nodes, const int64_t* cnt, int kb, int direct,
                             int64_t* sizes) {
    if (cnt[2]) {
        sizes[0] = -1;
        sizes[1] = -1;
        return;
    }
    sizes[0] = direct ? cnt[1] : n_real_nodes(nodes, cnt);
    sizes[1] = n_real_edges(keys, cnt, kb);
}

// Orientation u -> v iff (deg u, u) < (deg v, v): the pair (src, dst) of
// edge i goes to okey[i] / oval[i] (canonical order kept for the stable sort).
__global__ void orient_kernel(const int32_t* __restrict__ ca, const int32_t* __restrict__ cb, int64_t ne,
                              const int32_t* __restrict__ deg, uint32_t* okey, uint32_t* oval) {
    GRID_STRIDE(i, ne) {
        const int32_t a = ca[i], b = cb[i];
        const int32_t da = deg[a], db = deg[b];
        const bool first = (da < db) || (da == db && a < b);
        okey[i] = (uint32_t)(first ? a : b);
        oval[i] = (uint32_t)(first ? b : a);
    }
}

// row_ptr from the ascending sources src[0 .. ne): entry i is the first edge
// of every row s in (src[i-1], src[i]] (src[-1] = -1, src[ne] = n_nodes),
// so each of row_ptr[0 .. n_nodes] is written exactly once.
__global__ void row_ptr_kernel(const int32_t* __restrict__ src, int64_t ne, int64_t n_nodes, int32_t* row_ptr) {
    GRID_STRIDE(i, ne + 1) {
        const int64_t lo = i > 0 ? (int64_t)src[i - 1] : -1;
        const int64_t hi = i < ne ? (int64_t)src[i] : n_nodes;
        for (int64_t r = lo + 1; r <= hi; ++r) row_ptr[r] = (int32_t)i;
    }
}

__global__ void copy_nodes_kernel(const uint32_t* __restrict__ nodes, int64_t n, const int32_t* __restrict__ row_ptr,
                                  const int32_t* __restrict__ deg, int32_t* node_ids, int32_t* degrees,
                                  int32_t* undirected) {
    GRID_STRIDE(i, n) {
        node_ids[i] = (int32_t)nodes[i];
        degrees[i] = row_ptr[i + 1] - row_ptr[i];
        if (undirected) undirected[i] = deg[i];
    }
}

static int bits_for(int64_t maxv) {
    int b = 1;
    while (b < 63 && (maxv >> b) != 0) ++b;
    return b;
}

// ------------------------------------------------- forward_adj -> CSR ------
__global__ void iota_kernel(int64_t* a, int64_t n) {
    GRID_STRIDE(i, n) a[i] = i;
}

__global__ void gather_deg_kernel(const int64_t* __restrict__ lens, const int64_t* __restrict__ order, int64_t n,
                                  int32_t* degrees, int32_t* deg_scan_in) {
    GRID_STRIDE(i, n) {
        const int32_t d = (int32_t)lens[order[i]];
        degrees[i] = d;
        deg_scan_in[i] = d;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) deg_scan_in[n] = 0;
}

__device__ __forceinline__ int64_t upper_bound_i32(const int32_t* a, int64_t n, int64_t x) {
    int64_t lo = 0, hi = n;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if ((int64_t)a[mid] <= x) lo = mid + 1; else hi = mid;
    }
    return lo;
}

__global__ void adj_fill_kernel(const int64_t* __restrict__ sorted_keys, int64_t n,
                                const int64_t* __restrict__ order, const int64_t* __restrict__ dict_off,
                                const int32_t* __restrict__ row_ptr, const int64_t* __restrict__ values, int64_t nnz,
                                int32_t* col_idx, int32_t* edge_u, int32_t* edge_v, unsigned long long* missing) {
    unsigned long long miss = 0;
    GRID_STRIDE(k, nnz) {
        const int64_t row = upper_bound_i32(row_ptr, n + 1, k) - 1;
        const int64_t src = dict_off[order[row]] + (k - row_ptr[row]);
        const int64_t x = values[src];
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (sorted_keys[mid] < x) lo = mid + 1; else hi = mid;
        }
        int32_t c = (int32_t)lo;
        if (lo >= n || sorted_keys[lo] != x) {
            ++miss;
            c = -1;
        }
        col_idx[k] = c;
        edge_v[k] = c;
        edge_u[k] = (int32_t)row;
    }
    if (miss) atomicAdd(missing, miss);
}

__global__ void zero_kernel(int64_t* p) { *p = 0; }

}  // namespace tchll

using namespace tchll;

TCHLL_EXPORT int tchll_csr_workspace_bytes(int64_t n_raw, size_t* bytes) {
    TCHLL_ARG(bytes && n_raw >= 0, "bad arguments");
    TCHLL_ARG(n_raw < (int64_t)(INT32_MAX / 2), "edge list longer than 2^30 entries");
    CsrWs W;
    carve_csr(nullptr, 0, n_raw, W, bytes);
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_csr_build_phase1(const int32_t* raw_u, const int32_t* raw_v, int64_t n_raw, int64_t* sizes,
                                        void* workspace, size_t workspace_bytes, void* stream) {
    TCHLL_ARG(sizes != nullptr && n_raw >= 0, "bad arguments");
    TCHLL_ARG(n_raw == 0 || (raw_u && raw_v), "null edge arrays");
    TCHLL_ARG(n_raw < (int64_t)(INT32_MAX / 2), "edge list longer than 2^30 entries");
    CsrWs W;
    size_t need = 0;
    if (!carve_csr(workspace, workspace_bytes, n_raw, W, &need) || !workspace) {
        set_error("workspace too small: need %zu bytes, have %zu", need, workspace_bytes);
        return TCHLL_EWORKSPACE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const int R = (int)(n_raw > 0 ? n_raw : 1);
    TCHLL_CUDA(cudaMemsetAsync(W.cnt, 0, 4 * sizeof(int64_t), st));
    TCHLL_CUDA(cudaMemsetAsync(W.deg, 0, (2 * (size_t)R + 1) * sizeof(int32_t), st));
    if (n_raw == 0) {
        TCHLL_CUDA(cudaMemsetAsync(sizes, 0, 2 * sizeof(int64_t), st));
        return TCHLL_OK;
    }
    // the largest id sizes the keys and picks the node-table method: one
    // 16-byte read-back (the stream is waited for here)
    max_id_kernel<<<grid_n(n_raw), 256, 0, st>>>(raw_u, raw_v, n_raw, W.cnt);
    TCHLL_CHECK_LAUNCH("max_id_kernel");
    int64_t hc[2] = {0, 0};
    TCHLL_CUDA(cudaMemcpyAsync(hc, W.cnt + 2, sizeof(hc), cudaMemcpyDeviceToHost, st));
    TCHLL_CUDA(cudaStreamSynchronize(st));
    if (hc[0]) {  // a negative id: sizes -1, nothing else
        sizes_kernel<<<1, 1, 0, st>>>(W.k0, W.e0, W.cnt, 1, 0, sizes);
        TCHLL_CHECK_LAUNCH("sizes_kernel");
        return TCHLL_OK;
    }
    const int64_t max_id = hc[1];
    const int kb = bits_for(max_id);
    canon_kernel<<<grid_n(n_raw), 256, 0, st>>>(raw_u, raw_v, n_raw, kb, W.k0);
    TCHLL_CHECK_LAUNCH("canon_kernel");
    size_t tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceRadixSort::SortKeys(W.tmp, tb, W.k0, W.k1, R, 0, 2 * kb, st));
    count_launch();
    tb = W.tmp_bytes;
    TCHLL_CUDA(cub::DeviceSelect::Unique(W.tmp, tb, W.k1, W.k0, W.cnt + 0, R, st));
    count_launch();
    // direct rank table when ids 0 .. max_id (+ a zero flag) fit the 2R-entry
    // endpoint buffers, else sort and deduplicate the endpoints
    const int64_t ids = max_id + 2;
    const int direct = ids <= 2 * (int64_t)R ? 1 : 0;
    if (direct) {
        TCHLL_CUDA(cudaMemsetAsync(W.fdeg, 0, (size_t)ids * sizeof(int32_t), st));
        flag_ends_kernel<<<grid_n(n_raw), 256, 0, st>>>(W.k0, n_raw, W.cnt, kb, W.fdeg);
        TCHLL_CHECK_LAUNCH("flag_ends_kernel");
        int32_t* rank = reinterpret_cast<int32_t*>(W.e1);
        tb = W.tmp_bytes;
        TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(W.tmp, tb, W.fdeg, rank, (int)ids, st));
        count_launch();
        rank_nodes_kernel<<<grid_n(ids), 256, 0, st>>>(W.fdeg, rank, ids, W.e0, W.cnt);
        TCHLL_CHECK_LAUNCH("rank_nodes_kernel");
        remap_direct_kernel<<<grid_n(n_raw), 256, 0, st>>>(W.k0, n_raw, rank, W.cnt, kb, W.ca, W.cb, W.deg);
        TCHLL_CHECK_LAUNCH("remap_direct_kernel");
    } else {
        ends_kernel<<<grid_n(n_raw), 256, 0, st>>>(W.k0, n_raw, W.cnt, kb, W.e0);
        TCHLL_CHECK_LAUNCH("ends_kernel");
        tb = W.tmp_bytes;
        TCHLL_CUDA(cub::DeviceRadixSort::SortKeys(W.tmp, tb, W.e0, W.e1, 2 * R, 0, 32, st));
        count_launch();
        tb = W.tmp_bytes;
        TCHLL_CUDA(cub::DeviceSelect::Unique(W.tmp, tb, W.e1, W.e0, W.cnt + 1, 2 * R, st));
        count_launch();
        remap_kernel<<<grid_n(n_raw), 256, 0, st>>>(W.k0, n_raw, W.e0, W.cnt, kb, W.ca, W.cb, W.deg);
        TCHLL_CHECK_LAUNCH("remap_kernel");
    }
    sizes_kernel<<<1, 1, 0, st>>>(W.k0, W.e0, W.cnt, kb, direct, sizes);
    TCHLL_CHECK_LAUNCH("sizes_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_csr_build_phase2(int64_t n_raw, int64_t n_nodes, int64_t n_edges, int32_t* row_ptr,
                                        int32_t* col_idx, int32_t* degrees, int32_t* node_ids, int32_t* edge_u,
                                        int32_t* edge_v, int32_t* undirected_degrees, void* workspace,
                                        size_t workspace_bytes, void* stream) {
    TCHLL_ARG(n_nodes >= 0 && n_edges >= 0 && n_edges <= n_raw && n_nodes <= 2 * n_raw, "sizes out of range");
    TCHLL_ARG(row_ptr != nullptr, "row_ptr is null");
    TCHLL_ARG(n_nodes == 0 || (degrees && node_ids), "null node outputs");
    TCHLL_ARG(n_edges == 0 || (col_idx && edge_u && edge_v), "null edge outputs");
    CsrWs W;
    size_t need = 0;
    if (!carve_csr(workspace, workspace_bytes, n_raw, W, &need) || !workspace) {
        set_error("workspace too small: need %zu bytes, have %zu", need, workspace_bytes);
        return TCHLL_EWORKSPACE;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (n_edges > 0) {
        // the pairs in the first half of k1's bytes (2 n_raw uint32 >= 2 n_edges);
        // sorted by src straight into edge_u (src) and col_idx (dst)
        uint32_t* okey = reinterpret_cast<uint32_t*>(W.k1);
        uint32_t* oval = okey + n_edges;
        const int kn = bits_for(n_nodes > 1 ? n_nodes - 1 : 1);
        orient_kernel<<<grid_n(n_edges), 256, 0, st>>>(W.ca, W.cb, n_edges, W.deg, okey, oval);
        TCHLL_CHECK_LAUNCH("orient_kernel");
        size_t tb = W.tmp_bytes;
        TCHLL_CUDA(cub::DeviceRadixSort::SortPairs(W.tmp, tb, okey, reinterpret_cast<uint32_t*>(edge_u), oval,
                                                   reinterpret_cast<uint32_t*>(col_idx), (int)n_edges, 0, kn, st));
        count_launch();
        TCHLL_CUDA(cudaMemcpyAsync(edge_v, col_idx, (size_t)n_edges * sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    }
    row_ptr_kernel<<<grid_n(n_edges + 1), 256, 0, st>>>(edge_u, n_edges, n_nodes, row_ptr);
    TCHLL_CHECK_LAUNCH("row_ptr_kernel");
    if (n_nodes > 0) {
        copy_nodes_kernel<<<grid_n(n_nodes), 256, 0, st>>>(W.e0, n_nodes, row_ptr, W.deg, node_ids, degrees,
                                                            undirected_degrees);
        TCHLL_CHECK_LAUNCH("copy_nodes_kernel");
    }
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_adj_workspace_bytes(int64_t n, int64_t nnz, size_t* bytes) {
    TCHLL_ARG(bytes && n >= 0 && nnz >= 0, "bad arguments");
    TCHLL_ARG(n < (int64_t)INT32_MAX - 1 && nnz <= (int64_t)INT32_MAX, "int32 CSR limits exceeded");
    const int N = (int)(n > 0 ? n : 1);
    size_t a = 0, b = 0, c = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, a, (int64_t*)nullptr, (int64_t*)nullptr, N + 1);
    cub::DeviceRadixSort::SortPairs(nullptr, b, (int64_t*)nullptr, (int64_t*)nullptr, (int64_t*)nullptr,
                                    (int64_t*)nullptr, N);
    cub::DeviceScan::ExclusiveSum(nullptr, c, (int32_t*)nullptr, (int32_t*)nullptr, N + 1);
    size_t m = a > b ? a : b;
    if (c > m) m = c;
    Carve cv(nullptr, 0);
    cv.take<int64_t>((size_t)N + 1);  // dict offsets
    cv.take<int64_t>((size_t)N + 1);  // lens copy with trailing 0
    cv.take<int64_t>((size_t)N);      // iota
    cv.take<int32_t>((size_t)N + 1);  // degree scan input
    cv.take<char>(m);
    *bytes = cv.off;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_csr_from_adjacency(const int64_t* keys, const int64_t* lens, int64_t n,
                                          const int64_t* values, int64_t nnz, int64_t* node_ids, int32_t* row_ptr,
                                          int32_t* degrees, int32_t* col_idx, int32_t* edge_u, int32_t* edge_v,
                                          int64_t* order, int64_t* missing, void* workspace, size_t workspace_bytes,
                                          void* stream) {
    TCHLL_ARG(n >= 0 && nnz >= 0, "negative size");
    TCHLL_ARG(row_ptr && missing, "null output");
    TCHLL_ARG(n == 0 || (keys && lens && node_ids && degrees && order), "null node arrays");
    TCHLL_ARG(nnz == 0 || (values && col_idx && edge_u && edge_v), "null edge arrays");
    size_t need = 0;
    int rc = tchll_adj_workspace_bytes(n, nnz, &need);
    if (rc) return rc;
    TCHLL_ARG(workspace != nullptr && workspace_bytes >= need, "workspace too small: need %zu bytes", need);
    const int N = (int)(n > 0 ? n : 1);
    size_t a = 0, b = 0, c = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, a, (int64_t*)nullptr, (int64_t*)nullptr, N + 1);
    cub::DeviceRadixSort::SortPairs(nullptr, b, (int64_t*)nullptr, (int64_t*)nullptr, (int64_t*)nullptr,
                                    (int64_t*)nullptr, N);
    cub::DeviceScan::ExclusiveSum(nullptr, c, (int32_t*)nullptr, (int32_t*)nullptr, N + 1);
    size_t m = a > b ? a : b;
    if (c > m) m = c;
    Carve cv(workspace, workspace_bytes);
    int64_t* dict_off = cv.take<int64_t>((size_t)N + 1);
    int64_t* lens0 = cv.take<int64_t>((size_t)N + 1);
    int64_t* iota = cv.take<int64_t>((size_t)N);
    int32_t* dscan = cv.take<int32_t>((size_t)N + 1);
    void* tmp = cv.take<char>(m);
    cudaStream_t st = (cudaStream_t)stream;
    zero_kernel<<<1, 1, 0, st>>>(missing);
    TCHLL_CHECK_LAUNCH("zero_kernel");
    if (n == 0) {
        TCHLL_CUDA(cudaMemsetAsync(row_ptr, 0, sizeof(int32_t), st));
        return TCHLL_OK;
    }
    TCHLL_CUDA(cudaMemcpyAsync(lens0, lens, sizeof(int64_t) * n, cudaMemcpyDeviceToDevice, st));
    TCHLL_CUDA(cudaMemsetAsync(lens0 + n, 0, sizeof(int64_t), st));
    size_t tb = m;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, lens0, dict_off, (int)(n + 1), st));
    count_launch();
    iota_kernel<<<grid_n(n), 256, 0, st>>>(iota, n);
    TCHLL_CHECK_LAUNCH("iota_kernel");
    tb = m;
    TCHLL_CUDA(cub::DeviceRadixSort::SortPairs(tmp, tb, keys, node_ids, iota, order, (int)n, 0, 64, st));
    count_launch();
    gather_deg_kernel<<<grid_n(n), 256, 0, st>>>(lens, order, n, degrees, dscan);
    TCHLL_CHECK_LAUNCH("gather_deg_kernel");
    tb = m;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, dscan, row_ptr, (int)(n + 1), st));
    count_launch();
    if (nnz > 0) {
        adj_fill_kernel<<<grid_n(nnz), 256, 0, st>>>(node_ids, n, order, dict_off, row_ptr, values, nnz, col_idx,
                                                    edge_u, edge_v, (unsigned long long*)missing);
        TCHLL_CHECK_LAUNCH("adj_fill_kernel");
    }
    return TCHLL_OK;
}
