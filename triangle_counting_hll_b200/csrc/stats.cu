// stats.cu -- degree statistics and per-graph id helpers.
//
// tchll_degree_stats follows the reference's GPU degree statistics
// (experiment/gpu_graph_stats.py:100-140): for every vertex of positive
// degree, count it, sum d and d^2, track max / min, and histogram floor(log2 d)
// (bucket b holds degrees [2^b, 2^(b+1)-1]; the last bucket takes the rest).
// Here it feeds the launch-shape autotuner, keyed on the forward-degree
// histogram.
#include "common.cuh"

namespace tchll {

constexpr int kLogBuckets = 32;

__global__ void degree_stats_kernel(const int32_t* __restrict__ degrees, const int32_t* __restrict__ row_ptr,
                                    int64_t n, unsigned long long* log_hist, unsigned long long* sums,
                                    int32_t* minmax) {
    __shared__ unsigned long long h[kLogBuckets];
    for (int i = threadIdx.x; i < kLogBuckets; i += blockDim.x) h[i] = 0;
    __syncthreads();
    unsigned long long act = 0, sum = 0, sumsq = 0;
    int32_t mx = 0, mn = INT32_MAX;
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t d = degrees ? degrees[v] : row_ptr[v + 1] - row_ptr[v];
        if (d <= 0) continue;
        ++act;
        sum += (unsigned long long)d;
        sumsq += (unsigned long long)d * (unsigned long long)d;
        mx = d > mx ? d : mx;
        mn = d < mn ? d : mn;
        int b = 31 - __clz(d);
        if (b >= kLogBuckets) b = kLogBuckets - 1;
        atomicAdd(&h[b], 1ull);
    }
    act = warp_sum_u64(act);
    sum = warp_sum_u64(sum);
    sumsq = warp_sum_u64(sumsq);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = max(mx, __shfl_xor_sync(FULL, mx, o));
        mn = min(mn, __shfl_xor_sync(FULL, mn, o));
    }
    if ((threadIdx.x & 31) == 0) {
        if (act) {
            atomicAdd(sums + 0, act);
            atomicAdd(sums + 1, sum);
            atomicAdd(sums + 2, sumsq);
            atomicMax(minmax + 0, mx);
            atomicMin(minmax + 1, mn);
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < kLogBuckets; i += blockDim.x)
        if (h[i]) atomicAdd(log_hist + i, h[i]);
}

__global__ void stats_init_kernel(unsigned long long* log_hist, unsigned long long* sums, int32_t* minmax) {
    const int i = threadIdx.x;
    if (i < kLogBuckets) log_hist[i] = 0;
    if (i < 3) sums[i] = 0;
    if (i == 0) {
        minmax[0] = 0;
        minmax[1] = INT32_MAX;
    }
}

// local[v] = v - vbase[g] for v in graph g's range, v elsewhere.
__global__ void local_ids_kernel(const int32_t* __restrict__ vbase, int64_t n_graphs, int64_t n_nodes,
                                 int64_t* local) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n_nodes;
         v += (int64_t)gridDim.x * blockDim.x) {
        // graph of v: last g with vbase[g] <= v (ranges are non-decreasing)
        int64_t lo = 0, hi = n_graphs;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (vbase[mid] <= v) lo = mid + 1; else hi = mid;
        }
        const int64_t g = lo - 1;
        local[v] = (g >= 0 && g < n_graphs && v < vbase[g + 1]) ? v - vbase[g] : v;
    }
}

}  // namespace tchll

using namespace tchll;

TCHLL_EXPORT int tchll_degree_stats(const int32_t* degrees, const int32_t* row_ptr, int64_t n, uint64_t* log_hist32,
                                    uint64_t* sums3, int32_t* minmax2, void* stream) {
    TCHLL_ARG((degrees == nullptr) != (row_ptr == nullptr), "pass exactly one of degrees / row_ptr");
    TCHLL_ARG(n >= 0 && log_hist32 && sums3 && minmax2, "bad arguments");
    cudaStream_t st = (cudaStream_t)stream;
    stats_init_kernel<<<1, 32, 0, st>>>((unsigned long long*)log_hist32, (unsigned long long*)sums3, minmax2);
    TCHLL_CHECK_LAUNCH("stats_init_kernel");
    if (n == 0) return TCHLL_OK;
    int64_t g = (n + 255) / 256;
    if (g > (int64_t)sm_count() * 4) g = (int64_t)sm_count() * 4;
    degree_stats_kernel<<<(int)g, 256, 0, st>>>(degrees, row_ptr, n, (unsigned long long*)log_hist32,
                                                (unsigned long long*)sums3, minmax2);
    TCHLL_CHECK_LAUNCH("degree_stats_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_batch_local_ids(const int32_t* graph_vbase, int64_t n_graphs, int64_t n_nodes,
                                       int64_t* local_ids, void* stream) {
    TCHLL_ARG(n_graphs >= 0 && n_nodes >= 0 && (n_graphs == 0 || graph_vbase) && (n_nodes == 0 || local_ids),
              "bad arguments");
    if (n_nodes == 0) return TCHLL_OK;
    int64_t g = (n_nodes + 255) / 256;
    if (g > (int64_t)sm_count() * 8) g = (int64_t)sm_count() * 8;
    local_ids_kernel<<<(int)g, 256, 0, (cudaStream_t)stream>>>(graph_vbase, n_graphs, n_nodes, local_ids);
    TCHLL_CHECK_LAUNCH("local_ids_kernel");
    return TCHLL_OK;
}
