// hll.cu -- HyperLogLog sketch construction and estimation.
//
// Reference semantics (ChitandaEruQ/triangle_counting_hll):
//   hash       src/hll.py:13-19 (splitmix64 finaliser, bit for bit)
//   update     src/hll.py:81-91, src/gpu_hll.py:70-81
//   sketches   src/hybrid.py:15-41 (rows for forward degree >= theta),
//              src/gpu_hll.py:47-81 (dense n x 2^p layout + has_sketch)
//   estimate   src/hll.py:37-54,98-100,112-120
//
// Sketch build: one CTA per sketched vertex.  The CTA stages the 2^p-byte row
// in shared memory (words of four registers, byte max by compare-and-swap),
// hashes the vertex's neighbour list with coalesced loads, then writes the row
// out with 16-byte stores.  CTAs walk the vertex range in tiles of 256 ids,
// compacting the tile's sketched vertices with warp ballots, so vertices below
// the threshold cost one coalesced read.
#include <cub/cub.cuh>

#include "common.cuh"
#include "hll_device.cuh"

namespace tchll {

constexpr int kSketchThreads = 256;

template <bool DENSE>
__global__ void __launch_bounds__(kSketchThreads)
    sketch_kernel(const int32_t* __restrict__ row_ptr, int64_t n_nodes, const int32_t* __restrict__ col_idx,
                  const int64_t* __restrict__ keys, int64_t nnz, int64_t theta, int p, uint8_t* has,
                  const int64_t* __restrict__ slot, int64_t n_rows, uint8_t* rows) {
    extern __shared__ __align__(16) uint32_t words[];
    __shared__ int list[kSketchThreads];
    __shared__ int warp_cnt[kSketchThreads / 32];
    __shared__ int total;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int m = 1 << p;
    const int nwords = m >> 2;
    for (int64_t base = (int64_t)blockIdx.x * kSketchThreads; base < n_nodes;
         base += (int64_t)gridDim.x * kSketchThreads) {
        const int64_t u = base + tid;
        bool flag = false;
        if (u < n_nodes) {
            // Rows with a malformed extent or an out-of-range slot are skipped
            // (the counting kernels report such input through their status).
            const int32_t rs = row_ptr[u], re = row_ptr[u + 1];
            const bool row_ok = rs >= 0 && re >= rs && (int64_t)re <= nnz;
            if (DENSE) {
                flag = (int64_t)(re - rs) >= theta;
                has[u] = flag ? 1 : 0;
            } else {
                const int64_t s = slot[u];
                flag = s >= 0 && s < n_rows;
            }
            flag = flag && row_ok;
        }
        const unsigned bal = __ballot_sync(FULL, flag);
        if (lane == 0) warp_cnt[wid] = __popc(bal);
        __syncthreads();
        if (tid == 0) {
            int s = 0;
            for (int w = 0; w < kSketchThreads / 32; ++w) { int c = warp_cnt[w]; warp_cnt[w] = s; s += c; }
            total = s;
        }
        __syncthreads();
        if (flag) list[warp_cnt[wid] + __popc(bal & ((1u << lane) - 1u))] = (int)(u - base);
        __syncthreads();
        const int cnt = total;
        for (int t = 0; t < cnt; ++t) {
            const int64_t w = base + list[t];
            const int32_t rs = row_ptr[w], re = row_ptr[w + 1];
            uint8_t* row = DENSE ? rows + w * (int64_t)m : rows + slot[w] * (int64_t)m;
            uint4* row4 = reinterpret_cast<uint4*>(row);
            uint4* w4 = reinterpret_cast<uint4*>(words);
            if (DENSE) {
                for (int i = tid; i < (m >> 4); i += kSketchThreads) w4[i] = row4[i];
            } else {
                for (int i = tid; i < nwords; i += kSketchThreads) words[i] = 0u;
            }
            __syncthreads();
            for (int32_t k = rs + tid; k < re; k += kSketchThreads) {
                const int32_t c = col_idx[k];
                uint64_t x = (uint64_t)(int64_t)c;
                if (keys) {
                    if (c < 0 || (int64_t)c >= n_nodes) continue;  // malformed column: skipped
                    x = (uint64_t)keys[c];
                }
                uint32_t j, rho;
                hll_index_rank(x, p, j, rho);
                smem_byte_max(words, j, rho);
            }
            __syncthreads();
            for (int i = tid; i < (m >> 4); i += kSketchThreads) row4[i] = w4[i];
            __syncthreads();
        }
    }
}

__global__ void flag_kernel(const int32_t* __restrict__ row_ptr, int64_t n, int64_t theta, int64_t* out) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x)
        out[u] = ((int64_t)(row_ptr[u + 1] - row_ptr[u]) >= theta) ? 1 : 0;
}

__global__ void slot_fix_kernel(const int32_t* __restrict__ row_ptr, int64_t n, int64_t theta, const int64_t* scan,
                                int64_t* slot, int64_t* n_sketched) {
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const bool f = (int64_t)(row_ptr[u + 1] - row_ptr[u]) >= theta;
        slot[u] = f ? scan[u] : -1;
        if (u == n - 1) *n_sketched = scan[u] + (f ? 1 : 0);
    }
}

__global__ void zero_i64_kernel(int64_t* p) { *p = 0; }

__device__ __forceinline__ void global_byte_max(uint32_t* words, uint32_t j, uint32_t rho) {
    uint32_t* w = words + (j >> 2);
    const uint32_t sh = (j & 3u) * 8u;
    uint32_t old = *(volatile uint32_t*)w;
    while (((old >> sh) & 0xFFu) < rho) {
        const uint32_t nw = (old & ~(0xFFu << sh)) | (rho << sh);
        const uint32_t prev = atomicCAS(w, old, nw);
        if (prev == old) break;
        old = prev;
    }
}

__global__ void hll_add_kernel(uint32_t* regs, int p, const int64_t* __restrict__ values, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t j, rho;
        hll_index_rank((uint64_t)values[i], p, j, rho);
        global_byte_max(regs, j, rho);
    }
}

template <bool VEC>
__global__ void estimate_pairs_kernel(const uint8_t* rows, int64_t n_rows, int p, const int64_t* a, const int64_t* b,
                                      int64_t n_pairs, double* out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    const int64_t m = 1ll << p;
    for (int64_t i = warp; i < n_pairs; i += nwarps) {
        const int64_t sa = a[i];
        const int64_t sb = (b && b[i] >= 0) ? b[i] : sa;
        if (sa < 0 || sa >= n_rows || sb >= n_rows) {
            if (lane == 0) out[i] = __longlong_as_double(0x7FF8000000000000ll);  // NaN: bad row index
            continue;
        }
        const double E = warp_union_estimate<VEC>(rows + sa * m, rows + sb * m, p, lane, 0);
        if (lane == 0) out[i] = E;
    }
}

__global__ void hash_kernel(const int64_t* __restrict__ x, int64_t n, uint64_t* out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = splitmix64_fin((uint64_t)x[i]);
}

static int grid_for(int64_t n, int threads) {
    int64_t g = (n + threads - 1) / threads;
    const int64_t cap = (int64_t)sm_count() * 16;
    if (g > cap) g = cap;
    if (g < 1) g = 1;
    return (int)g;
}

template <bool DENSE>
static int launch_sketch(const int32_t* row_ptr, int64_t n, const int32_t* col_idx, const int64_t* keys,
                         int64_t nnz, int64_t theta, int p, uint8_t* has, const int64_t* slot, int64_t n_rows,
                         uint8_t* rows, cudaStream_t st) {
    if (n == 0) return TCHLL_OK;
    auto kern = sketch_kernel<DENSE>;
    const size_t smem = (size_t)1 << p;
    static size_t smem_set[kMaxDevices] = {};  // per device: the attribute is per device
    const int dev = current_device();
    if (dev < 0) return cuda_status(cudaErrorInvalidDevice, "cudaGetDevice");
    if (smem > smem_set[dev]) {
        TCHLL_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        smem_set[dev] = smem;
    }
    int bps = 1;
    TCHLL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, kern, kSketchThreads, smem));
    if (bps < 1) bps = 1;
    int64_t tiles = (n + kSketchThreads - 1) / kSketchThreads;
    int64_t g = (int64_t)sm_count() * bps;
    if (g > tiles) g = tiles;
    kern<<<(int)g, kSketchThreads, smem, st>>>(row_ptr, n, col_idx, keys, nnz, theta, p, has, slot, n_rows, rows);
    TCHLL_CHECK_LAUNCH("sketch_kernel");
    return TCHLL_OK;
}

}  // namespace tchll

using namespace tchll;

TCHLL_EXPORT int tchll_sketch_workspace_bytes(int64_t n_nodes, size_t* bytes) {
    TCHLL_ARG(bytes != nullptr && n_nodes >= 0, "bad arguments");
    size_t tmp = 0;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, (int64_t*)nullptr, (int64_t*)nullptr, (int)(n_nodes + 1)));
    Carve cv(nullptr, 0);
    cv.take<char>(tmp);
    cv.take<int64_t>((size_t)n_nodes + 1);
    *bytes = cv.off;
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_build_sketches_dense(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                            int64_t nnz, int64_t theta, int32_t p, uint8_t* sketch_regs,
                                            uint8_t* has_sketch, void* stream) {
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_nodes >= 0 && nnz >= 0, "negative size");
    TCHLL_ARG(n_nodes == 0 || (row_ptr && has_sketch && sketch_regs), "null pointer");
    TCHLL_ARG(((uintptr_t)sketch_regs & 15) == 0, "sketch_regs must be 16-byte aligned");
    return launch_sketch<true>(row_ptr, n_nodes, col_idx, nullptr, nnz, theta, p, has_sketch, nullptr, n_nodes,
                               sketch_regs, (cudaStream_t)stream);
}

TCHLL_EXPORT int tchll_sketch_slots(const int32_t* row_ptr, int64_t n_nodes, int64_t theta, int64_t* slot,
                                    int64_t* n_sketched, void* workspace, size_t workspace_bytes, void* stream) {
    TCHLL_ARG(n_nodes >= 0, "negative size");
    TCHLL_ARG(n_sketched != nullptr && (n_nodes == 0 || (row_ptr && slot)), "null pointer");
    cudaStream_t st = (cudaStream_t)stream;
    if (n_nodes == 0) {
        zero_i64_kernel<<<1, 1, 0, st>>>(n_sketched);
        TCHLL_CHECK_LAUNCH("zero_i64_kernel");
        return TCHLL_OK;
    }
    size_t need = 0;
    int rc = tchll_sketch_workspace_bytes(n_nodes, &need);
    if (rc) return rc;
    Carve cv(workspace, workspace_bytes);
    size_t tmp = 0;
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tmp, (int64_t*)nullptr, (int64_t*)nullptr, (int)(n_nodes + 1)));
    void* cub_tmp = cv.take<char>(tmp);
    int64_t* scan = cv.take<int64_t>((size_t)n_nodes + 1);
    if (!cv.ok() || workspace == nullptr) {
        set_error("workspace too small: need %zu bytes, have %zu", need, workspace_bytes);
        return TCHLL_EWORKSPACE;
    }
    const int g = grid_for(n_nodes, 256);
    flag_kernel<<<g, 256, 0, st>>>(row_ptr, n_nodes, theta, slot);
    TCHLL_CHECK_LAUNCH("flag_kernel");
    TCHLL_CUDA(cub::DeviceScan::ExclusiveSum(cub_tmp, tmp, slot, scan, (int)n_nodes, st));
    count_launch();
    slot_fix_kernel<<<g, 256, 0, st>>>(row_ptr, n_nodes, theta, scan, slot, n_sketched);
    TCHLL_CHECK_LAUNCH("slot_fix_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_build_sketches_compact(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                              const int64_t* keys, int64_t nnz, const int64_t* slot,
                                              int64_t n_rows, int32_t p, uint8_t* rows, void* stream) {
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_nodes >= 0 && nnz >= 0 && n_rows >= 0, "negative size");
    TCHLL_ARG(n_nodes == 0 || (row_ptr && slot), "null pointer");
    TCHLL_ARG(n_rows == 0 || rows, "rows is null");
    TCHLL_ARG(((uintptr_t)rows & 15) == 0, "rows must be 16-byte aligned");
    TCHLL_ARG(col_idx || nnz == 0, "col_idx is null");
    return launch_sketch<false>(row_ptr, n_nodes, col_idx, keys, nnz, 0, p, nullptr, slot, n_rows, rows,
                                (cudaStream_t)stream);
}

TCHLL_EXPORT int tchll_hll_add(uint8_t* regs, int32_t p, const int64_t* values, int64_t n, void* stream) {
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(regs && ((uintptr_t)regs & 3) == 0, "regs must be non-null and 4-byte aligned");
    TCHLL_ARG(n >= 0 && (n == 0 || values), "bad values");
    if (n == 0) return TCHLL_OK;
    hll_add_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>((uint32_t*)regs, p, values, n);
    TCHLL_CHECK_LAUNCH("hll_add_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_hll_estimate_pairs(const uint8_t* rows, int64_t n_rows, int32_t p, const int64_t* a,
                                          const int64_t* b, int64_t n_pairs, double* out, void* stream) {
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_pairs >= 0 && (n_pairs == 0 || (rows && a && out)), "bad arguments");
    if (n_pairs == 0) return TCHLL_OK;
    const int g = grid_for(n_pairs * 32, 256);
    if (((uintptr_t)rows & 15) == 0)
        estimate_pairs_kernel<true><<<g, 256, 0, (cudaStream_t)stream>>>(rows, n_rows, p, a, b, n_pairs, out);
    else
        estimate_pairs_kernel<false><<<g, 256, 0, (cudaStream_t)stream>>>(rows, n_rows, p, a, b, n_pairs, out);
    TCHLL_CHECK_LAUNCH("estimate_pairs_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_hash64(const int64_t* values, int64_t n, uint64_t* out, void* stream) {
    TCHLL_ARG(n >= 0 && (n == 0 || (values && out)), "bad arguments");
    if (n == 0) return TCHLL_OK;
    hash_kernel<<<grid_for(n, 256), 256, 0, (cudaStream_t)stream>>>(values, n, out);
    TCHLL_CHECK_LAUNCH("hash_kernel");
    return TCHLL_OK;
}

// cpu_exp register build (cpu_exp/triangle_hll_experiment.py:386-401,
// 526-540): dense rows for every vertex, seeded hash, low-p index; has_all[u]
// is set to 1 for every u (every vertex carries a sketch in that variant).
__global__ void cx_registers_kernel(const int32_t* __restrict__ row_ptr, int64_t n, const int32_t* __restrict__ col_idx,
                                    int64_t nnz, int p, uint64_t seed, uint8_t* regs, uint8_t* has_all) {
    const int lane = threadIdx.x & 31;
    const int64_t m = 1ll << p;
    for (int64_t u = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; u < n;
         u += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int32_t rs = row_ptr[u], re = row_ptr[u + 1];
        if (lane == 0) has_all[u] = 1;
        if (rs < 0 || re < rs || (int64_t)re > nnz) continue;
        uint32_t* row = reinterpret_cast<uint32_t*>(regs + u * m);
        for (int32_t k = rs + lane; k < re; k += 32) {
            uint32_t j, rho;
            hll_index_rank_cx((uint64_t)(int64_t)col_idx[k], seed, p, j, rho);
            global_byte_max(row, j, rho);
        }
    }
}

TCHLL_EXPORT int tchll_cx_build_registers(const int32_t* row_ptr, int64_t n_nodes, const int32_t* col_idx,
                                          int64_t nnz, int32_t p, uint64_t seed, uint8_t* regs, uint8_t* has_all,
                                          void* stream) {
    TCHLL_ARG(p >= 4 && p <= 16, "p must be in [4, 16], got %d", p);
    TCHLL_ARG(n_nodes >= 0 && (n_nodes == 0 || (row_ptr && regs && has_all)), "bad arguments");
    TCHLL_ARG(((uintptr_t)regs & 3) == 0, "regs must be 4-byte aligned");
    if (n_nodes == 0) return TCHLL_OK;
    cudaStream_t st = (cudaStream_t)stream;
    TCHLL_CUDA(cudaMemsetAsync(regs, 0, (size_t)n_nodes << p, st));
    cx_registers_kernel<<<grid_for(n_nodes * 32, 256), 256, 0, st>>>(row_ptr, n_nodes, col_idx, nnz, p, seed, regs,
                                                                     has_all);
    TCHLL_CHECK_LAUNCH("cx_registers_kernel");
    return TCHLL_OK;
}
