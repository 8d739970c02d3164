// gen.cu -- seeded synthetic edge-list generators (device).
//
// The reference reads SNAP edge lists (experiment/exp_gpu.py:131-144); the
// workloads here are synthetic stand-ins with the published shapes: R-MAT,
// Erdos-Renyi, a perturbed road-like lattice and Chung-Lu power-law graphs.
// Every random draw is a counter-based splitmix64 value, so a graph depends
// only on its parameters and seed:
//   key(seed, stream) = mix((seed + 1) * G ^ stream * C)
//   draw(key, i)      = mix(key + (i + 1) * G)
// mix = splitmix64 finaliser, G = 0x9E3779B97F4A7C15, C = 0xC2B2AE3D27D4EB4F.
// Streams: 1 R-MAT, 2 Erdos-Renyi, 3 lattice diagonals, 4 lattice deletions,
// 5 id permutation, 6 Chung-Lu.
#include "common.cuh"

namespace tchll {

constexpr uint64_t kG = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kC = 0xC2B2AE3D27D4EB4Full;

__host__ __device__ __forceinline__ uint64_t gen_key(uint64_t seed, uint64_t stream) {
    return splitmix64_fin((seed + 1ull) * kG ^ (stream * kC));
}
__host__ __device__ __forceinline__ uint64_t gen_draw(uint64_t key, uint64_t i) {
    return splitmix64_fin(key + (i + 1ull) * kG);
}

#define GRID_STRIDE(i, n) \
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < (n); i += (int64_t)gridDim.x * blockDim.x)

// R-MAT: `scale` quadrant choices per edge, two 32-bit draws per 64-bit value
// (high half for even levels, low half for odd), thresholds ta <= tab <= tabc.
__global__ void rmat_kernel(int scale, int64_t n_raw, uint32_t ta, uint32_t tab, uint32_t tabc, uint64_t key,
                            int32_t* out_u, int32_t* out_v) {
    const int64_t per = (scale + 1) / 2;
    GRID_STRIDE(i, n_raw) {
        uint32_t u = 0, v = 0;
        uint64_t x = 0;
        for (int l = 0; l < scale; ++l) {
            uint32_t r;
            if ((l & 1) == 0) {
                x = gen_draw(key, (uint64_t)i * per + (l >> 1));
                r = (uint32_t)(x >> 32);
            } else {
                r = (uint32_t)x;
            }
            const uint32_t bu = r >= tab;                   // quadrants c, d
            const uint32_t bv = (r >= ta && r < tab) || r >= tabc;  // quadrants b, d
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        out_u[i] = (int32_t)u;
        out_v[i] = (int32_t)v;
    }
}

__global__ void er_kernel(int64_t n, int64_t n_raw, uint64_t key, int32_t* out_u, int32_t* out_v) {
    GRID_STRIDE(i, n_raw) {
        out_u[i] = (int32_t)(((gen_draw(key, 2 * (uint64_t)i) >> 32) * (uint64_t)n) >> 32);
        out_v[i] = (int32_t)(((gen_draw(key, 2 * (uint64_t)i + 1) >> 32) * (uint64_t)n) >> 32);
    }
}

// Bijection of [0, n): 4-round balanced Feistel network over 2h bits, round
// keys draw(key(seed,5), r), cycle-walking until the value is below n.
struct Perm {
    uint64_t n;
    int h;
    uint64_t rk[4];
};

__host__ __device__ __forceinline__ uint64_t perm_apply(uint64_t x, const Perm& P) {
    const uint64_t mask = (1ull << P.h) - 1ull;
    do {
        uint64_t L = x >> P.h, R = x & mask;
        for (int r = 0; r < 4; ++r) {
            const uint64_t F = splitmix64_fin(R ^ P.rk[r]) & mask;
            const uint64_t nl = R;
            R = L ^ F;
            L = nl;
        }
        x = (L << P.h) | R;
    } while (x >= P.n);
    return x;
}

static Perm make_perm(uint64_t n, uint64_t seed) {
    Perm P;
    P.n = n;
    int b = 1;
    const uint64_t mx = n > 1 ? n - 1 : 1;
    while (b < 64 && (mx >> b) != 0) ++b;
    P.h = (b + 1) / 2;
    const uint64_t k = gen_key(seed, 5);
    for (int r = 0; r < 4; ++r) P.rk[r] = gen_draw(k, (uint64_t)r);
    return P;
}

// Candidates: right edges, down edges, then one diagonal per cell; absent or
// deleted candidates are emitted as (0, 0) self-loops, which ingest drops.
__global__ void lattice_kernel(int64_t R, int64_t C, uint32_t tdiag, uint32_t tdel, uint64_t kd, uint64_t kx,
                               Perm P, int32_t* out_u, int32_t* out_v) {
    const int64_t n_right = R * (C - 1), n_down = (R - 1) * C, n_diag = (R - 1) * (C - 1);
    const int64_t total = n_right + n_down + n_diag;
    GRID_STRIDE(k, total) {
        int64_t a, b;
        bool present = true;
        if (k < n_right) {
            const int64_t i = k / (C - 1), j = k % (C - 1);
            a = i * C + j;
            b = a + 1;
        } else if (k < n_right + n_down) {
            const int64_t q = k - n_right, i = q / C, j = q % C;
            a = i * C + j;
            b = a + C;
        } else {
            const int64_t q = k - n_right - n_down, i = q / (C - 1), j = q % (C - 1);
            a = i * C + j;
            b = a + C + 1;
            present = (uint32_t)(gen_draw(kd, (uint64_t)q) >> 32) < tdiag;
        }
        if (present && (uint32_t)(gen_draw(kx, (uint64_t)k) >> 32) < tdel) present = false;
        if (present) {
            out_u[k] = (int32_t)perm_apply((uint64_t)a, P);
            out_v[k] = (int32_t)perm_apply((uint64_t)b, P);
        } else {
            out_u[k] = 0;
            out_v[k] = 0;
        }
    }
}

// Chung-Lu: endpoint j (u_i = 2i, v_i = 2i+1) is the first index whose
// cumulative integer weight exceeds draw(key, j) mod total.
__global__ void chung_lu_kernel(const uint64_t* __restrict__ cum, int64_t n, int64_t n_raw, uint64_t key,
                                int32_t* out_u, int32_t* out_v) {
    const uint64_t total = cum[n - 1];
    GRID_STRIDE(j, 2 * n_raw) {
        const uint64_t t = gen_draw(key, (uint64_t)j) % total;
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            const int64_t mid = (lo + hi) >> 1;
            if (cum[mid] > t) hi = mid; else lo = mid + 1;
        }
        if (j & 1) out_v[j >> 1] = (int32_t)lo; else out_u[j >> 1] = (int32_t)lo;
    }
}

static int gen_grid(int64_t n) {
    int64_t g = (n + 255) / 256;
    const int64_t cap = (int64_t)sm_count() * 32;
    if (g > cap) g = cap;
    return g < 1 ? 1 : (int)g;
}

}  // namespace tchll

using namespace tchll;

TCHLL_EXPORT int tchll_gen_rmat(int32_t scale, int64_t n_raw, uint32_t ta, uint32_t tab, uint32_t tabc,
                                uint64_t seed, int32_t* u, int32_t* v, void* stream) {
    TCHLL_ARG(scale >= 1 && scale <= 31, "scale must be in [1, 31]");
    TCHLL_ARG(ta <= tab && tab <= tabc, "thresholds must be non-decreasing");
    TCHLL_ARG(n_raw >= 0 && (n_raw == 0 || (u && v)), "bad outputs");
    if (n_raw == 0) return TCHLL_OK;
    rmat_kernel<<<gen_grid(n_raw), 256, 0, (cudaStream_t)stream>>>(scale, n_raw, ta, tab, tabc, gen_key(seed, 1), u,
                                                                   v);
    TCHLL_CHECK_LAUNCH("rmat_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_gen_er(int64_t n, int64_t n_raw, uint64_t seed, int32_t* u, int32_t* v, void* stream) {
    TCHLL_ARG(n >= 1 && n <= (int64_t)INT32_MAX, "n must be in [1, 2^31)");
    TCHLL_ARG(n_raw >= 0 && (n_raw == 0 || (u && v)), "bad outputs");
    if (n_raw == 0) return TCHLL_OK;
    er_kernel<<<gen_grid(n_raw), 256, 0, (cudaStream_t)stream>>>(n, n_raw, gen_key(seed, 2), u, v);
    TCHLL_CHECK_LAUNCH("er_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int64_t tchll_gen_lattice_count(int64_t rows, int64_t cols) {
    if (rows < 1 || cols < 1) return 0;
    return rows * (cols - 1) + (rows - 1) * cols + (rows - 1) * (cols - 1);
}

TCHLL_EXPORT int tchll_gen_lattice(int64_t rows, int64_t cols, uint32_t tdiag, uint32_t tdel, uint64_t seed,
                                   int32_t* u, int32_t* v, void* stream) {
    TCHLL_ARG(rows >= 1 && cols >= 1 && rows * cols <= (int64_t)INT32_MAX, "bad lattice size");
    const int64_t total = tchll_gen_lattice_count(rows, cols);
    TCHLL_ARG(total == 0 || (u && v), "bad outputs");
    if (total == 0) return TCHLL_OK;
    Perm P = make_perm((uint64_t)(rows * cols), seed);
    lattice_kernel<<<gen_grid(total), 256, 0, (cudaStream_t)stream>>>(rows, cols, tdiag, tdel, gen_key(seed, 3),
                                                                      gen_key(seed, 4), P, u, v);
    TCHLL_CHECK_LAUNCH("lattice_kernel");
    return TCHLL_OK;
}

TCHLL_EXPORT int tchll_gen_chung_lu(const uint64_t* cum, int64_t n, int64_t n_raw, uint64_t seed, int32_t* u,
                                    int32_t* v, void* stream) {
    TCHLL_ARG(n >= 1 && n <= (int64_t)INT32_MAX && cum, "bad weight table");
    TCHLL_ARG(n_raw >= 0 && (n_raw == 0 || (u && v)), "bad outputs");
    if (n_raw == 0) return TCHLL_OK;
    chung_lu_kernel<<<gen_grid(2 * n_raw), 256, 0, (cudaStream_t)stream>>>(cum, n, n_raw, gen_key(seed, 6), u, v);
    TCHLL_CHECK_LAUNCH("chung_lu_kernel");
    return TCHLL_OK;
}
