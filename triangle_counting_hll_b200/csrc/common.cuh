// common.cuh -- shared device helpers and C-ABI plumbing for libtchll.
//
// Everything here is compiled for sm_100a only.  Host entry points never
// allocate device memory: callers pass every buffer, including scratch
// ("workspace"), whose size they obtain from the matching *_workspace_bytes
// query.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/tchll.h"

#define TCHLL_EXPORT extern "C" __attribute__((visibility("default")))

namespace tchll {

constexpr unsigned FULL = 0xFFFFFFFFu;

// ---------------------------------------------------------------- errors ----
void set_error(const char* fmt, ...);
int cuda_status(cudaError_t e, const char* what);
void count_launch(int n = 1);

#define TCHLL_CHECK_LAUNCH(what)                                   \
    do {                                                           \
        cudaError_t _e = cudaGetLastError();                       \
        if (_e != cudaSuccess) return ::tchll::cuda_status(_e, what); \
        ::tchll::count_launch();                                   \
    } while (0)

#define TCHLL_CUDA(call)                                           \
    do {                                                           \
        cudaError_t _e = (call);                                   \
        if (_e != cudaSuccess) return ::tchll::cuda_status(_e, #call); \
    } while (0)

#define TCHLL_ARG(cond, ...)                                       \
    do {                                                           \
        if (!(cond)) { ::tchll::set_error(__VA_ARGS__); return TCHLL_EINVAL; } \
    } while (0)

int sm_count();

// Current device ordinal, or -1 if it cannot be read or is >= kMaxDevices
// (per-device host caches are indexed by it).
constexpr int kMaxDevices = 64;
inline int current_device() {
    int d = -1;
    if (cudaGetDevice(&d) != cudaSuccess || d < 0 || d >= kMaxDevices) return -1;
    return d;
}

// Workspace carving: bump allocator over a caller-provided buffer.
struct Carve {
    char* base;
    size_t cap;
    size_t off = 0;
    bool dry;  // size query only
    Carve(void* b, size_t c) : base((char*)b), cap(c), dry(b == nullptr) {}
    template <class T>
    T* take(size_t n) {
        off = (off + 255) & ~size_t(255);
        T* p = dry ? nullptr : (T*)(base + off);
        off += n * sizeof(T);
        return p;
    }
    bool ok() const { return dry || off <= cap; }
};

// ---------------------------------------------------------------- hashing ---
// splitmix64 finaliser: the reference's _hash64 (src/hll.py:13-19) and
// _splitmix64 (src/gpu_hll.py:12-17), bit for bit.
__host__ __device__ __forceinline__ uint64_t splitmix64_fin(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// HLL register update target for value x at precision p: index = top p bits
// of the hash, rank = (64-p) - bit_length(low bits) + 1, or (64-p)+1 when the
// low bits are zero (src/hll.py:81-91, src/gpu_hll.py:74-79).
__device__ __forceinline__ void hll_index_rank(uint64_t x, int p, uint32_t& j, uint32_t& rho) {
    const int rem = 64 - p;
    uint64_t h = splitmix64_fin(x);
    j = (uint32_t)(h >> rem);
    uint64_t w = h & ((1ull << rem) - 1ull);
    // bit_length(w) = 64 - clz(w); w == 0 gives clz 64 -> rho = rem + 1.
    rho = (uint32_t)(rem - (64 - __clzll(w)) + 1);
}

// The cpu_exp estimator variant (cpu_exp/triangle_hll_experiment.py:369-381,
// 386-401): h = splitmix64(x + seed) with the +0x9E3779B97F4A7C15 increment,
// index = low p bits, rank from h >> p (bit_length rule as above).
__device__ __forceinline__ void hll_index_rank_cx(uint64_t x, uint64_t seed, int p, uint32_t& j, uint32_t& rho) {
    const int bits = 64 - p;
    const uint64_t h = splitmix64_fin(x + seed + 0x9E3779B97F4A7C15ull);
    j = (uint32_t)(h & ((1ull << p) - 1ull));
    const uint64_t w = h >> p;
    rho = (uint32_t)(bits - (64 - __clzll(w)) + 1);
}

// Byte-wise max into a shared-memory register row stored as 32-bit words.
__device__ __forceinline__ void smem_byte_max(uint32_t* words, uint32_t j, uint32_t rho) {
    uint32_t* w = words + (j >> 2);
    const uint32_t sh = (j & 3u) * 8u;
    uint32_t old = *(volatile uint32_t*)w;
    while (((old >> sh) & 0xFFu) < rho) {
        uint32_t nw = (old & ~(0xFFu << sh)) | (rho << sh);
        uint32_t prev = atomicCAS(w, old, nw);
        if (prev == old) break;
        old = prev;
    }
}

// ------------------------------------------------------------ warp helpers --
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

__device__ __forceinline__ int64_t warp_sum_i64(int64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}

// 128-bit unsigned accumulation (lo, hi) with carry.
struct U128 {
    uint64_t lo = 0, hi = 0;
    __device__ __forceinline__ void add(uint64_t x) {
        uint64_t n = lo + x;
        hi += (n < lo);
        lo = n;
    }
    __device__ __forceinline__ void add(U128 o) {
        uint64_t n = lo + o.lo;
        hi += o.hi + (n < lo);
        lo = n;
    }
};

__device__ __forceinline__ U128 warp_sum_u128(U128 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        U128 t;
        t.lo = __shfl_xor_sync(FULL, v.lo, o);
        t.hi = __shfl_xor_sync(FULL, v.hi, o);
        v.add(t);
    }
    return v;
}

// Global 128-bit accumulate: every add sees its own carry out of the low
// word, so concurrent adds compose exactly and order-independently.
__device__ __forceinline__ void atomic_add_u128(unsigned long long* lo_hi, U128 v) {
    if (v.lo == 0 && v.hi == 0) return;
    unsigned long long old = atomicAdd(lo_hi, (unsigned long long)v.lo);
    uint64_t carry = ((uint64_t)old + v.lo) < (uint64_t)old ? 1 : 0;
    if (v.hi + carry) atomicAdd(lo_hi + 1, (unsigned long long)(v.hi + carry));
}

// u128 -> double (two roundings, within 1 ulp).
__host__ __device__ __forceinline__ double u128_to_double(uint64_t lo, uint64_t hi) {
    return (double)hi * 18446744073709551616.0 + (double)lo;
}

}  // namespace tchll
