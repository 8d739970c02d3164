// hll_device.cuh -- device-side HyperLogLog union estimation shared by the
// counting kernels and the standalone estimate entry point.
#pragma once

#include "common.cuh"

namespace tchll {

// Exact sum 2^-r over the register-wise max of two rows, as an integer in
// units of 2^-S (S = 65 - p: every valid rank r in [1, 65-p] gives the
// integer 2^(S-r)); zero registers are counted separately (each is 2^S units);
// ranks above S (impossible for rows built from this hash) go to a double.
struct HllPartial {
    uint64_t sum = 0;
    uint32_t zeros = 0;
    double extra = 0.0;
};

__device__ __forceinline__ void hll_word(uint32_t w, int S, HllPartial& hp) {
    hp.zeros += __popc(__vcmpeq4(w, 0u)) >> 3;
    if (w == 0u) return;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t r = (w >> (8 * k)) & 0xFFu;
        if (r != 0u) {
            if ((int)r <= S) hp.sum += 1ull << (S - (int)r);
            else hp.extra += ldexp(1.0, S - (int)r);
        }
    }
}

// Union estimate for two register rows; every lane returns the same value.
template <bool VEC>
// variant 0: src/hll.py:37-54 (linear counting, then the 2^64 correction on
// the result); variant 1: cpu_exp's estimate_hll_cardinality
// (cpu_exp/triangle_hll_experiment.py:357-366: linear counting, else the
// 2^32 correction on the raw estimate).
__device__ __forceinline__ double warp_union_estimate(const uint8_t* ra, const uint8_t* rb, int p, int lane,
                                                      int variant = 0, uint32_t* zeros_out = nullptr) {
    const int m = 1 << p;
    const int S = 65 - p;
    HllPartial hp;
    // Per-lane sums stay below 2^64: a lane holds at most max(16, m/32) bytes
    // of rank >= 1, each worth at most 2^(64-p) units; p == 4 with 16 bytes on
    // one lane could reach 2^64, so p == 4 takes the byte path.
    if (VEC && p > 4) {
        const uint4* a4 = reinterpret_cast<const uint4*>(ra);
        const uint4* b4 = reinterpret_cast<const uint4*>(rb);
        for (int i = lane; i < (m >> 4); i += 32) {
            uint4 a = __ldg(a4 + i), b = __ldg(b4 + i);
            hll_word(__vmaxu4(a.x, b.x), S, hp);
            hll_word(__vmaxu4(a.y, b.y), S, hp);
            hll_word(__vmaxu4(a.z, b.z), S, hp);
            hll_word(__vmaxu4(a.w, b.w), S, hp);
        }
    } else {
        for (int i = lane; i < m; i += 32) {
            const uint32_t x = __ldg(ra + i), y = __ldg(rb + i);
            const uint32_t r = x > y ? x : y;
            if (r == 0u) ++hp.zeros;
            else if ((int)r <= S) hp.sum += 1ull << (S - (int)r);
            else hp.extra += ldexp(1.0, S - (int)r);
        }
    }
    U128 s;
    s.lo = hp.sum;
    s = warp_sum_u128(s);
    uint32_t zeros = hp.zeros;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) zeros += __shfl_xor_sync(FULL, zeros, o);
    double extra = hp.extra;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) extra += __shfl_xor_sync(FULL, extra, o);
    // zeros * 2^S added into the 128-bit sum
    U128 z;
    z.lo = (uint64_t)zeros << S;
    z.hi = (uint64_t)zeros >> (64 - S);
    s.add(z);
    const double Z = ldexp(u128_to_double(s.lo, s.hi) + extra, -S);
    // src/hll.py:26-34 (alpha) and :37-54 (corrections)
    double alpha;
    if (m == 16) alpha = 0.673;
    else if (m == 32) alpha = 0.697;
    else if (m == 64) alpha = 0.709;
    else alpha = 0.7213 / (1.0 + 1.079 / (double)m);
    double E = alpha * (double)m * (double)m / Z;
    if (zeros_out) *zeros_out = zeros;
    if (variant == 1) {
        if (E <= 2.5 * (double)m && zeros > 0) return (double)m * log((double)m / (double)zeros);
        const double two32 = 4294967296.0;
        if (E > two32 / 30.0) return -two32 * log(1.0 - E / two32);
        return E;
    }
    if (E <= 2.5 * (double)m) {
        if (zeros > 0) E = (double)m * log((double)m / (double)zeros);
    }
    const double two64 = 18446744073709551616.0;
    if (E > two64 / 30.0) E = -two64 * log(1.0 - E / two64);
    return E;
}

}  // namespace tchll
