/*
 * tchll_oracle.c -- CPU oracle for the hybrid exact / HyperLogLog triangle count.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker, never the product:
 * only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may load
 * the library built from it.  The product (triangle_counting_hll_b200) never
 * links, imports or calls it.
 *
 * It restates, in plain C, the reference implementation
 * (ChitandaEruQ/triangle_counting_hll, pure Python + Numba) for the hot path:
 *
 *   orc_hash64            src/hll.py:13-19          (splitmix64 finaliser)
 *   orc_alpha             src/hll.py:26-34
 *   orc_estimate          src/hll.py:37-54          (np.sum pairwise order kept)
 *   orc_hll_add           src/hll.py:81-96
 *   orc_union_estimate    src/hll.py:112-120
 *   orc_build_sketches_dense   src/gpu_hll.py:47-81  (max into existing rows)
 *   orc_build_sketches_compact src/hybrid.py:15-41   (rows for d+ >= theta)
 *   orc_intersect_*       src/exact.py:12-41
 *   orc_exact_count       src/exact.py:48-98, src/gpu_hybrid.py:96-130
 *   orc_hybrid_count      src/hybrid.py:95-164, src/gpu_hybrid.py:80-89,266-325
 *   orc_csr_build         experiment/exp_gpu.py:317-365 (array form of
 *                         src/graph.py:29-61 + src/gpu_graph.py:6-41)
 *   orc_cx_*              cpu_exp/triangle_hll_experiment.py:357-381,615-710
 *                         (the cpu_exp HLL variant: seeded hash, low-p index)
 *
 * Parity is pinned against the reference itself: tests/golden/make_golden.py
 * imports the reference's src/ modules and records registers, estimates and
 * counts; tests/test_oracle_golden.py checks this file against those fixtures.
 *
 * It also restates the seeded synthetic graph generators (R-MAT, Erdos-Renyi,
 * perturbed lattice, Chung-Lu) from their written specification, independently
 * of the product's device generators, so the two can be compared.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_API __attribute__((visibility("default")))

/* ------------------------------------------------------------------------- */
/* Hash and HLL helpers                                                       */
/* ------------------------------------------------------------------------- */

/* src/hll.py:13-19: splitmix64 finaliser on the masked 64-bit value. */
ORC_API uint64_t orc_hash64(uint64_t x) {
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

ORC_API void orc_hash64_array(const int64_t* x, int64_t n, uint64_t* out) {
    for (int64_t i = 0; i < n; ++i) out[i] = orc_hash64((uint64_t)x[i]);
}

/* src/hll.py:26-34 */
ORC_API double orc_alpha(int64_t m) {
    if (m == 16) return 0.673;
    if (m == 32) return 0.697;
    if (m == 64) return 0.709;
    return 0.7213 / (1.0 + 1.079 / (double)m);
}

/* numpy's pairwise summation (the order np.sum uses on a contiguous float64
 * array): blocks of at most 128 summed with 8 interleaved partials, larger
 * ranges split in two at a multiple of 8. */
static double pairwise_sum(const double* a, int64_t n) {
    if (n < 8) {
        double res = 0.0;
        for (int64_t i = 0; i < n; ++i) res += a[i];
        return res;
    } else if (n <= 128) {
        double r[8];
        int64_t i;
        for (int k = 0; k < 8; ++k) r[k] = a[k];
        for (i = 8; i < n - (n % 8); i += 8)
            for (int k = 0; k < 8; ++k) r[k] += a[i + k];
        double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; ++i) res += a[i];
        return res;
    } else {
        int64_t n2 = n / 2;
        n2 -= n2 % 8;
        return pairwise_sum(a, n2) + pairwise_sum(a + n2, n - n2);
    }
}

ORC_API double orc_pairwise_sum(const double* a, int64_t n) { return pairwise_sum(a, n); }

/* src/hll.py:37-54.  Z = np.sum(2.0 ** -registers) (pairwise order),
 * E = alpha*m*m/Z, linear counting when E <= 2.5m and zeros exist,
 * the 2^64 large-range correction when E > 2^64/30. */
static double estimate_regs(const uint8_t* regs, int64_t m, double alpha, double* tmp) {
    int64_t zeros = 0;
    for (int64_t j = 0; j < m; ++j) {
        tmp[j] = ldexp(1.0, -(int)regs[j]);
        zeros += (regs[j] == 0);
    }
    double Z = 0.0 + pairwise_sum(tmp, m);
    double E = alpha * (double)m * (double)m / Z;
    if (E <= 2.5 * (double)m) {
        if (zeros > 0) E = (double)m * log((double)m / (double)zeros);
    }
    const double two64 = 18446744073709551616.0;
    if (E > two64 / 30.0) E = -two64 * log(1.0 - E / two64);
    return E;
}

ORC_API double orc_estimate(const uint8_t* regs, int64_t m, double alpha) {
    double* tmp = (double*)malloc(sizeof(double) * (size_t)m);
    double e = estimate_regs(regs, m, alpha, tmp);
    free(tmp);
    return e;
}

/* src/hll.py:81-91: index = top p bits, rank = leading zeros of the low
 * (64-p) bits + 1, or (64-p)+1 when those bits are all zero. */
static inline void hll_update(uint8_t* regs, int p, uint64_t x) {
    const int rem = 64 - p;
    uint64_t h = orc_hash64(x);
    uint64_t j = h >> rem;
    uint64_t w = h & ((1ull << rem) - 1ull);
    int rho;
    if (w == 0) {
        rho = rem + 1;
    } else {
        int bl = 64 - __builtin_clzll(w);
        rho = rem - bl + 1;
    }
    if (rho > regs[j]) regs[j] = (uint8_t)rho;
}

ORC_API void orc_hll_add(uint8_t* regs, int p, const int64_t* x, int64_t n) {
    for (int64_t i = 0; i < n; ++i) hll_update(regs, p, (uint64_t)x[i]);
}

/* src/hll.py:112-120 (p equality is the caller's check). */
ORC_API double orc_union_estimate(const uint8_t* a, const uint8_t* b, int p) {
    int64_t m = 1ll << p;
    uint8_t* merged = (uint8_t*)malloc((size_t)m);
    double* tmp = (double*)malloc(sizeof(double) * (size_t)m);
    for (int64_t j = 0; j < m; ++j) merged[j] = a[j] > b[j] ? a[j] : b[j];
    double e = estimate_regs(merged, m, orc_alpha(m), tmp);
    free(tmp);
    free(merged);
    return e;
}

/* src/gpu_hll.py:47-81: dense rows regs[u*m ..], has[u] written for every u,
 * registers max-merged into whatever the rows already hold. */
ORC_API void orc_build_sketches_dense(const int32_t* row_ptr, const int32_t* col_idx,
                                      int64_t n_nodes, int64_t theta, int p,
                                      uint8_t* regs, uint8_t* has) {
    const int64_t m = 1ll << p;
    for (int64_t u = 0; u < n_nodes; ++u) {
        int64_t deg = (int64_t)row_ptr[u + 1] - row_ptr[u];
        if (deg < theta) { has[u] = 0; continue; }
        has[u] = 1;
        uint8_t* row = regs + u * m;
        for (int64_t k = row_ptr[u]; k < row_ptr[u + 1]; ++k)
            hll_update(row, p, (uint64_t)(int64_t)col_idx[k]);
    }
}

/* src/hybrid.py:15-41 in compact form: slot[u] = rank of u among vertices with
 * d+(u) >= theta (or -1); rows[slot*m ..] holds the sketch of N+(u), hashing the
 * values of `keys` (the ids forward_adj holds; the compacted ids on the GPU
 * path).  Pass rows == NULL to only count. Returns the number of sketches. */
ORC_API int64_t orc_build_sketches_compact(const int64_t* row_ptr, const int64_t* keys,
                                           int64_t n_nodes, int64_t theta, int p,
                                           int64_t* slot, uint8_t* rows) {
    const int64_t m = 1ll << p;
    int64_t ns = 0;
    for (int64_t u = 0; u < n_nodes; ++u) {
        int64_t deg = row_ptr[u + 1] - row_ptr[u];
        if (deg < theta) { if (slot) slot[u] = -1; continue; }
        if (slot) slot[u] = ns;
        if (rows) {
            uint8_t* row = rows + ns * m;
            memset(row, 0, (size_t)m);
            for (int64_t k = row_ptr[u]; k < row_ptr[u + 1]; ++k)
                hll_update(row, p, (uint64_t)keys[k]);
        }
        ++ns;
    }
    return ns;
}

/* ------------------------------------------------------------------------- */
/* Exact intersection (src/exact.py:12-41)                                    */
/* ------------------------------------------------------------------------- */

static int64_t intersect_merge(const int32_t* a, int64_t la, const int32_t* b, int64_t lb) {
    int64_t i = 0, j = 0, c = 0;
    while (i < la && j < lb) {
        if (a[i] == b[j]) { ++c; ++i; ++j; }
        else if (a[i] < b[j]) ++i;
        else ++j;
    }
    return c;
}

/* np.searchsorted(large, small) (left) then compare, src/exact.py:17-26 */
static int64_t intersect_bsearch(const int32_t* s, int64_t ls, const int32_t* l, int64_t ll) {
    int64_t c = 0;
    for (int64_t i = 0; i < ls; ++i) {
        int64_t lo = 0, hi = ll;
        int32_t x = s[i];
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (l[mid] < x) lo = mid + 1; else hi = mid;
        }
        if (lo < ll && l[lo] == x) ++c;
    }
    return c;
}

static int64_t intersect_adaptive(const int32_t* a, int64_t la, const int32_t* b, int64_t lb, double r) {
    if (la == 0 || lb == 0) return 0;
    if (la > lb) { const int32_t* t = a; a = b; b = t; int64_t tl = la; la = lb; lb = tl; }
    if ((double)lb / (double)la <= r) return intersect_merge(a, la, b, lb);
    return intersect_bsearch(a, la, b, lb);
}

ORC_API int64_t orc_intersect(const int32_t* a, int64_t la, const int32_t* b, int64_t lb, double r) {
    return intersect_adaptive(a, la, b, lb, r);
}

static inline void set_threads(int nthreads) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
}

ORC_API int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_num_procs();
#else
    return 1;
#endif
}

/* T = sum over the given oriented edges of |N+(u) cap N+(v)|.  The lists come
 * from the CSR (row_ptr/col_idx); edges are (edge_u[i], edge_v[i]).
 * per_edge (nullable) receives each edge's support. */
ORC_API uint64_t orc_exact_count(const int32_t* row_ptr, const int32_t* col_idx,
                                 const int32_t* eu, const int32_t* ev, int64_t n_edges,
                                 double r, int nthreads, int64_t* per_edge) {
    uint64_t total = 0;
    set_threads(nthreads);
#pragma omp parallel for reduction(+ : total) schedule(dynamic, 2048)
    for (int64_t i = 0; i < n_edges; ++i) {
        int32_t u = eu[i], v = ev[i];
        int64_t s = intersect_adaptive(col_idx + row_ptr[u], (int64_t)row_ptr[u + 1] - row_ptr[u],
                                       col_idx + row_ptr[v], (int64_t)row_ptr[v + 1] - row_ptr[v], r);
        if (per_edge) per_edge[i] = s;
        total += (uint64_t)s;
    }
    return total;
}

/* ------------------------------------------------------------------------- */
/* Hybrid (src/hybrid.py:95-164; GPU routing src/gpu_hybrid.py:80-89)          */
/* ------------------------------------------------------------------------- */

/* degrees: forward degree used for routing and for s_hat (the GPU path passes
 * its degrees array; the CPU path uses len(N+)).  slot[v] >= 0 iff v has a
 * sketch, rows[slot*m ..] its registers.  Sum order: edge order, one thread;
 * with several threads, contiguous chunks summed in chunk order.
 * stats[0..3] = n_approx, n_exact, n_fallback, n_clamped.
 * s_hat/s_clamped/method (nullable) receive per-edge details. */
ORC_API double orc_hybrid_count(const int32_t* row_ptr, const int32_t* col_idx,
                                const int32_t* eu, const int32_t* ev, int64_t n_edges,
                                const int32_t* degrees, const int64_t* slot,
                                const uint8_t* rows, int p, int64_t gamma, double r,
                                int nthreads, int64_t* stats, double* s_hat_out,
                                double* s_clamped_out, uint8_t* method_out) {
    const int64_t m = 1ll << p;
    const double alpha = orc_alpha(m);
    set_threads(nthreads);
    int nt = 1;
#ifdef _OPENMP
    nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    double* part = (double*)calloc((size_t)nt, sizeof(double));
    int64_t* pst = (int64_t*)calloc((size_t)nt * 4, sizeof(int64_t));
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        int64_t lo = n_edges * t / nt, hi = n_edges * (t + 1) / nt;
        uint8_t* merged = (uint8_t*)malloc((size_t)m);
        double* tmp = (double*)malloc(sizeof(double) * (size_t)m);
        double total = 0.0;
        int64_t n_approx = 0, n_exact = 0, n_fallback = 0, n_clamped = 0;
        for (int64_t i = lo; i < hi; ++i) {
            int32_t u = eu[i], v = ev[i];
            int64_t du = degrees[u], dv = degrees[v];
            int64_t proxy = du < dv ? du : dv;
            int wants = proxy >= gamma;
            int both = slot[u] >= 0 && slot[v] >= 0;
            if (wants && !both) ++n_fallback;
            if (wants && both) {
                ++n_approx;
                const uint8_t* a = rows + slot[u] * m;
                const uint8_t* b = rows + slot[v] * m;
                for (int64_t j = 0; j < m; ++j) merged[j] = a[j] > b[j] ? a[j] : b[j];
                double E = estimate_regs(merged, m, alpha, tmp);
                double s_hat = (double)(du + dv) - E;
                double upper = (double)proxy;
                /* max(0.0, min(s_hat, upper)) with Python's argument order */
                double s_cl = (upper < s_hat) ? upper : s_hat;
                s_cl = (s_cl > 0.0) ? s_cl : 0.0;
                if (s_hat < 0.0 || s_hat > upper) ++n_clamped;
                total += s_cl;
                if (s_hat_out) s_hat_out[i] = s_hat;
                if (s_clamped_out) s_clamped_out[i] = s_cl;
                if (method_out) method_out[i] = 1;
            } else {
                ++n_exact;
                int64_t s = intersect_adaptive(col_idx + row_ptr[u], (int64_t)row_ptr[u + 1] - row_ptr[u],
                                               col_idx + row_ptr[v], (int64_t)row_ptr[v + 1] - row_ptr[v], r);
                total += (double)s;
                if (s_hat_out) s_hat_out[i] = (double)s;
                if (s_clamped_out) s_clamped_out[i] = (double)s;
                if (method_out) method_out[i] = 0;
            }
        }
        part[t] = total;
        pst[4 * t + 0] = n_approx; pst[4 * t + 1] = n_exact;
        pst[4 * t + 2] = n_fallback; pst[4 * t + 3] = n_clamped;
        free(tmp);
        free(merged);
    }
    double total = 0.0;
    for (int k = 0; k < 4; ++k) stats[k] = 0;
    for (int t = 0; t < nt; ++t) {
        total += part[t];
        for (int k = 0; k < 4; ++k) stats[k] += pst[4 * t + k];
    }
    free(part);
    free(pst);
    return total;
}

/* ------------------------------------------------------------------------- */
/* Edge list -> oriented CSR (experiment/exp_gpu.py:317-365)                  */
/* ------------------------------------------------------------------------- */

static void radix_sort_u64(uint64_t* a, uint64_t* tmp, int64_t n, int bits) {
    /* LSD radix sort on the low `bits` bits, 16-bit digits. */
    int64_t* cnt = (int64_t*)malloc(sizeof(int64_t) * 65536);
    uint64_t* src = a;
    uint64_t* dst = tmp;
    int passes = (bits + 15) / 16;
    for (int ps = 0; ps < passes; ++ps) {
        int sh = 16 * ps;
        memset(cnt, 0, sizeof(int64_t) * 65536);
        for (int64_t i = 0; i < n; ++i) cnt[(src[i] >> sh) & 0xFFFF]++;
        int64_t s = 0;
        for (int d = 0; d < 65536; ++d) { int64_t c = cnt[d]; cnt[d] = s; s += c; }
        for (int64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> sh) & 0xFFFF]++] = src[i];
        uint64_t* t = src; src = dst; dst = t;
    }
    if (src != a) memcpy(a, src, sizeof(uint64_t) * (size_t)n);
    free(cnt);
}

static int bits_for(uint64_t maxv) {
    int b = 1;
    while (b < 64 && (maxv >> b) != 0) ++b;
    return b;
}

/* Canonical (min,max) pairs, self-loops dropped, duplicates dropped
 * (np.unique), node ids = sorted union of endpoints (np.union1d), undirected
 * degree, orientation u->v iff (deg u, id u) < (deg v, id v), forward CSR with
 * rows sorted by (src, dst) (np.lexsort).  Output capacities: row_ptr and
 * fdeg/node_ids 2*n_raw+1, col_idx/edge_u/edge_v n_raw.  Returns 0, or -1 when
 * an id is negative. */
ORC_API int orc_csr_build(const int32_t* ru, const int32_t* rv, int64_t n_raw,
                          int64_t* out_n_nodes, int64_t* out_n_edges,
                          int32_t* row_ptr, int32_t* col_idx, int32_t* fdeg,
                          int64_t* node_ids, int32_t* edge_u, int32_t* edge_v) {
    uint64_t* keys = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(n_raw > 0 ? n_raw : 1));
    uint64_t* tmp = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(2 * n_raw + 1));
    int64_t k = 0;
    uint32_t maxid = 0;
    for (int64_t i = 0; i < n_raw; ++i) {
        int32_t u = ru[i], v = rv[i];
        if (u < 0 || v < 0) { free(keys); free(tmp); return -1; }
        if (u == v) continue;
        uint32_t a = (uint32_t)(u < v ? u : v), b = (uint32_t)(u < v ? v : u);
        if (b > maxid) maxid = b;
        keys[k++] = ((uint64_t)a << 32) | b;
    }
    radix_sort_u64(keys, tmp, k, 64);
    int64_t e = 0;
    for (int64_t i = 0; i < k; ++i)
        if (i == 0 || keys[i] != keys[i - 1]) keys[e++] = keys[i];
    /* node ids: sorted unique endpoints */
    uint64_t* ends = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)(2 * e + 1));
    for (int64_t i = 0; i < e; ++i) { ends[2 * i] = keys[i] >> 32; ends[2 * i + 1] = keys[i] & 0xFFFFFFFFull; }
    radix_sort_u64(ends, tmp, 2 * e, bits_for(maxid));
    int64_t n = 0;
    for (int64_t i = 0; i < 2 * e; ++i)
        if (i == 0 || ends[i] != ends[i - 1]) ends[n++] = ends[i];
    for (int64_t i = 0; i < n; ++i) node_ids[i] = (int64_t)ends[i];
    /* remap + undirected degree */
    int32_t* deg = (int32_t*)calloc((size_t)(n > 0 ? n : 1), sizeof(int32_t));
    int32_t* ca = (int32_t*)malloc(sizeof(int32_t) * (size_t)(e > 0 ? e : 1));
    int32_t* cb = (int32_t*)malloc(sizeof(int32_t) * (size_t)(e > 0 ? e : 1));
    for (int64_t i = 0; i < e; ++i) {
        uint64_t a = keys[i] >> 32, b = keys[i] & 0xFFFFFFFFull;
        int64_t lo = 0, hi = n;
        while (lo < hi) { int64_t mid = (lo + hi) >> 1; if (ends[mid] < a) lo = mid + 1; else hi = mid; }
        ca[i] = (int32_t)lo;
        lo = 0; hi = n;
        while (lo < hi) { int64_t mid = (lo + hi) >> 1; if (ends[mid] < b) lo = mid + 1; else hi = mid; }
        cb[i] = (int32_t)lo;
        deg[ca[i]]++; deg[cb[i]]++;
    }
    /* orient, forward degree */
    for (int64_t i = 0; i < n; ++i) fdeg[i] = 0;
    for (int64_t i = 0; i < e; ++i) {
        int32_t a = ca[i], b = cb[i];
        int first = (deg[a] < deg[b]) || (deg[a] == deg[b] && a < b);
        int32_t s = first ? a : b, d = first ? b : a;
        fdeg[s]++;
        keys[i] = ((uint64_t)(uint32_t)s << 32) | (uint32_t)d;
    }
    row_ptr[0] = 0;
    for (int64_t i = 0; i < n; ++i) row_ptr[i + 1] = row_ptr[i] + fdeg[i];
    radix_sort_u64(keys, tmp, e, 32 + bits_for((uint64_t)(n > 0 ? n : 1)));
    for (int64_t i = 0; i < e; ++i) {
        edge_u[i] = (int32_t)(keys[i] >> 32);
        col_idx[i] = edge_v[i] = (int32_t)(keys[i] & 0xFFFFFFFFull);
    }
    *out_n_nodes = n;
    *out_n_edges = e;
    free(deg); free(ca); free(cb); free(ends); free(keys); free(tmp);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Seeded synthetic generators (specification restated independently of the  */
/* product's device generators)                                               */
/*                                                                            */
/*   key(seed, stream) = mix((seed + 1) * G  ^  stream * C)                    */
/*   draw(key, i)      = mix(key + (i + 1) * G)                                */
/* with mix the splitmix64 finaliser, G = 0x9E3779B97F4A7C15,                  */
/* C = 0xC2B2AE3D27D4EB4F.                                                     */
/* ------------------------------------------------------------------------- */

#define GEN_G 0x9E3779B97F4A7C15ull
#define GEN_C 0xC2B2AE3D27D4EB4Full

static inline uint64_t gen_key(uint64_t seed, uint64_t stream) {
    return orc_hash64((seed + 1ull) * GEN_G ^ (stream * GEN_C));
}
static inline uint64_t gen_draw(uint64_t key, uint64_t i) { return orc_hash64(key + (i + 1ull) * GEN_G); }

ORC_API uint64_t orc_gen_draw(uint64_t seed, uint64_t stream, uint64_t i) {
    return gen_draw(gen_key(seed, stream), i);
}

/* R-MAT: edge i descends `scale` levels; level l uses the high (l even) or low
 * (l odd) 32 bits of draw(key(seed,1), i*ceil(scale/2) + l/2) against the
 * cumulative thresholds ta <= tab <= tabc (probabilities * 2^32, floored). */
ORC_API void orc_gen_rmat(int scale, int64_t n_raw, uint32_t ta, uint32_t tab, uint32_t tabc,
                          uint64_t seed, int32_t* out_u, int32_t* out_v) {
    const uint64_t key = gen_key(seed, 1);
    const int64_t per = (scale + 1) / 2;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n_raw; ++i) {
        uint32_t u = 0, v = 0;
        uint64_t x = 0;
        for (int l = 0; l < scale; ++l) {
            uint32_t r;
            if ((l & 1) == 0) { x = gen_draw(key, (uint64_t)i * per + (l >> 1)); r = (uint32_t)(x >> 32); }
            else r = (uint32_t)x;
            uint32_t bu = 0, bv = 0;
            if (r < ta) { bu = 0; bv = 0; }
            else if (r < tab) { bu = 0; bv = 1; }
            else if (r < tabc) { bu = 1; bv = 0; }
            else { bu = 1; bv = 1; }
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        out_u[i] = (int32_t)u;
        out_v[i] = (int32_t)v;
    }
}

/* Erdos-Renyi endpoint pairs: u_i from draw(key(seed,2), 2i), v_i from
 * draw(.., 2i+1), each mapped to [0, n) by ((x >> 32) * n) >> 32. */
ORC_API void orc_gen_er(int64_t n, int64_t n_raw, uint64_t seed, int32_t* out_u, int32_t* out_v) {
    const uint64_t key = gen_key(seed, 2);
    for (int64_t i = 0; i < n_raw; ++i) {
        out_u[i] = (int32_t)(((gen_draw(key, 2 * (uint64_t)i) >> 32) * (uint64_t)n) >> 32);
        out_v[i] = (int32_t)(((gen_draw(key, 2 * (uint64_t)i + 1) >> 32) * (uint64_t)n) >> 32);
    }
}

/* Bijection of [0, n): balanced Feistel network over 2h bits (4 rounds, round
 * keys draw(key(seed,5), r)), cycle-walking until the value falls below n. */
static inline uint64_t feistel_perm(uint64_t x, uint64_t n, int h, const uint64_t* rk) {
    const uint64_t mask = (1ull << h) - 1ull;
    do {
        uint64_t L = x >> h, R = x & mask;
        for (int r = 0; r < 4; ++r) {
            uint64_t F = orc_hash64(R ^ rk[r]) & mask;
            uint64_t nl = R;
            R = L ^ F;
            L = nl;
        }
        x = (L << h) | R;
    } while (x >= n);
    return x;
}

ORC_API uint64_t orc_gen_perm(uint64_t x, uint64_t n, uint64_t seed) {
    int b = bits_for(n > 1 ? n - 1 : 1);
    int h = (b + 1) / 2;
    uint64_t key = gen_key(seed, 5), rk[4];
    for (int r = 0; r < 4; ++r) rk[r] = gen_draw(key, (uint64_t)r);
    return feistel_perm(x, n, h, rk);
}

/* Perturbed lattice on R x C cells.  Candidate k enumerates the right edges
 * (R*(C-1)), then the down edges ((R-1)*C), then one diagonal per cell
 * ((R-1)*(C-1), (i,j)-(i+1,j+1), present iff draw(key(seed,3), cell)>>32 <
 * tdiag).  Candidate k is deleted iff draw(key(seed,4), k)>>32 < tdel.  Ids
 * are permuted by orc_gen_perm.  Absent candidates are written as (0,0)
 * self-loops, which edge-list ingest drops.  Writes all candidates; returns
 * their number. */
ORC_API int64_t orc_gen_lattice(int64_t R, int64_t C, uint32_t tdiag, uint32_t tdel, uint64_t seed,
                                int32_t* out_u, int32_t* out_v) {
    const uint64_t kd = gen_key(seed, 3), kx = gen_key(seed, 4);
    const int64_t n_right = R * (C - 1), n_down = (R - 1) * C, n_diag = (R - 1) * (C - 1);
    const int64_t total = n_right + n_down + n_diag;
    const uint64_t N = (uint64_t)(R * C);
    int b = bits_for(N > 1 ? N - 1 : 1);
    int h = (b + 1) / 2;
    uint64_t kp = gen_key(seed, 5), rk[4];
    for (int r = 0; r < 4; ++r) rk[r] = gen_draw(kp, (uint64_t)r);
    if (!out_u) return total;
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < total; ++k) {
        int64_t a, bb;
        int present = 1;
        if (k < n_right) {
            int64_t i = k / (C - 1), j = k % (C - 1);
            a = i * C + j; bb = a + 1;
        } else if (k < n_right + n_down) {
            int64_t q = k - n_right, i = q / C, j = q % C;
            a = i * C + j; bb = a + C;
        } else {
            int64_t q = k - n_right - n_down, i = q / (C - 1), j = q % (C - 1);
            a = i * C + j; bb = a + C + 1;
            present = (uint32_t)(gen_draw(kd, (uint64_t)q) >> 32) < tdiag;
        }
        if (present && (uint32_t)(gen_draw(kx, (uint64_t)k) >> 32) < tdel) present = 0;
        if (present) {
            out_u[k] = (int32_t)feistel_perm((uint64_t)a, N, h, rk);
            out_v[k] = (int32_t)feistel_perm((uint64_t)bb, N, h, rk);
        } else {
            out_u[k] = 0; out_v[k] = 0;
        }
    }
    return total;
}

/* Chung-Lu: endpoints drawn in proportion to the integer weights whose
 * cumulative table `cum` (length n, cum[n-1] = total) the caller supplies:
 * endpoint = first index with cum[idx] > draw(key(seed,6), j) % total,
 * j = 2i for u_i and 2i+1 for v_i. */
ORC_API void orc_gen_chung_lu(const uint64_t* cum, int64_t n, int64_t n_raw, uint64_t seed,
                              int32_t* out_u, int32_t* out_v) {
    const uint64_t key = gen_key(seed, 6);
    const uint64_t total = cum[n - 1];
    for (int64_t i = 0; i < 2 * n_raw; ++i) {
        uint64_t t = gen_draw(key, (uint64_t)i) % total;
        int64_t lo = 0, hi = n;
        while (lo < hi) { int64_t mid = (lo + hi) >> 1; if (cum[mid] > t) hi = mid; else lo = mid + 1; }
        if (i & 1) out_v[i >> 1] = (int32_t)lo; else out_u[i >> 1] = (int32_t)lo;
    }
}

/* Chung-Lu weight table: w_i = (i+1)^(-1/(beta-1)), integer weight
 * max(1, llround(w_i * 2^24)), cumulative.  Returns the total. */
ORC_API uint64_t orc_chung_lu_table(int64_t n, double beta, uint64_t* cum) {
    double ex = -1.0 / (beta - 1.0);
    uint64_t s = 0;
    for (int64_t i = 0; i < n; ++i) {
        double w = pow((double)(i + 1), ex) * 16777216.0;
        long long iw = llround(w);
        if (iw < 1) iw = 1;
        s += (uint64_t)iw;
        cum[i] = s;
    }
    return s;
}

/* ------------------------------------------------------------------------- */
/* cpu_exp HLL variant (cpu_exp/triangle_hll_experiment.py:357-381,615-710)   */
/* ------------------------------------------------------------------------- */

#define CX_A 0x9E3779B97F4A7C15ull

/* splitmix64 with the +A increment, rank from h >> p, index = low p bits. */
ORC_API void orc_cx_build_registers(const int64_t* offsets, const int64_t* adj, int64_t n,
                                    int p, uint64_t seed, uint8_t* regs) {
    const int64_t m = 1ll << p;
    const int bits = 64 - p;
    for (int64_t u = 0; u < n; ++u) {
        uint8_t* row = regs + u * m;
        for (int64_t k = offsets[u]; k < offsets[u + 1]; ++k) {
            uint64_t h = orc_hash64((uint64_t)adj[k] + seed + CX_A);
            uint64_t idx = h & (uint64_t)(m - 1);
            uint64_t w = h >> p;
            int rho = (w == 0) ? bits + 1 : bits - (64 - __builtin_clzll(w)) + 1;
            if (rho > row[idx]) row[idx] = (uint8_t)rho;
        }
    }
}

/* estimate_hll_cardinality: sequential sum of ldexp(1,-r) (the Numba kernels'
 * order), 2^32 large-range constant. */
static double cx_estimate_pair(const uint8_t* a, const uint8_t* b, int64_t m) {
    double inv = 0.0;
    int64_t zeros = 0;
    for (int64_t j = 0; j < m; ++j) {
        int r = a[j] >= b[j] ? a[j] : b[j];
        inv += ldexp(1.0, -r);
        zeros += (r == 0);
    }
    double raw = orc_alpha(m) * (double)m * (double)m / inv;
    if (raw <= 2.5 * (double)m && zeros > 0) return (double)m * log((double)m / (double)zeros);
    if (raw > 4294967296.0 / 30.0) return -4294967296.0 * log(1.0 - raw / 4294967296.0);
    return raw;
}

/* hybrid_count (threshold: exact iff min(d+u, d+v) <= thr); a threshold below
 * zero gives the pure-HLL count.  out[0..5] = total, exact_edges, hll_edges,
 * exact_sum, hll_sum, clamp_count (as doubles). */
ORC_API void orc_cx_hybrid(const int64_t* offsets, const int64_t* adj, const int64_t* eu,
                           const int64_t* ev, int64_t n_edges, const int64_t* outdeg,
                           const uint8_t* regs, int p, int64_t threshold, double* out) {
    const int64_t m = 1ll << p;
    double exact_sum = 0.0, hll_sum = 0.0;
    int64_t exact_edges = 0, hll_edges = 0, clamp = 0;
    for (int64_t i = 0; i < n_edges; ++i) {
        int64_t u = eu[i], v = ev[i];
        int64_t cost = outdeg[u] < outdeg[v] ? outdeg[u] : outdeg[v];
        if (threshold >= 0 && cost <= threshold) {
            int64_t a0 = offsets[u], a1 = offsets[u + 1], b0 = offsets[v], b1 = offsets[v + 1];
            int64_t c = 0, x = a0, y = b0;
            while (x < a1 && y < b1) {
                if (adj[x] == adj[y]) { ++c; ++x; ++y; }
                else if (adj[x] < adj[y]) ++x;
                else ++y;
            }
            exact_sum += (double)c;
            ++exact_edges;
        } else {
            double ue = cx_estimate_pair(regs + u * m, regs + v * m, m);
            double est = (double)(outdeg[u] + outdeg[v]) - ue;
            double upper = (double)cost;
            if (est < 0.0) ++clamp;
            else if (est > upper) { hll_sum += upper; ++clamp; }
            else hll_sum += est;
            ++hll_edges;
        }
    }
    out[0] = exact_sum + hll_sum;
    out[1] = (double)exact_edges;
    out[2] = (double)hll_edges;
    out[3] = exact_sum;
    out[4] = hll_sum;
    out[5] = (double)clamp;
}
