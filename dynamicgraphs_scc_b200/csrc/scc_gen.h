// Seeded synthetic-graph formulas shared by the host generator and the device
// generator kernels.  Every function here is pure integer arithmetic on a
// counter-based RNG, so edge i of a graph is the same 64-bit computation on the
// CPU and on the GPU: the oracle and the CUDA path always see identical inputs.
//
// Graph families (the reference's benchmark inputs are not shipped, these stand
// in for them with the shapes the benchmark configurations name):
//   * R-MAT (a,b,c,d) = (.57,.19,.19,.05), scale s, edge factor ef,
//     vertex ids scrambled by a seeded bijection of [0, 2^s);
//   * a side x side 2D grid, every lattice edge oriented by a fair coin and
//     5% of them also given the reverse edge;
//   * planted directed cycles threaded through distinct vertex ids.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define SCC_HD __host__ __device__ __forceinline__
#else
#define SCC_HD static inline
#endif

// splitmix64 finaliser (Steele, Lea, Flood; public-domain constants from the
// published SplitMix64 algorithm).
SCC_HD uint64_t scc_mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Counter-based draw: stream `a`, index `b`, under `seed`.
SCC_HD uint64_t scc_rand3(uint64_t seed, uint64_t a, uint64_t b) {
    return scc_mix64(scc_mix64(seed ^ (a * 0xD1342543DE82EF95ull)) + b);
}

// Bijection of [0, 2^bits) used to scramble vertex ids (xor, odd multiply and
// xorshift are each invertible modulo 2^bits).
SCC_HD uint32_t scc_scramble(uint32_t v, int bits, uint64_t seed) {
    if (bits <= 0) return 0;
    uint64_t mask = (bits >= 32) ? 0xFFFFFFFFull : ((1ull << bits) - 1ull);
    uint64_t x = ((uint64_t)v ^ seed) & mask;
    int sh = bits / 2 + 1;
    x = (x * 0x9E3779B97F4A7C15ull) & mask;
    x ^= x >> sh;
    x = (x * (((seed >> 17) | 1ull) & 0xFFFFFFFFFFFFull)) & mask;
    x ^= x >> sh;
    x = (x * 0xBF58476D1CE4E5B9ull) & mask;
    x ^= x >> (sh > 1 ? sh - 1 : 1);
    return (uint32_t)x;
}

// R-MAT quadrant thresholds in 32-bit fixed point: a=.57, a+b=.76, a+b+c=.95.
#define SCC_RMAT_T0 2448131359u  // floor(0.57 * 2^32)
#define SCC_RMAT_T1 3264175145u  // floor(0.76 * 2^32)
#define SCC_RMAT_T2 4080218931u  // floor(0.95 * 2^32)

// Generated R-MAT edge `e` (before self-loop / duplicate removal).
SCC_HD void scc_rmat_edge(uint64_t seed, int scale, uint64_t e, uint32_t* src, uint32_t* dst) {
    uint32_t u = 0, v = 0;
    uint64_t r = 0;
    for (int l = 0; l < scale; ++l) {
        uint32_t x;
        if ((l & 1) == 0) { r = scc_rand3(seed, e, (uint64_t)(l >> 1)); x = (uint32_t)(r >> 32); }
        else { x = (uint32_t)r; }
        uint32_t ub = 0, vb = 0;
        if (x < SCC_RMAT_T0) { }
        else if (x < SCC_RMAT_T1) { vb = 1; }
        else if (x < SCC_RMAT_T2) { ub = 1; }
        else { ub = 1; vb = 1; }
        u = (u << 1) | ub;
        v = (v << 1) | vb;
    }
    *src = scc_scramble(u, scale, seed ^ 0x5CA7u);
    *dst = scc_scramble(v, scale, seed ^ 0x5CA7u);
}

// Undirected lattice edges of a side x side grid: side*(side-1) horizontal then
// side*(side-1) vertical.  Returns the two endpoints (row-major ids).
SCC_HD void scc_grid_lattice_edge(uint32_t side, uint64_t e, uint32_t* a, uint32_t* b) {
    uint64_t h = (uint64_t)side * (side - 1);
    if (e < h) {
        uint32_t r = (uint32_t)(e / (side - 1)), c = (uint32_t)(e % (side - 1));
        *a = r * side + c; *b = r * side + c + 1;
    } else {
        uint64_t f = e - h;
        uint32_t r = (uint32_t)(f / side), c = (uint32_t)(f % side);
        *a = r * side + c; *b = (r + 1) * side + c;
    }
}

// 5% of lattice edges are bidirectional: floor(0.05 * 2^32).
#define SCC_GRID_BIDIR_T 214748364u

// Directed edges contributed by lattice edge `e`: writes 1 or 2 edges, returns count.
SCC_HD int scc_grid_edges(uint64_t seed, uint32_t side, uint32_t base, uint64_t e,
                          uint32_t* s0, uint32_t* d0, uint32_t* s1, uint32_t* d1) {
    uint32_t a, b;
    scc_grid_lattice_edge(side, e, &a, &b);
    uint64_t r = scc_rand3(seed, 0x67726964ull, e);
    int flip = (int)(r & 1u);
    uint32_t x = (uint32_t)(r >> 32);
    uint32_t u = flip ? b : a, v = flip ? a : b;
    *s0 = base + u; *d0 = base + v;
    if (x < SCC_GRID_BIDIR_T) { *s1 = base + v; *d1 = base + u; return 2; }
    return 1;
}

// ---- batched uneven graphs
// Poisson CDF in 32-bit fixed point, thr[k] = floor(P(X <= k) * 2^32), built on
// the host; a draw is the first k with u < thr[k].
#define SCC_POIS_K 64
#define SCC_BATCH_MAX_DEG 255
SCC_HD int scc_poisson_draw(const uint32_t* thr, uint32_t u) {
    int k = 0;
    while (k < SCC_POIS_K - 1 && u >= thr[k]) ++k;
    return k < SCC_BATCH_MAX_DEG ? k : SCC_BATCH_MAX_DEG;
}

SCC_HD uint64_t scc_batch_graph_seed(uint64_t seed, uint32_t g) {
    return scc_mix64(seed ^ (0xBA7C4ull + (uint64_t)g * 0x9E3779B97F4A7C15ull));
}

SCC_HD int scc_ceil_log2(uint32_t n) {
    int s = 0;
    while ((1ull << s) < (uint64_t)n) ++s;
    return s;
}

SCC_HD int scc_batch_degree(const uint32_t* thr, uint64_t gseed, uint32_t lv) {
    return scc_poisson_draw(thr, (uint32_t)(scc_rand3(gseed, lv, 0) >> 32));
}

// Target of edge j of local vertex lv in a graph of n vertices: R-MAT column
// (reduced mod n) with probability rmat_thr / 2^32, else uniform.
SCC_HD uint32_t scc_batch_target(uint64_t gseed, uint32_t lv, uint32_t j, uint32_t n, uint32_t rmat_thr) {
    uint64_t r = scc_rand3(gseed, lv, 1 + (uint64_t)j);
    if ((uint32_t)r < rmat_thr) {
        uint32_t s, d;
        int scale = scc_ceil_log2(n);
        scc_rmat_edge(gseed ^ 0x77ull, scale > 0 ? scale : 1, ((uint64_t)lv << 8) | j, &s, &d);
        return d % n;
    }
    return (uint32_t)(((r >> 32) * (uint64_t)n) >> 32);
}

// Vertex of position `i` on planted cycle `k` (distinct within a cycle for
// i < 2^bits, since scc_scramble is a bijection).
SCC_HD uint32_t scc_cycle_vertex(uint64_t seed, uint32_t k, uint32_t i, int bits) {
    return scc_scramble(i, bits, scc_mix64(seed ^ (0xC1C1Eull + (uint64_t)k)));
}
