// Seeded synthetic graphs, generated on the host (for the oracle) and on the
// device (for the engine) from the same counter-based formulas (scc_gen.h), so
// both sides see the same edge multiset.  The reference's own datasets are not
// shipped; these stand in with the shapes of its benchmark configurations.
#include <math.h>
#include <string.h>
#include "scc_gen.h"
#include "scc_gen_api.h"
#include "scc_internal.cuh"

// Planted cycle lengths, log-uniform in [cycle_min, cycle_max] (host double
// math only; the device receives the integer lengths).
static void cycle_lengths(const scc_gen_params* p, std::vector<int64_t>& len) {
    len.resize((size_t)p->num_cycles);
    double lo = log((double)p->cycle_min), hi = log((double)p->cycle_max);
    for (int k = 0; k < p->num_cycles; ++k) {
        uint64_t r = scc_rand3(p->seed, 0xC7C1E5ull, (uint64_t)k);
        double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
        int64_t L = (int64_t)floor(exp(lo + u * (hi - lo)));
        if (L < p->cycle_min) L = p->cycle_min;
        if (L > p->cycle_max) L = p->cycle_max;
        len[(size_t)k] = L;
    }
}

static int check_params(const scc_gen_params* p) {
    SCC_REQUIRE(p, SCC_ERR_INVALID, "params is NULL");
    SCC_REQUIRE(p->rmat_scale >= 0 && p->rmat_scale <= 28, SCC_ERR_INVALID, "rmat_scale %d", p->rmat_scale);
    SCC_REQUIRE(p->edge_factor >= 0 && p->edge_factor <= 64, SCC_ERR_INVALID, "edge_factor %d", p->edge_factor);
    SCC_REQUIRE(p->grid_side >= 0 && p->grid_side <= 8192, SCC_ERR_INVALID, "grid_side %d", p->grid_side);
    SCC_REQUIRE(p->num_cycles >= 0, SCC_ERR_INVALID, "num_cycles %d", p->num_cycles);
    if (p->num_cycles > 0) {
        SCC_REQUIRE(p->rmat_scale >= 2, SCC_ERR_INVALID, "cycles need an R-MAT part");
        SCC_REQUIRE(p->cycle_min >= 2 && p->cycle_max >= p->cycle_min && p->cycle_max <= (1LL << p->rmat_scale),
                    SCC_ERR_INVALID, "cycle length range [%d, %d]", p->cycle_min, p->cycle_max);
    }
    int64_t n = 0;
    if (p->rmat_scale > 0) n += 1LL << p->rmat_scale;
    n += (int64_t)p->grid_side * p->grid_side;
    SCC_REQUIRE(n < SCC_WCC_ROOT_MASK, SCC_ERR_INVALID, "graph too large (n=%lld)", (long long)n);
    return SCC_OK;
}

extern "C" int scc_gen_sizes(const scc_gen_params* p, int32_t* n, int64_t* max_edges) {
    SCC_TRY(check_params(p));
    int64_t nn = 0, mm = 0;
    if (p->rmat_scale > 0 && p->edge_factor > 0) { nn += 1LL << p->rmat_scale; mm += (int64_t)p->edge_factor << p->rmat_scale; }
    else if (p->rmat_scale > 0) nn += 1LL << p->rmat_scale;
    if (p->grid_side > 1) mm += 4LL * p->grid_side * (p->grid_side - 1);
    nn += (int64_t)p->grid_side * p->grid_side;
    if (p->num_cycles > 0) {
        std::vector<int64_t> len;
        cycle_lengths(p, len);
        for (int64_t L : len) mm += L;
    }
    if (n) *n = (int32_t)nn;
    if (max_edges) *max_edges = mm;
    return SCC_OK;
}

// Host generation of the raw edge list (before self-loop / duplicate removal).
extern "C" int scc_gen_edges_host(const scc_gen_params* p, int32_t* src, int32_t* dst, int64_t capacity, int64_t* m) {
    SCC_TRY(check_params(p));
    SCC_REQUIRE(m, SCC_ERR_INVALID, "m is NULL");
    int64_t cap = 0;
    int32_t n = 0;
    SCC_TRY(scc_gen_sizes(p, &n, &cap));
    SCC_REQUIRE(capacity >= cap && src && dst, SCC_ERR_INVALID, "capacity %lld < %lld", (long long)capacity,
                (long long)cap);
    int64_t k = 0;
    if (p->rmat_scale > 0 && p->edge_factor > 0) {
        int64_t me = (int64_t)p->edge_factor << p->rmat_scale;
        for (int64_t e = 0; e < me; ++e) {
            uint32_t u, v;
            scc_rmat_edge(p->seed, p->rmat_scale, (uint64_t)e, &u, &v);
            src[k] = (int32_t)u; dst[k] = (int32_t)v; k++;
        }
    }
    if (p->grid_side > 1) {
        uint32_t base = p->rmat_scale > 0 ? (1u << p->rmat_scale) : 0u;
        uint64_t L = 2ull * p->grid_side * (p->grid_side - 1);
        for (uint64_t e = 0; e < L; ++e) {
            uint32_t s0, d0, s1, d1;
            int c = scc_grid_edges(p->seed ^ 0x9121Dull, (uint32_t)p->grid_side, base, e, &s0, &d0, &s1, &d1);
            src[k] = (int32_t)s0; dst[k] = (int32_t)d0; k++;
            if (c == 2) { src[k] = (int32_t)s1; dst[k] = (int32_t)d1; k++; }
        }
    }
    if (p->num_cycles > 0) {
        std::vector<int64_t> len;
        cycle_lengths(p, len);
        for (int c = 0; c < p->num_cycles; ++c) {
            int64_t L = len[(size_t)c];
            for (int64_t i = 0; i < L; ++i) {
                src[k] = (int32_t)scc_cycle_vertex(p->seed, (uint32_t)c, (uint32_t)i, p->rmat_scale);
                dst[k] = (int32_t)scc_cycle_vertex(p->seed, (uint32_t)c, (uint32_t)((i + 1) % L), p->rmat_scale);
                k++;
            }
        }
    }
    *m = k;
    return SCC_OK;
}

// ------------------------------------------------------------------ device generation
__global__ void k_gen_rmat(uint64_t seed, int scale, int64_t me, int32_t* __restrict__ src, int32_t* __restrict__ dst) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < me; e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t u, v;
        scc_rmat_edge(seed, scale, (uint64_t)e, &u, &v);
        src[e] = (int32_t)u; dst[e] = (int32_t)v;
    }
}

// Two slots per lattice edge; an unused second slot becomes a 0->0 self-loop
// that the build drops.
__global__ void k_gen_grid(uint64_t seed, uint32_t side, uint32_t base, uint64_t L, int32_t* __restrict__ src,
                           int32_t* __restrict__ dst) {
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < (int64_t)L; e += (int64_t)gridDim.x * blockDim.x) {
        uint32_t s0, d0, s1 = 0, d1 = 0;
        int c = scc_grid_edges(seed, side, base, (uint64_t)e, &s0, &d0, &s1, &d1);
        src[2 * e] = (int32_t)s0; dst[2 * e] = (int32_t)d0;
        if (c == 2) { src[2 * e + 1] = (int32_t)s1; dst[2 * e + 1] = (int32_t)d1; }
        else { src[2 * e + 1] = 0; dst[2 * e + 1] = 0; }
    }
}

__global__ void k_gen_cycles(uint64_t seed, int bits, int num_cycles, const int64_t* __restrict__ offs,
                             int32_t* __restrict__ src, int32_t* __restrict__ dst) {
    int64_t total = offs[num_cycles];
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = num_cycles - 1;
        while (lo < hi) { int mid = (lo + hi + 1) >> 1; if (offs[mid] <= t) lo = mid; else hi = mid - 1; }
        int64_t i = t - offs[lo], L = offs[lo + 1] - offs[lo];
        src[t] = (int32_t)scc_cycle_vertex(seed, (uint32_t)lo, (uint32_t)i, bits);
        dst[t] = (int32_t)scc_cycle_vertex(seed, (uint32_t)lo, (uint32_t)((i + 1) % L), bits);
    }
}

extern "C" int scc_gen_graph(const scc_gen_params* p, int flags, int device, scc_graph** out) {
    SCC_TRY(check_params(p));
    SCC_REQUIRE(out, SCC_ERR_INVALID, "out is NULL");
    SCC_CUDA(cudaSetDevice(device));
    int32_t n = 0;
    int64_t cap = 0;
    SCC_TRY(scc_gen_sizes(p, &n, &cap));
    int32_t *src = nullptr, *dst = nullptr;
    size_t bytes = sizeof(int32_t) * (size_t)(cap > 0 ? cap : 1);
    SCC_CUDA(cudaMalloc(&src, bytes));
    cudaError_t e = cudaMalloc(&dst, bytes);
    if (e != cudaSuccess) { cudaFree(src); return scc_cuda_status(e, "cudaMalloc", __FILE__, __LINE__); }
    int64_t k = 0;
    if (p->rmat_scale > 0 && p->edge_factor > 0) {
        int64_t me = (int64_t)p->edge_factor << p->rmat_scale;
        k_gen_rmat<<<scc_blocks(me, 256, 148 * 64), 256>>>(p->seed, p->rmat_scale, me, src, dst);
        k += me;
    }
    if (p->grid_side > 1) {
        uint32_t base = p->rmat_scale > 0 ? (1u << p->rmat_scale) : 0u;
        uint64_t L = 2ull * p->grid_side * (p->grid_side - 1);
        k_gen_grid<<<scc_blocks((int64_t)L, 256, 148 * 64), 256>>>(p->seed ^ 0x9121Dull, (uint32_t)p->grid_side, base, L,
                                                                  src + k, dst + k);
        k += 2 * (int64_t)L;
    }
    int64_t* d_offs = nullptr;
    if (p->num_cycles > 0) {
        std::vector<int64_t> len, offs((size_t)p->num_cycles + 1, 0);
        cycle_lengths(p, len);
        for (int c = 0; c < p->num_cycles; ++c) offs[(size_t)c + 1] = offs[(size_t)c] + len[(size_t)c];
        SCC_CUDA(cudaMalloc(&d_offs, sizeof(int64_t) * offs.size()));
        SCC_CUDA(cudaMemcpy(d_offs, offs.data(), sizeof(int64_t) * offs.size(), cudaMemcpyHostToDevice));
        k_gen_cycles<<<scc_blocks(offs.back(), 256, 148 * 64), 256>>>(p->seed, p->rmat_scale, p->num_cycles, d_offs,
                                                                      src + k, dst + k);
        k += offs.back();
    }
    SCC_CUDA(cudaPeekAtLastError());
    SCC_CUDA(cudaDeviceSynchronize());
    cudaFree(d_offs);
    int rc = scc_impl_build_graph_from_device_edges(n, k, src, dst, flags, device, out);
    cudaFree(src);
    cudaFree(dst);
    return rc;
}
