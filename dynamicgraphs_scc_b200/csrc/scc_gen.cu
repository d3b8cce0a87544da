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

// ------------------------------------------------------------------ batched uneven graphs
#include <cub/device/device_scan.cuh>

struct BatchTables {
    std::vector<int32_t> offsets;   // num_graphs + 1
    uint32_t pois[SCC_POIS_K];
    uint32_t rmat_thr;
};

static int batch_tables(const scc_batch_params* p, BatchTables& t) {
    SCC_REQUIRE(p, SCC_ERR_INVALID, "params is NULL");
    SCC_REQUIRE(p->num_graphs >= 1 && p->num_graphs <= (1 << 20), SCC_ERR_INVALID, "num_graphs %d", p->num_graphs);
    SCC_REQUIRE(p->n_min >= 1 && p->n_max >= p->n_min && p->n_max <= (1 << 24), SCC_ERR_INVALID,
                "vertex range [%d, %d]", p->n_min, p->n_max);
    SCC_REQUIRE(p->mean_degree >= 0.0 && p->mean_degree <= 32.0, SCC_ERR_INVALID, "mean_degree %f", p->mean_degree);
    SCC_REQUIRE(p->rmat_fraction >= 0.0 && p->rmat_fraction <= 1.0, SCC_ERR_INVALID, "rmat_fraction %f",
                p->rmat_fraction);
    t.offsets.assign((size_t)p->num_graphs + 1, 0);
    double lo = log((double)p->n_min), hi = log((double)p->n_max);
    int64_t total = 0;
    for (int32_t g = 0; g < p->num_graphs; ++g) {
        uint64_t r = scc_rand3(p->seed, 0xB47ull, (uint64_t)g);
        double u = (double)(r >> 11) * (1.0 / 9007199254740992.0);
        int64_t ni = (int64_t)floor(exp(lo + u * (hi - lo)));
        if (ni < p->n_min) ni = p->n_min;
        if (ni > p->n_max) ni = p->n_max;
        total += ni;
        SCC_REQUIRE(total < SCC_WCC_ROOT_MASK, SCC_ERR_INVALID, "batch too large (%lld vertices)", (long long)total);
        t.offsets[(size_t)g + 1] = (int32_t)total;
    }
    // Poisson(mean) CDF thresholds
    double pk = exp(-p->mean_degree), cdf = 0.0;
    for (int k = 0; k < SCC_POIS_K; ++k) {
        if (k > 0) pk *= p->mean_degree / k;
        cdf += pk;
        double x = cdf * 4294967296.0;
        t.pois[k] = (k == SCC_POIS_K - 1 || x >= 4294967295.0) ? 0xFFFFFFFFu : (uint32_t)x;
    }
    double rt = p->rmat_fraction * 4294967296.0;
    t.rmat_thr = rt >= 4294967295.0 ? 0xFFFFFFFFu : (uint32_t)rt;
    return SCC_OK;
}

extern "C" int scc_gen_batch_layout(const scc_batch_params* p, int32_t* offsets, int32_t* n, int64_t* max_edges) {
    BatchTables t;
    SCC_TRY(batch_tables(p, t));
    if (offsets) memcpy(offsets, t.offsets.data(), sizeof(int32_t) * t.offsets.size());
    if (n) *n = t.offsets.back();
    if (max_edges) *max_edges = (int64_t)t.offsets.back() * SCC_BATCH_MAX_DEG;
    return SCC_OK;
}

extern "C" int scc_gen_batch_edges_host(const scc_batch_params* p, int32_t* src, int32_t* dst, int64_t capacity,
                                        int64_t* m) {
    BatchTables t;
    SCC_TRY(batch_tables(p, t));
    SCC_REQUIRE(src && dst && m, SCC_ERR_INVALID, "NULL argument");
    int64_t k = 0;
    for (int32_t g = 0; g < p->num_graphs; ++g) {
        uint64_t gs = scc_batch_graph_seed(p->seed, (uint32_t)g);
        int32_t base = t.offsets[(size_t)g];
        uint32_t ni = (uint32_t)(t.offsets[(size_t)g + 1] - base);
        for (uint32_t lv = 0; lv < ni; ++lv) {
            int d = scc_batch_degree(t.pois, gs, lv);
            SCC_REQUIRE(k + d <= capacity, SCC_ERR_INVALID, "capacity %lld too small", (long long)capacity);
            for (int j = 0; j < d; ++j) {
                src[k] = base + (int32_t)lv;
                dst[k] = base + (int32_t)scc_batch_target(gs, lv, (uint32_t)j, ni, t.rmat_thr);
                k++;
            }
        }
    }
    *m = k;
    return SCC_OK;
}

struct BatchDev {
    const int32_t* offsets; int32_t num_graphs; uint64_t seed; uint32_t rmat_thr; uint32_t pois[SCC_POIS_K];
};

__device__ __forceinline__ int32_t batch_graph_of(const BatchDev& b, int32_t v) {
    int32_t lo = 0, hi = b.num_graphs - 1;
    while (lo < hi) { int32_t mid = (lo + hi + 1) >> 1; if (b.offsets[mid] <= v) lo = mid; else hi = mid - 1; }
    return lo;
}

__global__ void k_batch_degree(BatchDev b, int32_t n, int64_t* __restrict__ deg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = (int32_t)i, g = batch_graph_of(b, v);
        deg[i] = scc_batch_degree(b.pois, scc_batch_graph_seed(b.seed, (uint32_t)g), (uint32_t)(v - b.offsets[g]));
    }
}

__global__ void k_batch_edges(BatchDev b, int32_t n, const int64_t* __restrict__ eoff, int32_t* __restrict__ src,
                              int32_t* __restrict__ dst) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = (int32_t)i, g = batch_graph_of(b, v);
        int32_t base = b.offsets[g];
        uint32_t ni = (uint32_t)(b.offsets[g + 1] - base), lv = (uint32_t)(v - base);
        uint64_t gs = scc_batch_graph_seed(b.seed, (uint32_t)g);
        int d = scc_batch_degree(b.pois, gs, lv);
        int64_t o = eoff[i];
        for (int j = 0; j < d; ++j) {
            src[o + j] = v;
            dst[o + j] = base + (int32_t)scc_batch_target(gs, lv, (uint32_t)j, ni, b.rmat_thr);
        }
    }
}

extern "C" int scc_gen_batch_graph(const scc_batch_params* p, int flags, int device, scc_graph** out) {
    BatchTables t;
    SCC_TRY(batch_tables(p, t));
    SCC_REQUIRE(out, SCC_ERR_INVALID, "out is NULL");
    SCC_CUDA(cudaSetDevice(device));
    int32_t n = t.offsets.back();
    int32_t* d_off = nullptr;
    int64_t *deg = nullptr, *eoff = nullptr;
    SCC_CUDA(cudaMalloc(&d_off, sizeof(int32_t) * t.offsets.size()));
    SCC_CUDA(cudaMalloc(&deg, sizeof(int64_t) * ((size_t)n + 1)));
    SCC_CUDA(cudaMalloc(&eoff, sizeof(int64_t) * ((size_t)n + 1)));
    SCC_CUDA(cudaMemcpy(d_off, t.offsets.data(), sizeof(int32_t) * t.offsets.size(), cudaMemcpyHostToDevice));
    SCC_CUDA(cudaMemset(deg, 0, sizeof(int64_t) * ((size_t)n + 1)));
    BatchDev b;
    b.offsets = d_off; b.num_graphs = p->num_graphs; b.seed = p->seed; b.rmat_thr = t.rmat_thr;
    memcpy(b.pois, t.pois, sizeof(t.pois));
    k_batch_degree<<<scc_blocks(n, 256, 148 * 64), 256>>>(b, n, deg);
    SCC_CUDA(cudaPeekAtLastError());
    size_t bytes = 0;
    void* tmp = nullptr;
    SCC_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, deg, eoff, n + 1));
    SCC_CUDA(cudaMalloc(&tmp, bytes > 0 ? bytes : 16));
    SCC_CUDA(cub::DeviceScan::ExclusiveSum(tmp, bytes, deg, eoff, n + 1));
    int64_t m = 0;
    SCC_CUDA(cudaMemcpy(&m, eoff + n, sizeof(int64_t), cudaMemcpyDeviceToHost));
    cudaFree(tmp);
    int32_t *src = nullptr, *dst = nullptr;
    SCC_CUDA(cudaMalloc(&src, sizeof(int32_t) * (size_t)(m > 0 ? m : 1)));
    SCC_CUDA(cudaMalloc(&dst, sizeof(int32_t) * (size_t)(m > 0 ? m : 1)));
    k_batch_edges<<<scc_blocks(n, 256, 148 * 64), 256>>>(b, n, eoff, src, dst);
    SCC_CUDA(cudaPeekAtLastError());
    SCC_CUDA(cudaDeviceSynchronize());
    cudaFree(deg); cudaFree(eoff); cudaFree(d_off);
    int rc = scc_impl_build_graph_from_device_edges(n, m, src, dst, flags, device, out);
    cudaFree(src); cudaFree(dst);
    return rc;
}

// ------------------------------------------------------------------ subgraph of a closed id range
__global__ void k_sub_offsets(const int32_t* __restrict__ off, int32_t vb, int32_t nv, int32_t* __restrict__ out) {
    int32_t base = off[vb];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nv; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = off[vb + i] - base;
}

__global__ void k_sub_adj(const int32_t* __restrict__ adj, int64_t e0, int64_t cnt, int32_t vb, int32_t nv,
                          int32_t* __restrict__ out, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t w = adj[e0 + i] - vb;
        if (w < 0 || w >= nv) { atomicExch(bad, 1); w = 0; }
        out[i] = w;
    }
}

extern "C" int scc_graph_subgraph(const scc_graph* g, int32_t v_begin, int32_t v_end, scc_graph** out) {
    SCC_REQUIRE(g && out, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(v_begin >= 0 && v_end >= v_begin && v_end <= g->n, SCC_ERR_INVALID, "range [%d, %d)", v_begin, v_end);
    SCC_CUDA(cudaSetDevice(g->device));
    int32_t nv = v_end - v_begin;
    int32_t h[4];
    SCC_CUDA(cudaMemcpy(&h[0], g->begin + v_begin, sizeof(int32_t), cudaMemcpyDeviceToHost));
    SCC_CUDA(cudaMemcpy(&h[1], g->begin + v_end, sizeof(int32_t), cudaMemcpyDeviceToHost));
    SCC_CUDA(cudaMemcpy(&h[2], g->r_begin + v_begin, sizeof(int32_t), cudaMemcpyDeviceToHost));
    SCC_CUDA(cudaMemcpy(&h[3], g->r_begin + v_end, sizeof(int32_t), cudaMemcpyDeviceToHost));
    int64_t m = h[1] - h[0];
    SCC_REQUIRE(h[3] - h[2] == m, SCC_ERR_INVALID, "range [%d, %d) has edges leaving it", v_begin, v_end);
    scc_graph* s = new scc_graph();
    s->device = g->device; s->n = nv; s->m = m;
    int* bad = nullptr;
    cudaError_t e = cudaMalloc(&s->begin, sizeof(int32_t) * ((size_t)nv + 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->r_begin, sizeof(int32_t) * ((size_t)nv + 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->node_idx, sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    if (e == cudaSuccess) e = cudaMalloc(&s->r_node_idx, sizeof(int32_t) * (size_t)(m > 0 ? m : 1));
    if (e == cudaSuccess) e = cudaMalloc(&bad, sizeof(int));
    if (e == cudaSuccess) e = cudaMemset(bad, 0, sizeof(int));
    if (e != cudaSuccess) { scc_graph_free(s); cudaFree(bad); return scc_cuda_status(e, "subgraph", __FILE__, __LINE__); }
    k_sub_offsets<<<scc_blocks(nv + 1), 256>>>(g->begin, v_begin, nv, s->begin);
    k_sub_offsets<<<scc_blocks(nv + 1), 256>>>(g->r_begin, v_begin, nv, s->r_begin);
    if (m > 0) {
        k_sub_adj<<<scc_blocks(m), 256>>>(g->node_idx, h[0], m, v_begin, nv, s->node_idx, bad);
        k_sub_adj<<<scc_blocks(m), 256>>>(g->r_node_idx, h[2], m, v_begin, nv, s->r_node_idx, bad);
    }
    int hb = 0;
    e = cudaMemcpy(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(bad);
    if (e != cudaSuccess) { scc_graph_free(s); return scc_cuda_status(e, "subgraph", __FILE__, __LINE__); }
    if (hb) { scc_graph_free(s); scc_set_error("range [%d, %d) has edges leaving it", v_begin, v_end); return SCC_ERR_INVALID; }
    *out = s;
    return SCC_OK;
}
