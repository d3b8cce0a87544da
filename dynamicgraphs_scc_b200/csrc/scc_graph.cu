// Graph construction: edge list -> sorted CSR + sorted transpose, on the device.
//
// Replaces gm_graph add_node/add_edge + freeze + do_semi_sort +
// make_reverse_edges (gm_graph/src/gm_graph.cc:459-480, 60-101, 385-420,
// 193-287): one 64-bit radix sort of (src<<32 | dst) keys gives the out-CSR
// with each adjacency list sorted by destination (the semi-sort), a second
// sort of (dst<<32 | src) gives the transpose sorted by source.  Offsets are
// filled from the sorted keys by a gap-fill kernel.  Duplicates and self-loops
// are kept unless the caller asks otherwise, as gm_graph keeps them.
#include "scc_sort.cuh"
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include <algorithm>
#include <atomic>
#include <mutex>
#include "scc_internal.cuh"

// ------------------------------------------------------------------ errors
static thread_local char g_err[512] = "";

void scc_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int scc_cuda_status(cudaError_t e, const char* what, const char* file, int line) {
    scc_set_error("CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), what, file, line);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();  // clear the sticky-free allocation error
        return SCC_ERR_OOM;
    }
    return SCC_ERR_CUDA;
}

extern "C" const char* scc_last_error(void) { return g_err; }

extern "C" const char* scc_status_string(int status) {
    switch (status) {
        case SCC_OK: return "ok";
        case SCC_ERR_INVALID: return "invalid argument";
        case SCC_ERR_CUDA: return "CUDA error";
        case SCC_ERR_OOM: return "out of device memory";
        case SCC_ERR_TIMEOUT: return "bounded device wait gave up";
        case SCC_ERR_STATE: return "call out of order";
        case SCC_ERR_IO: return "file error";
        case SCC_ERR_NOT_FOUND: return "not found";
        case SCC_ERR_UNSUPPORTED: return "unsupported";
        case SCC_ERR_BUSY: return "busy (admission limit)";
        default: return "unknown status";
    }
}

extern "C" int scc_version(void) { return 100; }

extern "C" int scc_device_count(int* count) {
    SCC_REQUIRE(count, SCC_ERR_INVALID, "count is NULL");
    int c = 0;
    cudaError_t e = cudaGetDeviceCount(&c);
    if (e != cudaSuccess) { cudaGetLastError(); c = 0; }
    *count = c;
    return SCC_OK;
}

// ------------------------------------------------------------------ kernels
__global__ void k_make_keys(int64_t m, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                            unsigned long long* __restrict__ keys, int drop_self,
                            unsigned long long* __restrict__ dropped) {
    unsigned long long local = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        uint32_t x = (uint32_t)a[i], y = (uint32_t)b[i];
        if (drop_self && x == y) { keys[i] = ~0ull; local++; }
        else keys[i] = ((unsigned long long)x << 32) | y;
    }
    if (local) atomicAdd(dropped, local);
}

// Offsets from sorted keys: begin[v] = first index i with key(i) >= v, for v
// in [0, n].  Each key boundary fills at most FILL_SERIAL entries of the gap
// before it; entries of longer gaps (ids with no edges, e.g. a vertex range no
// edge of a chunk touches) stay at -1 and k_fill_gaps* finds them by binary
// search, so no thread walks millions of entries alone.  begin is preset to -1.
#define FILL_SERIAL 32

__device__ __forceinline__ int64_t key_hi(const unsigned long long* keys, int64_t i) { return (int64_t)(keys[i] >> 32); }
__device__ __forceinline__ int64_t key_hi(const int32_t* keys, int64_t i) { return (int64_t)keys[i]; }

template <class K>
__global__ void k_fill_offsets_t(int64_t m, int32_t n, const K* __restrict__ keys, int32_t* __restrict__ begin) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= m; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t prev = (i == 0) ? -1 : key_hi(keys, i - 1);
        int64_t cur = (i == m) ? (int64_t)n : key_hi(keys, i);
        int64_t last = min(min(cur, (int64_t)n), prev + FILL_SERIAL);
        for (int64_t v = prev + 1; v <= last; ++v) begin[v] = (int32_t)i;
    }
}

template <class K>
__global__ void k_fill_gaps_t(int64_t m, int32_t n, const K* __restrict__ keys, int32_t* __restrict__ begin) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v <= n; v += (int64_t)gridDim.x * blockDim.x) {
        if (begin[v] >= 0) continue;
        int64_t lo = 0, hi = m;                  // first index with key >= v
        while (lo < hi) {
            int64_t mid = (lo + hi) >> 1;
            if (key_hi(keys, mid) < v) lo = mid + 1; else hi = mid;
        }
        begin[v] = (int32_t)lo;
    }
}

template <class K>
static cudaError_t fill_offsets(int64_t m, int32_t n, const K* keys, int32_t* begin, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(begin, 0xFF, sizeof(int32_t) * ((size_t)n + 1), st);
    if (e != cudaSuccess) return e;
    k_fill_offsets_t<K><<<scc_blocks(m + 1, 256, 148 * 64), 256, 0, st>>>(m, n, keys, begin);
    k_fill_gaps_t<K><<<scc_blocks((int64_t)n + 1, 256, 148 * 64), 256, 0, st>>>(m, n, keys, begin);
    return cudaPeekAtLastError();
}

__global__ void k_low_words(int64_t m, const unsigned long long* __restrict__ keys, int32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = (int32_t)(uint32_t)(keys[i] & 0xFFFFFFFFull);
}

// src[e] = v for e in [begin[v], begin[v+1]) -- one warp per vertex.
__global__ void k_expand_sources(int32_t n, const int32_t* __restrict__ begin, int32_t* __restrict__ src) {
    int lane = threadIdx.x & 31;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < n;
         w += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        int32_t b = begin[w], e = begin[w + 1];
        for (int32_t k = b + lane; k < e; k += 32) src[k] = (int32_t)w;
    }
}

__global__ void k_check_ids(int64_t m, int32_t n, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                            int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        if (a[i] < 0 || a[i] >= n || b[i] < 0 || b[i] >= n) { atomicExch(bad, 1); return; }
    }
}

static int bits_for(int32_t n) {
    int b = 1;
    while (b < 31 && (1LL << b) < (int64_t)n) b++;
    return b;
}

// Stream-ordered scratch, released on the same stream.
struct AsyncScratch {
    void* p = nullptr;
    cudaStream_t st;
    explicit AsyncScratch(cudaStream_t s) : st(s) {}
    ~AsyncScratch() { if (p) cudaFreeAsync(p, st); }
    cudaError_t alloc(size_t bytes) { return scc_impl_malloc_async(&p, bytes > 0 ? bytes : 16, st); }
};

// Sort (hi<<32|lo) keys and write offsets + low words.  keys buffer is reused.
static int build_side(int32_t n, int64_t m, const int32_t* hi, const int32_t* lo, int flags, cudaStream_t st,
                      int32_t** begin_out, int32_t** idx_out, int64_t* m_out) {
    // temporaries come from the library's pool, stream-ordered on st (no
    // device-wide cudaMalloc/cudaFree of GB-sized key buffers per build)
    int64_t mm = m > 0 ? m : 1;
    AsyncScratch keys_b(st), keys2_b(st), dropped_b(st);
    SCC_CUDA(keys_b.alloc(sizeof(unsigned long long) * mm));
    SCC_CUDA(keys2_b.alloc(sizeof(unsigned long long) * mm));
    SCC_CUDA(dropped_b.alloc(sizeof(unsigned long long) * 2));
    unsigned long long* keys = (unsigned long long*)keys_b.p;
    unsigned long long* keys2 = (unsigned long long*)keys2_b.p;
    unsigned long long* dropped = (unsigned long long*)dropped_b.p;
    SCC_CUDA(cudaMemsetAsync(dropped, 0, sizeof(unsigned long long) * 2, st));
    int drop_self = (flags & SCC_BUILD_NO_SELF_LOOPS) ? 1 : 0;
    if (m > 0) {
        k_make_keys<<<scc_blocks(m, 256, 148 * 64), 256, 0, st>>>(m, hi, lo, keys, drop_self, dropped);
        SCC_CUDA(cudaPeekAtLastError());
    }
    int end_bit = 32 + bits_for(n + 1);
    if (drop_self) end_bit = 64;
    SCC_TRY(scc_impl_sort_keys_u64(keys, keys2, m, end_bit, st));
    unsigned long long* sorted = keys2;
    unsigned long long* other = keys;
    unsigned long long h_dropped = 0;
    SCC_CUDA(cudaMemcpyAsync(&h_dropped, dropped, sizeof(h_dropped), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    int64_t mk = m - (int64_t)h_dropped;   // self-loops sorted to the end
    if ((flags & SCC_BUILD_DEDUP) && mk > 0) {
        int64_t mu = 0;
        SCC_TRY(scc_impl_unique_u64(sorted, other, mk, &mu, st));
        mk = mu;
        unsigned long long* t = sorted; sorted = other; other = t;
    }
    int32_t *begin = nullptr, *idx = nullptr;
    SCC_CUDA(cudaMalloc(&begin, sizeof(int32_t) * ((size_t)n + 1)));
    cudaError_t e = cudaMalloc(&idx, sizeof(int32_t) * (size_t)(mk > 0 ? mk : 1));
    if (e != cudaSuccess) { cudaFree(begin); return scc_cuda_status(e, "cudaMalloc", __FILE__, __LINE__); }
    e = fill_offsets(mk, n, sorted, begin, st);
    if (e == cudaSuccess && mk > 0) {
        k_low_words<<<scc_blocks(mk, 256, 148 * 64), 256, 0, st>>>(mk, sorted, idx);
        e = cudaPeekAtLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { cudaFree(begin); cudaFree(idx); return scc_cuda_status(e, "build_side", __FILE__, __LINE__); }
    *begin_out = begin; *idx_out = idx; *m_out = mk;
    return SCC_OK;
}

int scc_impl_build_graph_from_device_edges(int32_t n, int64_t m, const int32_t* d_src, const int32_t* d_dst,
                                           int flags, int device, scc_graph** out) {
    SCC_REQUIRE(out, SCC_ERR_INVALID, "out is NULL");
    SCC_REQUIRE(n >= 0 && m >= 0, SCC_ERR_INVALID, "negative size n=%d m=%lld", n, (long long)m);
    SCC_REQUIRE(m < (1LL << 31) - 1, SCC_ERR_INVALID, "m=%lld exceeds int32 edge ids", (long long)m);
    SCC_REQUIRE(n < SCC_WCC_ROOT_MASK, SCC_ERR_INVALID, "n=%d exceeds 0x1FFFFFFF", n);
    SCC_CUDA(cudaSetDevice(device));
    cudaStream_t st;
    SCC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    if (m > 0) {
        int* bad = nullptr;
        SCC_CUDA(cudaMalloc(&bad, sizeof(int)));
        SCC_CUDA(cudaMemsetAsync(bad, 0, sizeof(int), st));
        k_check_ids<<<scc_blocks(m, 256, 148 * 64), 256, 0, st>>>(m, n, d_src, d_dst, bad);
        int hb = 0;
        SCC_CUDA(cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
        SCC_CUDA(cudaStreamSynchronize(st));
        cudaFree(bad);
        if (hb) { cudaStreamDestroy(st); scc_set_error("edge endpoint outside [0, %d)", n); return SCC_ERR_INVALID; }
    }
    scc_graph* g = new scc_graph();
    g->device = device;
    g->n = n;
    int64_t m1 = 0, m2 = 0;
    int s = build_side(n, m, d_src, d_dst, flags, st, &g->begin, &g->node_idx, &m1);
    if (s == SCC_OK) s = build_side(n, m, d_dst, d_src, flags, st, &g->r_begin, &g->r_node_idx, &m2);
    if (flags & SCC_BUILD_NO_SELF_LOOPS) g->self_loops = 0;
    cudaStreamDestroy(st);
    if (s != SCC_OK) { scc_graph_free(g); return s; }
    g->m = m1;
    *out = g;
    return SCC_OK;
}


// Transpose of g's forward CSR into g->r_begin / g->r_node_idx (allocated):
// a stable radix sort of (destination, source) pairs taken in edge order, so
// every in-list comes out sorted by source -- gm_graph's make_reverse_edges
// order (gm_graph/src/gm_graph.cc:193-287), duplicates kept.
static int transpose_into(scc_graph* g, cudaStream_t st) {
    const int64_t m = g->m;
    const int32_t n = g->n;
    if (m == 0) {
        SCC_CUDA(cudaMemsetAsync(g->r_begin, 0, sizeof(int32_t) * ((size_t)n + 1), st));
        return SCC_OK;
    }
    AsyncScratch src(st), keys(st);
    SCC_CUDA(src.alloc(sizeof(int32_t) * (size_t)m));
    SCC_CUDA(keys.alloc(sizeof(int32_t) * (size_t)m));
    k_expand_sources<<<scc_blocks((int64_t)n * 32, 256, 148 * 64), 256, 0, st>>>(n, g->begin, (int32_t*)src.p);
    SCC_CUDA(cudaPeekAtLastError());
    SCC_TRY(scc_impl_sort_pairs_u32(reinterpret_cast<const uint32_t*>(g->node_idx), (uint32_t*)keys.p,
                                    (const int32_t*)src.p, g->r_node_idx, m, bits_for(n), st));
    SCC_CUDA(fill_offsets(m, n, (const int32_t*)keys.p, g->r_begin, st));
    return SCC_OK;
}

int scc_impl_transpose(scc_graph* g, cudaStream_t st) {
    size_t nb = sizeof(int32_t) * ((size_t)g->n + 1), mb = sizeof(int32_t) * (size_t)(g->m > 0 ? g->m : 1);
    SCC_CUDA(cudaMalloc(&g->r_begin, nb));
    SCC_CUDA(cudaMalloc(&g->r_node_idx, mb));
    SCC_TRY(transpose_into(g, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    return SCC_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int scc_graph_create_edges_device(int32_t n, int64_t m, const int32_t* d_src, const int32_t* d_dst,
                                             int flags, int device, scc_graph** out) {
    SCC_REQUIRE(m == 0 || (d_src && d_dst), SCC_ERR_INVALID, "edge arrays are NULL");
    return scc_impl_build_graph_from_device_edges(n, m, d_src, d_dst, flags, device, out);
}

extern "C" int scc_graph_create_edges(int32_t n, int64_t m, const int32_t* src, const int32_t* dst, int flags,
                                      int device, scc_graph** out) {
    SCC_REQUIRE(m == 0 || (src && dst), SCC_ERR_INVALID, "edge arrays are NULL");
    SCC_REQUIRE(m >= 0 && n >= 0, SCC_ERR_INVALID, "negative size");
    SCC_CUDA(cudaSetDevice(device));
    int32_t *ds = nullptr, *dd = nullptr;
    size_t bytes = sizeof(int32_t) * (size_t)(m > 0 ? m : 1);
    SCC_CUDA(cudaMalloc(&ds, bytes));
    cudaError_t e = cudaMalloc(&dd, bytes);
    if (e != cudaSuccess) { cudaFree(ds); return scc_cuda_status(e, "cudaMalloc", __FILE__, __LINE__); }
    if (m > 0) {
        SCC_CUDA(cudaMemcpy(ds, src, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice));
        SCC_CUDA(cudaMemcpy(dd, dst, sizeof(int32_t) * (size_t)m, cudaMemcpyHostToDevice));
    }
    int s = scc_impl_build_graph_from_device_edges(n, m, ds, dd, flags, device, out);
    cudaFree(ds); cudaFree(dd);
    return s;
}

static int create_csr_common(int32_t n, int32_t m, const int32_t* begin, const int32_t* node_idx,
                             const int32_t* r_begin, const int32_t* r_node_idx, int device, scc_graph** out,
                             cudaMemcpyKind kind) {
    SCC_REQUIRE(out, SCC_ERR_INVALID, "out is NULL");
    SCC_REQUIRE(n >= 0 && m >= 0, SCC_ERR_INVALID, "negative size");
    SCC_REQUIRE(begin && (m == 0 || node_idx), SCC_ERR_INVALID, "CSR arrays are NULL");
    SCC_REQUIRE((r_begin == nullptr) == (r_node_idx == nullptr) || m == 0, SCC_ERR_INVALID,
                "give both transpose arrays or neither");
    SCC_REQUIRE(n < SCC_WCC_ROOT_MASK, SCC_ERR_INVALID, "n=%d exceeds 0x1FFFFFFF", n);
    SCC_CUDA(cudaSetDevice(device));
    scc_graph* g = new scc_graph();
    g->device = device; g->n = n; g->m = m;
    size_t nb = sizeof(int32_t) * ((size_t)n + 1), mb = sizeof(int32_t) * (size_t)(m > 0 ? m : 1);
    cudaError_t e = cudaMalloc(&g->begin, nb);
    if (e == cudaSuccess) e = cudaMalloc(&g->node_idx, mb);
    if (e == cudaSuccess) e = cudaMemcpy(g->begin, begin, nb, kind);
    if (e == cudaSuccess && m > 0) e = cudaMemcpy(g->node_idx, node_idx, sizeof(int32_t) * (size_t)m, kind);
    if (e == cudaSuccess && r_begin) {
        e = cudaMalloc(&g->r_begin, nb);
        if (e == cudaSuccess) e = cudaMalloc(&g->r_node_idx, mb);
        if (e == cudaSuccess) e = cudaMemcpy(g->r_begin, r_begin, nb, kind);
        if (e == cudaSuccess && m > 0) e = cudaMemcpy(g->r_node_idx, r_node_idx, sizeof(int32_t) * (size_t)m, kind);
    }
    if (e != cudaSuccess) { scc_graph_free(g); return scc_cuda_status(e, "csr upload", __FILE__, __LINE__); }
    if (!r_begin) {
        cudaStream_t st;
        SCC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        int s = scc_impl_transpose(g, st);
        cudaStreamDestroy(st);
        if (s != SCC_OK) { scc_graph_free(g); return s; }
    }
    *out = g;
    return SCC_OK;
}

extern "C" int scc_graph_create_csr(int32_t n, int32_t m, const int32_t* begin, const int32_t* node_idx,
                                    const int32_t* r_begin, const int32_t* r_node_idx, int device, scc_graph** out) {
    return create_csr_common(n, m, begin, node_idx, r_begin, r_node_idx, device, out, cudaMemcpyHostToDevice);
}

extern "C" int scc_graph_create_csr_device(int32_t n, int32_t m, const int32_t* d_begin, const int32_t* d_node_idx,
                                           const int32_t* d_r_begin, const int32_t* d_r_node_idx, int device,
                                           scc_graph** out) {
    return create_csr_common(n, m, d_begin, d_node_idx, d_r_begin, d_r_node_idx, device, out,
                             cudaMemcpyDeviceToDevice);
}

extern "C" int scc_graph_upload_csr(scc_graph* g, const int32_t* begin, const int32_t* node_idx,
                                    const int32_t* r_begin, const int32_t* r_node_idx, void* stream) {
    SCC_REQUIRE(g && begin && r_begin && (g->m == 0 || (node_idx && r_node_idx)), SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(g->device));
    cudaStream_t st = (cudaStream_t)stream;
    size_t nb = sizeof(int32_t) * ((size_t)g->n + 1), mb = sizeof(int32_t) * (size_t)g->m;
    g->self_loops = -1;                      // new contents: count again when needed
    SCC_CUDA(cudaMemcpyAsync(g->begin, begin, nb, cudaMemcpyHostToDevice, st));
    SCC_CUDA(cudaMemcpyAsync(g->r_begin, r_begin, nb, cudaMemcpyHostToDevice, st));
    if (g->m > 0) {
        SCC_CUDA(cudaMemcpyAsync(g->node_idx, node_idx, mb, cudaMemcpyHostToDevice, st));
        SCC_CUDA(cudaMemcpyAsync(g->r_node_idx, r_node_idx, mb, cudaMemcpyHostToDevice, st));
    }
    return SCC_OK;
}

// ------------------------------------------------------------------ pipelined upload
// The forward CSR crosses the bus in UPLOAD_RUNS chunks of whole source lists;
// each chunk's (destination, source) pairs are sorted by destination on a
// second stream while the next chunk is in flight.  A chunk's sorted pairs
// form a run; the stable sort keeps sources ascending inside a run and runs
// are in source order, so an in-list is the concatenation of its segments in
// the runs, in run order, which one scatter places.
#define UPLOAD_RUNS 4
#define UPLOAD_PIPELINE_MIN_EDGES (1LL << 22)

struct RunBounds {
    int64_t e[UPLOAD_RUNS + 1];      // edge range of each run
};

// r_begin[v] = sum over runs of the run-local offsets (edges with key < v)
__global__ void k_runs_begin(int32_t n, const int32_t* __restrict__ off, int32_t* __restrict__ r_begin) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v <= n; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t t = 0;
#pragma unroll
        for (int j = 0; j < UPLOAD_RUNS; ++j) t += off[(int64_t)j * (n + 1) + v];
        r_begin[v] = (int32_t)t;
    }
}

// pos = r_begin[v] + (v's edges in earlier runs) + (rank inside this run's segment)
__global__ void k_runs_scatter(int32_t n, RunBounds rb, const int32_t* __restrict__ keys,
                               const int32_t* __restrict__ vals, const int32_t* __restrict__ off,
                               const int32_t* __restrict__ r_begin, int32_t* __restrict__ out) {
    const int64_t m = rb.e[UPLOAD_RUNS];
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        int j = 0;
        while (j + 1 < UPLOAD_RUNS && i >= rb.e[j + 1]) ++j;
        const int32_t v = keys[i];
        int64_t pos = (int64_t)__ldg(r_begin + v) + (i - rb.e[j]) - __ldg(off + (int64_t)j * (n + 1) + v);
        for (int k = 0; k < j; ++k) {
            const int32_t* o = off + (int64_t)k * (n + 1);
            pos += __ldg(o + v + 1) - __ldg(o + v);
        }
        out[pos] = vals[i];
    }
}

// Source id of every edge of vertices [s0, s1): a lane per vertex, and the
// whole warp for a list of more than 32 entries (a warp per vertex spent most
// of its lanes idle on a grid's lists of one or two entries).
__global__ void k_expand_sources_range(int32_t s0, int32_t s1, const int32_t* __restrict__ begin,
                                       int32_t* __restrict__ src) {
    const int lane = threadIdx.x & 31;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t base = s0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x - lane; base < s1; base += stride) {
        const int64_t w = base + lane;             // base is warp-uniform
        int32_t b = 0, e = 0;
        if (w < s1) { b = begin[w]; e = begin[w + 1]; }
        const bool big = e - b > 32;
        if (!big)
            for (int32_t k = b; k < e; ++k) src[k] = (int32_t)w;
        unsigned m = __ballot_sync(0xFFFFFFFFu, big);
        while (m) {
            const int l = __ffs(m) - 1;
            m &= m - 1;
            const int32_t bb = __shfl_sync(0xFFFFFFFFu, b, l), be = __shfl_sync(0xFFFFFFFFu, e, l);
            const int32_t wv = (int32_t)__shfl_sync(0xFFFFFFFFu, (int32_t)w, l);
            for (int32_t k = bb + lane; k < be; k += 32) src[k] = wv;
        }
    }
}

namespace {
struct Events {
    cudaEvent_t ev[UPLOAD_RUNS + 1] = {};
    cudaStream_t cs = nullptr;
    ~Events() {
        for (auto& e : ev) if (e) cudaEventDestroy(e);
        if (cs) cudaStreamDestroy(cs);
    }
};
// Declared after the scratch buffers, so it runs before their frees on the
// caller's stream: that stream first waits for everything queued on the
// helper stream, on the error paths too.
struct JoinOnExit {
    cudaStream_t st;
    Events& evs;
    ~JoinOnExit() {
        if (evs.cs && evs.ev[UPLOAD_RUNS]) {
            cudaEventRecord(evs.ev[UPLOAD_RUNS], evs.cs);
            cudaStreamWaitEvent(st, evs.ev[UPLOAD_RUNS], 0);
        }
    }
};
}  // namespace

static int upload_pipelined(scc_graph* g, const int32_t* begin, const int32_t* node_idx, cudaStream_t st) {
    const int32_t n = g->n;
    const int64_t m = g->m;
    // Run boundaries at whole source lists.  Runs shrink: a run's sort is
    // about 2.5x faster than its transfer, so each sort ends before the next
    // run has landed and only the last, smallest sort (and the scatter) follow
    // the final byte.
    static const int cut_percent[UPLOAD_RUNS - 1] = {45, 75, 92};
    RunBounds rb;
    int64_t biggest = 0;
    int32_t sv[UPLOAD_RUNS + 1];
    sv[0] = 0;
    sv[UPLOAD_RUNS] = n;
    for (int j = 1; j < UPLOAD_RUNS; ++j) {
        const int64_t target = m * cut_percent[j - 1] / 100;
        sv[j] = (int32_t)(std::lower_bound(begin, begin + n + 1, (int32_t)target) - begin);
        if (sv[j] < sv[j - 1]) sv[j] = sv[j - 1];
        if (sv[j] > n) sv[j] = n;
    }
    for (int j = 0; j <= UPLOAD_RUNS; ++j) rb.e[j] = begin[sv[j]];
    for (int j = 0; j < UPLOAD_RUNS; ++j) biggest = std::max<int64_t>(biggest, rb.e[j + 1] - rb.e[j]);
    SCC_REQUIRE(rb.e[UPLOAD_RUNS] == m && rb.e[0] == 0, SCC_ERR_INVALID, "CSR offsets do not run from 0 to m");

    Events evs;
    SCC_CUDA(cudaStreamCreateWithFlags(&evs.cs, cudaStreamNonBlocking));
    for (auto& e : evs.ev) SCC_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    AsyncScratch src(st), keys(st), vals(st), off(st), sort_tmp(st);
    JoinOnExit join{st, evs};
    SCC_CUDA(src.alloc(sizeof(int32_t) * (size_t)m));
    SCC_CUDA(keys.alloc(sizeof(int32_t) * (size_t)m));
    SCC_CUDA(vals.alloc(sizeof(int32_t) * (size_t)m));
    SCC_CUDA(off.alloc(sizeof(int32_t) * (size_t)UPLOAD_RUNS * ((size_t)n + 1)));
    // every scratch buffer is taken before the first copy, so a failed
    // allocation leaves the graph as it was
    SCC_CUDA(sort_tmp.alloc(scc_impl_sort_scratch_bytes(biggest, sizeof(int32_t), true)));
    const int bits = bits_for(n);
    SCC_CUDA(cudaMemcpyAsync(g->begin, begin, sizeof(int32_t) * ((size_t)n + 1), cudaMemcpyHostToDevice, st));
    for (int j = 0; j < UPLOAD_RUNS; ++j) {
        const int64_t e0 = rb.e[j], c = rb.e[j + 1] - e0;
        if (c > 0)
            SCC_CUDA(cudaMemcpyAsync(g->node_idx + e0, node_idx + e0, sizeof(int32_t) * (size_t)c,
                                     cudaMemcpyHostToDevice, st));
        SCC_CUDA(cudaEventRecord(evs.ev[j], st));
    }
    int32_t* offp = (int32_t*)off.p;
    for (int j = 0; j < UPLOAD_RUNS; ++j) {
        const int64_t e0 = rb.e[j], c = rb.e[j + 1] - e0;
        SCC_CUDA(cudaStreamWaitEvent(evs.cs, evs.ev[j], 0));
        int32_t* oj = offp + (int64_t)j * (n + 1);
        if (c == 0) {
            SCC_CUDA(cudaMemsetAsync(oj, 0, sizeof(int32_t) * ((size_t)n + 1), evs.cs));
            continue;
        }
        k_expand_sources_range<<<scc_blocks((int64_t)(sv[j + 1] - sv[j]), 256, 148 * 64), 256, 0, evs.cs>>>(
            sv[j], sv[j + 1], g->begin, (int32_t*)src.p);
        SCC_CUDA(cudaPeekAtLastError());
        SCC_TRY(scc_impl_sort_pairs_u32(reinterpret_cast<const uint32_t*>(g->node_idx + e0), (uint32_t*)keys.p + e0,
                                        (const int32_t*)src.p + e0, (int32_t*)vals.p + e0, c, bits, evs.cs,
                                        sort_tmp.p));
        SCC_CUDA(fill_offsets(c, n, (const int32_t*)keys.p + e0, oj, evs.cs));
    }
    k_runs_begin<<<scc_blocks((int64_t)n + 1, 256, 148 * 64), 256, 0, evs.cs>>>(n, offp, g->r_begin);
    SCC_CUDA(cudaPeekAtLastError());
    k_runs_scatter<<<scc_blocks(m, 256, 148 * 64), 256, 0, evs.cs>>>(n, rb, (const int32_t*)keys.p,
                                                                     (const int32_t*)vals.p, offp, g->r_begin,
                                                                     g->r_node_idx);
    SCC_CUDA(cudaPeekAtLastError());
    return SCC_OK;      // `join` makes the caller's stream resume after the transpose
}

extern "C" int scc_graph_upload_csr_out(scc_graph* g, const int32_t* begin, const int32_t* node_idx, void* stream) {
    SCC_REQUIRE(g && begin && (g->m == 0 || node_idx), SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(g->device));
    cudaStream_t st = (cudaStream_t)stream;
    g->self_loops = -1;                      // new contents: count again when needed
    if (g->m >= UPLOAD_PIPELINE_MIN_EDGES) return upload_pipelined(g, begin, node_idx, st);
    SCC_CUDA(cudaMemcpyAsync(g->begin, begin, sizeof(int32_t) * ((size_t)g->n + 1), cudaMemcpyHostToDevice, st));
    if (g->m > 0)
        SCC_CUDA(cudaMemcpyAsync(g->node_idx, node_idx, sizeof(int32_t) * (size_t)g->m, cudaMemcpyHostToDevice, st));
    return transpose_into(g, st);
}

extern "C" int scc_graph_free(scc_graph* g) {
    if (!g) return SCC_OK;
    cudaSetDevice(g->device);
    if (g->owns) {
        cudaFree(g->begin); cudaFree(g->node_idx); cudaFree(g->r_begin); cudaFree(g->r_node_idx);
    }
    delete g;
    return SCC_OK;
}

extern "C" int scc_graph_num_nodes(const scc_graph* g, int32_t* n) {
    SCC_REQUIRE(g && n, SCC_ERR_INVALID, "NULL argument");
    *n = g->n;
    return SCC_OK;
}

extern "C" int scc_graph_num_edges(const scc_graph* g, int64_t* m) {
    SCC_REQUIRE(g && m, SCC_ERR_INVALID, "NULL argument");
    *m = g->m;
    return SCC_OK;
}

extern "C" int scc_graph_copy_csr(const scc_graph* g, int32_t* begin, int32_t* node_idx, int32_t* r_begin,
                                  int32_t* r_node_idx) {
    SCC_REQUIRE(g, SCC_ERR_INVALID, "graph is NULL");
    SCC_CUDA(cudaSetDevice(g->device));
    size_t nb = sizeof(int32_t) * ((size_t)g->n + 1), mb = sizeof(int32_t) * (size_t)g->m;
    if (begin) SCC_CUDA(cudaMemcpy(begin, g->begin, nb, cudaMemcpyDeviceToHost));
    if (r_begin) SCC_CUDA(cudaMemcpy(r_begin, g->r_begin, nb, cudaMemcpyDeviceToHost));
    if (g->m > 0) {
        if (node_idx) SCC_CUDA(cudaMemcpy(node_idx, g->node_idx, mb, cudaMemcpyDeviceToHost));
        if (r_node_idx) SCC_CUDA(cudaMemcpy(r_node_idx, g->r_node_idx, mb, cudaMemcpyDeviceToHost));
    }
    return SCC_OK;
}

extern "C" int scc_graph_device_csr(const scc_graph* g, const int32_t** d_begin, const int32_t** d_node_idx,
                                    const int32_t** d_r_begin, const int32_t** d_r_node_idx) {
    SCC_REQUIRE(g, SCC_ERR_INVALID, "graph is NULL");
    if (d_begin) *d_begin = g->begin;
    if (d_node_idx) *d_node_idx = g->node_idx;
    if (d_r_begin) *d_r_begin = g->r_begin;
    if (d_r_node_idx) *d_r_node_idx = g->r_node_idx;
    return SCC_OK;
}

// ------------------------------------------------------------------ files
extern "C" int scc_graph_save_binary(const scc_graph* g, const char* path) {
    SCC_REQUIRE(g && path, SCC_ERR_INVALID, "NULL argument");
    std::vector<int32_t> b((size_t)g->n + 1), a((size_t)g->m);
    SCC_TRY(scc_graph_copy_csr(g, b.data(), a.data(), nullptr, nullptr));
    FILE* f = fopen(path, "wb");
    SCC_REQUIRE(f, SCC_ERR_IO, "cannot open %s for writing", path);
    int64_t hdr[2] = {g->n, g->m};
    bool ok = fwrite("SCCCSR01", 1, 8, f) == 8 && fwrite(hdr, sizeof(hdr), 1, f) == 1 &&
              fwrite(b.data(), sizeof(int32_t), b.size(), f) == b.size() &&
              fwrite(a.data(), sizeof(int32_t), a.size(), f) == a.size();
    fclose(f);
    SCC_REQUIRE(ok, SCC_ERR_IO, "short write to %s", path);
    return SCC_OK;
}

extern "C" int scc_graph_load_binary(const char* path, int device, scc_graph** out) {
    SCC_REQUIRE(path && out, SCC_ERR_INVALID, "NULL argument");
    FILE* f = fopen(path, "rb");
    SCC_REQUIRE(f, SCC_ERR_IO, "cannot open %s", path);
    char magic[8];
    int64_t hdr[2];
    if (fread(magic, 1, 8, f) != 8 || memcmp(magic, "SCCCSR01", 8) != 0 || fread(hdr, sizeof(hdr), 1, f) != 1 ||
        hdr[0] < 0 || hdr[1] < 0 || hdr[0] >= SCC_WCC_ROOT_MASK || hdr[1] >= (1LL << 31)) {
        fclose(f);
        scc_set_error("%s is not an SCC binary CSR file", path);
        return SCC_ERR_IO;
    }
    std::vector<int32_t> b((size_t)hdr[0] + 1), a((size_t)hdr[1]);
    bool ok = fread(b.data(), sizeof(int32_t), b.size(), f) == b.size() &&
              fread(a.data(), sizeof(int32_t), a.size(), f) == a.size();
    fclose(f);
    SCC_REQUIRE(ok, SCC_ERR_IO, "truncated file %s", path);
    return scc_graph_create_csr((int32_t)hdr[0], (int32_t)hdr[1], b.data(), a.data(), nullptr, nullptr, device, out);
}

// Fast text parser: "u v" per line, 1-based, stored 0-based; returns the
// largest id, the reference's N (src/common_main.h:61-83,
// src_CUDA/scc_cuda_dynamic.cpp:59-147).
static int parse_edge_list(const char* path, std::vector<int32_t>& src, std::vector<int32_t>& dst, int64_t* max_id) {
    FILE* f = fopen(path, "rb");
    SCC_REQUIRE(f, SCC_ERR_IO, "cannot open %s", path);
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    std::vector<char> buf((size_t)(sz > 0 ? sz : 0) + 1);
    size_t rd = sz > 0 ? fread(buf.data(), 1, (size_t)sz, f) : 0;
    fclose(f);
    buf[rd] = 0;
    int64_t maxid = 0;
    const char* p = buf.data();
    const char* end = p + rd;
    while (p < end) {
        while (p < end && (*p == ' ' || *p == '\t' || *p == '\r' || *p == '\n')) p++;
        if (p >= end) break;
        if (*p == '%' || *p == '#') { while (p < end && *p != '\n') p++; continue; }
        int64_t v[2];
        for (int k = 0; k < 2; ++k) {
            while (p < end && (*p == ' ' || *p == '\t')) p++;
            if (p >= end || *p < '0' || *p > '9') { scc_set_error("%s: malformed line", path); return SCC_ERR_IO; }
            int64_t x = 0;
            while (p < end && *p >= '0' && *p <= '9') { x = x * 10 + (*p - '0'); p++; if (x > 0x7FFFFFFF) break; }
            if (x < 1 || x > 0x1FFFFFFE) { scc_set_error("%s: vertex id %lld out of range", path, (long long)x); return SCC_ERR_IO; }
            v[k] = x;
        }
        while (p < end && *p != '\n') p++;
        src.push_back((int32_t)(v[0] - 1));
        dst.push_back((int32_t)(v[1] - 1));
        if (v[0] > maxid) maxid = v[0];
        if (v[1] > maxid) maxid = v[1];
    }
    *max_id = maxid;
    return SCC_OK;
}

extern "C" int scc_graph_load_edge_list(const char* path, int device, scc_graph** out) {
    SCC_REQUIRE(path && out, SCC_ERR_INVALID, "NULL argument");
    std::vector<int32_t> src, dst;
    int64_t maxid = 0;
    SCC_TRY(parse_edge_list(path, src, dst, &maxid));
    return scc_graph_create_edges((int32_t)maxid, (int64_t)src.size(), src.data(), dst.data(), SCC_BUILD_KEEP_ALL,
                                  device, out);
}

extern "C" int scc_read_edge_list(const char* path, int64_t capacity, int32_t* src, int32_t* dst, int64_t* count,
                                  int32_t* max_id) {
    SCC_REQUIRE(path && count && capacity >= 0, SCC_ERR_INVALID, "bad argument");
    std::vector<int32_t> s, d;
    int64_t maxid = 0;
    SCC_TRY(parse_edge_list(path, s, d, &maxid));
    *count = (int64_t)s.size();
    if (max_id) *max_id = (int32_t)maxid;
    if (capacity > 0) {
        SCC_REQUIRE(src && dst, SCC_ERR_INVALID, "NULL output arrays");
        SCC_REQUIRE(capacity >= (int64_t)s.size(), SCC_ERR_INVALID, "capacity %lld below %lld edges",
                    (long long)capacity, (long long)s.size());
        memcpy(src, s.data(), sizeof(int32_t) * s.size());
        memcpy(dst, d.data(), sizeof(int32_t) * d.size());
    }
    return SCC_OK;
}

// ------------------------------------------------------------------ memory pool
// One pool per device, owned by the library (the device's default pool and
// other libraries' pools are left alone).  Its release threshold keeps freed
// blocks reserved, so repeated uploads and updates reuse them.
static std::mutex g_pool_mu;
static cudaMemPool_t g_pools[64] = {};

static cudaError_t pool_of(int device, cudaMemPool_t* out) {
    if (device < 0 || device >= 64) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_pool_mu);
    if (!g_pools[device]) {
        cudaMemPoolProps props;
        memset(&props, 0, sizeof(props));
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = device;
        cudaError_t e = cudaMemPoolCreate(&g_pools[device], &props);
        if (e != cudaSuccess) { g_pools[device] = nullptr; return e; }
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(g_pools[device], cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
    }
    *out = g_pools[device];
    return cudaSuccess;
}

// Host-side fault injection (scc_debug_inject): the n-th pool allocation from
// now fails; the next asynchronous drain gets one queue slot nobody fills.
static std::atomic<int64_t> g_fail_alloc_in{0};
static std::atomic<int> g_wait_hole{0};

extern "C" int scc_debug_inject(int what, int64_t countdown) {
    SCC_REQUIRE(countdown >= 0, SCC_ERR_INVALID, "countdown %lld", (long long)countdown);
    if (what == SCC_INJECT_ALLOC) { g_fail_alloc_in = countdown; return SCC_OK; }
    if (what == SCC_INJECT_WAIT) { g_wait_hole = countdown > 0 ? 1 : 0; return SCC_OK; }
    scc_set_error("unknown injection %d", what);
    return SCC_ERR_INVALID;
}

bool scc_impl_take_wait_injection() { return g_wait_hole.exchange(0) != 0; }

cudaError_t scc_impl_malloc_async(void** p, size_t bytes, cudaStream_t st) {
    int64_t k = g_fail_alloc_in.load();
    while (k > 0 && !g_fail_alloc_in.compare_exchange_weak(k, k - 1)) {}
    if (k == 1) { *p = nullptr; return cudaErrorMemoryAllocation; }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    cudaMemPool_t pool = nullptr;
    if (e == cudaSuccess) e = pool_of(device, &pool);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync(p, bytes, pool, st);
    return e;
}

extern "C" int scc_release_cached_memory(int device) {
    cudaMemPool_t pool = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_pool_mu);
        if (device < 0 || device >= 64 || !g_pools[device]) return SCC_OK;
        pool = g_pools[device];
    }
    SCC_CUDA(cudaSetDevice(device));
    SCC_CUDA(cudaDeviceSynchronize());
    SCC_CUDA(cudaMemPoolTrimTo(pool, 0));
    return SCC_OK;
}
