// State (G_Color / G_SCC and the phase globals), counters, and order-preserving
// compaction of the live vertex list (create_trim1_compact, src/scc_trim1.cc:211-275).
#include <algorithm>
#include <string.h>
#include "scc_internal.cuh"

// ------------------------------------------------------------------ kernels
__global__ void k_fill_i32(int64_t n, int32_t* __restrict__ a, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

// Compaction predicate modes
#define CMP_ALL_LIVE   0   // v in [0,n): color[v] != -2
#define CMP_LIST_LIVE  1   // v = list[i]: color[v] != -2
#define CMP_ALL_COLOR  2   // v in [0,n): color[v] == c
#define CMP_LIST_COLOR 3   // v = list[i]: color[v] == c

#define CMP_TILE 2048      // elements per block (256 threads x 8)

template <int MODE>
__device__ __forceinline__ bool cmp_pred(int64_t i, const int32_t* __restrict__ list, const int32_t* __restrict__ color,
                                         int32_t c, int32_t* v_out) {
    int32_t v = (MODE == CMP_ALL_LIVE || MODE == CMP_ALL_COLOR) ? (int32_t)i : list[i];
    *v_out = v;
    int32_t col = color[v];
    return (MODE == CMP_ALL_LIVE || MODE == CMP_LIST_LIVE) ? (col != SCC_COLOR_DONE) : (col == c);
}

// Pass 1: per-tile counts (ballot/popc per warp, summed per block).
template <int MODE>
__global__ void k_compact_count(int64_t n, const int32_t* __restrict__ list, const int32_t* __restrict__ color,
                                int32_t c, int32_t* __restrict__ tile_counts) {
    __shared__ int32_t warp_tot[SCC_THREADS / 32];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t base = (int64_t)blockIdx.x * CMP_TILE;
    int32_t tot = 0;
    for (int j = 0; j < CMP_TILE / SCC_THREADS; ++j) {
        int64_t i = base + (int64_t)j * SCC_THREADS + threadIdx.x;
        int32_t v;
        bool p = (i < n) && cmp_pred<MODE>(i, list, color, c, &v);
        tot += __popc(__ballot_sync(0xFFFFFFFFu, p));
    }
    if (lane == 0) warp_tot[wid] = tot;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t s = 0;
        for (int w = 0; w < SCC_THREADS / 32; ++w) s += warp_tot[w];
        tile_counts[blockIdx.x] = s;
    }
}

// Exclusive scan of tile counts by one block; total -> *total.
__global__ void k_scan_tiles(int32_t ntiles, int32_t* __restrict__ tile_counts, int32_t* __restrict__ total) {
    __shared__ int32_t part[1024];
    int t = threadIdx.x;
    int32_t per = (ntiles + 1023) / 1024;
    int32_t b = t * per, e = min(ntiles, b + per);
    int32_t s = 0;
    for (int32_t i = b; i < e; ++i) s += tile_counts[i];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        int32_t x = (t >= off) ? part[t - off] : 0;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    int32_t run = (t == 0) ? 0 : part[t - 1];
    for (int32_t i = b; i < e; ++i) { int32_t x = tile_counts[i]; tile_counts[i] = run; run += x; }
    if (t == 1023) *total = part[1023];
}

// Pass 2: write survivors in order.  Within a block the order is
// (j-slab, warp, lane), which is ascending index order.
template <int MODE>
__global__ void k_compact_write(int64_t n, const int32_t* __restrict__ list, const int32_t* __restrict__ color,
                                int32_t c, const int32_t* __restrict__ tile_offsets, int32_t* __restrict__ out) {
    __shared__ int32_t warp_cnt[SCC_THREADS / 32];
    __shared__ int32_t warp_off[SCC_THREADS / 32];
    __shared__ int32_t slab_base;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t base = (int64_t)blockIdx.x * CMP_TILE;
    if (threadIdx.x == 0) slab_base = tile_offsets[blockIdx.x];
    __syncthreads();
    for (int j = 0; j < CMP_TILE / SCC_THREADS; ++j) {
        int64_t i = base + (int64_t)j * SCC_THREADS + threadIdx.x;
        int32_t v = 0;
        bool p = (i < n) && cmp_pred<MODE>(i, list, color, c, &v);
        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
        if (lane == 0) warp_cnt[wid] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t s = slab_base;
            for (int w = 0; w < SCC_THREADS / 32; ++w) { warp_off[w] = s; s += warp_cnt[w]; }
            slab_base = s;
        }
        __syncthreads();
        if (p) out[warp_off[wid] + __popc(bal & ((1u << lane) - 1u))] = v;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ host helpers
int scc_sync_counters(scc_state* s) {
    SCC_CUDA(cudaMemcpyAsync(s->h_ctr, s->ctr, sizeof(int32_t) * CTR_MAX, cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}

int scc_zero_counters(scc_state* s, int first, int count) {
    SCC_CUDA(cudaMemsetAsync(s->ctr + first, 0, sizeof(int32_t) * count, s->stream));
    return SCC_OK;
}

int scc_check_device_error(scc_state* s) {
    SCC_TRY(scc_sync_counters(s));
    int e = s->h_ctr[CTR_ERROR];
    if (e == 0) return SCC_OK;
    int info = s->h_ctr[CTR_ERROR_INFO];
    SCC_CUDA(cudaMemsetAsync(s->ctr + CTR_ERROR, 0, sizeof(int32_t) * 2, s->stream));
    if (e == SCC_DEVERR_WAIT_LIMIT) {
        scc_set_error("bounded device wait gave up (site %d)", info);
        return SCC_ERR_TIMEOUT;
    }
    scc_set_error("device capacity error %d (info %d)", e, info);
    return SCC_ERR_OOM;
}

// Generic compaction into `out`; returns count through *count (synchronises).
template <int MODE>
static int compact(scc_state* s, int64_t n_items, const int32_t* list, int32_t c, int32_t* out, int32_t* count) {
    if (n_items <= 0) { *count = 0; return SCC_OK; }
    int64_t tiles = (n_items + CMP_TILE - 1) / CMP_TILE;
    k_compact_count<MODE><<<(unsigned)tiles, SCC_THREADS, 0, s->stream>>>(n_items, list, s->color, c, s->block_sums);
    SCC_LAUNCHED(s);
    k_scan_tiles<<<1, 1024, 0, s->stream>>>((int32_t)tiles, s->block_sums, s->ctr + CTR_QLEN2);
    SCC_LAUNCHED(s);
    k_compact_write<MODE><<<(unsigned)tiles, SCC_THREADS, 0, s->stream>>>(n_items, list, s->color, c, s->block_sums, out);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    *count = s->h_ctr[CTR_QLEN2];
    return SCC_OK;
}

// create_trim1_compact (scc_trim1.cc:266-275): from all vertices when no list
// exists yet (create_trim1_compact_1), else from the current list (_1b).
int scc_impl_compact_live(const scc_graph* g, scc_state* s, bool from_all) {
    int32_t cnt = 0;
    if (from_all || s->live_count < 0) {
        SCC_TRY(compact<CMP_ALL_LIVE>(s, g->n, nullptr, 0, s->live, &cnt));
    } else {
        SCC_TRY(compact<CMP_LIST_LIVE>(s, s->live_count, s->live, 0, s->live_tmp, &cnt));
        std::swap(s->live, s->live_tmp);
    }
    s->live_count = cnt;
    return SCC_OK;
}

int scc_impl_get_live_host(scc_state* s, std::vector<int32_t>& out) {
    if (s->live_count < 0) { out.clear(); return SCC_OK; }
    out.resize((size_t)s->live_count);
    if (s->live_count > 0)
        SCC_CUDA(cudaMemcpyAsync(out.data(), s->live, sizeof(int32_t) * (size_t)s->live_count,
                                 cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}

int scc_impl_count_colour(scc_state* s, int32_t color, int32_t* count) {
    // members of `color` among the live list if it exists, else among all vertices
    int32_t* tmp = s->live_tmp;
    if (s->live_count >= 0) return compact<CMP_LIST_COLOR>(s, s->live_count, s->live, color, tmp, count);
    return compact<CMP_ALL_COLOR>(s, s->n, nullptr, color, tmp, count);
}

int scc_impl_ensure_colour_cap(scc_state* s, int64_t need) {
    if (need <= s->colour_cap) return SCC_OK;
    int64_t cap = std::max<int64_t>(need, s->colour_cap * 2);
    cap = std::max<int64_t>(cap, 1024);
    cudaFree(s->slot_key); cudaFree(s->slot_pivot); cudaFree(s->slot_fw); cudaFree(s->slot_bw); cudaFree(s->slot_count);
    s->slot_key = nullptr; s->slot_pivot = s->slot_fw = s->slot_bw = s->slot_count = nullptr;
    SCC_CUDA(cudaMalloc(&s->slot_key, sizeof(unsigned long long) * cap));
    SCC_CUDA(cudaMalloc(&s->slot_pivot, sizeof(int32_t) * cap));
    SCC_CUDA(cudaMalloc(&s->slot_fw, sizeof(int32_t) * cap));
    SCC_CUDA(cudaMalloc(&s->slot_bw, sizeof(int32_t) * cap));
    SCC_CUDA(cudaMalloc(&s->slot_count, sizeof(int32_t) * cap));
    s->colour_cap = cap;
    return SCC_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int scc_state_reset(scc_state* s) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    SCC_CUDA(cudaSetDevice(s->device));
    int64_t n = s->n;
    if (n > 0) {
        k_fill_i32<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, s->color, SCC_COLOR_INIT);
        SCC_LAUNCHED(s);
        k_fill_i32<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, s->scc, SCC_NIL_NODE);
        SCC_LAUNCHED(s);
        k_fill_i32<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, s->wcc, SCC_NIL_NODE);
        SCC_LAUNCHED(s);
    }
    SCC_CUDA(cudaMemsetAsync(s->mark, 0, (size_t)((n + 4) & ~3LL), s->stream));
    SCC_CUDA(cudaMemsetAsync(s->ctr, 0, sizeof(int32_t) * CTR_MAX, s->stream));
    int32_t minus1 = -1;
    SCC_CUDA(cudaMemcpyAsync(s->ctr + CTR_NEXT_COLOR, &minus1, sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    s->live_count = -1;
    s->fresh = true;
    s->prefinished = false;
    s->cnt_valid = false;
    s->wq_colors.clear();
    s->wq_counts.clear();
    s->kernels = 0;
    s->traversal_steps = 0;
    return SCC_OK;
}

extern "C" int scc_state_free(scc_state* s) {
    if (!s) return SCC_OK;
    cudaSetDevice(s->device);
    cudaFree(s->color); cudaFree(s->scc); cudaFree(s->wcc); cudaFree(s->live); cudaFree(s->live_tmp);
    cudaFree(s->qa); cudaFree(s->qb); cudaFree(s->aq); cudaFree(s->uf); cudaFree(s->hq); cudaFree(s->hoff); cudaFree(s->cnt); cudaFree(s->ccnt); cudaFree(s->mark); cudaFree(s->aux); cudaFree(s->block_sums);
    cudaFree(s->tq); cudaFree(s->tctr); cudaFree(s->bkey);
    cudaFree(s->ctr);
    if (s->h_ctr) cudaFreeHost(s->h_ctr);
    cudaFree(s->slot_key); cudaFree(s->slot_pivot); cudaFree(s->slot_fw); cudaFree(s->slot_bw); cudaFree(s->slot_count);
    scc_impl_pivot_release(s);
    if (s->events) {
        for (int i = 0; i < 16; ++i) cudaEventDestroy(s->ev[i]);
        for (int i = 0; i < 2; ++i) cudaEventDestroy(s->lev[i]);
    }
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return SCC_OK;
}

extern "C" int scc_state_create(const scc_graph* g, scc_state** out) {
    SCC_REQUIRE(g && out, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(g->device));
    scc_state* s = new scc_state();
    s->device = g->device;
    s->n = g->n;
    int64_t n = g->n;
    size_t nb = sizeof(int32_t) * (size_t)(n > 0 ? n : 1);
    size_t qb = sizeof(int32_t) * (size_t)(2 * n + 64);
    int64_t tiles = (n + CMP_TILE - 1) / CMP_TILE + 1;
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&s->color, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->scc, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->wcc, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->live, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->live_tmp, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->aux, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->qa, qb);
    if (e == cudaSuccess) e = cudaMalloc(&s->qb, qb);
    if (e == cudaSuccess) e = cudaMalloc(&s->aq, qb);
    if (e == cudaSuccess) e = cudaMalloc(&s->uf, nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->cnt, 2 * nb);
    if (e == cudaSuccess) e = cudaMalloc(&s->hq, qb);
    if (e == cudaSuccess) e = cudaMalloc(&s->hoff, sizeof(long long) * (size_t)(2 * n + 64));
    if (e == cudaSuccess) e = cudaMemset(s->aq, 0xFF, qb);
    if (e == cudaSuccess) e = cudaMalloc(&s->mark, (size_t)((n + 4) & ~3LL) + 4);
    if (e == cudaSuccess) e = cudaMalloc(&s->block_sums, sizeof(int32_t) * (size_t)tiles);
    if (e == cudaSuccess) e = cudaMalloc(&s->ctr, sizeof(int32_t) * CTR_MAX);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_ctr, sizeof(int32_t) * CTR_MAX);
    if (e == cudaSuccess) {
        for (int i = 0; i < 16 && e == cudaSuccess; ++i) e = cudaEventCreate(&s->ev[i]);
        for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaEventCreate(&s->lev[i]);
        s->events = (e == cudaSuccess);
    }
    if (e != cudaSuccess) {
        int st = scc_cuda_status(e, "scc_state_create", __FILE__, __LINE__);
        scc_state_free(s);
        return st;
    }
    int st = scc_impl_ensure_colour_cap(s, 3 * n + 1024);
    if (st == SCC_OK) st = scc_state_reset(s);
    if (st != SCC_OK) { scc_state_free(s); return st; }
    *out = s;
    return SCC_OK;
}

extern "C" int scc_state_get_tuning(scc_state* s, scc_tuning* t) {
    SCC_REQUIRE(s && t, SCC_ERR_INVALID, "NULL argument");
    *t = s->tune;
    return SCC_OK;
}

extern "C" int scc_state_set_tuning(scc_state* s, const scc_tuning* t) {
    SCC_REQUIRE(s && t, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(t->async_keep <= 192, SCC_ERR_INVALID, "async_keep %d above 192", t->async_keep);
    SCC_REQUIRE(t->async_blocks_per_sm <= 8, SCC_ERR_INVALID, "async_blocks_per_sm %d above 8", t->async_blocks_per_sm);
    if (t->bu_alpha > 0) s->tune.bu_alpha = t->bu_alpha;
    if (t->bu_div > 0) s->tune.bu_div = t->bu_div;
    if (t->async_max > 0) s->tune.async_max = t->async_max;
    if (t->async_after > 0) s->tune.async_after = t->async_after;
    if (t->async_keep > 0) s->tune.async_keep = t->async_keep;
    if (t->async_blocks_per_sm > 0) s->tune.async_blocks_per_sm = t->async_blocks_per_sm;
    if (t->huge_deg > 0) s->tune.huge_deg = t->huge_deg;
    if (t->tile_min_live != 0) s->tune.tile_min_live = t->tile_min_live > 0 ? t->tile_min_live : -1;
    if (t->tile_min_span > 0) s->tune.tile_min_span = t->tile_min_span;
    if (t->pivot_salt != 0) s->tune.pivot_salt = t->pivot_salt == -1 ? 0 : t->pivot_salt;
    if (t->tail_live != 0) s->tune.tail_live = t->tail_live > 0 ? t->tail_live : -1;
    if (t->tail_class > 0) s->tune.tail_class = t->tail_class;
    if (t->cta_deg != 0) s->tune.cta_deg = t->cta_deg > 0 ? t->cta_deg : -1;
    return SCC_OK;
}

extern "C" int scc_state_profile(scc_state* s, int enable) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    s->ledger_on = enable != 0;
    s->ledger_ms = 0.0;
    s->ledger_launches = s->ledger_items = s->ledger_edges = 0;
    return SCC_OK;
}

extern "C" int scc_state_profile_read(scc_state* s, double* ms, int64_t* launches, int64_t* items, int64_t* edges) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    if (ms) *ms = s->ledger_ms;
    if (launches) *launches = s->ledger_launches;
    if (items) *items = s->ledger_items;
    if (edges) *edges = s->ledger_edges;
    return SCC_OK;
}

extern "C" int scc_state_synchronize(scc_state* s) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}

extern "C" int scc_state_stream(scc_state* s, void** stream) {
    SCC_REQUIRE(s && stream, SCC_ERR_INVALID, "NULL argument");
    *stream = (void*)s->stream;
    return SCC_OK;
}

static int copy_out(scc_state* s, int32_t* host, const int32_t* dev) {
    SCC_REQUIRE(s && host, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    if (s->n > 0) SCC_CUDA(cudaMemcpyAsync(host, dev, sizeof(int32_t) * (size_t)s->n, cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}
static int copy_in(scc_state* s, int32_t* dev, const int32_t* host) {
    SCC_REQUIRE(s && host, SCC_ERR_INVALID, "NULL argument");
    s->fresh = false;
    s->prefinished = false;
    SCC_CUDA(cudaSetDevice(s->device));
    if (s->n > 0) SCC_CUDA(cudaMemcpyAsync(dev, host, sizeof(int32_t) * (size_t)s->n, cudaMemcpyHostToDevice, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}

extern "C" int scc_state_get_color(scc_state* s, int32_t* color) { return copy_out(s, color, s ? s->color : nullptr); }
extern "C" int scc_state_get_scc(scc_state* s, int32_t* scc) { return copy_out(s, scc, s ? s->scc : nullptr); }
extern "C" int scc_state_get_wcc(scc_state* s, int32_t* wcc) { return copy_out(s, wcc, s ? s->wcc : nullptr); }
extern "C" int scc_state_set_color(scc_state* s, const int32_t* color) { return copy_in(s, s ? s->color : nullptr, color); }
extern "C" int scc_state_set_scc(scc_state* s, const int32_t* scc) { return copy_in(s, s ? s->scc : nullptr, scc); }

extern "C" int scc_state_get_trim_targets(scc_state* s, int32_t* out, int32_t capacity, int32_t* count) {
    SCC_REQUIRE(s && count, SCC_ERR_INVALID, "NULL argument");
    int32_t c = s->live_count < 0 ? 0 : s->live_count;
    *count = c;
    if (out && c > 0) {
        SCC_REQUIRE(capacity >= c, SCC_ERR_INVALID, "capacity %d < %d targets", capacity, c);
        SCC_CUDA(cudaMemcpyAsync(out, s->live, sizeof(int32_t) * (size_t)c, cudaMemcpyDeviceToHost, s->stream));
        SCC_CUDA(cudaStreamSynchronize(s->stream));
    }
    return SCC_OK;
}

extern "C" int scc_state_device_arrays(scc_state* s, int32_t** d_color, int32_t** d_scc) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    if (d_color) *d_color = s->color;
    if (d_scc) *d_scc = s->scc;
    return SCC_OK;
}

// get_new_color (src/scc_color.cc:38-54): single caller, so colours come out
// 0, 1, 2, ... exactly as the reference's thread 0 hands them out.
extern "C" int scc_get_new_color(scc_state* s, int32_t* color) {
    SCC_REQUIRE(s && color, SCC_ERR_INVALID, "NULL argument");
    SCC_TRY(scc_sync_counters(s));
    int32_t c = s->h_ctr[CTR_NEXT_COLOR] + 1;
    SCC_CUDA(cudaMemcpyAsync(s->ctr + CTR_NEXT_COLOR, &c, sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    *color = c;
    return SCC_OK;
}

// get_curr_color (src/scc_color.cc:56-61): the last colour handed out (-1 initially).
extern "C" int scc_get_curr_color(scc_state* s, int32_t* color) {
    SCC_REQUIRE(s && color, SCC_ERR_INVALID, "NULL argument");
    SCC_TRY(scc_sync_counters(s));
    *color = s->h_ctr[CTR_NEXT_COLOR];
    return SCC_OK;
}

extern "C" int scc_create_trim1_compact(const scc_graph* g, scc_state* s, int32_t* live_count) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    SCC_TRY(scc_impl_compact_live(g, s, false));
    if (live_count) *live_count = s->live_count;
    return SCC_OK;
}

extern "C" int scc_generate_compact_set(const scc_graph* g, scc_state* s, int32_t color, int32_t* out,
                                        int32_t capacity, int32_t* count) {
    SCC_REQUIRE(g && s && count, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t c = 0;
    SCC_TRY(scc_impl_count_colour(s, color, &c));
    *count = c;
    if (out && c > 0) {
        SCC_REQUIRE(capacity >= c, SCC_ERR_INVALID, "capacity %d < %d members", capacity, c);
        SCC_CUDA(cudaMemcpyAsync(out, s->live_tmp, sizeof(int32_t) * (size_t)c, cudaMemcpyDeviceToHost, s->stream));
        SCC_CUDA(cudaStreamSynchronize(s->stream));
    }
    return SCC_OK;
}
