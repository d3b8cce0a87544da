// WCC colouring (src/scc_weak.cc).
//
// do_global_wcc (scc_weak.cc:128-196): every live vertex t starts with the raw
// label t, or t|0x20000000 when its out-degree is >= 50 (:137-149);
// propagate_color (:65-125) repeats { label = min over same-colour
// out-neighbours; one pointer-jump hop } until nothing changes, so each label
// ends as the smallest raw value over the same-colour vertices reachable from
// t.  Every root (label & 0x1FFFFFFF == t) gets a new colour and its members
// copy it.  The classes are unions of SCCs, since vertices of one SCC reach
// the same set.
//
// Here the propagation is in place (atomicMin, so no update is lost) with the
// pointer jump in the same pass; roots are numbered in ascending vertex order
// so the colouring is deterministic.
#include "scc_internal.cuh"

__global__ void k_wcc_init(const int32_t* __restrict__ begin, const int32_t* __restrict__ live, int32_t n_items,
                           const int32_t* __restrict__ color, int32_t* __restrict__ wcc) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_items; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t t = live[i];
        if (color[t] == SCC_COLOR_DONE) { wcc[t] = SCC_NIL_NODE; continue; }
        int32_t deg = __ldg(begin + t + 1) - __ldg(begin + t);
        wcc[t] = (deg >= SCC_WCC_HIGH_DEG) ? (t | SCC_WCC_HIGH_DEG_FLAG) : t;
    }
}

__global__ void k_wcc_propagate(const int32_t* __restrict__ begin, const int32_t* __restrict__ node_idx,
                                const int32_t* __restrict__ live, int32_t n_items, const int32_t* __restrict__ color,
                                int32_t* __restrict__ wcc, int32_t* __restrict__ changed) {
    int any = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_items; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t t = live[i];
        int32_t c = __ldg(color + t);
        if (c == SCC_COLOR_DONE) continue;
        int32_t cur = __ldcg(wcc + t);
        int32_t mn = cur;
        int32_t b = __ldg(begin + t), e = __ldg(begin + t + 1);
        for (int32_t k = b; k < e; ++k) {
            int32_t w = __ldg(node_idx + k);
            if (__ldg(color + w) != c) continue;
            int32_t x = __ldcg(wcc + w);
            mn = min(mn, x);
        }
        // pointer jump (scc_weak.cc:107-118): label of the label's owner
        int32_t r = mn & SCC_WCC_ROOT_MASK;
        if (r != t) mn = min(mn, __ldcg(wcc + r));
        if (mn < cur) { atomicMin(wcc + t, mn); any = 1; }
    }
    if (__any_sync(0xFFFFFFFFu, any) && (threadIdx.x & 31) == 0) atomicExch(changed, 1);
}

__device__ __forceinline__ bool is_root(const int32_t* wcc, const int32_t* color, int32_t t) {
    return color[t] != SCC_COLOR_DONE && (wcc[t] & SCC_WCC_ROOT_MASK) == t;
}

// Roots in ascending order get colours base+rank: per-tile counts, scan, write.
#define WCC_TILE 2048
__global__ void k_root_count(const int32_t* __restrict__ live, int32_t n_items, const int32_t* __restrict__ color,
                             const int32_t* __restrict__ wcc, int32_t* __restrict__ tile_counts) {
    __shared__ int32_t wt[SCC_THREADS / 32];
    int64_t base = (int64_t)blockIdx.x * WCC_TILE;
    int32_t tot = 0;
    for (int j = 0; j < WCC_TILE / SCC_THREADS; ++j) {
        int64_t i = base + (int64_t)j * SCC_THREADS + threadIdx.x;
        bool p = i < n_items && is_root(wcc, color, live[i]);
        tot += __popc(__ballot_sync(0xFFFFFFFFu, p));
    }
    if ((threadIdx.x & 31) == 0) wt[threadIdx.x >> 5] = tot;
    __syncthreads();
    if (threadIdx.x == 0) {
        int32_t s = 0;
        for (int w = 0; w < SCC_THREADS / 32; ++w) s += wt[w];
        tile_counts[blockIdx.x] = s;
    }
}

__global__ void k_scan_tiles_wcc(int32_t ntiles, int32_t* __restrict__ tile_counts, int32_t* __restrict__ total) {
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

__global__ void k_root_color(const int32_t* __restrict__ live, int32_t n_items, int32_t* __restrict__ color,
                             const int32_t* __restrict__ wcc, const int32_t* __restrict__ tile_offsets,
                             int32_t first_color) {
    __shared__ int32_t wc[SCC_THREADS / 32];
    __shared__ int32_t wo[SCC_THREADS / 32];
    __shared__ int32_t slab;
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int64_t base = (int64_t)blockIdx.x * WCC_TILE;
    if (threadIdx.x == 0) slab = tile_offsets[blockIdx.x];
    __syncthreads();
    for (int j = 0; j < WCC_TILE / SCC_THREADS; ++j) {
        int64_t i = base + (int64_t)j * SCC_THREADS + threadIdx.x;
        int32_t t = i < n_items ? live[i] : 0;
        bool p = i < n_items && is_root(wcc, color, t);
        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
        if (lane == 0) wc[wid] = __popc(bal);
        __syncthreads();
        if (threadIdx.x == 0) {
            int32_t s = slab;
            for (int w = 0; w < SCC_THREADS / 32; ++w) { wo[w] = s; s += wc[w]; }
            slab = s;
        }
        __syncthreads();
        if (p) color[t] = first_color + wo[wid] + __popc(bal & ((1u << lane) - 1u));
        __syncthreads();
    }
}

// Members copy their root's colour (scc_weak.cc:465-473).  Roots were
// recoloured first, so a member is recognised by wcc root != itself.
__global__ void k_member_color(const int32_t* __restrict__ live, int32_t n_items, int32_t* __restrict__ color,
                               const int32_t* __restrict__ wcc) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_items; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t t = live[i];
        if (color[t] == SCC_COLOR_DONE) continue;
        int32_t r = wcc[t] & SCC_WCC_ROOT_MASK;
        if (r != t) color[t] = color[r];
    }
}

int scc_impl_wcc(const scc_graph* g, scc_state* s) {
    s->fresh = false;
    s->prefinished = false;
    if (s->live_count < 0) SCC_TRY(scc_impl_compact_live(g, s, true));
    int32_t n_items = s->live_count;
    if (n_items <= 0) return SCC_OK;
    unsigned blocks = scc_blocks(n_items);
    k_wcc_init<<<blocks, SCC_THREADS, 0, s->stream>>>(g->begin, s->live, n_items, s->color, s->wcc);
    SCC_LAUNCHED(s);
    for (int it = 0; it < (1 << 30); ++it) {
        SCC_TRY(scc_zero_counters(s, CTR_CHANGED, 1));
        k_wcc_propagate<<<blocks, SCC_THREADS, 0, s->stream>>>(g->begin, g->node_idx, s->live, n_items, s->color,
                                                               s->wcc, s->ctr + CTR_CHANGED);
        SCC_LAUNCHED(s);
        s->traversal_steps++;
        SCC_TRY(scc_sync_counters(s));
        if (!s->h_ctr[CTR_CHANGED]) break;
    }
    int32_t first = s->h_ctr[CTR_NEXT_COLOR] + 1;
    int64_t tiles = ((int64_t)n_items + WCC_TILE - 1) / WCC_TILE;
    k_root_count<<<(unsigned)tiles, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->wcc, s->block_sums);
    SCC_LAUNCHED(s);
    k_scan_tiles_wcc<<<1, 1024, 0, s->stream>>>((int32_t)tiles, s->block_sums, s->ctr + CTR_NUM_CLASSES);
    SCC_LAUNCHED(s);
    k_root_color<<<(unsigned)tiles, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->wcc, s->block_sums,
                                                                first);
    SCC_LAUNCHED(s);
    k_member_color<<<blocks, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->wcc);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    int32_t roots = s->h_ctr[CTR_NUM_CLASSES];
    int32_t last = first + roots - 1;
    SCC_CUDA(cudaMemcpyAsync(s->ctr + CTR_NEXT_COLOR, &last, sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    SCC_TRY(scc_impl_ensure_colour_cap(s, (int64_t)last + 2LL * n_items + 1024));
    return SCC_OK;
}

// ------------------------------------------------------------------ weak-component split
// Union-find over the live same-colour edges: every live vertex ends with
// uf[v] = the root of its weakly connected component inside its colour (the
// member of largest uf_rank).
// Components are unions of SCCs, so they are valid independent classes, and
// hooking converges in a few passes whatever the diameter (min-reach label
// propagation above needs O(diameter) passes on grids and long cycles).
__device__ __forceinline__ int32_t uf_find(int32_t* __restrict__ uf, int32_t x) {
    int32_t p = __ldcg(uf + x);
    while (p != x) {
        int32_t gp = __ldcg(uf + p);
        if (gp != p) uf[x] = gp;   // path halving; any ancestor is a valid parent
        x = p;
        p = gp;
    }
    return x;
}

// Roots are linked in the order of a bijective hash of their ids, not of the
// ids themselves: on a row-major grid, lowest-id linking chains parents along
// the rows and every find walks those chains.  Any total order keeps the
// concurrent linking acyclic, and the final root of a component is its
// vertex of largest hash whatever order the unions run in.
__device__ __forceinline__ uint32_t uf_rank(int32_t x) {
    uint32_t h = (uint32_t)x * 0x9E3779B1u;
    return h ^ (h >> 16);
}

__device__ __forceinline__ void uf_union(int32_t* __restrict__ uf, int32_t a, int32_t b) {
    for (;;) {
        a = uf_find(uf, a);
        b = uf_find(uf, b);
        if (a == b) return;
        int32_t lo = uf_rank(a) < uf_rank(b) ? a : b, hi = lo == a ? b : a;
        if (atomicCAS(uf + lo, lo, hi) == lo) return;
        a = lo; b = hi;
    }
}

__global__ void k_uf_init(const int32_t* __restrict__ live, int32_t n_items, int32_t* __restrict__ uf) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_items; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = live[i];
        uf[v] = v;
    }
}

// One warp per 32 live vertices; high-degree vertices are walked by the whole warp.
__global__ void k_uf_hook(const int32_t* __restrict__ begin, const int32_t* __restrict__ node_idx,
                          const int32_t* __restrict__ live, int32_t n_items, const int32_t* __restrict__ color,
                          int32_t* __restrict__ uf) {
    int lane = threadIdx.x & 31;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int64_t groups = ((int64_t)n_items + 31) >> 5;
    for (int64_t gi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; gi < groups; gi += nwarps) {
        int64_t idx = gi * 32 + lane;
        int32_t v = 0, b = 0, e = 0, c = SCC_COLOR_DONE;
        if (idx < n_items) {
            v = live[idx];
            c = __ldg(color + v);
            if (c != SCC_COLOR_DONE) { b = __ldg(begin + v); e = __ldg(begin + v + 1); }
        }
        int32_t deg = e - b;
        unsigned big = __ballot_sync(0xFFFFFFFFu, deg > 32);
        while (big) {
            int l = __ffs(big) - 1;
            big &= big - 1;
            int32_t bv = __shfl_sync(0xFFFFFFFFu, v, l), bb = __shfl_sync(0xFFFFFFFFu, b, l);
            int32_t be = __shfl_sync(0xFFFFFFFFu, e, l), bc = __shfl_sync(0xFFFFFFFFu, c, l);
            for (int32_t k = bb + lane; k < be; k += 32) {
                int32_t w = __ldg(node_idx + k);
                if (w != bv && __ldg(color + w) == bc) uf_union(uf, bv, w);
            }
        }
        if (deg <= 32) {
            // four neighbours' adjacency entries, then their colours, loaded together
            for (int32_t k = b; k < e; k += 4) {
                int32_t w[4], col[4];
#pragma unroll
                for (int j = 0; j < 4; ++j) w[j] = (k + j < e) ? __ldg(node_idx + k + j) : v;
#pragma unroll
                for (int j = 0; j < 4; ++j) col[j] = (w[j] != v) ? __ldg(color + w[j]) : SCC_COLOR_DONE;
#pragma unroll
                for (int j = 0; j < 4; ++j)
                    if (w[j] != v && col[j] == c) uf_union(uf, v, w[j]);
            }
        }
    }
}

__global__ void k_uf_flatten(const int32_t* __restrict__ live, int32_t n_items, const int32_t* __restrict__ color,
                             int32_t* __restrict__ uf, int32_t* __restrict__ label) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_items; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = live[i];
        if (color[v] == SCC_COLOR_DONE) continue;
        label[v] = uf_find(uf, v);
    }
}

// Recolour every live vertex by its weak component: roots (uf == itself) take
// colours 0..k-1 in ascending vertex order, members copy their root's colour.
// The colour counter restarts at k-1: all earlier colours of live vertices are
// overwritten, so colour ids stay below n.
int scc_impl_uf_split(const scc_graph* g, scc_state* s, int32_t* num_classes) {
    s->fresh = false;
    s->prefinished = false;
    int32_t n_items = s->live_count;
    *num_classes = 0;
    if (n_items <= 0) return SCC_OK;
    unsigned blocks = scc_blocks(n_items);
    k_uf_init<<<blocks, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->uf);
    SCC_LAUNCHED(s);
    k_uf_hook<<<scc_blocks(n_items, SCC_THREADS, 148 * 16), SCC_THREADS, 0, s->stream>>>(
        g->begin, g->node_idx, s->live, n_items, s->color, s->uf);
    SCC_LAUNCHED(s);
    k_uf_flatten<<<blocks, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->uf, s->wcc);
    SCC_LAUNCHED(s);
    int64_t tiles = ((int64_t)n_items + WCC_TILE - 1) / WCC_TILE;
    k_root_count<<<(unsigned)tiles, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->wcc, s->block_sums);
    SCC_LAUNCHED(s);
    k_scan_tiles_wcc<<<1, 1024, 0, s->stream>>>((int32_t)tiles, s->block_sums, s->ctr + CTR_NUM_CLASSES);
    SCC_LAUNCHED(s);
    k_root_color<<<(unsigned)tiles, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->wcc, s->block_sums, 0);
    SCC_LAUNCHED(s);
    k_member_color<<<blocks, SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->wcc);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    int32_t k = s->h_ctr[CTR_NUM_CLASSES];
    int32_t last = k - 1;
    SCC_CUDA(cudaMemcpyAsync(s->ctr + CTR_NEXT_COLOR, &last, sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
    s->h_ctr[CTR_NEXT_COLOR] = last;     // the host mirror stays current for the next round
    *num_classes = k;
    return SCC_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int scc_do_global_wcc(const scc_graph* g, scc_state* s) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    s->wq_colors.clear();
    s->wq_counts.clear();
    return scc_impl_wcc(g, s);
}

// create_work_items_from_wcc (scc_weak.cc:198-271): one item per root with its
// member count, in ascending root order.
extern "C" int scc_create_work_items_from_wcc(const scc_graph* g, scc_state* s, int32_t* num_items) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    std::vector<int32_t> live, col((size_t)s->n), w((size_t)s->n);
    SCC_TRY(scc_impl_get_live_host(s, live));
    SCC_TRY(scc_state_get_color(s, col.data()));
    SCC_TRY(scc_state_get_wcc(s, w.data()));
    s->wq_colors.clear();
    s->wq_counts.clear();
    std::vector<int32_t> idx_of_root;
    // roots ascending -> item index; counts via colour lookup
    std::vector<int64_t> slot;
    int32_t cmin = INT32_MAX, cmax = INT32_MIN;
    for (int32_t t : live) if (col[t] != SCC_COLOR_DONE) { cmin = std::min(cmin, col[t]); cmax = std::max(cmax, col[t]); }
    if (cmin <= cmax) {
        std::vector<int32_t> cnt((size_t)(cmax - cmin + 1), 0);
        for (int32_t t : live) if (col[t] != SCC_COLOR_DONE) cnt[(size_t)(col[t] - cmin)]++;
        for (int32_t t : live) {
            if (col[t] == SCC_COLOR_DONE) continue;
            if ((w[t] & SCC_WCC_ROOT_MASK) == t) {
                s->wq_colors.push_back(col[t]);
                s->wq_counts.push_back(cnt[(size_t)(col[t] - cmin)]);
            }
        }
    }
    if (num_items) *num_items = (int32_t)s->wq_colors.size();
    return SCC_OK;
}
