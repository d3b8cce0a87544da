// Batched decomposition of many independent small graphs in ONE persistent
// launch: each block takes whole graphs from a device counter (largest
// first) and runs the complete method on each inside the block -- Trim1 to
// the fixpoint, then rounds of pivot / FW+BW reachability / classify / peel
// over every class of that graph at once (the structure of
// do_baseline_global_wcc_fb and start_workers_fw_bw, src/scc_main.cc:272-351,
// src/scc_fb_seq2.cc:292-351) -- with __syncthreads between the steps instead
// of kernel boundaries and host round trips.  One launch per batch, so the
// run is captured once into a CUDA graph and replayed with one host
// submission.  Blocks never wait on one another.
//
// Per graph g with vertices [lo, hi) the block uses only slices of the
// state's arrays: colour/scc/mark/counts [lo, hi), the queue [2lo, 2hi), the
// live lists [lo, hi).  Colours are globally unique without an allocator:
// the graph starts as one class of colour 3*lo, and the FW-only / BW-only
// parts of the class pivoted on p become 3p+1 / 3p+2 (a pivot is finished in
// its round, so it never pivots again).  The per-colour pivot key lives in an
// array indexed by colour (3N entries).
#include <algorithm>
#include "scc_round.cuh"
#include "scc_batch.cuh"
#include "scc_sort.cuh"

struct BatchArgs {
    const int32_t* begin; const int32_t* adj; const int32_t* rbegin; const int32_t* radj;
    const int32_t* offs;        // [G+1] vertex offsets of the graphs
    const int32_t* order;       // [G] graphs, largest first
    int32_t G;
    int32_t* color; int32_t* scc; uint8_t* mark;
    uint32_t* cin; uint32_t* cout;   // live in/out counts within the class
    int32_t* q;                 // [2N] queue slices
    int32_t* live; int32_t* live2;   // [N] live-list slices
    unsigned long long* key;    // [3N] pivot key per colour
    int32_t* ctr;               // BATCH_CTR_* counters
    int32_t warp_deg;           // lists longer than this are expanded by a whole warp
    const int32_t* members;     // class mode: unit k is members[offs[k] .. offs[k+1]); NULL: vertex ids
};

__device__ __forceinline__ int32_t b_fw_colour(int32_t p) { return 3 * p + 1; }
__device__ __forceinline__ int32_t b_bw_colour(int32_t p) { return 3 * p + 2; }

// Warp-aggregated append of `item` (lanes with p) to q[base + tail++], tail in shared memory.
__device__ __forceinline__ void b_append(bool p, int32_t item, int32_t* q, int32_t* s_tail, int32_t cap,
                                         int32_t* err) {
    unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
    if (!bal) return;
    int lane = threadIdx.x & 31;
    int32_t base = 0;
    if (lane == __ffs(bal) - 1) base = atomicAdd(s_tail, __popc(bal));
    base = __shfl_sync(0xFFFFFFFFu, base, __ffs(bal) - 1);
    if (p) {
        int32_t pos = base + __popc(bal & ((1u << lane) - 1u));
        if (pos < cap) q[pos] = item;
        else atomicExch(err, SCC_DEVERR_QUEUE_OVERFLOW);
    }
}

// Block-wide exclusive scan of one int per thread; returns the prefix, *total the sum.
__device__ __forceinline__ int32_t b_scan(int32_t x, int32_t* s_warp, int32_t* total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    int32_t inc = x;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_warp[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int32_t w = lane < nw ? s_warp[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < nw) s_warp[lane] = w;       // inclusive warp totals
    }
    __syncthreads();
    int32_t before = (wid > 0 ? s_warp[wid - 1] : 0) + inc - x;
    *total = s_warp[nw - 1];
    __syncthreads();
    return before;
}

// ------------------------------------------------------------------ peel
// Counts of same-class neighbours (self-loops excluded) of every live vertex;
// vertices with a zero count are trimmed and queued with their class.
__device__ void b_count_and_seed(const BatchArgs& a, const int32_t* live, int32_t nlive, int32_t* q, int32_t* qc,
                                 int32_t* s_tail, int32_t cap) {
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5, wid = threadIdx.x >> 5;
    for (int32_t base = wid * 32; base < nlive; base += nwarps * 32) {
        int32_t i = base + lane;
        bool valid = i < nlive;
        int32_t v = valid ? live[i] : 0;
        int32_t c = valid ? a.color[v] : SCC_COLOR_DONE;
        uint32_t cnt[2] = {0u, 0u};
        for (int side = 0; side < 2; ++side) {
            const int32_t* off = side ? a.rbegin : a.begin;
            const int32_t* adj = side ? a.radj : a.adj;
            int32_t b = valid ? __ldg(off + v) : 0, e = valid ? __ldg(off + v + 1) : 0;
            int32_t deg = e - b;
            unsigned big = __ballot_sync(0xFFFFFFFFu, deg > a.warp_deg);
            while (big) {
                int l = __ffs(big) - 1;
                big &= big - 1;
                int32_t lb = __shfl_sync(0xFFFFFFFFu, b, l), le = __shfl_sync(0xFFFFFFFFu, e, l);
                int32_t lv = __shfl_sync(0xFFFFFFFFu, v, l), lc = __shfl_sync(0xFFFFFFFFu, c, l);
                uint32_t k = 0;
                for (int32_t j = lb + lane; j < le; j += 32) {
                    int32_t w = __ldg(adj + j);
                    k += (w != lv && a.color[w] == lc) ? 1u : 0u;
                }
                for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xFFFFFFFFu, k, o);
                if (lane == l) cnt[side] = k;
            }
            if (deg <= a.warp_deg && c != SCC_COLOR_DONE) {
                uint32_t k = 0;
                for (int32_t j = b; j < e; ++j) {
                    int32_t w = __ldg(adj + j);
                    k += (w != v && a.color[w] == c) ? 1u : 0u;
                }
                cnt[side] = k;
            }
        }
        if (valid && c != SCC_COLOR_DONE) { a.cout[v] = cnt[0]; a.cin[v] = cnt[1]; }
    }
    __syncthreads();
    for (int32_t base = wid * 32; base < nlive; base += nwarps * 32) {
        int32_t i = base + lane;
        bool p = false;
        int32_t v = 0, c = 0;
        if (i < nlive) {
            v = live[i];
            c = a.color[v];
            if (c != SCC_COLOR_DONE && (a.cin[v] == 0u || a.cout[v] == 0u) && atomicCAS(a.color + v, c, SCC_COLOR_DONE) == c) {
                a.scc[v] = v;
                p = true;
            }
        }
        // the queue holds the vertex; its class goes to the parallel slot
        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
        if (bal) {
            int32_t base2 = 0;
            if (lane == __ffs(bal) - 1) base2 = atomicAdd(s_tail, __popc(bal));
            base2 = __shfl_sync(0xFFFFFFFFu, base2, __ffs(bal) - 1);
            if (p) {
                int32_t pos = base2 + __popc(bal & ((1u << lane) - 1u));
                if (pos < cap) { q[pos] = v; qc[pos] = c; }
                else atomicExch(a.ctr + BATCH_CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW);
            }
        }
    }
    __syncthreads();
}

// The trimmed vertex x (class c) leaves its neighbours' counts; a count that
// reaches zero trims that neighbour (once: the colour CAS decides).
__device__ __forceinline__ bool b_peel_edge(const BatchArgs& a, int32_t w, int32_t x, int32_t c, int side) {
    if (w == x || a.color[w] != c) return false;
    uint32_t* cnt = side ? a.cout : a.cin;     // x's out-edge costs w an in-neighbour, and the reverse
    if (atomicSub(cnt + w, 1u) != 1u) return false;
    if (atomicCAS(a.color + w, c, SCC_COLOR_DONE) != c) return false;
    a.scc[w] = w;
    return true;
}

__device__ void b_peel(const BatchArgs& a, int32_t* q, int32_t* qc, int32_t* s_tail, int32_t cap) {
    const int lane = threadIdx.x & 31;
    const int nwarps = blockDim.x >> 5, wid = threadIdx.x >> 5;
    int32_t h = 0;
    while (true) {
        int32_t t = *s_tail;
        if (t > cap) t = cap;
        if (h >= t) break;
        for (int32_t base = h + wid * 32; base < t; base += nwarps * 32) {
            int32_t i = base + lane;
            bool valid = i < t;
            int32_t x = valid ? q[i] : 0, c = valid ? qc[i] : 0;
            for (int side = 0; side < 2; ++side) {
                const int32_t* off = side ? a.rbegin : a.begin;
                const int32_t* adj = side ? a.radj : a.adj;
                int32_t b = valid ? __ldg(off + x) : 0, e = valid ? __ldg(off + x + 1) : 0;
                int32_t deg = e - b;
                unsigned big = __ballot_sync(0xFFFFFFFFu, deg > a.warp_deg);
                while (big) {
                    int l = __ffs(big) - 1;
                    big &= big - 1;
                    int32_t lb = __shfl_sync(0xFFFFFFFFu, b, l), le = __shfl_sync(0xFFFFFFFFu, e, l);
                    int32_t lx = __shfl_sync(0xFFFFFFFFu, x, l), lc = __shfl_sync(0xFFFFFFFFu, c, l);
                    for (int32_t j0 = lb; j0 < le; j0 += 32) {
                        int32_t j = j0 + lane;
                        int32_t w = j < le ? __ldg(adj + j) : lx;
                        bool p = j < le && b_peel_edge(a, w, lx, lc, side);
                        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
                        if (bal) {
                            int32_t pos0 = 0;
                            if (lane == __ffs(bal) - 1) pos0 = atomicAdd(s_tail, __popc(bal));
                            pos0 = __shfl_sync(0xFFFFFFFFu, pos0, __ffs(bal) - 1);
                            if (p) {
                                int32_t pos = pos0 + __popc(bal & ((1u << lane) - 1u));
                                if (pos < cap) { q[pos] = w; qc[pos] = lc; }
                                else atomicExch(a.ctr + BATCH_CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW);
                            }
                        }
                    }
                }
                if (valid && deg <= a.warp_deg) {
                    for (int32_t j = b; j < e; ++j) {
                        int32_t w = __ldg(adj + j);
                        if (b_peel_edge(a, w, x, c, side)) {
                            int32_t pos = atomicAdd(s_tail, 1);
                            if (pos < cap) { q[pos] = w; qc[pos] = c; }
                            else atomicExch(a.ctr + BATCH_CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW);
                        }
                    }
                }
            }
        }
        h = t;
        __syncthreads();
    }
}

// ------------------------------------------------------------------ one graph
__device__ void b_graph(const BatchArgs& a, int32_t gi, int32_t* s) {
    int32_t* s_tail = s;          // queue tail
    int32_t* s_warp = s + 32;     // scan scratch (32 ints)
    const int32_t lo = a.offs[gi], hi = a.offs[gi + 1];
    const int32_t ng = hi - lo;
    if (ng <= 0) return;
    int32_t* q = a.q + 2LL * lo;          // [2 ng]: peel queue (vertices | classes) or BFS items
    int32_t* live = a.live + lo;
    int32_t* live2 = a.live2 + lo;
    // one class per unit: colour 3 x its first vertex (a multiple of 3, so it
    // never meets the 3p+1 / 3p+2 colours of a pivot's parts)
    const int32_t c0 = 3 * (a.members ? a.members[lo] : lo);
    for (int32_t i = threadIdx.x; i < ng; i += blockDim.x) {
        int32_t v = a.members ? a.members[lo + i] : lo + i;
        a.color[v] = c0;
        a.scc[v] = SCC_NIL_NODE;
        a.mark[v] = 0;
        live[i] = v;
    }
    int32_t nlive = ng;
    int32_t rounds = 0, levels = 0;
    __syncthreads();
    while (true) {
        // peel inside the classes
        if (threadIdx.x == 0) *s_tail = 0;
        __syncthreads();
        b_count_and_seed(a, live, nlive, q, q + ng, s_tail, ng);
        b_peel(a, q, q + ng, s_tail, ng);
        // compact the live list
        int32_t kept = 0;
        for (int32_t base = 0; base < nlive; base += blockDim.x) {
            int32_t i = base + threadIdx.x;
            int32_t v = i < nlive ? live[i] : 0;
            int32_t keep = (i < nlive && a.color[v] != SCC_COLOR_DONE) ? 1 : 0;
            int32_t tot = 0;
            int32_t pos = b_scan(keep, s_warp, &tot);
            if (keep) live2[kept + pos] = v;
            kept += tot;
        }
        { int32_t* t = live; live = live2; live2 = t; }
        nlive = kept;
        __syncthreads();
        if (nlive == 0) break;
        if (++rounds > ng + 2) {
            if (threadIdx.x == 0) atomicExch(a.ctr + BATCH_CTR_ERROR, SCC_DEVERR_WAIT_LIMIT);
            break;
        }
        // pivot of every class: largest in x out degree, ties by the id hash
        for (int32_t i = threadIdx.x; i < nlive; i += blockDim.x) a.key[a.color[live[i]]] = 0ull;
        __syncthreads();
        for (int32_t i = threadIdx.x; i < nlive; i += blockDim.x) {
            int32_t v = live[i];
            atomicMax(a.key + a.color[v], pivot_key(a.begin, a.rbegin, v));
        }
        __syncthreads();
        if (threadIdx.x == 0) *s_tail = 0;
        __syncthreads();
        for (int32_t base = 0; base < nlive; base += blockDim.x) {
            int32_t i = base + threadIdx.x;
            bool p = false;
            int32_t v = 0;
            if (i < nlive) {
                v = live[i];
                if (pivot_unhash((uint32_t)a.key[a.color[v]]) == v) { p = true; a.mark[v] = 3; }
            }
            b_append(p, v, q, s_tail, 2 * ng, a.ctr + BATCH_CTR_ERROR);
            b_append(p, v | (1 << DIR_SHIFT), q, s_tail, 2 * ng, a.ctr + BATCH_CTR_ERROR);
        }
        __syncthreads();
        // FW and BW of every class, level by level
        int32_t h = 0;
        const int lane = threadIdx.x & 31, nwarps = blockDim.x >> 5, wid = threadIdx.x >> 5;
        while (true) {
            int32_t t = min(*s_tail, 2 * ng);
            if (h >= t) break;
            ++levels;
            for (int32_t base = h + wid * 32; base < t; base += nwarps * 32) {
                int32_t i = base + lane;
                bool valid = i < t;
                int32_t it = valid ? q[i] : 0;
                int32_t v = it & ITEM_MASK, dir = (it >> DIR_SHIFT) & 1;
                const int32_t* off = dir ? a.rbegin : a.begin;
                int32_t b = valid ? __ldg(off + v) : 0, e = valid ? __ldg(off + v + 1) : 0;
                int32_t c = valid ? a.color[v] : 0;
                int32_t deg = e - b;
                unsigned big = __ballot_sync(0xFFFFFFFFu, deg > a.warp_deg);
                while (big) {
                    int l = __ffs(big) - 1;
                    big &= big - 1;
                    int32_t lb = __shfl_sync(0xFFFFFFFFu, b, l), le = __shfl_sync(0xFFFFFFFFu, e, l);
                    int32_t lc = __shfl_sync(0xFFFFFFFFu, c, l), ld = __shfl_sync(0xFFFFFFFFu, dir, l);
                    const int32_t* ladj = ld ? a.radj : a.adj;
                    const unsigned bit = 1u << ld;
                    for (int32_t j0 = lb; j0 < le; j0 += 32) {
                        int32_t j = j0 + lane;
                        bool p = false;
                        int32_t w = 0;
                        if (j < le) {
                            w = __ldg(ladj + j);
                            if (!(*(volatile uint8_t*)(a.mark + w) & bit) && a.color[w] == lc) {
                                unsigned sh = (unsigned)(w & 3) * 8u;
                                p = !((atomicOr(reinterpret_cast<unsigned*>(a.mark + (w & ~3)), bit << sh) >> sh) & bit);
                            }
                        }
                        b_append(p, w | (ld << DIR_SHIFT), q, s_tail, 2 * ng, a.ctr + BATCH_CTR_ERROR);
                    }
                }
                int32_t mydeg = (valid && deg <= a.warp_deg) ? deg : 0;
                int32_t maxd = (int32_t)__reduce_max_sync(0xFFFFFFFFu, (unsigned)mydeg);
                const int32_t* adj = dir ? a.radj : a.adj;
                const unsigned bit = 1u << dir;
                for (int32_t j = 0; j < maxd; ++j) {
                    bool p = false;
                    int32_t w = 0;
                    if (j < mydeg) {
                        w = __ldg(adj + b + j);
                        if (!(*(volatile uint8_t*)(a.mark + w) & bit) && a.color[w] == c) {
                            unsigned sh = (unsigned)(w & 3) * 8u;
                            p = !((atomicOr(reinterpret_cast<unsigned*>(a.mark + (w & ~3)), bit << sh) >> sh) & bit);
                        }
                    }
                    b_append(p, w | (dir << DIR_SHIFT), q, s_tail, 2 * ng, a.ctr + BATCH_CTR_ERROR);
                }
            }
            h = t;
            __syncthreads();
        }
        // classify: FW&BW -> SCC of the pivot, FW only / BW only -> the pivot's new classes
        for (int32_t i = threadIdx.x; i < nlive; i += blockDim.x) {
            int32_t v = live[i];
            uint8_t m = a.mark[v];
            if (!m) continue;
            int32_t p = pivot_unhash((uint32_t)a.key[a.color[v]]);
            if (m == 3) { a.scc[v] = p; a.color[v] = SCC_COLOR_DONE; }
            else a.color[v] = (m & 1) ? b_fw_colour(p) : b_bw_colour(p);
            a.mark[v] = 0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        atomicAdd(a.ctr + BATCH_CTR_ROUNDS, rounds);
        atomicAdd(a.ctr + BATCH_CTR_LEVELS, levels);
        atomicMax(a.ctr + BATCH_CTR_MAX_ROUNDS, rounds);
    }
    __syncthreads();
}

__global__ void k_batch_scc(BatchArgs a) {
    __shared__ int32_t s[64];
    __shared__ int32_t s_gi;
    while (true) {
        if (threadIdx.x == 0) {
            // a device error anywhere ends every block (read by one thread, so the block agrees)
            s_gi = *(volatile int32_t*)(a.ctr + BATCH_CTR_ERROR) ? a.G : atomicAdd(a.ctr + BATCH_CTR_NEXT, 1);
        }
        __syncthreads();
        int32_t k = s_gi;
        __syncthreads();
        if (k >= a.G) break;
        b_graph(a, a.order[k], s);
    }
}

// ------------------------------------------------------------------ host side
struct scc_batch_plan {
    const scc_graph* g = nullptr;
    scc_state* s = nullptr;
    int32_t G = 0;
    int32_t* d_offs = nullptr;
    int32_t* d_order = nullptr;
    unsigned long long* d_key = nullptr;
    int32_t* d_live2 = nullptr;
    int32_t* d_ctr = nullptr;
    int32_t* h_ctr = nullptr;
    scc_batch_tuning tune;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev[2];
};

static int batch_enqueue(scc_batch_plan* p, int sms) {
    scc_state* s = p->s;
    const scc_graph* g = p->g;
    BatchArgs a;
    a.begin = g->begin; a.adj = g->node_idx; a.rbegin = g->r_begin; a.radj = g->r_node_idx;
    a.offs = p->d_offs; a.order = p->d_order; a.G = p->G;
    a.color = s->color; a.scc = s->scc; a.mark = s->mark;
    a.cin = reinterpret_cast<uint32_t*>(s->cnt);
    a.cout = reinterpret_cast<uint32_t*>(s->cnt) + s->n;
    a.q = s->qa;
    a.live = s->live; a.live2 = p->d_live2;
    a.key = p->d_key;
    a.ctr = p->d_ctr;
    a.warp_deg = p->tune.warp_deg;
    a.members = nullptr;
    SCC_CUDA(cudaMemsetAsync(p->d_ctr, 0, sizeof(int32_t) * BATCH_CTR_WORDS, s->stream));
    k_batch_scc<<<sms * p->tune.blocks_per_sm, p->tune.threads, 0, s->stream>>>(a);
    SCC_CUDA(cudaPeekAtLastError());
    SCC_CUDA(cudaMemcpyAsync(p->h_ctr, p->d_ctr, sizeof(int32_t) * BATCH_CTR_WORDS, cudaMemcpyDeviceToHost,
                             s->stream));
    return SCC_OK;
}

static void batch_release(scc_batch_plan* p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    cudaFree(p->d_offs); cudaFree(p->d_order); cudaFree(p->d_key); cudaFree(p->d_live2); cudaFree(p->d_ctr);
    if (p->h_ctr) cudaFreeHost(p->h_ctr);
    cudaEventDestroy(p->ev[0]); cudaEventDestroy(p->ev[1]);
    delete p;
}

static bool batch_tuning_ok(const scc_batch_tuning* t) {
    return t->threads >= 64 && t->threads <= 1024 && (t->threads & 31) == 0 && t->blocks_per_sm >= 1 &&
           t->blocks_per_sm <= 8 && t->warp_deg >= 1;
}

extern "C" int scc_batch_default_tuning(scc_batch_tuning* t) {
    SCC_REQUIRE(t, SCC_ERR_INVALID, "NULL argument");
    t->threads = 512;
    t->blocks_per_sm = 2;
    t->warp_deg = 32;
    return SCC_OK;
}

extern "C" int scc_batch_plan_create(const scc_graph* g, scc_state* s, const int32_t* offsets, int32_t num_graphs,
                                     const scc_batch_tuning* tuning, scc_batch_plan** out) {
    SCC_REQUIRE(g && s && offsets && out && num_graphs >= 0, SCC_ERR_INVALID, "bad argument");
    SCC_REQUIRE(s->n == g->n, SCC_ERR_INVALID, "state of another graph");
    SCC_REQUIRE(offsets[0] == 0 && offsets[num_graphs] <= g->n, SCC_ERR_INVALID,
                "offsets must run from 0 to at most the graph's %d vertices", g->n);
    for (int32_t i = 0; i < num_graphs; ++i)
        SCC_REQUIRE(offsets[i + 1] >= offsets[i], SCC_ERR_INVALID, "offsets decrease at graph %d", i);
    SCC_REQUIRE((int64_t)g->n * 3 < (int64_t)INT32_MAX, SCC_ERR_INVALID, "too many vertices for batch colours");
    SCC_CUDA(cudaSetDevice(s->device));
    scc_batch_plan* p = new scc_batch_plan();
    p->g = g; p->s = s; p->G = num_graphs;
    if (tuning) p->tune = *tuning; else scc_batch_default_tuning(&p->tune);
    if (!batch_tuning_ok(&p->tune)) { delete p; scc_set_error("bad batch tuning"); return SCC_ERR_INVALID; }
    cudaEventCreate(&p->ev[0]); cudaEventCreate(&p->ev[1]);
    // graphs by decreasing size: the largest start first, the small ones fill in
    std::vector<int32_t> order((size_t)num_graphs);
    for (int32_t i = 0; i < num_graphs; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
        return offsets[x + 1] - offsets[x] > offsets[y + 1] - offsets[y];
    });
    int rc = SCC_OK;
    int sms = 148;
#define BATCH_TRY(call) do { cudaError_t _e = (call); if (_e != cudaSuccess) { rc = scc_cuda_status(_e, #call, __FILE__, __LINE__); goto fail; } } while (0)
    BATCH_TRY(cudaMalloc(&p->d_offs, sizeof(int32_t) * ((size_t)num_graphs + 1)));
    BATCH_TRY(cudaMalloc(&p->d_order, sizeof(int32_t) * std::max<size_t>(1, (size_t)num_graphs)));
    BATCH_TRY(cudaMalloc(&p->d_key, sizeof(unsigned long long) * (3 * (size_t)std::max(g->n, 1) + 3)));
    BATCH_TRY(cudaMalloc(&p->d_live2, sizeof(int32_t) * (size_t)std::max(g->n, 1)));
    BATCH_TRY(cudaMalloc(&p->d_ctr, sizeof(int32_t) * BATCH_CTR_WORDS));
    BATCH_TRY(cudaMallocHost(&p->h_ctr, sizeof(int32_t) * BATCH_CTR_WORDS));
    BATCH_TRY(cudaMemcpy(p->d_offs, offsets, sizeof(int32_t) * ((size_t)num_graphs + 1), cudaMemcpyHostToDevice));
    if (num_graphs > 0)
        BATCH_TRY(cudaMemcpy(p->d_order, order.data(), sizeof(int32_t) * (size_t)num_graphs, cudaMemcpyHostToDevice));
    // the whole run -- counter reset, the persistent launch, counters back --
    // captured once; every run is one graph launch
    BATCH_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    BATCH_TRY(cudaStreamSynchronize(s->stream));
    BATCH_TRY(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    rc = batch_enqueue(p, sms);
    {
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
        if (rc != SCC_OK) { if (graph) cudaGraphDestroy(graph); goto fail; }
        BATCH_TRY(e);
        p->graph = graph;
    }
    BATCH_TRY(cudaGraphInstantiate(&p->exec, p->graph, 0));
#undef BATCH_TRY
    *out = p;
    return SCC_OK;
fail:
    batch_release(p);
    return rc;
}

extern "C" int scc_batch_plan_run(scc_batch_plan* p, scc_batch_stats* stats) {
    SCC_REQUIRE(p, SCC_ERR_INVALID, "NULL plan");
    scc_state* s = p->s;
    SCC_CUDA(cudaSetDevice(s->device));
    SCC_CUDA(cudaEventRecord(p->ev[0], s->stream));
    SCC_CUDA(cudaGraphLaunch(p->exec, s->stream));
    SCC_CUDA(cudaEventRecord(p->ev[1], s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    SCC_CUDA(cudaEventElapsedTime(&ms, p->ev[0], p->ev[1]));
    s->live_count = -1;      // the live list slices no longer describe the whole graph
    s->fresh = false;
    s->prefinished = false;
    s->cnt_valid = false;
    if (p->h_ctr[BATCH_CTR_ERROR]) {
        scc_set_error("batched run: device error %d", p->h_ctr[BATCH_CTR_ERROR]);
        return p->h_ctr[BATCH_CTR_ERROR] == SCC_DEVERR_WAIT_LIMIT ? SCC_ERR_TIMEOUT : SCC_ERR_OOM;
    }
    if (stats) {
        stats->ms_total = ms;
        stats->graphs = p->G;
        stats->rounds = p->h_ctr[BATCH_CTR_ROUNDS];
        stats->levels = p->h_ctr[BATCH_CTR_LEVELS];
        stats->max_rounds = p->h_ctr[BATCH_CTR_MAX_ROUNDS];
        stats->host_submissions = 1;
        stats->kernels = 1;
    }
    return SCC_OK;
}

extern "C" int scc_batch_plan_free(scc_batch_plan* p) {
    if (!p) return SCC_OK;
    cudaSetDevice(p->s->device);
    batch_release(p);
    return SCC_OK;
}

// ------------------------------------------------------------------ autotuner
// Successive halving: every candidate runs on the first eighth of the graphs
// (ids are in generation order, so a prefix is a fair sample of the sizes),
// the faster half goes on to a quarter, then half, then the whole batch.
static int batch_time(const scc_graph* g, scc_state* s, const int32_t* offsets, int32_t k,
                      const scc_batch_tuning& t, double* ms) {
    scc_batch_plan* p = nullptr;
    SCC_TRY(scc_batch_plan_create(g, s, offsets, k, &t, &p));
    scc_batch_stats st;
    int rc = scc_batch_plan_run(p, &st);            // warm-up
    if (rc == SCC_OK) rc = scc_batch_plan_run(p, &st);
    *ms = st.ms_total;
    scc_batch_plan_free(p);
    return rc;
}

extern "C" int scc_batch_autotune(const scc_graph* g, scc_state* s, const int32_t* offsets, int32_t num_graphs,
                                  scc_batch_tuning* best, double* best_ms) {
    SCC_REQUIRE(g && s && offsets && num_graphs > 0, SCC_ERR_INVALID, "bad argument");
    std::vector<scc_batch_tuning> cand;
    const int32_t threads[] = {256, 512, 1024};
    const int32_t per_sm[] = {1, 2, 4};
    const int32_t warp_deg[] = {8, 16, 32, 64};
    for (int32_t t : threads)
        for (int32_t b : per_sm)
            for (int32_t w : warp_deg)
                if (t * b <= 2048) cand.push_back(scc_batch_tuning{t, b, w});
    std::vector<double> ms(cand.size());
    for (int stage = 3; stage >= 0; --stage) {
        int32_t k = std::max<int32_t>(1, num_graphs >> stage);
        for (size_t i = 0; i < cand.size(); ++i) SCC_TRY(batch_time(g, s, offsets, k, cand[i], &ms[i]));
        std::vector<size_t> idx(cand.size());
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return ms[x] < ms[y]; });
        size_t keep = stage > 0 ? std::max<size_t>(1, (cand.size() + 1) / 2) : 1;
        std::vector<scc_batch_tuning> next;
        std::vector<double> next_ms;
        for (size_t i = 0; i < keep; ++i) { next.push_back(cand[idx[i]]); next_ms.push_back(ms[idx[i]]); }
        cand.swap(next);
        ms.swap(next_ms);
    }
    if (best) *best = cand[0];
    if (best_ms) *best_ms = ms[0];
    return SCC_OK;
}

// ------------------------------------------------------------------ the recursion's tail
// Once few vertices are left (tail_live), every remaining class is an
// independent subproblem: the live vertices are grouped by class (a stable
// sort of (colour, vertex)), and one persistent launch decomposes each class
// inside a block, as for a batch of graphs, instead of further rounds of many
// launches and host round trips.  Classes are unions of SCCs, so the labels
// are the same.  Skipped (nothing done) when a class is larger than
// tail_class, which one block would take too long to finish alone.
__global__ void k_tail_keys(const int32_t* __restrict__ live, int32_t nl, const int32_t* __restrict__ color,
                            uint32_t* __restrict__ keys) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nl; i += (int64_t)gridDim.x * blockDim.x)
        keys[i] = (uint32_t)color[live[i]];
}

int scc_impl_resolve_tail(const scc_graph* g, scc_state* s, bool* taken) {
    *taken = false;
    const int32_t nl = s->live_count;
    if (nl <= 0) return SCC_OK;
    cudaStream_t st = s->stream;
    struct Pool {
        cudaStream_t st;
        std::vector<void*> v;
        ~Pool() { for (void* p : v) cudaFreeAsync(p, st); }
        cudaError_t get(void** p, size_t b) { cudaError_t e = scc_impl_malloc_async(p, b, st); if (e == cudaSuccess) v.push_back(*p); return e; }
    } pool{st, {}};
    uint32_t *keys = nullptr, *skeys = nullptr;
    int32_t *members = nullptr, *starts = nullptr, *order = nullptr, *ctr = nullptr;
    SCC_CUDA(pool.get((void**)&keys, sizeof(uint32_t) * (size_t)nl));
    SCC_CUDA(pool.get((void**)&skeys, sizeof(uint32_t) * (size_t)nl));
    SCC_CUDA(pool.get((void**)&members, sizeof(int32_t) * (size_t)nl));
    SCC_CUDA(pool.get((void**)&starts, sizeof(int32_t) * ((size_t)nl + 1)));
    k_tail_keys<<<scc_blocks(nl), SCC_THREADS, 0, st>>>(s->live, nl, s->color, keys);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_impl_sort_pairs_u32(keys, skeys, s->live, members, nl, 32, st));
    int64_t G = 0;
    SCC_TRY(scc_impl_segment_starts(skeys, nl, starts, &G, st));
    std::vector<int32_t> h((size_t)G + 1);
    SCC_CUDA(cudaMemcpyAsync(h.data(), starts, sizeof(int32_t) * (size_t)G, cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    h[(size_t)G] = nl;
    int32_t biggest = 0;
    for (int64_t k = 0; k < G; ++k) biggest = std::max(biggest, h[(size_t)k + 1] - h[(size_t)k]);
    if (biggest > s->tune.tail_class) return SCC_OK;
    std::vector<int32_t> ord((size_t)G);
    for (int64_t k = 0; k < G; ++k) ord[(size_t)k] = (int32_t)k;
    std::stable_sort(ord.begin(), ord.end(), [&](int32_t x, int32_t y) { return h[x + 1] - h[x] > h[y + 1] - h[y]; });
    if (!s->bkey) SCC_CUDA(cudaMalloc(&s->bkey, sizeof(unsigned long long) * (3 * (size_t)std::max(s->n, 1) + 3)));
    SCC_CUDA(pool.get((void**)&order, sizeof(int32_t) * (size_t)std::max<int64_t>(G, 1)));
    SCC_CUDA(pool.get((void**)&ctr, sizeof(int32_t) * BATCH_CTR_WORDS));
    SCC_CUDA(cudaMemcpyAsync(starts + G, &nl, sizeof(int32_t), cudaMemcpyHostToDevice, st));
    SCC_CUDA(cudaMemcpyAsync(order, ord.data(), sizeof(int32_t) * (size_t)G, cudaMemcpyHostToDevice, st));
    SCC_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int32_t) * BATCH_CTR_WORDS, st));
    BatchArgs a;
    a.begin = g->begin; a.adj = g->node_idx; a.rbegin = g->r_begin; a.radj = g->r_node_idx;
    a.offs = starts; a.order = order; a.G = (int32_t)G;
    a.color = s->color; a.scc = s->scc; a.mark = s->mark;
    a.cin = reinterpret_cast<uint32_t*>(s->cnt);
    a.cout = reinterpret_cast<uint32_t*>(s->cnt) + s->n;
    a.q = s->qa;
    a.live = s->live; a.live2 = s->live_tmp;
    a.key = s->bkey;
    a.ctr = ctr;
    a.warp_deg = 32;
    a.members = members;
    int sms = 148;
    SCC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device));
    k_batch_scc<<<sms * 2, 512, 0, st>>>(a);
    SCC_LAUNCHED(s);
    int32_t h_ctr[BATCH_CTR_WORDS];
    SCC_CUDA(cudaMemcpyAsync(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    if (h_ctr[BATCH_CTR_ERROR]) {
        scc_set_error("tail decomposition: device error %d", h_ctr[BATCH_CTR_ERROR]);
        return h_ctr[BATCH_CTR_ERROR] == SCC_DEVERR_WAIT_LIMIT ? SCC_ERR_TIMEOUT : SCC_ERR_OOM;
    }
    s->fb_rounds += h_ctr[BATCH_CTR_MAX_ROUNDS];
    s->cnt_valid = false;
    s->live_count = 0;
    *taken = true;
    if (scc_trace_on())
        fprintf(stderr, "[scc] tail: %d live vertices in %lld classes (largest %d) in one launch, up to %d rounds\n", nl,
                (long long)G, biggest, h_ctr[BATCH_CTR_MAX_ROUNDS]);
    return SCC_OK;
}
