// Trim1 and Trim2.
//
// Trim1 (trim_once_node, src/scc_trim1.cc:38-110): a vertex of colour c with
// no out-neighbour or no in-neighbour of colour c (self-loops ignored) is a
// singleton SCC: colour -2, scc = itself.  The reference repeats whole sweeps
// (repeat_global_trim1, scc_trim1.cc:195-209); here one launch peels to the
// fixpoint: a thread that trims x re-checks x's same-colour neighbours right
// away (after a device-scope fence, reading colours from L2) and follows the
// chain on a small per-thread stack; stack overflow and high-degree vertices
// go to an overflow list that the next launch expands one warp per vertex.
// Two threads that each trim one of w's last two live neighbours both fence
// before re-checking w, so at least one sees both trims and peels w: the
// fixpoint is exact.
//
// Trim2 (trim_2nd_new_main, src/scc_trim2_new.cc:45-78): {n,k}, n<k, where n's
// only live out-neighbour (ignoring self-loops and repeats) is k and k's is n,
// or the same on in-edges, is a 2-vertex SCC with scc = n.  Decisions are
// taken on the colours before the pass (a find kernel, then an apply kernel).
#include <algorithm>
#include "scc_internal.cuh"

#define TRIM_STACK 8
#define TRIM_BIG_DEG 512

__device__ __forceinline__ int32_t ld_cg(const int32_t* p) { return __ldcg(p); }

// true if v has a neighbour w != v of colour c in (off, adj).  Four entries
// at a time: their adjacency loads, then their colour loads, are issued
// together (short lists included), so a scan costs two round trips per four
// neighbours; every colour read still follows the caller's fence.
__device__ __forceinline__ bool has_live_nbr(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                             const int32_t* color, int32_t v, int32_t c) {
    int32_t b = __ldg(off + v), e = __ldg(off + v + 1);
    for (int32_t k = b; k < e; k += 4) {
        int32_t w[4], col[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) w[j] = (k + j < e) ? __ldg(adj + k + j) : v;
#pragma unroll
        for (int j = 0; j < 4; ++j) col[j] = (w[j] != v) ? ld_cg(color + w[j]) : SCC_COLOR_DONE;
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if (w[j] != v && col[j] == c) return true;
    }
    return false;
}

__device__ __forceinline__ bool trimmable(const scc_graph& g, const int32_t* color, int32_t v, int32_t c) {
    return !has_live_nbr(g.begin, g.node_idx, color, v, c) || !has_live_nbr(g.r_begin, g.r_node_idx, color, v, c);
}

struct TrimArgs {
    const int32_t* begin; const int32_t* node_idx; const int32_t* r_begin; const int32_t* r_node_idx;
    int32_t* color; int32_t* scc;
    int32_t* ovf; int32_t* ctr;
};

__device__ __forceinline__ scc_graph as_graph(const TrimArgs& a) {
    scc_graph g;
    g.begin = const_cast<int32_t*>(a.begin); g.node_idx = const_cast<int32_t*>(a.node_idx);
    g.r_begin = const_cast<int32_t*>(a.r_begin); g.r_node_idx = const_cast<int32_t*>(a.r_node_idx);
    return g;
}

__device__ __forceinline__ void push_overflow(const TrimArgs& a, int32_t x) {
    int32_t pos = atomicAdd(a.ctr + CTR_OVERFLOW, 1);
    a.ovf[pos] = x;   // each vertex is trimmed once, so the list never exceeds n
}

// Try to trim w (colour c); on success record it.
__device__ __forceinline__ bool try_trim(const TrimArgs& a, const scc_graph& g, int32_t w, int32_t c) {
    if (ld_cg(a.color + w) != c) return false;
    if (!trimmable(g, a.color, w, c)) return false;
    if (atomicCAS(a.color + w, c, SCC_COLOR_DONE) != c) return false;
    a.scc[w] = w;
    __threadfence();
    return true;
}

// Re-check the same-colour neighbours of trimmed x, following chains on a local stack.
__device__ void cascade(const TrimArgs& a, const scc_graph& g, int32_t x0, int32_t c, int32_t& cnt) {
    int32_t stk[TRIM_STACK];
    int sp = 0;
    stk[sp++] = x0;
    while (sp > 0) {
        int32_t x = stk[--sp];
        int32_t d = (__ldg(a.begin + x + 1) - __ldg(a.begin + x)) + (__ldg(a.r_begin + x + 1) - __ldg(a.r_begin + x));
        if (d > TRIM_BIG_DEG) { push_overflow(a, x); continue; }
        for (int pass = 0; pass < 2; ++pass) {
            const int32_t* off = pass ? a.r_begin : a.begin;
            const int32_t* adj = pass ? a.r_node_idx : a.node_idx;
            int32_t b = __ldg(off + x), e = __ldg(off + x + 1);
            for (int32_t k = b; k < e; ++k) {
                int32_t w = __ldg(adj + k);
                if (w == x) continue;
                if (try_trim(a, g, w, c)) {
                    cnt++;
                    if (sp < TRIM_STACK) stk[sp++] = w;
                    else push_overflow(a, w);
                }
            }
        }
    }
}

__device__ __forceinline__ void block_count_add(int32_t* dst, int32_t v) {
    v += __shfl_down_sync(0xFFFFFFFFu, v, 16);
    v += __shfl_down_sync(0xFFFFFFFFu, v, 8);
    v += __shfl_down_sync(0xFFFFFFFFu, v, 4);
    v += __shfl_down_sync(0xFFFFFFFFu, v, 2);
    v += __shfl_down_sync(0xFFFFFFFFu, v, 1);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

// Sweep: candidates are list[i] (or i when list == nullptr).
__global__ void k_trim1_sweep(TrimArgs a, const int32_t* __restrict__ list, int64_t n_items) {
    scc_graph g = as_graph(a);
    int32_t cnt = 0;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t start = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t limit = ((n_items + 31) / 32) * 32;   // keep whole warps for the final reduction
    for (int64_t i = start; i < limit; i += stride) {
        if (i < n_items) {
            int32_t v = list ? list[i] : (int32_t)i;
            int32_t c = ld_cg(a.color + v);
            if (c != SCC_COLOR_DONE && try_trim(a, g, v, c)) {
                cnt++;
                cascade(a, g, v, c, cnt);
            }
        }
    }
    block_count_add(a.ctr + CTR_COUNT, cnt);
}

// First sweep on a fresh state (every colour -1, nothing finished): v starts
// trimmable exactly when one of its sorted adjacency lists is empty or holds
// only v itself (self-loops do not count), which the offsets and the first and
// last entries decide without reading any colour.  Later peels cascade with
// the full colour test.
__device__ __forceinline__ bool has_other_nbr_sorted(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                                     int32_t v) {
    int32_t b = __ldg(off + v), e = __ldg(off + v + 1);
    if (b == e) return false;
    return __ldg(adj + b) != v || __ldg(adj + e - 1) != v;
}

__global__ void k_trim1_fresh(TrimArgs a, int32_t n) {
    scc_graph g = as_graph(a);
    int32_t cnt = 0;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += stride) {
        if (i < n) {
            int32_t v = (int32_t)i;
            if (!has_other_nbr_sorted(a.begin, a.node_idx, v) || !has_other_nbr_sorted(a.r_begin, a.r_node_idx, v)) {
                if (atomicCAS(a.color + v, SCC_COLOR_INIT, SCC_COLOR_DONE) == SCC_COLOR_INIT) {
                    a.scc[v] = v;
                    __threadfence();
                    cnt++;
                    cascade(a, g, v, SCC_COLOR_INIT, cnt);
                }
            }
        }
    }
    block_count_add(a.ctr + CTR_COUNT, cnt);
}

// ------------------------------------------------------------------ counting peel
// On a fresh state every vertex is live and of colour -1, so v's live
// out-neighbour count is its out-degree minus its self-loops (a contiguous run
// in the sorted list), from the offsets alone.  Both counts sit in one 64-bit
// word, (in << 32) | out.  Peeling needs one atomic per edge of a trimmed
// vertex: it decrements one half of the neighbour's word, and the atomic that
// takes the word from "both halves non-zero" to "one half zero" is unique, so
// whoever performs it trims that vertex with plain stores and continues the
// chain from it.  A vertex with a zero count from the start (a seed) never
// makes that transition: the count set-up marks it SEED and the sweep alone
// trims it.  Counts track the live counts exactly (a half is decremented once
// per edge to a trimmed neighbour, so it never borrows), and the result is
// the same fixpoint as the scanning peel.
#define SCC_COLOR_SEED (-3)
#define SCC_COLOR_PREDONE (-4)    // finished before the peel: expanded by the sweep, not trimmed again
#define CNT_NEVER 0x7FFFFFFF7FFFFFFFull   // a finished vertex's counts: no decrement brings a half to zero

__device__ __forceinline__ int32_t self_run(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                            int32_t v) {
    int32_t b = __ldg(off + v), e = __ldg(off + v + 1);
    if (b == e || __ldg(adj + b) > v || __ldg(adj + e - 1) < v) return 0;
    int32_t lo = b, hi = e;                 // first entry >= v
    while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (__ldg(adj + mid) < v) lo = mid + 1; else hi = mid; }
    int32_t first = lo;
    hi = e;                                 // first entry > v
    while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (__ldg(adj + mid) <= v) lo = mid + 1; else hi = mid; }
    return lo - first;
}

// Live-degree counts; the self-loop runs are looked up only when the graph has
// self-loops (graphs built without them skip the adjacency reads entirely).
// prefinished: vertices already finished (colour -2) count as trimmed; the
// sweep expands them, so their live neighbours' counts come out exact.
__global__ void k_count_init(const int32_t* __restrict__ begin, const int32_t* __restrict__ node_idx,
                             const int32_t* __restrict__ r_begin, const int32_t* __restrict__ r_node_idx, int32_t n,
                             int has_self, unsigned long long* __restrict__ cnt, int32_t* __restrict__ color,
                             int prefinished) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = (int32_t)i;
        if (prefinished && color[v] == SCC_COLOR_DONE) {
            cnt[v] = CNT_NEVER;
            color[v] = SCC_COLOR_PREDONE;
            continue;
        }
        int32_t co = __ldg(begin + v + 1) - __ldg(begin + v), ci = __ldg(r_begin + v + 1) - __ldg(r_begin + v);
        if (has_self) {
            co -= self_run(begin, node_idx, v);
            ci -= self_run(r_begin, r_node_idx, v);
        }
        cnt[v] = ((unsigned long long)(uint32_t)ci << 32) | (uint32_t)co;
        if (co == 0 || ci == 0) color[v] = SCC_COLOR_SEED;
    }
}

// Self-loops of the CSR (each appears once in the out-lists).
__global__ void k_count_self(const int32_t* __restrict__ begin, const int32_t* __restrict__ node_idx, int32_t n,
                             unsigned long long* __restrict__ total) {
    unsigned long long c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        c += (unsigned)self_run(begin, node_idx, (int32_t)i);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(total, c);
}

static int count_self_loops(const scc_graph* g, scc_state* s) {
    if (g->self_loops >= 0) return SCC_OK;
    SCC_TRY(scc_zero_counters(s, CTR_EDGES, 2));
    k_count_self<<<scc_blocks(g->n), SCC_THREADS, 0, s->stream>>>(g->begin, g->node_idx, g->n,
                                                                   reinterpret_cast<unsigned long long*>(s->ctr + CTR_EDGES));
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    g->self_loops = (int64_t)*reinterpret_cast<unsigned long long*>(s->h_ctr + CTR_EDGES);
    return SCC_OK;
}

struct CountArgs {
    const int32_t* begin; const int32_t* node_idx; const int32_t* r_begin; const int32_t* r_node_idx;
    int32_t* color; int32_t* scc; unsigned long long* cnt;
    int32_t* ovf; int32_t* ctr;
    int32_t* hub;           // trimmed vertices above PEEL_HUB edges, expanded edge-parallel (count CTR_SPARE3)
    const int32_t* snap;    // coloured peel: the colours before it (a trimmed vertex's class); else unused
};

#define PEEL_Q 256          // per-warp queue of trimmed vertices awaiting expansion
#define PEEL_HUB 4096       // a trimmed vertex with more edges is not expanded by one warp
#define CNT_IN_ONE (1ull << 32)

// One edge of trimmed x: out-edges take an in-neighbour from w, in-edges an
// out-neighbour; returns the neighbour this decrement trims, or -1.  COL: the
// counts are within colours, so only a neighbour still in x's class (cx) is
// decremented -- exactly the edges its count included.
template <bool COL>
__device__ __forceinline__ int32_t peel_edge(const CountArgs& a, int32_t x, int32_t ob, int32_t od, int32_t ib,
                                             int32_t k, int32_t cx) {
    int32_t nv = -1;
    if (k < od) {
        int32_t w = __ldg(a.node_idx + ob + k);
        if (w != x && (!COL || ld_cg(a.color + w) == cx)) {
            unsigned long long old = atomicAdd(a.cnt + w, 0ull - CNT_IN_ONE);
            if ((old >> 32) == 1ull && (uint32_t)old != 0u) nv = w;
        }
    } else {
        int32_t u = __ldg(a.r_node_idx + ib + (k - od));
        if (u != x && (!COL || ld_cg(a.color + u) == cx)) {
            unsigned long long old = atomicAdd(a.cnt + u, 0ull - 1ull);
            if ((uint32_t)old == 1u && (old >> 32) != 0ull) nv = u;
        }
    }
    if (nv >= 0) {
        a.color[nv] = SCC_COLOR_DONE;
        a.scc[nv] = nv;
    }
    return nv;
}

// Expand this warp's queued trimmed vertices, 32 at a time, with their edges
// spread over the lanes (a warp prefix sum of the degrees; each lane finds the
// vertex owning its edge by a binary search over the lanes): every trimmed x
// decrements a count of each neighbour -- out-neighbours lose an in-neighbour,
// in-neighbours an out-neighbour -- so a warp issues 32 independent atomics
// per round trip.  The atomic that zeroes the first half of a word trims that
// neighbour, which joins the queue, or the overflow list when the queue is full.
template <bool COL>
__device__ void peel_drain(const CountArgs& a, int32_t* wq, int32_t& qn, int32_t& cnt) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xFFFFFFFFu;
    while (qn > 0) {
        const int32_t take = min(qn, 32);
        qn -= take;
        const int32_t x = lane < take ? wq[qn + lane] : -1;
        __syncwarp();
        int32_t ob = 0, od = 0, ib = 0, id = 0, cx = 0;
        if (x >= 0) {
            if (COL) cx = a.snap[x];
            ob = __ldg(a.begin + x); od = __ldg(a.begin + x + 1) - ob;
            ib = __ldg(a.r_begin + x); id = __ldg(a.r_begin + x + 1) - ib;
            if (od + id > PEEL_HUB) {
                // one warp would take od + id atomics' round trips: the host
                // expands it over the whole grid instead
                a.hub[atomicAdd(a.ctr + CTR_SPARE3, 1)] = x;
                od = id = 0;
            }
        }
        const int32_t d = od + id;
        int32_t incl = d;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += t;
        }
        const int32_t total = __shfl_sync(full, incl, 31);
        const int32_t excl = incl - d;
        for (int32_t j0 = 0; j0 < total; j0 += 32) {
            const int32_t j = j0 + lane;
            int owner = 0;                                   // largest lane with excl <= j
            for (int step = 16; step > 0; step >>= 1) {
                int cand = owner + step;
                int32_t ev = __shfl_sync(full, excl, cand);
                if (ev <= j) owner = cand;
            }
            const int32_t k = j - __shfl_sync(full, excl, owner);
            const int32_t ox = __shfl_sync(full, x, owner);
            const int32_t oob = __shfl_sync(full, ob, owner), ood = __shfl_sync(full, od, owner);
            const int32_t oib = __shfl_sync(full, ib, owner);
            const int32_t ocx = COL ? __shfl_sync(full, cx, owner) : 0;
            int32_t nv = -1;
            if (j < total) nv = peel_edge<COL>(a, ox, oob, ood, oib, k, ocx);
            const unsigned bal = __ballot_sync(full, nv >= 0);
            if (bal) {
                const int32_t r = __popc(bal & ((1u << lane) - 1u)), nn = __popc(bal);
                if (qn + nn <= PEEL_Q) {
                    if (nv >= 0) wq[qn + r] = nv;
                    qn += nn;
                } else {
                    int32_t base = 0;
                    if (lane == 0) base = atomicAdd(a.ctr + CTR_OVERFLOW, nn);
                    base = __shfl_sync(full, base, 0);
                    if (nv >= 0) a.ovf[base + r] = nv;
                }
                cnt += nv >= 0;
                __syncwarp();
            }
        }
    }
}

// Sweep (items == NULL): every seed is trimmed and expanded.  List (items !=
// NULL): expand trimmed vertices that overflowed a queue, or, with
// trim_items, trim the listed seeds of a coloured peel and expand them.  Each
// warp drains its queue after every 32 vertices.
template <bool COL>
__global__ void __launch_bounds__(SCC_THREADS) k_count_peel(CountArgs a, int32_t n, const int32_t* __restrict__ items,
                                                            int trim_items) {
    __shared__ int32_t queues[SCC_THREADS / 32][PEEL_Q];
    const int lane = threadIdx.x & 31;
    int32_t* wq = queues[threadIdx.x >> 5];
    int32_t qn = 0, cnt = 0;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += nwarps * 32) {
        const int64_t i = base + lane;
        int32_t x = -1;
        if (i < n) {
            if (items) {
                x = items[i];
                if (trim_items) {
                    a.color[x] = SCC_COLOR_DONE;
                    a.scc[x] = x;
                    cnt++;
                }
            } else {
                // only the sweep writes a seed's colour, so a plain read decides
                int32_t v = (int32_t)i;
                const int32_t c = a.color[v];
                if (c == SCC_COLOR_SEED) {
                    a.color[v] = SCC_COLOR_DONE;
                    a.scc[v] = v;
                    x = v;
                    cnt++;
                } else if (c == SCC_COLOR_PREDONE) {     // finished already: expand only
                    a.color[v] = SCC_COLOR_DONE;
                    x = v;
                }
            }
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, x >= 0);
        if (x >= 0) wq[qn + __popc(bal & ((1u << lane) - 1u))] = x;    // qn == 0 here
        qn += __popc(bal);
        __syncwarp();
        peel_drain<COL>(a, wq, qn, cnt);
    }
    block_count_add(a.ctr + CTR_COUNT, cnt);
}

// Inclusive prefix of the hubs' edge counts (one block; hoff[j] = end of hub j).
__global__ void k_hub_prefix(const int32_t* __restrict__ begin, const int32_t* __restrict__ r_begin,
                             const int32_t* __restrict__ hubs, int32_t cnt, long long* __restrict__ hoff) {
    __shared__ long long part[1024];
    int t = threadIdx.x;
    int32_t per = (cnt + 1023) / 1024;
    int32_t b = t * per, e = min(cnt, b + per);
    long long sum = 0;
    for (int32_t j = b; j < e; ++j) {
        int32_t x = hubs[j];
        sum += (long long)(__ldg(begin + x + 1) - __ldg(begin + x)) + (__ldg(r_begin + x + 1) - __ldg(r_begin + x));
    }
    part[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        long long v = (t >= o) ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = (t == 0) ? 0 : part[t - 1];
    for (int32_t j = b; j < e; ++j) {
        int32_t x = hubs[j];
        run += (long long)(__ldg(begin + x + 1) - __ldg(begin + x)) + (__ldg(r_begin + x + 1) - __ldg(r_begin + x));
        hoff[j] = run;
    }
}

// Edge-parallel expansion of trimmed hubs: thread t takes edge t of their
// concatenated lists; trims it causes go to the overflow list, expanded by the
// next list launch of k_count_peel.
template <bool COL>
__global__ void k_hub_peel(CountArgs a, const int32_t* __restrict__ hubs, int32_t cnt,
                           const long long* __restrict__ hoff) {
    const long long total = hoff[cnt - 1];
    int32_t trims = 0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long limit = ((total + 31) / 32) * 32;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < limit; t += stride) {
        int32_t nv = -1;
        if (t < total) {
            int32_t lo = 0, hi = cnt - 1;
            while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (hoff[mid] > t) hi = mid; else lo = mid + 1; }
            const int32_t x = hubs[lo];
            const long long start = lo ? hoff[lo - 1] : 0;
            const int32_t ob = __ldg(a.begin + x), od = __ldg(a.begin + x + 1) - ob, ib = __ldg(a.r_begin + x);
            nv = peel_edge<COL>(a, x, ob, od, ib, (int32_t)(t - start), COL ? a.snap[x] : 0);
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, nv >= 0);
        if (bal) {
            const int lane = threadIdx.x & 31;
            int32_t base = 0;
            if (lane == 0) base = atomicAdd(a.ctr + CTR_OVERFLOW, __popc(bal));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (nv >= 0) a.ovf[base + __popc(bal & ((1u << lane) - 1u))] = nv;
            trims += nv >= 0;
        }
    }
    block_count_add(a.ctr + CTR_COUNT, trims);
}

static int trim1_counting(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    int32_t n = g->n;
    CountArgs a;
    a.begin = g->begin; a.node_idx = g->node_idx; a.r_begin = g->r_begin; a.r_node_idx = g->r_node_idx;
    a.color = s->color; a.scc = s->scc; a.cnt = s->cnt;
    a.ovf = s->qa; a.ctr = s->ctr; a.hub = s->hq; a.snap = nullptr;
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
    SCC_TRY(scc_zero_counters(s, CTR_OVERFLOW, 1));
    SCC_TRY(scc_zero_counters(s, CTR_SPARE3, 1));
    SCC_TRY(count_self_loops(g, s));
    k_count_init<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(g->begin, g->node_idx, g->r_begin, g->r_node_idx, n,
                                                               g->self_loops > 0 ? 1 : 0, s->cnt, s->color,
                                                               s->prefinished ? 1 : 0);
    SCC_LAUNCHED(s);
    k_count_peel<false><<<scc_blocks(n, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(a, n, nullptr, 0);
    SCC_LAUNCHED(s);
    int64_t total = 0;
    // Rounds: overflowed trims are expanded by a list launch, hubs edge-parallel
    // (their trims join the overflow list).  Every vertex is trimmed once, so
    // the lists together never exceed n and the rounds end.
    for (int round = 0;; ++round) {
        SCC_REQUIRE(round < SCC_HOST_ROUND_LIMIT, SCC_ERR_TIMEOUT, "Trim1: no fixpoint after %d rounds", round);
        SCC_TRY(scc_sync_counters(s));
        total += s->h_ctr[CTR_COUNT];
        int32_t novf = s->h_ctr[CTR_OVERFLOW];
        int32_t nhub = s->h_ctr[CTR_SPARE3];
        if (novf == 0 && nhub == 0) break;
        SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
        if (novf > 0)
            SCC_CUDA(cudaMemcpyAsync(s->qb, s->qa, sizeof(int32_t) * (size_t)novf, cudaMemcpyDeviceToDevice, s->stream));
        if (nhub > 0)
            SCC_CUDA(cudaMemcpyAsync(s->aux, s->hq, sizeof(int32_t) * (size_t)nhub, cudaMemcpyDeviceToDevice, s->stream));
        SCC_TRY(scc_zero_counters(s, CTR_OVERFLOW, 1));
        SCC_TRY(scc_zero_counters(s, CTR_SPARE3, 1));
        if (nhub > 0) {
            k_hub_prefix<<<1, 1024, 0, s->stream>>>(g->begin, g->r_begin, s->aux, nhub, s->hoff);
            SCC_LAUNCHED(s);
            k_hub_peel<false><<<148 * 8, SCC_THREADS, 0, s->stream>>>(a, s->aux, nhub, s->hoff);
            SCC_LAUNCHED(s);
        }
        if (novf > 0) {
            k_count_peel<false><<<scc_blocks(novf, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(a, novf, s->qb, 0);
            SCC_LAUNCHED(s);
        }
    }
    *trimmed = (int32_t)total;
    s->cnt_valid = !s->prefinished;      // the residue of finished vertices is not a count
    s->fresh = false;
    s->prefinished = false;
    return SCC_OK;
}

// ---------------------------------------------------------------- coloured counting peel
// Later peels run inside colours over the live list.  The scanning sweep
// re-reads a neighbour's lists at every trim next to it, and its cascades run
// in single threads (a grid's chains of trimmable vertices left 3 lanes of 32
// busy).  Instead, count each live vertex's same-colour in- and out-
// neighbours once, list the vertices with a zero count, and peel with the warp
// queues of the first peel, decrementing only neighbours still in the trimmed
// vertex's class (its colour before the peel is in the snapshot).  The set
// peeled is the same unique fixpoint.
#define CCOUNT_WARP_DEG 64   // a live vertex with more edges is counted by its whole warp
#define CCOUNT_MIN_LIVE 32768   // smaller live lists: one scanning sweep costs less than the extra round trip

__global__ void k_ccount_init(CountArgs a, const int32_t* __restrict__ live, int32_t n_items,
                              int32_t* __restrict__ seeds, int32_t* __restrict__ nseeds) {
    const unsigned full = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n_items;
         base += nwarps * 32) {
        const int64_t i = base + lane;
        int32_t v = 0, c = SCC_COLOR_DONE, ob = 0, oe = 0, ib = 0, ie = 0;
        if (i < n_items) {
            v = live[i];
            c = a.color[v];
            if (c != SCC_COLOR_DONE) {
                ob = __ldg(a.begin + v); oe = __ldg(a.begin + v + 1);
                ib = __ldg(a.r_begin + v); ie = __ldg(a.r_begin + v + 1);
            }
        }
        const bool on = c != SCC_COLOR_DONE;
        const bool wide = on && (oe - ob) + (ie - ib) > CCOUNT_WARP_DEG;
        uint32_t co = 0, ci = 0;
        if (on && !wide) {
            for (int32_t k = ob; k < oe; ++k) { int32_t w = __ldg(a.node_idx + k); co += (w != v && a.color[w] == c); }
            for (int32_t k = ib; k < ie; ++k) { int32_t u = __ldg(a.r_node_idx + k); ci += (u != v && a.color[u] == c); }
        }
        unsigned wm = __ballot_sync(full, wide);
        while (wm) {
            const int l = __ffs(wm) - 1;
            wm &= wm - 1;
            const int32_t lv = __shfl_sync(full, v, l), lc = __shfl_sync(full, c, l);
            const int32_t lob = __shfl_sync(full, ob, l), loe = __shfl_sync(full, oe, l);
            const int32_t lib = __shfl_sync(full, ib, l), lie = __shfl_sync(full, ie, l);
            uint32_t so = 0, si = 0;
            for (int32_t k = lob + lane; k < loe; k += 32) { int32_t w = __ldg(a.node_idx + k); so += (w != lv && a.color[w] == lc); }
            for (int32_t k = lib + lane; k < lie; k += 32) { int32_t u = __ldg(a.r_node_idx + k); si += (u != lv && a.color[u] == lc); }
            so = __reduce_add_sync(full, so);
            si = __reduce_add_sync(full, si);
            if (lane == l) { co = so; ci = si; }
        }
        const bool seed = on && (co == 0 || ci == 0);
        if (on) a.cnt[v] = ((unsigned long long)ci << 32) | co;
        const unsigned sb = __ballot_sync(full, seed);
        if (sb) {
            int32_t at = 0;
            if (lane == 0) at = atomicAdd(nseeds, __popc(sb));
            at = __shfl_sync(full, at, 0);
            if (seed) seeds[at + __popc(sb & ((1u << lane) - 1u))] = v;
        }
    }
}

// Buffers: seeds in qb (read by the first peel launch only), overflow in qa
// (copied to qb for each list launch), hubs in hq (copied to live_tmp), class
// snapshot in aux, counts in the state's own coloured-count array.
__global__ void k_copy_list_i32(const int32_t* __restrict__ list, int64_t n, const int32_t* __restrict__ a,
                                int32_t* __restrict__ b);

static int trim1_coloured(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    const int32_t n_items = s->live_count;
    if (!s->ccnt) SCC_CUDA(cudaMalloc(&s->ccnt, sizeof(unsigned long long) * (size_t)std::max<int32_t>(g->n, 1)));
    CountArgs a;
    a.begin = g->begin; a.node_idx = g->node_idx; a.r_begin = g->r_begin; a.r_node_idx = g->r_node_idx;
    a.color = s->color; a.scc = s->scc; a.cnt = s->ccnt;
    a.ovf = s->qa; a.ctr = s->ctr; a.hub = s->hq; a.snap = s->aux;
    k_copy_list_i32<<<scc_blocks(n_items), SCC_THREADS, 0, s->stream>>>(s->live, n_items, s->color, s->aux);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
    SCC_TRY(scc_zero_counters(s, CTR_OVERFLOW, 1));
    SCC_TRY(scc_zero_counters(s, CTR_SPARE3, 1));
    SCC_TRY(scc_zero_counters(s, CTR_QLEN, 1));
    k_ccount_init<<<scc_blocks(n_items, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(
        a, s->live, n_items, s->qb, s->ctr + CTR_QLEN);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    const int32_t nseeds = s->h_ctr[CTR_QLEN];
    int64_t total = 0;
    if (nseeds > 0) {
        k_count_peel<true><<<scc_blocks(nseeds, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(a, nseeds, s->qb, 1);
        SCC_LAUNCHED(s);
        for (int round = 0;; ++round) {
            SCC_REQUIRE(round < SCC_HOST_ROUND_LIMIT, SCC_ERR_TIMEOUT, "Trim1: no fixpoint after %d rounds", round);
            SCC_TRY(scc_sync_counters(s));
            total += s->h_ctr[CTR_COUNT];
            int32_t novf = s->h_ctr[CTR_OVERFLOW];
            int32_t nhub = s->h_ctr[CTR_SPARE3];
            if (novf == 0 && nhub == 0) break;
            SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
            if (novf > 0)
                SCC_CUDA(cudaMemcpyAsync(s->qb, s->qa, sizeof(int32_t) * (size_t)novf, cudaMemcpyDeviceToDevice, s->stream));
            if (nhub > 0)
                SCC_CUDA(cudaMemcpyAsync(s->live_tmp, s->hq, sizeof(int32_t) * (size_t)nhub, cudaMemcpyDeviceToDevice,
                                         s->stream));
            SCC_TRY(scc_zero_counters(s, CTR_OVERFLOW, 1));
            SCC_TRY(scc_zero_counters(s, CTR_SPARE3, 1));
            if (nhub > 0) {
                k_hub_prefix<<<1, 1024, 0, s->stream>>>(g->begin, g->r_begin, s->live_tmp, nhub, s->hoff);
                SCC_LAUNCHED(s);
                k_hub_peel<true><<<148 * 8, SCC_THREADS, 0, s->stream>>>(a, s->live_tmp, nhub, s->hoff);
                SCC_LAUNCHED(s);
            }
            if (novf > 0) {
                k_count_peel<true><<<scc_blocks(novf, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(a, novf, s->qb, 0);
                SCC_LAUNCHED(s);
            }
        }
    }
    *trimmed = (int32_t)total;
    s->fresh = false;
    s->prefinished = false;
    return SCC_OK;
}

// Overflow expansion: one warp per already-trimmed vertex x, lanes stride its
// neighbours; newly trimmed neighbours cascade per lane.
__global__ void k_trim1_overflow(TrimArgs a, const int32_t* __restrict__ items, int32_t n_items,
                                 const int32_t* __restrict__ item_colors) {
    scc_graph g = as_graph(a);
    int lane = threadIdx.x & 31;
    int32_t cnt = 0;
    int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t wi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; wi < n_items; wi += wstride) {
        int32_t x = items[wi];
        int32_t c = item_colors[wi];
        for (int pass = 0; pass < 2; ++pass) {
            const int32_t* off = pass ? a.r_begin : a.begin;
            const int32_t* adj = pass ? a.r_node_idx : a.node_idx;
            int32_t b = __ldg(off + x), e = __ldg(off + x + 1);
            for (int32_t k = b + lane; k < e; k += 32) {
                int32_t w = __ldg(adj + k);
                if (w != x && try_trim(a, g, w, c)) { cnt++; cascade(a, g, w, c, cnt); }
            }
        }
    }
    block_count_add(a.ctr + CTR_COUNT, cnt);
}

// Edge-parallel overflow expansion (the engine's own peel): thread t takes edge
// t of the overflowed vertices' concatenated out- and in-lists, so a hub's
// neighbours are re-checked by the whole grid instead of one warp.
__global__ void k_ovf_prefix(const int32_t* __restrict__ begin, const int32_t* __restrict__ r_begin,
                             const int32_t* __restrict__ items, int32_t cnt, long long* __restrict__ hoff) {
    __shared__ long long part[1024];
    int t = threadIdx.x;
    int32_t per = (cnt + 1023) / 1024;
    int32_t b = t * per, e = min(cnt, b + per);
    long long sum = 0;
    for (int32_t j = b; j < e; ++j) {
        int32_t x = items[j];
        sum += (long long)(__ldg(begin + x + 1) - __ldg(begin + x)) + (__ldg(r_begin + x + 1) - __ldg(r_begin + x));
    }
    part[t] = sum;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        long long v = (t >= o) ? part[t - o] : 0;
        __syncthreads();
        part[t] += v;
        __syncthreads();
    }
    long long run = (t == 0) ? 0 : part[t - 1];
    for (int32_t j = b; j < e; ++j) {
        int32_t x = items[j];
        run += (long long)(__ldg(begin + x + 1) - __ldg(begin + x)) + (__ldg(r_begin + x + 1) - __ldg(r_begin + x));
        hoff[j] = run;
    }
}

__global__ void k_trim1_overflow_edges(TrimArgs a, const int32_t* __restrict__ items, int32_t n_items,
                                       const int32_t* __restrict__ item_colors, const long long* __restrict__ hoff) {
    scc_graph g = as_graph(a);
    int32_t cnt = 0;
    const long long total = hoff[n_items - 1];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long limit = ((total + 31) / 32) * 32;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < limit; t += stride) {
        if (t < total) {
            int32_t lo = 0, hi = n_items - 1;
            while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (hoff[mid] > t) hi = mid; else lo = mid + 1; }
            const int32_t x = items[lo], c = item_colors[lo];
            const int32_t k = (int32_t)(t - (lo ? hoff[lo - 1] : 0));
            const int32_t ob = __ldg(a.begin + x), od = __ldg(a.begin + x + 1) - ob;
            const int32_t w = k < od ? __ldg(a.node_idx + ob + k) : __ldg(a.r_node_idx + __ldg(a.r_begin + x) + (k - od));
            if (w != x && try_trim(a, g, w, c)) { cnt++; cascade(a, g, w, c, cnt); }
        }
    }
    block_count_add(a.ctr + CTR_COUNT, cnt);
}

// Re-checking an overflowed vertex's neighbours needs the colour it had before
// it was trimmed (the list holds vertices already set to -2): this kernel
// copies it from the snapshot, alongside the list.
__global__ void k_save_colors(const int32_t* __restrict__ items, int32_t n, const int32_t* __restrict__ saved_src,
                              int32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = saved_src[items[i]];
}

__global__ void k_fill_aux(int64_t n, int32_t* __restrict__ b, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = v;
}

// Colour snapshot used to recover the colour a vertex had before it was trimmed.
__global__ void k_copy_i32(int64_t n, const int32_t* __restrict__ a, int32_t* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}
__global__ void k_copy_list_i32(const int32_t* __restrict__ list, int64_t n, const int32_t* __restrict__ a,
                                int32_t* __restrict__ b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = list[i];
        b[v] = a[v];
    }
}

// Peel to the fixpoint over the live list (use_live) or all vertices.
int scc_impl_trim1(const scc_graph* g, scc_state* s, bool use_live, int32_t* trimmed) {
    int64_t n_items = use_live ? s->live_count : g->n;
    const int32_t* list = use_live ? s->live : nullptr;
    *trimmed = 0;
    if (n_items <= 0) return SCC_OK;
    // snapshot colours (aux) so overflowed vertices keep their pre-trim colour
    if ((s->fresh || s->prefinished) && !use_live && s->cnt) return trim1_counting(g, s, trimmed);
    if (use_live && n_items >= CCOUNT_MIN_LIVE) return trim1_coloured(g, s, trimmed);
    s->prefinished = false;
    bool fresh = s->fresh && !use_live;
    if (fresh) {
        // every colour is -1: the snapshot the overflow path reads is that constant
        k_fill_aux<<<scc_blocks(n_items), SCC_THREADS, 0, s->stream>>>(n_items, s->aux, SCC_COLOR_INIT);
    } else if (use_live) {
        k_copy_list_i32<<<scc_blocks(n_items), SCC_THREADS, 0, s->stream>>>(list, n_items, s->color, s->aux);
    } else {
        k_copy_i32<<<scc_blocks(n_items), SCC_THREADS, 0, s->stream>>>(n_items, s->color, s->aux);
    }
    SCC_LAUNCHED(s);
    TrimArgs a;
    a.begin = g->begin; a.node_idx = g->node_idx; a.r_begin = g->r_begin; a.r_node_idx = g->r_node_idx;
    a.color = s->color; a.scc = s->scc; a.ctr = s->ctr;
    a.ovf = s->qa;
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
    SCC_TRY(scc_zero_counters(s, CTR_OVERFLOW, 1));
    if (fresh)
        k_trim1_fresh<<<scc_blocks(n_items, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(a, (int32_t)n_items);
    else
        k_trim1_sweep<<<scc_blocks(n_items, SCC_THREADS, 148 * 8), SCC_THREADS, 0, s->stream>>>(a, list, n_items);
    SCC_LAUNCHED(s);
    s->fresh = false;
    s->prefinished = false;
    int64_t total = 0;
    for (int round = 0;; ++round) {
        SCC_REQUIRE(round < SCC_HOST_ROUND_LIMIT, SCC_ERR_TIMEOUT, "Trim1: no fixpoint after %d rounds", round);
        SCC_TRY(scc_sync_counters(s));
        total += s->h_ctr[CTR_COUNT];
        int32_t novf = s->h_ctr[CTR_OVERFLOW];
        if (novf == 0) break;
        // expand overflowed vertices: move list qa -> qb, colours of items into live_tmp
        SCC_CUDA(cudaMemcpyAsync(s->qb, s->qa, sizeof(int32_t) * (size_t)novf, cudaMemcpyDeviceToDevice, s->stream));
        k_save_colors<<<scc_blocks(novf), SCC_THREADS, 0, s->stream>>>(s->qb, novf, s->aux, s->live_tmp);
        SCC_LAUNCHED(s);
        SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
        SCC_TRY(scc_zero_counters(s, CTR_OVERFLOW, 1));
        k_ovf_prefix<<<1, 1024, 0, s->stream>>>(g->begin, g->r_begin, s->qb, novf, s->hoff);
        SCC_LAUNCHED(s);
        k_trim1_overflow_edges<<<148 * 8, SCC_THREADS, 0, s->stream>>>(a, s->qb, novf, s->live_tmp, s->hoff);
        SCC_LAUNCHED(s);
    }
    *trimmed = (int32_t)total;
    return SCC_OK;
}

// Trim1 to the fixpoint over all n vertices of caller-owned arrays, with every
// scratch buffer supplied by the caller (snapshot, two overflow lists and the
// overflow items' colours: n ints each; ctr: CTR_MAX ints).  It computes the
// same fixpoint as scc_do_global_trim1 with the scanning peel over all
// vertices (k_trim1_sweep, whose cascades overflow to a list expanded a warp
// per item by k_trim1_overflow) rather than the counting peel, which needs the
// state's per-vertex count words; used by the allocation-free entry point.
int scc_trim1_with_scratch(int32_t n, const int32_t* begin, const int32_t* node_idx, const int32_t* r_begin,
                           const int32_t* r_node_idx, int32_t* color, int32_t* scc, int32_t* snapshot,
                           int32_t* ovf_a, int32_t* ovf_b, int32_t* item_colors, int32_t* ctr, cudaStream_t st,
                           int32_t* trimmed) {
    *trimmed = 0;
    if (n <= 0) return SCC_OK;
    int32_t h_ctr[CTR_MAX];
    k_copy_i32<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, color, snapshot);
    SCC_CUDA(cudaPeekAtLastError());
    TrimArgs a;
    a.begin = begin; a.node_idx = node_idx; a.r_begin = r_begin; a.r_node_idx = r_node_idx;
    a.color = color; a.scc = scc; a.ctr = ctr;
    a.ovf = ovf_a;
    SCC_CUDA(cudaMemsetAsync(ctr, 0, sizeof(int32_t) * CTR_MAX, st));
    k_trim1_sweep<<<scc_blocks(n, SCC_THREADS, 148 * 8), SCC_THREADS, 0, st>>>(a, nullptr, n);
    SCC_CUDA(cudaPeekAtLastError());
    int64_t total = 0;
    for (int round = 0;; ++round) {
        SCC_REQUIRE(round < SCC_HOST_ROUND_LIMIT, SCC_ERR_TIMEOUT, "Trim1: no fixpoint after %d rounds", round);
        SCC_CUDA(cudaMemcpyAsync(h_ctr, ctr, sizeof(h_ctr), cudaMemcpyDeviceToHost, st));
        SCC_CUDA(cudaStreamSynchronize(st));
        total += h_ctr[CTR_COUNT];
        int32_t novf = h_ctr[CTR_OVERFLOW];
        if (novf == 0) break;
        SCC_CUDA(cudaMemcpyAsync(ovf_b, ovf_a, sizeof(int32_t) * (size_t)novf, cudaMemcpyDeviceToDevice, st));
        k_save_colors<<<scc_blocks(novf), SCC_THREADS, 0, st>>>(ovf_b, novf, snapshot, item_colors);
        SCC_CUDA(cudaPeekAtLastError());
        SCC_CUDA(cudaMemsetAsync(ctr + CTR_COUNT, 0, sizeof(int32_t), st));
        SCC_CUDA(cudaMemsetAsync(ctr + CTR_OVERFLOW, 0, sizeof(int32_t), st));
        k_trim1_overflow<<<scc_blocks((int64_t)novf * 32, SCC_THREADS, 148 * 8), SCC_THREADS, 0, st>>>(
            a, ovf_b, novf, item_colors);
        SCC_CUDA(cudaPeekAtLastError());
    }
    *trimmed = (int32_t)total;
    return SCC_OK;
}

// ------------------------------------------------------------------ trim2
__device__ __forceinline__ bool degree_is_one(const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                              const int32_t* __restrict__ color, int32_t c, int32_t v, int32_t* nbr) {
    int32_t the = SCC_NIL_NODE;
    int cnt = 0;
    int32_t b = __ldg(off + v), e = __ldg(off + v + 1);
    for (int32_t k = b; k < e; ++k) {
        int32_t w = __ldg(adj + k);
        if (w == v || w == the) continue;   // self edge, repeated edge
        if (color[w] != c) continue;
        cnt++;
        the = w;
        if (cnt == 2) return false;
    }
    *nbr = the;
    return cnt == 1;
}

__global__ void k_trim2_find(const int32_t* __restrict__ begin, const int32_t* __restrict__ node_idx,
                             const int32_t* __restrict__ r_begin, const int32_t* __restrict__ r_node_idx,
                             const int32_t* __restrict__ color, const int32_t* __restrict__ list, int64_t n_items,
                             int32_t* __restrict__ mate) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n_items; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t n = list ? list[i] : (int32_t)i;
        int32_t c = color[n];
        int32_t res = SCC_NIL_NODE;
        if (c != SCC_COLOR_DONE) {
            int32_t k, kk;
            if (degree_is_one(begin, node_idx, color, c, n, &k) && n < k &&
                degree_is_one(begin, node_idx, color, c, k, &kk) && kk == n)
                res = k;
            else if (degree_is_one(r_begin, r_node_idx, color, c, n, &k) && n < k &&
                     degree_is_one(r_begin, r_node_idx, color, c, k, &kk) && kk == n)
                res = k;
        }
        mate[n] = res;
    }
}

__global__ void k_trim2_apply(int32_t* __restrict__ color, int32_t* __restrict__ scc, const int32_t* __restrict__ list,
                              int64_t n_items, const int32_t* __restrict__ mate, int32_t* __restrict__ count) {
    int32_t cnt = 0;
    int64_t limit = ((n_items + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n_items) {
            int32_t n = list ? list[i] : (int32_t)i;
            int32_t k = (color[n] != SCC_COLOR_DONE) ? mate[n] : SCC_NIL_NODE;
            if (k >= 0) {
                color[n] = SCC_COLOR_DONE; color[k] = SCC_COLOR_DONE;
                scc[n] = n; scc[k] = n;
                cnt += 2;
            }
        }
    }
    block_count_add(count, cnt);
}

int scc_impl_trim2(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    *trimmed = 0;
    s->fresh = false;
    s->prefinished = false;
    bool use_live = s->live_count >= 0;
    int64_t n_items = use_live ? s->live_count : g->n;
    const int32_t* list = use_live ? s->live : nullptr;
    if (n_items <= 0) return SCC_OK;
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
    k_trim2_find<<<scc_blocks(n_items), SCC_THREADS, 0, s->stream>>>(g->begin, g->node_idx, g->r_begin, g->r_node_idx,
                                                                    s->color, list, n_items, s->aux);
    SCC_LAUNCHED(s);
    k_trim2_apply<<<scc_blocks(n_items), SCC_THREADS, 0, s->stream>>>(s->color, s->scc, list, n_items, s->aux,
                                                                     s->ctr + CTR_COUNT);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    *trimmed = s->h_ctr[CTR_COUNT];
    return SCC_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int scc_do_global_trim1(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t t = 0;
    SCC_TRY(scc_impl_trim1(g, s, false, &t));
    if (trimmed) *trimmed = t;
    return SCC_OK;
}

extern "C" int scc_do_global_trim1_compact(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t t = 0;
    SCC_TRY(scc_impl_trim1(g, s, s->live_count >= 0, &t));
    if (trimmed) *trimmed = t;
    return SCC_OK;
}

extern "C" int scc_repeat_global_trim1(const scc_graph* g, scc_state* s, int32_t trim_stop, int32_t* trimmed) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    (void)trim_stop;
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t t = 0;
    SCC_TRY(scc_impl_trim1(g, s, false, &t));
    // scc_trim1.cc:203-205: once >= 10% are trimmed the reference continues on
    // the compact list, which leaves trim_targets built.
    if ((double)t >= (double)g->n * 0.1 && g->n > 0) SCC_TRY(scc_impl_compact_live(g, s, s->live_count < 0));
    if (trimmed) *trimmed = t;
    return SCC_OK;
}

extern "C" int scc_repeat_global_trim1_compact(const scc_graph* g, scc_state* s, int32_t trim_stop, int32_t* trimmed) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    (void)trim_stop;
    SCC_CUDA(cudaSetDevice(s->device));
    SCC_TRY(scc_impl_compact_live(g, s, false));
    int32_t t = 0;
    SCC_TRY(scc_impl_trim1(g, s, true, &t));
    if (trimmed) *trimmed = t;
    return SCC_OK;
}

extern "C" int scc_do_global_trim2_new(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t t = 0;
    SCC_TRY(scc_impl_trim2(g, s, &t));
    if (trimmed) *trimmed = t;
    return SCC_OK;
}

extern "C" int scc_do_global_trim2(const scc_graph* g, scc_state* s, int32_t* trimmed) {
    return scc_do_global_trim2_new(g, s, trimmed);
}

extern "C" int scc_repeat_global_trim2_new(const scc_graph* g, scc_state* s, int32_t exit_count, int32_t* trimmed) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    int64_t total = 0;
    for (;;) {
        int32_t t = 0;
        SCC_TRY(scc_impl_trim2(g, s, &t));
        total += t;
        if (t <= exit_count || t == 0) break;
    }
    if (trimmed) *trimmed = (int32_t)total;
    return SCC_OK;
}
