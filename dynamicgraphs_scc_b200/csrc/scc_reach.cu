// Forward/backward reachability inside colour classes, the traversal under
// every FW-BW step (fw_trim_global / bw_trim_global, src/scc_fb_global.cc:32-130,
// and the per-item searches of src/scc_fb_seq2.cc:10-177).
//
// Items are (vertex | direction << 30); direction 0 walks out-edges (FW),
// 1 walks in-edges (BW).  A vertex is claimed once per direction with an
// atomicOr on its mark byte, so FW and BW of every class advance together.
// Three execution modes, chosen per step by the host from the frontier size:
//
//  * top-down level (k_reach_level): one launch per BFS level; a warp takes 32
//    items, vertices with more than 32 neighbours are expanded by the whole
//    warp (coalesced adjacency reads), the rest lane by lane; new items go to
//    a per-warp shared-memory buffer and reach the global queue in batches;
//  * bottom-up sweep (k_reach_bottomup): when the frontier is a large share of
//    the live vertices (the "RD" state of gm_bfs_template.h:418-487), every
//    unvisited live vertex looks for an already visited parent among its
//    in-neighbours (FW) / out-neighbours (BW) and stops at the first one;
//  * asynchronous drain (k_reach_async): once the frontier has stayed narrow
//    for a few levels (long-diameter inputs such as grids and long cycles),
//    one persistent launch finishes the traversal with no level barriers and
//    no host round trips.  Each warp works LIFO from its own shared-memory
//    list and spills surplus items to a global queue that idle warps drain.
//    A global `work` counter (items claimed but not yet expanded) detects the
//    end.  Every wait is bounded: past its limit a warp records
//    SCC_DEVERR_WAIT_LIMIT and returns, and the host reports SCC_ERR_TIMEOUT.
#include <stdlib.h>
#include <algorithm>
#include "scc_round.cuh"
#include "scc_tile.cuh"

// switch points come from the state's tunables (scc_tuning)
#define ASYNC_EMPTY (-1)
#define ASYNC_IDLE_LIMIT (1 << 22)
#define PRE_NONE (-2)      // an item's neighbours were not loaded with it
// Drain block: four warps.  Idle warps poll the queue counters that working
// warps update atomically; on the C2 workload 4 resident warps per SM beat 8
// (33.3 vs 35.8 ms a step) and 2 (37.5 ms).
#define ASYNC_THREADS 128
#define ASYNC_SLOT_LIMIT (1 << 20)

// ------------------------------------------------------------------ warp expansion
// Expand one item per lane (valid lanes only); push(p, item) is warp-collective.
// Items whose degree exceeds a.huge_deg are handed to k_reach_huge (edge-parallel
// over the whole grid) when huge_list is given, so one hub never serialises a level.
template <class Push>
__device__ __forceinline__ void expand_warp(const RoundArgs& a, bool valid, int32_t it, Push& push,
                                            int32_t* huge_list = nullptr, int32_t* huge_cnt = nullptr,
                                            long long* edge_acc = nullptr) {
    int lane = threadIdx.x & 31;
    int32_t v = 0, dir = 0, b = 0, e = 0, c = 0;
    if (valid) {
        v = it & ITEM_MASK;
        dir = (it >> DIR_SHIFT) & 1;
        const int32_t* off = dir ? a.r_begin : a.begin;
        b = __ldg(off + v);
        e = __ldg(off + v + 1);
        c = __ldg(a.color + v);
        if (edge_acc) *edge_acc += e - b;
        if (huge_list && e - b > a.huge_deg) {
            huge_list[atomicAdd(huge_cnt, 1)] = it;
            e = b;
        }
    }
    int32_t deg = e - b;
    unsigned big = __ballot_sync(0xFFFFFFFFu, deg > 32);
    while (big) {
        int l = __ffs(big) - 1;
        big &= big - 1;
        int32_t bb = __shfl_sync(0xFFFFFFFFu, b, l), be = __shfl_sync(0xFFFFFFFFu, e, l);
        int32_t bc = __shfl_sync(0xFFFFFFFFu, c, l), bd = __shfl_sync(0xFFFFFFFFu, dir, l);
        const int32_t* adj = bd ? a.r_node_idx : a.node_idx;
        for (int32_t k0 = bb; k0 < be; k0 += 32) {
            int32_t k = k0 + lane;
            bool p = false;
            int32_t w = 0;
            if (k < be) { w = __ldg(adj + k); p = visit(a, w, bc, bd); }
            push(p, w | (bd << DIR_SHIFT));
        }
    }
    // Low-degree lists, four neighbours at a time: the adjacency loads, then the
    // mark and colour loads, then the claims are each issued together, so a hop
    // costs three memory round trips rather than three per neighbour.
    int32_t mydeg = deg <= 32 ? deg : 0;
    int32_t maxd = (int32_t)__reduce_max_sync(0xFFFFFFFFu, (unsigned)mydeg);
    const int32_t* adj = dir ? a.r_node_idx : a.node_idx;
    const unsigned bit = 1u << dir;
    for (int32_t j0 = 0; j0 < maxd; j0 += 4) {
        int32_t w[4];
        bool p[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            p[u] = (j0 + u) < mydeg;
            w[u] = p[u] ? __ldg(adj + b + j0 + u) : 0;
        }
        unsigned mk[4];
        int32_t col[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            mk[u] = p[u] ? (unsigned)*(volatile uint8_t*)(a.mark + w[u]) : bit;
            col[u] = p[u] ? __ldg(a.color + w[u]) : c;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            p[u] = p[u] && !(mk[u] & bit) && col[u] == c;
            if (p[u]) {
                unsigned sh = (unsigned)(w[u] & 3) * 8u;
                unsigned old = atomicOr(reinterpret_cast<unsigned*>(a.mark + (w[u] & ~3)), bit << sh);
                p[u] = ((old >> sh) & bit) == 0u;
            }
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) push(p[u], w[u] | (dir << DIR_SHIFT));
    }
}

// ------------------------------------------------------------------ level mode
struct GlobalPush {
    int32_t* buf;          // warp's shared buffer
    int32_t count;         // warp-uniform
    int32_t* qout;
    int32_t* qlen;
    const int32_t* off_fw; // degree of pushed items (frontier edge count), nullptr = skip
    const int32_t* off_bw;
    unsigned long long edges;   // per lane
    __device__ __forceinline__ void finish(unsigned long long* total) {
        flush();
        if (off_fw) {
            unsigned long long e = edges;
            for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xFFFFFFFFu, e, o);
            if ((threadIdx.x & 31) == 0 && e) atomicAdd(total, e);
        }
    }
    __device__ __forceinline__ void flush() {
        int lane = threadIdx.x & 31;
        __syncwarp();
        if (count > 0) {
            int32_t base = 0;
            if (lane == 0) base = atomicAdd(qlen, count);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            for (int j = lane; j < count; j += 32) qout[base + j] = buf[j];
        }
        __syncwarp();
        count = 0;
    }
    __device__ __forceinline__ void operator()(bool p, int32_t item) {
        int lane = threadIdx.x & 31;
        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
        if (p) {
            buf[count + __popc(bal & ((1u << lane) - 1u))] = item;
            if (off_fw) {
                int32_t w = item & ITEM_MASK;
                const int32_t* off = (item >> DIR_SHIFT) ? off_bw : off_fw;
                edges += (unsigned)(__ldg(off + w + 1) - __ldg(off + w));
            }
        }
        count += __popc(bal);
        if (count > WBUF - 32) flush();
    }
};

__global__ void __launch_bounds__(REACH_THREADS) k_reach_level(RoundArgs a, const int32_t* __restrict__ qin,
                                                                int32_t nin, int32_t* __restrict__ qout,
                                                                int32_t* __restrict__ huge_list) {
    __shared__ int32_t sbuf[REACH_THREADS / 32][WBUF];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    GlobalPush push{sbuf[wid], 0, qout, a.ctr + CTR_QLEN, a.begin, a.r_begin, 0ull};
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int64_t groups = ((int64_t)nin + 31) >> 5;
    for (int64_t gi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; gi < groups; gi += nwarps) {
        int64_t idx = gi * 32 + lane;
        bool valid = idx < nin;
        int32_t it = valid ? qin[idx] : 0;
        expand_warp(a, valid, it, push, huge_list, a.ctr + CTR_SPARE4);
    }
    push.finish(reinterpret_cast<unsigned long long*>(a.ctr + CTR_EDGES));
}

// Inclusive prefix of the deferred items' degrees (one block; hoff[j] = end of item j).
__global__ void k_huge_prefix(RoundArgs a, const int32_t* __restrict__ list, int32_t cnt,
                              long long* __restrict__ hoff) {
    __shared__ long long part[1024];
    int t = threadIdx.x;
    int32_t per = (cnt + 1023) / 1024;
    int32_t b = t * per, e = min(cnt, b + per);
    long long s = 0;
    for (int32_t j = b; j < e; ++j) {
        int32_t it = list[j], v = it & ITEM_MASK;
        const int32_t* off = (it >> DIR_SHIFT) ? a.r_begin : a.begin;
        s += __ldg(off + v + 1) - __ldg(off + v);
    }
    part[t] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {
        long long x = (t >= o) ? part[t - o] : 0;
        __syncthreads();
        part[t] += x;
        __syncthreads();
    }
    long long run = (t == 0) ? 0 : part[t - 1];
    for (int32_t j = b; j < e; ++j) {
        int32_t it = list[j], v = it & ITEM_MASK;
        const int32_t* off = (it >> DIR_SHIFT) ? a.r_begin : a.begin;
        run += __ldg(off + v + 1) - __ldg(off + v);
        hoff[j] = run;
    }
}

// Edge-parallel expansion of the deferred high-degree items: thread t takes
// edge t of the concatenated adjacency lists (consecutive lanes, consecutive edges).
__global__ void __launch_bounds__(REACH_THREADS) k_reach_huge(RoundArgs a, const int32_t* __restrict__ list,
                                                               int32_t cnt, const long long* __restrict__ hoff,
                                                               int32_t* __restrict__ qout) {
    __shared__ int32_t sbuf[REACH_THREADS / 32][WBUF];
    int wid = threadIdx.x >> 5;
    GlobalPush push{sbuf[wid], 0, qout, a.ctr + CTR_QLEN, a.begin, a.r_begin, 0ull};
    long long total = hoff[cnt - 1];
    long long stride = (long long)gridDim.x * blockDim.x;
    long long limit = ((total + 31) / 32) * 32;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < limit; t += stride) {
        bool p = false;
        int32_t w = 0, d = 0;
        if (t < total) {
            int32_t lo = 0, hi = cnt - 1;
            while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (hoff[mid] > t) hi = mid; else lo = mid + 1; }
            int32_t it = list[lo], v = it & ITEM_MASK;
            d = (it >> DIR_SHIFT) & 1;
            long long start = lo ? hoff[lo - 1] : 0;
            const int32_t* off = d ? a.r_begin : a.begin;
            const int32_t* adj = d ? a.r_node_idx : a.node_idx;
            w = __ldg(adj + __ldg(off + v) + (t - start));
            p = visit(a, w, __ldg(a.color + v), d);
        }
        push(p, w | (d << DIR_SHIFT));
    }
    push.finish(reinterpret_cast<unsigned long long*>(a.ctr + CTR_EDGES));
}

// ------------------------------------------------------------------ bottom-up mode
// True if a neighbour of v carries `bit` in its mark and belongs to v's class.
// Four neighbours at a time: their adjacency entries, then their marks, are
// loaded together, so a long scan costs two round trips per four.  A round
// over one class (use_only) traverses only that class, so a marked neighbour
// is of colour c and its colour need not be read; with several classes a
// mark may come from another class's traversal.
__device__ __forceinline__ bool parent_ok(const RoundArgs& a, int32_t u, int32_t c) {
    return a.use_only || __ldg(a.color + u) == c;
}

__device__ __forceinline__ bool has_marked_parent(const RoundArgs& a, const int32_t* __restrict__ off,
                                                  const int32_t* __restrict__ adj, int32_t v, int32_t c,
                                                  unsigned bit) {
    int32_t b = __ldg(off + v), e = __ldg(off + v + 1);
    int32_t k = b;
    for (; k + 4 <= e; k += 4) {
        int32_t u[4];
        unsigned m[4];
#pragma unroll
        for (int j = 0; j < 4; ++j) u[j] = __ldg(adj + k + j);
#pragma unroll
        for (int j = 0; j < 4; ++j) m[j] = *(volatile uint8_t*)(a.mark + u[j]);
#pragma unroll
        for (int j = 0; j < 4; ++j)
            if ((m[j] & bit) && parent_ok(a, u[j], c)) return true;
    }
    for (; k < e; ++k) {
        int32_t u = __ldg(adj + k);
        if ((*(volatile uint8_t*)(a.mark + u) & bit) && parent_ok(a, u, c)) return true;
    }
    return false;
}

__global__ void __launch_bounds__(REACH_THREADS) k_reach_bottomup(RoundArgs a, int32_t* __restrict__ qout) {
    __shared__ int32_t sbuf[REACH_THREADS / 32][WBUF];
    int wid = threadIdx.x >> 5;
    GlobalPush push{sbuf[wid], 0, qout, a.ctr + CTR_QLEN, nullptr, nullptr, 0ull};
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t limit = (((int64_t)a.live_count + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += stride) {
        bool p0 = false, p1 = false;
        int32_t v = 0;
        if (i < a.live_count) {
            v = a.live[i];
            int32_t c = __ldg(a.color + v);
            if (c != SCC_COLOR_DONE && (!a.use_only || c == a.only_color)) {
                unsigned m = *(volatile uint8_t*)(a.mark + v);
                if (!(m & 1u)) p0 = has_marked_parent(a, a.r_begin, a.r_node_idx, v, c, 1u);
                if (!(m & 2u)) p1 = has_marked_parent(a, a.begin, a.node_idx, v, c, 2u);
                if (p0 || p1) {
                    unsigned sh = (unsigned)(v & 3) * 8u;
                    unsigned bits = (p0 ? 1u : 0u) | (p1 ? 2u : 0u);
                    unsigned old = atomicOr(reinterpret_cast<unsigned*>(a.mark + (v & ~3)), bits << sh);
                    // push only directions this thread newly set
                    p0 = p0 && !((old >> sh) & 1u);
                    p1 = p1 && !((old >> sh) & 2u);
                }
            }
        }
        push(p0, v);
        push(p1, v | (1 << DIR_SHIFT));
    }
    push.flush();
}

// ------------------------------------------------------------------ asynchronous mode
struct LocalPush {
    int32_t* buf;          // warp's shared list: items
    int32_t* bb;           //   and their adjacency range [bb, be) in the item's direction
    int32_t* be;
    int32_t* x0;           //   and, for an item of at most four neighbours, those
    int32_t* x1;           //   neighbours (x0 = PRE_NONE when not preloaded)
    int32_t* x2;
    int32_t* x3;
    int32_t count;         // warp-uniform
    int32_t pushed;        // items added since the last work-counter update
    int32_t* q; int32_t* tail; int32_t* work; int64_t qcap; int32_t* err;
    int32_t keep;          // items kept for this warp when sharing
    __device__ __forceinline__ void spill(int32_t keep) {
        int lane = threadIdx.x & 31;
        __syncwarp();
        int32_t ns = count - keep;
        if (ns > 0) {
            int32_t base = 0;
            if (lane == 0) {
                if (pushed) { atomicAdd(work, pushed); }
                base = atomicAdd(tail, ns);
                if ((int64_t)base + ns > qcap) atomicExch(err, SCC_DEVERR_QUEUE_OVERFLOW);
            }
            pushed = 0;
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if ((int64_t)base + ns <= qcap)
                for (int j = lane; j < ns; j += 32) *(volatile int32_t*)(q + base + j) = buf[keep + j];
            count = keep;
        }
        __syncwarp();
    }
    // Items spilled to the global queue lose their range (the taker reloads it).
    __device__ __forceinline__ void operator()(bool p, int32_t item, int32_t b, int32_t e, int32_t n0, int32_t n1, int32_t n2, int32_t n3) {
        int lane = threadIdx.x & 31;
        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
        if (p) {
            int32_t pos = count + __popc(bal & ((1u << lane) - 1u));
            buf[pos] = item; bb[pos] = b; be[pos] = e; x0[pos] = n0; x1[pos] = n1; x2[pos] = n2; x3[pos] = n3;
        }
        int32_t k = __popc(bal);
        count += k;
        pushed += k;
        if (count > WBUF - 32) spill(keep > 64 ? keep : 64);
    }
};

// Asynchronous-mode expansion.  Each item arrives with its adjacency range
// when it was claimed locally (b < 0 when it came through the global queue);
// a claim loads the claimed vertex's range in the same round trip as the
// atomic, so the next hop starts at the adjacency read.
__device__ __forceinline__ void expand_warp_async(const RoundArgs& a, bool valid, int32_t it, int32_t b, int32_t e,
                                                  int32_t x0, int32_t x1, int32_t x2, int32_t x3, LocalPush& push,
                                                  long long* edge_acc) {
    int lane = threadIdx.x & 31;
    int32_t dir = 0, c = 0;
    if (valid) {
        int32_t v = it & ITEM_MASK;
        dir = (it >> DIR_SHIFT) & 1;
        const int32_t* off = dir ? a.r_begin : a.begin;
        if (b < 0) { b = __ldg(off + v); e = __ldg(off + v + 1); }
        c = __ldg(a.color + v);
        *edge_acc += e - b;
    } else {
        b = e = 0;
    }
    int32_t deg = e - b;
    unsigned big = __ballot_sync(0xFFFFFFFFu, deg > 32);
    while (big) {
        int l = __ffs(big) - 1;
        big &= big - 1;
        int32_t lb = __shfl_sync(0xFFFFFFFFu, b, l), le = __shfl_sync(0xFFFFFFFFu, e, l);
        int32_t lc = __shfl_sync(0xFFFFFFFFu, c, l), ld = __shfl_sync(0xFFFFFFFFu, dir, l);
        const int32_t* adj = ld ? a.r_node_idx : a.node_idx;
        const int32_t* off = ld ? a.r_begin : a.begin;
        for (int32_t k0 = lb; k0 < le; k0 += 32) {
            int32_t k = k0 + lane;
            bool p = false;
            int32_t w = 0, wb = -1, we = -1;
            if (k < le) {
                w = __ldg(adj + k);
                p = visit(a, w, lc, ld);
                if (p) { wb = __ldg(off + w); we = __ldg(off + w + 1); }
            }
            push(p, w | (ld << DIR_SHIFT), wb, we, PRE_NONE, 0, 0, 0);
        }
    }
    int32_t mydeg = deg <= 32 ? deg : 0;
    int32_t maxd = (int32_t)__reduce_max_sync(0xFFFFFFFFu, (unsigned)mydeg);
    const int32_t* adj = dir ? a.r_node_idx : a.node_idx;
    const int32_t* off = dir ? a.r_begin : a.begin;
    const unsigned bit = 1u << dir;
    const bool pre = x0 != PRE_NONE;   // at most four neighbours, already loaded
    for (int32_t j0 = 0; j0 < maxd; j0 += 4) {
        int32_t w[4], wb[4], we[4];
        bool p[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            p[u] = (j0 + u) < mydeg;
            w[u] = p[u] ? (pre ? (u == 0 ? x0 : u == 1 ? x1 : u == 2 ? x2 : x3) : __ldg(adj + b + j0 + u)) : 0;
        }
        // the neighbour's range is loaded with its mark and colour (speculatively:
        // most neighbours on a narrow frontier are new), so the claim that
        // follows waits only on the L2-resident mark word
        unsigned mk[4];
        int32_t col[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            mk[u] = p[u] ? (unsigned)*(volatile uint8_t*)(a.mark + w[u]) : bit;
            col[u] = p[u] ? __ldg(a.color + w[u]) : c;
            wb[u] = p[u] ? __ldg(off + w[u]) : -1;
            we[u] = p[u] ? __ldg(off + w[u] + 1) : -1;
        }
        unsigned old[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            p[u] = p[u] && !(mk[u] & bit) && col[u] == c;
            old[u] = p[u] ? atomicOr(reinterpret_cast<unsigned*>(a.mark + (w[u] & ~3)), bit << ((w[u] & 3) * 8u)) : 0u;
        }
        // a claimed vertex of at most four neighbours brings them along, loaded
        // while its claim is in flight: its own expansion then starts at the
        // neighbours' marks instead of an adjacency read
        int32_t n0[4], n1[4], n2[4], n3[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            int32_t dg = we[u] - wb[u];
            bool small = p[u] && dg <= 4;
            n0[u] = small ? (dg >= 1 ? __ldg(adj + wb[u]) : -1) : PRE_NONE;
            n1[u] = small && dg >= 2 ? __ldg(adj + wb[u] + 1) : -1;
            n2[u] = small && dg >= 3 ? __ldg(adj + wb[u] + 2) : -1;
            n3[u] = small && dg >= 4 ? __ldg(adj + wb[u] + 3) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u) p[u] = p[u] && ((old[u] >> ((w[u] & 3) * 8u)) & bit) == 0u;
#pragma unroll
        for (int u = 0; u < 4; ++u) push(p[u], w[u] | (dir << DIR_SHIFT), wb[u], we[u], n0[u], n1[u], n2[u], n3[u]);
    }
}

__device__ __forceinline__ int32_t ld_volatile(const int32_t* p) { return *(const volatile int32_t*)p; }

__global__ void __launch_bounds__(ASYNC_THREADS, 1) k_reach_async(RoundArgs a, int32_t* __restrict__ q, int64_t qcap) {
    __shared__ int32_t sbuf[ASYNC_THREADS / 32][WBUF];
    __shared__ int32_t sbeg[ASYNC_THREADS / 32][WBUF];
    __shared__ int32_t send[ASYNC_THREADS / 32][WBUF];
    __shared__ int32_t sx0[ASYNC_THREADS / 32][WBUF];
    __shared__ int32_t sx1[ASYNC_THREADS / 32][WBUF];
    __shared__ int32_t sx2[ASYNC_THREADS / 32][WBUF];
    __shared__ int32_t sx3[ASYNC_THREADS / 32][WBUF];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t* head = a.ctr + CTR_AHEAD;
    int32_t* tail = a.ctr + CTR_ATAIL;
    int32_t* work = a.ctr + CTR_AWORK;
    int32_t* err = a.ctr + CTR_ERROR;
    int32_t* bail = a.ctr + CTR_ABAIL;
    LocalPush push{sbuf[wid], sbeg[wid], send[wid], sx0[wid], sx1[wid], sx2[wid], sx3[wid], 0, 0, q, tail, work, qcap, err, a.async_keep};
    int idle = 0;
    uint32_t iter = 0;
    int32_t last_work = -1;
    long long my_edges = 0;     // per lane
    long long my_items = 0;     // warp-uniform
    while (true) {
        if (push.count == 0) {
            // publish this warp's net change to the outstanding work before it
            // waits: the count reaches zero only once every warp has done so
            if (lane == 0 && push.pushed != 0) atomicAdd(work, push.pushed);
            push.pushed = 0;
            int32_t got = 0, base = 0;
            if (lane == 0) {
                int32_t t = ld_volatile(tail), h = ld_volatile(head);
                if (h < t) {
                    int32_t k = min(32, t - h);
                    if (atomicCAS(head, h, h + k) == h) { got = k; base = h; }
                }
            }
            got = __shfl_sync(0xFFFFFFFFu, got, 0);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (got == 0) {
                ++idle;
                if ((idle & 7) == 1) {
                    int32_t w = 1, e = 0, bl = 0;
                    if (lane == 0) { w = ld_volatile(work); e = ld_volatile(err); bl = ld_volatile(bail); }
                    w = __shfl_sync(0xFFFFFFFFu, w, 0);
                    e = __shfl_sync(0xFFFFFFFFu, e, 0);
                    bl = __shfl_sync(0xFFFFFFFFu, bl, 0);
                    if (w == 0 || e != 0 || bl != 0) break;
                    // the limit bounds a stall, not a long traversal: progress elsewhere resets it
                    if (w != last_work) { last_work = w; idle = 1; }
                }
                if (idle > ASYNC_IDLE_LIMIT) {
                    if (lane == 0) { atomicExch(err, SCC_DEVERR_WAIT_LIMIT); atomicExch(a.ctr + CTR_ERROR_INFO, 1); }
                    break;
                }
                __nanosleep(idle < 16 ? 100 : 500);
                continue;
            }
            idle = 0;
            int32_t item = ASYNC_EMPTY;
            if (lane < got) {
                volatile int32_t* slot = q + base + lane;
                int spins = 0;
                while ((item = *slot) == ASYNC_EMPTY && spins < ASYNC_SLOT_LIMIT) { spins++; __nanosleep(20); }
                if (item != ASYNC_EMPTY) *slot = ASYNC_EMPTY;
            }
            if (__any_sync(0xFFFFFFFFu, lane < got && item == ASYNC_EMPTY)) {
                if (lane == 0) { atomicExch(err, SCC_DEVERR_WAIT_LIMIT); atomicExch(a.ctr + CTR_ERROR_INFO, 2); }
                break;
            }
            if (lane < got) { push.buf[lane] = item; push.bb[lane] = -1; push.be[lane] = -1; push.x0[lane] = PRE_NONE; }
            __syncwarp();
            push.count = got;
        }
        int32_t k = min(32, push.count);
        int32_t top = push.count - k + lane;
        int32_t it = (lane < k) ? push.buf[top] : 0;
        int32_t ib = (lane < k) ? push.bb[top] : 0;
        int32_t ie = (lane < k) ? push.be[top] : 0;
        int32_t ix0 = (lane < k) ? push.x0[top] : PRE_NONE;
        int32_t ix1 = (lane < k) ? push.x1[top] : 0;
        int32_t ix2 = (lane < k) ? push.x2[top] : 0;
        int32_t ix3 = (lane < k) ? push.x3[top] : 0;
        __syncwarp();
        push.count -= k;
        expand_warp_async(a, lane < k, it, ib, ie, ix0, ix1, ix2, ix3, push, &my_edges);
        my_items += k;
        // the net change (pushed - expanded) accumulates in push.pushed and is
        // published every 8th iteration, before a spill makes items visible,
        // and before the warp waits: one counter update per 8 iterations
        // instead of one per iteration, on a line every idle warp polls
        push.pushed -= k;
        if ((++iter & 7) == 0) {
            // read back the outstanding work; a frontier that has grown wide is
            // handed back to the level-synchronous kernels, which expand wide
            // frontiers far better than one queue
            int32_t stop = 0;
            if (lane == 0) {
                int32_t w = atomicAdd(work, push.pushed) + push.pushed;
                if (w > a.async_bail) atomicExch(bail, 1);
                stop = ld_volatile(bail);
            }
            push.pushed = 0;
            if (__shfl_sync(0xFFFFFFFFu, stop, 0)) {
                push.spill(0);
                break;
            }
        }
        // keep one iteration's worth (this warp's own continuation), share the rest
        if (push.count > push.keep) push.spill(push.keep);
    }
    // work done by this warp, for the kernel ledger (items expanded, edges scanned)
    for (int o = 16; o > 0; o >>= 1) my_edges += __shfl_down_sync(0xFFFFFFFFu, my_edges, o);
    if (lane == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + CTR_ASYNC_ITEMS), (unsigned long long)my_items);
        atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + CTR_ASYNC_EDGES), (unsigned long long)my_edges);
    }
}

// ------------------------------------------------------------------ host driver
bool scc_trace_on() {
    static int t = -1;
    if (t < 0) { const char* e = getenv("SCC_TRACE"); t = (e && *e && *e != '0') ? 1 : 0; }
    return t == 1;
}

static int async_blocks(int device, int want_per_sm) {
    static int cached_sms[64] = {0}, cached_per[64] = {0};
    int sms = 148, per = 1;
    if (device >= 0 && device < 64 && cached_sms[device]) {
        sms = cached_sms[device];
        per = cached_per[device];
    } else {
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_reach_async, ASYNC_THREADS, 0);
        if (per < 1) per = 1;
        if (device >= 0 && device < 64) { cached_sms[device] = sms; cached_per[device] = per; }
    }
    // every block must be resident (warps wait on each other's items): never
    // more than the occupancy limit; a few per SM cover a narrow frontier
    // without flooding the queue with pollers
    if (want_per_sm < per) per = want_per_sm;
    if (per < 1) per = 1;
    return sms * per;
}

static double now_ms() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}

// The tile drain takes a round's narrow frontiers when the round has enough
// live vertices and its live id range splits into tiles that fit shared
// memory.  The live list is ascending, so its ends give the range.
static bool tile_round(scc_state* s, int32_t* lo, int32_t* hi) {
    if (s->tune.tile_min_live <= 0 || s->live_count < s->tune.tile_min_live) return false;
    if (*lo < 0) {
        int32_t ends[2] = {0, 0};
        if (cudaMemcpyAsync(ends, s->live, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream) != cudaSuccess ||
            cudaMemcpyAsync(ends + 1, s->live + s->live_count - 1, sizeof(int32_t), cudaMemcpyDeviceToHost,
                            s->stream) != cudaSuccess ||
            cudaStreamSynchronize(s->stream) != cudaSuccess)
            return false;
        *lo = ends[0];
        *hi = ends[1];
    }
    return scc_impl_tile_eligible(s, *lo, *hi);
}

// Direction choice (Beamer's rule as in the reference's BFS state machine,
// gm_bfs_template.h:418-487): go bottom-up when the next frontier's edges
// times bu_alpha exceed the edges of the vertices being traversed; stay
// bottom-up while the frontier holds more than 2*live/bu_div items.

int scc_impl_reach(const scc_graph* g, scc_state* s, RoundArgs& a, int32_t qlen) {
    int32_t* qin = s->qa;
    int32_t* qout = s->qb;
    int64_t live2 = 2LL * (a.live_count > 0 ? a.live_count : 1);
    unsigned long long live_edges = *reinterpret_cast<unsigned long long*>(s->h_ctr + CTR_LIVE_EDGES);
    if (live_edges == 0) live_edges = 1;
    // a small round (at most 4x the drain's entry threshold of live vertices)
    // goes straight to the drain: its frontier cannot outgrow the drain, and
    // level steps would cost a launch and a host round trip each -- unless it
    // holds a hub, which a drain warp would expand alone while the level
    // kernels expand it over the whole grid
    int narrow = ((int64_t)a.live_count <= 4LL * s->tune.async_max && s->h_ctr[CTR_MAXDEG] <= a.huge_deg)
                     ? s->tune.async_after : 0;
    bool bottom_up = false;
    double t0 = scc_trace_on() ? now_ms() : 0.0;
    int32_t live_lo = -1, live_hi = -1;     // live id range, read once when the tile drain is considered
    while (qlen > 0) {
        const char* mode;
        bool synced = false;      // the counters on the host already hold this step's results
        if (bottom_up) {
            SCC_TRY(scc_zero_counters(s, CTR_QLEN, 1));
            k_reach_bottomup<<<scc_blocks(a.live_count, REACH_THREADS, 148 * 16), REACH_THREADS, 0, s->stream>>>(a, qout);
            SCC_LAUNCHED(s);
            narrow = 0;
            mode = "bottom-up";
        } else if (qlen <= s->tune.async_max && narrow >= s->tune.async_after && tile_round(s, &live_lo, &live_hi)) {
            // narrow frontier over a large live range: the tile drain
            int32_t handed = 0;
            SCC_TRY(scc_impl_reach_tile(g, s, a, qin, qlen, qout, live_lo, live_hi, &handed));
            if (handed == 0) return SCC_OK;
            qlen = handed;
            int32_t* t = qin; qin = qout; qout = t;
            narrow = 0;
            bottom_up = false;
            if (scc_trace_on()) fprintf(stderr, "[scc] reach tile handed back %d items\n", qlen);
            continue;
        } else if (qlen <= s->tune.async_max && narrow >= s->tune.async_after) {
            int64_t qcap = 2LL * s->n + 64;
            SCC_CUDA(cudaMemcpyAsync(s->aq, qin, sizeof(int32_t) * (size_t)qlen, cudaMemcpyDeviceToDevice, s->stream));
            int32_t init[CTR_AWORK - CTR_AHEAD + 1] = {0};   // head, tail, work on separate lines
            init[CTR_ATAIL - CTR_AHEAD] = qlen;
            init[CTR_AWORK - CTR_AHEAD] = qlen;
            if (scc_impl_take_wait_injection()) {
                // injected failure: one more item is announced than written, so
                // the warp that takes slot qlen (kept at -1) waits until its
                // bound runs out and the drain reports SCC_ERR_TIMEOUT
                init[CTR_ATAIL - CTR_AHEAD] = qlen + 1;
                init[CTR_AWORK - CTR_AHEAD] = qlen + 1;
            }
            SCC_CUDA(cudaMemcpyAsync(s->ctr + CTR_AHEAD, init, sizeof(init), cudaMemcpyHostToDevice, s->stream));
            SCC_TRY(scc_zero_counters(s, CTR_ASYNC_ITEMS, 4));
            SCC_TRY(scc_zero_counters(s, CTR_ABAIL, 1));
            a.async_bail = std::max<int32_t>(8 * s->tune.async_max, 1 << 16);
            if (s->ledger_on) SCC_CUDA(cudaEventRecord(s->lev[0], s->stream));
            k_reach_async<<<async_blocks(s->device, s->tune.async_blocks_per_sm), ASYNC_THREADS, 0, s->stream>>>(a, s->aq, qcap);
            SCC_LAUNCHED(s);
            if (s->ledger_on) SCC_CUDA(cudaEventRecord(s->lev[1], s->stream));
            s->traversal_steps++;
            SCC_TRY(scc_sync_counters(s));
            if (s->ledger_on) {
                float ms = 0.f;
                SCC_CUDA(cudaEventElapsedTime(&ms, s->lev[0], s->lev[1]));
                s->ledger_ms += ms;
                s->ledger_launches++;
                s->ledger_items += *reinterpret_cast<long long*>(s->h_ctr + CTR_ASYNC_ITEMS);
                s->ledger_edges += *reinterpret_cast<long long*>(s->h_ctr + CTR_ASYNC_EDGES);
            }
            if (scc_trace_on()) {
                double t1 = now_ms();
                fprintf(stderr, "[scc] reach async seeds=%d spilled=%d %.3f ms\n", qlen, s->h_ctr[CTR_ATAIL], t1 - t0);
            }
            if (s->h_ctr[CTR_ERROR] == SCC_DEVERR_WAIT_LIMIT && s->h_ctr[CTR_ERROR_INFO] == 1 &&
                (s->h_ctr[CTR_AWORK] == 0 || s->h_ctr[CTR_ABAIL])) {
                // Idle warps gave up while a warp walked a long chain of single
                // hops: the chain stays in that warp's own buffer, so the work
                // count sits still for seconds and their idle bound cannot tell it
                // from a stall.  Warps still busy drain the queue before they read
                // the error word, so a drain that ended with no work outstanding,
                // or that handed its frontier back, is complete.
                if (scc_trace_on()) fprintf(stderr, "[scc] reach async: idle warps left a long chain early\n");
                s->h_ctr[CTR_ERROR] = 0;
                SCC_CUDA(cudaMemsetAsync(s->ctr + CTR_ERROR, 0, sizeof(int32_t) * 2, s->stream));
            }
            if (s->h_ctr[CTR_ERROR]) {
                // leave the queue clean for the next traversal, then report
                SCC_CUDA(cudaMemsetAsync(s->aq, 0xFF, sizeof(int32_t) * (size_t)qcap, s->stream));
                return scc_check_device_error(s);
            }
            if (!s->h_ctr[CTR_ABAIL]) return SCC_OK;
            // the frontier grew wide: its unexpanded items are aq[head, tail)
            // (every warp spilled its own before leaving); continue level by level
            int32_t h = s->h_ctr[CTR_AHEAD], t = s->h_ctr[CTR_ATAIL];
            qlen = t - h;
            if (qlen > 0) {
                SCC_CUDA(cudaMemcpyAsync(qin, s->aq + h, sizeof(int32_t) * (size_t)qlen, cudaMemcpyDeviceToDevice,
                                         s->stream));
                SCC_CUDA(cudaMemsetAsync(s->aq + h, 0xFF, sizeof(int32_t) * (size_t)qlen, s->stream));
            }
            narrow = 0;
            bottom_up = false;
            if (scc_trace_on()) fprintf(stderr, "[scc] reach async handed back %d items\n", qlen);
            continue;
        } else {
            SCC_TRY(scc_zero_counters(s, CTR_QLEN, 1));
            SCC_TRY(scc_zero_counters(s, CTR_SPARE4, 1));
            SCC_TRY(scc_zero_counters(s, CTR_EDGES, 2));
            k_reach_level<<<scc_blocks((int64_t)qlen, REACH_THREADS, 148 * 8), REACH_THREADS, 0, s->stream>>>(
                a, qin, qlen, qout, s->hq);
            SCC_LAUNCHED(s);
            SCC_TRY(scc_sync_counters(s));
            int32_t nhuge = s->h_ctr[CTR_SPARE4];
            if (nhuge > 0) {
                k_huge_prefix<<<1, 1024, 0, s->stream>>>(a, s->hq, nhuge, s->hoff);
                SCC_LAUNCHED(s);
                k_reach_huge<<<148 * 8, REACH_THREADS, 0, s->stream>>>(a, s->hq, nhuge, s->hoff, qout);
                SCC_LAUNCHED(s);
            } else {
                synced = true;
            }
            mode = nhuge > 0 ? "top-down+huge" : "top-down";
        }
        s->traversal_steps++;
        if (!synced) SCC_TRY(scc_sync_counters(s));
        int32_t next = s->h_ctr[CTR_QLEN];
        if (bottom_up) {
            bottom_up = (int64_t)next * s->tune.bu_div > live2;
        } else {
            unsigned long long fe = *reinterpret_cast<unsigned long long*>(s->h_ctr + CTR_EDGES);
            bottom_up = fe * (unsigned long long)s->tune.bu_alpha > live_edges;
        }
        if (scc_trace_on()) {
            double t1 = now_ms();
            fprintf(stderr, "[scc] reach %s in=%d out=%d %.3f ms\n", mode, qlen, next, t1 - t0);
            t0 = t1;
        }
        narrow = (!bottom_up && next <= s->tune.async_max) ? narrow + 1 : 0;
        qlen = next;
        int32_t* t = qin; qin = qout; qout = t;
    }
    return SCC_OK;
}
