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
//    items; vertices above huge_deg neighbours go edge-parallel over the
//    grid (k_reach_huge), those above cta_deg are expanded by the whole block
//    with their adjacency streamed into shared memory by bulk copies, those
//    above 32 by the whole warp (coalesced adjacency reads), the rest lane by
//    lane; new items go to a per-warp shared-memory buffer and reach the
//    global queue in batches;
//  * bottom-up sweep (k_reach_bottomup): when the frontier is a large share of
//    the live vertices (the "RD" state of gm_bfs_template.h:418-487), every
//    unvisited live vertex looks for an already visited parent among its
//    in-neighbours (FW) and a visited child among its out-neighbours (BW),
//    both searches in step, int4 chunks of adjacency at a time, and stops
//    each at its first hit;
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
                                            long long* edge_acc = nullptr, int32_t* cta_list = nullptr,
                                            int32_t* cta_cnt = nullptr) {
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
        } else if (cta_list && e - b > a.cta_deg) {
            cta_list[atomicAdd(cta_cnt, 1)] = it;      // the block expands it (expand_block)
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

// ------------------------------------------------------------------ block-wide expansion
// A top-down item of degree in (cta_deg, huge_deg] is expanded by the whole
// block: its adjacency list is streamed into shared memory in chunks of
// CTA_STAGE entries by 1-D bulk copies (cp.async.bulk, global memory of this
// GPU into this CTA's shared memory, completion counted on an mbarrier), two
// buffers deep, so the next chunk is in flight while the block visits the
// current one.  A copy starts and ends on 16-byte boundaries: the staged
// range is [b & ~3, e & ~3) (entries before b are masked) and the last
// (e & 3) entries are read directly.
#define CTA_STAGE 1024
#define BULK_WAIT_LIMIT (1 << 20)

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Copy `bytes` (a multiple of 16, both addresses 16-byte aligned) from global
// memory into shared memory; the copy's bytes complete the barrier's phase.
__device__ __forceinline__ void bulk_stage(void* dst, const void* src, uint32_t bytes, unsigned long long* bar) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                 ::"r"(smem_u32(dst)), "l"(src), "r"(bytes), "r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the barrier's phase of the given parity.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, uint32_t parity) {
    for (int i = 0; i < BULK_WAIT_LIMIT; ++i) {
        uint32_t ok;
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
                     " selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(ok) : "r"(smem_u32(bar)), "r"(parity) : "memory");
        if (ok) return true;
    }
    return false;
}

struct BlockStage {
    int32_t buf[2][CTA_STAGE];
    unsigned long long bar[2];
    int32_t list[REACH_THREADS];     // items deferred to the block in this pass
    int32_t count;
};

// Expand [b, e) (direction dir, class c) with every thread of the block.
// Block-uniform; returns false (error word set) if a copy did not complete
// within its bound, after waiting once more, bounded, for copies in flight.
template <class Push>
__device__ bool expand_block(const RoundArgs& a, int32_t b, int32_t e, int32_t c, int32_t dir, BlockStage& st,
                             uint32_t& parity, Push& push) {
    const int32_t* adj = dir ? a.r_node_idx : a.node_idx;
    const int tid = threadIdx.x;
    const int32_t lo = b & ~3, hi = e & ~3;
    const int32_t nchunks = (a.vec_adj && hi > lo) ? (hi - lo + CTA_STAGE - 1) / CTA_STAGE : 0;
    if (nchunks > 0 && tid == 0)
        bulk_stage(st.buf[0], adj + lo, 4u * (uint32_t)min(CTA_STAGE, hi - lo), &st.bar[0]);
    for (int32_t t = 0; t < nchunks; ++t) {
        const int32_t x0 = lo + t * CTA_STAGE, x1 = min(hi, x0 + CTA_STAGE);
        const int nb = (t + 1) & 1;
        if (t + 1 < nchunks && tid == 0)   // buffer nb was released by the barrier that ended chunk t - 1
            bulk_stage(st.buf[nb], adj + x1, 4u * (uint32_t)(min(hi, x1 + CTA_STAGE) - x1), &st.bar[nb]);
        const int cb = t & 1;
        const uint32_t ph = (parity >> cb) & 1u;
        bool ok = mbar_wait(&st.bar[cb], ph);
        parity ^= 1u << cb;
        if (__syncthreads_or(!ok)) {
            if (tid == 0) {
                atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_WAIT_LIMIT);
                atomicExch(a.ctr + CTR_ERROR_INFO, 3);
            }
            if (!ok) mbar_wait(&st.bar[cb], ph);
            if (t + 1 < nchunks) mbar_wait(&st.bar[nb], (parity >> nb) & 1u);
            return false;
        }
        for (int32_t k0 = max(b, x0); k0 < x1; k0 += REACH_THREADS) {
            const int32_t k = k0 + tid;
            bool p = false;
            int32_t w = 0;
            if (k < x1) { w = st.buf[cb][k - x0]; p = visit(a, w, c, dir); }
            push(p, w | (dir << DIR_SHIFT));
        }
        __syncthreads();
    }
    for (int32_t k0 = nchunks > 0 ? max(b, hi) : b; k0 < e; k0 += REACH_THREADS) {
        const int32_t k = k0 + tid;
        bool p = false;
        int32_t w = 0;
        if (k < e) { w = __ldg(adj + k); p = visit(a, w, c, dir); }
        push(p, w | (dir << DIR_SHIFT));
    }
    return true;
}

// One top-down level.  BLOCK: items of degree in (cta_deg, huge_deg] are
// collected per pass of REACH_THREADS items and expanded by the whole block
// after the pass's warp and lane expansions.
template <bool BLOCK>
__global__ void __launch_bounds__(REACH_THREADS) k_reach_level(RoundArgs a, const int32_t* __restrict__ qin,
                                                                int32_t nin, int32_t* __restrict__ qout,
                                                                int32_t* __restrict__ huge_list) {
    __shared__ int32_t sbuf[REACH_THREADS / 32][WBUF];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    GlobalPush push{sbuf[wid], 0, qout, a.ctr + CTR_QLEN, a.begin, a.r_begin, 0ull};
    if constexpr (!BLOCK) {
        int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
        int64_t groups = ((int64_t)nin + 31) >> 5;
        for (int64_t gi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; gi < groups; gi += nwarps) {
            int64_t idx = gi * 32 + lane;
            bool valid = idx < nin;
            int32_t it = valid ? qin[idx] : 0;
            expand_warp(a, valid, it, push, huge_list, a.ctr + CTR_SPARE4);
        }
    } else {
        __shared__ __align__(16) BlockStage st;
        if (threadIdx.x == 0) {
            mbar_init(&st.bar[0], 1);
            mbar_init(&st.bar[1], 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
            st.count = 0;
        }
        __syncthreads();
        uint32_t parity = 0;
        bool ok = true;
        for (int64_t base = (int64_t)blockIdx.x * REACH_THREADS; base < nin && ok;
             base += (int64_t)gridDim.x * REACH_THREADS) {
            int64_t idx = base + threadIdx.x;
            bool valid = idx < nin;
            int32_t it = valid ? qin[idx] : 0;
            expand_warp(a, valid, it, push, huge_list, a.ctr + CTR_SPARE4, nullptr, st.list, &st.count);
            __syncthreads();
            const int32_t nc = st.count;
            for (int32_t j = 0; j < nc && ok; ++j) {
                const int32_t ci = st.list[j], v = ci & ITEM_MASK, d = (ci >> DIR_SHIFT) & 1;
                const int32_t* off = d ? a.r_begin : a.begin;
                ok = expand_block(a, __ldg(off + v), __ldg(off + v + 1), __ldg(a.color + v), d, st, parity, push);
            }
            __syncthreads();
            if (threadIdx.x == 0) st.count = 0;
            __syncthreads();
        }
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
// A round over one class (use_only) traverses only that class, so a marked
// neighbour is of colour c and its colour need not be read; with several
// classes a mark may come from another class's traversal.
// Entries [k, e) of one adjacency list seen through the aligned chunk
// [k & ~3, (k & ~3) + P): P/4 int4 loads (a 32-byte sector for P = 8) when
// the chunk lies inside the array and the array is 16-byte aligned, else one
// load per entry that lies in [k, e).  Entries outside [k, e) are masked.
template <int P>
__device__ __forceinline__ void probe_chunk(const RoundArgs& a, const int32_t* __restrict__ adj, int32_t k,
                                            int32_t e, int32_t (&u)[P], bool (&p)[P]) {
    const int32_t c0 = k & ~3;
#pragma unroll
    for (int j = 0; j < P; ++j) p[j] = k < e && c0 + j >= k && c0 + j < e;
    if (k < e && a.vec_adj && (int64_t)c0 + P <= a.adj_len) {
#pragma unroll
        for (int q = 0; q < P / 4; ++q) {
            int4 x = __ldg(reinterpret_cast<const int4*>(adj + c0) + q);
            u[4 * q] = x.x; u[4 * q + 1] = x.y; u[4 * q + 2] = x.z; u[4 * q + 3] = x.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < P; ++j) u[j] = p[j] ? __ldg(adj + c0 + j) : 0;
    }
}

// One thread per live vertex, both directions at once: the vertex's colour,
// mark and both adjacency ranges are loaded together, then each probe loads
// an aligned chunk of each still-open list, then the marks of both chunks'
// neighbours, then (in a round over several classes) the colours of the
// marked ones -- three dependent round trips per probe for the two searches
// together, where searching one direction after the other costs six.
// P = 4 (one int4 per list and probe, 40 registers): R-MAT s24 1.274 ->
// 1.243 ms and C3 2.29 -> 2.17 ms a decomposition against one direction
// after the other; P = 8 (a whole 32-byte sector per probe) needs 64
// registers, halves the resident warps and is slower on both (1.38, 2.48 ms).
template <int P>
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
            unsigned m = *(volatile uint8_t*)(a.mark + v);
            int32_t k0 = __ldg(a.r_begin + v), e0 = __ldg(a.r_begin + v + 1);   // FW: a marked in-neighbour
            int32_t k1 = __ldg(a.begin + v), e1 = __ldg(a.begin + v + 1);       // BW: a marked out-neighbour
            bool in = c != SCC_COLOR_DONE && (!a.use_only || c == a.only_color);
            if (!in || (m & 1u)) e0 = k0;
            if (!in || (m & 2u)) e1 = k1;
            while (k0 < e0 || k1 < e1) {
                int32_t u0[P], u1[P];
                bool q0[P], q1[P];
                probe_chunk<P>(a, a.r_node_idx, k0, e0, u0, q0);
                probe_chunk<P>(a, a.node_idx, k1, e1, u1, q1);
                unsigned m0[P], m1[P];
#pragma unroll
                for (int j = 0; j < P; ++j) m0[j] = q0[j] ? (unsigned)*(volatile uint8_t*)(a.mark + u0[j]) : 0u;
#pragma unroll
                for (int j = 0; j < P; ++j) m1[j] = q1[j] ? (unsigned)*(volatile uint8_t*)(a.mark + u1[j]) : 0u;
#pragma unroll
                for (int j = 0; j < P; ++j) {
                    q0[j] = q0[j] && (m0[j] & 1u);
                    q1[j] = q1[j] && (m1[j] & 2u);
                }
                if (!a.use_only) {
                    // a mark may come from another class's traversal
#pragma unroll
                    for (int j = 0; j < P; ++j) {
                        int32_t c0 = q0[j] ? __ldg(a.color + u0[j]) : c;
                        int32_t c1 = q1[j] ? __ldg(a.color + u1[j]) : c;
                        q0[j] = q0[j] && c0 == c;
                        q1[j] = q1[j] && c1 == c;
                    }
                }
                bool h0 = false, h1 = false;
#pragma unroll
                for (int j = 0; j < P; ++j) { h0 = h0 || q0[j]; h1 = h1 || q1[j]; }
                if (h0) { p0 = true; e0 = k0; } else { k0 = (k0 & ~3) + P; }
                if (h1) { p1 = true; e1 = k1; } else { k1 = (k1 & ~3) + P; }
            }
            if (p0 || p1) {
                unsigned sh = (unsigned)(v & 3) * 8u;
                unsigned bits = (p0 ? 1u : 0u) | (p1 ? 2u : 0u);
                unsigned old = atomicOr(reinterpret_cast<unsigned*>(a.mark + (v & ~3)), bits << sh);
                // push only directions this thread newly set
                p0 = p0 && !((old >> sh) & 1u);
                p1 = p1 && !((old >> sh) & 2u);
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
                // a queue that overflowed (its error already recorded by the
                // spill) is read no further than its capacity
                if ((int64_t)t > qcap) t = (int32_t)qcap;
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
            k_reach_bottomup<4><<<scc_blocks(a.live_count, REACH_THREADS, 148 * 16), REACH_THREADS, 0, s->stream>>>(
                a, qout);
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
            const int lblocks = scc_blocks((int64_t)qlen, REACH_THREADS, 148 * 8);
            RoundArgs la = a;
            bool block_bucket = a.cta_deg > 0 && a.cta_deg < a.huge_deg;
            if (block_bucket && lblocks < 148) {
                // a level of fewer blocks than SMs would expand each mid-degree
                // item in one block while most SMs idle: those items go
                // edge-parallel over the whole GPU instead (the pivot's own
                // lists, the first levels after it)
                la.huge_deg = a.cta_deg;
                block_bucket = false;
            }
            if (block_bucket)
                k_reach_level<true><<<lblocks, REACH_THREADS, 0, s->stream>>>(la, qin, qlen, qout, s->hq);
            else
                k_reach_level<false><<<lblocks, REACH_THREADS, 0, s->stream>>>(la, qin, qlen, qout, s->hq);
            SCC_LAUNCHED(s);
            SCC_TRY(scc_sync_counters(s));
            if (s->h_ctr[CTR_ERROR]) return scc_check_device_error(s);
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
        // a frontier of few items may still hold hubs: it counts as narrow
        // only while its edges stay under the drain's hand-back bound, else
        // the drain would take it, grow past the bound and hand it back
        bool edges_small = true;
        if (bottom_up) {
            bottom_up = (int64_t)next * s->tune.bu_div > live2;
        } else {
            unsigned long long fe = *reinterpret_cast<unsigned long long*>(s->h_ctr + CTR_EDGES);
            bottom_up = fe * (unsigned long long)s->tune.bu_alpha > live_edges;
            edges_small = fe <= (unsigned long long)a.async_bail;
        }
        if (scc_trace_on()) {
            double t1 = now_ms();
            fprintf(stderr, "[scc] reach %s in=%d out=%d %.3f ms\n", mode, qlen, next, t1 - t0);
            t0 = t1;
        }
        narrow = (!bottom_up && next <= s->tune.async_max && edges_small) ? narrow + 1 : 0;
        qlen = next;
        int32_t* t = qin; qin = qout; qout = t;
    }
    return SCC_OK;
}
