// Method 7's level analytics on the condensation graph: topological levels of
// the DAG (the BFS in create_scc_edges, src/common_main.h:85-108, 210-219),
// the levels an inserted batch can affect (affect_level and its prefix sum,
// :232-262), and the trim shortcut that finishes every node of an unaffected
// level as its own SCC (src/scc_trim1.cc:67-73).
//
// The reference computes levels with a FIFO queue (Kahn's order): a node is
// queued when its last predecessor is processed, and every processed edge
// overwrites the child's level with the parent's level + 1.  The queue's
// levels never decrease, so the last write is the largest, and a level is the
// longest path from a source.  Here the peel runs without an order: released
// nodes are expanded from per-warp queues in shared memory, each edge raises
// its child's level with atomicMax before it decrements the child's
// in-count, and whoever brings the count to zero releases the child.  Nodes
// that are never released (on or behind a cycle, when the labels are not the
// SCCs of the graph) keep the largest level + 1 of their released
// predecessors, or 0 -- what the reference's queue leaves them.
#include "scc_internal.cuh"
#include "scc_sort.cuh"

#define LEVEL_Q 256          // per-warp queue of released nodes awaiting expansion
#define LEVEL_HUB 4096       // a released node with more out-edges is expanded over the whole grid

struct LevelArgs {
    const int32_t* begin; const int32_t* node_idx; const int32_t* r_begin;
    int32_t* cnt; int32_t* level; int32_t* ovf; int32_t* ovf_count;
    int32_t* hub; int32_t* hub_count;      // released hubs set aside for k_level_hub
};

// One out-edge of released x (whose level is lx - 1): raise the child's level,
// then take its in-count; returns the child if this released it, else -1.
__device__ __forceinline__ int32_t level_edge(const LevelArgs& a, int32_t w, int32_t lx) {
    atomicMax(a.level + w, lx);
    __threadfence();
    return atomicSub(a.cnt + w, 1) == 1 ? w : -1;
}

__global__ void k_level_init(int32_t n, const int32_t* __restrict__ r_begin, int32_t* __restrict__ cnt,
                             int32_t* __restrict__ level) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        cnt[i] = __ldg(r_begin + i + 1) - __ldg(r_begin + i);
        level[i] = 0;
    }
}

// Expand this warp's released nodes 32 at a time, their out-edges spread over
// the lanes (warp prefix sum of the degrees, owner found by a binary search
// over the lanes).  A released node's level is final: each of its
// predecessors raised it before the fence that precedes their decrement.
__device__ void level_drain(const LevelArgs& a, int32_t* wq, int32_t& qn) {
    const int lane = threadIdx.x & 31;
    const unsigned full = 0xFFFFFFFFu;
    while (qn > 0) {
        const int32_t take = min(qn, 32);
        qn -= take;
        const int32_t x = lane < take ? wq[qn + lane] : -1;
        __syncwarp();
        __threadfence();
        int32_t ob = 0, od = 0, lx = 0;
        if (x >= 0) {
            ob = __ldg(a.begin + x);
            od = __ldg(a.begin + x + 1) - ob;
            lx = __ldcg(a.level + x) + 1;
            if (od > LEVEL_HUB) {          // too many edges for one warp: the host expands it
                a.hub[atomicAdd(a.hub_count, 1)] = x;
                od = 0;
            }
        }
        int32_t incl = od;
        for (int o = 1; o < 32; o <<= 1) {
            int32_t t = __shfl_up_sync(full, incl, o);
            if (lane >= o) incl += t;
        }
        const int32_t total = __shfl_sync(full, incl, 31);
        const int32_t excl = incl - od;
        for (int32_t j0 = 0; j0 < total; j0 += 32) {
            const int32_t j = j0 + lane;
            int owner = 0;                                   // largest lane with excl <= j
            for (int step = 16; step > 0; step >>= 1) {
                int cand = owner + step;
                int32_t ev = __shfl_sync(full, excl, cand);
                if (ev <= j) owner = cand;
            }
            const int32_t k = j - __shfl_sync(full, excl, owner);
            const int32_t oob = __shfl_sync(full, ob, owner);
            const int32_t olx = __shfl_sync(full, lx, owner);
            int32_t nv = -1;
            if (j < total) nv = level_edge(a, __ldg(a.node_idx + oob + k), olx);
            const unsigned bal = __ballot_sync(full, nv >= 0);
            if (bal) {
                const int32_t r = __popc(bal & ((1u << lane) - 1u)), nn = __popc(bal);
                if (qn + nn <= LEVEL_Q) {
                    if (nv >= 0) wq[qn + r] = nv;
                    qn += nn;
                } else {
                    int32_t base = 0;
                    if (lane == 0) base = atomicAdd(a.ovf_count, nn);
                    base = __shfl_sync(full, base, 0);
                    if (nv >= 0) a.ovf[base + r] = nv;
                }
                __syncwarp();
            }
        }
    }
}

// Sweep (items == NULL): the sources (no in-edges, decided from the offsets,
// so no decrement can release one twice) start the peel.  List: expand
// released nodes that overflowed a queue.
__global__ void __launch_bounds__(SCC_THREADS) k_level_peel(LevelArgs a, int32_t n, const int32_t* __restrict__ items) {
    __shared__ int32_t queues[SCC_THREADS / 32][LEVEL_Q];
    const int lane = threadIdx.x & 31;
    int32_t* wq = queues[threadIdx.x >> 5];
    int32_t qn = 0;
    const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t base = ((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5) * 32; base < n; base += nwarps * 32) {
        const int64_t i = base + lane;
        int32_t x = -1;
        if (i < n) {
            if (items) x = items[i];
            else if (__ldg(a.r_begin + i + 1) == __ldg(a.r_begin + i)) x = (int32_t)i;
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, x >= 0);
        if (x >= 0) wq[__popc(bal & ((1u << lane) - 1u))] = x;    // qn == 0 here
        qn = __popc(bal);
        __syncwarp();
        level_drain(a, wq, qn);
    }
}

// Inclusive prefix of the hubs' out-degrees (one block; hoff[j] = end of hub j).
__global__ void k_level_hub_prefix(const int32_t* __restrict__ begin, const int32_t* __restrict__ hubs, int32_t cnt,
                                   long long* __restrict__ hoff) {
    __shared__ long long part[1024];
    int t = threadIdx.x;
    int32_t per = (cnt + 1023) / 1024;
    int32_t b = t * per, e = min(cnt, b + per);
    long long sum = 0;
    for (int32_t j = b; j < e; ++j) sum += __ldg(begin + hubs[j] + 1) - __ldg(begin + hubs[j]);
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
        run += __ldg(begin + hubs[j] + 1) - __ldg(begin + hubs[j]);
        hoff[j] = run;
    }
}

// Edge-parallel expansion of released hubs: thread t takes edge t of their
// concatenated out-lists; the children it releases join the overflow list.
__global__ void k_level_hub(LevelArgs a, const int32_t* __restrict__ hubs, int32_t cnt,
                            const long long* __restrict__ hoff) {
    const long long total = hoff[cnt - 1];
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long limit = ((total + 31) / 32) * 32;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < limit; t += stride) {
        int32_t nv = -1;
        if (t < total) {
            int32_t lo = 0, hi = cnt - 1;
            while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (hoff[mid] > t) hi = mid; else lo = mid + 1; }
            const int32_t x = hubs[lo];
            const long long start = lo ? hoff[lo - 1] : 0;
            nv = level_edge(a, __ldg(a.node_idx + __ldg(a.begin + x) + (t - start)), __ldcg(a.level + x) + 1);
        }
        const unsigned bal = __ballot_sync(0xFFFFFFFFu, nv >= 0);
        if (bal) {
            const int lane = threadIdx.x & 31;
            int32_t base = 0;
            if (lane == 0) base = atomicAdd(a.ovf_count, __popc(bal));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (nv >= 0) a.ovf[base + __popc(bal & ((1u << lane) - 1u))] = nv;
        }
    }
}

__global__ void k_level_max(int32_t n, const int32_t* __restrict__ level, int32_t* __restrict__ out) {
    int32_t m = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        m = max(m, level[i]);
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_down_sync(0xFFFFFFFFu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, m);
}

namespace {
struct Buf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~Buf() { if (p) cudaFreeAsync(p, st); }
    template <class T> T* as() { return (T*)p; }
};
int get(Buf& b, size_t bytes, cudaStream_t st) {
    b.st = st;
    SCC_CUDA(scc_impl_malloc_async(&b.p, bytes > 0 ? bytes : 16, st));
    return SCC_OK;
}
struct Stream {
    cudaStream_t st = nullptr;
    ~Stream() { if (st) { cudaStreamSynchronize(st); cudaStreamDestroy(st); } }
};
}  // namespace

// Levels into d_level (device, n ints); *max_level from the device.
static int levels_on_device(const scc_graph* g, cudaStream_t st, int32_t* d_level, int32_t* max_level) {
    int32_t n = g->n;
    *max_level = 0;
    if (n == 0) return SCC_OK;
    Buf cnt, ovf, list, ctr, hub, hubs, hoff;
    SCC_TRY(get(cnt, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(get(ovf, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(get(list, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(get(hub, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(get(hubs, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(get(hoff, sizeof(long long) * (size_t)n, st));
    SCC_TRY(get(ctr, sizeof(int32_t) * 4, st));      // overflow count, max level, hub count
    LevelArgs a;
    a.begin = g->begin; a.node_idx = g->node_idx; a.r_begin = g->r_begin;
    a.cnt = cnt.as<int32_t>(); a.level = d_level; a.ovf = ovf.as<int32_t>(); a.ovf_count = ctr.as<int32_t>();
    a.hub = hub.as<int32_t>(); a.hub_count = ctr.as<int32_t>() + 2;
    k_level_init<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, g->r_begin, a.cnt, d_level);
    SCC_CUDA(cudaPeekAtLastError());
    SCC_CUDA(cudaMemsetAsync(ctr.p, 0, sizeof(int32_t) * 4, st));
    k_level_peel<<<scc_blocks(n, SCC_THREADS, 148 * 8), SCC_THREADS, 0, st>>>(a, n, nullptr);
    SCC_CUDA(cudaPeekAtLastError());
    // Rounds: overflowed releases expanded by a list launch, hubs edge-parallel
    // (their releases join the overflow list).  Each node is released once,
    // so the lists together hold at most n and the rounds end.
    for (int round = 0;; ++round) {
        SCC_REQUIRE(round < SCC_HOST_ROUND_LIMIT, SCC_ERR_TIMEOUT, "topological levels: no fixpoint after %d rounds", round);
        int32_t c[4] = {0, 0, 0, 0};
        SCC_CUDA(cudaMemcpyAsync(c, ctr.p, sizeof(c), cudaMemcpyDeviceToHost, st));
        SCC_CUDA(cudaStreamSynchronize(st));
        const int32_t novf = c[0], nhub = c[2];
        if (novf == 0 && nhub == 0) break;
        if (novf > 0)
            SCC_CUDA(cudaMemcpyAsync(list.p, ovf.p, sizeof(int32_t) * (size_t)novf, cudaMemcpyDeviceToDevice, st));
        if (nhub > 0)
            SCC_CUDA(cudaMemcpyAsync(hubs.p, hub.p, sizeof(int32_t) * (size_t)nhub, cudaMemcpyDeviceToDevice, st));
        SCC_CUDA(cudaMemsetAsync(ctr.p, 0, sizeof(int32_t), st));
        SCC_CUDA(cudaMemsetAsync(ctr.as<int32_t>() + 2, 0, sizeof(int32_t), st));
        if (nhub > 0) {
            k_level_hub_prefix<<<1, 1024, 0, st>>>(g->begin, hubs.as<int32_t>(), nhub, hoff.as<long long>());
            SCC_CUDA(cudaPeekAtLastError());
            k_level_hub<<<148 * 8, SCC_THREADS, 0, st>>>(a, hubs.as<int32_t>(), nhub, hoff.as<long long>());
            SCC_CUDA(cudaPeekAtLastError());
        }
        if (novf > 0) {
            k_level_peel<<<scc_blocks(novf, SCC_THREADS, 148 * 8), SCC_THREADS, 0, st>>>(a, novf, list.as<int32_t>());
            SCC_CUDA(cudaPeekAtLastError());
        }
    }
    int32_t* d_max = ctr.as<int32_t>() + 1;
    k_level_max<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, d_level, d_max);
    SCC_CUDA(cudaPeekAtLastError());
    SCC_CUDA(cudaMemcpyAsync(max_level, d_max, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    return SCC_OK;
}

extern "C" int scc_topological_levels(const scc_graph* dag, int32_t* levels, int32_t* max_level) {
    SCC_REQUIRE(dag && levels && max_level, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(dag->device));
    Stream s;
    SCC_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    Buf lev;
    SCC_TRY(get(lev, sizeof(int32_t) * (size_t)dag->n, s.st));
    SCC_TRY(levels_on_device(dag, s.st, lev.as<int32_t>(), max_level));
    if (dag->n > 0)
        SCC_CUDA(cudaMemcpyAsync(levels, lev.p, sizeof(int32_t) * (size_t)dag->n, cudaMemcpyDeviceToHost, s.st));
    SCC_CUDA(cudaStreamSynchronize(s.st));
    return SCC_OK;
}

// ------------------------------------------------------------------ affected levels
// Every inserted edge joining two SCCs adds one over the level interval
// [min, max] of its endpoints' SCCs: +1 at min, -1 at max + 1.
__global__ void k_affect_diff(int64_t k, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                              const int32_t* __restrict__ label, int32_t n, const int32_t* __restrict__ level,
                              int32_t num_sccs, int32_t max_level, int32_t* __restrict__ diff, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t x = a[i], y = b[i];
        if (x < 0 || x >= n || y < 0 || y >= n) { atomicExch(bad, 1); continue; }
        int32_t cx = label[x], cy = label[y];
        if (cx < 0 || cx >= num_sccs || cy < 0 || cy >= num_sccs) { atomicExch(bad, 2); continue; }
        if (cx == cy) continue;
        int32_t lx = level[cx], ly = level[cy];
        if (lx < 0 || lx > max_level || ly < 0 || ly > max_level) { atomicExch(bad, 3); continue; }
        atomicAdd(diff + min(lx, ly), 1);
        atomicAdd(diff + max(lx, ly) + 1, -1);
    }
}

__global__ void k_count_zero(int32_t n, const int32_t* __restrict__ v, int32_t* __restrict__ out) {
    int32_t c = 0;
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x)
        c += (i < n && v[i] == 0);
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

extern "C" int scc_affected_levels(const scc_graph* dag, const int32_t* levels, int32_t max_level, int32_t n,
                                   const int32_t* labels, int64_t n_ins, const int32_t* ins_src,
                                   const int32_t* ins_dst, int32_t* affected, int32_t* num_unaffected) {
    SCC_REQUIRE(dag && levels && labels && affected && num_unaffected && n >= 0 && max_level >= 0 && n_ins >= 0,
                SCC_ERR_INVALID, "bad argument");
    SCC_REQUIRE(n_ins == 0 || (ins_src && ins_dst), SCC_ERR_INVALID, "NULL batch arrays");
    SCC_CUDA(cudaSetDevice(dag->device));
    Stream s;
    SCC_CUDA(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
    cudaStream_t st = s.st;
    const int32_t L = max_level + 1;
    Buf lab, lev, src, dst, diff, out, bad;
    SCC_TRY(get(lab, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(get(lev, sizeof(int32_t) * (size_t)dag->n, st));
    SCC_TRY(get(src, sizeof(int32_t) * (size_t)n_ins, st));
    SCC_TRY(get(dst, sizeof(int32_t) * (size_t)n_ins, st));
    SCC_TRY(get(diff, sizeof(int32_t) * ((size_t)L + 1), st));
    SCC_TRY(get(out, sizeof(int32_t) * (size_t)L, st));
    SCC_TRY(get(bad, sizeof(int32_t) * 2, st));
    SCC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int32_t) * 2, st));
    SCC_CUDA(cudaMemsetAsync(diff.p, 0, sizeof(int32_t) * ((size_t)L + 1), st));
    if (n > 0) SCC_CUDA(cudaMemcpyAsync(lab.p, labels, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, st));
    if (dag->n > 0)
        SCC_CUDA(cudaMemcpyAsync(lev.p, levels, sizeof(int32_t) * (size_t)dag->n, cudaMemcpyHostToDevice, st));
    if (n_ins > 0) {
        SCC_CUDA(cudaMemcpyAsync(src.p, ins_src, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st));
        SCC_CUDA(cudaMemcpyAsync(dst.p, ins_dst, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st));
        k_affect_diff<<<scc_blocks(n_ins), SCC_THREADS, 0, st>>>(n_ins, src.as<int32_t>(), dst.as<int32_t>(),
                                                                lab.as<int32_t>(), n, lev.as<int32_t>(), dag->n,
                                                                max_level, diff.as<int32_t>(), bad.as<int>());
        SCC_CUDA(cudaPeekAtLastError());
    }
    SCC_TRY(scc_impl_scan_i32(diff.as<int32_t>(), out.as<int32_t>(), L, true, st));
    k_count_zero<<<scc_blocks(L), SCC_THREADS, 0, st>>>(L, out.as<int32_t>(), bad.as<int32_t>() + 1);
    SCC_CUDA(cudaPeekAtLastError());
    int32_t h[2] = {0, 0};
    SCC_CUDA(cudaMemcpyAsync(affected, out.p, sizeof(int32_t) * (size_t)L, cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaMemcpyAsync(h, bad.p, sizeof(h), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    SCC_REQUIRE(h[0] != 1, SCC_ERR_INVALID, "inserted endpoint outside [0, %d)", n);
    SCC_REQUIRE(h[0] != 2, SCC_ERR_INVALID, "label outside [0, %d)", dag->n);
    SCC_REQUIRE(h[0] != 3, SCC_ERR_INVALID, "level outside [0, %d]", max_level);
    *num_unaffected = h[1];
    return SCC_OK;
}

// ------------------------------------------------------------------ trim shortcut
__global__ void k_finish_unaffected(int32_t n, const int32_t* __restrict__ level, const int32_t* __restrict__ affected,
                                    int32_t max_level, int32_t* __restrict__ color, int32_t* __restrict__ scc,
                                    int32_t* __restrict__ count) {
    int32_t c = 0;
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n) {
            int32_t l = level[i];
            if (l >= 0 && l <= max_level && affected[l] == 0) {
                color[i] = SCC_COLOR_DONE;
                scc[i] = (int32_t)i;
                c++;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

extern "C" int scc_state_finish_unaffected(scc_state* s, const int32_t* levels, const int32_t* affected,
                                           int32_t max_level, int32_t* finished) {
    SCC_REQUIRE(s && levels && affected && max_level >= 0, SCC_ERR_INVALID, "bad argument");
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t n = s->n;
    Buf lev, aff;
    SCC_TRY(get(lev, sizeof(int32_t) * (size_t)n, s->stream));
    SCC_TRY(get(aff, sizeof(int32_t) * ((size_t)max_level + 1), s->stream));
    if (n > 0) SCC_CUDA(cudaMemcpyAsync(lev.p, levels, sizeof(int32_t) * (size_t)n, cudaMemcpyHostToDevice, s->stream));
    SCC_CUDA(cudaMemcpyAsync(aff.p, affected, sizeof(int32_t) * ((size_t)max_level + 1), cudaMemcpyHostToDevice,
                             s->stream));
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 1));
    if (n > 0) {
        k_finish_unaffected<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, lev.as<int32_t>(), aff.as<int32_t>(),
                                                                           max_level, s->color, s->scc,
                                                                           s->ctr + CTR_COUNT);
        SCC_LAUNCHED(s);
    }
    SCC_TRY(scc_sync_counters(s));
    s->prefinished = s->fresh || s->prefinished;   // the counting peel still applies
    s->fresh = false;
    s->cnt_valid = false;
    if (finished) *finished = s->h_ctr[CTR_COUNT];
    return SCC_OK;
}
