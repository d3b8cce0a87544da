// Edge-batch updates of a decomposed graph (methods 5-11 of the reference:
// insert_idea1/insert_idea2, src/scc_incremental.cc:7-27, create_scc_edges,
// src/common_main.h:180-314; delete_idea1, src/scc_decremental.cc:7-24, and
// read_file2, src/common_main.h:343-393).
//
// The reference rebuilds gm_graph on the host and either recomputes
// everything (method 5), decomposes the condensation graph (methods 6, 7, 11),
// or re-runs the pipeline with the SCCs that lost an edge (methods 8-10, only
// SCC index 5 in its code).  Here a batch is applied on the device:
//
//  1. CSR merge: deleted (u,v) pairs remove every copy of that edge, inserted
//     pairs are added (kept sorted, duplicates allowed as add_edge allows
//     them), on the CSR and on the transpose.
//  2. Deletions: only an old SCC that lost an internal edge can split.  Those
//     SCCs become classes and the device recursion re-decomposes them; every
//     other SCC keeps its label.  Afterwards every label class is strongly
//     connected in the new graph.
//  3. Insertions: a merge needs a cycle through an inserted edge (u,v) whose
//     ends are in different classes (the old condensation had no cycle), so
//     every merged SCC lies in R = FW(those v) and BW(those u).  R is a union
//     of classes closed under strong connectivity; SCCs are recomputed inside
//     R only.
#include <algorithm>
#include <string.h>
#include "scc_round.cuh"
#include "scc_sort.cuh"

// ------------------------------------------------------------------ kernels
__global__ void k_upd_keys(int64_t k, const int32_t* __restrict__ a, const int32_t* __restrict__ b, int32_t n,
                           unsigned long long* __restrict__ keys, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t x = a[i], y = b[i];
        if (x < 0 || x >= n || y < 0 || y >= n) { atomicExch(bad, 1); keys[i] = ~0ull; continue; }
        keys[i] = ((unsigned long long)(uint32_t)x << 32) | (uint32_t)y;
    }
}

// For each deleted key (row, col): mark every copy of col in row's sorted list.
__global__ void k_upd_mark_deleted(int64_t k, const unsigned long long* __restrict__ keys,
                                   const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                                   uint8_t* __restrict__ dead, int32_t* __restrict__ ndead) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long key = keys[i];
        if (key == ~0ull || (i > 0 && keys[i - 1] == key)) continue;   // skip repeats of the same pair
        int32_t r = (int32_t)(key >> 32), c = (int32_t)(uint32_t)key;
        int32_t lo = off[r], hi = off[r + 1];
        while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (adj[mid] < c) lo = mid + 1; else hi = mid; }
        int32_t cnt = 0;
        for (int32_t e = lo; e < off[r + 1] && adj[e] == c; ++e) { dead[e] = 1; cnt++; }
        if (cnt) atomicAdd(ndead + r, cnt);
    }
}

// new degree = old - dead + inserted
__global__ void k_upd_degrees(int32_t n, const int32_t* __restrict__ off, const int32_t* __restrict__ ndead,
                              const unsigned long long* __restrict__ ins, int64_t kins, int32_t* __restrict__ ins_begin,
                              int32_t* __restrict__ deg) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        // inserted keys of row v: [lower_bound(v<<32), lower_bound((v+1)<<32))
        unsigned long long lo_key = (unsigned long long)v << 32;
        int64_t lo = 0, hi = kins;
        while (lo < hi) { int64_t mid = (lo + hi) >> 1; if (ins[mid] < lo_key) lo = mid + 1; else hi = mid; }
        int64_t a = lo;
        hi = kins;
        unsigned long long hi_key = (unsigned long long)(v + 1) << 32;
        while (lo < hi) { int64_t mid = (lo + hi) >> 1; if (ins[mid] < hi_key) lo = mid + 1; else hi = mid; }
        ins_begin[v] = (int32_t)a;
        deg[v] = (off[v + 1] - off[v]) - ndead[v] + (int32_t)(lo - a);
    }
}

// Per-vertex merge of the kept old entries and the inserted ones (both sorted).
__global__ void k_upd_merge(int32_t n, const int32_t* __restrict__ off, const int32_t* __restrict__ adj,
                            const uint8_t* __restrict__ dead, const int32_t* __restrict__ ndead,
                            const unsigned long long* __restrict__ ins, const int32_t* __restrict__ ins_begin,
                            const int32_t* __restrict__ new_off, int32_t* __restrict__ new_adj,
                            int32_t* __restrict__ kp) {
    int lane = threadIdx.x & 31;
    int64_t wstride = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t w = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; w < n; w += wstride) {
        int32_t v = (int32_t)w;
        int32_t b = off[v], e = off[v + 1];
        int32_t nb = new_off[v];
        int32_t nins = (new_off[v + 1] - nb) - ((e - b) - ndead[v]);
        if (nins == 0 && ndead[v] == 0) {            // unchanged list: coalesced copy
            for (int32_t k = lane; k < e - b; k += 32) new_adj[nb + k] = adj[b + k];
            continue;
        }
        // Changed list, merged by the whole warp.  A kept old entry x lands at
        // (kept entries before it) + (inserted entries < x); an inserted y at
        // (its index) + (kept old entries <= y), so equal values keep old-first
        // order.  kp[i] records the kept count before old position i.
        const unsigned long long* iv = ins + ins_begin[v];
        int32_t kept_base = 0;
        for (int32_t i0 = b; i0 < e; i0 += 32) {
            int32_t i = i0 + lane;
            bool valid = i < e;
            int32_t x = valid ? adj[i] : 0;
            bool kept = valid && !dead[i];
            unsigned bal = __ballot_sync(0xFFFFFFFFu, kept);
            int32_t r = __popc(bal & ((1u << lane) - 1u));
            if (valid) kp[i] = kept_base + r;
            if (kept) {
                int32_t lo = 0, hi = nins;
                while (lo < hi) { int32_t mid = (lo + hi) >> 1; if ((int32_t)(uint32_t)iv[mid] < x) lo = mid + 1; else hi = mid; }
                new_adj[nb + kept_base + r + lo] = x;
            }
            kept_base += __popc(bal);
        }
        __syncwarp();
        for (int32_t j = lane; j < nins; j += 32) {
            int32_t y = (int32_t)(uint32_t)iv[j];
            int32_t lo = b, hi = e;          // first old entry > y
            while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (adj[mid] <= y) lo = mid + 1; else hi = mid; }
            int32_t before = (lo < e) ? kp[lo] : kept_base;
            new_adj[nb + j + before] = y;
        }
        __syncwarp();
    }
}

__global__ void k_upd_fill(int64_t n, int32_t* __restrict__ a, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) a[i] = v;
}

// Deleted pairs inside one SCC flag that SCC's representative.
__global__ void k_upd_flag_split(int64_t k, const unsigned long long* __restrict__ keys, const int32_t* __restrict__ scc,
                                 int32_t* __restrict__ flag) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long key = keys[i];
        if (key == ~0ull) continue;
        int32_t u = (int32_t)(key >> 32), w = (int32_t)(uint32_t)key;
        int32_t r = scc[u];
        if (r >= 0 && r == scc[w]) flag[r] = 1;
    }
}

// Vertices of flagged SCCs become live with their old representative as class
// colour; all others are finished.
__global__ void k_upd_colour_flagged(int32_t n, const int32_t* __restrict__ scc, const int32_t* __restrict__ flag,
                                     int32_t* __restrict__ color, int32_t* __restrict__ count) {
    int32_t c = 0;
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n) {
            int32_t r = scc[i];
            bool live = r >= 0 && flag[r];
            color[i] = live ? r : SCC_COLOR_DONE;
            c += live;
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// Seeds of the merge region: for inserted (u,v) across classes, FW from v, BW from u.
__global__ void k_upd_seed_region(int64_t k, const unsigned long long* __restrict__ keys, const int32_t* __restrict__ scc,
                                  uint8_t* __restrict__ mark, int32_t* __restrict__ q, int32_t* __restrict__ qlen) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        unsigned long long key = keys[i];
        if (key == ~0ull) continue;
        int32_t u = (int32_t)(key >> 32), v = (int32_t)(uint32_t)key;
        if (scc[u] == scc[v]) continue;
        unsigned sh = (unsigned)(v & 3) * 8u;
        unsigned old = atomicOr(reinterpret_cast<unsigned*>(mark + (v & ~3)), 1u << sh);
        if (!((old >> sh) & 1u)) q[atomicAdd(qlen, 1)] = v;
        sh = (unsigned)(u & 3) * 8u;
        old = atomicOr(reinterpret_cast<unsigned*>(mark + (u & ~3)), 2u << sh);
        if (!((old >> sh) & 2u)) q[atomicAdd(qlen, 1)] = u | (1 << DIR_SHIFT);
    }
}

// R = reached both ways: class 0, live; everything else finished.  Marks cleared.
__global__ void k_upd_colour_region(int32_t n, uint8_t* __restrict__ mark, int32_t* __restrict__ color,
                                    int32_t* __restrict__ count) {
    int32_t c = 0;
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < n) {
            bool in = (mark[i] & 3) == 3;
            color[i] = in ? 0 : SCC_COLOR_DONE;
            mark[i] = 0;
            c += in;
        }
    }
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(count, c);
}

// ------------------------------------------------------------------ host helpers
// Stream-ordered scratch: cudaFree would synchronise the whole device and
// serialise updates that run concurrently on other streams.
struct DevBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    ~DevBuf() { if (p) cudaFreeAsync(p, st); }
    template <class T> T* as() { return (T*)p; }
};

static int alloc(DevBuf& b, size_t bytes, cudaStream_t st) {
    b.st = st;
    SCC_CUDA(scc_impl_malloc_async(&b.p, bytes > 0 ? bytes : 16, st));
    return SCC_OK;
}

// Replace a graph's arrays with stream-ordered ones.
static void release_graph_arrays(scc_graph* g, cudaStream_t st) {
    int32_t* arr[4] = {g->begin, g->node_idx, g->r_begin, g->r_node_idx};
    for (int i = 0; i < 4; ++i) {
        if (!arr[i]) continue;
        if (g->async_arrays) cudaFreeAsync(arr[i], st);
        else cudaFree(arr[i]);
    }
}

// keys (a<<32|b) sorted ascending into out (k entries); invalid ids flagged in *bad.
static int sorted_keys(int64_t k, const int32_t* d_a, const int32_t* d_b, int32_t n, cudaStream_t st,
                       DevBuf& out, int* d_bad) {
    DevBuf tmpk;
    SCC_TRY(alloc(out, sizeof(unsigned long long) * (size_t)k, st));
    SCC_TRY(alloc(tmpk, sizeof(unsigned long long) * (size_t)k, st));
    if (k == 0) return SCC_OK;
    k_upd_keys<<<scc_blocks(k), SCC_THREADS, 0, st>>>(k, d_a, d_b, n, tmpk.as<unsigned long long>(), d_bad);
    SCC_CUDA(cudaPeekAtLastError());
    // a < n in the high word: the bits above 32 + log2(n) are zero
    int hb = 1;
    while (hb < 31 && (1LL << hb) < (int64_t)n) hb++;
    return scc_impl_sort_keys_u64(tmpk.as<unsigned long long>(), out.as<unsigned long long>(), k, 32 + hb, st);
}

// Merge one side (off/adj) with sorted deleted and inserted keys; returns new arrays.
static int merge_side(int32_t n, int64_t m, const int32_t* off, const int32_t* adj, const unsigned long long* del,
                      int64_t kdel, const unsigned long long* ins, int64_t kins, cudaStream_t st, int32_t** new_off,
                      int32_t** new_adj, int64_t* new_m) {
    DevBuf dead, ndead, insb, deg, kp;
    SCC_TRY(alloc(kp, sizeof(int32_t) * (size_t)(m > 0 ? m : 1), st));
    SCC_TRY(alloc(dead, (size_t)(m > 0 ? m : 1), st));
    SCC_TRY(alloc(ndead, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(alloc(insb, sizeof(int32_t) * (size_t)n, st));
    SCC_TRY(alloc(deg, sizeof(int32_t) * ((size_t)n + 1), st));
    SCC_CUDA(cudaMemsetAsync(dead.p, 0, (size_t)(m > 0 ? m : 1), st));
    SCC_CUDA(cudaMemsetAsync(ndead.p, 0, sizeof(int32_t) * (size_t)n, st));
    SCC_CUDA(cudaMemsetAsync(deg.p, 0, sizeof(int32_t) * ((size_t)n + 1), st));
    if (kdel > 0) {
        k_upd_mark_deleted<<<scc_blocks(kdel), SCC_THREADS, 0, st>>>(kdel, del, off, adj, dead.as<uint8_t>(),
                                                                     ndead.as<int32_t>());
        SCC_CUDA(cudaPeekAtLastError());
    }
    if (n > 0) {
        k_upd_degrees<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, off, ndead.as<int32_t>(), ins, kins, insb.as<int32_t>(),
                                                             deg.as<int32_t>());
        SCC_CUDA(cudaPeekAtLastError());
    }
    int32_t* noff = nullptr;
    SCC_CUDA(scc_impl_malloc_async((void**)&noff, sizeof(int32_t) * ((size_t)n + 1), st));
    {
        int rc = scc_impl_scan_i32(deg.as<int32_t>(), noff, (int64_t)n + 1, false, st);
        if (rc != SCC_OK) { cudaFreeAsync(noff, st); return rc; }
    }
    int32_t nm = 0;
    SCC_CUDA(cudaMemcpyAsync(&nm, noff + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    int32_t* nadj = nullptr;
    cudaError_t e = scc_impl_malloc_async((void**)&nadj, sizeof(int32_t) * (size_t)(nm > 0 ? nm : 1), st);
    if (e != cudaSuccess) { cudaFreeAsync(noff, st); return scc_cuda_status(e, "scratch allocation", __FILE__, __LINE__); }
    if (n > 0) {
        k_upd_merge<<<scc_blocks((int64_t)n * 32, SCC_THREADS, 148 * 16), SCC_THREADS, 0, st>>>(
            n, off, adj, dead.as<uint8_t>(), ndead.as<int32_t>(), ins, insb.as<int32_t>(), noff, nadj,
            kp.as<int32_t>());
        SCC_CUDA(cudaPeekAtLastError());
    }
    SCC_CUDA(cudaStreamSynchronize(st));
    *new_off = noff; *new_adj = nadj; *new_m = nm;
    return SCC_OK;
}

static RoundArgs update_round_args(const scc_graph* g, scc_state* s) {
    RoundArgs a;
    a.begin = g->begin; a.node_idx = g->node_idx; a.r_begin = g->r_begin; a.r_node_idx = g->r_node_idx;
    a.color = s->color; a.scc = s->scc; a.mark = s->mark;
    a.slot_key = s->slot_key; a.slot_pivot = s->slot_pivot; a.slot_fw = s->slot_fw; a.slot_bw = s->slot_bw;
    a.slot_count = s->slot_count;
    a.colour_cap = s->colour_cap;
    a.ctr = s->ctr;
    a.live = s->live; a.live_count = s->live_count;
    a.only_color = 0; a.use_only = 1;
    a.huge_deg = s->tune.huge_deg;
    a.async_keep = s->tune.async_keep;
    a.async_bail = std::max<int32_t>(8 * s->tune.async_max, 1 << 16);
    a.pivot_salt = 0;
    a.cta_deg = s->tune.cta_deg;
    round_args_adjacency(a, g->node_idx, g->r_node_idx, g->m);
    return a;
}

static double ev_ms(cudaEvent_t a, cudaEvent_t b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, a, b) != cudaSuccess) { cudaGetLastError(); return 0.0; }
    return ms;
}

// ------------------------------------------------------------------ C ABI
extern "C" int scc_update_batch(scc_graph* g, scc_state* s, int64_t n_ins, const int32_t* ins_src,
                                const int32_t* ins_dst, int64_t n_del, const int32_t* del_src, const int32_t* del_dst,
                                int on_device, scc_update_stats* stats) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(s->n == g->n, SCC_ERR_INVALID, "state and graph differ in size");
    SCC_REQUIRE(n_ins >= 0 && n_del >= 0, SCC_ERR_INVALID, "negative batch size");
    SCC_REQUIRE((n_ins == 0 || (ins_src && ins_dst)) && (n_del == 0 || (del_src && del_dst)), SCC_ERR_INVALID,
                "NULL batch arrays");
    SCC_REQUIRE(g->m + n_ins < (1LL << 31) - 1, SCC_ERR_INVALID, "edge count would exceed int32");
    SCC_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    scc_update_stats out;
    memset(&out, 0, sizeof(out));
    SCC_CUDA(cudaEventRecord(s->ev[8], st));
    int32_t n = g->n;
    // batch to the device
    DevBuf d_is, d_id, d_ds, d_dd, bad;
    const int32_t *is = ins_src, *id = ins_dst, *ds = del_src, *dd = del_dst;
    if (!on_device) {
        SCC_TRY(alloc(d_is, sizeof(int32_t) * (size_t)n_ins, st)); SCC_TRY(alloc(d_id, sizeof(int32_t) * (size_t)n_ins, st));
        SCC_TRY(alloc(d_ds, sizeof(int32_t) * (size_t)n_del, st)); SCC_TRY(alloc(d_dd, sizeof(int32_t) * (size_t)n_del, st));
        if (n_ins) {
            SCC_CUDA(cudaMemcpyAsync(d_is.p, ins_src, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st));
            SCC_CUDA(cudaMemcpyAsync(d_id.p, ins_dst, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st));
        }
        if (n_del) {
            SCC_CUDA(cudaMemcpyAsync(d_ds.p, del_src, sizeof(int32_t) * (size_t)n_del, cudaMemcpyHostToDevice, st));
            SCC_CUDA(cudaMemcpyAsync(d_dd.p, del_dst, sizeof(int32_t) * (size_t)n_del, cudaMemcpyHostToDevice, st));
        }
        is = d_is.as<int32_t>(); id = d_id.as<int32_t>(); ds = d_ds.as<int32_t>(); dd = d_dd.as<int32_t>();
    }
    SCC_TRY(alloc(bad, sizeof(int), st));
    SCC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    DevBuf ins_k, ins_t, del_k, del_t;
    SCC_TRY(sorted_keys(n_ins, is, id, n, st, ins_k, bad.as<int>()));
    SCC_TRY(sorted_keys(n_ins, id, is, n, st, ins_t, bad.as<int>()));
    SCC_TRY(sorted_keys(n_del, ds, dd, n, st, del_k, bad.as<int>()));
    SCC_TRY(sorted_keys(n_del, dd, ds, n, st, del_t, bad.as<int>()));
    int hbad = 0;
    SCC_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    SCC_REQUIRE(!hbad, SCC_ERR_INVALID, "batch edge endpoint outside [0, %d)", n);

    // 1. CSR merge, both sides
    int32_t *nb = nullptr, *na = nullptr, *nrb = nullptr, *nra = nullptr;
    int64_t m1 = 0, m2 = 0;
    SCC_TRY(merge_side(n, g->m, g->begin, g->node_idx, del_k.as<unsigned long long>(), n_del,
                       ins_k.as<unsigned long long>(), n_ins, st, &nb, &na, &m1));
    int rc = merge_side(n, g->m, g->r_begin, g->r_node_idx, del_t.as<unsigned long long>(), n_del,
                        ins_t.as<unsigned long long>(), n_ins, st, &nrb, &nra, &m2);
    if (rc != SCC_OK) { cudaFreeAsync(nb, st); cudaFreeAsync(na, st); return rc; }
    release_graph_arrays(g, st);
    g->begin = nb; g->node_idx = na; g->r_begin = nrb; g->r_node_idx = nra; g->m = m1;
    g->self_loops = -1;
    g->async_arrays = true;
    SCC_CUDA(cudaEventRecord(s->ev[9], st));

    // 2. deletions: re-decompose the SCCs that lost an internal edge
    int32_t* flag = reinterpret_cast<int32_t*>(s->cnt);   // scratch, n ints: the peel residue is gone
    s->cnt_valid = false;
    if (n_del > 0) {
        k_upd_fill<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, flag, 0);
        SCC_LAUNCHED(s);
        k_upd_flag_split<<<scc_blocks(n_del), SCC_THREADS, 0, st>>>(n_del, del_k.as<unsigned long long>(), s->scc, flag);
        SCC_LAUNCHED(s);
        SCC_TRY(scc_zero_counters(s, CTR_SPARE0, 1));
        k_upd_colour_flagged<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, s->scc, flag, s->color, s->ctr + CTR_SPARE0);
        SCC_LAUNCHED(s);
        SCC_TRY(scc_sync_counters(s));
        out.affected_delete = s->h_ctr[CTR_SPARE0];
        if (out.affected_delete > 0) {
            s->fresh = false;
            s->prefinished = false;
            s->live_count = -1;
            SCC_TRY(scc_impl_resolve_all(g, s));
        }
    }
    SCC_CUDA(cudaEventRecord(s->ev[10], st));

    // 3. insertions: recompute inside R = FW(targets) & BW(sources) of cross-class inserted edges
    if (n_ins > 0) {
        // every vertex one traversal class
        k_upd_fill<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, s->color, 0);
        SCC_LAUNCHED(s);
        SCC_CUDA(cudaMemsetAsync(s->mark, 0, (size_t)((n + 4) & ~3LL), st));
        SCC_TRY(scc_zero_counters(s, CTR_QLEN, 1));
        k_upd_seed_region<<<scc_blocks(n_ins), SCC_THREADS, 0, st>>>(n_ins, ins_k.as<unsigned long long>(), s->scc,
                                                                     s->mark, s->qa, s->ctr + CTR_QLEN);
        SCC_LAUNCHED(s);
        SCC_TRY(scc_sync_counters(s));
        int32_t qlen = s->h_ctr[CTR_QLEN];
        if (qlen > 0) {
            // traversal over all vertices: the live list is every vertex
            SCC_TRY(scc_impl_compact_live(g, s, true));
            RoundArgs a = update_round_args(g, s);
            *reinterpret_cast<unsigned long long*>(s->h_ctr + CTR_LIVE_EDGES) = 2ull * (unsigned long long)g->m;
            s->h_ctr[CTR_MAXDEG] = INT32_MAX;      // degrees not scanned here: no shortcut to the drain
            SCC_TRY(scc_impl_reach(g, s, a, qlen));
            SCC_TRY(scc_zero_counters(s, CTR_SPARE0, 1));
            k_upd_colour_region<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, s->mark, s->color, s->ctr + CTR_SPARE0);
            SCC_LAUNCHED(s);
            SCC_TRY(scc_sync_counters(s));
            out.affected_insert = s->h_ctr[CTR_SPARE0];
            s->fresh = false;
            s->prefinished = false;
            s->live_count = -1;
            if (out.affected_insert > 0) SCC_TRY(scc_impl_resolve_all(g, s));
        } else {
            k_upd_fill<<<scc_blocks(n), SCC_THREADS, 0, st>>>(n, s->color, SCC_COLOR_DONE);
            SCC_LAUNCHED(s);
        }
    }
    SCC_CUDA(cudaEventRecord(s->ev[11], st));
    SCC_CUDA(cudaStreamSynchronize(st));
    SCC_TRY(scc_check_device_error(s));
    out.ms_merge = ev_ms(s->ev[8], s->ev[9]);
    out.ms_delete = ev_ms(s->ev[9], s->ev[10]);
    out.ms_insert = ev_ms(s->ev[10], s->ev[11]);
    out.ms_total = ev_ms(s->ev[8], s->ev[11]);
    out.m_after = g->m;
    int32_t k = 0;
    SCC_TRY(scc_count_sccs(s, &k));
    out.num_sccs = k;
    if (stats) *stats = out;
    return SCC_OK;
}

extern "C" int scc_incremental_insert(scc_graph* g, scc_state* s, int64_t n_ins, const int32_t* src,
                                      const int32_t* dst, scc_update_stats* stats) {
    return scc_update_batch(g, s, n_ins, src, dst, 0, nullptr, nullptr, 0, stats);
}

extern "C" int scc_decremental_delete(scc_graph* g, scc_state* s, int64_t n_del, const int32_t* src,
                                      const int32_t* dst, scc_update_stats* stats) {
    return scc_update_batch(g, s, 0, nullptr, nullptr, n_del, src, dst, 0, stats);
}

// insert_idea1 (src/scc_incremental.cc:7-17): the graph plus the inserted
// edges, decomposed from scratch (method 5).
extern "C" int scc_insert_idea1(scc_graph* g, scc_state* s, int64_t n_ins, const int32_t* src, const int32_t* dst,
                                scc_run_stats* stats) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    int32_t *nb = nullptr, *na = nullptr, *nrb = nullptr, *nra = nullptr;
    int64_t m1 = 0, m2 = 0;
    SCC_CUDA(cudaSetDevice(s->device));
    cudaStream_t st = s->stream;
    DevBuf d_s, d_d, bad, ins_k, ins_t;
    SCC_TRY(alloc(d_s, sizeof(int32_t) * (size_t)n_ins, st)); SCC_TRY(alloc(d_d, sizeof(int32_t) * (size_t)n_ins, st));
    if (n_ins) {
        SCC_CUDA(cudaMemcpyAsync(d_s.p, src, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st));
        SCC_CUDA(cudaMemcpyAsync(d_d.p, dst, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st));
    }
    SCC_TRY(alloc(bad, sizeof(int), st));
    SCC_CUDA(cudaMemsetAsync(bad.p, 0, sizeof(int), st));
    SCC_TRY(sorted_keys(n_ins, d_s.as<int32_t>(), d_d.as<int32_t>(), g->n, st, ins_k, bad.as<int>()));
    SCC_TRY(sorted_keys(n_ins, d_d.as<int32_t>(), d_s.as<int32_t>(), g->n, st, ins_t, bad.as<int>()));
    int hbad = 0;
    SCC_CUDA(cudaMemcpyAsync(&hbad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, st));
    SCC_CUDA(cudaStreamSynchronize(st));
    SCC_REQUIRE(!hbad, SCC_ERR_INVALID, "inserted edge endpoint outside [0, %d)", g->n);
    SCC_TRY(merge_side(g->n, g->m, g->begin, g->node_idx, nullptr, 0, ins_k.as<unsigned long long>(), n_ins, st, &nb,
                       &na, &m1));
    SCC_TRY(merge_side(g->n, g->m, g->r_begin, g->r_node_idx, nullptr, 0, ins_t.as<unsigned long long>(), n_ins, st,
                       &nrb, &nra, &m2));
    release_graph_arrays(g, st);
    g->begin = nb; g->node_idx = na; g->r_begin = nrb; g->r_node_idx = nra; g->m = m1;
    g->self_loops = -1;
    g->async_arrays = true;
    SCC_TRY(scc_state_reset(s));
    return scc_run(g, s, SCC_METHOD_GLOBAL_WCC_FB, SCC_PIVOT_DEGREE, stats);
}

// create_scc_edges + insert_idea2 (src/common_main.h:180-314,
// src/scc_incremental.cc:19-27): the condensation graph over the SCC ids of
// `labels` (ids < num_sccs), with every cross-SCC edge of g and of the
// inserted batch mapped to (id(u), id(v)); duplicates dropped.
// Condensation edges (create_scc_edges, src/common_main.h:180-314): every
// edge (u, v) becomes (label[u], label[v]); pairs inside one SCC would be
// self-loops the build drops, so only cross-SCC pairs are written, appended
// to a compact list.  Edge-balanced: a block takes COND_CHUNK consecutive
// edges, stages the offsets and labels of the vertices owning them in shared
// memory, and each thread finds its edges' sources there by binary search.
// Adjacency is streamed (evict-first) so the label array stays in L2 for
// the random destination gathers.
#define COND_ITEMS 8
#define COND_CHUNK (SCC_THREADS * COND_ITEMS)
#define COND_TILE_V COND_CHUNK

// largest v in [lo, hi] with off[v] <= k (off[lo] <= k)
__device__ __forceinline__ int32_t cond_owner(const int32_t* off, int32_t lo, int32_t hi, int32_t k) {
    while (lo < hi) {
        int32_t mid = lo + ((hi - lo + 1) >> 1);
        if (off[mid] <= k) lo = mid; else hi = mid - 1;
    }
    return lo;
}

// owner[c] = source vertex of edge c * COND_CHUNK; owner[chunks] = n - 1
__global__ void k_cond_owners(int32_t n, int64_t chunks, const int32_t* __restrict__ off, int32_t* __restrict__ owner) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c <= chunks; c += (int64_t)gridDim.x * blockDim.x)
        owner[c] = c == chunks ? n - 1 : cond_owner(off, 0, n - 1, (int32_t)(c * COND_CHUNK));
}

__global__ void k_cond_check_labels(int32_t n, const int32_t* __restrict__ label, int32_t num_sccs, int* __restrict__ bad) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t l = label[v];
        if (l < 0 || l >= num_sccs) atomicExch(bad, 1);
    }
}

__global__ void __launch_bounds__(SCC_THREADS) k_cond_cross(int32_t m, int64_t chunks, const int32_t* __restrict__ off,
                                                            const int32_t* __restrict__ adj,
                                                            const int32_t* __restrict__ label,
                                                            const int32_t* __restrict__ owner,
                                                            int32_t* __restrict__ out_src, int32_t* __restrict__ out_dst,
                                                            int32_t* __restrict__ count) {
    __shared__ int32_t scan_w[SCC_THREADS / 32];
    __shared__ int32_t s_off[COND_TILE_V + 1];
    __shared__ int32_t s_lab[COND_TILE_V];
    __shared__ int32_t s_base;
    const bool vec = (((uintptr_t)adj) & 15) == 0;
    for (int64_t c = blockIdx.x; c < chunks; c += gridDim.x) {
        const int32_t e0 = (int32_t)(c * COND_CHUNK);
        const int32_t e1 = (int32_t)min((int64_t)m, (c + 1) * COND_CHUNK);
        const int32_t vs = owner[c], hi = owner[c + 1];   // every source of the chunk lies in [vs, hi]
        const int32_t nv = hi - vs + 1;
        const bool tiled = nv <= COND_TILE_V;
        if (tiled) {
            for (int i = threadIdx.x; i <= nv; i += SCC_THREADS) s_off[i] = off[vs + i];
            for (int i = threadIdx.x; i < nv; i += SCC_THREADS) s_lab[i] = label[vs + i];
        }
        const int32_t k0 = e0 + threadIdx.x * COND_ITEMS;
        int32_t d[COND_ITEMS];
        if (vec && k0 + COND_ITEMS <= e1) {
#pragma unroll
            for (int j = 0; j < COND_ITEMS; j += 4) {
                int4 q = __ldcs((const int4*)(adj + k0 + j));
                d[j] = q.x; d[j + 1] = q.y; d[j + 2] = q.z; d[j + 3] = q.w;
            }
        } else {
#pragma unroll
            for (int j = 0; j < COND_ITEMS; j++) d[j] = k0 + j < e1 ? __ldcs(adj + k0 + j) : 0;
        }
#pragma unroll
        for (int j = 0; j < COND_ITEMS; j++) d[j] = k0 + j < e1 ? __ldg(label + d[j]) : 0;
        __syncthreads();
        int32_t sl[COND_ITEMS];
        int keep = 0;
        if (k0 < e1) {
            if (tiled) {
                int32_t i = cond_owner(s_off, 0, nv - 1, k0);
#pragma unroll
                for (int j = 0; j < COND_ITEMS; j++) {
                    sl[j] = 0;
                    if (k0 + j < e1) {   // off[hi + 1] > k0 + j stops the walk inside the tile
                        while (s_off[i + 1] <= k0 + j) i++;
                        sl[j] = s_lab[i];
                    }
                }
            } else {
                int32_t v = cond_owner(off, vs, hi, k0);
#pragma unroll
                for (int j = 0; j < COND_ITEMS; j++) {
                    sl[j] = 0;
                    if (k0 + j < e1) {
                        while (v < hi && off[v + 1] <= k0 + j) v++;
                        sl[j] = label[v];
                    }
                }
            }
#pragma unroll
            for (int j = 0; j < COND_ITEMS; j++)
                if (k0 + j < e1 && sl[j] != d[j]) keep |= 1 << j;
        }
        int32_t total = 0;
        const int32_t pre = scc_block_excl_sum256(__popc(keep), scan_w, &total);
        if (threadIdx.x == 0 && total > 0) s_base = atomicAdd(count, total);
        __syncthreads();
        if (keep) {
            int32_t at = s_base + pre;
#pragma unroll
            for (int j = 0; j < COND_ITEMS; j++)
                if (keep & (1 << j)) { out_src[at] = sl[j]; out_dst[at] = d[j]; at++; }
        }
        __syncthreads();   // shared tiles and scan storage are reused
    }
}

// inserted pairs (insert_idea2, src/scc_incremental.cc:18-27) mapped through
// the labels and appended when they join two SCCs
__global__ void k_cond_batch(int64_t k, const int32_t* __restrict__ a, const int32_t* __restrict__ b,
                             const int32_t* __restrict__ label, int32_t n, int32_t* __restrict__ out_src,
                             int32_t* __restrict__ out_dst, int32_t* __restrict__ count, int* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t x = a[i], y = b[i];
        if (x < 0 || x >= n || y < 0 || y >= n) { atomicExch(bad, 1); continue; }
        int32_t lx = label[x], ly = label[y];
        if (lx == ly) continue;
        int32_t at = atomicAdd(count, 1);
        out_src[at] = lx;
        out_dst[at] = ly;
    }
}

extern "C" int scc_condensation_graph(const scc_graph* g, const int32_t* labels, int32_t num_sccs, int64_t n_ins,
                                      const int32_t* ins_src, const int32_t* ins_dst, scc_graph** out) {
    SCC_REQUIRE(g && labels && out && num_sccs >= 0, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(n_ins == 0 || (ins_src && ins_dst), SCC_ERR_INVALID, "NULL batch arrays");
    SCC_REQUIRE(n_ins >= 0 && g->m + n_ins < (1LL << 31) - 1, SCC_ERR_INVALID, "batch of %lld edges too large",
                (long long)n_ins);
    SCC_CUDA(cudaSetDevice(g->device));
    cudaStream_t st;
    SCC_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    const int64_t total = g->m + n_ins;
    const int64_t chunks = (g->m + COND_CHUNK - 1) / COND_CHUNK;
    int rc = SCC_OK;
    {   // buffers are freed on `st` before it is destroyed
    DevBuf lab, osrc, odst, own, bs, bd, ctr;
    if ((rc = alloc(lab, sizeof(int32_t) * (size_t)g->n, st)) == SCC_OK &&
        (rc = alloc(osrc, sizeof(int32_t) * (size_t)total, st)) == SCC_OK &&
        (rc = alloc(odst, sizeof(int32_t) * (size_t)total, st)) == SCC_OK &&
        (rc = alloc(own, sizeof(int32_t) * (size_t)(chunks + 1), st)) == SCC_OK &&
        (rc = alloc(bs, sizeof(int32_t) * (size_t)n_ins, st)) == SCC_OK &&
        (rc = alloc(bd, sizeof(int32_t) * (size_t)n_ins, st)) == SCC_OK &&
        (rc = alloc(ctr, 2 * sizeof(int), st)) == SCC_OK) {
        int* bad = ctr.as<int>();
        int32_t* count = ctr.as<int32_t>() + 1;
        cudaMemsetAsync(ctr.p, 0, 2 * sizeof(int), st);
        cudaMemcpyAsync(lab.p, labels, sizeof(int32_t) * (size_t)g->n, cudaMemcpyHostToDevice, st);
        if (g->n > 0)
            k_cond_check_labels<<<scc_blocks(g->n, SCC_THREADS, 148 * 8), SCC_THREADS, 0, st>>>(
                g->n, lab.as<int32_t>(), num_sccs, bad);
        if (g->m > 0) {
            k_cond_owners<<<scc_blocks(chunks + 1), SCC_THREADS, 0, st>>>(g->n, chunks, g->begin, own.as<int32_t>());
            // one resident wave: a grid-stride loop over chunks with a second
            // wave would leave its blocks a full share of chunks to run late
            int sms = 148, per = 1;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_cond_cross, SCC_THREADS, 0);
            k_cond_cross<<<(unsigned)std::min<int64_t>(chunks, (int64_t)sms * std::max(per, 1)), SCC_THREADS, 0, st>>>(
                (int32_t)g->m, chunks, g->begin, g->node_idx, lab.as<int32_t>(), own.as<int32_t>(),
                osrc.as<int32_t>(), odst.as<int32_t>(), count);
        }
        if (n_ins > 0) {
            cudaMemcpyAsync(bs.p, ins_src, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st);
            cudaMemcpyAsync(bd.p, ins_dst, sizeof(int32_t) * (size_t)n_ins, cudaMemcpyHostToDevice, st);
            k_cond_batch<<<scc_blocks(n_ins), SCC_THREADS, 0, st>>>(n_ins, bs.as<int32_t>(), bd.as<int32_t>(),
                                                                    lab.as<int32_t>(), g->n, osrc.as<int32_t>(),
                                                                    odst.as<int32_t>(), count, bad);
        }
        int h[2] = {0, 0};
        cudaError_t e = cudaPeekAtLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(h, ctr.p, 2 * sizeof(int), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) rc = scc_cuda_status(e, "condensation map", __FILE__, __LINE__);
        else if (h[0]) { scc_set_error("label or inserted endpoint out of range"); rc = SCC_ERR_INVALID; }
        else rc = scc_impl_build_graph_from_device_edges(num_sccs, h[1], osrc.as<int32_t>(), odst.as<int32_t>(),
                                                         SCC_BUILD_DEDUP | SCC_BUILD_NO_SELF_LOOPS, g->device, out);
    }
    }
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
    return rc;
}
