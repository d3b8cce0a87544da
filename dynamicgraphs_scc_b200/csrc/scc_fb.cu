// FW-BW: pivot selection, forward/backward reachability inside colour classes,
// and the split of every class into SCC / FW-only / BW-only / rest.
//
// Reference: do_fw_bw_global_main (src/scc_fb_global.cc:133-219) runs a FW
// BFS from one pivot over vertices of the base colour (navigator
// fw_trim_global::check_navigator, :65-68), then a BW BFS over the transpose
// over {fw, base} colours (:124-128): intersection -> SCC (scc = pivot, colour
// -2), BW-only -> bw colour.  The per-class recursion (do_fw_bw_dfs,
// src/scc_fb_seq2.cc:180-289) does the same inside each work item.
//
// Here one device round handles every live colour class at once: each class
// picks its pivot (largest in-degree x out-degree, ties by a fixed id hash),
// FW and BW reachability run in the same frontier (items tagged with their
// direction, visited bits in a byte per vertex), and a classify pass gives
// each class the reference's outcome.  A single class (curr_color) is the
// global step.
#include "scc_internal.cuh"

#define DIR_SHIFT 30
#define ITEM_MASK 0x3FFFFFFF
#define WBUF 256          // per-warp push buffer (shared memory)
#define REACH_THREADS 256

__device__ __forceinline__ uint32_t pivot_hash(uint32_t v) {
    uint32_t x = v * 0x9E3779B1u;
    x ^= x >> 16; x *= 0x85EBCA6Bu; x ^= x >> 13;
    return x;
}

// Pivot key: (min(in*out, 2^32-2)+1) << 32 | hash(v); never 0, unique per vertex.
__device__ __forceinline__ unsigned long long pivot_key(const int32_t* __restrict__ begin,
                                                        const int32_t* __restrict__ r_begin, int32_t v) {
    unsigned long long outd = (unsigned)(__ldg(begin + v + 1) - __ldg(begin + v));
    unsigned long long ind = (unsigned)(__ldg(r_begin + v + 1) - __ldg(r_begin + v));
    unsigned long long prod = outd * ind;
    if (prod > 0xFFFFFFFEull) prod = 0xFFFFFFFEull;
    return ((prod + 1ull) << 32) | pivot_hash((uint32_t)v);
}

struct RoundArgs {
    const int32_t* begin; const int32_t* node_idx; const int32_t* r_begin; const int32_t* r_node_idx;
    int32_t* color; int32_t* scc; uint8_t* mark;
    unsigned long long* slot_key; int32_t* slot_pivot; int32_t* slot_fw; int32_t* slot_bw;
    int64_t colour_cap;
    int32_t* ctr;
    const int32_t* live; int32_t live_count;
    int32_t only_color;   // INT32_MIN = every class
    int32_t use_only;
};

__global__ void k_slot_reset(RoundArgs a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.live_count; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = a.live[i];
        int32_t c = a.color[v];
        if (c == SCC_COLOR_DONE) continue;
        a.slot_key[c + 1] = 0ull;
        a.slot_pivot[c + 1] = SCC_NIL_NODE;
    }
}

__global__ void k_pivot_key(RoundArgs a) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.live_count; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = a.live[i];
        int32_t c = a.color[v];
        if (c == SCC_COLOR_DONE || (a.use_only && c != a.only_color)) continue;
        unsigned long long k = pivot_key(a.begin, a.r_begin, v);
        if (k > a.slot_key[c + 1]) atomicMax(a.slot_key + c + 1, k);
    }
}

// The pivot of each class claims two fresh colours and seeds the frontier.
__device__ __forceinline__ void seed_pivot(const RoundArgs& a, int32_t v, int32_t c, int32_t* q) {
    a.slot_pivot[c + 1] = v;
    int32_t old = atomicAdd(a.ctr + CTR_NEXT_COLOR, 2);
    if ((int64_t)old + 4 >= a.colour_cap) { atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_COLOR_OVERFLOW); }
    a.slot_fw[c + 1] = old + 1;
    a.slot_bw[c + 1] = old + 2;
    a.mark[v] = 3;
    int32_t pos = atomicAdd(a.ctr + CTR_QLEN, 2);
    q[pos] = v;
    q[pos + 1] = v | (1 << DIR_SHIFT);
    atomicAdd(a.ctr + CTR_NUM_CLASSES, 1);
}

__global__ void k_pivot_pick(RoundArgs a, int32_t* q) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.live_count; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = a.live[i];
        int32_t c = a.color[v];
        if (c == SCC_COLOR_DONE || (a.use_only && c != a.only_color)) continue;
        if (pivot_key(a.begin, a.r_begin, v) == a.slot_key[c + 1]) seed_pivot(a, v, c, q);
    }
}

__global__ void k_pivot_forced(RoundArgs a, int32_t v, int32_t* q) {
    if (blockIdx.x == 0 && threadIdx.x == 0) seed_pivot(a, v, a.color[v], q);
}

// ------------------------------------------------------------------ one BFS level
struct WarpPush {
    int32_t* buf;     // this warp's shared buffer
    int32_t count;    // warp-uniform
};

__device__ __forceinline__ void warp_flush(WarpPush& wp, int32_t* __restrict__ qout, int32_t* __restrict__ qlen) {
    int lane = threadIdx.x & 31;
    __syncwarp();
    if (wp.count > 0) {
        int32_t base = 0;
        if (lane == 0) base = atomicAdd(qlen, wp.count);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        for (int j = lane; j < wp.count; j += 32) qout[base + j] = wp.buf[j];
    }
    __syncwarp();
    wp.count = 0;
}

__device__ __forceinline__ void warp_push(WarpPush& wp, bool p, int32_t item, int32_t* __restrict__ qout,
                                          int32_t* __restrict__ qlen) {
    int lane = threadIdx.x & 31;
    unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
    if (p) wp.buf[wp.count + __popc(bal & ((1u << lane) - 1u))] = item;
    wp.count += __popc(bal);
    if (wp.count > WBUF - 32) warp_flush(wp, qout, qlen);
}

// Claim w for direction `dir` inside colour c; true if this thread claimed it.
__device__ __forceinline__ bool visit(const RoundArgs& a, int32_t w, int32_t c, int dir) {
    unsigned bit = 1u << dir;
    if (a.mark[w] & bit) return false;
    if (__ldg(a.color + w) != c) return false;
    unsigned sh = (unsigned)(w & 3) * 8u;
    unsigned old = atomicOr(reinterpret_cast<unsigned*>(a.mark + (w & ~3)), bit << sh);
    return ((old >> sh) & bit) == 0u;
}

__global__ void __launch_bounds__(REACH_THREADS) k_reach_level(RoundArgs a, const int32_t* __restrict__ qin,
                                                                int32_t nin, int32_t* __restrict__ qout) {
    __shared__ int32_t sbuf[REACH_THREADS / 32][WBUF];
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpPush wp{sbuf[wid], 0};
    int32_t* qlen = a.ctr + CTR_QLEN;
    int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
    int64_t groups = ((int64_t)nin + 31) >> 5;
    for (int64_t gi = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; gi < groups; gi += nwarps) {
        int64_t idx = gi * 32 + lane;
        int32_t v = 0, dir = 0, b = 0, e = 0, c = 0;
        if (idx < nin) {
            int32_t it = qin[idx];
            v = it & ITEM_MASK;
            dir = (it >> DIR_SHIFT) & 1;
            const int32_t* off = dir ? a.r_begin : a.begin;
            b = __ldg(off + v);
            e = __ldg(off + v + 1);
            c = __ldg(a.color + v);
        }
        int32_t deg = e - b;
        // high-degree vertices: the whole warp strides the adjacency
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
                warp_push(wp, p, w | (bd << DIR_SHIFT), qout, qlen);
            }
        }
        // low-degree vertices: each lane walks its own list, warp-uniform trip count
        int32_t mydeg = deg <= 32 ? deg : 0;
        int32_t maxd = __reduce_max_sync(0xFFFFFFFFu, (unsigned)mydeg);
        const int32_t* adj = dir ? a.r_node_idx : a.node_idx;
        for (int32_t j = 0; j < maxd; ++j) {
            bool p = false;
            int32_t w = 0;
            if (j < mydeg) { w = __ldg(adj + b + j); p = visit(a, w, c, dir); }
            warp_push(wp, p, w | (dir << DIR_SHIFT), qout, qlen);
        }
    }
    warp_flush(wp, qout, qlen);
}

// ------------------------------------------------------------------ classify
// FW&BW -> SCC (scc = pivot of the class), FW only -> fw colour, BW only -> bw
// colour, neither -> unchanged.  Marks are cleared for the next round.
__global__ void k_classify(RoundArgs a) {
    int32_t n_scc = 0, n_fw = 0, n_bw = 0;
    int64_t limit = (((int64_t)a.live_count + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        if (i < a.live_count) {
            int32_t v = a.live[i];
            uint8_t m = a.mark[v];
            if (m) {
                int32_t c = a.color[v];
                if ((m & 3) == 3) { a.scc[v] = a.slot_pivot[c + 1]; a.color[v] = SCC_COLOR_DONE; n_scc++; }
                else if (m & 1) { a.color[v] = a.slot_fw[c + 1]; n_fw++; }
                else { a.color[v] = a.slot_bw[c + 1]; n_bw++; }
                a.mark[v] = 0;
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        n_scc += __shfl_down_sync(0xFFFFFFFFu, n_scc, o);
        n_fw += __shfl_down_sync(0xFFFFFFFFu, n_fw, o);
        n_bw += __shfl_down_sync(0xFFFFFFFFu, n_bw, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (n_scc) atomicAdd(a.ctr + CTR_COUNT, n_scc);
        if (n_fw) atomicAdd(a.ctr + CTR_COUNT2, n_fw);
        if (n_bw) atomicAdd(a.ctr + CTR_COUNT3, n_bw);
    }
}

static RoundArgs round_args(const scc_graph* g, scc_state* s) {
    RoundArgs a;
    a.begin = g->begin; a.node_idx = g->node_idx; a.r_begin = g->r_begin; a.r_node_idx = g->r_node_idx;
    a.color = s->color; a.scc = s->scc; a.mark = s->mark;
    a.slot_key = s->slot_key; a.slot_pivot = s->slot_pivot; a.slot_fw = s->slot_fw; a.slot_bw = s->slot_bw;
    a.colour_cap = s->colour_cap;
    a.ctr = s->ctr;
    a.live = s->live; a.live_count = s->live_count;
    a.only_color = 0; a.use_only = 0;
    return a;
}

// Run reachability from the queue in s->qa (length qlen) to completion.
static int reach_to_completion(const scc_graph* g, scc_state* s, RoundArgs& a, int32_t qlen) {
    int32_t* qin = s->qa;
    int32_t* qout = s->qb;
    while (qlen > 0) {
        SCC_TRY(scc_zero_counters(s, CTR_QLEN, 1));
        unsigned blocks = scc_blocks((int64_t)qlen, REACH_THREADS, 148 * 8);
        k_reach_level<<<blocks, REACH_THREADS, 0, s->stream>>>(a, qin, qlen, qout);
        SCC_LAUNCHED(s);
        s->traversal_steps++;
        SCC_TRY(scc_sync_counters(s));
        qlen = s->h_ctr[CTR_QLEN];
        int32_t* t = qin; qin = qout; qout = t;
    }
    return SCC_OK;
}

// One FW-BW round over every live class (only_color == INT32_MIN) or one class.
// Requires the live list.  *scc_found = vertices finished, *active = classes pivoted.
int scc_impl_fb_round(const scc_graph* g, scc_state* s, int32_t only_color, int32_t forced_pivot,
                      int32_t* scc_found, int32_t* active) {
    *scc_found = 0;
    if (active) *active = 0;
    if (s->live_count <= 0) return SCC_OK;
    SCC_TRY(scc_sync_counters(s));
    SCC_TRY(scc_impl_ensure_colour_cap(s, (int64_t)s->h_ctr[CTR_NEXT_COLOR] + 2LL * s->live_count + 1024));
    RoundArgs a = round_args(g, s);
    a.use_only = (only_color != INT32_MIN);
    a.only_color = only_color;
    unsigned blocks = scc_blocks(s->live_count);
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 4));
    SCC_TRY(scc_zero_counters(s, CTR_NUM_CLASSES, 1));
    if (forced_pivot >= 0) {
        k_pivot_forced<<<1, 32, 0, s->stream>>>(a, forced_pivot, s->qa);
        SCC_LAUNCHED(s);
    } else {
        k_slot_reset<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
        SCC_LAUNCHED(s);
        k_pivot_key<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
        SCC_LAUNCHED(s);
        k_pivot_pick<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->qa);
        SCC_LAUNCHED(s);
    }
    SCC_TRY(scc_sync_counters(s));
    if (s->h_ctr[CTR_ERROR]) SCC_TRY(scc_check_device_error(s));
    int32_t qlen = s->h_ctr[CTR_QLEN];
    if (active) *active = s->h_ctr[CTR_NUM_CLASSES];
    SCC_TRY(reach_to_completion(g, s, a, qlen));
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 3));
    k_classify<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
    SCC_LAUNCHED(s);
    SCC_TRY(scc_sync_counters(s));
    *scc_found = s->h_ctr[CTR_COUNT];
    return SCC_OK;
}

// Resolve every live class to SCCs: trim, FW-BW round, repeat (the device
// replacement for start_workers_fw_bw[_dfs], src/scc_fb_seq2.cc:292-351).
int scc_impl_resolve_all(const scc_graph* g, scc_state* s) {
    if (s->live_count < 0) SCC_TRY(scc_impl_compact_live(g, s, true));
    for (int round = 0; round < (1 << 30); ++round) {
        int32_t t = 0;
        SCC_TRY(scc_impl_trim1(g, s, true, &t));
        SCC_TRY(scc_impl_compact_live(g, s, false));
        if (s->live_count == 0) break;
        int32_t found = 0, act = 0;
        SCC_TRY(scc_impl_fb_round(g, s, INT32_MIN, -1, &found, &act));
        SCC_TRY(scc_impl_compact_live(g, s, false));
        if (s->live_count == 0) break;
        if (found == 0) { scc_set_error("FW-BW round made no progress"); return SCC_ERR_STATE; }
    }
    s->wq_colors.clear();
    s->wq_counts.clear();
    return SCC_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" int scc_choose_pivot_from_color(const scc_graph* g, scc_state* s, int32_t color, int32_t* pivot) {
    SCC_REQUIRE(g && s && pivot, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    *pivot = SCC_NIL_NODE;
    if (s->live_count < 0) SCC_TRY(scc_impl_compact_live(g, s, true));
    SCC_REQUIRE(color >= -1 && (int64_t)color + 1 < s->colour_cap, SCC_ERR_INVALID, "colour %d out of range", color);
    RoundArgs a = round_args(g, s);
    a.use_only = 1;
    a.only_color = color;
    unsigned blocks = scc_blocks(s->live_count);
    unsigned long long zero = 0;
    SCC_CUDA(cudaMemcpyAsync(s->slot_key + color + 1, &zero, sizeof(zero), cudaMemcpyHostToDevice, s->stream));
    if (s->live_count > 0) {
        k_pivot_key<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
        SCC_LAUNCHED(s);
    }
    unsigned long long key = 0;
    SCC_CUDA(cudaMemcpyAsync(&key, s->slot_key + color + 1, sizeof(key), cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    if (key == 0) return SCC_ERR_NOT_FOUND;
    // invert the hash over the candidates: find the member whose key matches
    std::vector<int32_t> live;
    SCC_TRY(scc_impl_get_live_host(s, live));
    std::vector<int32_t> col((size_t)s->n);
    SCC_TRY(scc_state_get_color(s, col.data()));
    std::vector<int32_t> b((size_t)g->n + 1), rb((size_t)g->n + 1);
    SCC_TRY(scc_graph_copy_csr(g, b.data(), nullptr, rb.data(), nullptr));
    for (int32_t v : live) {
        if (col[v] != color) continue;
        unsigned long long outd = (unsigned)(b[v + 1] - b[v]), ind = (unsigned)(rb[v + 1] - rb[v]);
        unsigned long long prod = outd * ind;
        if (prod > 0xFFFFFFFEull) prod = 0xFFFFFFFEull;
        uint32_t x = (uint32_t)v * 0x9E3779B1u;
        x ^= x >> 16; x *= 0x85EBCA6Bu; x ^= x >> 13;
        if ((((prod + 1ull) << 32) | x) == key) { *pivot = v; return SCC_OK; }
    }
    return SCC_ERR_NOT_FOUND;
}

static int fw_bw_global(const scc_graph* g, scc_state* s, int32_t curr_color, int32_t pivot, int create_work_items,
                        int32_t* scc_size) {
    SCC_CUDA(cudaSetDevice(s->device));
    if (s->live_count < 0) SCC_TRY(scc_impl_compact_live(g, s, true));
    int32_t found = 0, act = 0;
    SCC_TRY(scc_impl_fb_round(g, s, curr_color, pivot, &found, &act));
    SCC_REQUIRE(act > 0, SCC_ERR_NOT_FOUND, "no vertex of colour %d", curr_color);
    int32_t fw = s->h_ctr[CTR_COUNT2], bw = s->h_ctr[CTR_COUNT3];
    if (scc_size) *scc_size = found;
    s->wq_colors.clear();
    s->wq_counts.clear();
    if (create_work_items) {
        // scc_fb_global.cc:188-216: fw, bw, base items
        SCC_TRY(scc_sync_counters(s));
        int32_t last = s->h_ctr[CTR_NEXT_COLOR];
        int32_t base_count = 0;
        SCC_TRY(scc_impl_count_colour(s, curr_color, &base_count));
        if (fw > 0) { s->wq_colors.push_back(last - 1); s->wq_counts.push_back(fw); }
        if (bw > 0) { s->wq_colors.push_back(last); s->wq_counts.push_back(bw); }
        if (base_count > 0) { s->wq_colors.push_back(curr_color); s->wq_counts.push_back(base_count); }
    }
    return SCC_OK;
}

extern "C" int scc_do_fw_bw_global_main(const scc_graph* g, scc_state* s, int32_t curr_color, int32_t count,
                                        int create_work_items, int32_t* scc_size) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    (void)count;
    return fw_bw_global(g, s, curr_color, -1, create_work_items, scc_size);
}

extern "C" int scc_do_fw_bw_global_pivot(const scc_graph* g, scc_state* s, int32_t curr_color, int32_t pivot,
                                         int create_work_items, int32_t* scc_size) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(pivot >= 0 && pivot < g->n, SCC_ERR_INVALID, "pivot %d out of range", pivot);
    std::vector<int32_t> c1(1);
    SCC_CUDA(cudaMemcpy(c1.data(), s->color + pivot, sizeof(int32_t), cudaMemcpyDeviceToHost));
    SCC_REQUIRE(c1[0] == curr_color, SCC_ERR_INVALID, "pivot %d has colour %d, not %d", pivot, c1[0], curr_color);
    return fw_bw_global(g, s, curr_color, pivot, create_work_items, scc_size);
}

extern "C" int scc_create_works_after_bfs_trim(const scc_graph* g, scc_state* s, int32_t* num_items) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    // classes of the live list (scc_fb_global.cc:223-283 counts fw/bw/base over the compact targets)
    if (s->live_count < 0) SCC_TRY(scc_impl_compact_live(g, s, true));
    SCC_TRY(scc_sync_counters(s));
    int32_t last = s->h_ctr[CTR_NEXT_COLOR];
    s->wq_colors.clear();
    s->wq_counts.clear();
    int32_t cand[3] = {last - 1, last, SCC_COLOR_INIT};
    for (int i = 0; i < 3; ++i) {
        if (cand[i] < -1) continue;
        int32_t c = 0;
        SCC_TRY(scc_impl_count_colour(s, cand[i], &c));
        if (c > 0) { s->wq_colors.push_back(cand[i]); s->wq_counts.push_back(c); }
    }
    if (num_items) *num_items = (int32_t)s->wq_colors.size();
    return SCC_OK;
}

extern "C" int scc_start_workers_fw_bw(const scc_graph* g, scc_state* s, int32_t local_items) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    (void)local_items;
    SCC_CUDA(cudaSetDevice(s->device));
    return scc_impl_resolve_all(g, s);
}

extern "C" int scc_start_workers_fw_bw_dfs(const scc_graph* g, scc_state* s, int32_t local_items) {
    return scc_start_workers_fw_bw(g, s, local_items);
}

extern "C" int scc_work_q_size(scc_state* s, int32_t* size) {
    SCC_REQUIRE(s && size, SCC_ERR_INVALID, "NULL argument");
    *size = (int32_t)s->wq_colors.size();
    return SCC_OK;
}

extern "C" int scc_work_q_items(scc_state* s, int32_t* colors, int32_t* counts, int32_t capacity, int32_t* num_items) {
    SCC_REQUIRE(s && num_items, SCC_ERR_INVALID, "NULL argument");
    int32_t k = (int32_t)s->wq_colors.size();
    *num_items = k;
    if (colors || counts) {
        SCC_REQUIRE(capacity >= k, SCC_ERR_INVALID, "capacity %d < %d items", capacity, k);
        for (int32_t i = 0; i < k; ++i) {
            if (colors) colors[i] = s->wq_colors[i];
            if (counts) counts[i] = s->wq_counts[i];
        }
    }
    return SCC_OK;
}
