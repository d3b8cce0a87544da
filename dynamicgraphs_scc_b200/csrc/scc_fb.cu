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
#include <time.h>
#include <algorithm>
#include "scc_round.cuh"

static double trace_ms() {
    struct timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec * 1e3 + t.tv_nsec * 1e-6;
}

// Reset the per-colour pivot slots of the classes present and total the
// in+out degree of the vertices this round will traverse (the direction rule
// of the traversal compares frontier edges against it).  Lanes of a warp that
// share a class reset its slots once, and a thread skips the class it reset
// last, so a round over one huge class does not pile stores onto one address.
// Also the largest single degree (a hub keeps a round out of the
// asynchronous drain, whose warps would each expand it alone).
__device__ __forceinline__ void max_degree_add(int32_t* dst, unsigned d) {
    for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_down_sync(0xFFFFFFFFu, d, o));
    if ((threadIdx.x & 31) == 0 && d) atomicMax(dst, (int32_t)min(d, 0x7FFFFFFFu));
}

__global__ void k_slot_reset(RoundArgs a, int reset_slots) {
    unsigned long long deg = 0;
    unsigned dmax = 0;
    int32_t last = INT32_MIN;
    const int lane = threadIdx.x & 31;
    int64_t limit = (((int64_t)a.live_count + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t c = SCC_COLOR_DONE;
        if (i < a.live_count) {
            int32_t v = a.live[i];
            c = a.color[v];
            if (c != SCC_COLOR_DONE && !(a.use_only && c != a.only_color)) {
                unsigned dv = (unsigned)(__ldg(a.begin + v + 1) - __ldg(a.begin + v)) +
                              (unsigned)(__ldg(a.r_begin + v + 1) - __ldg(a.r_begin + v));
                deg += dv;
                dmax = max(dmax, dv);
            } else {
                c = SCC_COLOR_DONE;
            }
        }
        if (!reset_slots) continue;
        unsigned grp = __match_any_sync(0xFFFFFFFFu, c);
        if (c != SCC_COLOR_DONE && lane == __ffs(grp) - 1 && c != last) {
            a.slot_key[c + 1] = 0ull;
            a.slot_pivot[c + 1] = SCC_NIL_NODE;
            a.slot_count[c + 1] = 0;
            last = c;
        }
    }
    for (int o = 16; o > 0; o >>= 1) deg += __shfl_down_sync(0xFFFFFFFFu, deg, o);
    if ((threadIdx.x & 31) == 0 && deg)
        atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + CTR_LIVE_EDGES), deg);
    max_degree_add(a.ctr + CTR_MAXDEG, dmax);
}

// One class (the global step): its slots are the only ones to reset.
__global__ void k_slot_reset_one(RoundArgs a, int32_t c) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        a.slot_key[c + 1] = 0ull;
        a.slot_pivot[c + 1] = SCC_NIL_NODE;
        a.slot_count[c + 1] = 0;
    }
}

// Per-class maximum of the pivot keys.  A warp whose lanes all belong to one
// class reduces its keys first and issues one atomic.  The atomic that first
// raises a class's slot from zero (keys are never zero) lists the class, so the
// pivots are seeded from the list, not by another pass over the live vertices.
// sum_degrees: also total the in+out degree of the traversed vertices (what
// k_slot_reset does when the classes' slots need resetting first).
__global__ void k_pivot_key(RoundArgs a, int32_t* __restrict__ class_list, int32_t* __restrict__ class_count,
                            int sum_degrees) {
    const int lane = threadIdx.x & 31;
    unsigned long long deg = 0;
    unsigned dmax = 0;
    int64_t limit = (((int64_t)a.live_count + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t c = SCC_COLOR_DONE;
        unsigned long long k = 0ull;
        if (i < a.live_count) {
            int32_t v = a.live[i];
            c = a.color[v];
            if (c == SCC_COLOR_DONE || (a.use_only && c != a.only_color)) {
                c = SCC_COLOR_DONE;
            } else {
                unsigned outd = (unsigned)(__ldg(a.begin + v + 1) - __ldg(a.begin + v));
                unsigned ind = (unsigned)(__ldg(a.r_begin + v + 1) - __ldg(a.r_begin + v));
                unsigned long long prod = (unsigned long long)outd * ind;
                if (prod > 0xFFFFFFFEull) prod = 0xFFFFFFFEull;
                k = ((prod + 1ull) << 32) | pivot_hash((uint32_t)v ^ a.pivot_salt);
                deg += outd + ind;
                dmax = max(dmax, outd + ind);
            }
        }
        unsigned grp = __match_any_sync(0xFFFFFFFFu, c);
        if (grp == 0xFFFFFFFFu) {
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long other = __shfl_xor_sync(0xFFFFFFFFu, k, o);
                k = other > k ? other : k;
            }
            if (lane != 0) continue;
        }
        if (c != SCC_COLOR_DONE && k > a.slot_key[c + 1]) {
            if (atomicMax(a.slot_key + c + 1, k) == 0ull) class_list[atomicAdd(class_count, 1)] = c;
        }
    }
    if (sum_degrees) {
        for (int o = 16; o > 0; o >>= 1) deg += __shfl_down_sync(0xFFFFFFFFu, deg, o);
        if (lane == 0 && deg) atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + CTR_LIVE_EDGES), deg);
        max_degree_add(a.ctr + CTR_MAXDEG, dmax);
    }
}

// Each listed class pivots on the vertex its best key names.
__global__ void k_pivot_seed(RoundArgs a, const int32_t* __restrict__ class_list,
                             const int32_t* __restrict__ class_count, int32_t* q) {
    const int32_t nc = *class_count;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nc; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t c = class_list[i];
        seed_pivot(a, (int32_t)((uint32_t)pivot_unhash((uint32_t)a.slot_key[c + 1]) ^ a.pivot_salt), c, q);
    }
}

__global__ void k_pivot_forced(RoundArgs a, int32_t v, int32_t* q) {
    if (blockIdx.x == 0 && threadIdx.x == 0) seed_pivot(a, v, a.color[v], q);
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
    a.slot_count = s->slot_count;
    a.colour_cap = s->colour_cap;
    a.ctr = s->ctr;
    a.live = s->live; a.live_count = s->live_count;
    a.only_color = 0; a.use_only = 0;
    a.huge_deg = s->tune.huge_deg;
    a.async_keep = s->tune.async_keep;
    a.async_bail = std::max<int32_t>(8 * s->tune.async_max, 1 << 16);
    a.pivot_salt = (uint32_t)s->tune.pivot_salt;
    a.cta_deg = s->tune.cta_deg;
    round_args_adjacency(a, g->node_idx, g->r_node_idx, g->m);
    return a;
}

// One FW-BW round over every live class (only_color == INT32_MIN) or one class.
// Requires the live list.  *scc_found = vertices finished, *active = classes pivoted.
int scc_impl_fb_round(const scc_graph* g, scc_state* s, int32_t only_color, int32_t forced_pivot,
                      int32_t* scc_found, int32_t* active, bool pipeline) {
    *scc_found = 0;
    if (active) *active = 0;
    s->fresh = false;
    s->prefinished = false;
    if (s->live_count <= 0) return SCC_OK;
    // inside the pipeline the host counters are current here (the last step
    // synchronised them or set the colour counter itself); from the phase API
    // they are read again
    if (!pipeline) SCC_TRY(scc_sync_counters(s));
    SCC_TRY(scc_impl_ensure_colour_cap(s, (int64_t)s->h_ctr[CTR_NEXT_COLOR] + 2LL * s->live_count + 1024));
    RoundArgs a = round_args(g, s);
    a.use_only = (only_color != INT32_MIN);
    a.only_color = only_color;
    unsigned blocks = scc_blocks(s->live_count);
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 4));
    SCC_TRY(scc_zero_counters(s, CTR_NUM_CLASSES, 1));
    SCC_TRY(scc_zero_counters(s, CTR_LIVE_EDGES, 2));
    SCC_TRY(scc_zero_counters(s, CTR_MAXDEG, 1));
    // one class: reset its slots alone and total the degrees in the key pass
    const bool one_class = a.use_only && forced_pivot < 0;
    if (one_class) {
        k_slot_reset_one<<<1, 32, 0, s->stream>>>(a, only_color);
    } else {
        k_slot_reset<<<blocks, SCC_THREADS, 0, s->stream>>>(a, forced_pivot < 0 ? 1 : 0);
    }
    SCC_LAUNCHED(s);
    if (forced_pivot >= 0) {
        k_pivot_forced<<<1, 32, 0, s->stream>>>(a, forced_pivot, s->qa);
        SCC_LAUNCHED(s);
    } else {
        // the class list lives in hq (free until the traversal), its length in CTR_SPARE4
        int32_t* nclass = s->ctr + CTR_SPARE4;
        SCC_TRY(scc_zero_counters(s, CTR_SPARE4, 1));
        k_pivot_key<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->hq, nclass, one_class ? 1 : 0);
        SCC_LAUNCHED(s);
        const bool learned = s->pivot_mode == SCC_PIVOT_LEARNED && s->pivot_model;
        bool seeded = false;
        if (learned || s->log_cap > 0) SCC_TRY(scc_impl_pivot_prepare(g, s, a, learned, s->qa, &seeded));
        if (!seeded) {
            k_pivot_seed<<<scc_blocks(s->live_count, SCC_THREADS, 148 * 4), SCC_THREADS, 0, s->stream>>>(a, s->hq, nclass,
                                                                                                     s->qa);
            SCC_LAUNCHED(s);
        }
    }
    SCC_TRY(scc_sync_counters(s));
    if (s->h_ctr[CTR_ERROR]) SCC_TRY(scc_check_device_error(s));
    int32_t qlen = s->h_ctr[CTR_QLEN];
    if (active) *active = s->h_ctr[CTR_NUM_CLASSES];
    SCC_TRY(scc_impl_reach(g, s, a, qlen));
    SCC_TRY(scc_zero_counters(s, CTR_COUNT, 3));
    k_classify<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
    SCC_LAUNCHED(s);
    if (pipeline) {
        // the caller's compaction synchronises next; it leaves CTR_COUNT alone
        *scc_found = -1;
        return SCC_OK;
    }
    SCC_TRY(scc_sync_counters(s));
    *scc_found = s->h_ctr[CTR_COUNT];
    return SCC_OK;
}

// Resolve every live class to SCCs: trim, FW-BW round, repeat (the device
// replacement for start_workers_fw_bw[_dfs], src/scc_fb_seq2.cc:292-351).
// Each round: peel (trim1 inside colours), split every class into its weak
// components (so independent pieces get their own pivot), then one FW-BW
// round over all classes at once.  Every class loses at least its pivot's SCC
// per round, so the loop ends.
int scc_impl_resolve_all(const scc_graph* g, scc_state* s, bool classes_split) {
    if (s->live_count < 0) SCC_TRY(scc_impl_compact_live(g, s, true));
    double t_round = scc_trace_on() ? trace_ms() : 0.0;
    for (int round = 0; round < (1 << 30); ++round) {
        int32_t t = 0;
        int32_t classes = 0;
        if (round >= 1 && s->tune.tail_live > 0 && s->live_count <= s->tune.tail_live &&
            s->pivot_mode == SCC_PIVOT_DEGREE && s->log_cap == 0) {
            // few vertices left: every class in one launch, a block per class
            bool taken = false;
            SCC_TRY(scc_impl_resolve_tail(g, s, &taken));
            if (taken) break;
        }
        if (round == 0 && classes_split) {
            // the caller peeled to the fixpoint, compacted, then split: a split
            // only recolours weakly disconnected parts, so no live vertex loses
            // a same-colour neighbour and this round's peel would find nothing
            classes = -1;
        } else {
            SCC_TRY(scc_impl_trim1(g, s, true, &t));
            SCC_TRY(scc_impl_compact_live(g, s, false));
            if (s->live_count == 0) break;
            SCC_TRY(scc_impl_uf_split(g, s, &classes));
        }
        int32_t live_before = s->live_count;
        int32_t found = 0, act = 0;
        SCC_TRY(scc_impl_fb_round(g, s, INT32_MIN, -1, &found, &act, true));
        SCC_TRY(scc_impl_compact_live(g, s, false));   // synchronises: classify's count is current
        found = s->h_ctr[CTR_COUNT];
        if (scc_trace_on()) {
            double t1 = trace_ms();
            fprintf(stderr, "[scc] round %d: trimmed=%d live=%d classes=%d scc_found=%d left=%d %.3f ms\n", round, t,
                    live_before, classes, found, s->live_count, t1 - t_round);
            t_round = t1;
        }
        s->fb_rounds++;
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
        SCC_TRY(scc_zero_counters(s, CTR_SPARE4, 1));     // the key pass lists the class in hq
        k_pivot_key<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->hq, s->ctr + CTR_SPARE4, 0);
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
