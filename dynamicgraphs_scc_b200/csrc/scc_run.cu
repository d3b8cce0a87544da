// Driver pipeline (my_main::run, src/scc_main.cc:120-145 and the method bodies
// :282-444), SCC counting (post_process, :147-178), canonical labels, and the
// scc_list.txt / histogram outputs (src/scc_post_analyze.cc:31-82, 235-261).
#include <algorithm>
#include <map>
#include <string.h>
#include <nvtx3/nvToolsExt.h>
#include "scc_internal.cuh"

// ------------------------------------------------------------------ kernels
__global__ void k_count_roots(int32_t n, const int32_t* __restrict__ scc, int32_t* __restrict__ out) {
    int32_t c = 0;
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x)
        if (i < n && scc[i] == (int32_t)i) c++;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_down_sync(0xFFFFFFFFu, c, o);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

// minm[rep] = smallest member; warps first reduce lanes that share a representative.
__global__ void k_min_member(int32_t n, const int32_t* __restrict__ scc, int32_t* __restrict__ minm) {
    int64_t limit = (((int64_t)n + 31) / 32) * 32;
    int lane = threadIdx.x & 31;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = (int32_t)i;
        int32_t r = (i < n) ? scc[v] : -1;
        unsigned grp = __match_any_sync(0xFFFFFFFFu, r);
        int leader = __ffs(grp) - 1;   // lowest lane = smallest v of the group in this warp
        if (lane == leader && r >= 0) {
            if (__ldcg(minm + r) > v) atomicMin(minm + r, v);
        }
    }
}

__global__ void k_apply_min(int32_t n, const int32_t* __restrict__ scc, const int32_t* __restrict__ minm,
                            int32_t* __restrict__ out) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t r = scc[i];
        out[i] = r >= 0 ? minm[r] : -1;
    }
}

__global__ void k_fill(int64_t n, int32_t* __restrict__ a, int32_t v) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = v;
}

// ------------------------------------------------------------------ helpers
static int canonical_into(scc_state* s, int32_t* d_out) {
    int32_t n = s->n;
    if (n == 0) return SCC_OK;
    int32_t* minm = s->aux;
    k_fill<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, minm, INT32_MAX);
    SCC_LAUNCHED(s);
    k_min_member<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, s->scc, minm);
    SCC_LAUNCHED(s);
    k_apply_min<<<scc_blocks(n), SCC_THREADS, 0, s->stream>>>(n, s->scc, minm, d_out);
    SCC_LAUNCHED(s);
    return SCC_OK;
}

// Phase markers: a CUDA event on the state's stream (the run statistics) and
// an NVTX range per phase for profilers, named like the reference's -d output.
static const char* const kPhase[5] = {"TRIM1", "GLOBAL_FW_BW", "TRIM1_TRIM2", "WCC", "FW_BW"};
static thread_local int t_nvtx_open = 0;

static int record(scc_state* s, int i) {
    SCC_CUDA(cudaEventRecord(s->ev[i], s->stream));
    if (t_nvtx_open) { nvtxRangePop(); t_nvtx_open = 0; }
    if (i < 5) { nvtxRangePushA(kPhase[i]); t_nvtx_open = 1; }
    return SCC_OK;
}
static double elapsed(scc_state* s, int a, int b) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, s->ev[a], s->ev[b]) != cudaSuccess) { cudaGetLastError(); return 0.0; }
    return (double)ms;
}

// ------------------------------------------------------------------ pipeline
static int run_method(const scc_graph* g, scc_state* s, int method, scc_run_stats* st) {
    int32_t t = 0;
    // TRIM1: repeat_global_trim1 then the compact list (scc_main.cc:369 / :288 / :319)
    SCC_TRY(record(s, 0));
    SCC_TRY(scc_impl_trim1(g, s, false, &t));
    st->trimmed_first = t;
    SCC_TRY(scc_impl_compact_live(g, s, true));
    SCC_TRY(record(s, 1));
    if (s->live_count == 0 || method == SCC_METHOD_BASELINE) {
        // method 0: one work item of colour -1 resolved by the FB workers (scc_main.cc:301-311)
        SCC_TRY(record(s, 2));
        SCC_TRY(record(s, 3));
        SCC_TRY(record(s, 4));
        if (s->live_count > 0) SCC_TRY(scc_impl_resolve_all(g, s));
        SCC_TRY(record(s, 5));
        return SCC_OK;
    }
    // GLOBAL_BFS: do_fw_bw_global_main(G, -1, count, false)
    int32_t found = 0, act = 0;
    SCC_TRY(scc_impl_fb_round(g, s, SCC_COLOR_INIT, -1, &found, &act, true));
    SCC_TRY(record(s, 2));
    // TRIM1 (+ TRIM2 + TRIM1 for method 2, scc_main.cc:410-423)
    SCC_TRY(scc_impl_compact_live(g, s, false));   // synchronises: classify's count is current
    st->first_scc_size = s->h_ctr[CTR_COUNT];
    int32_t t2 = 0;
    SCC_TRY(scc_impl_trim1(g, s, true, &t));
    t2 += t;
    if (method == SCC_METHOD_GLOBAL_WCC_FB) {
        SCC_TRY(scc_impl_compact_live(g, s, false));
        SCC_TRY(scc_impl_trim2(g, s, &t));
        t2 += t;
        SCC_TRY(scc_impl_trim1(g, s, true, &t));
        t2 += t;
    }
    SCC_TRY(scc_impl_compact_live(g, s, false));
    st->trimmed_second = t2;
    SCC_TRY(record(s, 3));
    if (s->live_count > 0 && method == SCC_METHOD_GLOBAL_WCC_FB) {
        // WCC: colour the remainder into independent classes (create_work_items_from_wcc).
        // The pipeline splits by weak components (union-find, a few passes whatever
        // the diameter); the min-reach colouring of do_global_wcc is offered unchanged
        // as scc_do_global_wcc.  Both give unions of SCCs, so the labels are the same.
        int32_t classes = 0;
        SCC_TRY(scc_impl_uf_split(g, s, &classes));
        st->num_wcc_classes = classes;
    }
    SCC_TRY(record(s, 4));
    // FB: start_workers_fw_bw_dfs
    if (s->live_count > 0) SCC_TRY(scc_impl_resolve_all(g, s, method == SCC_METHOD_GLOBAL_WCC_FB));
    SCC_TRY(record(s, 5));
    return SCC_OK;
}

extern "C" int scc_run(const scc_graph* g, scc_state* s, int method, int pivot_mode, scc_run_stats* stats) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(s->n == g->n, SCC_ERR_INVALID, "state built for n=%d, graph has n=%d", s->n, g->n);
    if (method >= 5 && method <= 11) method = SCC_METHOD_GLOBAL_WCC_FB;   // scc_main.cc:170-171
    if (method == 3 || method == 4) {
        scc_set_error("method %d (Tarjan) is the sequential oracle and is not offered by the GPU engine", method);
        return SCC_ERR_UNSUPPORTED;
    }
    SCC_REQUIRE(method >= 0 && method <= 2, SCC_ERR_INVALID, "method %d outside 0..11", method);
    SCC_REQUIRE(pivot_mode == SCC_PIVOT_DEGREE || pivot_mode == SCC_PIVOT_LEARNED, SCC_ERR_INVALID,
                "unknown pivot mode %d", pivot_mode);
    SCC_CUDA(cudaSetDevice(s->device));
    scc_run_stats st;
    memset(&st, 0, sizeof(st));
    st.pivot_mode = pivot_mode;
    int k0 = s->kernels;
    int64_t steps0 = s->traversal_steps;
    int32_t rounds0 = s->fb_rounds;
    if (pivot_mode == SCC_PIVOT_LEARNED)
        SCC_REQUIRE(s->pivot_model, SCC_ERR_INVALID, "learned pivots need a model (scc_state_set_pivot_model)");
    s->pivot_mode = pivot_mode;
    nvtxRangePushA("scc_run");
    int rc = run_method(g, s, method, &st);
    if (t_nvtx_open) { nvtxRangePop(); t_nvtx_open = 0; }
    nvtxRangePop();
    s->pivot_mode = SCC_PIVOT_DEGREE;
    if (rc != SCC_OK) return rc;
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    SCC_TRY(scc_check_device_error(s));
    st.ms_trim1 = elapsed(s, 0, 1);
    st.ms_global_fb = elapsed(s, 1, 2);
    st.ms_trim12 = elapsed(s, 2, 3);
    st.ms_wcc = elapsed(s, 3, 4);
    st.ms_fb = elapsed(s, 4, 5);
    st.ms_total = elapsed(s, 0, 5);
    st.kernels_launched = s->kernels - k0;
    st.traversal_steps = s->traversal_steps - steps0;
    st.fb_rounds = s->fb_rounds - rounds0;
    int32_t nscc = 0;
    SCC_TRY(scc_count_sccs(s, &nscc));
    st.num_sccs = nscc;
    if (stats) *stats = st;
    return SCC_OK;
}

extern "C" int scc_count_sccs(scc_state* s, int32_t* count) {
    SCC_REQUIRE(s && count, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    SCC_TRY(scc_zero_counters(s, CTR_SPARE0, 1));
    if (s->n > 0) {
        k_count_roots<<<scc_blocks(s->n), SCC_THREADS, 0, s->stream>>>(s->n, s->scc, s->ctr + CTR_SPARE0);
        SCC_LAUNCHED(s);
    }
    SCC_TRY(scc_sync_counters(s));
    *count = s->h_ctr[CTR_SPARE0];
    return SCC_OK;
}

extern "C" int scc_canonical_labels_device(scc_state* s, int32_t* d_labels) {
    SCC_REQUIRE(s && d_labels, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    SCC_TRY(canonical_into(s, d_labels));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}

extern "C" int scc_canonical_labels(scc_state* s, int32_t* labels) {
    SCC_REQUIRE(s && labels, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(s->device));
    if (s->n == 0) return SCC_OK;
    SCC_TRY(canonical_into(s, s->live_tmp));
    SCC_CUDA(cudaMemcpyAsync(labels, s->live_tmp, sizeof(int32_t) * (size_t)s->n, cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}

// output_scc_list: "i id" with ids numbered by first appearance over i.
extern "C" int scc_output_scc_list(scc_state* s, const char* path) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    const char* p = path ? path : "scc_list.txt";
    std::vector<int32_t> rep((size_t)s->n);
    SCC_TRY(scc_state_get_scc(s, rep.data()));
    FILE* f = fopen(p, "w");
    SCC_REQUIRE(f, SCC_ERR_IO, "Error: Cannot open scc_list output file %s", p);
    std::vector<int32_t> id((size_t)s->n, -1);
    int32_t next = 0;
    std::vector<char> line(32);
    for (int32_t i = 0; i < s->n; ++i) {
        int32_t r = rep[i];
        int32_t k;
        if (r >= 0 && r < s->n) {
            if (id[r] < 0) id[r] = next++;
            k = id[r];
        } else {
            k = next++;   // unfinished vertex: its own id
        }
        fprintf(f, "%d %d\n", i, k);
    }
    int bad = ferror(f);
    fclose(f);
    SCC_REQUIRE(!bad, SCC_ERR_IO, "write error on %s", p);
    return SCC_OK;
}

extern "C" int scc_read_scc_list(const char* path, int32_t n, int32_t* labels, int32_t* num_sccs) {
    SCC_REQUIRE(path && labels && n >= 0, SCC_ERR_INVALID, "bad argument");
    FILE* f = fopen(path, "r");
    SCC_REQUIRE(f, SCC_ERR_IO, "cannot open %s", path);
    for (int32_t i = 0; i < n; ++i) labels[i] = -1;
    int32_t mx = 0;
    long long a, b;
    while (fscanf(f, "%lld %lld", &a, &b) == 2) {
        if (a < 0 || a >= n || b < 0 || b > INT32_MAX - 1) { fclose(f); scc_set_error("%s: bad line", path); return SCC_ERR_IO; }
        labels[a] = (int32_t)b;
        if (b + 1 > mx) mx = (int32_t)(b + 1);
    }
    fclose(f);
    if (num_sccs) *num_sccs = mx;
    return SCC_OK;
}

extern "C" int scc_histogram(scc_state* s, int32_t* sizes, int32_t* counts, int32_t capacity, int32_t* num_bins) {
    SCC_REQUIRE(s && num_bins, SCC_ERR_INVALID, "NULL argument");
    std::vector<int32_t> rep((size_t)s->n);
    SCC_TRY(scc_state_get_scc(s, rep.data()));
    std::vector<int32_t> sz((size_t)s->n, 0);
    for (int32_t i = 0; i < s->n; ++i) if (rep[i] >= 0 && rep[i] < s->n) sz[rep[i]]++;
    std::map<int32_t, int32_t> h;
    for (int32_t i = 0; i < s->n; ++i) if (rep[i] == i) h[sz[i]]++;
    *num_bins = (int32_t)h.size();
    if (sizes || counts) {
        SCC_REQUIRE(capacity >= (int32_t)h.size(), SCC_ERR_INVALID, "capacity too small");
        int32_t k = 0;
        for (auto& kv : h) {
            if (sizes) sizes[k] = kv.first;
            if (counts) counts[k] = kv.second;
            k++;
        }
    }
    return SCC_OK;
}

extern "C" int scc_decompose_csr(int32_t n, int32_t m, const int32_t* begin, const int32_t* node_idx,
                                 const int32_t* r_begin, const int32_t* r_node_idx, int method, int device,
                                 int32_t* labels, int32_t* num_sccs, scc_run_stats* stats) {
    scc_graph* g = nullptr;
    scc_state* s = nullptr;
    int rc = scc_graph_create_csr(n, m, begin, node_idx, r_begin, r_node_idx, device, &g);
    if (rc == SCC_OK) rc = scc_state_create(g, &s);
    scc_run_stats st;
    if (rc == SCC_OK) rc = scc_run(g, s, method, SCC_PIVOT_DEGREE, &st);
    if (rc == SCC_OK && labels) rc = scc_canonical_labels(s, labels);
    if (rc == SCC_OK && num_sccs) *num_sccs = st.num_sccs;
    if (rc == SCC_OK && stats) *stats = st;
    scc_state_free(s);
    scc_graph_free(g);
    return rc;
}
