// Harness around the reference's own CUDA engine -- the GPU comparator, TEST
// AND MEASUREMENT INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile with the reference's src_CUDA/*.cu (all but its
// main and its dynamic-method loaders, scc_cuda_main.cpp and
// scc_cuda_dynamic.cpp) into oracle/_ref/libscc_ref_cuda.so for sm_100a
// (-include cstdint: scc_cuda.h uses uint32_t without <cstdint>).  It replaces
// the reference's main() for method 2 only: instead of reading a text file
// into gm_graph it takes the CSR and its transpose that gm_graph's
// make_reverse_edges would give, then makes the same calls, in the same
// order, as scc_cuda_main.cpp:408-500 (graph_upload, state_allocate/init, the
// initialize_* calls of :296-301, repeat_global_trim1, create_trim1_compact,
// do_global_fw_bw_main, repeat_global_trim1_compact, do_global_trim2_new,
// repeat_global_trim1_compact(100), do_global_wcc, create_work_items_from_wcc,
// start_workers_fw_bw_dfs_host(40)), timed over the same region as the
// reference's R1..R2, and copies G_SCC back.  Methods 0 and 1 of the CUDA path
// are not offered: their per-work BFS never clears its visited bits.
#include <omp.h>
#include <sys/time.h>
#include <vector>
#include "scc_cuda.h"

// host CSR the reference's host-side FW-BW reads (defined by its main)
const edge_t* g_h_begin = NULL;
const node_t* g_h_node_idx = NULL;
const edge_t* g_h_r_begin = NULL;
const node_t* g_h_r_node_idx = NULL;
int g_h_N = 0;

static double ms_since(const struct timeval& a, const struct timeval& b) {
    return (b.tv_sec - a.tv_sec) * 1000.0 + (b.tv_usec - a.tv_usec) * 0.001;
}

extern "C" int refcuda_method2(int32_t n, int64_t m, const int32_t* begin, const int32_t* node_idx,
                               const int32_t* r_begin, const int32_t* r_node_idx, int threads, int32_t* scc_out,
                               double* ms_out) {
    if (n <= 0 || m < 0 || m > 0x7FFFFFFF) return 1;
    const int N = n, M = (int)m;
    std::vector<edge_t> h_begin(begin, begin + N + 1), h_r_begin(r_begin, r_begin + N + 1);
    std::vector<node_t> h_node_idx(node_idx, node_idx + M), h_r_node_idx(r_node_idx, r_node_idx + M);
    omp_set_num_threads(threads);            // what gm_rt_set_num_threads does for its OpenMP loops
    GPUGraph gpuG;
    graph_upload(gpuG, h_begin, h_node_idx, h_r_begin, h_r_node_idx, N, M);
    g_h_begin = h_begin.data();
    g_h_node_idx = h_node_idx.data();
    g_h_r_begin = h_r_begin.data();
    g_h_r_node_idx = h_r_node_idx.data();
    g_h_N = N;

    GPUState st;
    state_allocate(st, N);
    state_init(st);
    initialize_trim1_full(N);
    initialize_trim2(N);
    initialize_WCC(N);
    work_q_init(threads);
    int* d_count = NULL;
    CUDA_CHECK(cudaMalloc(&d_count, sizeof(int)));
    DynamicArrays da;
    memset(&da, 0, sizeof(da));
    int flag11 = 0;
    const int met_algo = 2;
    CUDA_CHECK(cudaDeviceSynchronize());

    struct timeval R1, R2;
    gettimeofday(&R1, NULL);
    int trimmed = repeat_global_trim1(st, gpuG, d_count, met_algo, flag11, da, NULL, 0);
    int curr_count = N - trimmed;
    if (curr_count > 0) {
        create_trim1_compact(st, gpuG);
        initialize_global_fb(N);
        do_global_fw_bw_main(st, gpuG, COLOR_UNASSIGNED, curr_count, -1, false);
        trimmed = repeat_global_trim1_compact(st, gpuG, d_count, met_algo, flag11, da, NULL, 0);
        int trim_total = do_global_trim2_new(st, gpuG, d_count);
        trim_total += repeat_global_trim1_compact(st, gpuG, d_count, met_algo, flag11, da, NULL, 100);
        (void)trim_total;
        curr_count = d_trim_targets_count;
        if (curr_count > 0) {
            do_global_wcc(st, gpuG);
            create_work_items_from_wcc(st, gpuG);
            start_workers_fw_bw_dfs_host(st, gpuG, 40);
        }
        finalize_global_fb();
    }
    gettimeofday(&R2, NULL);
    if (ms_out) *ms_out = ms_since(R1, R2);
    CUDA_CHECK(cudaMemcpy(scc_out, st.d_SCC, sizeof(int32_t) * (size_t)N, cudaMemcpyDeviceToHost));

    cudaFree(d_count);
    finalize_WCC();
    finalize_trim2();
    finalize_trim1();
    state_free(st);
    graph_free(gpuG);
    return 0;
}
