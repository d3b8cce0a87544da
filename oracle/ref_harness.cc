// Harness around the reference's own OpenMP SCC engine -- TEST INFRASTRUCTURE ONLY.
//
// Compiled by oracle/Makefile together with the reference sources
// (gm_graph/src/*.cc, src/*.cc of ShashwaTTrigunayaT/DynamicGraphs_SCC) into
// oracle/_ref/libscc_ref.so.  It exposes two C entry points that build the
// reference's gm_graph from a CSR and then call the reference's own code:
//   ref_method2: my_main::prepare() + my_main::run() with method 2, the same
//                region src/common_main.h:794-807 times;
//   ref_tarjan:  initialize_color/initialize_tarjan + do_tarjan_all
//                (src/scc_tarjan.cc:62-149), on a thread with a large stack,
//                because the CLI's methods 3/4 load no graph (common_main.h:733).
// The reference's scc_main.cc is included with its main() renamed so that its
// driver class and globals are available here unchanged.
#include <bits/stdc++.h>
#include <omp.h>
#include <pthread.h>
#include <sys/resource.h>
#include <sys/time.h>
#include "gm.h"
#include "my_work_queue.h"
#include "scc.h"

#define private public
#define protected public
#define main scc_reference_cli_main
#include "scc_main.cc"
#undef main
#undef protected
#undef private

static void build_graph(gm_graph& G, int32_t n, int64_t m, const int32_t* begin, const int32_t* node_idx) {
    G.prepare_external_creation(n, (edge_t)m);
    memcpy(G.begin, begin, sizeof(int32_t) * ((size_t)n + 1));
    if (m > 0) memcpy(G.node_idx, node_idx, sizeof(int32_t) * (size_t)m);
    G.do_semi_sort();          // what freeze() does after add_edge (gm_graph.cc:100)
    G.make_reverse_edges();    // sorted transpose, as the loader path builds it
}

static double now_ms() {
    struct timeval t;
    gettimeofday(&t, NULL);
    return t.tv_sec * 1000.0 + t.tv_usec * 0.001;
}

// Method 0, 1 or 2 of my_main::run (src/scc_main.cc:120-145) with its own
// phase selection, timed over run() like the reference's timer.
extern "C" int ref_method(int method, int32_t n, int64_t m, const int32_t* begin, const int32_t* node_idx,
                          int threads, int pin, int32_t* scc_out, double* ms_out) {
    if (method < 0 || method > 2) return 2;
    gm_rt_set_num_threads(threads);
    my_main T;
    char a0[2] = {(char)('0' + method), 0};
    char* av[] = {a0};
    if (!T.check_args(1, av)) return 1;
    met_algo = method;
    build_graph(T.G, n, m, begin, node_idx);
    if (pin) T.pin_CPU();
    T.prepare();
    double t0 = now_ms();
    T.run();
    double t1 = now_ms();
    if (ms_out) *ms_out = t1 - t0;
    memcpy(scc_out, G_SCC, sizeof(int32_t) * (size_t)n);
    finalize_color();
    finalize_tarjan();
    finalize_trim2();
    finalize_WCC();
    finalize_analyze();
    delete[] G_SCC;
    G_SCC = NULL;
    met_algo = 2;
    return 0;
}

extern "C" int ref_method2(int32_t n, int64_t m, const int32_t* begin, const int32_t* node_idx, int threads,
                           int pin, int32_t* scc_out, double* ms_out) {
    return ref_method(2, n, m, begin, node_idx, threads, pin, scc_out, ms_out);
}

struct tarjan_job {
    int32_t n; int64_t m; const int32_t* begin; const int32_t* node_idx; int32_t* out; double ms;
};

static void* tarjan_thread(void* arg) {
    tarjan_job* j = (tarjan_job*)arg;
    gm_rt_set_num_threads(1);
    gm_rt_initialize();
    gm_graph G;
    build_graph(G, j->n, j->m, j->begin, j->node_idx);
    G_num_nodes = G.num_nodes();
    G_SCC = new node_t[G_num_nodes];
    for (int i = 0; i < G_num_nodes; ++i) G_SCC[i] = gm_graph::NIL_NODE;
    initialize_color();
    initialize_tarjan();
    double t0 = now_ms();
    do_tarjan_all(G);
    j->ms = now_ms() - t0;
    memcpy(j->out, G_SCC, sizeof(int32_t) * (size_t)j->n);
    finalize_color();
    finalize_tarjan();
    delete[] G_SCC;
    G_SCC = NULL;
    return NULL;
}

extern "C" int ref_tarjan(int32_t n, int64_t m, const int32_t* begin, const int32_t* node_idx, int32_t* scc_out,
                          double* ms_out) {
    tarjan_job j{n, m, begin, node_idx, scc_out, 0.0};
    pthread_attr_t attr;
    pthread_attr_init(&attr);
    size_t stack = (size_t)256 * (size_t)(n > 0 ? n : 1) + ((size_t)64 << 20);
    pthread_attr_setstacksize(&attr, stack);
    pthread_t th;
    if (pthread_create(&th, &attr, tarjan_thread, &j) != 0) return 1;
    pthread_join(th, NULL);
    pthread_attr_destroy(&attr);
    if (ms_out) *ms_out = j.ms;
    return 0;
}

// Method 7's preprocessing by the reference's own main_t::create_scc_edges
// (src/common_main.h:180-262) with met_algo = 7: the condensation edges, the
// BFS levels of the original condensation (level_ver) and the prefix-summed
// affect_level.  One OpenMP thread: its loops push into shared vectors
// without locks.  Its closing loop runs to unaffected_levels.size() - 1 on an
// unsigned size, so callers only pass batches that leave a level unaffected.
// ids: the scc_list ids (read_file1) of the nv vertices; edges 0-based.
extern "C" int ref_method7_levels(int32_t nv, int64_t m, const int32_t* osrc, const int32_t* odst, int64_t k,
                                  const int32_t* isrc, const int32_t* idst, const int32_t* ids, int32_t num_sccs,
                                  int32_t* level_out, int32_t* affect_out) {
    gm_rt_set_num_threads(1);
    omp_set_num_threads(1);
    my_main T;
    met_algo = 7;
    scc_list.assign(ids, ids + nv);
    level_ver.clear();
    affect_level.clear();
    new_edge_nodes.clear();
    std::vector<std::pair<int, int>> orig((size_t)m), ins((size_t)k), scc_edges;
    for (int64_t i = 0; i < m; ++i) orig[(size_t)i] = std::make_pair(osrc[i], odst[i]);
    for (int64_t i = 0; i < k; ++i) ins[(size_t)i] = std::make_pair(isrc[i], idst[i]);
    T.create_scc_edges(orig, ins, scc_edges, nv, num_sccs);
    for (int32_t i = 0; i < num_sccs; ++i) level_out[i] = level_ver[(size_t)i];
    for (int32_t i = 0; i < num_sccs + 5; ++i) affect_out[i] = affect_level[(size_t)i];
    met_algo = 2;
    return 0;
}
