// scc -- drop-in command-line driver for the GPU engine.
//
// Same command line and stdout lines as the reference driver
// (src/common_main.h:451-486, 764, 804; src/scc_main.cc:57-93, 147-178), so
// the reference's scripts (exec_auto.py, info_extract.py) parse its output
// unchanged:
//
//   scc <graph_file> <num_threads> <method> [-d|-a|-p]
//
//   graph_file   text edge list "u v", 1-based, N = max id (common_main.h:61-83)
//   num_threads  accepted and echoed (the work runs on the GPU)
//   method       0, 1, 2: decompose graph_file
//                5-11: the dynamic experiments (common_main.h:500-732).  graph_file
//                is the update batch; the original graph is refined_edges.txt
//                in the same directory; methods 6-11 start from the previous
//                decomposition in scc_list.txt, as a "-p" run writes it (the
//                reference reads a fixed path; here $SCC_LIST, else
//                ./scc_list.txt).  5: inserts, full recompute (insert_idea1);
//                6, 11: inserts on the condensation graph (insert_idea2); 7: the
//                same with the unaffected topological levels finished first;
//                8-10: deletions, recomputed inside the SCCs that lost an edge.
//   -d           per-phase times;  -a  SCC size histogram;  -p  write scc_list.txt
//
// The timed region is the SCC run only, like the reference's prepare()+run()
// timer (common_main.h:801-807); loading and CSR construction are reported
// separately.  Errors print scc_last_error() and exit with status 1.
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <string>
#include <vector>
#include "scc_capi.h"

static double now_ms() {
    struct timeval t;
    gettimeofday(&t, NULL);
    return t.tv_sec * 1000.0 + t.tv_usec * 0.001;
}

static void usage(const char* prog) {
    printf("%s <graph_name> <num_threads> ", prog);
    printf("<method> {-d|-a|-p}\n");
    printf("   method  0: Trim1 + FW-BW (Baseline) \n");
    printf("   method  1: Trim1 + Global FW-BW + Trim1 + FW-BW (Method 1)\n");
    printf("   method  2: Trim1 + Global FW-BW + Trim1/2 + WCC + FW-BW (Method 2)\n");
    printf("   method  3: Tarjan (sequential oracle; not offered on the GPU)\n");
    printf("   method  4: Trim1 + Tarjan (sequential oracle; not offered on the GPU)\n");
    printf("   -d: Print detailed execution time breakdown\n");
    printf("   -a: Print SCC size histogram\n");
    printf("   -p: Output SCC list to file\n");
    printf("\n");
}

static int fail(const char* what, int rc) {
    fprintf(stderr, "%s failed: %s (%s)\n", what, scc_status_string(rc), scc_last_error());
    return 1;
}

static void print_phases(const scc_run_stats& st) {
    printf("\t[TRIM1 phase: %f ms]\n", st.ms_trim1);
    printf("\t[GLOBAL_BFS phase: %f ms]\n", st.ms_global_fb);
    printf("\t[TRIM1 phase: %f ms]\n", st.ms_trim12);
    printf("\t[WCC phase: %f ms]\n", st.ms_wcc);
    printf("\t[FB phase: %f ms]\n", st.ms_fb);
}

// ------------------------------------------------------------------ methods 5-11
struct Edges {
    std::vector<int32_t> s, d;
    int32_t max_id = 0;
};

static int read_edges(const char* path, Edges& e) {
    int64_t m = 0;
    int rc = scc_read_edge_list(path, 0, NULL, NULL, &m, &e.max_id);
    if (rc != SCC_OK || m == 0) return rc;
    e.s.resize((size_t)m);
    e.d.resize((size_t)m);
    return scc_read_edge_list(path, m, e.s.data(), e.d.data(), &m, &e.max_id);
}

// refined_edges.txt beside the batch file (common_main.h:503-504)
static std::string original_graph_path(const char* fname) {
    std::string f(fname);
    size_t slash = f.rfind('/');
    return (slash == std::string::npos ? std::string(".") : f.substr(0, slash)) + "/refined_edges.txt";
}

static int update_flow(const char* fname, int num, int method, int detail, int analyze, int print) {
    double t1 = now_ms();
    Edges orig, batch;
    std::string orig_path = original_graph_path(fname);
    int rc = read_edges(orig_path.c_str(), orig);
    if (rc != SCC_OK) return fail("reading the original graph", rc);
    rc = read_edges(fname, batch);
    if (rc != SCC_OK) return fail("reading the update batch", rc);
    const int32_t n = orig.max_id;
    if (batch.max_id > n) {
        fprintf(stderr, "update batch names vertex %d beyond the original graph's %d vertices\n", batch.max_id, n);
        return 1;
    }
    const int64_t k = (int64_t)batch.s.size();
    const int32_t* bs = k ? batch.s.data() : NULL;
    const int32_t* bd = k ? batch.d.data() : NULL;
    scc_graph* g0 = NULL;
    rc = scc_graph_create_edges(n, (int64_t)orig.s.size(), orig.s.data(), orig.d.data(), SCC_BUILD_KEEP_ALL, 0, &g0);
    if (rc != SCC_OK) return fail("building the original graph", rc);

    // previous decomposition: scc_list.txt ids (read_file1, common_main.h:316-341)
    std::vector<int32_t> ids((size_t)n, -1);
    int32_t num_sccs = 0;
    if (method >= 6) {
        const char* env = getenv("SCC_LIST");
        const char* list = (env && *env) ? env : "scc_list.txt";
        rc = scc_read_scc_list(list, n, ids.data(), &num_sccs);
        if (rc != SCC_OK) return fail("reading scc_list.txt", rc);
        for (int32_t v = 0; v < n; ++v)
            if (ids[(size_t)v] < 0) {
                fprintf(stderr, "%s does not list vertex %d\n", list, v);
                return 1;
            }
    }

    // the graph the run decomposes, and method 7's level analytics
    scc_graph* g = NULL;
    std::vector<int32_t> levels, affected;
    int32_t max_level = 0;
    if (method == 5) {
        Edges all = orig;
        all.s.insert(all.s.end(), batch.s.begin(), batch.s.end());
        all.d.insert(all.d.end(), batch.d.begin(), batch.d.end());
        rc = scc_graph_create_edges(n, (int64_t)all.s.size(), all.s.data(), all.d.data(), SCC_BUILD_KEEP_ALL, 0, &g);
        if (rc != SCC_OK) return fail("building the graph with the inserted edges", rc);
    } else if (method == 6 || method == 7 || method == 11) {
        if (method == 7) {
            scc_graph* dag = NULL;
            rc = scc_condensation_graph(g0, ids.data(), num_sccs, 0, NULL, NULL, &dag);
            if (rc != SCC_OK) return fail("scc_condensation_graph", rc);
            levels.resize((size_t)num_sccs);
            rc = scc_topological_levels(dag, levels.data(), &max_level);
            if (rc != SCC_OK) return fail("scc_topological_levels", rc);
            printf("max_level:%d\n", max_level);
            affected.resize((size_t)max_level + 1);
            int32_t unaffected = 0;
            rc = scc_affected_levels(dag, levels.data(), max_level, n, ids.data(), k, bs, bd, affected.data(),
                                     &unaffected);
            if (rc != SCC_OK) return fail("scc_affected_levels", rc);
            printf("size of unaffected_levels:%d\n", unaffected);
            scc_graph_free(dag);
        }
        rc = scc_condensation_graph(g0, ids.data(), num_sccs, k, bs, bd, &g);
        if (rc != SCC_OK) return fail("scc_condensation_graph", rc);
    }
    double t2 = now_ms();
    printf("graph loading time=%lf\n", t2 - t1);
    printf("reverse edge creation time=%lf\n", 0.0);
    printf("data=%s %d %d\n", fname, method, num);
    printf("\n");

    int32_t total = 0;
    double r1 = 0.0, r2 = 0.0;
    scc_state* s = NULL;
    if (method <= 7 || method == 11) {
        rc = scc_state_create(g, &s);
        if (rc != SCC_OK) return fail("creating the state", rc);
        printf("Running Method 2: Trim1 + Global FW-BW + Trim1/2 + WCC + FW-BW\n");
        scc_run_stats st;
        r1 = now_ms();
        if (method == 7) {
            rc = scc_state_finish_unaffected(s, levels.data(), affected.data(), max_level, NULL);
            if (rc != SCC_OK) return fail("scc_state_finish_unaffected", rc);
        }
        rc = scc_run(g, s, 2, SCC_PIVOT_DEGREE, &st);
        r2 = now_ms();
        if (rc != SCC_OK) return fail("scc_run", rc);
        if (detail) print_phases(st);
        total = st.num_sccs;
    } else {
        // deletions against the previous decomposition: each SCC's
        // representative is its first vertex; read_file2's counts of SCCs
        // holding a deleted edge (common_main.h:343-393)
        std::vector<int32_t> first((size_t)num_sccs, -1), rep((size_t)n), colour((size_t)n, SCC_COLOR_DONE);
        for (int32_t v = 0; v < n; ++v) {
            int32_t id = ids[(size_t)v];
            if (first[(size_t)id] < 0) first[(size_t)id] = v;
            rep[(size_t)v] = first[(size_t)id];
        }
        if (method == 9) {
            std::vector<char> hit((size_t)num_sccs, 0);
            int32_t affect = 0;
            for (int64_t i = 0; i < k; ++i) {
                int32_t a = ids[(size_t)batch.s[(size_t)i]];
                if (a == ids[(size_t)batch.d[(size_t)i]] && !hit[(size_t)a]) { hit[(size_t)a] = 1; affect++; }
            }
            printf("affect_sccs:%d unaffect_sccs:%d\n", affect, num_sccs - affect);
        }
        g = g0;
        g0 = NULL;
        rc = scc_state_create(g, &s);
        if (rc == SCC_OK) rc = scc_state_set_scc(s, rep.data());
        if (rc == SCC_OK) rc = scc_state_set_color(s, colour.data());
        if (rc != SCC_OK) return fail("creating the state", rc);
        printf("Running Method 2: Trim1 + Global FW-BW + Trim1/2 + WCC + FW-BW\n");
        scc_update_stats us;
        r1 = now_ms();
        rc = scc_decremental_delete(g, s, k, bs, bd, &us);
        r2 = now_ms();
        if (rc != SCC_OK) return fail("scc_decremental_delete", rc);
        if (detail) printf("\t[DELETE phase: %f ms]\n", us.ms_total);
        total = us.num_sccs;
    }
    printf("[%d]running_time(ms)=%lf\n", num, r2 - r1);
    fflush(stdout);
    printf("Total # SCCs = %d\n", total);
    if (method == 7) printf("Trimmed nodes=%d\n", 0);   // trim_7 is never incremented (scc_main.cc:27, 162-163)
    if (analyze) {
        int32_t bins = 0;
        rc = scc_histogram(s, NULL, NULL, 0, &bins);
        if (rc != SCC_OK) return fail("scc_histogram", rc);
        std::vector<int32_t> sizes((size_t)bins), counts((size_t)bins);
        rc = scc_histogram(s, sizes.data(), counts.data(), bins, &bins);
        if (rc != SCC_OK) return fail("scc_histogram", rc);
        for (int32_t i = 0; i < bins; ++i) printf("%d => %d\n", sizes[(size_t)i], counts[(size_t)i]);
        printf("\n");
    }
    if (print) {
        rc = scc_output_scc_list(s, "scc_list.txt");
        if (rc != SCC_OK) return fail("scc_output_scc_list", rc);
    }
    scc_state_free(s);
    scc_graph_free(g);
    scc_graph_free(g0);
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 4) {
        usage(argv[0]);
        return EXIT_FAILURE;
    }
    const char* fname = argv[1];
    int num = atoi(argv[2]);
    int method = atoi(argv[3]);
    int detail = 0, analyze = 0, print = 0;
    if (method < 0 || method > 11) {
        printf("error procesing argument\n");
        usage(argv[0]);
        return EXIT_FAILURE;
    }
    if (argc >= 5) {
        if (strncmp(argv[4], "-d", 2) == 0) detail = 1;
        else if (strncmp(argv[4], "-a", 2) == 0) analyze = 1;
        else if (strncmp(argv[4], "-p", 2) == 0) print = 1;
        else printf("ignoring %s\n", argv[4]);
    }
    printf("running with %d threads\n", num);
    if (method >= 5) return update_flow(fname, num, method, detail, analyze, print);
    int run_method = method;

    double t1 = now_ms();
    scc_graph* g = NULL;
    int rc = scc_graph_load_edge_list(fname, 0, &g);
    if (rc != SCC_OK) return fail("loading the graph", rc);
    double t2 = now_ms();
    printf("graph loading time=%lf\n", t2 - t1);
    printf("reverse edge creation time=%lf\n", 0.0);   // built on the device together with the CSR
    printf("data=%s %d %d\n", fname, method, num);
    printf("\n");

    scc_state* s = NULL;
    rc = scc_state_create(g, &s);
    if (rc != SCC_OK) return fail("creating the state", rc);
    if (run_method == 0) printf("Running Baseline: Trim1 + FW-BW\n");
    else if (run_method == 1) printf("Running Method 1: Trim1 + Global FW-BW + Trim1 + FW-BW\n");
    else if (run_method == 2) printf("Running Method 2: Trim1 + Global FW-BW + Trim1/2 + WCC + FW-BW\n");
    scc_run_stats st;
    double r1 = now_ms();
    rc = scc_run(g, s, run_method, SCC_PIVOT_DEGREE, &st);
    double r2 = now_ms();
    if (rc != SCC_OK) return fail("scc_run", rc);
    if (detail) print_phases(st);
    if (analyze) {
        printf("trimmed = %d\n", st.trimmed_first);
        printf("First_SCC_size = %d\n", st.first_scc_size);
    }
    printf("[%d]running_time(ms)=%lf\n", num, r2 - r1);
    fflush(stdout);
    printf("Total # SCCs = %d\n", st.num_sccs);
    if (analyze) {
        int32_t bins = 0;
        rc = scc_histogram(s, NULL, NULL, 0, &bins);
        if (rc != SCC_OK) return fail("scc_histogram", rc);
        std::vector<int32_t> sizes((size_t)bins), counts((size_t)bins);
        rc = scc_histogram(s, sizes.data(), counts.data(), bins, &bins);
        if (rc != SCC_OK) return fail("scc_histogram", rc);
        for (int32_t i = 0; i < bins; ++i) printf("%d => %d\n", sizes[(size_t)i], counts[(size_t)i]);
        printf("\n");
    }
    if (print) {
        rc = scc_output_scc_list(s, "scc_list.txt");
        if (rc != SCC_OK) return fail("scc_output_scc_list", rc);
    }
    scc_state_free(s);
    scc_graph_free(g);
    return 0;
}
