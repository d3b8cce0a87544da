// Autotuner for the traversal switch points and launch shapes (scc_tuning):
// a grid search that times full decompositions of the caller's graph (or a
// sample of it) and keeps the fastest setting in the state.  The reference
// fixes these constants in its BFS template (gm_bfs_template.h:841-842) and
// trim/WCC thresholds (src/scc_trim1.cc:203, src/scc_weak.cc:143).
#include <string.h>
#include "scc_internal.cuh"

static int time_run(const scc_graph* g, scc_state* s, int method, double* ms) {
    SCC_TRY(scc_state_reset(s));
    scc_run_stats st;
    SCC_TRY(scc_run(g, s, method, SCC_PIVOT_DEGREE, &st));
    *ms = st.ms_total;
    return SCC_OK;
}

extern "C" int scc_autotune(const scc_graph* g, scc_state* s, int method, int max_trials, scc_tuning* best,
                            double* best_ms) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(max_trials >= 1, SCC_ERR_INVALID, "max_trials %d", max_trials);
    const int32_t keeps[] = {16, 32};
    const int32_t blocks[] = {1, 2};
    const int32_t narrow[] = {1 << 14, 1 << 16};
    const int32_t after[] = {1, 2};
    const int32_t alphas[] = {14, 40};
    scc_tuning start = s->tune, top = s->tune;
    double warm = 0.0, top_ms = 0.0;
    SCC_TRY(time_run(g, s, method, &warm));       // warm caches and allocations
    SCC_TRY(time_run(g, s, method, &top_ms));     // the current setting is the first candidate
    int trials = 1;
    for (int a = 0; a < 2 && trials < max_trials; ++a)
        for (int k = 0; k < 2 && trials < max_trials; ++k)
            for (int b = 0; b < 2 && trials < max_trials; ++b)
                for (int nw = 0; nw < 2 && trials < max_trials; ++nw)
                    for (int af = 0; af < 2 && trials < max_trials; ++af) {
                        scc_tuning t = start;
                        t.bu_alpha = alphas[a]; t.async_keep = keeps[k]; t.async_blocks_per_sm = blocks[b];
                        t.async_max = narrow[nw]; t.async_after = after[af];
                        if (memcmp(&t, &start, sizeof(t)) == 0) continue;
                        s->tune = t;
                        double ms = 0.0;
                        int rc = time_run(g, s, method, &ms);
                        if (rc != SCC_OK) { s->tune = start; return rc; }
                        trials++;
                        if (ms < top_ms) { top_ms = ms; top = t; }
                    }
    s->tune = top;
    SCC_TRY(scc_state_reset(s));
    if (best) *best = top;
    if (best_ms) *best_ms = top_ms;
    return SCC_OK;
}
