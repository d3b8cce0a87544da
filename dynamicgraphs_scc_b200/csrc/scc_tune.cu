// Autotuner for the traversal switch points and launch shapes (scc_tuning).
// The reference fixes these constants in its BFS template
// (gm_bfs_template.h:841-842) and its trim/WCC thresholds
// (src/scc_trim1.cc:203, src/scc_weak.cc:143); here they are searched per
// graph by successive halving: a seeded sample of the knob grid (the current
// setting always among them) is timed with one full decomposition each, the
// faster half is timed again with two runs each, and so on until one remains;
// it is kept in the state.
#include <string.h>
#include <algorithm>
#include <vector>
#include "scc_internal.cuh"

static int time_run(const scc_graph* g, scc_state* s, int method, double* ms) {
    SCC_TRY(scc_state_reset(s));
    scc_run_stats st;
    SCC_TRY(scc_run(g, s, method, SCC_PIVOT_DEGREE, &st));
    *ms = st.ms_total;
    return SCC_OK;
}

// The knobs and their candidate values.
static const int32_t K_ALPHA[] = {8, 14, 24, 40};                 // bottom-up switch (Beamer's alpha)
static const int32_t K_BUDIV[] = {12, 24, 48};                    // stay bottom-up while frontier > 2 live / div
static const int32_t K_AMAX[] = {1 << 12, 1 << 14, 1 << 16};      // a frontier this small is narrow
static const int32_t K_AFTER[] = {1, 2};                          // narrow levels before the drain
static const int32_t K_KEEP[] = {16, 32, 64};                     // items a drain warp keeps
static const int32_t K_BLOCKS[] = {1, 2};                         // drain blocks per SM
static const int32_t K_HUGE[] = {1024, 4096, 16384};              // edge-parallel hub expansion above this degree
static const int32_t K_TILE[] = {-1, 1 << 18, 1 << 20};           // tile drain from this many live vertices
static const int32_t K_SPAN[] = {2048, 16384};                    // smallest tile
static const int32_t K_TAIL[] = {-1, 1 << 14, 1 << 16};           // one-launch tail from this many live vertices
static const int32_t K_CTA[] = {-1, 256, 1024};                   // block-wide expansion above this degree

static scc_tuning candidate(uint64_t& rng) {
    auto pick = [&](const int32_t* v, int k) {
        rng = rng * 6364136223846793005ull + 1442695040888963407ull;
        return v[(rng >> 33) % (uint64_t)k];
    };
    scc_tuning t;
    t.bu_alpha = pick(K_ALPHA, 4);
    t.bu_div = pick(K_BUDIV, 3);
    t.async_max = pick(K_AMAX, 3);
    t.async_after = pick(K_AFTER, 2);
    t.async_keep = pick(K_KEEP, 3);
    t.async_blocks_per_sm = pick(K_BLOCKS, 2);
    t.huge_deg = pick(K_HUGE, 3);
    t.tile_min_live = pick(K_TILE, 3);
    t.tile_min_span = pick(K_SPAN, 2);
    t.pivot_salt = 0;
    t.tail_live = pick(K_TAIL, 3);
    t.tail_class = 1024;
    t.cta_deg = pick(K_CTA, 3);
    return t;
}

extern "C" int scc_autotune(const scc_graph* g, scc_state* s, int method, int max_trials, scc_tuning* best,
                            double* best_ms) {
    SCC_REQUIRE(g && s, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(max_trials >= 1, SCC_ERR_INVALID, "max_trials %d", max_trials);
    const scc_tuning start = s->tune;
    // the budget of full decompositions buys a first stage of k candidates:
    // k + k/2*2 + k/4*4 + ... ~ k * stages
    int k = std::max(1, max_trials / 3);
    std::vector<scc_tuning> cand{start};
    uint64_t rng = 0x5CC0B200ull;
    for (int tries = 0; (int)cand.size() < k && tries < 64 * k; ++tries) {
        scc_tuning t = candidate(rng);
        bool dup = false;
        for (const auto& c : cand) dup = dup || memcmp(&c, &t, sizeof(t)) == 0;
        if (!dup) cand.push_back(t);
    }
    double warm = 0.0;
    SCC_TRY(time_run(g, s, method, &warm));       // warm caches and allocations
    std::vector<double> ms(cand.size(), 0.0);
    int runs = 1, used = 0;
    while (true) {
        for (size_t i = 0; i < cand.size(); ++i) {
            s->tune = cand[i];
            double sum = 0.0;
            for (int r = 0; r < runs; ++r) {
                double t = 0.0;
                int rc = time_run(g, s, method, &t);
                if (rc != SCC_OK) { s->tune = start; return rc; }
                sum += t;
                ++used;
            }
            ms[i] = sum / runs;
        }
        if (cand.size() == 1) break;
        std::vector<size_t> idx(cand.size());
        for (size_t i = 0; i < idx.size(); ++i) idx[i] = i;
        std::sort(idx.begin(), idx.end(), [&](size_t x, size_t y) { return ms[x] < ms[y]; });
        size_t keep = (cand.size() + 1) / 2;
        // out of budget: keep the best so far
        if (used + (int)keep * runs * 2 > max_trials) keep = 1;
        std::vector<scc_tuning> next;
        std::vector<double> next_ms;
        for (size_t i = 0; i < keep; ++i) { next.push_back(cand[idx[i]]); next_ms.push_back(ms[idx[i]]); }
        cand.swap(next);
        ms.swap(next_ms);
        if (cand.size() == 1) break;
        runs *= 2;
    }
    s->tune = cand[0];
    SCC_TRY(scc_state_reset(s));
    if (best) *best = cand[0];
    if (best_ms) *best_ms = ms[0];
    return SCC_OK;
}
