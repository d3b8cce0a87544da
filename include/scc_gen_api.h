/*
 * scc_gen_api.h -- seeded synthetic graph generators of the B200 SCC engine.
 *
 * The reference benchmarks on SNAP / MatrixMarket files read by
 * src/common_main.h:61-83 and generated update batches (dataset_handler.py),
 * none of which ship with it.  These generators stand in for them with the
 * shapes of its benchmark configurations.  Host and device generation use
 * the same counter-based formulas, so the oracle and the engine decompose the
 * same graphs.  Output graphs drop self-loops and duplicates when built with
 * SCC_BUILD_DEDUP | SCC_BUILD_NO_SELF_LOOPS.
 */
#ifndef SCC_GEN_API_H
#define SCC_GEN_API_H

#include <stdint.h>
#include "scc_capi.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct scc_gen_params {
    int rmat_scale;        /* R-MAT part: 2^rmat_scale vertices (0 = none) */
    int edge_factor;       /* R-MAT edges = edge_factor << rmat_scale, a/b/c/d = .57/.19/.19/.05 */
    int grid_side;         /* grid part: side^2 vertices after the R-MAT ids (0 = none) */
    int num_cycles;        /* planted directed cycles through R-MAT vertex ids */
    int cycle_min, cycle_max;   /* cycle lengths log-uniform in [cycle_min, cycle_max] */
    uint64_t seed;
} scc_gen_params;

/* Vertex count and an upper bound on the raw edge count. */
int scc_gen_sizes(const scc_gen_params* p, int32_t* n, int64_t* max_edges);
/* Raw edge list on the host (before self-loop / duplicate removal). */
int scc_gen_edges_host(const scc_gen_params* p, int32_t* src, int32_t* dst, int64_t capacity, int64_t* m);
/* Generate on the device and build the CSR + transpose (flags: SCC_BUILD_*). */
int scc_gen_graph(const scc_gen_params* p, int flags, int device, scc_graph** out);

/* Many independent uneven graphs (the batched configuration): graph i has
 * n_i vertices, log-uniform in [n_min, n_max]; each vertex gets a Poisson
 * (mean_degree) number of out-edges, each aimed at an R-MAT-distributed
 * target (probability rmat_fraction) or a uniform one, inside graph i.  The
 * graphs are laid out one after another: graph i owns the ids
 * [offsets[i], offsets[i+1]).  Seeded per graph. */
typedef struct scc_batch_params {
    int32_t num_graphs;
    int32_t n_min, n_max;
    double mean_degree;
    double rmat_fraction;
    uint64_t seed;
} scc_batch_params;

/* offsets: num_graphs + 1 ints; *n = offsets[num_graphs]; *max_edges bounds the raw edge count. */
int scc_gen_batch_layout(const scc_batch_params* p, int32_t* offsets, int32_t* n, int64_t* max_edges);
int scc_gen_batch_edges_host(const scc_batch_params* p, int32_t* src, int32_t* dst, int64_t capacity, int64_t* m);
int scc_gen_batch_graph(const scc_batch_params* p, int flags, int device, scc_graph** out);
/* The induced subgraph on ids [v_begin, v_end), rebased to start at 0.  The
 * range must have no edge leaving it (one graph of a batch). */
int scc_graph_subgraph(const scc_graph* g, int32_t v_begin, int32_t v_end, scc_graph** out);

#ifdef __cplusplus
}
#endif
#endif
