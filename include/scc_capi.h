/*
 * scc_capi.h -- C ABI of the B200 strongly-connected-components engine.
 *
 * Drop-in boundary for the SCC path of ShashwaTTrigunayaT/DynamicGraphs_SCC.
 * The reference exposes that path as a global-state C++ phase API
 * (src/scc.h:18-92) over gm_graph's int32 CSR (gm_graph/inc/gm_graph.h) and as
 * a CUDA host API over GPUGraph/GPUState (src_CUDA/scc_cuda.h:26-490).  This
 * header replaces both with opaque handles and plain pointers:
 *
 *   gm_graph / GPUGraph       -> scc_graph  (device CSR + transpose, int32)
 *   G_Color, G_SCC / GPUState -> scc_state  (device colour / SCC arrays + work space)
 *   global work queue         -> device-resident colour classes inside scc_state
 *
 * Every entry point returns an int status (SCC_OK == 0) instead of the
 * reference's assert()/exit(1) (src_CUDA/scc_cuda.h:61-67); counts come back
 * through out-parameters.  scc_last_error() describes the last failure on the
 * calling thread.  All arrays are int32 (gm_graph/inc/gm_graph_typedef.h:17-20).
 *
 * Colours follow the reference (src/scc.h:19-22): -1 initial, -2 SCC found,
 * fresh colours >= 0 from scc_get_new_color().  scc[v] is the representative
 * vertex of v's SCC (G_SCC); scc_canonical_labels() turns it into the
 * smallest member id of the component.
 *
 * Threading: one handle may be used by one host thread at a time; work on a
 * state is ordered on the state's CUDA stream.  Host pointers may be pageable
 * or pinned; "_device" variants take device pointers.
 */
#ifndef SCC_CAPI_H
#define SCC_CAPI_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------------- */
#define SCC_OK               0
#define SCC_ERR_INVALID      1   /* bad argument (null handle, negative size, id out of range) */
#define SCC_ERR_CUDA         2   /* CUDA runtime error (message in scc_last_error) */
#define SCC_ERR_OOM          3   /* device allocation failed or budget exceeded */
#define SCC_ERR_TIMEOUT      4   /* a bounded device wait gave up; the state is still usable after scc_state_reset */
#define SCC_ERR_STATE        5   /* call out of order (e.g. phase before scc_state_create) */
#define SCC_ERR_IO           6   /* file could not be read or written */
#define SCC_ERR_NOT_FOUND    7   /* no vertex of the requested colour (NIL_NODE in the reference) */
#define SCC_ERR_UNSUPPORTED  8   /* method or flag not offered by this engine */
#define SCC_ERR_BUSY         9   /* serving loop: the queue is over its admission limit; retry later */

#define SCC_NIL_NODE (-1)        /* gm_graph::NIL_NODE */
#define SCC_COLOR_INIT (-1)
#define SCC_COLOR_DONE (-2)

typedef struct scc_graph scc_graph;
typedef struct scc_state scc_state;

const char* scc_status_string(int status);
const char* scc_last_error(void);
int scc_version(void);                       /* major*10000 + minor*100 + patch */
int scc_device_count(int* count);
/* Scratch of uploads, updates and graph merges comes from one memory pool per
 * device owned by this library, which keeps freed blocks for reuse; this hands
 * them back to the driver (after synchronising the device). */
int scc_release_cached_memory(int device);
/* Host-side fault injection for failure-path tests (the reference's only
 * failure path is CUDA_CHECK -> exit(1), src_CUDA/scc_cuda.h:61-67).
 * SCC_INJECT_ALLOC: the countdown-th scratch allocation of an upload or update
 * from now fails (SCC_ERR_OOM); 0 disarms.  SCC_INJECT_WAIT (countdown > 0):
 * the next asynchronous reachability drain is given one queue slot that is
 * never filled, so its bounded wait gives up and the call returns
 * SCC_ERR_TIMEOUT; the state is usable again after scc_state_reset.  No
 * injection faults, traps or hangs the GPU. */
#define SCC_INJECT_ALLOC 1
#define SCC_INJECT_WAIT  2
int scc_debug_inject(int what, int64_t countdown);

/* ---- graph (gm_graph / GPUGraph) ---------------------------------------------------- */
/* Build flags for scc_graph_create_edges*. */
#define SCC_BUILD_KEEP_ALL      0   /* keep duplicates and self-loops (gm_graph semantics) */
#define SCC_BUILD_DEDUP         1   /* drop duplicate edges */
#define SCC_BUILD_NO_SELF_LOOPS 2   /* drop self-loops */

/* Edge list -> sorted CSR + sorted transpose on the device.  Replaces gm_graph
 * add_node()/add_edge() + freeze() + do_semi_sort() + make_reverse_edges()
 * (gm_graph/src/gm_graph.cc:459-480, 60-101, 385-420, 193-287) and
 * graph_upload() (src_CUDA/scc_cuda_graph.cu:4).  Ids must be in [0, n). */
int scc_graph_create_edges(int32_t n, int64_t m, const int32_t* src, const int32_t* dst,
                           int flags, int device, scc_graph** out);
int scc_graph_create_edges_device(int32_t n, int64_t m, const int32_t* d_src, const int32_t* d_dst,
                                  int flags, int device, scc_graph** out);
/* CSR (+ optional transpose; NULL r_begin/r_node_idx = build it on the device).
 * Mirrors graph_upload(GPUGraph&, h_begin, h_node_idx, h_r_begin, h_r_node_idx, N, M)
 * (src_CUDA/scc_cuda.h:72-77).  Adjacency lists must be sorted (gm_graph keeps them
 * semi-sorted); the engine does not re-sort a caller's CSR. */
int scc_graph_create_csr(int32_t n, int32_t m, const int32_t* begin, const int32_t* node_idx,
                         const int32_t* r_begin, const int32_t* r_node_idx, int device, scc_graph** out);
int scc_graph_create_csr_device(int32_t n, int32_t m, const int32_t* d_begin, const int32_t* d_node_idx,
                                const int32_t* d_r_begin, const int32_t* d_r_node_idx, int device,
                                scc_graph** out);
/* Text edge list "u v" per line, 1-based, N = max id (src/common_main.h:61-83,
 * the fast parser of src_CUDA/scc_cuda_dynamic.cpp:59-147).  Lines starting
 * with '%' or '#' are skipped.  Duplicates and self-loops are kept. */
int scc_graph_load_edge_list(const char* path, int device, scc_graph** out);
/* read_file (src/common_main.h:61-83) into host arrays, 0-based: *count edges, *max_id = N
 * (the largest 1-based id).  capacity 0 only counts; otherwise src/dst hold capacity
 * entries, at least *count. */
int scc_read_edge_list(const char* path, int64_t capacity, int32_t* src, int32_t* dst, int64_t* count,
                       int32_t* max_id);
/* Re-upload host CSR arrays into an existing graph of the same n and m (no
 * allocation): the per-request H2D of graph_upload (src_CUDA/scc_cuda_graph.cu:4)
 * for callers that keep the device graph between runs.  Ordered on `stream`
 * (cudaStream_t as void*, NULL = legacy default stream). */
int scc_graph_upload_csr(scc_graph* g, const int32_t* begin, const int32_t* node_idx,
                         const int32_t* r_begin, const int32_t* r_node_idx, void* stream);
/* Re-upload only the forward CSR (host arrays of the graph's n and m; begin
 * must be a valid CSR offset array) and rebuild the transpose on the device --
 * stable radix sorts of (destination, source) pairs, so in-lists come out
 * sorted by source exactly as make_reverse_edges (gm_graph/src/gm_graph.cc:193-287)
 * leaves them.  From 4 M edges the CSR crosses the bus in four chunks of whole
 * source lists, each sorted on a helper stream while the next is in flight,
 * then merged by one scatter.  Half the host-to-device bytes of
 * scc_graph_upload_csr; ordered on `stream`, whose memory pool holds the
 * scratch until the stream reaches it. */
int scc_graph_upload_csr_out(scc_graph* g, const int32_t* begin, const int32_t* node_idx, void* stream);
int scc_graph_free(scc_graph* g);                             /* graph_free() */
int scc_graph_num_nodes(const scc_graph* g, int32_t* n);
int scc_graph_num_edges(const scc_graph* g, int64_t* m);
/* Copy the CSR and transpose back to host arrays (n+1, m, n+1, m ints; any may be NULL). */
int scc_graph_copy_csr(const scc_graph* g, int32_t* begin, int32_t* node_idx,
                       int32_t* r_begin, int32_t* r_node_idx);
/* Device pointers of the CSR arrays (borrowed; valid until scc_graph_free). */
int scc_graph_device_csr(const scc_graph* g, const int32_t** d_begin, const int32_t** d_node_idx,
                         const int32_t** d_r_begin, const int32_t** d_r_node_idx);
/* Binary CSR snapshot (own format, little-endian: magic "SCCCSR01", n, m, begin, node_idx). */
int scc_graph_save_binary(const scc_graph* g, const char* path);
int scc_graph_load_binary(const char* path, int device, scc_graph** out);

/* ---- state (G_Color / G_SCC / GPUState + phase globals) ------------------------------ */
/* prepare() of src/scc_main.cc:96-118: G_SCC = NIL, colours = -1, colour
 * counter reset, work queue empty, compact trim targets empty. */
int scc_state_create(const scc_graph* g, scc_state** out);
int scc_state_reset(scc_state* s);
int scc_state_free(scc_state* s);
int scc_state_synchronize(scc_state* s);
/* The CUDA stream all work on this state is ordered on (cudaStream_t as void*). */
int scc_state_stream(scc_state* s, void** stream);
/* Host <-> device copies of G_Color / G_SCC (n ints each). */
int scc_state_get_color(scc_state* s, int32_t* color);
int scc_state_get_scc(scc_state* s, int32_t* scc);
int scc_state_set_color(scc_state* s, const int32_t* color);
int scc_state_set_scc(scc_state* s, const int32_t* scc);
/* G_WCC labels (raw, with the 0x20000000 high-degree flag; -1 for finished vertices). */
int scc_state_get_wcc(scc_state* s, int32_t* wcc);
/* Compact trim targets (get_compact_trim_targets, src/scc_trim1.cc:32). */
int scc_state_get_trim_targets(scc_state* s, int32_t* out, int32_t capacity, int32_t* count);
int scc_state_device_arrays(scc_state* s, int32_t** d_color, int32_t** d_scc);
/* Kernel ledger (no counterpart in the reference; its phase timers are
 * gettimeofday, src/scc_main.cc:180-184): when enabled, every launch of the
 * asynchronous reachability drain is timed with CUDA events on the state's
 * stream and its work counted (items expanded, edges scanned).  Enabling or
 * disabling resets the totals. */
int scc_state_profile(scc_state* s, int enable);
int scc_state_profile_read(scc_state* s, double* ms, int64_t* launches, int64_t* items, int64_t* edges);

/* Traversal tunables (the reference hard-codes its BFS switch points,
 * gm_graph/inc/gm_bfs_template.h:418-487, 841-842): the autotuner
 * (scc_autotune) and callers may change them per state.  Any value <= 0
 * keeps the current setting. */
typedef struct scc_tuning {
    int32_t bu_alpha;             /* bottom-up when frontier edges * bu_alpha > traversed edges (14) */
    int32_t bu_div;               /* stay bottom-up while frontier > 2 * live / bu_div (24) */
    int32_t async_max;            /* a frontier this small counts as narrow (16384) */
    int32_t async_after;          /* narrow levels before the asynchronous drain (1) */
    int32_t async_keep;           /* items a warp keeps for itself before sharing (16, max 192) */
    int32_t async_blocks_per_sm;  /* resident blocks per SM in the drain (1, max 8) */
    int32_t huge_deg;             /* degree above which a top-down item is expanded edge-parallel (4096) */
    int32_t tile_min_live;        /* rounds with at least this many live vertices drain narrow frontiers
                                     tile by tile (one id range per SM, marks in shared memory); negative =
                                     never (the default) */
    int32_t tile_min_span;        /* smallest id range of a tile (2048) */
    int32_t pivot_salt;           /* xor on vertex ids before the degree rule's tie-break hash (0): picks
                                     another of the equally good pivots; changes speed, never labels */
    int32_t tail_live;            /* from the second recursion round on, at most this many live vertices are
                                     finished in one launch, a block per class (65536); negative = never */
    int32_t tail_class;           /* ... provided no class has more vertices than this (1024) */
    int32_t cta_deg;              /* top-down items above this degree (up to huge_deg) are expanded by a whole
                                     block, their adjacency staged in shared memory by bulk copies; negative =
                                     never */
} scc_tuning;
int scc_state_get_tuning(scc_state* s, scc_tuning* t);
/* Fields <= 0 keep their current value, except tile_min_live, tail_live and
 * cta_deg, where a negative value turns that path off, and pivot_salt, which any
 * non-zero value sets (and -1 resets to 0). */
int scc_state_set_tuning(scc_state* s, const scc_tuning* t);
/* Autotuner: successive halving over the tunables with a budget of max_trials full
 * decompositions (method) of g: a seeded sample of settings (the current one among
 * them) is timed once each, the faster half twice each, and so on; the winner is kept
 * in s (which is reset) and reported with its mean time. */
int scc_autotune(const scc_graph* g, scc_state* s, int method, int max_trials, scc_tuning* best, double* best_ms);

/* ---- colour (src/scc_color.cc) --------------------------------------------------------- */
int scc_get_new_color(scc_state* s, int32_t* color);          /* get_new_color,  scc_color.cc:38-54 */
int scc_get_curr_color(scc_state* s, int32_t* color);         /* get_curr_color, scc_color.cc:56-61 */
/* choose_pivot_from_color (scc_color.cc:64-93).  This engine's rule: the vertex
 * of that colour with the largest in-degree x out-degree (ties: fixed id hash).
 * SCC_ERR_NOT_FOUND and *pivot = SCC_NIL_NODE when the colour is empty. */
int scc_choose_pivot_from_color(const scc_graph* g, scc_state* s, int32_t color, int32_t* pivot);
/* generate_compact_set (scc_color.cc:95-113): members of a colour, ascending. */
int scc_generate_compact_set(const scc_graph* g, scc_state* s, int32_t color,
                             int32_t* out, int32_t capacity, int32_t* count);

/* ---- trim1 (src/scc_trim1.cc) ---------------------------------------------------------- */
/* One sweep: do_global_trim1 (scc_trim1.cc:112-135).  Trimmed vertices cascade
 * inside the sweep; *trimmed counts them. */
int scc_do_global_trim1(const scc_graph* g, scc_state* s, int32_t* trimmed);
/* do_global_trim1_compact (scc_trim1.cc:137-163): same over the compact targets. */
int scc_do_global_trim1_compact(const scc_graph* g, scc_state* s, int32_t* trimmed);
/* repeat_global_trim1(G, TRIM_STOP) (scc_trim1.cc:195-209): sweeps until a
 * sweep trims <= trim_stop vertices; this engine peels to the fixpoint whatever
 * trim_stop is (the CUDA reference's TRIM_STOP=0), and also rebuilds the
 * compact targets as the reference does once 10% are trimmed. */
int scc_repeat_global_trim1(const scc_graph* g, scc_state* s, int32_t trim_stop, int32_t* trimmed);
/* repeat_global_trim1_compact (scc_trim1.cc:277-290): create_trim1_compact + sweeps. */
int scc_repeat_global_trim1_compact(const scc_graph* g, scc_state* s, int32_t trim_stop, int32_t* trimmed);
/* create_trim1_compact (scc_trim1.cc:266-275): live vertices (colour != -2), ascending. */
int scc_create_trim1_compact(const scc_graph* g, scc_state* s, int32_t* live_count);

/* Trim1 with no device allocation.  No counterpart in the reference.
 * For callers that cannot call cudaMalloc: a serving process that reserves
 * its device-memory budget at start-up and must not fail or stall on an
 * allocation mid-request, or a host that lends the library a fixed pool.
 * Same result as scc_do_global_trim1 (peel to the fixpoint inside each
 * colour) on caller-owned device arrays of the current device: the CSR and
 * transpose (n+1 / m ints), d_color and d_scc (n ints, updated in place).
 * The scratch lives in one file-scope __device__ array of
 * 4 * SCC_NOALLOC_MAX_NODES + 128 ints (about 16 MiB); n above
 * SCC_NOALLOC_MAX_NODES is rejected with SCC_ERR_INVALID.  With CUDA's lazy
 * module loading (the default) the array is reserved on a device when the
 * first call on that device looks up its address, so call once with n = 0
 * (NULL arrays are accepted then) at start-up, before any stream capture: that
 * call reserves the array and does nothing else, and from then on the device
 * holds it until the process exits.  Every call looks the address up again,
 * with no allocation.  All calls share the array, so calls that overlap on the
 * GPU (other streams, other host threads) race; serialise them.  Work is
 * ordered on `stream` (cudaStream_t as void*, NULL = legacy default stream);
 * the call reads its counters back on that stream and returns once the work
 * is done. */
#define SCC_NOALLOC_MAX_NODES (1 << 20)
int scc_trim1_noalloc(int32_t n, const int32_t* d_begin, const int32_t* d_node_idx,
                      const int32_t* d_r_begin, const int32_t* d_r_node_idx,
                      int32_t* d_color, int32_t* d_scc, int32_t* trimmed, void* stream);

/* ---- trim2 (src/scc_trim2_new.cc, src/scc_trim2.cc) ---------------------------------- */
/* do_global_trim2_new (scc_trim2_new.cc:80-102): 2-vertex SCCs among the compact
 * targets, decided on the colours as they stood before the pass. */
int scc_do_global_trim2_new(const scc_graph* g, scc_state* s, int32_t* trimmed);
/* do_global_trim2 (scc_trim2.cc:24-152): same 2-SCC rule (alias). */
int scc_do_global_trim2(const scc_graph* g, scc_state* s, int32_t* trimmed);
/* repeat_global_trim2_new (scc_trim2_new.cc:105-114): until a pass trims <= exit_count. */
int scc_repeat_global_trim2_new(const scc_graph* g, scc_state* s, int32_t exit_count, int32_t* trimmed);

/* ---- FW-BW (src/scc_fb_global.cc, src/scc_fb_seq*.cc) ------------------------------- */
/* do_fw_bw_global_main(G, curr_color, count, create_work_items) (scc_fb_global.cc:133-219).
 * Pivot by scc_choose_pivot_from_color; FW set -> new colour, FW&BW -> SCC
 * (scc = pivot), BW only -> second new colour, rest keeps curr_color.  Returns
 * the SCC size.  count == 1 finishes the pivot alone, as the reference does. */
int scc_do_fw_bw_global_main(const scc_graph* g, scc_state* s, int32_t curr_color, int32_t count,
                             int create_work_items, int32_t* scc_size);
/* Same with an explicit pivot (the met 6/11 good_init_pivot override, scc_fb_global.cc:140-147). */
int scc_do_fw_bw_global_pivot(const scc_graph* g, scc_state* s, int32_t curr_color, int32_t pivot,
                              int create_work_items, int32_t* scc_size);
/* create_works_after_bfs_trim (scc_fb_global.cc:223-283): queue the fw/bw/base classes. */
int scc_create_works_after_bfs_trim(const scc_graph* g, scc_state* s, int32_t* num_items);
/* start_workers_fw_bw(G, N) (scc_fb_seq.cc:303-349) and start_workers_fw_bw_dfs(G, N)
 * (scc_fb_seq2.cc:292-351): resolve every queued colour class to SCCs.  Here
 * all classes advance together on the device (pivot per class, FW and BW
 * reachability, split, trim) until none is left; local_items is accepted for
 * interface parity. */
int scc_start_workers_fw_bw(const scc_graph* g, scc_state* s, int32_t local_items);
int scc_start_workers_fw_bw_dfs(const scc_graph* g, scc_state* s, int32_t local_items);
int scc_work_q_size(scc_state* s, int32_t* size);            /* work_q_size, my_work_queue.cc */
/* Work item table: colour and member count of each queued class (my_work{color,count}). */
int scc_work_q_items(scc_state* s, int32_t* colors, int32_t* counts, int32_t capacity, int32_t* num_items);

/* ---- WCC (src/scc_weak.cc) ------------------------------------------------------------ */
/* do_global_wcc (scc_weak.cc:128-196): over the compact targets, label =
 * minimum raw id (t, or t|0x20000000 when out-degree >= 50) over the same-colour
 * vertices reachable from t; each root (label == itself) gets a new colour and
 * its members take it. */
int scc_do_global_wcc(const scc_graph* g, scc_state* s);
/* create_work_items_from_wcc (scc_weak.cc:198-271): one queued class per root. */
int scc_create_work_items_from_wcc(const scc_graph* g, scc_state* s, int32_t* num_items);

/* ---- driver (src/scc_main.cc) ---------------------------------------------------------- */
#define SCC_METHOD_BASELINE       0   /* Trim1 + FW-BW */
#define SCC_METHOD_GLOBAL_FB      1   /* Trim1 + Global FW-BW + Trim1 + FW-BW */
#define SCC_METHOD_GLOBAL_WCC_FB  2   /* Trim1 + Global FW-BW + Trim1/2 + WCC + FW-BW */

#define SCC_PIVOT_DEGREE  0           /* max in-degree x out-degree */
#define SCC_PIVOT_LEARNED 1           /* MLP-scored pivot (scc_pivot_model_* must be loaded) */

typedef struct scc_run_stats {
    double ms_total;                  /* device time of the run (CUDA events) */
    double ms_trim1, ms_global_fb, ms_trim12, ms_wcc, ms_fb;   /* PHASE timers */
    int32_t trimmed_first;            /* first repeat_global_trim1 */
    int32_t first_scc_size;           /* do_fw_bw_global_main result */
    int32_t trimmed_second;           /* trim1 + trim2 + trim1 after the global step */
    int32_t num_sccs;                 /* "Total # SCCs" */
    int32_t num_wcc_classes;          /* work items created from WCC */
    int32_t fb_rounds;                /* device FW-BW rounds of the recursive phase */
    int64_t traversal_steps;          /* reachability steps launched */
    int32_t kernels_launched;         /* kernels this run launched */
    int32_t pivot_mode;
} scc_run_stats;

/* my_main::run (src/scc_main.cc:120-145) for methods 0, 1, 2 (5-7 and 11 map
 * to 2 as in check_args, scc_main.cc:170-171).  Method 3/4 (Tarjan) are the
 * sequential oracle in the reference and are not offered here
 * (SCC_ERR_UNSUPPORTED).  stats may be NULL. */
int scc_run(const scc_graph* g, scc_state* s, int method, int pivot_mode, scc_run_stats* stats);
/* post_process count (scc_main.cc:147-178): #v with scc[v] == v. */
int scc_count_sccs(scc_state* s, int32_t* count);
/* Canonical labels: smallest member id of each vertex's SCC (n ints). */
int scc_canonical_labels(scc_state* s, int32_t* labels);
int scc_canonical_labels_device(scc_state* s, int32_t* d_labels);
/* output_scc_list (src/scc_post_analyze.cc:31-53): "i id" lines, ids numbered
 * by first appearance.  path NULL = "scc_list.txt". */
int scc_output_scc_list(scc_state* s, const char* path);
/* read_file1 (src/common_main.h:316-341): labels from an scc_list.txt; *num_sccs = max id + 1. */
int scc_read_scc_list(const char* path, int32_t n, int32_t* labels, int32_t* num_sccs);
/* create_histogram_and_print (scc_post_analyze.cc:235-261): sizes[i], counts[i] ascending by size. */
int scc_histogram(scc_state* s, int32_t* sizes, int32_t* counts, int32_t capacity, int32_t* num_bins);

/* ---- updates (src/scc_incremental.cc, src/scc_decremental.cc, src/common_main.h:180-393) -- */
typedef struct scc_update_stats {
    double ms_total, ms_merge, ms_delete, ms_insert;   /* device time: CSR merge, split, merge phases */
    int32_t affected_delete;    /* vertices re-decomposed because their SCC lost an internal edge */
    int32_t affected_insert;    /* vertices in the merge region FW(inserted targets) & BW(inserted sources) */
    int64_t m_after;            /* edges after the batch */
    int32_t num_sccs;           /* SCC count after the batch */
} scc_update_stats;

/* Apply a batch to a graph whose state holds a complete decomposition (after
 * scc_run or a previous update): every copy of each deleted (u,v) is removed,
 * each inserted (u,v) is added (add_edge semantics: duplicates kept), on the
 * CSR and the transpose, lists kept sorted.  Labels are then recomputed only
 * where they can change: SCCs that lost an internal edge (the decremental
 * idea of delete_idea1 / method 9, src/scc_decremental.cc:7-24,
 * src/scc_trim1.cc:61-66) and the region reachable from the targets and
 * reaching the sources of inserted cross-SCC edges (where every merge of the
 * condensation graph of methods 6/7/11 happens, src/common_main.h:180-314).
 * on_device = 1: the four batch arrays are device pointers. */
int scc_update_batch(scc_graph* g, scc_state* s, int64_t n_ins, const int32_t* ins_src, const int32_t* ins_dst,
                     int64_t n_del, const int32_t* del_src, const int32_t* del_dst, int on_device,
                     scc_update_stats* stats);
int scc_incremental_insert(scc_graph* g, scc_state* s, int64_t n_ins, const int32_t* src, const int32_t* dst,
                           scc_update_stats* stats);
int scc_decremental_delete(scc_graph* g, scc_state* s, int64_t n_del, const int32_t* src, const int32_t* dst,
                           scc_update_stats* stats);
/* insert_idea1 (src/scc_incremental.cc:7-17, method 5): add the edges, then
 * reset the state and decompose from scratch. */
int scc_insert_idea1(scc_graph* g, scc_state* s, int64_t n_ins, const int32_t* src, const int32_t* dst,
                     scc_run_stats* stats);
/* create_scc_edges + insert_idea2 (src/common_main.h:180-314, src/scc_incremental.cc:19-27,
 * methods 6/7/11): the condensation graph over SCC ids labels[v] in [0, num_sccs)
 * (host array, e.g. from scc_read_scc_list), with every cross-SCC edge of g and of
 * the inserted batch (host arrays) mapped to (id(u), id(v)), duplicates dropped. */
int scc_condensation_graph(const scc_graph* g, const int32_t* labels, int32_t num_sccs, int64_t n_ins,
                           const int32_t* ins_src, const int32_t* ins_dst, scc_graph** out);
/* Method 7, the BFS of create_scc_edges (src/common_main.h:85-108, 210-219): topological
 * levels of a condensation DAG (scc_condensation_graph with no inserted edges).  levels[c]
 * (host array of dag's n) is the longest path from a source; a node on or behind a cycle
 * keeps the largest level + 1 of its released predecessors, or 0, as the reference's queue
 * leaves it.  *max_level = the largest level (the reference's "max_level:" line). */
int scc_topological_levels(const scc_graph* dag, int32_t* levels, int32_t* max_level);
/* Method 7, affect_level (src/common_main.h:232-262): every inserted edge (u, v) of the
 * original graph's n vertices with labels[u] != labels[v] covers the levels between those
 * of its two SCCs, inclusive.  affected[l], l in [0, max_level] (host array of
 * max_level + 1), receives how many edges cover level l (the prefix-summed affect_level);
 * *num_unaffected counts the levels no edge covers ("size of unaffected_levels:").  Sums
 * are exact int32 (the reference accumulates in float). */
int scc_affected_levels(const scc_graph* dag, const int32_t* levels, int32_t max_level, int32_t n,
                        const int32_t* labels, int64_t n_ins, const int32_t* ins_src, const int32_t* ins_dst,
                        int32_t* affected, int32_t* num_unaffected);
/* Method 7's trim shortcut (src/scc_trim1.cc:67-73) on a state of the condensation graph
 * with inserted edges: every node c with affected[levels[c]] == 0 is finished as its own
 * SCC (G_SCC = c, colour -2) before scc_run, which then decomposes only the rest.  No
 * inserted edge can join such a node to another.  *finished may be NULL. */
int scc_state_finish_unaffected(scc_state* s, const int32_t* levels, const int32_t* affected, int32_t max_level,
                                int32_t* finished);

/* ---- batched small graphs (no counterpart in the reference, which decomposes one
 * graph per process) -------------------------------------------------------------------- */
/* Many independent graphs stored as one disjoint union (graph i owns the vertices
 * [offsets[i], offsets[i+1]), no edge leaves a graph) are decomposed by ONE
 * persistent launch: each block takes whole graphs, largest first, and runs the
 * method (Trim1 to the fixpoint, then rounds of pivot / FW+BW / classify / peel over
 * every class of the graph) inside the block.  The plan captures the run (counter
 * reset, the launch, the counters back) into a CUDA graph once; each run is one
 * graph launch.  Results land in the state's colour and SCC arrays, so
 * scc_canonical_labels and the other output calls work on the union. */
typedef struct scc_batch_tuning {
    int32_t threads;              /* threads per block (512) */
    int32_t blocks_per_sm;        /* resident blocks per SM (2) */
    int32_t warp_deg;             /* lists longer than this are expanded by a whole warp (32) */
} scc_batch_tuning;
typedef struct scc_batch_stats {
    double ms_total;              /* device time of the run (events around the graph launch) */
    int32_t graphs, rounds, levels, max_rounds;
    int32_t host_submissions;     /* graph launches of the run (1) */
    int32_t kernels;              /* kernel launches inside it (1) */
} scc_batch_stats;
typedef struct scc_batch_plan scc_batch_plan;
int scc_batch_default_tuning(scc_batch_tuning* t);
/* offsets: host array of num_graphs + 1 vertex offsets, 0 .. g's vertex count.  The
 * plan keeps g and s (both must outlive it); tuning may be NULL (defaults). */
int scc_batch_plan_create(const scc_graph* g, scc_state* s, const int32_t* offsets, int32_t num_graphs,
                          const scc_batch_tuning* tuning, scc_batch_plan** out);
/* One run: every graph decomposed; synchronises.  stats may be NULL. */
int scc_batch_plan_run(scc_batch_plan* p, scc_batch_stats* stats);
int scc_batch_plan_free(scc_batch_plan* p);
/* Autotuner of the batched run: successive halving over threads per block, blocks
 * per SM and the warp cut-off.  Every candidate runs on a prefix of the graphs
 * (a quarter, then half, then all of them), the faster half goes on; the winner
 * is returned in *best with its time on the whole batch. */
int scc_batch_autotune(const scc_graph* g, scc_state* s, const int32_t* offsets, int32_t num_graphs,
                       scc_batch_tuning* best, double* best_ms);

/* ---- serving loop (no counterpart in the reference, whose dynamic methods read one
 * update file per process, src/common_main.h:500-732) ----------------------------------- */
typedef struct scc_server scc_server;
typedef struct scc_request_result {
    int status;                 /* SCC_OK; SCC_ERR_OOM when the batch can never fit the budget;
                                   SCC_ERR_BUSY when it waited longer than the admission age limit */
    int32_t session;
    double latency_ms;          /* completion - submission */
    double queue_ms;            /* admission - submission */
    scc_update_stats update;
} scc_request_result;
typedef struct scc_server_stats {
    int64_t completed, rejected, updates, max_inflight, bytes_in_use;
    double p50_ms, p99_ms, max_ms, updates_per_s;
    int64_t groups;             /* device updates applied (fewer than completed when requests coalesce) */
    int64_t offered_edges;      /* edges of every submission, shed ones included */
    int64_t shed;               /* submissions refused at the queue limit (SCC_ERR_BUSY from submit) */
    int64_t shed_edges;
    int64_t expired;            /* requests dropped at the age limit (status SCC_ERR_BUSY) */
    int64_t max_queued_edges;   /* largest backlog seen (edges queued, not yet admitted) */
    double offered_per_s;       /* offered edges / (last submission - first submission) */
} scc_server_stats;

/* num_slots worker threads; admission keeps resident graphs + admitted batches
 * under hbm_budget_bytes (estimates).  Requests of different sessions overlap
 * on the device (one stream per session); a session's requests run in order. */
int scc_server_create(int device, int num_slots, int64_t hbm_budget_bytes, scc_server** out);
/* Takes ownership of g and decomposes it (method 2); *session names it. */
int scc_server_add_graph(scc_server* sv, scc_graph* g, int32_t* session);
/* Copies the batch (host arrays) and queues it; returns at once. */
int scc_server_submit(scc_server* sv, int32_t session, int64_t n_ins, const int32_t* ins_src, const int32_t* ins_dst,
                      int64_t n_del, const int32_t* del_src, const int32_t* del_dst, int64_t* request_id);
/* Coalescing, off by default (max_requests = 1): a session's queued requests,
 * up to max_requests and max_edges edges in all, are composed into one batch
 * with the same final graph as applying them in order (an insert survives
 * unless a later request of the group deletes that pair) and applied by one
 * update.  Each request of a group then reports the group's result. */
int scc_server_set_coalesce(scc_server* sv, int32_t max_requests, int64_t max_edges);
/* Backpressure, off by default (0 = no limit).  A submission whose edges would
 * take the backlog (edges queued and not yet admitted, all sessions) above
 * max_queued_edges is refused: submit returns SCC_ERR_BUSY, queues nothing and
 * sets *request_id to -1.  A request still queued max_queue_ms after its
 * submission is dropped when a slot reaches it: it completes with status
 * SCC_ERR_BUSY and changes nothing.  Either way the client decides whether to
 * resend; the graph stays as the admitted requests left it. */
int scc_server_set_admission(scc_server* sv, int64_t max_queued_edges, double max_queue_ms);
int scc_server_wait(scc_server* sv, int64_t request_id, scc_request_result* out);
int scc_server_drain(scc_server* sv);
int scc_server_get_stats(scc_server* sv, scc_server_stats* out);
/* Canonical labels of an idle session (n ints). */
int scc_server_labels(scc_server* sv, int32_t session, int32_t* labels);
/* The session's graph (owned by the server; valid until scc_server_free). */
int scc_server_session_graph(scc_server* sv, int32_t session, scc_graph** g);
int scc_server_free(scc_server* sv);

/* ---- learned pivot proposer (no counterpart in the reference, whose pivot is the
 * first vertex of the colour, src/scc_color.cc:64-93) ------------------------------------
 * An 8 -> 64 -> 64 -> 1 ReLU network (4,801 parameters; parameter order W1[8][64],
 * b1[64], W2[64][64], b2[64], w3[64], b3) scores the vertices of every class; with
 * SCC_PIVOT_LEARNED each class pivots on its highest-scoring vertex.  Weights are
 * used in BF16 with FP32 accumulation (tensor cores for inference).  A pivot only
 * changes the speed of a run, never its labels.
 * Features per vertex (log1p-scaled, rounded to BF16): out-degree, in-degree, their
 * product, live out- and in-neighbours after the first peel (trim residue), size of
 * the vertex's class, mean degree of its first 4 out-neighbours, largest degree of
 * its first 4 in-neighbours. */
#define SCC_MLP_FEATURES 8
#define SCC_MLP_HIDDEN 64
#define SCC_MLP_PARAMS 4801
typedef struct scc_pivot_model scc_pivot_model;
/* Uniform He initialisation from a seed. */
int scc_pivot_model_create(int device, uint64_t seed, scc_pivot_model** out);
int scc_pivot_model_free(scc_pivot_model* m);
int scc_pivot_model_get_params(const scc_pivot_model* m, float* params);      /* FP32 master copy */
int scc_pivot_model_set_params(scc_pivot_model* m, const float* params);
int scc_pivot_model_save(const scc_pivot_model* m, const char* path);
int scc_pivot_model_load(int device, const char* path, scc_pivot_model** out);
/* Scores of count host feature rows.  tensor_cores = 1: the inference kernel
 * (tcgen05 MMA, BF16 activations); 0: FP32 activations on the CUDA cores. */
int scc_pivot_model_forward(const scc_pivot_model* m, const float* x, int64_t count, int tensor_cores, float* y);
/* Device time of one inference launch over count resident rows (CUDA events,
 * mean of iters launches after one warm-up): the tensor-core kernel alone. */
int scc_pivot_model_bench(const scc_pivot_model* m, int64_t count, int iters, double* ms_per_launch);
/* Mean squared error over count rows and its gradient w.r.t. the parameters as
 * used (BF16 weights, FP32 activations) -- the training kernels' gradient. */
int scc_pivot_model_loss_grad(const scc_pivot_model* m, const float* x, const float* t, int64_t count,
                              float* grad, float* loss);
/* Adam (beta 0.9 / 0.999) on shuffled mini-batches, on the device.
 * epoch_loss (may be NULL) receives the mean loss of each epoch. */
int scc_pivot_model_train(scc_pivot_model* m, const float* x, const float* t, int64_t count, int epochs,
                          int batch, float lr, uint64_t seed, float* epoch_loss);
/* Attach a model to a state (NULL detaches); runs with SCC_PIVOT_LEARNED need one. */
int scc_state_set_pivot_model(scc_state* s, scc_pivot_model* m);
/* Pivot logging for training: each FW-BW round of the following runs records
 * the features of about per_round sampled vertices of the classes it pivots,
 * up to capacity records in all (capacity 0 turns logging off and drops them). */
int scc_state_pivot_log(scc_state* s, int64_t capacity, int32_t per_round);
/* After a run: the records (features x[count][8], vertex v, size of its class at
 * the time) and targets t = log1p(|SCC(v)|) / log1p(class size), the share of
 * the class that v resolves as a pivot.  count receives the number written. */
int scc_state_pivot_records(scc_state* s, float* x, float* t, int32_t* v, int32_t* class_size, int64_t cap,
                            int64_t* count);

/* One-call convenience: host CSR in, canonical labels out (H2D + run + D2H). */
int scc_decompose_csr(int32_t n, int32_t m, const int32_t* begin, const int32_t* node_idx,
                      const int32_t* r_begin, const int32_t* r_node_idx, int method, int device,
                      int32_t* labels, int32_t* num_sccs, scc_run_stats* stats);

#ifdef __cplusplus
}
#endif
#endif /* SCC_CAPI_H */
