// Internal definitions shared by the engine's translation units.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>
#include <vector>
#include "scc_capi.h"

// ---------------------------------------------------------------- error plumbing
void scc_set_error(const char* fmt, ...);
int scc_cuda_status(cudaError_t e, const char* what, const char* file, int line);

#define SCC_CUDA(call)                                                            \
    do {                                                                          \
        cudaError_t _e = (call);                                                  \
        if (_e != cudaSuccess) return scc_cuda_status(_e, #call, __FILE__, __LINE__); \
    } while (0)
#define SCC_TRY(call)                                                             \
    do { int _s = (call); if (_s != SCC_OK) return _s; } while (0)
#define SCC_REQUIRE(cond, code, ...)                                              \
    do { if (!(cond)) { scc_set_error(__VA_ARGS__); return (code); } } while (0)
// launch check: cudaGetLastError after each launch
#define SCC_LAUNCHED(st) SCC_CUDA(cudaPeekAtLastError()); (st)->kernels++

// ---------------------------------------------------------------- constants
#define SCC_THREADS 256
// Host loops that repeat a device pass until a counter reads zero (peel
// overflow rounds, level releases) shrink their list every round, so they end
// well before this; reaching it reports SCC_ERR_TIMEOUT instead of a partial result.
#define SCC_HOST_ROUND_LIMIT 1000000
#define SCC_WCC_HIGH_DEG_FLAG 0x20000000   // scc_weak.cc:141-146
#define SCC_WCC_ROOT_MASK 0x1FFFFFFF
#define SCC_WCC_HIGH_DEG 50                // scc_weak.cc:143

// ---------------------------------------------------------------- graph
struct scc_graph {
    int device = 0;
    int32_t n = 0;
    int64_t m = 0;
    int32_t* begin = nullptr;     // [n+1]  out-CSR offsets      (gm_graph::begin)
    int32_t* node_idx = nullptr;  // [m]    out-neighbours       (gm_graph::node_idx)
    int32_t* r_begin = nullptr;   // [n+1]  in-CSR offsets       (gm_graph::r_begin)
    int32_t* r_node_idx = nullptr;// [m]    in-neighbours        (gm_graph::r_node_idx)
    bool owns = true;
    bool async_arrays = false;    // arrays come from cudaMallocAsync (after an update)
    mutable int64_t self_loops = -1;  // edges u->u in the CSR; -1 = not counted yet
};

// Device counters block (one allocation, mirrored to pinned host memory).
enum {
    CTR_COUNT = 0,       // generic per-launch counter (trimmed, visited, ...)
    CTR_COUNT2,
    CTR_COUNT3,
    CTR_QLEN,            // length of the produced queue
    CTR_QLEN2,
    CTR_NEXT_COLOR,      // colour allocator (last colour handed out)
    CTR_OVERFLOW,        // trim cascade overflow length
    CTR_CHANGED,         // label propagation change flag
    CTR_ERROR,           // device-side error code (bounded waits, capacity)
    CTR_ERROR_INFO,
    CTR_NUM_CLASSES,
    CTR_SPARE0,
    CTR_SPARE1,
    CTR_ABAIL,           // asynchronous drain: hand the frontier back to level steps
    CTR_SPARE3,
    CTR_SPARE4,
    CTR_EDGES = 16,      // u64 (slots 16-17): edges of the next top-down frontier
    CTR_LIVE_EDGES = 18, // u64 (slots 18-19): in+out degree of the vertices being traversed
    CTR_ASYNC_ITEMS = 20,// u64 (slots 20-21): items expanded by the asynchronous drain (ledger)
    CTR_ASYNC_EDGES = 22,// u64 (slots 22-23): edges scanned by it
    CTR_MAXDEG = 24,     // largest in+out degree among the vertices a round traverses
    // asynchronous traversal queue counters, one 128-byte line each (polled by idle warps)
    CTR_AHEAD = 32,
    CTR_ATAIL = 64,
    CTR_AWORK = 96,
    CTR_MAX = 128
};

// device error codes written to CTR_ERROR
#define SCC_DEVERR_QUEUE_OVERFLOW 1
#define SCC_DEVERR_WAIT_LIMIT     2
#define SCC_DEVERR_COLOR_OVERFLOW 3

struct scc_state {
    int device = 0;
    int32_t n = 0;
    cudaStream_t stream = nullptr;
    int kernels = 0;                 // kernels launched (statistics)
    int64_t traversal_steps = 0;
    int32_t fb_rounds = 0;           // recursion rounds (statistics)
    bool fresh = false;              // colours all -1 and nothing finished (set by reset, cleared by any phase)
    bool prefinished = false;        // fresh except vertices finished as their own SCC (method 7's shortcut)

    int32_t* color = nullptr;        // G_Color [n]
    int32_t* scc = nullptr;          // G_SCC   [n]
    int32_t* wcc = nullptr;          // G_WCC   [n]
    int32_t* live = nullptr;         // compact trim targets [n]
    int32_t live_count = 0;          // host mirror; -1 = not built (trim_targets.size()==0)
    int32_t* live_tmp = nullptr;     // [n] scratch list
    int32_t* qa = nullptr;           // [2n+64] traversal queue A
    int32_t* qb = nullptr;           // [2n+64] traversal queue B
    int32_t* aq = nullptr;           // [2n+64] asynchronous traversal queue, kept at -1 between uses
    int32_t* uf = nullptr;           // [n] union-find parents (weak-component split)
    unsigned long long* cnt = nullptr;   // [n] live counts of the counting peel, (in << 32) | out; also n ints of scratch for updates
    unsigned long long* ccnt = nullptr;  // [n] counts within colours of later peels (allocated at first use)
    int32_t* hq = nullptr;           // [2n+64] high-degree items deferred by a top-down level
    long long* hoff = nullptr;       // [2n+64] prefix of their degrees
    uint8_t* mark = nullptr;         // [n rounded to 4] reachability marks (bit0 FW, bit1 BW)
    int32_t* aux = nullptr;          // [n] per-vertex scratch (trim2 mates, pivot slots...)
    int32_t* tq = nullptr;           // tile drain inboxes [tq_cap], kept at -1 between uses (allocated at first use)
    int64_t tq_cap = 0;
    int32_t* tctr = nullptr;         // tile drain counters (allocated at first use)
    unsigned long long* bkey = nullptr;  // [3n] pivot key per colour of the one-launch tail (allocated at first use)
    int32_t* block_sums = nullptr;   // scan scratch
    int32_t* ctr = nullptr;          // device counters [CTR_MAX]
    int32_t* h_ctr = nullptr;        // pinned host mirror [CTR_MAX]

    // per-colour slot arrays (index = colour id), capacity colour_cap
    int64_t colour_cap = 0;
    unsigned long long* slot_key = nullptr;  // pivot key per colour
    int32_t* slot_pivot = nullptr;           // pivot vertex per colour
    int32_t* slot_fw = nullptr;              // new fw colour per colour
    int32_t* slot_bw = nullptr;              // new bw colour per colour
    int32_t* slot_count = nullptr;           // member count per colour

    // work queue (my_work items): classes that still need resolving
    std::vector<int32_t> wq_colors;
    std::vector<int32_t> wq_counts;

    // learned pivot (scc_mlp.cu)
    scc_pivot_model* pivot_model = nullptr;  // attached model (not owned)
    int pivot_mode = SCC_PIVOT_DEGREE;       // mode of the run in progress
    bool cnt_valid = false;                  // cnt holds the first peel's residue
    int32_t* pivot_cand = nullptr;           // [n] candidates of the learned choice (vertex ids)
    float* pivot_score = nullptr;            // [n] their scores
    void* pivot_x = nullptr;                 // [n] their BF16 feature rows (16 B each)
    // pivot logging (training records)
    int64_t log_cap = 0;
    int32_t log_per_round = 0;
    uint32_t log_salt = 0;
    float* log_x = nullptr;                  // [log_cap][8]
    int32_t* log_v = nullptr;                // [log_cap]
    int32_t* log_size = nullptr;             // [log_cap]
    int32_t* log_ctr = nullptr;              // records appended (may exceed log_cap)

    cudaEvent_t ev[16];
    bool events = false;

    // defaults from a B200 sweep on the mixed R-MAT + grid workload (fewer
    // resident warps in the drain mean less contention on its queue)
    // (the tile drain and the one-launch tail are off by default: measured
    // slower than the shared-queue drain and the round engine on C2)
    scc_tuning tune = {14, 24, 1 << 14, 1, 16, 1, 4096, -1, 2048, 0, 1 << 16, 1024, 256};

    // kernel ledger (scc_state_profile): device time and algorithmic bytes of
    // the asynchronous reachability drain, timed with events on `stream`
    bool ledger_on = false;
    cudaEvent_t lev[2];
    double ledger_ms = 0.0;
    long long ledger_launches = 0;
    long long ledger_items = 0;
    long long ledger_edges = 0;
};

// ---------------------------------------------------------------- helpers (host)
static inline unsigned scc_blocks(int64_t n, int threads = SCC_THREADS, int64_t cap = 148LL * 16) {
    int64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return (unsigned)b;
}
int scc_sync_counters(scc_state* s);   // D2H copy of ctr -> h_ctr and stream sync
int scc_zero_counters(scc_state* s, int first, int count);
int scc_check_device_error(scc_state* s);

// phase implementations shared between translation units
int scc_impl_compact_live(const scc_graph* g, scc_state* s, bool from_all);
int scc_impl_trim1(const scc_graph* g, scc_state* s, bool use_live, int32_t* trimmed);
int scc_impl_trim2(const scc_graph* g, scc_state* s, int32_t* trimmed);
int scc_impl_ensure_colour_cap(scc_state* s, int64_t need);
int scc_impl_fb_round(const scc_graph* g, scc_state* s, int32_t only_color, int32_t forced_pivot,
                      int32_t* scc_found, int32_t* active_classes, bool pipeline = false);
int scc_impl_wcc(const scc_graph* g, scc_state* s);
int scc_impl_uf_split(const scc_graph* g, scc_state* s, int32_t* num_classes);
bool scc_trace_on();
// Stream-ordered scratch from the library's own memory pool on the current
// device: freed blocks stay reserved for the next call (no re-mapping of
// gigabytes per upload or update) until scc_release_cached_memory.
cudaError_t scc_impl_malloc_async(void** p, size_t bytes, cudaStream_t st);
bool scc_impl_take_wait_injection();   // consumes a pending SCC_INJECT_WAIT
void scc_impl_pivot_release(scc_state* s);   // frees the learned-pivot and logging buffers
// classes_split: the live classes are already weak components (a split ran last)
int scc_impl_resolve_all(const scc_graph* g, scc_state* s, bool classes_split = false);
// Decomposes every remaining class in one launch (a block per class); *taken is
// false, with nothing done, when a class is above tune.tail_class vertices.
int scc_impl_resolve_tail(const scc_graph* g, scc_state* s, bool* taken);
int scc_impl_get_live_host(scc_state* s, std::vector<int32_t>& out);
int scc_impl_count_colour(scc_state* s, int32_t color, int32_t* count);
int scc_impl_build_graph_from_device_edges(int32_t n, int64_t m, const int32_t* d_src,
                                           const int32_t* d_dst, int flags, int device,
                                           scc_graph** out);
int scc_impl_transpose(scc_graph* g, cudaStream_t st);
