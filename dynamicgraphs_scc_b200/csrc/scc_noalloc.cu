// Allocation-free Trim1.
//
// Some callers cannot call cudaMalloc: a serving process that reserves its
// whole device-memory budget at start-up and must not fail or stall on an
// allocation in the middle of a request, or a host that hands this library a
// fixed memory pool it may not grow.  scc_trim1_noalloc gives them Trim1 to
// the fixpoint (the same kernels and result as scc_do_global_trim1) without
// any device allocation: the caller passes the CSR, the transpose and the
// colour / SCC arrays, and the scratch the peel needs (a colour snapshot, two
// overflow lists, the overflowed vertices' colours and the counters) lives in
// the file-scope array below, which every GPU that loads this library holds
// until the process exits.
#include "scc_internal.cuh"

// Scratch layout (int32 words): snapshot | overflow A | overflow B | item colours | counters.
#define NOALLOC_WORDS (4 * SCC_NOALLOC_MAX_NODES + CTR_MAX)
static __device__ __align__(256) int32_t g_trim1_scratch[NOALLOC_WORDS];

int scc_trim1_with_scratch(int32_t n, const int32_t* begin, const int32_t* node_idx, const int32_t* r_begin,
                           const int32_t* r_node_idx, int32_t* color, int32_t* scc, int32_t* snapshot,
                           int32_t* ovf_a, int32_t* ovf_b, int32_t* item_colors, int32_t* ctr, cudaStream_t st,
                           int32_t* trimmed);

// Device address of the scratch array on the current device.  In host code
// the array's name is only a host-side stand-in, so the address is looked up
// with the device current.  The lookup is cheap and runs on every call, so an
// address never outlives the context it came from (a cudaDeviceReset between
// calls makes the next call look it up afresh).  With lazy module loading the
// first lookup on a device is what loads this library's module there and
// reserves the array.
static int scratch_for_current_device(int32_t** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_trim1_scratch);
    if (e != cudaSuccess) return scc_cuda_status(e, "cudaGetSymbolAddress(g_trim1_scratch)", __FILE__, __LINE__);
    *out = (int32_t*)p;
    return SCC_OK;
}

extern "C" int scc_trim1_noalloc(int32_t n, const int32_t* d_begin, const int32_t* d_node_idx,
                                 const int32_t* d_r_begin, const int32_t* d_r_node_idx, int32_t* d_color,
                                 int32_t* d_scc, int32_t* trimmed, void* stream) {
    SCC_REQUIRE(trimmed, SCC_ERR_INVALID, "trimmed is NULL");
    SCC_REQUIRE(n >= 0, SCC_ERR_INVALID, "negative vertex count %d", n);
    SCC_REQUIRE(n <= SCC_NOALLOC_MAX_NODES, SCC_ERR_INVALID,
                "scc_trim1_noalloc handles at most %d vertices (got %d); use scc_do_global_trim1",
                SCC_NOALLOC_MAX_NODES, n);
    SCC_REQUIRE(n == 0 || (d_begin && d_node_idx && d_r_begin && d_r_node_idx && d_color && d_scc), SCC_ERR_INVALID,
                "NULL device array");
    *trimmed = 0;
    // the scratch is reserved on this device before anything else, so a call
    // with n = 0 at start-up makes every later call allocation-free
    int32_t* base = nullptr;
    SCC_TRY(scratch_for_current_device(&base));
    if (n == 0) return SCC_OK;
    const int64_t M = SCC_NOALLOC_MAX_NODES;
    return scc_trim1_with_scratch(n, d_begin, d_node_idx, d_r_begin, d_r_node_idx, d_color, d_scc, base, base + M,
                                  base + 2 * M, base + 3 * M, base + 4 * M, (cudaStream_t)stream, trimmed);
}
