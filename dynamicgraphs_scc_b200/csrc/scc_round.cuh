// Shared definitions for one FW-BW round: arguments, pivot key, visit/claim.
#pragma once
#include "scc_internal.cuh"

#define DIR_SHIFT 30
#define ITEM_MASK 0x3FFFFFFF
#define REACH_THREADS 256
#define WBUF 256          // per-warp shared-memory buffer (items)

struct RoundArgs {
    const int32_t* begin; const int32_t* node_idx; const int32_t* r_begin; const int32_t* r_node_idx;
    int32_t* color; int32_t* scc; uint8_t* mark;
    unsigned long long* slot_key; int32_t* slot_pivot; int32_t* slot_fw; int32_t* slot_bw;
    int32_t* slot_count;        // members per colour (learned-pivot feature)
    int64_t colour_cap;
    int32_t* ctr;
    const int32_t* live; int32_t live_count;
    int32_t only_color;   // used when use_only
    int32_t use_only;
    int32_t huge_deg;           // top-down items above this degree go edge-parallel
    int32_t async_keep;         // items a warp keeps before sharing in the asynchronous drain
    int32_t async_bail;         // outstanding items at which the drain hands back to level steps
    uint32_t pivot_salt;        // xor on the vertex id before the tie-break hash of the degree rule (0 = none)
    int32_t cta_deg = -1;       // top-down items above this degree are expanded by the whole block (-1 = never)
    int64_t adj_len = 0;        // entries in node_idx and in r_node_idx (int4 probes stay below it)
    int32_t vec_adj = 0;        // both adjacency arrays start on a 16-byte boundary (int4 probes allowed)
};

// Adjacency arrays of g as RoundArgs needs them: int4 probes only where both
// arrays are 16-byte aligned, never past their m entries.
__host__ inline void round_args_adjacency(RoundArgs& a, const int32_t* node_idx, const int32_t* r_node_idx,
                                          int64_t m) {
    a.adj_len = m;
    a.vec_adj = ((reinterpret_cast<uintptr_t>(node_idx) | reinterpret_cast<uintptr_t>(r_node_idx)) & 15u) == 0;
}

__device__ __forceinline__ uint32_t pivot_hash(uint32_t v) {
    uint32_t x = v * 0x9E3779B1u;
    x ^= x >> 16; x *= 0x85EBCA6Bu; x ^= x >> 13;
    return x;
}

// The hash is a bijection (odd multipliers and xor-shifts), so a class's best
// key names its pivot: multiply by the inverses mod 2^32 and undo the shifts.
__device__ __forceinline__ int32_t pivot_unhash(uint32_t x) {
    x ^= (x >> 13) ^ (x >> 26);
    x *= 0xA5CB9243u;            // 0x85EBCA6B^-1 mod 2^32
    x ^= x >> 16;
    x *= 0x0E8B2F51u;            // 0x9E3779B1^-1 mod 2^32
    return (int32_t)x;
}

// Pivot key: (min(in*out, 2^32-2)+1) << 32 | hash(v); never 0, unique per vertex.
__device__ __forceinline__ unsigned long long pivot_key(const int32_t* __restrict__ begin,
                                                        const int32_t* __restrict__ r_begin, int32_t v) {
    unsigned long long outd = (unsigned)(__ldg(begin + v + 1) - __ldg(begin + v));
    unsigned long long ind = (unsigned)(__ldg(r_begin + v + 1) - __ldg(r_begin + v));
    unsigned long long prod = outd * ind;
    if (prod > 0xFFFFFFFEull) prod = 0xFFFFFFFEull;
    return ((prod + 1ull) << 32) | pivot_hash((uint32_t)v);
}

// The pivot of class c claims two fresh colours and seeds the frontier with
// its FW and BW items.
__device__ __forceinline__ void seed_pivot(const RoundArgs& a, int32_t v, int32_t c, int32_t* q) {
    a.slot_pivot[c + 1] = v;
    int32_t old = atomicAdd(a.ctr + CTR_NEXT_COLOR, 2);
    if ((int64_t)old + 4 >= a.colour_cap) { atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_COLOR_OVERFLOW); }
    a.slot_fw[c + 1] = old + 1;
    a.slot_bw[c + 1] = old + 2;
    a.mark[v] = 3;
    int32_t pos = atomicAdd(a.ctr + CTR_QLEN, 2);
    q[pos] = v;
    q[pos + 1] = v | (1 << DIR_SHIFT);
    atomicAdd(a.ctr + CTR_NUM_CLASSES, 1);
}

// Learned-pivot work of a round (scc_mlp.cu), after the degree keys are in
// slot_key: class sizes, training records when logging is on, and, when
// `learned`, the pivot of every class chosen by the network among the class's
// degree candidates and seeded into q (instead of the degree pick).
// *seeded: whether q was seeded; false when no class has a second candidate
// (the network would have no choice), and the caller seeds the degree pivots.
int scc_impl_pivot_prepare(const scc_graph* g, scc_state* s, RoundArgs& a, bool learned, int32_t* q, bool* seeded);

// Claim w for direction `dir` inside colour c; true if this thread claimed it.
__device__ __forceinline__ bool visit(const RoundArgs& a, int32_t w, int32_t c, int dir) {
    unsigned bit = 1u << dir;
    if (*(volatile uint8_t*)(a.mark + w) & bit) return false;
    if (__ldg(a.color + w) != c) return false;
    unsigned sh = (unsigned)(w & 3) * 8u;
    unsigned old = atomicOr(reinterpret_cast<unsigned*>(a.mark + (w & ~3)), bit << sh);
    return ((old >> sh) & bit) == 0u;
}

int scc_impl_reach(const scc_graph* g, scc_state* s, RoundArgs& a, int32_t qlen);
