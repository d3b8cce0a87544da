// Tile-owned asynchronous reachability (scc_tile.cu): constants shared with
// the host driver in scc_reach.cu.
#pragma once
#include "scc_round.cuh"

#define TILE_THREADS 512
#define TILE_WBUF 256                 // per-warp list (items)

#define TILE_MARK_WORDS 16384         // shared marks: 2 bits per vertex
#define TILE_MAX_SPAN (TILE_MARK_WORDS * 16)
#define TILE_MAX_TILES 160            // at least one per SM of a B200 (148)
// counters: per tile a head and a tail on separate 64-byte halves of a line,
// then the outstanding-item count, a progress word, the bail flag and the
// grid-barrier count, one line each
#define TILE_CTR_STRIDE 32
#define TILE_TAIL_OFF 16
#define TILE_W (TILE_MAX_TILES * TILE_CTR_STRIDE)
#define TILE_PROG (TILE_W + 32)
#define TILE_BAIL (TILE_W + 64)
#define TILE_BAR (TILE_W + 96)
#define TILE_CTR_WORDS (TILE_W + 128)

// True when the round may use the tile drain: the state's tunables enable it
// for this many live vertices, and the live id range [live_lo, live_hi]
// splits into one tile per SM of at most TILE_MAX_SPAN vertices.
bool scc_impl_tile_eligible(const scc_state* s, int32_t live_lo, int32_t live_hi);
// Runs the tile drain from the qlen items of qin.  On return either the
// traversal is complete (*handed_back = 0) or the frontier grew wide and its
// *handed_back unexpanded items are in qout for the level-synchronous kernels.
int scc_impl_reach_tile(const scc_graph* g, scc_state* s, RoundArgs& a, const int32_t* qin, int32_t qlen,
                        int32_t* qout, int32_t live_lo, int32_t live_hi, int32_t* handed_back);
