// Tile-owned asynchronous reachability: the deep, narrow waves of FW-BW
// (fw_trim_global / bw_trim_global, src/scc_fb_global.cc:32-130) over inputs
// whose vertex ids carry locality, such as a grid numbered row by row.
//
// The live id range [lo, lo + ntiles * span) is cut into one contiguous tile
// per block (one block per SM, all resident).  A block keeps its tile's
// reachability marks in shared memory, two bits per vertex, and expands its
// own vertices only:
//  * a neighbour inside the tile is claimed with a shared-memory atomic, and
//    the global mark byte is set with a reduction nobody waits on, so a hop
//    inside a tile costs the adjacency and colour loads and no global atomic
//    round trip;
//  * a neighbour in another tile is claimed with the global atomicOr (as the
//    shared-queue drain does) and, if newly claimed, appended to the owner's
//    inbox, a slice of one queue kept at -1 between launches.
// The two claims can race (an owner's shared claim while another block's
// global claim is in flight); the owner then finds the inbox copy already set
// in shared memory and drops it, so no vertex is expanded twice.  An item that
// arrives with TILE_PRE set (a seed, or an item the owner spilled from a
// warp's full list) was claimed for the owner already and is expanded as is.
// Each (vertex, direction) enters an inbox at most once by a global claim and
// at most once as a spill, so an inbox of 4 x span slots cannot overflow.
//
// Termination: `W` counts items that exist anywhere (inbox slots, warp lists,
// items being expanded), published lazily as in the shared-queue drain: a
// warp adds its net change before it waits, every 8th iteration, and before
// it makes items visible to anyone else (remote pushes, spills).  W reaches 0
// only when no item exists, and then every warp leaves.  Idle warps reset
// their wait bound while W or the progress word (bumped by busy warps every
// 32 iterations) moves.  When W passes `bail_at` the frontier has grown wide:
// every warp hands its list back, the blocks meet at a grid barrier (all sends
// done), and each block hands back its inbox; the host continues with the
// level-synchronous kernels.  Every wait is bounded and reports
// SCC_DEVERR_WAIT_LIMIT through the state's error word.
#include <stdlib.h>
#include <algorithm>
#include "scc_round.cuh"
#include "scc_tile.cuh"

#define TILE_WARPS (TILE_THREADS / 32)
#define TILE_EMPTY (-1)
#define TILE_PRE 0x80000000u
#define TILE_IDLE_LIMIT (1 << 22)
#define TILE_SLOT_LIMIT (1 << 20)
#define TILE_BAR_LIMIT (1 << 24)
#define TILE_SMEM_BYTES (4 * TILE_MARK_WORDS + 16 * TILE_WARPS * TILE_WBUF)

struct TileArgs {
    int32_t lo;          // first vertex of tile 0 (a multiple of 16)
    int32_t span;        // vertices per tile (a multiple of 16, at most TILE_MAX_SPAN)
    int32_t ntiles;      // tiles = blocks
    int32_t n;
    int64_t inbox_cap;   // slots per tile inbox (4 x span + 64)
    int32_t* tq;         // ntiles x inbox_cap slots, TILE_EMPTY between launches
    int32_t* tctr;       // TILE_CTR_WORDS counters, zero at launch except W
    int32_t* qout;       // hand-back list of a bail (its length in CTR_QLEN)
    int64_t qcap;        // its capacity
    int32_t bail_at;
    int32_t keep;        // items a warp keeps when it shares the rest with the block
};

__device__ __forceinline__ int32_t tld(const int32_t* p) { return *(const volatile int32_t*)p; }

__device__ __forceinline__ void tile_error(const RoundArgs& a, int info) {
    atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_WAIT_LIMIT);
    atomicExch(a.ctr + CTR_ERROR_INFO, info);
}

// Seeds go to their owners' inboxes, flagged as already claimed.
__global__ void k_tile_seed(RoundArgs a, TileArgs t, const int32_t* __restrict__ q, int32_t qlen) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < qlen; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t it = q[i];
        int32_t v = it & ITEM_MASK;
        uint32_t o = v >= t.lo ? (uint32_t)(v - t.lo) / (uint32_t)t.span : 0xFFFFFFFFu;
        if (o >= (uint32_t)t.ntiles) { atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW); continue; }
        int32_t pos = atomicAdd(t.tctr + (int64_t)o * TILE_CTR_STRIDE + TILE_TAIL_OFF, 1);
        if (pos >= t.inbox_cap) { atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW); continue; }
        t.tq[(int64_t)o * t.inbox_cap + pos] = (int32_t)((uint32_t)it | TILE_PRE);
    }
}

struct TileList {
    int32_t* it; int32_t* b; int32_t* e; int32_t* c;   // this warp's list in shared memory
    int32_t count;                                      // warp-uniform
    int32_t pushed;                                     // net change since the last publish
    int32_t* W; int32_t* tail; int32_t* inbox; int64_t cap; int32_t* err; int32_t keep;
    // Items beyond `keep` go to this tile's inbox (flagged: already claimed
    // here), where idle warps of the block take them.  The count is published
    // first, and the fence orders it before the items become visible.
    __device__ __forceinline__ bool spill(int32_t keep) {
        int lane = threadIdx.x & 31;
        int32_t ns = count - keep;
        if (ns <= 0) return true;
        int32_t pos = 0;
        if (lane == 0) {
            if (pushed) atomicAdd(W, pushed);
            __threadfence();
            pos = atomicAdd(tail, ns);
        }
        pushed = 0;
        pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
        if ((int64_t)pos + ns > cap) {
            // cannot happen (each item enters an inbox at most twice); the
            // items are dropped and the launch reports an error
            if (lane == 0) atomicExch(err, SCC_DEVERR_QUEUE_OVERFLOW);
            count = keep;
            return false;
        }
        __syncwarp();
        for (int32_t j = lane; j < ns; j += 32)
            *(volatile int32_t*)(inbox + pos + j) = (int32_t)((uint32_t)it[keep + j] | TILE_PRE);
        __syncwarp();
        count = keep;
        return true;
    }
    __device__ __forceinline__ void push(bool p, int32_t item, int32_t bb, int32_t ee, int32_t cc) {
        int lane = threadIdx.x & 31;
        unsigned bal = __ballot_sync(0xFFFFFFFFu, p);
        if (p) {
            int32_t pos = count + __popc(bal & ((1u << lane) - 1u));
            it[pos] = item; b[pos] = bb; e[pos] = ee; c[pos] = cc;
        }
        count += __popc(bal);
        pushed += __popc(bal);
        if (count > TILE_WBUF - 32) spill(keep);
    }
};

// Claim neighbour w (direction dir, class c) found by a lane.  Returns 1 for a
// new vertex of this tile (push locally), 2 for a new vertex of another tile
// (send to its owner), 0 otherwise.
__device__ __forceinline__ int tile_claim(const RoundArgs& a, uint32_t* smark, int32_t lo_k, int32_t span,
                                          int32_t w, int dir, unsigned gmark) {
    uint32_t li = (uint32_t)(w - lo_k);
    const unsigned bit = 1u << dir;
    if (li < (uint32_t)span) {
        uint32_t sh = (li & 15u) * 2u + (uint32_t)dir;
        uint32_t old = atomicOr(smark + (li >> 4), 1u << sh);
        if (old & (1u << sh)) return 0;
        // publish the claim to other tiles' senders; nobody waits for it
        atomicOr(reinterpret_cast<unsigned*>(a.mark + (w & ~3)), bit << ((w & 3) * 8u));
        return 1;
    }
    if (gmark & bit) return 0;
    unsigned sh = (unsigned)(w & 3) * 8u;
    unsigned old = atomicOr(reinterpret_cast<unsigned*>(a.mark + (w & ~3)), bit << sh);
    return ((old >> sh) & bit) ? 0 : 2;
}

// Send the lanes' remote items (flag r) to their owners' inboxes: W is raised
// first, and the fence orders that before the items become visible.
__device__ __forceinline__ bool tile_send(const RoundArgs& a, const TileArgs& t, bool r, int32_t item) {
    unsigned bal = __ballot_sync(0xFFFFFFFFu, r);
    if (!bal) return true;
    int lane = threadIdx.x & 31;
    if (lane == 0) {
        atomicAdd(t.tctr + TILE_W, __popc(bal));
        __threadfence();
    }
    __syncwarp();
    bool ok = true;
    if (r) {
        int32_t v = item & ITEM_MASK;
        uint32_t o = v >= t.lo ? (uint32_t)(v - t.lo) / (uint32_t)t.span : 0xFFFFFFFFu;
        if (o >= (uint32_t)t.ntiles) {
            atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW);
            ok = false;
        } else {
            int32_t pos = atomicAdd(t.tctr + (int64_t)o * TILE_CTR_STRIDE + TILE_TAIL_OFF, 1);
            if (pos < t.inbox_cap) {
                *(volatile int32_t*)(t.tq + (int64_t)o * t.inbox_cap + pos) = item;
            } else {
                atomicExch(a.ctr + CTR_ERROR, SCC_DEVERR_QUEUE_OVERFLOW);
                ok = false;
            }
        }
    }
    return __all_sync(0xFFFFFFFFu, ok);
}

// Expand one item per lane (valid lanes).  b < 0: range and class not known yet.
__device__ __forceinline__ void tile_expand(const RoundArgs& a, const TileArgs& t, uint32_t* smark, int32_t lo_k,
                                            bool valid, int32_t it, int32_t b, int32_t e, int32_t c,
                                            TileList& L, long long* edge_acc) {
    const int lane = threadIdx.x & 31;
    int32_t dir = 0;
    if (valid) {
        int32_t v = it & ITEM_MASK;
        dir = (it >> DIR_SHIFT) & 1;
        if (b < 0) {
            const int32_t* off = dir ? a.r_begin : a.begin;
            b = __ldg(off + v); e = __ldg(off + v + 1);
            c = __ldg(a.color + v);
        }
        *edge_acc += e - b;
    } else {
        b = e = 0;
    }
    int32_t deg = e - b;
    // long lists: the whole warp, 32 neighbours per step
    unsigned big = __ballot_sync(0xFFFFFFFFu, deg > 32);
    while (big) {
        int l = __ffs(big) - 1;
        big &= big - 1;
        int32_t lb = __shfl_sync(0xFFFFFFFFu, b, l), le = __shfl_sync(0xFFFFFFFFu, e, l);
        int32_t lc = __shfl_sync(0xFFFFFFFFu, c, l), ld = __shfl_sync(0xFFFFFFFFu, dir, l);
        const int32_t* adj = ld ? a.r_node_idx : a.node_idx;
        const int32_t* off = ld ? a.r_begin : a.begin;
        for (int32_t k0 = lb; k0 < le; k0 += 32) {
            int32_t k = k0 + lane;
            int r = 0;
            int32_t w = 0, wb = -1, we = -1;
            if (k < le) {
                w = __ldg(adj + k);
                unsigned gm = *(volatile uint8_t*)(a.mark + w);
                int32_t col = __ldg(a.color + w);
                wb = __ldg(off + w); we = __ldg(off + w + 1);
                if (col == lc) r = tile_claim(a, smark, lo_k, t.span, w, ld, gm);
            }
            L.push(r == 1, w | (ld << DIR_SHIFT), wb, we, lc);
            tile_send(a, t, r == 2, w | (ld << DIR_SHIFT));
        }
    }
    // short lists: four neighbours per step, loads issued together
    int32_t mydeg = deg <= 32 ? deg : 0;
    int32_t maxd = (int32_t)__reduce_max_sync(0xFFFFFFFFu, (unsigned)mydeg);
    const int32_t* adj = dir ? a.r_node_idx : a.node_idx;
    const int32_t* off = dir ? a.r_begin : a.begin;
    for (int32_t j0 = 0; j0 < maxd; j0 += 4) {
        int32_t w[4], col[4], wb[4], we[4];
        unsigned gm[4];
        int r[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) w[u] = (j0 + u) < mydeg ? __ldg(adj + b + j0 + u) : -1;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            bool p = w[u] >= 0;
            gm[u] = p ? (unsigned)*(volatile uint8_t*)(a.mark + w[u]) : 0u;
            col[u] = p ? __ldg(a.color + w[u]) : 0;
            wb[u] = p ? __ldg(off + w[u]) : -1;
            we[u] = p ? __ldg(off + w[u] + 1) : -1;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
            r[u] = (w[u] >= 0 && col[u] == c) ? tile_claim(a, smark, lo_k, t.span, w[u], dir, gm[u]) : 0;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            L.push(r[u] == 1, w[u] | (dir << DIR_SHIFT), wb[u], we[u], c);
            tile_send(a, t, r[u] == 2, w[u] | (dir << DIR_SHIFT));
        }
    }
}

__global__ void __launch_bounds__(TILE_THREADS, 1) k_reach_tile(RoundArgs a, TileArgs t) {
    extern __shared__ uint32_t tsm[];
    __shared__ int s_stop;
    uint32_t* smark = tsm;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t* lists = reinterpret_cast<int32_t*>(tsm + TILE_MARK_WORDS);
    const int32_t k = blockIdx.x;
    const int32_t lo_k = t.lo + k * t.span;
    int32_t* W = t.tctr + TILE_W;
    int32_t* prog = t.tctr + TILE_PROG;
    int32_t* bail = t.tctr + TILE_BAIL;
    int32_t* err = a.ctr + CTR_ERROR;
    int32_t* my_head = t.tctr + k * TILE_CTR_STRIDE;
    int32_t* my_tail = my_head + TILE_TAIL_OFF;
    int32_t* inbox = t.tq + (int64_t)k * t.inbox_cap;
    TileList L{lists + (0 * TILE_WARPS + wid) * TILE_WBUF, lists + (1 * TILE_WARPS + wid) * TILE_WBUF,
               lists + (2 * TILE_WARPS + wid) * TILE_WBUF, lists + (3 * TILE_WARPS + wid) * TILE_WBUF, 0, 0,
               W, my_tail, inbox, t.inbox_cap, err, t.keep};

    // this tile's marks, two bits per vertex
    const int32_t words = t.span >> 4;
    for (int32_t j = threadIdx.x; j < words; j += blockDim.x) {
        int32_t v0 = lo_k + 16 * j;
        uint32_t packed = 0;
        if (v0 + 16 <= t.n) {
            uint4 m = __ldcg(reinterpret_cast<const uint4*>(a.mark + v0));
            uint32_t x[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
            for (int q = 0; q < 16; ++q) packed |= ((x[q >> 2] >> ((q & 3) * 8)) & 3u) << (2 * q);
        } else {
            for (int q = 0; q < 16; ++q)
                if (v0 + q < t.n) packed |= ((uint32_t)a.mark[v0 + q] & 3u) << (2 * q);
        }
        smark[j] = packed;
    }
    if (threadIdx.x == 0) s_stop = 0;
    __syncthreads();
    // no block claims a vertex of another tile before every tile has read its marks
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(t.tctr + TILE_BAR, 1);
        int spins = 0;
        while (tld(t.tctr + TILE_BAR) < t.ntiles && tld(err) == 0 && spins < TILE_BAR_LIMIT) {
            ++spins;
            __nanosleep(64);
        }
        if (spins >= TILE_BAR_LIMIT) tile_error(a, 3);
        if (tld(err)) s_stop = 1;
    }
    __syncthreads();
    if (s_stop) return;

    int idle = 0;
    uint32_t iter = 0;
    int32_t last_w = -1, last_p = -1;
    long long my_edges = 0, my_items = 0;
    bool bailed = false;
    while (true) {
        if (L.count == 0) {
            if (lane == 0 && L.pushed != 0) atomicAdd(W, L.pushed);
            L.pushed = 0;
            int32_t got = 0, base = 0;
            if (lane == 0) {
                int32_t tl = tld(my_tail), h = tld(my_head);
                if (tl > t.inbox_cap) tl = (int32_t)t.inbox_cap;
                if (h < tl) {
                    int32_t kk = min(32, tl - h);
                    if (atomicCAS(my_head, h, h + kk) == h) { got = kk; base = h; }
                }
            }
            got = __shfl_sync(0xFFFFFFFFu, got, 0);
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (got == 0) {
                ++idle;
                if ((idle & 7) == 1) {
                    int32_t w = 1, e = 0, bl = 0, p = 0;
                    if (lane == 0) { w = tld(W); e = tld(err); bl = tld(bail); p = tld(prog); }
                    w = __shfl_sync(0xFFFFFFFFu, w, 0);
                    e = __shfl_sync(0xFFFFFFFFu, e, 0);
                    bl = __shfl_sync(0xFFFFFFFFu, bl, 0);
                    p = __shfl_sync(0xFFFFFFFFu, p, 0);
                    if (bl) { bailed = true; break; }
                    if (w == 0 || e != 0) break;
                    if (w != last_w || p != last_p) { last_w = w; last_p = p; idle = 1; }
                }
                if (idle > TILE_IDLE_LIMIT) {
                    if (lane == 0) tile_error(a, 4);
                    break;
                }
                __nanosleep(idle < 16 ? 64 : 256);
                continue;
            }
            idle = 0;
            int32_t item = TILE_EMPTY;
            if (lane < got) {
                volatile int32_t* slot = inbox + base + lane;
                int spins = 0;
                while ((item = *slot) == TILE_EMPTY && spins < TILE_SLOT_LIMIT) { ++spins; __nanosleep(20); }
                if (item != TILE_EMPTY) *slot = TILE_EMPTY;
            }
            if (__any_sync(0xFFFFFFFFu, lane < got && item == TILE_EMPTY)) {
                if (lane == 0) tile_error(a, 5);
                break;
            }
            bool acc = false;
            if (lane < got) {
                if ((uint32_t)item & TILE_PRE) {
                    acc = true;
                } else {
                    // claimed by another tile's sender: expand unless this tile claimed it itself
                    uint32_t li = (uint32_t)((item & ITEM_MASK) - lo_k);
                    uint32_t sh = (li & 15u) * 2u + (uint32_t)((item >> DIR_SHIFT) & 1);
                    acc = !(atomicOr(smark + (li >> 4), 1u << sh) & (1u << sh));
                }
            }
            unsigned bal = __ballot_sync(0xFFFFFFFFu, acc);
            L.pushed -= got - __popc(bal);          // dropped copies leave the count
            if (acc) {
                int32_t pos = __popc(bal & ((1u << lane) - 1u));
                L.it[pos] = (int32_t)((uint32_t)item & ~TILE_PRE); L.b[pos] = -1; L.e[pos] = -1; L.c[pos] = 0;
            }
            __syncwarp();
            L.count = __popc(bal);
            if (L.count == 0) continue;
        }
        int32_t kk = min(32, L.count);
        int32_t top = L.count - kk + lane;
        int32_t it = (lane < kk) ? L.it[top] : 0;
        int32_t ib = (lane < kk) ? L.b[top] : 0;
        int32_t ie = (lane < kk) ? L.e[top] : 0;
        int32_t ic = (lane < kk) ? L.c[top] : 0;
        __syncwarp();
        L.count -= kk;
        tile_expand(a, t, smark, lo_k, lane < kk, it, ib, ie, ic, L, &my_edges);
        my_items += kk;
        L.pushed -= kk;
        if ((++iter & 7) == 0) {
            int32_t stop = 0;
            if (lane == 0) {
                int32_t w = atomicAdd(W, L.pushed) + L.pushed;
                if (w > t.bail_at) atomicExch(bail, 1);
                if ((iter & 31) == 0) atomicAdd(prog, 1);
                stop = tld(bail) ? 1 : (tld(err) ? 2 : 0);
            }
            L.pushed = 0;
            stop = __shfl_sync(0xFFFFFFFFu, stop, 0);
            if (stop) { bailed = stop == 1; break; }
        }
        // share what this warp cannot expand in its next iteration
        if (L.count > 2 * t.keep && !L.spill(t.keep)) break;
    }
    for (int o = 16; o > 0; o >>= 1) my_edges += __shfl_down_sync(0xFFFFFFFFu, my_edges, o);
    if (lane == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + CTR_ASYNC_ITEMS), (unsigned long long)my_items);
        atomicAdd(reinterpret_cast<unsigned long long*>(a.ctr + CTR_ASYNC_EDGES), (unsigned long long)my_edges);
    }
    if (bailed) {
        // this warp's unexpanded items go back to the host's frontier
        int32_t pos = 0;
        if (lane == 0 && L.count > 0) pos = atomicAdd(a.ctr + CTR_QLEN, L.count);
        pos = __shfl_sync(0xFFFFFFFFu, pos, 0);
        if ((int64_t)pos + L.count > t.qcap) {
            if (lane == 0) atomicExch(err, SCC_DEVERR_QUEUE_OVERFLOW);
        } else {
            for (int32_t j = lane; j < L.count; j += 32) t.qout[pos + j] = L.it[j];
        }
        if (lane == 0) atomicExch(&s_stop, 2);
    }
    __threadfence();
    __syncthreads();
    if (s_stop != 2) return;
    // hand-back: wait until every block has stopped sending, then return the
    // inbox items not yet taken (dropping copies this tile claimed itself)
    if (threadIdx.x == 0) {
        atomicAdd(t.tctr + TILE_BAR, 1);
        int spins = 0;
        while (tld(t.tctr + TILE_BAR) < 2 * t.ntiles && tld(err) == 0 && spins < TILE_BAR_LIMIT) {
            ++spins;
            __nanosleep(64);
        }
        if (spins >= TILE_BAR_LIMIT) tile_error(a, 6);
    }
    __syncthreads();
    if (tld(err)) return;
    int32_t h = tld(my_head), tl = tld(my_tail);
    if (tl > t.inbox_cap) tl = (int32_t)t.inbox_cap;
    for (int32_t j = h + threadIdx.x; j < tl; j += blockDim.x) {
        volatile int32_t* slot = inbox + j;
        int32_t item = TILE_EMPTY;
        int spins = 0;
        while ((item = *slot) == TILE_EMPTY && spins < TILE_SLOT_LIMIT) { ++spins; __nanosleep(20); }
        if (item == TILE_EMPTY) { tile_error(a, 7); continue; }
        *slot = TILE_EMPTY;
        bool keep_it = true;
        if (!((uint32_t)item & TILE_PRE)) {
            uint32_t li = (uint32_t)((item & ITEM_MASK) - lo_k);
            uint32_t sh = (li & 15u) * 2u + (uint32_t)((item >> DIR_SHIFT) & 1);
            keep_it = !(atomicOr(smark + (li >> 4), 1u << sh) & (1u << sh));
        }
        if (keep_it) {
            int32_t pos = atomicAdd(a.ctr + CTR_QLEN, 1);
            if (pos < t.qcap) t.qout[pos] = (int32_t)((uint32_t)item & ~TILE_PRE);
            else atomicExch(err, SCC_DEVERR_QUEUE_OVERFLOW);
        }
    }
}

// ------------------------------------------------------------------ host driver
static int tile_blocks(int device) {
    static int cached[64] = {0};
    if (device >= 0 && device < 64 && cached[device]) return cached[device];
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (sms > TILE_MAX_TILES) sms = TILE_MAX_TILES;
    if (device >= 0 && device < 64) cached[device] = sms;
    return sms;
}

bool scc_impl_tile_eligible(const scc_state* s, int32_t live_lo, int32_t live_hi) {
    if (s->tune.tile_min_live <= 0 || s->live_count < s->tune.tile_min_live) return false;
    if (s->n >= ITEM_MASK) return false;
    int64_t lo = live_lo & ~15;
    int64_t range = (int64_t)live_hi + 1 - lo;
    int64_t per = (range + tile_blocks(s->device) - 1) / tile_blocks(s->device);
    return per <= TILE_MAX_SPAN;
}

int scc_impl_reach_tile(const scc_graph* g, scc_state* s, RoundArgs& a, const int32_t* qin, int32_t qlen,
                        int32_t* qout, int32_t live_lo, int32_t live_hi, int32_t* handed_back) {
    (void)g;
    *handed_back = 0;
    int blocks = tile_blocks(s->device);
    TileArgs t;
    t.lo = live_lo & ~15;
    int64_t range = (int64_t)live_hi + 1 - t.lo;
    int64_t per = (range + blocks - 1) / blocks;
    per = std::max<int64_t>(per, s->tune.tile_min_span);
    per = (per + 15) & ~15LL;
    SCC_REQUIRE(per <= TILE_MAX_SPAN, SCC_ERR_STATE, "tile span %lld above %d", (long long)per, TILE_MAX_SPAN);
    t.span = (int32_t)per;
    t.ntiles = (int32_t)((range + per - 1) / per);
    t.n = s->n;
    t.inbox_cap = 4LL * per + 64;
    t.bail_at = std::max<int32_t>(8 * s->tune.async_max, 1 << 16);
    // inbox storage (kept at -1 between launches) and counters, allocated at first use
    int64_t need = (int64_t)t.ntiles * t.inbox_cap;
    if (s->tq_cap < need) {
        cudaFree(s->tq);
        s->tq = nullptr;
        s->tq_cap = 0;
        int64_t cap = std::max<int64_t>(need, 4LL * s->n + 64LL * TILE_MAX_TILES + 64);
        SCC_CUDA(cudaMalloc(&s->tq, sizeof(int32_t) * (size_t)cap));
        SCC_CUDA(cudaMemsetAsync(s->tq, 0xFF, sizeof(int32_t) * (size_t)cap, s->stream));
        s->tq_cap = cap;
    }
    if (!s->tctr) SCC_CUDA(cudaMalloc(&s->tctr, sizeof(int32_t) * TILE_CTR_WORDS));
    t.tq = s->tq;
    t.tctr = s->tctr;
    t.qout = qout;
    t.qcap = 2LL * s->n + 64;
    t.keep = std::min<int32_t>(std::max<int32_t>(s->tune.async_keep, 4), 64);
    SCC_CUDA(cudaMemsetAsync(s->tctr, 0, sizeof(int32_t) * TILE_CTR_WORDS, s->stream));
    SCC_CUDA(cudaMemcpyAsync(s->tctr + TILE_W, &qlen, sizeof(int32_t), cudaMemcpyHostToDevice, s->stream));
    SCC_TRY(scc_zero_counters(s, CTR_QLEN, 1));
    SCC_TRY(scc_zero_counters(s, CTR_ASYNC_ITEMS, 4));
    k_tile_seed<<<scc_blocks(qlen, SCC_THREADS, 148 * 4), SCC_THREADS, 0, s->stream>>>(a, t, qin, qlen);
    SCC_LAUNCHED(s);
    static bool attr_set[64] = {false};
    if (s->device >= 0 && s->device < 64 && !attr_set[s->device]) {
        SCC_CUDA(cudaFuncSetAttribute(k_reach_tile, cudaFuncAttributeMaxDynamicSharedMemorySize, TILE_SMEM_BYTES));
        attr_set[s->device] = true;
    }
    if (s->ledger_on) SCC_CUDA(cudaEventRecord(s->lev[0], s->stream));
    k_reach_tile<<<t.ntiles, TILE_THREADS, TILE_SMEM_BYTES, s->stream>>>(a, t);
    SCC_LAUNCHED(s);
    if (s->ledger_on) SCC_CUDA(cudaEventRecord(s->lev[1], s->stream));
    s->traversal_steps++;
    SCC_TRY(scc_sync_counters(s));
    if (s->ledger_on) {
        float ms = 0.f;
        SCC_CUDA(cudaEventElapsedTime(&ms, s->lev[0], s->lev[1]));
        s->ledger_ms += ms;
        s->ledger_launches++;
        s->ledger_items += *reinterpret_cast<long long*>(s->h_ctr + CTR_ASYNC_ITEMS);
        s->ledger_edges += *reinterpret_cast<long long*>(s->h_ctr + CTR_ASYNC_EDGES);
    }
    if (s->h_ctr[CTR_ERROR]) {
        // leave the inboxes clean for the next launch, then report
        SCC_CUDA(cudaMemsetAsync(s->tq, 0xFF, sizeof(int32_t) * (size_t)s->tq_cap, s->stream));
        return scc_check_device_error(s);
    }
    *handed_back = s->h_ctr[CTR_QLEN];
    if (scc_trace_on())
        fprintf(stderr, "[scc] reach tile seeds=%d tiles=%d span=%d handed_back=%d\n", qlen, t.ntiles, t.span,
                *handed_back);
    return SCC_OK;
}
