// Device sorting for CSR construction: a stable least-significant-digit radix
// sort of 32- or 64-bit keys with optional int32 values, and the removal of
// repeated keys from a sorted array.  gm_graph builds its CSR by sorting each
// adjacency list (do_semi_sort, gm_graph/src/gm_graph.cc:385-420) and its
// transpose by scattering edges in source order (make_reverse_edges,
// :193-287); on the device both become one sort of packed keys.
//
// Each pass handles 8 bits, over tiles of 4,096 elements (256 threads x 16):
//  1. k_rs_hist: a shared-memory histogram of the digit per tile (one per
//     warp, summed), written digit-major (counts[digit * tiles + tile]);
//  2. an exclusive scan of those counts gives every (digit, tile) its first
//     output position;
//  3. k_rs_scatter: each warp ranks its own contiguous segment of the tile
//     (per-warp digit counts in shared memory, lanes of one digit found by
//     ballots inside a round); a block scan over (digit, warp) turns the
//     counts into slots.
//     The tile is reordered by digit in shared memory first, then written
//     out run by run, so the writes are coalesced.  Elements keep their
//     input order within each digit, so the sort is stable.
#include "scc_internal.cuh"
#include "scc_sort.cuh"

#define RS_THREADS 256
#define RS_ITEMS 16
#define RS_TILE (RS_THREADS * RS_ITEMS)
#define RS_BINS 256
#define RS_WARPS (RS_THREADS / 32)
#define SCAN_CHUNK 4096

// ------------------------------------------------------------------ exclusive scan (int32, in place)
__device__ __forceinline__ int32_t warp_incl(int32_t x) {
    int lane = threadIdx.x & 31;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    return x;
}

// Exclusive prefix of one value per thread over a 256-thread block; *total = the sum.
__device__ __forceinline__ int32_t block_excl256(int32_t x, int32_t* s_w, int32_t* total) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t inc = warp_incl(x);
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int32_t w = lane < RS_WARPS ? s_w[lane] : 0;
        w = warp_incl(w);
        if (lane < RS_WARPS) s_w[lane] = w;
    }
    __syncthreads();
    int32_t r = (wid ? s_w[wid - 1] : 0) + inc - x;
    *total = s_w[RS_WARPS - 1];
    __syncthreads();
    return r;
}

__global__ void k_scan_reduce(const int32_t* __restrict__ a, int64_t L, int32_t* __restrict__ sums) {
    __shared__ int32_t s_w[RS_WARPS];
    int64_t base = (int64_t)blockIdx.x * SCAN_CHUNK;
    int32_t x = 0;
    for (int r = 0; r < SCAN_CHUNK / RS_THREADS; ++r) {
        int64_t i = base + r * RS_THREADS + threadIdx.x;
        if (i < L) x += a[i];
    }
    int32_t tot = 0;
    block_excl256(x, s_w, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One block: exclusive scan of the chunk sums, in place.
__global__ void k_scan_top(int32_t* __restrict__ sums, int32_t nb) {
    __shared__ int32_t s_w[RS_WARPS];
    int32_t carry = 0;
    for (int32_t b0 = 0; b0 < nb; b0 += RS_THREADS) {
        int32_t i = b0 + threadIdx.x;
        int32_t x = i < nb ? sums[i] : 0;
        int32_t tot = 0;
        int32_t e = block_excl256(x, s_w, &tot);
        if (i < nb) sums[i] = carry + e;
        carry += tot;
    }
}

__global__ void k_scan_down(int32_t* __restrict__ a, int64_t L, const int32_t* __restrict__ sums) {
    __shared__ int32_t s_w[RS_WARPS];
    int64_t base = (int64_t)blockIdx.x * SCAN_CHUNK;
    int32_t run = sums[blockIdx.x];
    for (int r = 0; r < SCAN_CHUNK / RS_THREADS; ++r) {
        int64_t i = base + r * RS_THREADS + threadIdx.x;
        int32_t x = i < L ? a[i] : 0;
        int32_t tot = 0;
        int32_t e = block_excl256(x, s_w, &tot);
        if (i < L) a[i] = run + e;
        run += tot;
    }
}

static cudaError_t scan_excl(int32_t* a, int64_t L, int32_t* sums, cudaStream_t st) {
    int64_t nb = (L + SCAN_CHUNK - 1) / SCAN_CHUNK;
    if (nb == 0) return cudaSuccess;
    k_scan_reduce<<<(unsigned)nb, RS_THREADS, 0, st>>>(a, L, sums);
    k_scan_top<<<1, RS_THREADS, 0, st>>>(sums, (int32_t)nb);
    k_scan_down<<<(unsigned)nb, RS_THREADS, 0, st>>>(a, L, sums);
    return cudaPeekAtLastError();
}

// ------------------------------------------------------------------ radix passes
// Per-warp sub-histograms in shared memory (eight warps' atomics never meet
// on one counter), summed per digit at the end of the tile.
template <typename K>
__global__ void __launch_bounds__(RS_THREADS) k_rs_hist(const K* __restrict__ keys, int64_t m, int shift,
                                                        int32_t ntiles, int32_t* __restrict__ counts) {
    __shared__ int32_t h[RS_WARPS][RS_BINS];
    const int wid = threadIdx.x >> 5;
    for (int32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) h[w][threadIdx.x] = 0;
        __syncthreads();
        const int64_t base = (int64_t)tile * RS_TILE;
        K k[RS_ITEMS];
#pragma unroll
        for (int r = 0; r < RS_ITEMS; ++r) {
            int64_t i = base + r * RS_THREADS + threadIdx.x;
            k[r] = i < m ? keys[i] : (K)0;
        }
#pragma unroll
        for (int r = 0; r < RS_ITEMS; ++r)
            if (base + r * RS_THREADS + threadIdx.x < m)
                atomicAdd(&h[wid][(unsigned)(k[r] >> shift) & (RS_BINS - 1)], 1);
        __syncthreads();
        int32_t c = 0;
#pragma unroll
        for (int w = 0; w < RS_WARPS; ++w) c += h[w][threadIdx.x];
        counts[(int64_t)threadIdx.x * ntiles + tile] = c;
        __syncthreads();
    }
}

// One tile per pass of the loop.  Warp w owns the tile's elements
// [w * RS_SEG, (w + 1) * RS_SEG), read 32 consecutive ones per round, all
// rounds' loads issued before any is ranked.  Its lanes rank them inside the
// warp (earlier rounds first, then earlier lanes) against per-warp digit
// counts in shared memory; the lanes of a round that share a digit are found
// with eight ballots, one per digit bit.  One block scan over (digit, warp)
// then gives each warp's slot for each digit; the tile is reordered by digit
// in shared memory and written out run by run, each digit's output position
// read once per tile into shared memory.  Within a digit the order is rounds,
// lanes, warps -- the input order -- so the sort is stable.  Two blocks per
// SM (registers capped at 128): a third of the time of one block per SM.
#define RS_SEG (RS_TILE / RS_WARPS)
template <typename K, bool VALS>
__global__ void __launch_bounds__(RS_THREADS, 2) k_rs_scatter(const K* __restrict__ kin, K* __restrict__ kout,
                                                              const int32_t* __restrict__ vin,
                                                              int32_t* __restrict__ vout, int64_t m, int shift,
                                                              int32_t ntiles, const int32_t* __restrict__ offs) {
    __shared__ int32_t wcnt[RS_WARPS][RS_BINS];   // per-warp digit counts, then each warp's slot per digit
    __shared__ int32_t dst[RS_BINS];              // output position of the digit's tile-local slot 0
    __shared__ K skey[RS_TILE];
    __shared__ int32_t sval[VALS ? RS_TILE : 1];
    __shared__ int32_t s_w[RS_WARPS];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        const int64_t base = (int64_t)tile * RS_TILE;
        const int32_t cnt = (m - base < RS_TILE) ? (int32_t)(m - base) : RS_TILE;
        const int32_t seg = wid * RS_SEG;
        K k[RS_ITEMS];
        int32_t v[RS_ITEMS];
        int32_t rank[RS_ITEMS];
        // __ldcg (cached in L2 only): on this kernel's 32 outstanding loads
        // per thread the read-only path that `const __restrict__` selects
        // takes 1.6x as long per pass (5.98 against 3.70 ms over 4 passes of
        // C2's largest 134 M-pair upload run)
#pragma unroll
        for (int r = 0; r < RS_ITEMS; ++r) {
            const int32_t j = seg + r * 32 + lane;
            k[r] = j < cnt ? __ldcg(kin + base + j) : (K)0;
            v[r] = (VALS && j < cnt) ? __ldcg(vin + base + j) : 0;
        }
        const int32_t gofs = offs[(int64_t)threadIdx.x * ntiles + tile];    // digit threadIdx.x
#pragma unroll
        for (int q = lane; q < RS_BINS; q += 32) wcnt[wid][q] = 0;
        __syncwarp();
#pragma unroll
        for (int r = 0; r < RS_ITEMS; ++r) {
            const bool valid = seg + r * 32 + lane < cnt;
            const int d = (int)((unsigned)(k[r] >> shift) & (RS_BINS - 1));
            unsigned peers = __ballot_sync(0xFFFFFFFFu, valid);
#pragma unroll
            for (int bit = 0; bit < 8; ++bit) {
                const unsigned x = __ballot_sync(0xFFFFFFFFu, (d >> bit) & 1);
                peers &= ((d >> bit) & 1) ? x : ~x;
            }
            // an invalid lane may see valid peers of digit d; it neither reads nor writes
            const int leader = __ffs(peers) - 1;
            int32_t cur = (valid && lane == leader) ? wcnt[wid][d] : 0;
            cur = __shfl_sync(0xFFFFFFFFu, cur, leader < 0 ? lane : leader);
            rank[r] = cur + __popc(peers & lt);
            if (valid && lane == leader) wcnt[wid][d] = cur + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        // thread t owns digit t: the tile's start of the digit, then each warp's slot
        {
            int32_t c[RS_WARPS];
            int32_t tot = 0;
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) { c[w] = wcnt[w][threadIdx.x]; tot += c[w]; }
            int32_t all = 0;
            int32_t run = block_excl256(tot, s_w, &all);
            dst[threadIdx.x] = gofs - run;
#pragma unroll
            for (int w = 0; w < RS_WARPS; ++w) { wcnt[w][threadIdx.x] = run; run += c[w]; }
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < RS_ITEMS; ++r) {
            const int32_t j = seg + r * 32 + lane;
            if (j < cnt) {
                const int d = (int)((unsigned)(k[r] >> shift) & (RS_BINS - 1));
                const int32_t pos = wcnt[wid][d] + rank[r];
                skey[pos] = k[r];
                if (VALS) sval[pos] = v[r];
            }
        }
        __syncthreads();
        // the tile leaves in digit order: consecutive threads write consecutive
        // slots of each digit's run
#pragma unroll 4
        for (int32_t j = threadIdx.x; j < cnt; j += RS_THREADS) {
            const K kk = skey[j];
            const int d = (int)((unsigned)(kk >> shift) & (RS_BINS - 1));
            const int64_t pos = (int64_t)dst[d] + j;
            kout[pos] = kk;
            if (VALS) vout[pos] = sval[j];
        }
        __syncthreads();
    }
}

static inline size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Scratch of one sort: the alternate key and value buffers, the per-(digit,
// tile) counts and the scan's chunk sums.
static size_t sort_scratch(int64_t m, size_t key_bytes, bool vals) {
    const int64_t ntiles = (m + RS_TILE - 1) / RS_TILE;
    const int64_t L = (int64_t)RS_BINS * ntiles;
    return align256(key_bytes * (size_t)m) + (vals ? align256(sizeof(int32_t) * (size_t)m) : 0) +
           align256(sizeof(int32_t) * (size_t)L) + align256(sizeof(int32_t) * (size_t)(L / SCAN_CHUNK + 2));
}

size_t scc_impl_sort_scratch_bytes(int64_t m, size_t key_bytes, bool vals) {
    return sort_scratch(m > 0 ? m : 1, key_bytes, vals);
}

template <typename K>
static int radix_sort(const K* keys_in, K* keys_out, const int32_t* vals_in, int32_t* vals_out, int64_t m,
                      int bits, cudaStream_t st, void* scratch) {
    SCC_REQUIRE(m >= 0 && m < (1LL << 31), SCC_ERR_INVALID, "sort of %lld elements", (long long)m);
    const bool vals = vals_in != nullptr;
    if (m == 0) return SCC_OK;
    const int passes = (bits + 7) / 8;
    if (passes == 0) {
        SCC_CUDA(cudaMemcpyAsync(keys_out, keys_in, sizeof(K) * (size_t)m, cudaMemcpyDeviceToDevice, st));
        if (vals) SCC_CUDA(cudaMemcpyAsync(vals_out, vals_in, sizeof(int32_t) * (size_t)m, cudaMemcpyDeviceToDevice, st));
        return SCC_OK;
    }
    const int32_t ntiles = (int32_t)((m + RS_TILE - 1) / RS_TILE);
    const int64_t L = (int64_t)RS_BINS * ntiles;
    void* own = nullptr;
    cudaError_t e = cudaSuccess;
    if (!scratch) {
        e = scc_impl_malloc_async(&own, sort_scratch(m, sizeof(K), vals), st);
        scratch = own;
    }
    int rc = SCC_OK;
    if (e == cudaSuccess) {
        char* p = (char*)scratch;
        K* kt = (K*)p;                     p += align256(sizeof(K) * (size_t)m);
        int32_t* vt = nullptr;
        if (vals) { vt = (int32_t*)p;      p += align256(sizeof(int32_t) * (size_t)m); }
        int32_t* cnt = (int32_t*)p;        p += align256(sizeof(int32_t) * (size_t)L);
        int32_t* sums = (int32_t*)p;
        // the last pass must write keys_out: start in keys_out when the pass count is odd
        const K* ksrc = keys_in;
        const int32_t* vsrc = vals_in;
        K* kbuf[2] = {keys_out, kt};
        int32_t* vbuf[2] = {vals_out, vt};
        int cur = (passes & 1) ? 0 : 1;
        unsigned blocks = (unsigned)std::min<int32_t>(ntiles, 148 * 8);
        for (int p2 = 0; p2 < passes && e == cudaSuccess; ++p2) {
            int shift = 8 * p2;
            k_rs_hist<K><<<blocks, RS_THREADS, 0, st>>>(ksrc, m, shift, ntiles, cnt);
            e = cudaPeekAtLastError();
            if (e == cudaSuccess) e = scan_excl(cnt, L, sums, st);
            if (e != cudaSuccess) break;
            if constexpr (sizeof(K) == 4) {      // values ride along with 32-bit keys only
                if (vals)
                    k_rs_scatter<K, true><<<blocks, RS_THREADS, 0, st>>>(ksrc, kbuf[cur], vsrc, vbuf[cur], m, shift,
                                                                        ntiles, cnt);
                else
                    k_rs_scatter<K, false><<<blocks, RS_THREADS, 0, st>>>(ksrc, kbuf[cur], nullptr, nullptr, m,
                                                                         shift, ntiles, cnt);
            } else
                k_rs_scatter<K, false><<<blocks, RS_THREADS, 0, st>>>(ksrc, kbuf[cur], nullptr, nullptr, m, shift,
                                                                     ntiles, cnt);
            e = cudaPeekAtLastError();
            ksrc = kbuf[cur];
            vsrc = vbuf[cur];
            cur ^= 1;
        }
    }
    if (e != cudaSuccess) rc = scc_cuda_status(e, "radix sort", __FILE__, __LINE__);
    if (own) cudaFreeAsync(own, st);
    return rc;
}

int scc_impl_sort_pairs_u32(const uint32_t* keys_in, uint32_t* keys_out, const int32_t* vals_in, int32_t* vals_out,
                            int64_t m, int bits, cudaStream_t st, void* scratch) {
    return radix_sort<uint32_t>(keys_in, keys_out, vals_in, vals_out, m, bits, st, scratch);
}

__global__ void k_add_i32(const int32_t* __restrict__ in, int32_t* __restrict__ out, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        out[i] += in[i];
}

int scc_impl_scan_i32(const int32_t* in, int32_t* out, int64_t n, bool inclusive, cudaStream_t st) {
    SCC_REQUIRE(n >= 0 && n < (1LL << 31), SCC_ERR_INVALID, "scan of %lld elements", (long long)n);
    SCC_REQUIRE(!(inclusive && in == out), SCC_ERR_INVALID, "inclusive scan in place");
    if (n == 0) return SCC_OK;
    if (in != out) SCC_CUDA(cudaMemcpyAsync(out, in, sizeof(int32_t) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    void* sums = nullptr;
    SCC_CUDA(scc_impl_malloc_async(&sums, sizeof(int32_t) * (size_t)(n / SCAN_CHUNK + 2), st));
    cudaError_t e = scan_excl(out, n, (int32_t*)sums, st);
    if (e == cudaSuccess && inclusive) {
        k_add_i32<<<scc_blocks(n, RS_THREADS, 148 * 8), RS_THREADS, 0, st>>>(in, out, n);
        e = cudaPeekAtLastError();
    }
    cudaFreeAsync(sums, st);
    SCC_CUDA(e);
    return SCC_OK;
}

int scc_impl_sort_keys_u64(const unsigned long long* keys_in, unsigned long long* keys_out, int64_t m, int bits,
                           cudaStream_t st) {
    return radix_sort<unsigned long long>(keys_in, keys_out, nullptr, nullptr, m, bits, st, nullptr);
}

// ------------------------------------------------------------------ unique of a sorted array
// Per tile the kept elements (first of each run of equal keys) are counted,
// the counts scanned, and each tile writes its kept elements in order: the
// key itself, or (POS) its index.
template <typename K>
__global__ void k_uniq_count(const K* __restrict__ a, int64_t m, int32_t ntiles, int32_t* __restrict__ counts) {
    __shared__ int32_t s_w[RS_WARPS];
    for (int32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int64_t base = (int64_t)tile * RS_TILE;
        int32_t c = 0;
        for (int r = 0; r < RS_ITEMS; ++r) {
            int64_t i = base + r * RS_THREADS + threadIdx.x;
            if (i < m && (i == 0 || a[i] != a[i - 1])) ++c;
        }
        int32_t tot = 0;
        block_excl256(c, s_w, &tot);
        if (threadIdx.x == 0) counts[tile] = tot;
    }
}

template <typename K, typename O, bool POS>
__global__ void k_uniq_write(const K* __restrict__ a, O* __restrict__ out, int64_t m, int32_t ntiles,
                             const int32_t* __restrict__ offs) {
    __shared__ int32_t s_w[RS_WARPS];
    for (int32_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        int64_t base = (int64_t)tile * RS_TILE;
        int32_t run = offs[tile];
        for (int r = 0; r < RS_ITEMS; ++r) {
            int64_t i = base + r * RS_THREADS + threadIdx.x;
            bool keep = i < m && (i == 0 || a[i] != a[i - 1]);
            int32_t tot = 0;
            int32_t e = block_excl256(keep ? 1 : 0, s_w, &tot);
            if (keep) out[(int64_t)run + e] = POS ? (O)i : (O)a[i];
            run += tot;
        }
    }
}

template <typename K, typename O, bool POS>
static int uniq(const K* a, O* out, int64_t m, int64_t* m_out, cudaStream_t st) {
    *m_out = 0;
    if (m <= 0) return SCC_OK;
    SCC_REQUIRE(m < (1LL << 31), SCC_ERR_INVALID, "unique of %lld elements", (long long)m);
    const int32_t ntiles = (int32_t)((m + RS_TILE - 1) / RS_TILE);
    void *cnt = nullptr, *sums = nullptr;
    SCC_CUDA(scc_impl_malloc_async(&cnt, sizeof(int32_t) * ((size_t)ntiles + 1), st));
    cudaError_t e = scc_impl_malloc_async(&sums, sizeof(int32_t) * ((size_t)ntiles / SCAN_CHUNK + 2), st);
    int32_t total = 0;
    if (e == cudaSuccess) {
        unsigned blocks = (unsigned)std::min<int32_t>(ntiles, 148 * 8);
        k_uniq_count<K><<<blocks, RS_THREADS, 0, st>>>(a, m, ntiles, (int32_t*)cnt);
        e = cudaPeekAtLastError();
        // one extra zero entry after the tiles: its exclusive prefix is the total
        if (e == cudaSuccess) e = cudaMemsetAsync((int32_t*)cnt + ntiles, 0, sizeof(int32_t), st);
        if (e == cudaSuccess) e = scan_excl((int32_t*)cnt, (int64_t)ntiles + 1, (int32_t*)sums, st);
        if (e == cudaSuccess) {
            k_uniq_write<K, O, POS><<<blocks, RS_THREADS, 0, st>>>(a, out, m, ntiles, (const int32_t*)cnt);
            e = cudaPeekAtLastError();
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&total, (int32_t*)cnt + ntiles, sizeof(int32_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (cnt) cudaFreeAsync(cnt, st);
    if (sums) cudaFreeAsync(sums, st);
    if (e != cudaSuccess) return scc_cuda_status(e, "unique", __FILE__, __LINE__);
    *m_out = total;
    return SCC_OK;
}

int scc_impl_unique_u64(const unsigned long long* a, unsigned long long* out, int64_t m, int64_t* m_out,
                        cudaStream_t st) {
    return uniq<unsigned long long, unsigned long long, false>(a, out, m, m_out, st);
}

int scc_impl_segment_starts(const uint32_t* keys, int64_t m, int32_t* starts, int64_t* count, cudaStream_t st) {
    return uniq<uint32_t, int32_t, true>(keys, starts, m, count, st);
}
