// Learned pivot proposer: an 8 -> 64 -> 64 -> 1 ReLU network (4,801
// parameters) that scores live vertices as FW-BW pivots.  The reference picks
// the first vertex of a colour (src/scc_color.cc:64-93; the CUDA path the
// smallest id, src_CUDA/scc_cuda_fb_global.cu:426-440); this engine's plain rule
// is the largest in-degree x out-degree.  A pivot only changes how fast the
// classes shrink, never the labels.
//
// Features of vertex v (log1p-scaled, then rounded to BF16 so that training and
// inference see the same inputs): out-degree, in-degree, their product, live
// out- and in-neighbours left by the first peel (trim residue), size of v's
// colour class, mean log-degree of v's first 4 out-neighbours and largest
// log-degree of its first 4 in-neighbours.
//
// Inference (k_mlp_score_tc): 128 vertices per tile; both hidden layers are
// tcgen05.mma (kind::f16, BF16 operands from shared memory, FP32 accumulators
// in tensor memory) issued by one thread; the epilogues (bias, ReLU, BF16
// repack, last layer) read the accumulators back with tcgen05.ld, one row per
// thread.  Training (k_mlp_train): one fused kernel per mini-batch runs the
// forward and backward passes of 128 samples per block on the CUDA cores
// (BF16 weights, FP32 activations and accumulation) and reduces the weight
// gradients in shared memory as small register-tiled GEMMs (dW2 = H1^T dZ2,
// dW1 = X^T dZ1) before one atomicAdd per parameter per block; Adam updates
// the FP32 master copy and refreshes the BF16 copy.
//
// Training records come from plain runs: with logging on, each FW-BW round
// stores the features of sampled vertices of the classes it pivots and the
// class size; after the run the target is log1p(|SCC(v)|) / log1p(class size),
// the share of its class that v resolves when it is the pivot.
#include <cuda_bf16.h>
#include <math.h>
#include <cmath>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <vector>
#include "scc_round.cuh"

#define MLP_IN SCC_MLP_FEATURES
#define MLP_H SCC_MLP_HIDDEN
#define OFF_W1 0                              // [MLP_IN][MLP_H]
#define OFF_B1 (OFF_W1 + MLP_IN * MLP_H)      // [MLP_H]
#define OFF_W2 (OFF_B1 + MLP_H)               // [MLP_H][MLP_H]
#define OFF_B2 (OFF_W2 + MLP_H * MLP_H)       // [MLP_H]
#define OFF_W3 (OFF_B2 + MLP_H)               // [MLP_H]
#define OFF_B3 (OFF_W3 + MLP_H)               // [1]
#define MLP_PARAMS (OFF_B3 + 1)
static_assert(MLP_PARAMS == SCC_MLP_PARAMS, "parameter count");

#define TC_ROWS 128                           // vertices per inference tile (MMA M)
#define TRAIN_B 128                           // samples per training block
#define TRAIN_S (TRAIN_B + 1)                 // padded stride of the per-sample columns
#define NEIGH_SAMPLE 4                        // neighbours read for the neighbour-degree features
#define WAIT_LIMIT (1 << 24)                  // mbarrier polls before giving up

struct scc_pivot_model {
    int device = 0;
    float* master = nullptr;         // FP32 [MLP_PARAMS]
    __nv_bfloat16* w16 = nullptr;    // BF16 copy used by every forward pass
    float* grad = nullptr;           // FP32 gradient accumulator (kept zero between steps)
    float* m1 = nullptr;             // Adam moments
    float* m2 = nullptr;
    float* loss = nullptr;           // device scalar: sum of squared errors
    int32_t* err = nullptr;          // device error flag of the inference kernel
    int64_t steps = 0;
};

// ------------------------------------------------------------------ features
__device__ __forceinline__ float lg1p(float x) { return log1pf(fmaxf(x, 0.f)); }
__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float degree_log(const int32_t* __restrict__ off, int32_t v) {
    return lg1p((float)(__ldg(off + v + 1) - __ldg(off + v)));
}

__device__ void vertex_features(const RoundArgs& a, const unsigned long long* __restrict__ cnt, int32_t v,
                                int32_t c, float* f) {
    int32_t ob = __ldg(a.begin + v), oe = __ldg(a.begin + v + 1);
    int32_t ib = __ldg(a.r_begin + v), ie = __ldg(a.r_begin + v + 1);
    float od = (float)(oe - ob), id = (float)(ie - ib);
    f[0] = lg1p(od);
    f[1] = lg1p(id);
    f[2] = lg1p(od * id);
    const unsigned long long r = cnt ? cnt[v] : 0ull;        // peel residue, (in << 32) | out
    f[3] = cnt ? lg1p((float)(uint32_t)r) : f[0];
    f[4] = cnt ? lg1p((float)(uint32_t)(r >> 32)) : f[1];
    f[5] = lg1p((float)a.slot_count[c + 1]);
    float s = 0.f, mx = 0.f;
    int k = 0;
    for (int32_t e = ob; e < oe && k < NEIGH_SAMPLE; ++e, ++k) s += degree_log(a.begin, __ldg(a.node_idx + e));
    f[6] = k ? s / (float)k : 0.f;
    k = 0;
    for (int32_t e = ib; e < ie && k < NEIGH_SAMPLE; ++e, ++k) mx = fmaxf(mx, degree_log(a.r_begin, __ldg(a.r_node_idx + e)));
    f[7] = mx;
#pragma unroll
    for (int j = 0; j < MLP_IN; ++j) f[j] = bf16r(f[j]);
}

__device__ __forceinline__ bool traversed(const RoundArgs& a, int32_t c) {
    return c != SCC_COLOR_DONE && (!a.use_only || c == a.only_color);
}

// Members per class of this round (slot_count, reset by the slot reset).
// Lanes of a warp that share a colour add once; a warp whose lanes all share
// one colour keeps a running count and adds it when the colour changes, so a
// round over one huge class costs one atomic per warp.
__global__ void k_class_sizes(RoundArgs a) {
    int lane = threadIdx.x & 31;
    int32_t run_c = SCC_COLOR_DONE, run_n = 0;
    int64_t limit = (((int64_t)a.live_count + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t c = SCC_COLOR_DONE;
        if (i < a.live_count) {
            c = a.color[a.live[i]];
            if (!traversed(a, c)) c = SCC_COLOR_DONE;
        }
        unsigned grp = __match_any_sync(0xFFFFFFFFu, c);
        if (c == SCC_COLOR_DONE) continue;
        if (grp == 0xFFFFFFFFu) {
            if (lane == 0) {
                if (c != run_c) {
                    if (run_n) atomicAdd(a.slot_count + run_c + 1, run_n);
                    run_c = c; run_n = 0;
                }
                run_n += 32;
            }
        } else if (lane == __ffs(grp) - 1) {
            atomicAdd(a.slot_count + c + 1, __popc(grp));
        }
    }
    if (lane == 0 && run_n) atomicAdd(a.slot_count + run_c + 1, run_n);
}

struct LogArgs {
    float* x; int32_t* v; int32_t* size; int32_t* ctr;
    int64_t cap;
    uint32_t thresh;     // keep a vertex when its salted hash (16 bits) is below this
    uint32_t salt;
};

__device__ __forceinline__ uint4 pack_row(const float* f) {
    __nv_bfloat162 p0 = __floats2bfloat162_rn(f[0], f[1]), p1 = __floats2bfloat162_rn(f[2], f[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(f[4], f[5]), p3 = __floats2bfloat162_rn(f[6], f[7]);
    uint4 r;
    r.x = *reinterpret_cast<uint32_t*>(&p0); r.y = *reinterpret_cast<uint32_t*>(&p1);
    r.z = *reinterpret_cast<uint32_t*>(&p2); r.w = *reinterpret_cast<uint32_t*>(&p3);
    return r;
}

// Training records: features of sampled vertices of the classes being pivoted.
__global__ void k_pivot_log(RoundArgs a, const unsigned long long* __restrict__ cnt,
                            LogArgs lg) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < a.live_count; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = a.live[i];
        int32_t c = a.color[v];
        if (!traversed(a, c) || (pivot_hash((uint32_t)v ^ lg.salt) & 0xFFFFu) >= lg.thresh) continue;
        float f[MLP_IN];
        vertex_features(a, cnt, v, c, f);
        int32_t k = atomicAdd(lg.ctr, 1);
        if (k < lg.cap) {
#pragma unroll
            for (int j = 0; j < MLP_IN; ++j) lg.x[(int64_t)k * MLP_IN + j] = f[j];
            lg.v[k] = v;
            lg.size[k] = a.slot_count[c + 1];
        }
    }
}

// Candidates of the learned choice: vertices whose in x out degree is within a
// factor CAND_DIV of the best of their class (slot_key holds the degree keys).
// The network re-ranks these; a class's degree pivot is always among them.
// CAND_DIV 1 keeps the vertices tied at the best: on C2 a window of 4x let the
// network pick grid vertices outside the grid's giant SCC, each miss one more
// 17-18 ms wave (learned/plain 0.50-0.82 over three trainings; 2x: 0.54-0.60;
// ties only: 0.86-0.99), while C3 measured the same with all three (0.91-0.93).
#define CAND_DIV 1ull
__global__ void k_pivot_candidates(RoundArgs a, int32_t* __restrict__ cand, int32_t* __restrict__ ncand) {
    int lane = threadIdx.x & 31;
    int64_t limit = (((int64_t)a.live_count + 31) / 32) * 32;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < limit; i += (int64_t)gridDim.x * blockDim.x) {
        bool take = false;
        if (i < a.live_count) {
            int32_t v = a.live[i];
            int32_t c = a.color[v];
            if (traversed(a, c)) {
                unsigned long long best = a.slot_key[c + 1] >> 32;            // max(in*out) + 1
                unsigned long long mine = pivot_key(a.begin, a.r_begin, v) >> 32;
                take = mine * CAND_DIV >= best;
            }
        }
        unsigned bal = __ballot_sync(0xFFFFFFFFu, take);
        int32_t base = 0;
        if (lane == 0 && bal) base = atomicAdd(ncand, __popc(bal));
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (take) cand[base + __popc(bal & ((1u << lane) - 1u))] = a.live[i];
    }
}

__global__ void k_cand_features(RoundArgs a, const unsigned long long* __restrict__ cnt,
                                const int32_t* __restrict__ cand, const int32_t* __restrict__ ncand,
                                uint4* __restrict__ rows) {
    const int32_t k = *ncand;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = cand[i];
        float f[MLP_IN];
        vertex_features(a, cnt, v, a.color[v], f);
        rows[i] = pack_row(f);
    }
}

// Learned key: the score in unsigned order (NaN lowest), ties by the id hash.
__device__ __forceinline__ unsigned long long learned_key(float sc, int32_t v) {
    uint32_t hi = 1u;
    if (sc == sc) {
        uint32_t u = __float_as_uint(sc);
        hi = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
        if (hi == 0u) hi = 1u;
    }
    return ((unsigned long long)hi << 32) | pivot_hash((uint32_t)v);
}

__global__ void k_cand_reset(RoundArgs a, const int32_t* __restrict__ cand, const int32_t* __restrict__ ncand) {
    const int32_t k = *ncand;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x)
        a.slot_key[a.color[cand[i]] + 1] = 0ull;
}

__global__ void k_cand_key(RoundArgs a, const int32_t* __restrict__ cand, const int32_t* __restrict__ ncand,
                           const float* __restrict__ score) {
    const int32_t k = *ncand;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = cand[i];
        int32_t c = a.color[v];
        unsigned long long key = learned_key(score[i], v);
        if (key > a.slot_key[c + 1]) atomicMax(a.slot_key + c + 1, key);
    }
}

__global__ void k_cand_pick(RoundArgs a, const int32_t* __restrict__ cand, const int32_t* __restrict__ ncand,
                            const float* __restrict__ score, int32_t* q) {
    const int32_t k = *ncand;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t v = cand[i];
        int32_t c = a.color[v];
        if (learned_key(score[i], v) == a.slot_key[c + 1]) seed_pivot(a, v, c, q);
    }
}

// ------------------------------------------------------------------ tcgen05 helpers
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor: K-major, no swizzle (8-row x 16-byte core
// matrices), lbo = byte distance between the two K halves of a 16-wide slice,
// sbo = byte distance between 8-row groups; descriptor version 1 (sm_100).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}
// Instruction descriptor, kind::f16: D FP32 (bit 4), A and B BF16 (bits 7, 10),
// both K-major, N = 64 (bits 17-22 hold N/8), M = 128 (bits 24-28 hold M/16).
#define MLP_IDESC ((1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) | ((128u >> 4) << 24))

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
                 :: "r"(tmem_d), "l"(da), "l"(db), "r"((uint32_t)MLP_IDESC), "r"(accumulate) : "memory");
}
__device__ __forceinline__ void umma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(mbar) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint32_t mbar, uint32_t parity) {
    uint32_t ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}\n" : "=r"(ok) : "r"(mbar), "r"(parity) : "memory");
    return ok != 0u;
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// 16 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* r) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Byte offset of element (row, k) in a K-major no-swizzle operand whose 8-row
// groups are sbo bytes apart (the two K halves of each 16-wide slice 128 B apart).
__host__ __device__ __forceinline__ uint32_t canon_off(int row, int k, uint32_t sbo) {
    return (uint32_t)((row & 7) * 16 + (row >> 3) * sbo + (k & 7) * 2 + (k >> 3) * 128);
}

// Shared-memory plan of the inference kernel (bytes).
#define TC_A1 0          // X tile   [128 x 16] BF16, sbo 256
#define TC_A2 4096       // H1 tile  [128 x 64] BF16, sbo 1024
#define TC_B1 20480      // W1^T     [64 x 16]  BF16, sbo 256
#define TC_B2 22528      // W2^T     [64 x 64]  BF16, sbo 1024
#define TC_F32 30720     // b1, b2, w3 (64 floats each), b3
#define TC_BAR 31504     // mbarrier (8 B) + TMEM base (4 B)
#define TC_SMEM 31616
#define TC_TMEM_COLS 128 // D1 in columns 0-63, D2 in 64-127

// count_ptr (device) gives the row count when not NULL, else count.
__global__ void __launch_bounds__(TC_ROWS) k_mlp_score_tc(const uint4* __restrict__ rows, int32_t count,
                                                          const int32_t* __restrict__ count_ptr,
                                                          const __nv_bfloat16* __restrict__ w16,
                                                          float* __restrict__ score, int32_t* __restrict__ err) {
    if (count_ptr) count = *count_ptr;
    extern __shared__ __align__(1024) uint8_t sm[];
    const int tid = threadIdx.x, warp = tid >> 5;
    __nv_bfloat16* b1s = reinterpret_cast<__nv_bfloat16*>(sm + TC_B1);
    __nv_bfloat16* b2s = reinterpret_cast<__nv_bfloat16*>(sm + TC_B2);
    float* fb1 = reinterpret_cast<float*>(sm + TC_F32);
    float* fb2 = fb1 + MLP_H;
    float* fw3 = fb2 + MLP_H;
    float* fb3 = fw3 + MLP_H;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + TC_BAR);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + TC_BAR + 8);
    const __nv_bfloat16 zero = __float2bfloat16_rn(0.f);
    // B operands: row j = output unit, column k = input (W^T, K-major)
    for (int e = tid; e < MLP_H * 16; e += TC_ROWS) {
        int j = e >> 4, k = e & 15;
        b1s[canon_off(j, k, 256) >> 1] = k < MLP_IN ? w16[OFF_W1 + k * MLP_H + j] : zero;
    }
    for (int e = tid; e < MLP_H * MLP_H; e += TC_ROWS) {
        int j = e >> 6, k = e & 63;
        b2s[canon_off(j, k, 1024) >> 1] = w16[OFF_W2 + k * MLP_H + j];
    }
    // the upper K half of the X tile stays zero
    *reinterpret_cast<uint4*>(sm + TC_A1 + canon_off(tid, 8, 256)) = make_uint4(0u, 0u, 0u, 0u);
    if (tid < MLP_H) {
        fb1[tid] = __bfloat162float(w16[OFF_B1 + tid]);
        fb2[tid] = __bfloat162float(w16[OFF_B2 + tid]);
        fw3[tid] = __bfloat162float(w16[OFF_W3 + tid]);
    }
    if (tid == 0) {
        fb3[0] = __bfloat162float(w16[OFF_B3]);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(smem_addr(bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     :: "r"(smem_addr(tslot)), "r"((uint32_t)TC_TMEM_COLS) : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;
    const uint32_t d1 = tmem, d2 = tmem + MLP_H;
    const uint32_t lane_base = (uint32_t)(warp * 32) << 16;
    const uint32_t bar_a = smem_addr(bar);
    const uint64_t da1 = umma_desc(smem_addr(sm + TC_A1), 128, 256);
    const uint64_t db1 = umma_desc(smem_addr(sm + TC_B1), 128, 256);
    uint32_t parity = 0;
    int failed = 0;
    const int32_t tiles = (count + TC_ROWS - 1) / TC_ROWS;
    for (int32_t tile = blockIdx.x; tile < tiles && !failed; tile += gridDim.x) {
        const int64_t row = (int64_t)tile * TC_ROWS + tid;
        uint4 xv = row < count ? rows[row] : make_uint4(0u, 0u, 0u, 0u);
        *reinterpret_cast<uint4*>(sm + TC_A1 + canon_off(tid, 0, 256)) = xv;
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
            umma_bf16(d1, da1, db1, 0u);                       // D1 = X W1
            umma_commit(bar_a);
        }
        int ok = 0;
        for (int it = 0; it < WAIT_LIMIT && !ok; ++it) ok = mbar_try_wait(bar_a, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) { failed = 1; break; }
        tc_fence_after();
        uint32_t r[MLP_H];
        tmem_ld16(d1 + lane_base + 0, r);
        tmem_ld16(d1 + lane_base + 16, r + 16);
        tmem_ld16(d1 + lane_base + 32, r + 32);
        tmem_ld16(d1 + lane_base + 48, r + 48);
        tmem_wait_ld();
#pragma unroll
        for (int c8 = 0; c8 < MLP_H / 8; ++c8) {               // H1 = relu(D1 + b1) -> BF16, row tid
            uint32_t pk[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                int j = c8 * 8 + q * 2;
                float h0 = fmaxf(__uint_as_float(r[j]) + fb1[j], 0.f);
                float h1 = fmaxf(__uint_as_float(r[j + 1]) + fb1[j + 1], 0.f);
                __nv_bfloat162 p = __floats2bfloat162_rn(h0, h1);
                pk[q] = *reinterpret_cast<uint32_t*>(&p);
            }
            *reinterpret_cast<uint4*>(sm + TC_A2 + canon_off(tid, c8 * 8, 1024)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        proxy_fence();
        tc_fence_before();
        __syncthreads();
        tc_fence_after();
        if (tid == 0) {
#pragma unroll
            for (int kk = 0; kk < MLP_H / 16; ++kk)            // D2 = H1 W2, K in four slices of 16
                umma_bf16(d2, umma_desc(smem_addr(sm + TC_A2 + kk * 256), 128, 1024),
                          umma_desc(smem_addr(sm + TC_B2 + kk * 256), 128, 1024), kk > 0 ? 1u : 0u);
            umma_commit(bar_a);
        }
        ok = 0;
        for (int it = 0; it < WAIT_LIMIT && !ok; ++it) ok = mbar_try_wait(bar_a, parity);
        parity ^= 1u;
        if (__syncthreads_or(!ok)) { failed = 1; break; }
        tc_fence_after();
        tmem_ld16(d2 + lane_base + 0, r);
        tmem_ld16(d2 + lane_base + 16, r + 16);
        tmem_ld16(d2 + lane_base + 32, r + 32);
        tmem_ld16(d2 + lane_base + 48, r + 48);
        tmem_wait_ld();
        float y = fb3[0];
#pragma unroll
        for (int j = 0; j < MLP_H; ++j) y = fmaf(fmaxf(__uint_as_float(r[j]) + fb2[j], 0.f), fw3[j], y);
        if (row < count) score[row] = y;
    }
    if (failed && tid == 0) atomicExch(err, SCC_DEVERR_WAIT_LIMIT);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"((uint32_t)TC_TMEM_COLS)
                     : "memory");
}

// ------------------------------------------------------------------ CUDA-core forward (FP32 activations)
__global__ void __launch_bounds__(128) k_mlp_forward_rows(const float* __restrict__ x, int64_t count,
                                                          const __nv_bfloat16* __restrict__ w16, float* __restrict__ y) {
    __shared__ float sw[MLP_PARAMS];
    for (int i = threadIdx.x; i < MLP_PARAMS; i += blockDim.x) sw[i] = __bfloat162float(w16[i]);
    __syncthreads();
    // one row per thread: a grid-stride loop would let the compiler hoist every
    // shared-memory weight into registers across iterations
    const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (i < count) {
        float f[MLP_IN], h1[MLP_H];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) f[k] = x[i * MLP_IN + k];
#pragma unroll
        for (int j = 0; j < MLP_H; ++j) {
            float acc = sw[OFF_B1 + j];
#pragma unroll
            for (int k = 0; k < MLP_IN; ++k) acc = fmaf(f[k], sw[OFF_W1 + k * MLP_H + j], acc);
            h1[j] = fmaxf(acc, 0.f);
        }
        float out = sw[OFF_B3];
#pragma unroll 1
        for (int j = 0; j < MLP_H; ++j) {
            float acc = sw[OFF_B2 + j];
#pragma unroll
            for (int k = 0; k < MLP_H; ++k) acc = fmaf(h1[k], sw[OFF_W2 + k * MLP_H + j], acc);
            out = fmaf(fmaxf(acc, 0.f), sw[OFF_W3 + j], out);
        }
        y[i] = out;
    }
}

__global__ void k_rows_bf16(const float* __restrict__ x, int64_t count, uint4* __restrict__ rows) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        const float* f = x + i * MLP_IN;
        __nv_bfloat162 p0 = __floats2bfloat162_rn(f[0], f[1]), p1 = __floats2bfloat162_rn(f[2], f[3]);
        __nv_bfloat162 p2 = __floats2bfloat162_rn(f[4], f[5]), p3 = __floats2bfloat162_rn(f[6], f[7]);
        uint4 r;
        r.x = *reinterpret_cast<uint32_t*>(&p0); r.y = *reinterpret_cast<uint32_t*>(&p1);
        r.z = *reinterpret_cast<uint32_t*>(&p2); r.w = *reinterpret_cast<uint32_t*>(&p3);
        rows[i] = r;
    }
}

// ------------------------------------------------------------------ training (fused forward + backward)
// Shared plan (floats): weights (MLP_PARAMS, padded to 4804), then per-sample
// columns with stride TRAIN_S: X [8], H1 [64], H2 [64], dZ2 [64], dZ1 [64], dy.
#define TRAIN_W_PAD 4804
#define TRAIN_SMEM_FLOATS (TRAIN_W_PAD + (MLP_IN + 4 * MLP_H) * TRAIN_S + TRAIN_B)

__global__ void __launch_bounds__(TRAIN_B) k_mlp_train(const float* __restrict__ x, const float* __restrict__ t,
                                                       const int32_t* __restrict__ perm, int64_t first, int32_t nb,
                                                       const __nv_bfloat16* __restrict__ w16, float* __restrict__ grad,
                                                       float* __restrict__ loss_sum, float inv_n) {
    extern __shared__ float tsm[];
    float* sw = tsm;
    float* sx = sw + TRAIN_W_PAD;
    float* sh1 = sx + MLP_IN * TRAIN_S;
    float* sh2 = sh1 + MLP_H * TRAIN_S;
    float* sd2 = sh2 + MLP_H * TRAIN_S;
    float* sd1 = sd2 + MLP_H * TRAIN_S;
    float* sdy = sd1 + MLP_H * TRAIN_S;
    const int s = threadIdx.x;
    for (int i = s; i < MLP_PARAMS; i += TRAIN_B) sw[i] = __bfloat162float(w16[i]);
    const int32_t local = blockIdx.x * TRAIN_B + s;
    const bool valid = local < nb;
    int64_t idx = 0;
    if (valid) idx = perm ? (int64_t)perm[first + local] : first + local;
    float xi[MLP_IN];
#pragma unroll
    for (int k = 0; k < MLP_IN; ++k) {
        xi[k] = valid ? x[idx * MLP_IN + k] : 0.f;
        sx[k * TRAIN_S + s] = xi[k];
    }
    __syncthreads();
    // forward
    float h1[MLP_H];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        float acc = sw[OFF_B1 + j];
#pragma unroll
        for (int k = 0; k < MLP_IN; ++k) acc = fmaf(xi[k], sw[OFF_W1 + k * MLP_H + j], acc);
        h1[j] = fmaxf(acc, 0.f);
        sh1[j * TRAIN_S + s] = h1[j];
    }
    float y = sw[OFF_B3];
    for (int j = 0; j < MLP_H; ++j) {
        float acc = sw[OFF_B2 + j];
#pragma unroll
        for (int k = 0; k < MLP_H; ++k) acc = fmaf(h1[k], sw[OFF_W2 + k * MLP_H + j], acc);
        float h2 = fmaxf(acc, 0.f);
        sh2[j * TRAIN_S + s] = h2;
        y = fmaf(h2, sw[OFF_W3 + j], y);
    }
    // backward of the mean squared error
    const float diff = valid ? (y - t[idx]) : 0.f;
    const float dy = 2.f * diff * inv_n;
    sdy[s] = dy;
    float sq = diff * diff;
    for (int o = 16; o > 0; o >>= 1) sq += __shfl_down_sync(0xFFFFFFFFu, sq, o);
    if ((s & 31) == 0 && sq != 0.f) atomicAdd(loss_sum, sq);
    float dz2[MLP_H];
#pragma unroll
    for (int j = 0; j < MLP_H; ++j) {
        dz2[j] = sh2[j * TRAIN_S + s] > 0.f ? dy * sw[OFF_W3 + j] : 0.f;
        sd2[j * TRAIN_S + s] = dz2[j];
    }
    for (int k = 0; k < MLP_H; ++k) {
        float acc = 0.f;
#pragma unroll
        for (int j = 0; j < MLP_H; ++j) acc = fmaf(dz2[j], sw[OFF_W2 + k * MLP_H + j], acc);
        sd1[k * TRAIN_S + s] = sh1[k * TRAIN_S + s] > 0.f ? acc : 0.f;
    }
    __syncthreads();
    // dW2[k][j] = sum_s H1[s][k] dZ2[s][j]: a 4 x 8 register tile per thread
    {
        const int kb = (s >> 3) * 4, jb = (s & 7) * 8;
        float acc[4][8];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) acc[a][b] = 0.f;
        for (int q = 0; q < TRAIN_B; ++q) {
            float av[4], bv[8];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = sh1[(kb + a) * TRAIN_S + q];
#pragma unroll
            for (int b = 0; b < 8; ++b) bv[b] = sd2[(jb + b) * TRAIN_S + q];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 8; ++b) acc[a][b] = fmaf(av[a], bv[b], acc[a][b]);
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 8; ++b) atomicAdd(grad + OFF_W2 + (kb + a) * MLP_H + jb + b, acc[a][b]);
    }
    // dW1[k][j] = sum_s X[s][k] dZ1[s][j]: 4 outputs per thread
    {
        const int k = s >> 4, jb = (s & 15) * 4;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int q = 0; q < TRAIN_B; ++q) {
            float xv = sx[k * TRAIN_S + q];
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[b] = fmaf(xv, sd1[(jb + b) * TRAIN_S + q], acc[b]);
        }
#pragma unroll
        for (int b = 0; b < 4; ++b) atomicAdd(grad + OFF_W1 + k * MLP_H + jb + b, acc[b]);
    }
    // biases and the last layer
    if (s < MLP_H) {
        float a1 = 0.f, a2 = 0.f;
        for (int q = 0; q < TRAIN_B; ++q) { a1 += sd1[s * TRAIN_S + q]; a2 += sd2[s * TRAIN_S + q]; }
        atomicAdd(grad + OFF_B1 + s, a1);
        atomicAdd(grad + OFF_B2 + s, a2);
    } else {
        const int j = s - MLP_H;
        float a3 = 0.f;
        for (int q = 0; q < TRAIN_B; ++q) a3 = fmaf(sh2[j * TRAIN_S + q], sdy[q], a3);
        atomicAdd(grad + OFF_W3 + j, a3);
        if (j == 0) {
            float b3 = 0.f;
            for (int q = 0; q < TRAIN_B; ++q) b3 += sdy[q];
            atomicAdd(grad + OFF_B3, b3);
        }
    }
}

// Adam step on the master copy; clears the gradient and refreshes the BF16 copy.
__global__ void k_adam(float* __restrict__ p, float* __restrict__ g, float* __restrict__ m1, float* __restrict__ m2,
                       __nv_bfloat16* __restrict__ w16, float lr, float c1, float c2) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= MLP_PARAMS) return;
    float gi = g[i];
    g[i] = 0.f;
    float a = 0.9f * m1[i] + 0.1f * gi;
    float b = 0.999f * m2[i] + 0.001f * gi * gi;
    m1[i] = a;
    m2[i] = b;
    float v = p[i] - lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
    p[i] = v;
    w16[i] = __float2bfloat16_rn(v);
}

__global__ void k_refresh_bf16(const float* __restrict__ p, __nv_bfloat16* __restrict__ w16) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < MLP_PARAMS) w16[i] = __float2bfloat16_rn(p[i]);
}

// ------------------------------------------------------------------ training targets
__global__ void k_scc_sizes(int32_t n, const int32_t* __restrict__ scc, int32_t* __restrict__ hist) {
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int32_t r = scc[v];
        if (r >= 0 && r < n) atomicAdd(hist + r, 1);
    }
}

__global__ void k_targets(int64_t count, const int32_t* __restrict__ lv, const int32_t* __restrict__ lsize,
                          const int32_t* __restrict__ scc, const int32_t* __restrict__ hist, int32_t n,
                          float* __restrict__ t, int32_t* __restrict__ bad) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        int32_t r = scc[lv[i]];
        if (r < 0 || r >= n) { atomicExch(bad, 1); t[i] = 0.f; continue; }
        t[i] = log1pf((float)hist[r]) / log1pf((float)max(lsize[i], 1));
    }
}

// ------------------------------------------------------------------ host: round preparation
static int ensure_pivot_buffers(scc_state* s) {
    size_t n = (size_t)std::max<int32_t>(s->n, 1);
    if (!s->pivot_score) SCC_CUDA(cudaMalloc(&s->pivot_score, sizeof(float) * n));
    if (!s->pivot_x) SCC_CUDA(cudaMalloc(&s->pivot_x, 16 * n));
    if (!s->pivot_cand) SCC_CUDA(cudaMalloc(&s->pivot_cand, sizeof(int32_t) * n));
    return SCC_OK;
}

static unsigned tc_blocks(int64_t count) {
    int64_t tiles = (count + TC_ROWS - 1) / TC_ROWS;
    return (unsigned)std::max<int64_t>(1, std::min<int64_t>(tiles, 148LL * 4));
}

int scc_impl_pivot_prepare(const scc_graph* g, scc_state* s, RoundArgs& a, bool learned, int32_t* q, bool* seeded) {
    (void)g;
    *seeded = false;
    const bool logging = s->log_cap > 0;
    if ((!learned && !logging) || a.live_count <= 0) return SCC_OK;
    unsigned blocks = scc_blocks(a.live_count);
    if (logging) {
        k_class_sizes<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
        SCC_LAUNCHED(s);
    }
    const unsigned long long* cr = s->cnt_valid ? s->cnt : nullptr;
    if (logging) {
        LogArgs lg;
        lg.x = s->log_x; lg.v = s->log_v; lg.size = s->log_size; lg.ctr = s->log_ctr; lg.cap = s->log_cap;
        double p = (double)s->log_per_round / (double)a.live_count;
        lg.thresh = p >= 1.0 ? 0x10000u : (uint32_t)std::max(1.0, p * 65536.0);
        lg.salt = 0x9E3779B9u * (++s->log_salt);
        k_pivot_log<<<blocks, SCC_THREADS, 0, s->stream>>>(a, cr, lg);
        SCC_LAUNCHED(s);
    }
    if (!learned) return SCC_OK;
    scc_pivot_model* m = s->pivot_model;
    SCC_REQUIRE(m->device == s->device, SCC_ERR_INVALID, "pivot model on device %d, state on %d", m->device, s->device);
    SCC_TRY(ensure_pivot_buffers(s));
    int32_t* ncand = s->ctr + CTR_SPARE1;
    SCC_TRY(scc_zero_counters(s, CTR_SPARE1, 1));
    k_pivot_candidates<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->pivot_cand, ncand);
    SCC_LAUNCHED(s);
    // every listed class's degree pivot is one of its candidates, so no more
    // candidates than classes (CTR_SPARE4, counted by k_pivot_key) means no
    // class has a choice: the degree pivots are the learned ones, unscored
    SCC_TRY(scc_sync_counters(s));
    if (s->h_ctr[CTR_SPARE1] <= s->h_ctr[CTR_SPARE4]) return SCC_OK;
    if (!logging) {
        k_class_sizes<<<blocks, SCC_THREADS, 0, s->stream>>>(a);
        SCC_LAUNCHED(s);
    }
    k_cand_features<<<blocks, SCC_THREADS, 0, s->stream>>>(a, cr, s->pivot_cand, ncand, (uint4*)s->pivot_x);
    SCC_LAUNCHED(s);
    k_mlp_score_tc<<<tc_blocks(a.live_count), TC_ROWS, TC_SMEM, s->stream>>>(
        (const uint4*)s->pivot_x, a.live_count, ncand, m->w16, s->pivot_score, s->ctr + CTR_ERROR);
    SCC_LAUNCHED(s);
    k_cand_reset<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->pivot_cand, ncand);
    SCC_LAUNCHED(s);
    k_cand_key<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->pivot_cand, ncand, s->pivot_score);
    SCC_LAUNCHED(s);
    k_cand_pick<<<blocks, SCC_THREADS, 0, s->stream>>>(a, s->pivot_cand, ncand, s->pivot_score, q);
    SCC_LAUNCHED(s);
    *seeded = true;
    return SCC_OK;
}

void scc_impl_pivot_release(scc_state* s) {
    cudaFree(s->pivot_score); cudaFree(s->pivot_x); cudaFree(s->pivot_cand);
    cudaFree(s->log_x); cudaFree(s->log_v); cudaFree(s->log_size); cudaFree(s->log_ctr);
    s->pivot_score = nullptr; s->pivot_x = nullptr; s->pivot_cand = nullptr;
    s->log_x = nullptr; s->log_v = nullptr; s->log_size = nullptr; s->log_ctr = nullptr;
    s->log_cap = 0;
}

// ------------------------------------------------------------------ host: model
static inline uint64_t mix64(uint64_t& st) {
    uint64_t z = (st += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline double unit(uint64_t& st) { return (double)(mix64(st) >> 11) * (1.0 / 9007199254740992.0); }

static void free_model(scc_pivot_model* m) {
    if (!m) return;
    cudaSetDevice(m->device);
    cudaFree(m->master); cudaFree(m->w16); cudaFree(m->grad); cudaFree(m->m1); cudaFree(m->m2); cudaFree(m->loss);
    cudaFree(m->err);
    delete m;
}

static int upload_params(scc_pivot_model* m, const float* host) {
    SCC_CUDA(cudaMemcpy(m->master, host, sizeof(float) * MLP_PARAMS, cudaMemcpyHostToDevice));
    k_refresh_bf16<<<(MLP_PARAMS + 255) / 256, 256>>>(m->master, m->w16);
    SCC_CUDA(cudaGetLastError());
    SCC_CUDA(cudaMemset(m->m1, 0, sizeof(float) * MLP_PARAMS));
    SCC_CUDA(cudaMemset(m->m2, 0, sizeof(float) * MLP_PARAMS));
    SCC_CUDA(cudaDeviceSynchronize());
    m->steps = 0;
    return SCC_OK;
}

static int alloc_model(int device, scc_pivot_model** out) {
    SCC_REQUIRE(out, SCC_ERR_INVALID, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    SCC_CUDA(cudaGetDeviceCount(&ndev));
    SCC_REQUIRE(device >= 0 && device < ndev, SCC_ERR_INVALID, "device %d of %d", device, ndev);
    SCC_CUDA(cudaSetDevice(device));
    scc_pivot_model* m = new scc_pivot_model();
    m->device = device;
    cudaError_t e = cudaMalloc(&m->master, sizeof(float) * MLP_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->w16, sizeof(__nv_bfloat16) * MLP_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->grad, sizeof(float) * MLP_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->m1, sizeof(float) * MLP_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->m2, sizeof(float) * MLP_PARAMS);
    if (e == cudaSuccess) e = cudaMalloc(&m->loss, sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&m->err, sizeof(int32_t));
    if (e == cudaSuccess) e = cudaMemset(m->grad, 0, sizeof(float) * MLP_PARAMS);
    if (e == cudaSuccess) e = cudaMemset(m->err, 0, sizeof(int32_t));
    if (e != cudaSuccess) {
        free_model(m);
        return scc_cuda_status(e, "pivot model allocation", __FILE__, __LINE__);
    }
    *out = m;
    return SCC_OK;
}

extern "C" int scc_pivot_model_create(int device, uint64_t seed, scc_pivot_model** out) {
    SCC_TRY(alloc_model(device, out));
    std::vector<float> p(MLP_PARAMS, 0.f);
    uint64_t st = seed ^ 0x5CC0B200ull;
    const double a1 = sqrt(6.0 / MLP_IN), a2 = sqrt(6.0 / MLP_H);
    for (int i = 0; i < MLP_IN * MLP_H; ++i) p[OFF_W1 + i] = (float)((2.0 * unit(st) - 1.0) * a1);
    for (int i = 0; i < MLP_H * MLP_H; ++i) p[OFF_W2 + i] = (float)((2.0 * unit(st) - 1.0) * a2);
    for (int i = 0; i < MLP_H; ++i) p[OFF_W3 + i] = (float)((2.0 * unit(st) - 1.0) * a2 * 0.5);
    for (int i = 0; i < MLP_H; ++i) { p[OFF_B1 + i] = 0.01f; p[OFF_B2 + i] = 0.01f; }
    int rc = upload_params(*out, p.data());
    if (rc != SCC_OK) { free_model(*out); *out = nullptr; }
    return rc;
}

extern "C" int scc_pivot_model_free(scc_pivot_model* m) {
    free_model(m);
    return SCC_OK;
}

extern "C" int scc_pivot_model_get_params(const scc_pivot_model* m, float* params) {
    SCC_REQUIRE(m && params, SCC_ERR_INVALID, "NULL argument");
    SCC_CUDA(cudaSetDevice(m->device));
    SCC_CUDA(cudaMemcpy(params, m->master, sizeof(float) * MLP_PARAMS, cudaMemcpyDeviceToHost));
    return SCC_OK;
}

extern "C" int scc_pivot_model_set_params(scc_pivot_model* m, const float* params) {
    SCC_REQUIRE(m && params, SCC_ERR_INVALID, "NULL argument");
    for (int i = 0; i < MLP_PARAMS; ++i)
        SCC_REQUIRE(std::isfinite(params[i]), SCC_ERR_INVALID, "parameter %d is not finite", i);
    SCC_CUDA(cudaSetDevice(m->device));
    return upload_params(m, params);
}

static const char kMagic[8] = {'S', 'C', 'C', 'P', 'I', 'V', 'T', '1'};

extern "C" int scc_pivot_model_save(const scc_pivot_model* m, const char* path) {
    SCC_REQUIRE(m && path, SCC_ERR_INVALID, "NULL argument");
    std::vector<float> p(MLP_PARAMS);
    SCC_TRY(scc_pivot_model_get_params(m, p.data()));
    FILE* f = fopen(path, "wb");
    SCC_REQUIRE(f, SCC_ERR_IO, "cannot write %s", path);
    int32_t cnt = MLP_PARAMS;
    bool ok = fwrite(kMagic, 1, 8, f) == 8 && fwrite(&cnt, 4, 1, f) == 1 &&
              fwrite(p.data(), sizeof(float), MLP_PARAMS, f) == (size_t)MLP_PARAMS;
    ok = (fclose(f) == 0) && ok;
    SCC_REQUIRE(ok, SCC_ERR_IO, "short write to %s", path);
    return SCC_OK;
}

extern "C" int scc_pivot_model_load(int device, const char* path, scc_pivot_model** out) {
    SCC_REQUIRE(path && out, SCC_ERR_INVALID, "NULL argument");
    FILE* f = fopen(path, "rb");
    SCC_REQUIRE(f, SCC_ERR_IO, "cannot open %s", path);
    char magic[8];
    int32_t cnt = 0;
    std::vector<float> p(MLP_PARAMS);
    bool ok = fread(magic, 1, 8, f) == 8 && memcmp(magic, kMagic, 8) == 0 && fread(&cnt, 4, 1, f) == 1 &&
              cnt == MLP_PARAMS && fread(p.data(), sizeof(float), MLP_PARAMS, f) == (size_t)MLP_PARAMS;
    fclose(f);
    SCC_REQUIRE(ok, SCC_ERR_IO, "%s is not a pivot model file", path);
    SCC_TRY(alloc_model(device, out));
    int rc = scc_pivot_model_set_params(*out, p.data());
    if (rc != SCC_OK) { free_model(*out); *out = nullptr; }
    return rc;
}

// RAII device buffer for the host entry points below.
template <class T>
struct DevArr {
    T* p = nullptr;
    ~DevArr() { if (p) cudaFree(p); }
    int alloc(size_t n) {
        SCC_CUDA(cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)));
        return SCC_OK;
    }
};

extern "C" int scc_pivot_model_forward(const scc_pivot_model* m, const float* x, int64_t count, int tensor_cores,
                                       float* y) {
    SCC_REQUIRE(m && (count == 0 || (x && y)), SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(count >= 0 && count < (1LL << 31), SCC_ERR_INVALID, "count %lld", (long long)count);
    if (count == 0) return SCC_OK;
    SCC_CUDA(cudaSetDevice(m->device));
    DevArr<float> dx, dy;
    SCC_TRY(dx.alloc((size_t)count * MLP_IN));
    SCC_TRY(dy.alloc((size_t)count));
    SCC_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice));
    if (tensor_cores) {
        DevArr<uint4> rows;
        SCC_TRY(rows.alloc((size_t)count));
        k_rows_bf16<<<scc_blocks(count), SCC_THREADS>>>(dx.p, count, rows.p);
        SCC_CUDA(cudaGetLastError());
        SCC_CUDA(cudaMemset(m->err, 0, sizeof(int32_t)));
        k_mlp_score_tc<<<tc_blocks(count), TC_ROWS, TC_SMEM>>>(rows.p, (int32_t)count, nullptr, m->w16, dy.p, m->err);
        SCC_CUDA(cudaGetLastError());
        SCC_CUDA(cudaDeviceSynchronize());
        int32_t err = 0;
        SCC_CUDA(cudaMemcpy(&err, m->err, sizeof(int32_t), cudaMemcpyDeviceToHost));
        SCC_REQUIRE(err == 0, SCC_ERR_TIMEOUT, "tensor-core inference: MMA completion wait ran out");
    } else {
        k_mlp_forward_rows<<<(unsigned)((count + 127) / 128), 128>>>(dx.p, count, m->w16, dy.p);
        SCC_CUDA(cudaGetLastError());
    }
    SCC_CUDA(cudaMemcpy(y, dy.p, sizeof(float) * (size_t)count, cudaMemcpyDeviceToHost));
    return SCC_OK;
}

extern "C" int scc_pivot_model_bench(const scc_pivot_model* m, int64_t count, int iters, double* ms_per_launch) {
    SCC_REQUIRE(m && ms_per_launch && iters > 0, SCC_ERR_INVALID, "NULL argument or iters %d", iters);
    SCC_REQUIRE(count > 0 && count < (1LL << 31), SCC_ERR_INVALID, "count %lld", (long long)count);
    SCC_CUDA(cudaSetDevice(m->device));
    DevArr<uint4> rows;
    DevArr<float> y;
    SCC_TRY(rows.alloc((size_t)count));
    SCC_TRY(y.alloc((size_t)count));
    // rows of small positive features (0x3F80 = 1.0 in BF16): any input gives the same work
    SCC_CUDA(cudaMemset(rows.p, 0x3F, sizeof(uint4) * (size_t)count));
    SCC_CUDA(cudaMemset(m->err, 0, sizeof(int32_t)));
    cudaEvent_t e0, e1;
    SCC_CUDA(cudaEventCreate(&e0));
    SCC_CUDA(cudaEventCreate(&e1));
    k_mlp_score_tc<<<tc_blocks(count), TC_ROWS, TC_SMEM>>>(rows.p, (int32_t)count, nullptr, m->w16, y.p, m->err);
    cudaEventRecord(e0);
    for (int i = 0; i < iters; ++i)
        k_mlp_score_tc<<<tc_blocks(count), TC_ROWS, TC_SMEM>>>(rows.p, (int32_t)count, nullptr, m->w16, y.p, m->err);
    cudaEventRecord(e1);
    cudaError_t e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    SCC_CUDA(e);
    int32_t err = 0;
    SCC_CUDA(cudaMemcpy(&err, m->err, sizeof(int32_t), cudaMemcpyDeviceToHost));
    SCC_REQUIRE(err == 0, SCC_ERR_TIMEOUT, "tensor-core inference: MMA completion wait ran out");
    *ms_per_launch = (double)ms / iters;
    return SCC_OK;
}

static int train_smem_attr(int device) {
    static int done[64] = {0};
    if (device >= 0 && device < 64 && done[device]) return SCC_OK;
    SCC_CUDA(cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)(sizeof(float) * TRAIN_SMEM_FLOATS)));
    if (device >= 0 && device < 64) done[device] = 1;
    return SCC_OK;
}

static int launch_train(const scc_pivot_model* m, const float* dx, const float* dt, const int32_t* perm, int64_t first,
                        int32_t nb) {
    unsigned blocks = (unsigned)((nb + TRAIN_B - 1) / TRAIN_B);
    k_mlp_train<<<blocks, TRAIN_B, sizeof(float) * TRAIN_SMEM_FLOATS>>>(dx, dt, perm, first, nb, m->w16, m->grad,
                                                                        m->loss, 1.f / (float)nb);
    SCC_CUDA(cudaGetLastError());
    return SCC_OK;
}

extern "C" int scc_pivot_model_loss_grad(const scc_pivot_model* m, const float* x, const float* t, int64_t count,
                                         float* grad, float* loss) {
    SCC_REQUIRE(m && x && t && grad, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(count > 0 && count < (1LL << 31), SCC_ERR_INVALID, "count %lld", (long long)count);
    SCC_CUDA(cudaSetDevice(m->device));
    SCC_TRY(train_smem_attr(m->device));
    DevArr<float> dx, dt;
    SCC_TRY(dx.alloc((size_t)count * MLP_IN));
    SCC_TRY(dt.alloc((size_t)count));
    SCC_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice));
    SCC_CUDA(cudaMemcpy(dt.p, t, sizeof(float) * (size_t)count, cudaMemcpyHostToDevice));
    SCC_CUDA(cudaMemset(m->grad, 0, sizeof(float) * MLP_PARAMS));
    SCC_CUDA(cudaMemset(m->loss, 0, sizeof(float)));
    SCC_TRY(launch_train(m, dx.p, dt.p, nullptr, 0, (int32_t)count));
    SCC_CUDA(cudaMemcpy(grad, m->grad, sizeof(float) * MLP_PARAMS, cudaMemcpyDeviceToHost));
    float l = 0.f;
    SCC_CUDA(cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
    SCC_CUDA(cudaMemset(m->grad, 0, sizeof(float) * MLP_PARAMS));
    if (loss) *loss = l / (float)count;
    return SCC_OK;
}

extern "C" int scc_pivot_model_train(scc_pivot_model* m, const float* x, const float* t, int64_t count, int epochs,
                                     int batch, float lr, uint64_t seed, float* epoch_loss) {
    SCC_REQUIRE(m && x && t, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(count > 0 && count < (1LL << 31), SCC_ERR_INVALID, "count %lld", (long long)count);
    SCC_REQUIRE(epochs >= 0 && batch > 0 && lr > 0.f && std::isfinite(lr), SCC_ERR_INVALID,
                "epochs %d batch %d lr %g", epochs, batch, (double)lr);
    for (int64_t i = 0; i < count; ++i) SCC_REQUIRE(std::isfinite(t[i]), SCC_ERR_INVALID, "target %lld", (long long)i);
    SCC_CUDA(cudaSetDevice(m->device));
    SCC_TRY(train_smem_attr(m->device));
    DevArr<float> dx, dt;
    DevArr<int32_t> dperm;
    SCC_TRY(dx.alloc((size_t)count * MLP_IN));
    SCC_TRY(dt.alloc((size_t)count));
    SCC_TRY(dperm.alloc((size_t)count));
    SCC_CUDA(cudaMemcpy(dx.p, x, sizeof(float) * MLP_IN * (size_t)count, cudaMemcpyHostToDevice));
    SCC_CUDA(cudaMemcpy(dt.p, t, sizeof(float) * (size_t)count, cudaMemcpyHostToDevice));
    std::vector<int32_t> perm((size_t)count);
    for (int64_t i = 0; i < count; ++i) perm[(size_t)i] = (int32_t)i;
    uint64_t st = seed ^ 0xA5A5F00Dull;
    for (int ep = 0; ep < epochs; ++ep) {
        for (int64_t i = count - 1; i > 0; --i) std::swap(perm[(size_t)i], perm[(size_t)(mix64(st) % (uint64_t)(i + 1))]);
        SCC_CUDA(cudaMemcpy(dperm.p, perm.data(), sizeof(int32_t) * (size_t)count, cudaMemcpyHostToDevice));
        SCC_CUDA(cudaMemset(m->loss, 0, sizeof(float)));
        for (int64_t b = 0; b < count; b += batch) {
            int32_t nb = (int32_t)std::min<int64_t>(batch, count - b);
            SCC_TRY(launch_train(m, dx.p, dt.p, dperm.p, b, nb));
            m->steps++;
            float c1 = 1.f - powf(0.9f, (float)m->steps), c2 = 1.f - powf(0.999f, (float)m->steps);
            k_adam<<<(MLP_PARAMS + 255) / 256, 256>>>(m->master, m->grad, m->m1, m->m2, m->w16, lr, c1, c2);
            SCC_CUDA(cudaGetLastError());
        }
        float l = 0.f;
        SCC_CUDA(cudaMemcpy(&l, m->loss, sizeof(float), cudaMemcpyDeviceToHost));
        if (epoch_loss) epoch_loss[ep] = l / (float)count;
    }
    SCC_CUDA(cudaDeviceSynchronize());
    return SCC_OK;
}

// ------------------------------------------------------------------ host: state hooks
extern "C" int scc_state_set_pivot_model(scc_state* s, scc_pivot_model* m) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    SCC_REQUIRE(!m || m->device == s->device, SCC_ERR_INVALID, "model on device %d, state on %d", m ? m->device : -1,
                s->device);
    s->pivot_model = m;
    return SCC_OK;
}

extern "C" int scc_state_pivot_log(scc_state* s, int64_t capacity, int32_t per_round) {
    SCC_REQUIRE(s, SCC_ERR_INVALID, "state is NULL");
    SCC_REQUIRE(capacity >= 0 && capacity < (1LL << 31) && (capacity == 0 || per_round > 0), SCC_ERR_INVALID,
                "capacity %lld per_round %d", (long long)capacity, per_round);
    SCC_CUDA(cudaSetDevice(s->device));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    cudaFree(s->log_x); cudaFree(s->log_v); cudaFree(s->log_size); cudaFree(s->log_ctr);
    s->log_x = nullptr; s->log_v = nullptr; s->log_size = nullptr; s->log_ctr = nullptr;
    s->log_cap = 0;
    if (capacity == 0) return SCC_OK;
    SCC_CUDA(cudaMalloc(&s->log_x, sizeof(float) * MLP_IN * (size_t)capacity));
    SCC_CUDA(cudaMalloc(&s->log_v, sizeof(int32_t) * (size_t)capacity));
    SCC_CUDA(cudaMalloc(&s->log_size, sizeof(int32_t) * (size_t)capacity));
    SCC_CUDA(cudaMalloc(&s->log_ctr, sizeof(int32_t)));
    SCC_CUDA(cudaMemset(s->log_ctr, 0, sizeof(int32_t)));
    s->log_cap = capacity;
    s->log_per_round = per_round;
    return SCC_OK;
}

extern "C" int scc_state_pivot_records(scc_state* s, float* x, float* t, int32_t* v, int32_t* class_size, int64_t cap,
                                       int64_t* count) {
    SCC_REQUIRE(s && count, SCC_ERR_INVALID, "NULL argument");
    SCC_REQUIRE(s->log_cap > 0, SCC_ERR_STATE, "pivot logging is off (scc_state_pivot_log)");
    SCC_CUDA(cudaSetDevice(s->device));
    int32_t c = 0;
    SCC_CUDA(cudaMemcpyAsync(&c, s->log_ctr, sizeof(int32_t), cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    int64_t have = std::min<int64_t>(c, s->log_cap);
    *count = have;
    if (cap <= 0 || have == 0) return SCC_OK;
    int64_t k = std::min<int64_t>(have, cap);
    *count = k;
    if (t) {
        DevArr<float> dt;
        SCC_TRY(dt.alloc((size_t)k));
        SCC_CUDA(cudaMemsetAsync(s->aux, 0, sizeof(int32_t) * (size_t)s->n, s->stream));
        k_scc_sizes<<<scc_blocks(s->n), SCC_THREADS, 0, s->stream>>>(s->n, s->scc, s->aux);
        SCC_LAUNCHED(s);
        SCC_TRY(scc_zero_counters(s, CTR_SPARE3, 1));
        k_targets<<<scc_blocks(k), SCC_THREADS, 0, s->stream>>>(k, s->log_v, s->log_size, s->scc, s->aux, s->n, dt.p,
                                                                s->ctr + CTR_SPARE3);
        SCC_LAUNCHED(s);
        SCC_CUDA(cudaMemcpyAsync(t, dt.p, sizeof(float) * (size_t)k, cudaMemcpyDeviceToHost, s->stream));
        SCC_TRY(scc_sync_counters(s));
        SCC_REQUIRE(s->h_ctr[CTR_SPARE3] == 0, SCC_ERR_STATE, "records need a finished run (unlabelled vertices)");
    }
    if (x) SCC_CUDA(cudaMemcpyAsync(x, s->log_x, sizeof(float) * MLP_IN * (size_t)k, cudaMemcpyDeviceToHost, s->stream));
    if (v) SCC_CUDA(cudaMemcpyAsync(v, s->log_v, sizeof(int32_t) * (size_t)k, cudaMemcpyDeviceToHost, s->stream));
    if (class_size)
        SCC_CUDA(cudaMemcpyAsync(class_size, s->log_size, sizeof(int32_t) * (size_t)k, cudaMemcpyDeviceToHost, s->stream));
    SCC_CUDA(cudaStreamSynchronize(s->stream));
    return SCC_OK;
}
