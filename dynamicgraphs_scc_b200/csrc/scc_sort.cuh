// Device sorting for CSR construction (scc_sort.cu): a stable LSD radix sort
// and the removal of repeated keys from a sorted array.  Scratch comes from the
// library's stream-ordered pool on `st`; results are ordered on `st`.
#pragma once
#include "scc_internal.cuh"

// Sorts m (key, value) pairs by the low `bits` bits of the key, stably;
// vals_in may be NULL (keys only).  Inputs are not modified.  scratch: NULL
// (taken from the pool) or at least scc_impl_sort_scratch_bytes(m, 4, vals)
// bytes, 256-byte aligned, that the caller allocated beforehand.
int scc_impl_sort_pairs_u32(const uint32_t* keys_in, uint32_t* keys_out, const int32_t* vals_in, int32_t* vals_out,
                            int64_t m, int bits, cudaStream_t st, void* scratch = nullptr);
size_t scc_impl_sort_scratch_bytes(int64_t m, size_t key_bytes, bool vals);
int scc_impl_sort_keys_u64(const unsigned long long* keys_in, unsigned long long* keys_out, int64_t m, int bits,
                           cudaStream_t st);
// out = a with repeated neighbours removed; *m_out its length (synchronises st).
int scc_impl_unique_u64(const unsigned long long* a, unsigned long long* out, int64_t m, int64_t* m_out,
                        cudaStream_t st);
// out[i] = sum of in[0, i) (inclusive: in[0, i]) in int32, n entries; out may
// equal in only for the exclusive form.  Scratch from the pool on `st`.
int scc_impl_scan_i32(const int32_t* in, int32_t* out, int64_t n, bool inclusive, cudaStream_t st);

// Exclusive prefix sum of one value per thread over a 256-thread block; *total
// = the block's sum.  s_w: 8 ints of shared memory.  Every thread must call it.
__device__ __forceinline__ int32_t scc_block_excl_sum256(int32_t x, int32_t* s_w, int32_t* total) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int32_t inc = x;
    for (int o = 1; o < 32; o <<= 1) {
        int32_t y = __shfl_up_sync(0xFFFFFFFFu, inc, o);
        if (lane >= o) inc += y;
    }
    if (lane == 31) s_w[wid] = inc;
    __syncthreads();
    if (wid == 0) {
        int32_t w = lane < 8 ? s_w[lane] : 0;
        for (int o = 1; o < 8; o <<= 1) {
            int32_t y = __shfl_up_sync(0xFFFFFFFFu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < 8) s_w[lane] = w;
    }
    __syncthreads();
    const int32_t r = (wid ? s_w[wid - 1] : 0) + inc - x;
    *total = s_w[7];
    __syncthreads();
    return r;
}

// starts[j] = index where the j-th run of equal keys of a sorted array begins;
// *count = the number of runs (synchronises st).
int scc_impl_segment_starts(const uint32_t* keys, int64_t m, int32_t* starts, int64_t* count, cudaStream_t st);
