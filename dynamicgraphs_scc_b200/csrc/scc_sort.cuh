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
// starts[j] = index where the j-th run of equal keys of a sorted array begins;
// *count = the number of runs (synchronises st).
int scc_impl_segment_starts(const uint32_t* keys, int64_t m, int32_t* starts, int64_t* count, cudaStream_t st);
