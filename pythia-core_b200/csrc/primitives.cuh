// Device-wide primitives shared across libpyg sources (host-callable).
#pragma once

#include "pyg_internal.cuh"

namespace pyg {

// Exclusive prefix sum of n 64-bit counts (in and out may alias).
// Writes the total to *total_dev if not null.
int exclusive_scan_u64(pyg_ctx* ctx, const unsigned long long* in, unsigned long long* out, int64_t n,
                       unsigned long long* total_dev);

// Stable LSD radix sort of (key, value) pairs by unsigned key over bits
// [begin_bit, end_bit).  Sorted data ends in (keys, vals) or (keys_alt,
// vals_alt); *in_alt tells which.  vals may be null (keys only).
int radix_sort_pairs(pyg_ctx* ctx, uint64_t* keys, uint64_t* vals, uint64_t* keys_alt, uint64_t* vals_alt,
                     int64_t n, int begin_bit, int end_bit, int* in_alt);

// [begin, end) bit range over which the n keys differ (computed on device,
// read back with a stream sync).  begin == end when all keys are equal.
int key_bit_range(pyg_ctx* ctx, const uint64_t* keys, int64_t n, int* begin_bit, int* end_bit);

// Order-preserving map of a signed 64-bit value to an unsigned one.
__host__ __device__ __forceinline__ uint64_t to_sortable(int64_t v)
{
    return (uint64_t)v ^ 0x8000000000000000ULL;
}
__host__ __device__ __forceinline__ int64_t from_sortable(uint64_t u)
{
    return (int64_t)(u ^ 0x8000000000000000ULL);
}

// Sortable form of a packed key word (KeySpec): signed order of the single
// column, or lexicographic signed order of an (int32, int32) pair.
__host__ __device__ __forceinline__ uint64_t packed_to_sortable(uint64_t k, int nkeys)
{
    return nkeys == 2 ? (k ^ 0x8000000080000000ULL) : (k ^ 0x8000000000000000ULL);
}

// Distinct-key estimate for n tuples (device, tb bytes each) from the
// packed keys of a strided sample of CDF_ESTIMATE_SAMPLE tuples: the GEE
// estimate carried by the learned CDF model trained on that sample
// (cdf.cu).  Sizes hash tables when a caller gives no group estimate.
constexpr int64_t CDF_ESTIMATE_SAMPLE = (int64_t)1 << 18;
// Largest key sample the MPSM join draws for its learned splitters.
constexpr int64_t CDF_MPSM_SAMPLE = (int64_t)1 << 21;
int estimate_distinct_keys(pyg_ctx* ctx, const uint8_t* base, int64_t n, int32_t tb, const KeySpec& ks,
                           int64_t* out);

// Gather rows: out[i] = in[idx[i]] for tuples of tb bytes.
int gather_rows(pyg_ctx* ctx, const uint8_t* in, const uint64_t* idx, int64_t n, int32_t tb, uint8_t* out);

}  // namespace pyg
