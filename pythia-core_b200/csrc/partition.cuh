// Partitioning internals shared by the partition entry point, the MPSM join
// and the partitioned hash join.
#pragma once

#include "pyg_internal.cuh"

namespace pyg {

// Bucket function of one partition pass.
struct BucketFn {
    int32_t kind;         // PYG_SPLIT_*
    uint32_t fanout;
    int32_t log2f;        // RADIX / HASH
    int64_t mn, br;       // EXACTRANGE: min and bucket range
    const int64_t* spl;   // SPLITTERS: device array of fanout-1 values
};

__device__ __forceinline__ uint32_t bucket_of(const BucketFn& f, int64_t v, const int64_t* spl_smem)
{
    switch (f.kind) {
    case PYG_SPLIT_EXACTRANGE: {
        int64_t q = (v - f.mn) / f.br;
        return (q < 0 || q >= (int64_t)f.fanout) ? 0xFFFFFFFFu : (uint32_t)q;
    }
    case PYG_SPLIT_SPLITTERS: {
        const int64_t* s = spl_smem ? spl_smem : f.spl;
        uint32_t lo = 0, hi = f.fanout - 1;  // number of splitters <= v
        while (lo < hi) {
            uint32_t m = (lo + hi) >> 1;
            if (s[m] <= v) lo = m + 1;
            else hi = m;
        }
        return lo;
    }
    case PYG_SPLIT_RADIX:
        return (uint32_t)((uint64_t)v & (uint64_t)(f.fanout - 1));
    default:
        return f.log2f == 0 ? 0u : (uint32_t)(mix64((uint64_t)v) >> (64 - f.log2f));
    }
}

// Builds the device bucket function for a splitter spec.  For SPLITTERS the
// host splitters are copied to *spl_dev (caller frees with dfree).
int make_bucket_fn(pyg_ctx* ctx, const pyg_splitter* spl, BucketFn* f, int64_t** spl_dev);

// Partitions a device relation by key column into out (device), writing
// fanout+1 offsets to offsets_dev (device, unsigned long long).  Returns
// PYG_ERR_ARG (with a message) if a key falls outside an EXACTRANGE.
int partition_device(pyg_ctx* ctx, const pyg_rel* in, int32_t key_col, const BucketFn& f, void* out,
                     unsigned long long* offsets_dev);

}  // namespace pyg
