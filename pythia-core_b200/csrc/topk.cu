// Top-k (the reference's `sortlimit` operator, operators/sortlimit.cpp):
// the first `limit` tuples of a stable sort by the key columns, ascending
// or descending, ties in input order.
//
// Radix select instead of a full sort, since limit is usually far below n:
//   1. histogram of the top 12 bits of every tuple's order key (a 64-bit
//      unsigned word whose order is the requested order);
//   2. the host finds the bin b* holding the limit-th tuple;
//   3. every tuple below b* (all of them are in the answer) and every tuple
//      in b* (candidates) is appended as an (order key, row) pair;
//   4. those pairs are sorted by (order key, row) with the stable LSD radix
//      sort (row first, then key), and the first `limit` rows gathered.
// Two reads of the relation plus work on about limit + n / 4096 pairs.
#include <string.h>

#include <algorithm>
#include <vector>

#include "primitives.cuh"

namespace pyg {

constexpr int TK_BITS = 12;
constexpr int TK_BINS = 1 << TK_BITS;
constexpr int TK_THREADS = 256;

// Order key: signed order of the (packed) key, complemented for descending.
__device__ __forceinline__ uint64_t tk_order(const uint8_t* t, const KeySpec& ks, bool asc)
{
    const uint64_t s = packed_to_sortable(load_key(t, ks), ks.nkeys);
    return asc ? s : ~s;
}

__global__ void __launch_bounds__(TK_THREADS) tk_hist_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb,
                                                             KeySpec ks, int asc, unsigned long long* __restrict__ hist)
{
    __shared__ unsigned h[TK_BINS];
    for (int b = threadIdx.x; b < TK_BINS; b += TK_THREADS) h[b] = 0;
    __syncthreads();
    for (int64_t i = blockIdx.x * (int64_t)TK_THREADS + threadIdx.x; i < n; i += (int64_t)gridDim.x * TK_THREADS)
        atomicAdd(&h[tk_order(base + i * tb, ks, asc) >> (64 - TK_BITS)], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < TK_BINS; b += TK_THREADS)
        if (h[b]) atomicAdd(&hist[b], (unsigned long long)h[b]);
}

// Appends (order key, row) of every tuple whose top bits are <= bstar.
__global__ void __launch_bounds__(TK_THREADS) tk_select_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb,
                                                               KeySpec ks, int asc, unsigned bstar,
                                                               uint64_t* __restrict__ okey, uint64_t* __restrict__ row,
                                                               unsigned long long* __restrict__ cursor)
{
    const unsigned lane = threadIdx.x & 31;
    // Whole warps step together so that one atomic reserves the warp's slots.
    for (int64_t w0 = (blockIdx.x * (int64_t)TK_THREADS + threadIdx.x) & ~31LL; w0 < n;
         w0 += (int64_t)gridDim.x * TK_THREADS) {
        const int64_t i = w0 + lane;
        uint64_t k = 0;
        bool take = false;
        if (i < n) {
            k = tk_order(base + i * tb, ks, asc);
            take = (unsigned)(k >> (64 - TK_BITS)) <= bstar;
        }
        const unsigned m = __ballot_sync(0xffffffffu, take);
        if (!m) continue;
        unsigned long long at = 0;
        if (lane == 0) at = atomicAdd(cursor, (unsigned long long)__popc(m));
        at = __shfl_sync(0xffffffffu, at, 0);
        if (take) {
            const unsigned long long p = at + __popc(m & ((1u << lane) - 1u));
            okey[p] = k;
            row[p] = (uint64_t)i;
        }
    }
}

// Every tuple's (order key, row), for limit >= n.
__global__ void tk_all_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb, KeySpec ks, int asc,
                              uint64_t* __restrict__ okey, uint64_t* __restrict__ row)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        okey[i] = tk_order(base + i * tb, ks, asc);
        row[i] = (uint64_t)i;
    }
}

}  // namespace pyg

using namespace pyg;

extern "C" int pyg_sortlimit(pyg_ctx* ctx, const pyg_rel* in, const int32_t* key_cols, int32_t nkeys, int32_t asc,
                             int64_t limit, void* out, int64_t out_capacity, int64_t* out_n)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out_n || limit < 0 || (out_capacity > 0 && !out)) {
        set_error("pyg_sortlimit: bad arguments");
        return PYG_ERR_ARG;
    }
    if ((rc = check_rel(in, "sortlimit input"))) return rc;
    KeySpec ks;
    if ((rc = make_keyspec(in, key_cols, nkeys, &ks))) return rc;
    const int64_t n = in->ntuples;
    const int64_t k = limit < n ? limit : n;
    *out_n = k;
    if (k == 0) return PYG_OK;
    if (k > out_capacity) {
        set_error("pyg_sortlimit: %lld tuples exceed the output capacity %lld", (long long)k, (long long)out_capacity);
        return PYG_ERR_CAPACITY;
    }
    DevRel R;
    if ((rc = R.stage(ctx, in))) return rc;
    const uint8_t* base = (const uint8_t*)R.rel.base;
    const int32_t tb = in->tuple_bytes;
    uint64_t* pairs = nullptr;  // okey, row, okey_alt, row_alt
    unsigned long long* hist = nullptr;
    int64_t w = n;              // pairs selected
    do {
        if (k < n) {
            if ((rc = dalloc(ctx, (void**)&hist, (size_t)TK_BINS * 8))) break;
            PYG_CUDA(cudaMemsetAsync(hist, 0, (size_t)TK_BINS * 8, ctx->stream));
            tk_hist_kernel<<<grid_for(ctx, n, TK_THREADS, 8, 4), TK_THREADS, 0, ctx->stream>>>(base, n, tb, ks, asc,
                                                                                                 hist);
            PYG_LAUNCHED(ctx);
            std::vector<unsigned long long> h(TK_BINS);
            PYG_CUDA(cudaMemcpyAsync(h.data(), hist, (size_t)TK_BINS * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            unsigned bstar = 0;
            unsigned long long below = 0;
            while (below + h[bstar] < (unsigned long long)k) below += h[bstar++];
            w = (int64_t)(below + h[bstar]);
            if ((rc = dalloc(ctx, (void**)&pairs, (size_t)w * 32))) break;
            unsigned long long* cursor = ctx->dcounters + 120;
            PYG_CUDA(cudaMemsetAsync(cursor, 0, 8, ctx->stream));
            tk_select_kernel<<<grid_for(ctx, n, TK_THREADS, 8, 4), TK_THREADS, 0, ctx->stream>>>(
                base, n, tb, ks, asc, bstar, pairs, pairs + w, cursor);
            PYG_LAUNCHED(ctx);
        } else {
            if ((rc = dalloc(ctx, (void**)&pairs, (size_t)n * 32))) break;
            tk_all_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(base, n, tb, ks, asc, pairs,
                                                                                pairs + n);
            PYG_LAUNCHED(ctx);
        }
        // Sort by row, then (stably) by order key: (order key, row) order.
        uint64_t *key = pairs, *row = pairs + w, *key2 = pairs + 2 * w, *row2 = pairs + 3 * w;
        int rbits = 1;
        while (rbits < 64 && ((uint64_t)1 << rbits) < (uint64_t)n) ++rbits;
        int alt = 0;
        if ((rc = radix_sort_pairs(ctx, row, key, row2, key2, w, 0, rbits, &alt))) break;
        if (alt) {
            std::swap(row, row2);
            std::swap(key, key2);
        }
        int b0 = 0, b1 = 0;
        if ((rc = key_bit_range(ctx, key, w, &b0, &b1))) break;
        if ((rc = radix_sort_pairs(ctx, key, row, key2, row2, w, b0, b1, &alt))) break;
        if (alt) row = row2;
        rc = gather_rows(ctx, base, row, k, tb, (uint8_t*)out);
    } while (0);
    dfree(ctx, hist);
    dfree(ctx, pairs);
    R.release(ctx);
    if (!rc) PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    return rc;
}
