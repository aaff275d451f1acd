// Scan, stable LSD radix sort, gather, and the sort / lower-bound entry
// points (reference SortOp and TupleBuffer::sort / findsmallest).
#include <string.h>

#include "primitives.cuh"

namespace pyg {

// ---------------------------------------------------------------------------
// Exclusive scan (three phases: block reduce, scan of block totals, scan).

constexpr int SCAN_THREADS = 1024;

__device__ __forceinline__ unsigned long long block_incl_scan(unsigned long long v, unsigned long long* warp_tot)
{
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        unsigned long long t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    if (lane == 31) warp_tot[w] = v;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        unsigned long long x = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long t = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += t;
        }
        if (lane < nw) warp_tot[lane] = x;
    }
    __syncthreads();
    unsigned long long r = v + (w > 0 ? warp_tot[w - 1] : 0);
    __syncthreads();
    return r;
}

__global__ void scan_reduce_kernel(const unsigned long long* __restrict__ in, int64_t n, int64_t chunk,
                                   unsigned long long* __restrict__ partial)
{
    __shared__ unsigned long long red[32];
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    unsigned long long s = 0;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) s += in[i];
    s = warp_sum_u64(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned long long x = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0;
        x = warp_sum_u64(x);
        if (threadIdx.x == 0) partial[blockIdx.x] = x;
    }
}

// Exclusive scan of `partial` (nb entries, one block), total to *total.
__global__ void scan_partials_kernel(unsigned long long* partial, int nb, unsigned long long* total)
{
    __shared__ unsigned long long warp_tot[32];
    unsigned long long carry = 0;
    for (int base = 0; base < nb; base += blockDim.x) {
        int i = base + threadIdx.x;
        unsigned long long v = i < nb ? partial[i] : 0;
        unsigned long long incl = block_incl_scan(v, warp_tot);
        if (i < nb) partial[i] = carry + incl - v;
        __shared__ unsigned long long last;
        if (threadIdx.x == blockDim.x - 1) last = incl;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

__global__ void scan_apply_kernel(const unsigned long long* in, unsigned long long* out, int64_t n, int64_t chunk,
                                  const unsigned long long* __restrict__ partial)
{
    __shared__ unsigned long long warp_tot[32];
    __shared__ unsigned long long last;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    unsigned long long carry = partial[blockIdx.x];
    for (int64_t base = lo; base < hi; base += blockDim.x) {
        int64_t i = base + threadIdx.x;
        unsigned long long v = i < hi ? in[i] : 0;
        unsigned long long incl = block_incl_scan(v, warp_tot);
        if (threadIdx.x == blockDim.x - 1) last = incl;
        if (i < hi) out[i] = carry + incl - v;
        __syncthreads();
        carry += last;
        __syncthreads();
    }
}

int exclusive_scan_u64(pyg_ctx* ctx, const unsigned long long* in, unsigned long long* out, int64_t n,
                       unsigned long long* total_dev)
{
    if (n <= 0) {
        if (total_dev) PYG_CUDA(cudaMemsetAsync(total_dev, 0, 8, ctx->stream));
        return PYG_OK;
    }
    int nb = (int)((n + 65535) / 65536);
    if (nb > 4096) nb = 4096;
    int64_t chunk = (n + nb - 1) / nb;
    nb = (int)((n + chunk - 1) / chunk);
    unsigned long long* partial;
    int rc = dalloc(ctx, (void**)&partial, nb * sizeof(unsigned long long));
    if (rc) return rc;
    scan_reduce_kernel<<<nb, SCAN_THREADS, 0, ctx->stream>>>(in, n, chunk, partial);
    PYG_LAUNCHED(ctx);
    scan_partials_kernel<<<1, SCAN_THREADS, 0, ctx->stream>>>(partial, nb, total_dev);
    PYG_LAUNCHED(ctx);
    scan_apply_kernel<<<nb, SCAN_THREADS, 0, ctx->stream>>>(in, out, n, chunk, partial);
    PYG_LAUNCHED(ctx);
    dfree(ctx, partial);
    return PYG_OK;
}

// ---------------------------------------------------------------------------
// Key bit range.

__global__ void bit_range_kernel(const uint64_t* __restrict__ keys, int64_t n, unsigned long long* out)
{
    uint64_t first = keys[0];
    uint64_t diff = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        diff |= keys[i] ^ first;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) diff |= __shfl_xor_sync(0xffffffffu, diff, o);
    if ((threadIdx.x & 31) == 0 && diff) atomicOr(out, (unsigned long long)diff);
}

int key_bit_range(pyg_ctx* ctx, const uint64_t* keys, int64_t n, int* begin_bit, int* end_bit)
{
    *begin_bit = *end_bit = 0;
    if (n <= 1) return PYG_OK;
    unsigned long long* d = ctx->dcounters + 32;
    PYG_CUDA(cudaMemsetAsync(d, 0, 8, ctx->stream));
    bit_range_kernel<<<grid_for(ctx, n, 256, 8, 4), 256, 0, ctx->stream>>>(keys, n, d);
    PYG_LAUNCHED(ctx);
    unsigned long long* h = (unsigned long long*)ctx->pinned + 64;
    PYG_CUDA(cudaMemcpyAsync(h, d, 8, cudaMemcpyDeviceToHost, ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    uint64_t diff = *h;
    if (!diff) return PYG_OK;
    *begin_bit = __builtin_ctzll(diff);
    *end_bit = 64 - __builtin_clzll(diff);
    return PYG_OK;
}

// ---------------------------------------------------------------------------
// LSD radix sort: 8-bit digits; per pass a histogram kernel, a scan, and a
// stable scatter.  A block owns a contiguous run of 2048-item sub-tiles;
// inside a sub-tile each warp ranks 8 rows of 32 items with match_any, so
// the order (warp, row, lane) equals the input order and the sort is stable.

constexpr int RS_THREADS = 256;
constexpr int RS_WARPS = RS_THREADS / 32;
constexpr int RS_ROWS = 8;
constexpr int RS_SUB = RS_THREADS * RS_ROWS;  // 2048 items per sub-tile
constexpr int RS_BINS = 256;

__global__ void __launch_bounds__(RS_THREADS) rs_hist_kernel(const uint64_t* __restrict__ keys, int64_t n,
                                                             int64_t subs_per_block, int shift,
                                                             unsigned long long* __restrict__ counts)
{
    __shared__ unsigned int hist[RS_BINS];
    hist[threadIdx.x] = 0;
    __syncthreads();
    int64_t lo = blockIdx.x * subs_per_block * RS_SUB;
    int64_t hi = min(n, lo + subs_per_block * RS_SUB);
    for (int64_t i = lo + threadIdx.x; i < hi; i += RS_THREADS)
        atomicAdd(&hist[(keys[i] >> shift) & 0xFF], 1u);
    __syncthreads();
    counts[(int64_t)threadIdx.x * gridDim.x + blockIdx.x] = hist[threadIdx.x];
}

__global__ void __launch_bounds__(RS_THREADS) rs_scatter_kernel(
    const uint64_t* __restrict__ keys, const uint64_t* __restrict__ vals, uint64_t* __restrict__ okeys,
    uint64_t* __restrict__ ovals, int64_t n, int64_t subs_per_block, int shift,
    const unsigned long long* __restrict__ offsets)
{
    __shared__ unsigned long long running[RS_BINS];
    __shared__ unsigned int wcnt[RS_WARPS][RS_BINS];
    __shared__ unsigned int total[RS_BINS];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    running[threadIdx.x] = offsets[(int64_t)threadIdx.x * gridDim.x + blockIdx.x];
    int64_t lo = blockIdx.x * subs_per_block * RS_SUB;
    int64_t hi = min(n, lo + subs_per_block * RS_SUB);
    const unsigned lt = (1u << lane) - 1;
    for (int64_t sub = lo; sub < hi; sub += RS_SUB) {
        for (int ww = 0; ww < RS_WARPS; ++ww) wcnt[ww][threadIdx.x] = 0;
        __syncthreads();
        uint64_t k[RS_ROWS], v[RS_ROWS];
        unsigned pos[RS_ROWS];
        int dg[RS_ROWS];
#pragma unroll
        for (int j = 0; j < RS_ROWS; ++j) {
            int64_t i = sub + w * (RS_ROWS * 32) + j * 32 + lane;
            bool valid = i < hi;
            k[j] = valid ? keys[i] : 0;
            v[j] = (valid && vals) ? vals[i] : 0;
            int d = valid ? (int)((k[j] >> shift) & 0xFF) : RS_BINS;
            dg[j] = d;
            unsigned mask = __match_any_sync(0xffffffffu, d);
            int leader = __ffs(mask) - 1;
            unsigned old = 0;
            if (lane == leader && valid) {
                old = wcnt[w][d];
                wcnt[w][d] = old + __popc(mask);
            }
            old = __shfl_sync(0xffffffffu, old, leader);
            pos[j] = old + __popc(mask & lt);
            __syncwarp();
        }
        __syncthreads();
        {
            unsigned base = 0;
#pragma unroll
            for (int ww = 0; ww < RS_WARPS; ++ww) {
                unsigned t = wcnt[ww][threadIdx.x];
                wcnt[ww][threadIdx.x] = base;
                base += t;
            }
            total[threadIdx.x] = base;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < RS_ROWS; ++j) {
            if (dg[j] == RS_BINS) continue;
            unsigned long long p = running[dg[j]] + wcnt[w][dg[j]] + pos[j];
            okeys[p] = k[j];
            if (vals) ovals[p] = v[j];
        }
        __syncthreads();
        running[threadIdx.x] += total[threadIdx.x];
        __syncthreads();
    }
}

int radix_sort_pairs(pyg_ctx* ctx, uint64_t* keys, uint64_t* vals, uint64_t* keys_alt, uint64_t* vals_alt,
                     int64_t n, int begin_bit, int end_bit, int* in_alt)
{
    *in_alt = 0;
    if (n <= 1 || end_bit <= begin_bit) return PYG_OK;
    int64_t subs = (n + RS_SUB - 1) / RS_SUB;
    int64_t max_blocks = (int64_t)ctx->sm_count * 4;
    int64_t spb = (subs + max_blocks - 1) / max_blocks;
    int blocks = (int)((subs + spb - 1) / spb);
    unsigned long long* counts;
    int rc = dalloc(ctx, (void**)&counts, (size_t)RS_BINS * blocks * sizeof(unsigned long long));
    if (rc) return rc;
    uint64_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
    for (int shift = begin_bit; shift < end_bit; shift += 8) {
        rs_hist_kernel<<<blocks, RS_THREADS, 0, ctx->stream>>>(ki, n, spb, shift, counts);
        PYG_LAUNCHED(ctx);
        if ((rc = exclusive_scan_u64(ctx, counts, counts, (int64_t)RS_BINS * blocks, nullptr))) break;
        rs_scatter_kernel<<<blocks, RS_THREADS, 0, ctx->stream>>>(ki, vi, ko, vo, n, spb, shift, counts);
        PYG_LAUNCHED(ctx);
        uint64_t* t = ki; ki = ko; ko = t;
        t = vi; vi = vo; vo = t;
        *in_alt ^= 1;
    }
    dfree(ctx, counts);
    return rc;
}

// ---------------------------------------------------------------------------
// Gather, key extraction, sort entry point.

template <typename V>
__global__ void gather_kernel(const V* __restrict__ in, const uint64_t* __restrict__ idx, int64_t n, int words,
                              V* __restrict__ out)
{
    int64_t total = n * words;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        int64_t r = t / words;
        int c = (int)(t - r * words);
        out[t] = in[idx[r] * words + c];
    }
}

int gather_rows(pyg_ctx* ctx, const uint8_t* in, const uint64_t* idx, int64_t n, int32_t tb, uint8_t* out)
{
    if (n <= 0) return PYG_OK;
    int threads = 256;
    if (tb % 16 == 0 && (uintptr_t)in % 16 == 0 && (uintptr_t)out % 16 == 0) {
        gather_kernel<uint4><<<grid_for(ctx, n * (tb / 16), threads, 4, 8), threads, 0, ctx->stream>>>(
            (const uint4*)in, idx, n, tb / 16, (uint4*)out);
    } else if (tb % 8 == 0 && (uintptr_t)in % 8 == 0 && (uintptr_t)out % 8 == 0) {
        gather_kernel<uint2><<<grid_for(ctx, n * (tb / 8), threads, 4, 8), threads, 0, ctx->stream>>>(
            (const uint2*)in, idx, n, tb / 8, (uint2*)out);
    } else if (tb % 4 == 0 && (uintptr_t)in % 4 == 0 && (uintptr_t)out % 4 == 0) {
        gather_kernel<unsigned><<<grid_for(ctx, n * (tb / 4), threads, 4, 8), threads, 0, ctx->stream>>>(
            (const unsigned*)in, idx, n, tb / 4, (unsigned*)out);
    } else {
        gather_kernel<unsigned char><<<grid_for(ctx, n * tb, threads, 4, 8), threads, 0, ctx->stream>>>(
            in, idx, n, tb, out);
    }
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

// Extract (sortable key, row index) from tuples.
__global__ void extract_keys_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb, int32_t off, int32_t type,
                                    uint64_t* __restrict__ keys, uint64_t* __restrict__ idx)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        keys[i] = to_sortable(load_col(base + i * (int64_t)tb, off, type));
        idx[i] = (uint64_t)i;
    }
}

// 16-byte tuples of two int64 columns: split into (sortable key, other).
__global__ void split16_kernel(const longlong2* __restrict__ in, int64_t n, int key_hi, uint64_t* __restrict__ keys,
                               uint64_t* __restrict__ other)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        longlong2 t = __ldcs(&in[i]);
        keys[i] = to_sortable(key_hi ? t.y : t.x);
        other[i] = (uint64_t)(key_hi ? t.x : t.y);
    }
}

__global__ void join16_kernel(const uint64_t* __restrict__ keys, const uint64_t* __restrict__ other, int64_t n,
                              int key_hi, longlong2* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        long long k = from_sortable(keys[i]);
        long long o = (long long)other[i];
        __stcs(&out[i], key_hi ? make_longlong2(o, k) : make_longlong2(k, o));
    }
}

// Sorts a device relation by one column into out (device).  Shared by the
// sort entry point and the MPSM join.
int sort_relation(pyg_ctx* ctx, const pyg_rel* r, int32_t key_col, void* out)
{
    int64_t n = r->ntuples;
    if (n == 0) return PYG_OK;
    int32_t off = r->col_offset[key_col], type = r->col_type[key_col];
    bool fast16 = r->tuple_bytes == 16 && r->ncols >= 1 && type == PYG_INT64 && (off == 0 || off == 8) &&
                  (uintptr_t)r->base % 16 == 0 && (uintptr_t)out % 16 == 0;
    uint64_t* buf;
    int rc = dalloc(ctx, (void**)&buf, (size_t)4 * n * sizeof(uint64_t));
    if (rc) return rc;
    uint64_t *k0 = buf, *v0 = buf + n, *k1 = buf + 2 * n, *v1 = buf + 3 * n;
    int threads = 256, grid = grid_for(ctx, n, threads, 4, 8);
    if (fast16) split16_kernel<<<grid, threads, 0, ctx->stream>>>((const longlong2*)r->base, n, off == 8, k0, v0);
    else extract_keys_kernel<<<grid, threads, 0, ctx->stream>>>((const uint8_t*)r->base, n, r->tuple_bytes, off, type, k0, v0);
    PYG_LAUNCHED(ctx);
    int b, e, alt = 0;
    if ((rc = key_bit_range(ctx, k0, n, &b, &e)) == PYG_OK) {
        rc = radix_sort_pairs(ctx, k0, v0, k1, v1, n, b, e, &alt);
    }
    if (rc == PYG_OK) {
        uint64_t* ks = alt ? k1 : k0;
        uint64_t* vs = alt ? v1 : v0;
        if (fast16) {
            join16_kernel<<<grid, threads, 0, ctx->stream>>>(ks, vs, n, off == 8, (longlong2*)out);
            PYG_LAUNCHED(ctx);
        } else {
            rc = gather_rows(ctx, (const uint8_t*)r->base, vs, n, r->tuple_bytes, (uint8_t*)out);
        }
    }
    dfree(ctx, buf);
    return rc;
}

__global__ void lower_bound_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb, int32_t off, int32_t type,
                                   const int64_t* __restrict__ q, int64_t nq, int64_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nq; i += (int64_t)gridDim.x * blockDim.x) {
        int64_t key = q[i];
        int64_t lo = 0, hi = n;
        while (lo < hi) {
            int64_t mid = lo + (hi - lo) / 2;
            if (load_col(base + mid * (int64_t)tb, off, type) < key) lo = mid + 1;
            else hi = mid;
        }
        out[i] = lo;
    }
}

}  // namespace pyg

using namespace pyg;

extern "C" {

int pyg_sort(pyg_ctx* ctx, const pyg_rel* in, int32_t key_col, void* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_rel(in, "sort input"))) return rc;
    if (key_col < 0 || key_col >= in->ncols || (in->ntuples > 0 && !out)) {
        set_error("pyg_sort: bad key column %d or null out", key_col);
        return PYG_ERR_ARG;
    }
    DevRel r;
    if ((rc = r.stage(ctx, in))) return rc;
    rc = sort_relation(ctx, &r.rel, key_col, out);
    r.release(ctx);
    if (rc) return rc;
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PYG_OK;
}

int pyg_lower_bound(pyg_ctx* ctx, const pyg_rel* sorted, int32_t key_col, const int64_t* queries, int64_t nq,
                    int64_t* out_idx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_rel(sorted, "sorted"))) return rc;
    if (key_col < 0 || key_col >= sorted->ncols || nq < 0 || (nq > 0 && (!queries || !out_idx))) {
        set_error("pyg_lower_bound: bad arguments");
        return PYG_ERR_ARG;
    }
    if (!sorted->on_device) {
        set_error("pyg_lower_bound: the sorted relation must be device-resident");
        return PYG_ERR_ARG;
    }
    if (nq == 0) return PYG_OK;
    lower_bound_kernel<<<grid_for(ctx, nq, 256, 1, 8), 256, 0, ctx->stream>>>(
        (const uint8_t*)sorted->base, sorted->ntuples, sorted->tuple_bytes, sorted->col_offset[key_col],
        sorted->col_type[key_col], queries, nq, out_idx);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

}  // extern "C"
