// Page sort of 8-byte records (the reference's TupleBuffer::bitonicsort,
// util/buffer.cpp:97-110, and its SIMD merge sort, util/bitonicsort.cpp):
// records {int32 rid; int32 key} ordered by the signed key.
//
//   1. page sort   each CTA receives one 4096-record page (32 KB, the
//                  reference's CACHE_SIZE block) by bulk copy into shared
//                  memory (completion on an mbarrier, bounded wait), sorts it
//                  with a bitonic network (stages of stride >= 32 across the
//                  CTA with barriers, smaller strides inside each warp's
//                  registers by shuffles) and writes it back;
//   2. merge       merge-path passes double the sorted run length until one
//                  run remains (ping-pong with a scratch buffer).
//
// Items compare as one unsigned 64-bit word: the record read little-endian
// is (key << 32) | rid, so flipping the top bit orders by (signed key,
// unsigned rid); equal keys end in rid order (the reference leaves their
// order open).
#include <string.h>

#include "bulk.cuh"
#include "pyg_internal.cuh"

namespace pyg {

constexpr int BS_PAGE = 4096;           // records per page
constexpr int BS_THREADS = 1024;        // 4 records per thread
constexpr int BS_PER = BS_PAGE / BS_THREADS;
constexpr unsigned long long kBsWaitNs = 2000000000ULL;
constexpr uint64_t kFlip = 0x8000000000000000ULL;

__device__ __forceinline__ void cmp_swap(uint64_t& a, uint64_t& b, bool up)
{
    if ((a > b) == up) {
        const uint64_t t = a;
        a = b;
        b = t;
    }
}

// Sorts page `blockIdx.x` of in (n records) into out; a last partial page is
// padded with all-ones items, which sort after every record.
__global__ void __launch_bounds__(BS_THREADS) bs_page_kernel(const uint64_t* __restrict__ in, int64_t n,
                                                             uint64_t* __restrict__ out, unsigned* __restrict__ err)
{
    __shared__ __align__(128) uint64_t page[BS_PAGE];
    __shared__ uint64_t bar;
    const int64_t base = (int64_t)blockIdx.x * BS_PAGE;
    const int cnt = n - base < (int64_t)BS_PAGE ? (int)(n - base) : BS_PAGE;
    const int tid = threadIdx.x;
    // Bulk copy of the page's whole 16-byte units; an odd last record is
    // read by a plain load.
    const int units = cnt / 2;
    if (tid == 0) {
        mbar_init(&bar, 1);
        mbar_fence_init();
        if (units > 0) {
            mbar_arrive_expect_tx(&bar, (unsigned)units * 16u);
            bulk_load(page, in + base, (unsigned)units * 16u, &bar);
        } else {
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&bar)) : "memory");
        }
    }
    __shared__ int ok;
    if (tid == 0) ok = 1;
    __syncthreads();
    // Every thread waits (bounded); a wait that runs out fails the whole
    // CTA after the barrier, so no thread is left at a barrier alone.
    if (!mbar_wait(&bar, 0, kBsWaitNs)) ok = 0;
    if (tid == 0 && 2 * units < cnt) page[cnt - 1] = in[base + cnt - 1];  // odd last record
    __syncthreads();
    if (!ok) {
        if (tid == 0) atomicOr(err, 1u);
        return;
    }
    // Order-preserving flip of the records; padding is the largest item.
    for (int i = tid; i < BS_PAGE; i += BS_THREADS) page[i] = i < cnt ? page[i] ^ kFlip : ~0ULL;
    __syncthreads();
    // Strides >= 32 pair items across the CTA between barriers; smaller
    // strides run inside warps on 32 consecutive items, by shuffles.
    for (int k = 2; k <= BS_PAGE; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                for (int p = tid; p < BS_PAGE / 2; p += BS_THREADS) {
                    const int i = 2 * p - (p & (j - 1));  // lower index of pair p at stride j
                    const bool up = (i & k) == 0;
                    uint64_t a = page[i], b = page[i + j];
                    cmp_swap(a, b, up);
                    page[i] = a;
                    page[i + j] = b;
                }
                __syncthreads();
            } else {
                // Remaining strides j .. 1 of this k inside warps: each
                // warp owns runs of 32 consecutive items.
                const int lane = tid & 31;
                for (int r = 0; r < BS_PER; ++r) {
                    const int i = ((tid >> 5) + r * (BS_THREADS / 32)) * 32 + lane;
                    uint64_t v = page[i];
                    for (int jj = j; jj > 0; jj >>= 1) {
                        const uint64_t o = __shfl_xor_sync(0xffffffffu, v, jj);
                        const bool up = (i & k) == 0;
                        const bool lower = (lane & jj) == 0;
                        // Lower element keeps the smaller item when ascending.
                        const bool take_min = (lower == up);
                        v = take_min ? (v < o ? v : o) : (v > o ? v : o);
                    }
                    page[i] = v;
                }
                __syncthreads();
                break;  // strides below 32 of this k are done
            }
        }
    }
    for (int i = tid; i < cnt; i += BS_THREADS) out[base + i] = page[i] ^ kFlip;
}

// One merge pass: runs of `run` items of in (flipped order) merged pairwise
// into out; each thread produces BS_MPER consecutive outputs found by a
// merge-path search.
constexpr int BS_MPER = 8;

__global__ void bs_merge_kernel(const uint64_t* __restrict__ in, int64_t n, int64_t run, uint64_t* __restrict__ out)
{
    const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    const int64_t d0 = t * BS_MPER;  // first output index of this thread
    if (d0 >= n) return;
    const int64_t pair = d0 / (2 * run);
    const int64_t a0 = pair * 2 * run, a1 = min(n, a0 + run), b1 = min(n, a0 + 2 * run);
    const int64_t la = a1 - a0, lb = b1 - a1;
    const int64_t diag = d0 - a0;  // position on the merge path of this pair
    // Largest i in [max(0, diag - lb), min(diag, la)] with A[i - 1] <= B[diag - i] ...
    int64_t lo = diag > lb ? diag - lb : 0, hi = diag < la ? diag : la;
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;  // take mid items of A: valid when A[mid] <= B[diag - mid - 1]
        if ((in[a0 + mid] ^ kFlip) <= (in[a1 + diag - mid - 1] ^ kFlip)) lo = mid + 1;
        else hi = mid;
    }
    int64_t i = a0 + lo, j = a1 + (diag - lo);
    const int64_t end = min(d0 + BS_MPER, a0 + la + lb);
    for (int64_t d = d0; d < end; ++d) {
        bool takeA;
        if (i >= a1) takeA = false;
        else if (j >= b1) takeA = true;
        else takeA = (in[i] ^ kFlip) <= (in[j] ^ kFlip);
        out[d] = takeA ? in[i++] : in[j++];
    }
}

}  // namespace pyg

using namespace pyg;

extern "C" int pyg_bitonic_sort(pyg_ctx* ctx, void* records, int64_t n)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (n < 0 || (n > 0 && !records) || ((uintptr_t)records % 16)) {
        set_error("pyg_bitonic_sort: bad arguments (16-byte aligned device records)");
        return PYG_ERR_ARG;
    }
    if (n <= 1) return PYG_OK;
    uint64_t* buf = nullptr;
    if ((rc = dalloc(ctx, (void**)&buf, (size_t)n * 8))) return rc;
    unsigned* err = (unsigned*)(ctx->dcounters + 124);
    PYG_CUDA(cudaMemsetAsync(err, 0, 4, ctx->stream));
    const int64_t pages = (n + BS_PAGE - 1) / BS_PAGE;
    uint64_t* a = (uint64_t*)records;
    uint64_t* b = buf;
    // Pages sorted from the caller's buffer into the scratch buffer, then
    // merge passes ping-pong until one run remains.
    bs_page_kernel<<<(unsigned)pages, BS_THREADS, 0, ctx->stream>>>(a, n, b, err);
    PYG_LAUNCHED(ctx);
    for (int64_t run = BS_PAGE; run < n; run *= 2) {
        const int64_t threads = (n + BS_MPER - 1) / BS_MPER;
        bs_merge_kernel<<<(unsigned)((threads + 255) / 256), 256, 0, ctx->stream>>>(b, n, run, a);
        PYG_LAUNCHED(ctx);
        uint64_t* t = a;
        a = b;
        b = t;
    }
    if (b != (uint64_t*)records) PYG_CUDA(cudaMemcpyAsync(records, b, (size_t)n * 8, cudaMemcpyDeviceToDevice, ctx->stream));
    unsigned h = 0;
    PYG_CUDA(cudaMemcpyAsync(ctx->pinned, err, 4, cudaMemcpyDeviceToHost, ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    memcpy(&h, ctx->pinned, 4);
    dfree(ctx, buf);
    if (h) {
        set_error("pyg_bitonic_sort: a page copy did not complete in time");
        return PYG_ERR_TIMEOUT;
    }
    return PYG_OK;
}
