// Radix / range partitioning: per-block shared-memory histograms, one
// exclusive scan over (bucket, block), then a scatter pass in which each
// warp reserves output slots for lanes of the same bucket with one shared
// atomic (__match_any_sync).  Follows PartitionOp::scanStart
// (operators/partition.cpp:272-359): histogram, prefix, exact allocation,
// scatter.  The fan-out is not limited to 127 as the reference's is (the
// number of partitions there is the number of threads).
#include <string.h>

#include "partition.cuh"
#include "primitives.cuh"

namespace pyg {

constexpr int PT_THREADS = 512;
constexpr int PT_SMEM_SPLITTERS = 4096;

__device__ __forceinline__ const int64_t* load_splitters(const BucketFn& f, int64_t* sm)
{
    if (f.kind != PYG_SPLIT_SPLITTERS || f.fanout - 1 > (uint32_t)PT_SMEM_SPLITTERS) return nullptr;
    for (uint32_t i = threadIdx.x; i + 1 < f.fanout; i += blockDim.x) sm[i] = f.spl[i];
    return sm;
}

__global__ void __launch_bounds__(PT_THREADS) pt_hist_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb,
                                                             int32_t off, int32_t type, BucketFn f, int64_t chunk,
                                                             unsigned long long* __restrict__ hist,
                                                             unsigned long long* __restrict__ err)
{
    extern __shared__ unsigned char smraw[];
    unsigned* h = (unsigned*)smraw;
    int64_t* ssp = (int64_t*)(smraw + (((size_t)f.fanout * 4 + 15) & ~(size_t)15));
    for (uint32_t i = threadIdx.x; i < f.fanout; i += blockDim.x) h[i] = 0;
    const int64_t* sp = load_splitters(f, ssp);
    __syncthreads();
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    bool bad = false;
    for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
        uint32_t b = bucket_of(f, load_col(base + i * (int64_t)tb, off, type), sp);
        if (b >= f.fanout) {
            bad = true;
            continue;
        }
        atomicAdd(&h[b], 1u);
    }
    if (bad) atomicOr(err, 1ULL);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < f.fanout; i += blockDim.x)
        hist[(int64_t)i * gridDim.x + blockIdx.x] = h[i];
}

template <typename W>
__global__ void __launch_bounds__(PT_THREADS) pt_scatter_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb,
                                                                int32_t off, int32_t type, BucketFn f, int64_t chunk,
                                                                const unsigned long long* __restrict__ offs,
                                                                uint8_t* __restrict__ out)
{
    extern __shared__ unsigned char smraw[];
    unsigned long long* cur = (unsigned long long*)smraw;
    int64_t* ssp = (int64_t*)(smraw + (size_t)f.fanout * 8);
    for (uint32_t i = threadIdx.x; i < f.fanout; i += blockDim.x) cur[i] = offs[(int64_t)i * gridDim.x + blockIdx.x];
    const int64_t* sp = load_splitters(f, ssp);
    __syncthreads();
    const int words = tb / (int)sizeof(W);
    const unsigned lane = threadIdx.x & 31;
    int64_t lo = blockIdx.x * chunk, hi = min(n, lo + chunk);
    for (int64_t wb = lo + (threadIdx.x & ~31u); wb < hi; wb += blockDim.x) {
        int64_t i = wb + lane;
        bool valid = i < hi;
        const W* src = (const W*)(base + i * (int64_t)tb);
        uint32_t b = valid ? bucket_of(f, load_col((const uint8_t*)src, off, type), sp) : 0xFFFFFFFFu;
        if (b >= f.fanout) valid = false;
        unsigned mask = __match_any_sync(0xffffffffu, valid ? b : 0xFFFFFFFFu);
        int leader = __ffs(mask) - 1;
        unsigned long long p = 0;
        if (valid && (int)lane == leader) p = atomicAdd(&cur[b], (unsigned long long)__popc(mask));
        p = __shfl_sync(0xffffffffu, p, leader);
        if (!valid) continue;
        p += __popc(mask & ((1u << lane) - 1));
        W* dst = (W*)(out + (int64_t)p * tb);
        for (int w = 0; w < words; ++w) dst[w] = src[w];
    }
}

__global__ void pt_offsets_kernel(const unsigned long long* __restrict__ scanned, uint32_t fanout, int blocks,
                                  int64_t n, unsigned long long* __restrict__ offsets)
{
    for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b <= fanout; b += gridDim.x * blockDim.x)
        offsets[b] = b == fanout ? (unsigned long long)n : scanned[(int64_t)b * blocks];
}

int make_bucket_fn(pyg_ctx* ctx, const pyg_splitter* spl, BucketFn* f, int64_t** spl_dev)
{
    memset(f, 0, sizeof(*f));
    *spl_dev = nullptr;
    if (!spl || spl->fanout < 1 || spl->fanout > (1 << 20)) {
        set_error("partition: fan-out must be in [1, 2^20]");
        return PYG_ERR_ARG;
    }
    f->kind = spl->kind;
    f->fanout = (uint32_t)spl->fanout;
    switch (spl->kind) {
    case PYG_SPLIT_EXACTRANGE: {
        if (spl->range_max < spl->range_min) {
            set_error("partition: exactrange max < min");
            return PYG_ERR_ARG;
        }
        // ExactRangeValueHasher (hash.h:452-487): bucket range
        // (max - min + k) / k, bucket = (value - min) / range.
        f->mn = spl->range_min;
        f->br = (spl->range_max - spl->range_min + (int64_t)spl->fanout) / (int64_t)spl->fanout;
        return PYG_OK;
    }
    case PYG_SPLIT_SPLITTERS: {
        if (spl->fanout > 1 && !spl->splitters) {
            set_error("partition: null splitters");
            return PYG_ERR_ARG;
        }
        for (int i = 0; i + 2 < spl->fanout; ++i)
            if (spl->splitters[i] > spl->splitters[i + 1]) {
                set_error("partition: splitters not ascending at %d", i);
                return PYG_ERR_ARG;
            }
        if (spl->fanout > 1) {
            int rc = dalloc(ctx, (void**)spl_dev, (spl->fanout - 1) * sizeof(int64_t));
            if (rc) return rc;
            PYG_CUDA(cudaMemcpyAsync(*spl_dev, spl->splitters, (spl->fanout - 1) * sizeof(int64_t),
                                     cudaMemcpyHostToDevice, ctx->stream));
        }
        f->spl = *spl_dev;
        return PYG_OK;
    }
    case PYG_SPLIT_RADIX:
    case PYG_SPLIT_HASH: {
        if (spl->fanout & (spl->fanout - 1)) {
            set_error("partition: radix/hash fan-out must be a power of two");
            return PYG_ERR_ARG;
        }
        f->log2f = __builtin_ctz((unsigned)spl->fanout);
        return PYG_OK;
    }
    default:
        set_error("partition: unknown splitter kind %d", spl->kind);
        return PYG_ERR_ARG;
    }
}

int partition_device(pyg_ctx* ctx, const pyg_rel* in, int32_t key_col, const BucketFn& f, void* out,
                     unsigned long long* offsets_dev)
{
    int64_t n = in->ntuples;
    int threads = PT_THREADS;
    // A few large chunks per SM keep the (bucket x block) histogram small.
    int blocks = grid_for(ctx, n, threads, 16, 2);
    int64_t chunk = (n + blocks - 1) / blocks;
    if (chunk < 1) chunk = 1;
    blocks = (int)((n + chunk - 1) / chunk);
    if (blocks < 1) blocks = 1;
    size_t spl_smem = (f.kind == PYG_SPLIT_SPLITTERS && f.fanout - 1 <= (uint32_t)PT_SMEM_SPLITTERS)
                          ? (size_t)(f.fanout - 1) * 8 : 0;
    size_t hist_smem = (((size_t)f.fanout * 4 + 15) & ~(size_t)15) + spl_smem;
    size_t scat_smem = (size_t)f.fanout * 8 + spl_smem;
    if (scat_smem > 200 * 1024 || hist_smem > 200 * 1024) {
        set_error("partition: fan-out %u too large for one pass", f.fanout);
        return PYG_ERR_ARG;
    }
    unsigned long long* hist;
    int rc = dalloc(ctx, (void**)&hist, (size_t)f.fanout * blocks * sizeof(unsigned long long));
    if (rc) return rc;
    unsigned long long* err = ctx->dcounters + 64;
    PYG_CUDA(cudaMemsetAsync(err, 0, 8, ctx->stream));
    int32_t off = in->col_offset[key_col], type = in->col_type[key_col];
    const uint8_t* base = (const uint8_t*)in->base;
    PYG_CUDA(cudaFuncSetAttribute(pt_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hist_smem));
    pt_hist_kernel<<<blocks, threads, hist_smem, ctx->stream>>>(base, n, in->tuple_bytes, off, type, f, chunk, hist, err);
    PYG_LAUNCHED(ctx);
    unsigned long long* h = (unsigned long long*)ctx->pinned + 72;
    PYG_CUDA(cudaMemcpyAsync(h, err, 8, cudaMemcpyDeviceToHost, ctx->stream));
    if ((rc = exclusive_scan_u64(ctx, hist, hist, (int64_t)f.fanout * blocks, nullptr))) {
        dfree(ctx, hist);
        return rc;
    }
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    if (*h) {
        dfree(ctx, hist);
        set_error("partition: a key falls outside the exactrange bounds");
        return PYG_ERR_ARG;
    }
    int tb = in->tuple_bytes;
    bool a16 = tb % 16 == 0 && (uintptr_t)base % 16 == 0 && (uintptr_t)out % 16 == 0;
    bool a8 = tb % 8 == 0 && (uintptr_t)base % 8 == 0 && (uintptr_t)out % 8 == 0;
    bool a4 = tb % 4 == 0 && (uintptr_t)base % 4 == 0 && (uintptr_t)out % 4 == 0;
    if (n > 0) {
        if (a16) {
            PYG_CUDA(cudaFuncSetAttribute(pt_scatter_kernel<uint4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scat_smem));
            pt_scatter_kernel<uint4><<<blocks, threads, scat_smem, ctx->stream>>>(base, n, tb, off, type, f, chunk, hist, (uint8_t*)out);
        } else if (a8) {
            PYG_CUDA(cudaFuncSetAttribute(pt_scatter_kernel<uint2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scat_smem));
            pt_scatter_kernel<uint2><<<blocks, threads, scat_smem, ctx->stream>>>(base, n, tb, off, type, f, chunk, hist, (uint8_t*)out);
        } else if (a4) {
            PYG_CUDA(cudaFuncSetAttribute(pt_scatter_kernel<unsigned>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scat_smem));
            pt_scatter_kernel<unsigned><<<blocks, threads, scat_smem, ctx->stream>>>(base, n, tb, off, type, f, chunk, hist, (uint8_t*)out);
        } else {
            PYG_CUDA(cudaFuncSetAttribute(pt_scatter_kernel<unsigned char>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)scat_smem));
            pt_scatter_kernel<unsigned char><<<blocks, threads, scat_smem, ctx->stream>>>(base, n, tb, off, type, f, chunk, hist, (uint8_t*)out);
        }
        PYG_LAUNCHED(ctx);
    }
    pt_offsets_kernel<<<grid_for(ctx, f.fanout + 1, 256, 1, 4), 256, 0, ctx->stream>>>(hist, f.fanout, blocks, n,
                                                                                      offsets_dev);
    PYG_LAUNCHED(ctx);
    dfree(ctx, hist);
    return PYG_OK;
}

}  // namespace pyg

using namespace pyg;

extern "C" int pyg_partition(pyg_ctx* ctx, const pyg_rel* in, int32_t key_col, const pyg_splitter* spl, void* out,
                             int64_t* offsets)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_rel(in, "partition input"))) return rc;
    if (key_col < 0 || key_col >= in->ncols || !offsets || (in->ntuples > 0 && !out)) {
        set_error("pyg_partition: bad key column or null output");
        return PYG_ERR_ARG;
    }
    BucketFn f;
    int64_t* spl_dev = nullptr;
    if ((rc = make_bucket_fn(ctx, spl, &f, &spl_dev))) return rc;
    DevRel r;
    if ((rc = r.stage(ctx, in))) {
        dfree(ctx, spl_dev);
        return rc;
    }
    unsigned long long* offs;
    if ((rc = dalloc(ctx, (void**)&offs, ((size_t)f.fanout + 1) * 8))) {
        r.release(ctx);
        dfree(ctx, spl_dev);
        return rc;
    }
    rc = partition_device(ctx, &r.rel, key_col, f, out, offs);
    if (rc == PYG_OK) {
        cudaError_t e = cudaMemcpyAsync(offsets, offs, ((size_t)f.fanout + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_status(e, "partition offsets");
    }
    dfree(ctx, offs);
    r.release(ctx);
    dfree(ctx, spl_dev);
    return rc;
}
