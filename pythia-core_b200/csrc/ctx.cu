// Context, errors, memory and relation staging for libpyg.
#include <stdarg.h>
#include <string.h>

#include "pyg_internal.cuh"

namespace pyg {

static thread_local char g_err[512] = "";

void set_error(const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int cuda_status(cudaError_t e, const char* what)
{
    set_error("CUDA error in %s: %s", what, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return PYG_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver || e == cudaErrorNoKernelImageForDevice)
        return PYG_ERR_NO_DEVICE;
    return PYG_ERR_CUDA;
}

int check_ctx(pyg_ctx* ctx)
{
    if (!ctx) {
        set_error("null context");
        return PYG_ERR_ARG;
    }
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return cuda_status(e, "cudaSetDevice");
    return PYG_OK;
}

int check_rel(const pyg_rel* r, const char* name)
{
    if (!r) {
        set_error("%s: null relation", name);
        return PYG_ERR_ARG;
    }
    if (r->ntuples < 0 || r->tuple_bytes <= 0 || r->ncols <= 0 || r->ncols > PYG_MAX_COLS) {
        set_error("%s: bad shape (ntuples=%lld tuple_bytes=%d ncols=%d)", name, (long long)r->ntuples,
                  r->tuple_bytes, r->ncols);
        return PYG_ERR_ARG;
    }
    if (r->ntuples > 0 && !r->base) {
        set_error("%s: null base with %lld tuples", name, (long long)r->ntuples);
        return PYG_ERR_ARG;
    }
    for (int c = 0; c < r->ncols; ++c) {
        int sz = r->col_type[c] == PYG_INT32 ? 4 : (r->col_type[c] == PYG_INT64 ? 8 : 0);
        if (!sz || r->col_offset[c] < 0 || r->col_offset[c] + sz > r->tuple_bytes) {
            set_error("%s: column %d has bad type %d or offset %d", name, c, r->col_type[c], r->col_offset[c]);
            return PYG_ERR_ARG;
        }
    }
    return PYG_OK;
}

int stage_h2d(pyg_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    if (bytes == 0) return PYG_OK;
    if (bytes > kPinnedUploadBytes) {
        PYG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
        return PYG_OK;
    }
    size_t at = (ctx->up_cursor + 255) & ~(size_t)255;
    if (at + bytes > kPinnedUploadBytes) {
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        at = 0;
    }
    unsigned char* area = (unsigned char*)ctx->pinned + kPinnedScalarBytes + kPinnedStageBytes;
    memcpy(area + at, src, bytes);
    ctx->up_cursor = at + bytes;
    PYG_CUDA(cudaMemcpyAsync(dst, area + at, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return PYG_OK;
}

int dalloc(pyg_ctx* ctx, void** p, size_t bytes)
{
    *p = nullptr;
    if (bytes == 0) bytes = 256;
    cudaError_t e = cudaMallocAsync(p, bytes, ctx->stream);
    if (e != cudaSuccess) {
        *p = nullptr;
        return cuda_status(e, "cudaMallocAsync");
    }
    return PYG_OK;
}

void dfree(pyg_ctx* ctx, void* p)
{
    if (p) cudaFreeAsync(p, ctx->stream);
}

int DevRel::stage(pyg_ctx* ctx, const pyg_rel* in)
{
    rel = *in;
    owned = nullptr;
    if (in->on_device || in->ntuples == 0) {
        rel.on_device = 1;
        return PYG_OK;
    }
    size_t bytes = (size_t)in->ntuples * in->tuple_bytes;
    int rc = dalloc(ctx, &owned, bytes);
    if (rc) return rc;
    PYG_CUDA(cudaMemcpyAsync(owned, in->base, bytes, cudaMemcpyHostToDevice, ctx->stream));
    rel.base = owned;
    rel.on_device = 1;
    return PYG_OK;
}

void DevRel::release(pyg_ctx* ctx)
{
    if (owned) dfree(ctx, owned);
    owned = nullptr;
}

int make_keyspec(const pyg_rel* r, const int32_t* cols, int32_t nkeys, KeySpec* ks)
{
    memset(ks, 0, sizeof(*ks));
    if (nkeys < 1 || nkeys > 2 || !cols) {
        set_error("keys: 1 or 2 key columns supported (got %d)", nkeys);
        return PYG_ERR_ARG;
    }
    for (int i = 0; i < nkeys; ++i)
        if (cols[i] < 0 || cols[i] >= r->ncols) {
            set_error("keys: column %d out of range", cols[i]);
            return PYG_ERR_ARG;
        }
    ks->nkeys = nkeys;
    ks->off0 = r->col_offset[cols[0]];
    ks->type0 = r->col_type[cols[0]];
    if (nkeys == 2) {
        ks->off1 = r->col_offset[cols[1]];
        ks->type1 = r->col_type[cols[1]];
        if (ks->type0 != PYG_INT32 || ks->type1 != PYG_INT32) {
            set_error("keys: a composite key must be two int32 columns (8 bytes total)");
            return PYG_ERR_ARG;
        }
    }
    return PYG_OK;
}

}  // namespace pyg

using namespace pyg;

extern "C" {

const char* pyg_last_error(void) { return g_err; }

const char* pyg_version(void) { return "pyg-b200 0.1 (sm_100a)"; }

int pyg_ctx_create(int device, pyg_ctx** out)
{
    if (!out) {
        set_error("pyg_ctx_create: null out");
        return PYG_ERR_ARG;
    }
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        set_error("no CUDA device available (%s)", e == cudaSuccess ? "0 devices" : cudaGetErrorString(e));
        return PYG_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= n) {
        set_error("device %d out of range (%d devices)", device, n);
        return PYG_ERR_ARG;
    }
    PYG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    PYG_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major < 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a", device, prop.major, prop.minor);
        return PYG_ERR_NO_DEVICE;
    }
    pyg_ctx* c = new pyg_ctx();
    memset(c, 0, sizeof(*c));
    c->device = device;
    c->sm_count = prop.multiProcessorCount;
    c->launches = 0;
    // A blocking stream: ordered with the legacy default stream that callers
    // (and frameworks) use unless they pass their own stream.
    e = cudaStreamCreate(&c->own_stream);
    if (e != cudaSuccess) {
        delete c;
        return cuda_status(e, "cudaStreamCreate");
    }
    c->stream = c->own_stream;
    c->pinned_bytes = kPinnedScalarBytes + kPinnedStageBytes + kPinnedUploadBytes;
    e = cudaMallocHost(&c->pinned, c->pinned_bytes);
    if (e == cudaSuccess) e = cudaMalloc((void**)&c->dcounters, 4096);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->copy_stream, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&c->copied[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->consumed[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        cudaStreamDestroy(c->own_stream);
        if (c->pinned) cudaFreeHost(c->pinned);
        delete c;
        return cuda_status(e, "context buffers");
    }
    // Keep freed pool memory cached across calls (no release at sync).
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    *out = c;
    return PYG_OK;
}

int pyg_ctx_destroy(pyg_ctx* ctx)
{
    if (!ctx) return PYG_OK;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamSynchronize(ctx->copy_stream);
    for (int i = 0; i < 2; ++i) {
        cudaEventDestroy(ctx->copied[i]);
        cudaEventDestroy(ctx->consumed[i]);
    }
    cudaStreamDestroy(ctx->copy_stream);
    if (ctx->join_arena) cudaFree(ctx->join_arena);  // synchronous: the caller's stream may be gone
    cudaFree(ctx->dcounters);
    cudaFreeHost(ctx->pinned);
    cudaStreamDestroy(ctx->own_stream);
    delete ctx;
    return PYG_OK;
}

int pyg_ctx_set_stream(pyg_ctx* ctx, void* s)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    ctx->stream = s ? (cudaStream_t)s : ctx->own_stream;
    return PYG_OK;
}

void* pyg_ctx_stream(pyg_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

int pyg_ctx_sync(pyg_ctx* ctx)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PYG_OK;
}

int64_t pyg_ctx_kernel_launches(pyg_ctx* ctx) { return ctx ? ctx->launches : 0; }

int pyg_alloc(pyg_ctx* ctx, size_t bytes, void** out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) {
        set_error("pyg_alloc: null out");
        return PYG_ERR_ARG;
    }
    return dalloc(ctx, out, bytes);
}

int pyg_free(pyg_ctx* ctx, void* p)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    dfree(ctx, p);
    return PYG_OK;
}

int pyg_host_alloc(size_t bytes, void** out)
{
    if (!out) {
        set_error("pyg_host_alloc: null out");
        return PYG_ERR_ARG;
    }
    PYG_CUDA(cudaMallocHost(out, bytes ? bytes : 1));
    return PYG_OK;
}

int pyg_host_free(void* p)
{
    if (p) PYG_CUDA(cudaFreeHost(p));
    return PYG_OK;
}

int pyg_memcpy_h2d(pyg_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (bytes) PYG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return PYG_OK;
}

int pyg_memcpy_d2h(pyg_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (bytes) PYG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    return PYG_OK;
}

int pyg_memcpy_d2d(pyg_ctx* ctx, void* dst, const void* src, size_t bytes)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (bytes) PYG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
    return PYG_OK;
}

}  // extern "C"
