// Internal definitions shared by the libpyg CUDA sources (sm_100a only).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string>

#include "../../include/pyg.h"

constexpr size_t kPinnedScalarBytes = (size_t)1 << 16;  // scalar read-backs (fixed word offsets)
constexpr size_t kPinnedStageBytes = (size_t)1 << 21;   // two relations x 2^16 partition counts x 8 B, x2
constexpr size_t kPinnedUploadBytes = (size_t)1 << 23;  // host arrays staged for device copies (stage_h2d)

struct pyg_ctx {
    int device;
    int sm_count;
    cudaStream_t own_stream;
    cudaStream_t stream;
    int64_t launches;
    // Pinned host staging: kPinnedScalarBytes for scalar results read back
    // per call, then kPinnedStageBytes for per-partition counts.
    void* pinned;
    size_t pinned_bytes;
    // Device scratch for scalar counters (zeroed per use).
    unsigned long long* dcounters;
    // Second stream and events for overlapping host->device copies with
    // kernels when an input relation lives in host memory.
    cudaStream_t copy_stream;
    cudaEvent_t copied[2], consumed[2];
    // Grow-only device buffer reused by the one-shot direct join for its
    // table and side list (no allocation per call once it is large enough;
    // freed with the context).
    void* join_arena;
    size_t join_arena_bytes;
    // Bump cursor into the pinned upload area (after the scalar and stage
    // areas) used by stage_h2d.
    size_t up_cursor;
};

namespace pyg {

void set_error(const char* fmt, ...);

// Records the error (if any) of the last CUDA call and maps it to a status.
int cuda_status(cudaError_t e, const char* what);

#define PYG_CUDA(call)                                                  \
    do {                                                                \
        cudaError_t _e = (call);                                        \
        if (_e != cudaSuccess) return ::pyg::cuda_status(_e, #call);    \
    } while (0)

#define PYG_LAUNCHED(ctx)                                               \
    do {                                                                \
        (ctx)->launches++;                                              \
        cudaError_t _e = cudaGetLastError();                            \
        if (_e != cudaSuccess) return ::pyg::cuda_status(_e, "launch"); \
    } while (0)

int check_ctx(pyg_ctx* ctx);
int check_rel(const pyg_rel* r, const char* name);

// Host -> device copy on ctx->stream through the context's pinned upload
// area: src is copied into pinned memory first, so the asynchronous copy
// neither blocks on pageable staging nor depends on src afterwards.  The
// area is used as a bump allocator; when it is full, the stream is
// synchronised (every earlier copy out of it has then completed) and it
// starts over.  Copies larger than the area go directly from src
// (pageable, synchronously staged by the driver).
int stage_h2d(pyg_ctx* ctx, void* dst, const void* src, size_t bytes);
// Marks the upload area free; call only right after ctx->stream was
// synchronised.
inline void stage_reset(pyg_ctx* ctx) { ctx->up_cursor = 0; }

// Device memory from the stream-ordered pool.
int dalloc(pyg_ctx* ctx, void** p, size_t bytes);
void dfree(pyg_ctx* ctx, void* p);

// A relation staged on the device: either the caller's device buffer or a
// temporary copy of a host buffer (freed by release()).
struct DevRel {
    pyg_rel rel;
    void* owned = nullptr;
    int stage(pyg_ctx* ctx, const pyg_rel* in);
    void release(pyg_ctx* ctx);
};

// Key of up to 8 bytes packed into one 64-bit word.  A single int64 column
// is the value itself; a single int32 column is sign-extended; a pair of
// int32 columns is (first << 32) | (uint32)second, so the packed word's
// signed order is the lexicographic order of the pair.
struct KeySpec {
    int32_t nkeys;
    int32_t off0, off1;
    int32_t type0, type1;
};
int make_keyspec(const pyg_rel* r, const int32_t* cols, int32_t nkeys, KeySpec* ks);

// Column reader description for up to PYG_MAX_COLS value columns.
struct ColSpec {
    int32_t n;
    int32_t off[PYG_MAX_COLS];
    int32_t type[PYG_MAX_COLS];
};

// Column access.  Every column of a packed relation is 4 or 8 bytes wide
// and starts at a multiple of 4 bytes (columns are packed back to back and
// buffers are at least 16-byte aligned), so a column is read with one
// 32-bit load, or one 64-bit load when 8-byte aligned, else two 32-bit loads.
__device__ __forceinline__ int64_t load_col(const uint8_t* t, int32_t off, int32_t type)
{
    const uint8_t* p = t + off;
    if (type == PYG_INT32) return (int64_t)*reinterpret_cast<const int32_t*>(p);
    if (((uintptr_t)p & 7) == 0) return *reinterpret_cast<const int64_t*>(p);
    const uint32_t* q = reinterpret_cast<const uint32_t*>(p);
    return (int64_t)(((uint64_t)q[1] << 32) | (uint64_t)q[0]);
}

__device__ __forceinline__ void store_col(uint8_t* t, int32_t off, int32_t type, uint64_t v)
{
    uint8_t* p = t + off;
    if (type == PYG_INT32) {
        *reinterpret_cast<uint32_t*>(p) = (uint32_t)v;
    } else if (((uintptr_t)p & 7) == 0) {
        *reinterpret_cast<uint64_t*>(p) = v;
    } else {
        uint32_t* q = reinterpret_cast<uint32_t*>(p);
        q[0] = (uint32_t)v;
        q[1] = (uint32_t)(v >> 32);
    }
}

__device__ __forceinline__ uint64_t load_key(const uint8_t* t, const KeySpec& ks)
{
    if (ks.nkeys == 1) return (uint64_t)load_col(t, ks.off0, ks.type0);
    uint32_t a = *reinterpret_cast<const uint32_t*>(t + ks.off0);
    uint32_t b = *reinterpret_cast<const uint32_t*>(t + ks.off1);
    return ((uint64_t)a << 32) | (uint64_t)b;
}

// 64-bit finaliser (the MurmurHash3 fmix64 mixing function).  It is a
// bijection, so distinct keys never share a mixed value.
__host__ __device__ __forceinline__ uint64_t mix64(uint64_t k)
{
    k ^= k >> 33;
    k *= 0xff51afd7ed558ccdULL;
    k ^= k >> 33;
    k *= 0xc4ceb9fe1a85ec53ULL;
    k ^= k >> 33;
    return k;
}

// Slot index in [0, cap) from a mixed hash: multiply-high range reduction.
__device__ __forceinline__ uint64_t reduce_range(uint64_t h, uint64_t cap)
{
    return __umul64hi(h, cap);
}

constexpr uint64_t kEmptyKey = 0x8000000000000000ULL;

inline int grid_for(pyg_ctx* ctx, int64_t work, int threads, int per_thread, int blocks_per_sm)
{
    int64_t need = (work + (int64_t)threads * per_thread - 1) / ((int64_t)threads * per_thread);
    int64_t cap = (int64_t)ctx->sm_count * blocks_per_sm;
    if (need < 1) need = 1;
    return (int)(need < cap ? need : cap);
}

// Warp-level 64-bit sum.
__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace pyg
