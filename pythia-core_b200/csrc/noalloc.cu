// Hash join + sum that allocates nothing: the table lives in a fixed
// file-scope device array instead of memory obtained from cudaMalloc.
//
// For callers that cannot allocate device memory at the point of the call:
// engines whose memory is owned by another allocator (a framework's pool
// or a query runtime's arena) that the library must not bypass, or
// real-time paths where an allocation may block on the device.  The
// caller passes device inputs and a device output; the call only enqueues
// kernels on the caller's stream.
//
// Limits and sharing: the scratch array holds one table of
// kNoAllocSlots 32-byte slots, enough for PYG_NOALLOC_MAX_BUILD build
// tuples at a load factor of 0.5; every GPU that loads the library keeps
// the array (about 16 MiB) until the process exits.  All calls on a device
// share the one array and each call starts by clearing it, so calls whose
// kernels overlap on the GPU (different streams without ordering between
// them) race and give wrong results: order such calls on one stream.
#include <mutex>

#include "pyg_internal.cuh"

namespace pyg {

constexpr uint64_t kNoAllocSlots = 1ULL << 19;  // 2 x PYG_NOALLOC_MAX_BUILD
constexpr int kNoAllocHeader = 16;              // u64 accumulators before the table
constexpr size_t kNoAllocBytes = kNoAllocHeader * 8 + kNoAllocSlots * 32;

// The scratch.  Host code never uses this name as an address (on the host
// it is a stand-in symbol); the address comes from cudaGetSymbolAddress.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

// Header words: [0] count, [1] build-payload sum, [2] probe-value sum,
// [3] / [4] build tuples with the empty-marker key (count / payload sum),
// [5] / [6] probe tuples with that key (count / value sum).
__global__ void noalloc_clear_kernel(unsigned long long* head, ulonglong4* table, uint64_t cap)
{
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < kNoAllocHeader) head[i] = 0;
    for (; i < cap; i += (uint64_t)gridDim.x * blockDim.x) table[i] = make_ulonglong4(kEmptyKey, 0, 0, 0);
}

__global__ void noalloc_build_kernel(const longlong2* __restrict__ R, int64_t n, unsigned long long* head,
                                     ulonglong4* table, uint64_t cap)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        longlong2 t = R[i];
        uint64_t k = (uint64_t)t.x;
        if (k == kEmptyKey) {
            atomicAdd(&head[3], 1ULL);
            atomicAdd(&head[4], (unsigned long long)t.y);
            continue;
        }
        // cap >= 2n, so an empty slot is always found.
        uint64_t s = reduce_range(mix64(k), cap);
        for (uint64_t steps = 0; steps < cap; ++steps) {
            unsigned long long* slot = (unsigned long long*)&table[s];
            unsigned long long prev = atomicCAS(slot, kEmptyKey, k);
            if (prev == kEmptyKey || prev == k) {
                atomicAdd(slot + 1, (unsigned long long)t.y);
                atomicAdd(slot + 2, 1ULL);
                break;
            }
            s = (s + 1 == cap) ? 0 : s + 1;
        }
    }
}

__global__ void noalloc_probe_kernel(const longlong2* __restrict__ S, int64_t n, unsigned long long* head,
                                     const ulonglong4* table, uint64_t cap)
{
    uint64_t cnt = 0, bs = 0, ps = 0, ec = 0, es = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        longlong2 t = __ldcs(&S[i]);
        uint64_t k = (uint64_t)t.x;
        if (k == kEmptyKey) {
            ++ec;
            es += (uint64_t)t.y;
            continue;
        }
        uint64_t s = reduce_range(mix64(k), cap);
        for (uint64_t steps = 0; steps < cap; ++steps) {
            ulonglong4 e = table[s];
            if (e.x == k) {
                cnt += e.z;
                bs += e.y;
                ps += e.z * (uint64_t)t.y;
                break;
            }
            if (e.x == kEmptyKey) break;
            s = (s + 1 == cap) ? 0 : s + 1;
        }
    }
    cnt = warp_sum_u64(cnt);
    bs = warp_sum_u64(bs);
    ps = warp_sum_u64(ps);
    ec = warp_sum_u64(ec);
    es = warp_sum_u64(es);
    if ((threadIdx.x & 31) == 0) {
        if (cnt) atomicAdd(&head[0], (unsigned long long)cnt);
        if (bs) atomicAdd(&head[1], (unsigned long long)bs);
        if (ps) atomicAdd(&head[2], (unsigned long long)ps);
        if (ec) atomicAdd(&head[5], (unsigned long long)ec);
        if (es) atomicAdd(&head[6], (unsigned long long)es);
    }
}

// Empty-marker keys join among themselves; write the caller's output.
__global__ void noalloc_finish_kernel(const unsigned long long* head, int64_t* out)
{
    uint64_t bc = head[3], bsum = head[4], pc = head[5], psum = head[6];
    out[0] = (int64_t)(head[0] + bc * pc);
    out[1] = (int64_t)(head[1] + bsum * pc);
    out[2] = (int64_t)(head[2] + bc * psum);
}

// Device address of the scratch array, looked up once per device (with that
// device current).  A device reset unloads the module that holds the array,
// so the cached address is only valid until then: reload the library after
// cudaDeviceReset.
static std::mutex g_noalloc_mu;
static void* g_noalloc_addr[64];

static int noalloc_scratch(int device, void** out)
{
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (device < 0 || device >= 64) {
        set_error("pyg_hashjoin_agg_noalloc: device %d out of range", device);
        return PYG_ERR_ARG;
    }
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(noalloc scratch)");
        g_noalloc_addr[device] = p;
    }
    *out = g_noalloc_addr[device];
    return PYG_OK;
}

}  // namespace pyg

using namespace pyg;

extern "C" int pyg_hashjoin_agg_noalloc(const void* build, int64_t nbuild, const void* probe, int64_t nprobe,
                                        int64_t* out_dev, void* stream)
{
    if (nbuild < 0 || nprobe < 0 || !out_dev || (nbuild > 0 && !build) || (nprobe > 0 && !probe) ||
        ((uintptr_t)build % 16) || ((uintptr_t)probe % 16) || ((uintptr_t)out_dev % 8)) {
        set_error("pyg_hashjoin_agg_noalloc: bad arguments (16-byte aligned device tuples, 8-byte aligned output)");
        return PYG_ERR_ARG;
    }
    if (nbuild > PYG_NOALLOC_MAX_BUILD) {
        set_error("pyg_hashjoin_agg_noalloc: %lld build tuples exceed the fixed scratch limit of %d",
                  (long long)nbuild, PYG_NOALLOC_MAX_BUILD);
        return PYG_ERR_ARG;
    }
    // An error left pending by an earlier, unrelated call is reported as
    // such and left pending for its owner; the launch checks below then
    // only see errors of this call's own launches.
    cudaError_t pending = cudaPeekAtLastError();
    if (pending != cudaSuccess) {
        set_error("pyg_hashjoin_agg_noalloc: a CUDA error from an earlier call is pending: %s",
                  cudaGetErrorString(pending));
        return PYG_ERR_CUDA;
    }
    int device = 0;
    PYG_CUDA(cudaGetDevice(&device));
    void* scratch = nullptr;
    int rc = noalloc_scratch(device, &scratch);
    if (rc) return rc;
    unsigned long long* head = (unsigned long long*)scratch;
    ulonglong4* table = (ulonglong4*)((unsigned char*)scratch + kNoAllocHeader * 8);
    uint64_t cap = (uint64_t)(2 * nbuild) + 64;
    if (cap > kNoAllocSlots) cap = kNoAllocSlots;
    cudaStream_t s = (cudaStream_t)stream;
    const int threads = 256;
    // Grids are clamped in 64-bit arithmetic before narrowing to int.
    auto grid_of = [&](int64_t n, int64_t most) {
        const int64_t g = (n + threads - 1) / threads;
        return (int)(g < most ? g : most);
    };
    noalloc_clear_kernel<<<grid_of((int64_t)cap, 4096), threads, 0, s>>>(head, table, cap);
    PYG_CUDA(cudaGetLastError());
    if (nbuild > 0) {
        noalloc_build_kernel<<<grid_of(nbuild, 4096), threads, 0, s>>>((const longlong2*)build, nbuild, head, table,
                                                                        cap);
        PYG_CUDA(cudaGetLastError());
    }
    if (nprobe > 0) {
        noalloc_probe_kernel<<<grid_of(nprobe, 8192), threads, 0, s>>>((const longlong2*)probe, nprobe, head, table,
                                                                        cap);
        PYG_CUDA(cudaGetLastError());
    }
    noalloc_finish_kernel<<<1, 1, 0, s>>>(head, out_dev);
    PYG_CUDA(cudaGetLastError());
    return PYG_OK;
}
