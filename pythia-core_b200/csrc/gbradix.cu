// Group-by (sum and/or count) of 16-byte (int64 key, int64 value) device
// tuples, aggregated in shared memory.
//
// Same result table as the generic group-by kernel (groupby.cu): 32-byte
// slots {key, sum, count, -} in HBM plus the flags {full, groups, sum and
// count of the INT64_MIN key}; compaction and ordering by key are shared.
// What differs is how the table is filled:
//
//   very few     (expected <= GBR_TINY_GROUPS) every warp folds into its own
//                128-slot table, so atomics of different warps never meet.
//   few groups   (expected <= GBR_DIRECT_GROUPS) every CTA folds its slice
//                of the input into a 160 KB shared-memory table and flushes
//                it once: one HBM read of the input, G atomics per CTA.
//   many groups  the input is hash-partitioned (radixpart.cu) into
//                partitions of about GBR_PART_GROUPS distinct keys; a
//                persistent CTA folds each partition chunk into its shared
//                table and flushes it.  Traffic: the partition passes plus
//                one read.
//
// A key that does not fit a full shared table goes straight to the HBM
// table, so the result never depends on the group estimate being right.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "gbradix.cuh"
#include "radixpart.cuh"

namespace pyg {

constexpr int GBR_THREADS = 1024;
constexpr unsigned GBR_SLOTS = 8192;            // shared table: keys (8 B), sums (8 B), counts (4 B)
constexpr int GBR_SMEM = GBR_SLOTS * 20;        // 160 KB
constexpr int64_t GBR_DIRECT_GROUPS = 3072;     // fold without partitioning up to this many groups
constexpr int64_t GBR_PART_GROUPS = 2048;       // distinct keys per partition when partitioned
constexpr uint64_t GBR_PROBE_LIMIT = 4096;      // HBM table probe limit (then "full")
constexpr int64_t GBR_CHUNK = (int64_t)1 << 22; // tuples per work item (partitioned mode)
constexpr int64_t GBR_COMBINE_GROUPS = 256;   // few-groups mode combines lanes up to this many groups

struct GbrArgs {
    const longlong2* in;
    int64_t n;                   // direct mode: the input; partitioned: unused
    const unsigned long long* item_start;  // partitioned: first tuple of each item
    const unsigned* item_len;              // partitioned: tuples of each item
    long long nitems;
    unsigned* next;              // work queue head (partitioned)
    int fine_bits;               // slot bits below the partition bits (0 in direct mode)
    int want_sum;
    ulonglong4* table;           // HBM result table
    uint64_t cap;
    unsigned long long* flags;   // [0] full, [1] groups, [2] INT64_MIN sum, [3] INT64_MIN count
};

// Adds (sum, cnt) for key k to the HBM table; false if the probe limit was hit.
__device__ __forceinline__ bool gbr_global_add(const GbrArgs& a, uint64_t k, uint64_t sum, uint64_t cnt,
                                               unsigned long long& fresh)
{
    uint64_t s = reduce_range(mix64(k), a.cap);
    for (uint64_t steps = 0; steps < GBR_PROBE_LIMIT && steps < a.cap; ++steps) {
        unsigned long long* slot = (unsigned long long*)&a.table[s];
        unsigned long long prev = slot[0];
        if (prev == kEmptyKey) {
            prev = atomicCAS(slot, kEmptyKey, k);
            if (prev == kEmptyKey) ++fresh;
        }
        if (prev == kEmptyKey || prev == k) {
            if (a.want_sum) atomicAdd(slot + 1, (unsigned long long)sum);
            atomicAdd(slot + 2, (unsigned long long)cnt);
            return true;
        }
        s = (s + 1 == a.cap) ? 0 : s + 1;
    }
    return false;
}

struct GbrTable {
    unsigned long long* key;
    unsigned long long* sum;
    unsigned* cnt;
};

// Folds one tuple into the shared table; false if the table is full.
__device__ __forceinline__ bool gbr_fold(const GbrTable& t, uint64_t k, uint64_t v, int want_sum, int fb)
{
    unsigned pos = rj_slot(k, fb, GBR_SLOTS);
    for (unsigned steps = 0; steps < GBR_SLOTS; ++steps) {
        unsigned long long prev = t.key[pos];
        if (prev == kEmptyKey) prev = atomicCAS(&t.key[pos], kEmptyKey, (unsigned long long)k);
        if (prev == kEmptyKey || prev == k) {
            if (want_sum) atomicAdd(&t.sum[pos], (unsigned long long)v);
            atomicAdd(&t.cnt[pos], 1u);
            return true;
        }
        pos = pos + 1 == GBR_SLOTS ? 0 : pos + 1;
    }
    return false;
}

// Folds (sum, cnt) for key k into the shared table, else into the HBM
// table; false if both are full.
__device__ __forceinline__ bool gbr_fold_n(const GbrArgs& a, const GbrTable& t, uint64_t k, uint64_t sum, unsigned cnt,
                                           unsigned long long& fresh)
{
    unsigned pos = rj_slot(k, a.fine_bits, GBR_SLOTS);
    for (unsigned steps = 0; steps < GBR_SLOTS; ++steps) {
        unsigned long long prev = t.key[pos];
        if (prev == kEmptyKey) prev = atomicCAS(&t.key[pos], kEmptyKey, (unsigned long long)k);
        if (prev == kEmptyKey || prev == k) {
            if (a.want_sum) atomicAdd(&t.sum[pos], (unsigned long long)sum);
            atomicAdd(&t.cnt[pos], cnt);
            return true;
        }
        pos = pos + 1 == GBR_SLOTS ? 0 : pos + 1;
    }
    return gbr_global_add(a, k, sum, cnt, fresh);
}

// Folds tuples [0, n) of p into the shared table.
// Lane combining in gbr_fold_range: never, always, or adaptive (a warp
// stops combining after four batches in a row whose rounds found no key
// group of three or more lanes, and tries again 64 batches later).
enum GbrFold { kFoldPlain = 0, kFoldCombine = 1, kFoldAdaptive = 2 };

template <int MODE>
__device__ void gbr_fold_range(const GbrArgs& a, const GbrTable& t, const longlong2* __restrict__ p, int64_t n,
                               uint64_t& sent_sum, uint64_t& sent_cnt, unsigned long long& fresh, bool& full)
{
    constexpr int U = MODE == kFoldPlain ? 8 : 4;
    const int lane = threadIdx.x & 31;
    bool comb = MODE != kFoldPlain, hit = false;
    int cool = 0, miss = 0;
    // The warp's hot key: combined groups of it are added to these
    // registers (the same values in every lane) instead of the shared
    // table, where every warp's groups of that key would meet on one slot;
    // they are folded in when another key of a large group takes its
    // place, and at the end.
    uint64_t hot_k = kEmptyKey, hot_s = 0;
    unsigned hot_c = 0;
    // While combining, the lanes holding the key of a leader lane are combined
    // with one shuffle reduction and folded once, for up to two leaders per
    // warp; each round takes the larger key group of two candidates (the
    // lowest and the highest unplaced lanes).  Hot keys (skew, very few
    // groups) cost one shared atomic per warp instead of one per lane.
    auto one = [&](const longlong2 x, bool valid) {
        const uint64_t k = (uint64_t)x.x, v = (uint64_t)x.y;
        if (valid && k == kEmptyKey) {
            sent_sum += v;
            sent_cnt += 1;
        }
        unsigned rem = __ballot_sync(0xffffffffu, valid && k != kEmptyKey);
#pragma unroll
        for (int r = 0; r < (MODE != kFoldPlain ? 2 : 0); ++r) {
            if (!comb || !rem) break;
            // Two candidate leaders, the lowest and the highest unplaced
            // lanes; the larger of their key groups is combined.
            const int la = __ffs(rem) - 1, lb = 31 - __clz(rem);
            const uint64_t ka = __shfl_sync(0xffffffffu, k, la), kb = __shfl_sync(0xffffffffu, k, lb);
            const unsigned ma = __ballot_sync(0xffffffffu, ((rem >> lane) & 1) && k == ka);
            const unsigned mb = __ballot_sync(0xffffffffu, ((rem >> lane) & 1) && k == kb);
            const bool pa = __popc(ma) >= __popc(mb);
            const unsigned m = pa ? ma : mb;
            const int leader = pa ? la : lb;
            const uint64_t kl = pa ? ka : kb;
            const int c = __popc(m);
            if (c < 3) break;
            hit = true;
            uint64_t sv = ((m >> lane) & 1) ? v : 0;
#pragma unroll
            for (int o = 16; o; o >>= 1) sv += __shfl_xor_sync(0xffffffffu, sv, o);
            if (kl == hot_k) {
                hot_s += sv;
                hot_c += (unsigned)c;
            } else if (c >= 8) {
                // A large group: its key becomes the warp's hot key.
                if (lane == leader && hot_c && !gbr_fold_n(a, t, hot_k, hot_s, hot_c, fresh)) full = true;
                hot_k = kl;
                hot_s = sv;
                hot_c = (unsigned)c;
            } else if (lane == leader && !gbr_fold_n(a, t, kl, sv, (unsigned)c, fresh)) {
                full = true;
            }
            rem &= ~m;
        }
        if ((rem >> lane) & 1) {
            if (!gbr_fold(t, k, v, a.want_sum, a.fine_bits) && !gbr_global_add(a, k, v, 1, fresh)) full = true;
        }
    };
    // Loop bounds are uniform across each warp (the whole-warp test in
    // `one` needs all 32 lanes): wb is the warp's first position.
    int64_t wb = (int64_t)(threadIdx.x - lane);
    for (; wb + 31 + (int64_t)(U - 1) * GBR_THREADS < n; wb += (int64_t)U * GBR_THREADS) {
        longlong2 x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) x[u] = __ldcs(&p[wb + lane + (int64_t)u * GBR_THREADS]);
#pragma unroll
        for (int u = 0; u < U; ++u) one(x[u], true);
        if (MODE == kFoldAdaptive) {
            if (comb) {
                miss = hit ? 0 : miss + 1;
                hit = false;
                if (miss == 4) {
                    comb = false;
                    miss = 0;
                    cool = 64;
                }
            } else if (--cool == 0) {
                comb = true;
            }
        }
    }
    for (; wb < n; wb += GBR_THREADS) {
        const int64_t j = wb + lane;
        const bool valid = j < n;
        one(valid ? __ldcs(&p[j]) : make_longlong2((long long)kEmptyKey, 0), valid);
    }
    if (lane == 0 && hot_c && !gbr_fold_n(a, t, hot_k, hot_s, hot_c, fresh)) full = true;
}

__device__ void gbr_clear(const GbrTable& t)
{
    for (unsigned s = threadIdx.x; s < GBR_SLOTS; s += GBR_THREADS) {
        t.key[s] = kEmptyKey;
        t.sum[s] = 0;
        t.cnt[s] = 0;
    }
}

__device__ void gbr_flush(const GbrArgs& a, const GbrTable& t, unsigned long long& fresh, bool& full)
{
    for (unsigned s = threadIdx.x; s < GBR_SLOTS; s += GBR_THREADS) {
        const uint64_t k = t.key[s];
        if (k != kEmptyKey && !gbr_global_add(a, k, t.sum[s], t.cnt[s], fresh)) full = true;
    }
}

__device__ void gbr_finish(const GbrArgs& a, uint64_t sent_sum, uint64_t sent_cnt, unsigned long long fresh, bool full)
{
    sent_sum = warp_sum_u64(sent_sum);
    sent_cnt = warp_sum_u64(sent_cnt);
    fresh = warp_sum_u64(fresh);
    const bool anyfull = __any_sync(0xffffffffu, full);
    if ((threadIdx.x & 31) == 0) {
        if (sent_cnt) {
            atomicAdd(&a.flags[2], (unsigned long long)sent_sum);
            atomicAdd(&a.flags[3], (unsigned long long)sent_cnt);
        }
        if (fresh) atomicAdd(&a.flags[1], fresh);
        if (anyfull) a.flags[0] = 1;
    }
}

// Few groups: CTA b folds the b-th slice of the input, then flushes once.
template <int MODE>
__global__ void __launch_bounds__(GBR_THREADS, 1) gbr_direct_kernel(GbrArgs a)
{
    extern __shared__ __align__(16) unsigned char gbr_smem[];
    GbrTable t{(unsigned long long*)gbr_smem, (unsigned long long*)gbr_smem + GBR_SLOTS,
               (unsigned*)((unsigned long long*)gbr_smem + 2 * GBR_SLOTS)};
    gbr_clear(t);
    __syncthreads();
    uint64_t sent_sum = 0, sent_cnt = 0;
    unsigned long long fresh = 0;
    bool full = false;
    const int64_t per = (a.n + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = (int64_t)blockIdx.x * per;
    const int64_t b1 = min(a.n, b0 + per);
    if (b0 < b1) gbr_fold_range<MODE>(a, t, a.in + b0, b1 - b0, sent_sum, sent_cnt, fresh, full);
    __syncthreads();
    gbr_flush(a, t, fresh, full);
    gbr_finish(a, sent_sum, sent_cnt, fresh, full);
}

// Very few groups: every warp folds into its own 128-slot table, so the
// shared atomics of different warps never meet on one address.  The 32
// warp tables are flushed at the end.
constexpr int GBR_TINY_SLOTS = 128;
constexpr int64_t GBR_TINY_GROUPS = 64;

__global__ void __launch_bounds__(GBR_THREADS, 1) gbr_tiny_kernel(GbrArgs a)
{
    extern __shared__ __align__(16) unsigned char gbr_smem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int NW = GBR_THREADS / 32;
    unsigned long long* keys = (unsigned long long*)gbr_smem + w * GBR_TINY_SLOTS;
    unsigned long long* sums = (unsigned long long*)gbr_smem + NW * GBR_TINY_SLOTS + w * GBR_TINY_SLOTS;
    unsigned* cnts = (unsigned*)((unsigned long long*)gbr_smem + 2 * NW * GBR_TINY_SLOTS) + w * GBR_TINY_SLOTS;
    for (int i = lane; i < GBR_TINY_SLOTS; i += 32) {
        keys[i] = kEmptyKey;
        sums[i] = 0;
        cnts[i] = 0;
    }
    __syncwarp();
    uint64_t sent_sum = 0, sent_cnt = 0;
    unsigned long long fresh = 0;
    bool full = false;
    const int64_t per = (a.n + gridDim.x - 1) / gridDim.x;
    const int64_t b0 = (int64_t)blockIdx.x * per;
    const int64_t b1 = min(a.n, b0 + per);
    // Every lane adds its tuple with shared atomics, but only into its own
    // warp's table, so atomics of different warps never meet.  (Combining
    // the lanes that hold a leader lane's key first, by a shuffle reduction,
    // measured slower at every shape tried: 2^28 tuples, G = 16 2.23 against
    // 1.38 ms, G = 64 1.48 against 1.32 ms, Zipf(1.0) ids 2.69 against 1.95 ms.)
    auto add = [&](uint64_t k, uint64_t s, unsigned c) {
        unsigned pos = rj_slot(k, 0, GBR_TINY_SLOTS);
        for (int steps = 0; steps < GBR_TINY_SLOTS; ++steps) {
            unsigned long long prev = keys[pos];
            if (prev == kEmptyKey) prev = atomicCAS(&keys[pos], kEmptyKey, (unsigned long long)k);
            if (prev == kEmptyKey || prev == k) {
                if (a.want_sum) atomicAdd(&sums[pos], (unsigned long long)s);
                atomicAdd(&cnts[pos], c);
                return;
            }
            pos = (pos + 1) & (GBR_TINY_SLOTS - 1);
        }
        if (!gbr_global_add(a, k, s, c, fresh)) full = true;
    };
    auto one = [&](const longlong2 x, bool valid) {
        const uint64_t k = (uint64_t)x.x, v = (uint64_t)x.y;
        if (!valid) return;
        if (k == kEmptyKey) {
            sent_sum += v;
            sent_cnt += 1;
        } else {
            add(k, v, 1u);
        }
    };
    int64_t wb = b0 + w * 32;
    constexpr int U = 4;
    for (; wb + 31 + (int64_t)(U - 1) * GBR_THREADS < b1; wb += (int64_t)U * GBR_THREADS) {
        longlong2 x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) x[u] = __ldcs(&a.in[wb + lane + (int64_t)u * GBR_THREADS]);
#pragma unroll
        for (int u = 0; u < U; ++u) one(x[u], true);
    }
    for (; wb < b1; wb += GBR_THREADS) {
        const int64_t j = wb + lane;
        const bool valid = j < b1;
        one(valid ? __ldcs(&a.in[j]) : make_longlong2((long long)kEmptyKey, 0), valid);
    }
    __syncwarp();
    for (int i = lane; i < GBR_TINY_SLOTS; i += 32) {
        const uint64_t k = keys[i];
        if (k != kEmptyKey && !gbr_global_add(a, k, sums[i], cnts[i], fresh)) full = true;
    }
    gbr_finish(a, sent_sum, sent_cnt, fresh, full);
}

// Many groups: persistent CTAs claim (partition chunk) items.
__global__ void __launch_bounds__(GBR_THREADS, 1) gbr_part_kernel(GbrArgs a)
{
    extern __shared__ __align__(16) unsigned char gbr_smem[];
    GbrTable t{(unsigned long long*)gbr_smem, (unsigned long long*)gbr_smem + GBR_SLOTS,
               (unsigned*)((unsigned long long*)gbr_smem + 2 * GBR_SLOTS)};
    __shared__ long long item;
    uint64_t sent_sum = 0, sent_cnt = 0;
    unsigned long long fresh = 0;
    bool full = false;
    for (;;) {
        if (threadIdx.x == 0) item = (long long)atomicAdd(a.next, 1u);
        gbr_clear(t);
        __syncthreads();
        const long long it = item;
        if (it >= a.nitems) break;
        // Skew concentrates in partitions: warps combine lanes wherever they
        // find repeated keys.
        gbr_fold_range<kFoldAdaptive>(a, t, a.in + a.item_start[it], (int64_t)a.item_len[it], sent_sum, sent_cnt, fresh,
                                      full);
        __syncthreads();
        gbr_flush(a, t, fresh, full);
        __syncthreads();
    }
    gbr_finish(a, sent_sum, sent_cnt, fresh, full);
}

bool groupby16_eligible(int64_t expected_groups) { return expected_groups > 0; }

int groupby16_fill(pyg_ctx* ctx, const void* in, int64_t n, int want_sum, int64_t expected_groups, ulonglong4* table,
                   uint64_t cap, unsigned long long* flags)
{
    GbrArgs a;
    memset(&a, 0, sizeof(a));
    a.want_sum = want_sum;
    a.table = table;
    a.cap = cap;
    a.flags = flags;
    if (n <= 0) return PYG_OK;
    if (expected_groups <= GBR_DIRECT_GROUPS) {
        a.in = (const longlong2*)in;
        a.n = n;
        const int64_t want0 = (n + 64 * GBR_THREADS - 1) / (64 * GBR_THREADS);
        const int grid0 = (int)std::max<int64_t>(1, std::min<int64_t>(want0, ctx->sm_count));
        if (expected_groups <= GBR_TINY_GROUPS) {
            const int smem = (GBR_THREADS / 32) * GBR_TINY_SLOTS * 20;
            PYG_CUDA(cudaFuncSetAttribute(gbr_tiny_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            gbr_tiny_kernel<<<grid0, GBR_THREADS, smem, ctx->stream>>>(a);
            PYG_LAUNCHED(ctx);
            return PYG_OK;
        }
        const bool combine = expected_groups <= GBR_COMBINE_GROUPS;
        void* fn = combine ? (void*)gbr_direct_kernel<kFoldCombine> : (void*)gbr_direct_kernel<kFoldPlain>;
        PYG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, GBR_SMEM));
        const int64_t want = (n + 64 * GBR_THREADS - 1) / (64 * GBR_THREADS);
        const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, ctx->sm_count));
        if (combine) gbr_direct_kernel<kFoldCombine><<<grid, GBR_THREADS, GBR_SMEM, ctx->stream>>>(a);
        else gbr_direct_kernel<kFoldPlain><<<grid, GBR_THREADS, GBR_SMEM, ctx->stream>>>(a);
        PYG_LAUNCHED(ctx);
        return PYG_OK;
    }
    // Partition so that each partition holds about GBR_PART_GROUPS keys.
    int FB = 1;
    while (FB < RJ_MAX_FINE_BITS && (double)expected_groups / (double)(1 << FB) > (double)GBR_PART_GROUPS) ++FB;
    const bool two = FB > RJ_MAX_LOCAL_BITS;
    const int CB = two ? (FB + 1) / 2 : FB;
    const int F = 1 << FB, C = 1 << CB, sub = FB - CB;
    const bool sample = two && n >= ((int64_t)1 << 25);
    const int64_t step = sample ? std::max<int64_t>(1, n >> RJ_SAMPLE_LOG2) : 1;
    const longlong2* src = (const longlong2*)in;
    const size_t side = RJSideDev::words(F, C);
    unsigned long long* meta = nullptr;
    void *P1 = nullptr, *P2 = nullptr;
    unsigned long long* dstart = nullptr;
    int rc = PYG_OK;
    do {
        if ((rc = dalloc(ctx, (void**)&meta, (side + F) * 8))) break;
        RJSideDev d;
        d.carve(meta, F, C);
        unsigned long long* hist = meta + side;
        unsigned* pflags = (unsigned*)(ctx->dcounters + 204);  // [0] a bulk copy never landed, [1] overflow
        PYG_CUDA(cudaMemsetAsync(pflags, 0, 8, ctx->stream));
        if ((rc = hist_launch(ctx, src, n, step, FB, hist))) break;
        std::vector<unsigned long long> h(F);
        PYG_CUDA(cudaMemcpyAsync(h.data(), hist, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        RJLayout L;
        if (sample) layout_sampled(h, step, C, sub, L);
        else layout_exact(h, C, sub, L);
        unsigned* hp = (unsigned*)ctx->pinned + 64;
        for (int attempt = 0; attempt < 2; ++attempt) {
            if ((rc = upload_layout(ctx, L, d, F, C, n))) break;
            dfree(ctx, P1);
            dfree(ctx, P2);
            P1 = P2 = nullptr;
            if ((rc = dalloc(ctx, &P1, (size_t)L.p1 * 16))) break;
            if (two && (rc = dalloc(ctx, &P2, (size_t)L.p2 * 16))) break;
            if ((rc = run_passes(ctx, src, n, L, d, two, FB, CB, P1, P2, pflags, pflags + 1))) break;
            PYG_CUDA(cudaMemcpyAsync(hp, pflags, 8, cudaMemcpyDeviceToHost, ctx->stream));
            if (L.sampled) {
                L.count.resize(F);
                PYG_CUDA(cudaMemcpyAsync(L.count.data(), d.cur2, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
            }
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            if (hp[0]) {
                set_error("pyg_groupby: a partition tile copy did not complete in time");
                rc = PYG_ERR_TIMEOUT;
                break;
            }
            if (!hp[1]) break;
            // A sampled region overflowed: redo from an exact histogram.
            if ((rc = hist_launch(ctx, src, n, 1, FB, hist))) break;
            PYG_CUDA(cudaMemcpyAsync(h.data(), hist, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            layout_exact(h, C, sub, L);
            PYG_CUDA(cudaMemsetAsync(pflags, 0, 8, ctx->stream));
        }
        if (rc) break;
        // Work items: chunks of each partition, small enough for about four
        // items per SM (each chunk costs one flush of its distinct keys).
        const unsigned long long chunk = (unsigned long long)std::max<int64_t>(
            (int64_t)1 << 16, std::min<int64_t>(GBR_CHUNK, n / (4 * (int64_t)ctx->sm_count) + 1));
        std::vector<unsigned long long> istart;
        std::vector<unsigned> ilen;
        for (int f = 0; f < F; ++f)
            for (unsigned long long o = 0; o < L.count[f]; o += chunk) {
                istart.push_back(L.fstart[f] + o);
                ilen.push_back((unsigned)std::min<unsigned long long>(chunk, L.count[f] - o));
            }
        if (istart.empty()) break;
        const size_t ni = istart.size();
        if ((rc = dalloc(ctx, (void**)&dstart, ni * 12 + 16))) break;
        unsigned* dlen = (unsigned*)(dstart + ni);
        if ((rc = stage_h2d(ctx, dstart, istart.data(), ni * 8)) || (rc = stage_h2d(ctx, dlen, ilen.data(), ni * 4))) break;
        unsigned* next = (unsigned*)(ctx->dcounters + 206);
        PYG_CUDA(cudaMemsetAsync(next, 0, 8, ctx->stream));
        a.in = (const longlong2*)(two ? P2 : P1);
        a.item_start = dstart;
        a.item_len = dlen;
        a.nitems = (long long)ni;
        a.next = next;
        a.fine_bits = FB;
        PYG_CUDA(cudaFuncSetAttribute(gbr_part_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, GBR_SMEM));
        const unsigned grid = (unsigned)std::min<long long>((long long)ctx->sm_count, (long long)ni);
        gbr_part_kernel<<<grid, GBR_THREADS, GBR_SMEM, ctx->stream>>>(a);
        PYG_LAUNCHED(ctx);
    } while (0);
    // Stream-ordered frees: the kernels above finish before the memory is reused.
    dfree(ctx, dstart);
    dfree(ctx, P1);
    dfree(ctx, P2);
    dfree(ctx, meta);
    return rc;
}

}  // namespace pyg
