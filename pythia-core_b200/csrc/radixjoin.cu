// Radix hash join + aggregation with shared-memory tables.
//
// Restates the reference's partitioned hash join (the `hashjoin` node over
// `partition` outputs, operators/hashjoin.cpp and operators/partition.cpp)
// for the 16-byte (int64 key, int64 payload) case, B200-first:
//
//   1. histogram  one read of each relation counts the top `fine_bits`
//                 bits of rj_hash(key) in a shared-memory histogram per CTA;
//                 the host turns the counts into exact partition offsets.
//   2. partition  one or two tile passes (coarse bits, then the remaining
//                 bits inside each coarse partition).  A CTA groups a
//                 2048-tuple tile by partition in shared memory and writes
//                 each group as one contiguous run; exact offsets mean no
//                 capacity slack and no overflow path.
//   3. join       a persistent kernel takes work items (a build partition,
//                 or a chunk of it, and a chunk of the matching probe
//                 partition) from a queue.  The CTA builds the partition's
//                 table in 192 KB of shared memory, then streams the probe
//                 chunk from HBM against it.  No grid-wide barrier: CTAs
//                 never wait for one another, and table lookups never leave
//                 the SM.
//
// Build keys equal to the table's empty marker (INT64_MIN) are counted on
// the side per work item: they all hash to one fine partition, as do the
// probe keys they match.

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

#include "pyg_internal.cuh"
#include "radixjoin.cuh"

namespace pyg {

#ifndef PYG_RJ_JOIN_THREADS
#define PYG_RJ_JOIN_THREADS 1024
#endif
#ifndef PYG_RJ_JOIN_BLOCKS
#define PYG_RJ_JOIN_BLOCKS 1
#endif
#ifndef PYG_RJ_TABLE_KB
#define PYG_RJ_TABLE_KB 192
#endif
#ifndef PYG_RJ_RCAP_PCT
#define PYG_RJ_RCAP_PCT 50
#endif
constexpr int RJ_JOIN_THREADS = PYG_RJ_JOIN_THREADS;
constexpr int RJ_JOIN_BLOCKS = PYG_RJ_JOIN_BLOCKS;  // join CTAs per SM
#ifndef PYG_RJ_PROBE_UNROLL
#define PYG_RJ_PROBE_UNROLL 4
#endif
constexpr int RJ_PROBE_UNROLL = PYG_RJ_PROBE_UNROLL;  // probe tuples in flight per thread
constexpr int RJ_TABLE_BYTES = PYG_RJ_TABLE_KB * 1024;
constexpr int RJ_SLOTS_UNIQUE = RJ_TABLE_BYTES / 16;   // {key, payload}
constexpr int RJ_SLOTS_COUNTED = RJ_TABLE_BYTES / 32;  // {key, payload sum, count, -}
// Build tuples per work item: at most this share of the table's slots.
constexpr unsigned RJ_RCAP_UNIQUE = RJ_SLOTS_UNIQUE * PYG_RJ_RCAP_PCT / 100;
constexpr unsigned RJ_RCAP_COUNTED = RJ_SLOTS_COUNTED * PYG_RJ_RCAP_PCT / 100;
constexpr int64_t RJ_SCHUNK = 1 << 16;                 // probe tuples per work item (at most)

// ---------------------------------------------------------------------------
// Join: persistent CTAs, one shared-memory table each (partitioning is in
// radixpart.cu).

struct RJItem {
    unsigned long long r0, s0;  // first build / probe tuple of the item
    unsigned rn, sn;            // build tuples (<= table capacity / 2), probe tuples
};

struct RJJoinArgs {
    const void* R;              // 16-byte tuples, or packed words when RP
    const void* S;              // 16-byte tuples, or packed words when SP
    const RJItem* items;
    long long nitems;
    unsigned* next;             // work queue head, zeroed
    int fine_bits;              // the table's slot uses the hash bits below these
    unsigned long long* acc;    // count, build sum, probe sum
    unsigned* dup;              // set when a build key repeats (UNIQUE)
    unsigned long long rk, rp;  // frame of packed build words: key = rk + low half, payload = rp + high half
    unsigned long long sk, sp;  // frame of packed probe words
};

// Tuple i of a partitioned relation as (key, payload).
template <bool PACKED>
__device__ __forceinline__ longlong2 rj_tuple(const void* base, unsigned long long i, unsigned long long kb,
                                              unsigned long long pb)
{
    if constexpr (PACKED) {
        const unsigned long long w = reinterpret_cast<const unsigned long long*>(base)[i];
        return make_longlong2((long long)(kb + (w & 0xFFFFFFFFULL)), (long long)(pb + (w >> 32)));
    } else {
        return reinterpret_cast<const longlong2*>(base)[i];
    }
}

// Streaming load of a probe element and its decoding.
template <bool PACKED>
struct RJProbeElem {
    using T = typename std::conditional<PACKED, unsigned long long, longlong2>::type;
    static __device__ __forceinline__ T load(const void* base, unsigned long long i)
    {
        return __ldcs(reinterpret_cast<const T*>(base) + i);
    }
    static __device__ __forceinline__ longlong2 decode(const T& e, unsigned long long kb, unsigned long long pb)
    {
        if constexpr (PACKED) return make_longlong2((long long)(kb + (e & 0xFFFFFFFFULL)), (long long)(pb + (e >> 32)));
        else return e;
    }
};

// Warms L2 with [p, p + bytes) (16-byte aligned start; bytes rounded down
// to a multiple of 16); no registers are held for it.
__device__ __forceinline__ void rj_prefetch_l2(const void* p, unsigned long long bytes)
{
    bytes &= ~15ULL;
    if (bytes == 0) return;
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"((unsigned long long)__cvta_generic_to_global(p)),
                 "r"((unsigned)bytes)
                 : "memory");
}

template <bool UNIQUE, bool RP, bool SP>
__global__ void __launch_bounds__(RJ_JOIN_THREADS, RJ_JOIN_BLOCKS) rj_join_kernel(RJJoinArgs a)
{
    extern __shared__ __align__(16) unsigned char rj_table[];
    constexpr unsigned TS = UNIQUE ? RJ_SLOTS_UNIQUE : RJ_SLOTS_COUNTED;
    // Probe elements in flight per thread: the same bytes for 8-byte words.
    constexpr int U = SP ? 2 * RJ_PROBE_UNROLL : RJ_PROBE_UNROLL;
    constexpr unsigned RB = RP ? 8 : 16, SB = SP ? 8 : 16;  // bytes per build / probe element
    using PE = RJProbeElem<SP>;
    __shared__ long long item_cur, item_next;
    __shared__ unsigned long long side_cnt, side_sum;
    ulonglong2* T2 = reinterpret_cast<ulonglong2*>(rj_table);  // UNIQUE slots
    ulonglong4* T4 = reinterpret_cast<ulonglong4*>(rj_table);  // counted slots
    uint64_t cnt = 0, bsum = 0, psum = 0;
    bool dup = false;
    // One item of look-ahead: while this CTA works on an item, the next
    // one is already claimed and its build partition (and the head of its
    // probe chunk) is being pulled into L2.
    if (threadIdx.x == 0) item_next = (long long)atomicAdd(a.next, 1u);
    for (;;) {
        __syncthreads();  // previous item done with the table and item slots
        if (threadIdx.x == 0) {
            item_cur = item_next;
            side_cnt = side_sum = 0;
            if (item_cur < a.nitems) {
                item_next = (long long)atomicAdd(a.next, 1u);
                if (item_next < a.nitems) {
                    const RJItem nx = a.items[item_next];
                    rj_prefetch_l2((const char*)a.R + nx.r0 * RB, (unsigned long long)nx.rn * RB);
                    rj_prefetch_l2((const char*)a.S + nx.s0 * SB, (unsigned long long)min(nx.sn, 4096u) * SB);
                }
            }
        }
        for (unsigned i = threadIdx.x; i < TS; i += RJ_JOIN_THREADS) {
            if constexpr (UNIQUE) T2[i] = make_ulonglong2(kEmptyKey, 0);
            else T4[i] = make_ulonglong4(kEmptyKey, 0, 0, 0);
        }
        __syncthreads();
        const long long it = item_cur;
        if (it >= a.nitems) break;
        const RJItem item = a.items[it];
        // Build: linear probing with 64-bit shared-memory CAS.  At most
        // TS / 2 tuples per item, so a free slot always exists.
        for (unsigned i = threadIdx.x; i < item.rn; i += RJ_JOIN_THREADS) {
            const longlong2 t = rj_tuple<RP>(a.R, item.r0 + i, a.rk, a.rp);
            const uint64_t k = (uint64_t)t.x;
            if (k == kEmptyKey) {
                atomicAdd(&side_cnt, 1ULL);
                atomicAdd(&side_sum, (unsigned long long)t.y);
                continue;
            }
            unsigned pos = rj_slot(k, a.fine_bits, TS);
            for (unsigned steps = 0; steps < TS; ++steps) {
                unsigned long long* key = UNIQUE ? &T2[pos].x : &T4[pos].x;
                const unsigned long long prev = atomicCAS(key, kEmptyKey, k);
                if (prev == kEmptyKey || prev == k) {
                    if constexpr (UNIQUE) {
                        if (prev == k) dup = true;
                        else T2[pos].y = (unsigned long long)t.y;  // the CAS owns the slot
                    } else {
                        atomicAdd(&T4[pos].y, (unsigned long long)t.y);
                        atomicAdd(&T4[pos].z, 1ULL);
                    }
                    break;
                }
                pos = pos + 1 == TS ? 0 : pos + 1;
            }
        }
        __syncthreads();
        const uint64_t scnt = side_cnt, ssum = side_sum;
        if (UNIQUE && scnt > 1) dup = true;
        // Probe: U independent streaming loads per thread, lookups in
        // shared memory.
        auto probe = [&](const longlong2 t) {
            const uint64_t k = (uint64_t)t.x;
            if (k == kEmptyKey) {
                cnt += scnt;
                bsum += ssum;
                psum += scnt * (uint64_t)t.y;
                return;
            }
            unsigned pos = rj_slot(k, a.fine_bits, TS);
            for (unsigned steps = 0; steps < TS; ++steps) {
                if constexpr (UNIQUE) {
                    const ulonglong2 e = T2[pos];
                    if (e.x == k) {
                        cnt += 1;
                        bsum += e.y;
                        psum += (uint64_t)t.y;
                        return;
                    }
                    if (e.x == kEmptyKey) return;
                } else {
                    const ulonglong4 e = T4[pos];
                    if (e.x == k) {
                        cnt += e.z;
                        bsum += e.y;
                        psum += e.z * (uint64_t)t.y;
                        return;
                    }
                    if (e.x == kEmptyKey) return;
                }
                pos = pos + 1 == TS ? 0 : pos + 1;
            }
        };
        const unsigned long long s0 = item.s0;
        const unsigned sn = item.sn;
        unsigned i = threadIdx.x;
        for (; i + (U - 1) * RJ_JOIN_THREADS < sn; i += U * RJ_JOIN_THREADS) {
            typename PE::T t[U];
#pragma unroll
            for (int u = 0; u < U; ++u) t[u] = PE::load(a.S, s0 + i + u * RJ_JOIN_THREADS);
#pragma unroll
            for (int u = 0; u < U; ++u) probe(PE::decode(t[u], a.sk, a.sp));
        }
        for (; i < sn; i += RJ_JOIN_THREADS) probe(PE::decode(PE::load(a.S, s0 + i), a.sk, a.sp));
    }
    cnt = warp_sum_u64(cnt);
    bsum = warp_sum_u64(bsum);
    psum = warp_sum_u64(psum);
    if ((threadIdx.x & 31) == 0 && (cnt | bsum | psum)) {
        atomicAdd(&a.acc[0], (unsigned long long)cnt);
        atomicAdd(&a.acc[1], (unsigned long long)bsum);
        atomicAdd(&a.acc[2], (unsigned long long)psum);
    }
    if (__any_sync(0xffffffffu, dup) && (threadIdx.x & 31) == 0) atomicOr(a.dup, 1u);
}

// ---------------------------------------------------------------------------
// Join of packed partitions that share one key frame.  The low halves of
// both relations' words are then comparable 32-bit key offsets, so a table
// slot is the build word itself (key offset, payload offset): 8 bytes, one
// 64-bit CAS to insert, one 64-bit shared load per probe, no key decoding,
// and a 32-bit slot hash.  Offsets never reach 2^32 - 1, so the all-ones
// word marks an empty slot.  Two 512-thread CTAs per SM, 96 KB tables of
// 12288 slots (a build chunk fills at most half).  Sums are kept over the
// payload offsets and rebased at the end: sum = count x base + sum of
// offsets, modulo 2^64.

#ifndef PYG_RJ32_TABLE_KB
#define PYG_RJ32_TABLE_KB 96
#endif
#ifndef PYG_RJ32_BLOCKS
#define PYG_RJ32_BLOCKS 2
#endif
constexpr int RJ32_THREADS = 512;
constexpr int RJ32_BLOCKS = PYG_RJ32_BLOCKS;  // CTAs per SM
constexpr int RJ32_TABLE_BYTES = PYG_RJ32_TABLE_KB * 1024;
constexpr unsigned RJ32_SLOTS = RJ32_TABLE_BYTES / 8;
constexpr unsigned RJ32_RCAP = RJ32_SLOTS / 2;
#ifndef PYG_RJ32_U
#define PYG_RJ32_U 8
#endif
#ifndef PYG_RJ32_PREFETCH
#define PYG_RJ32_PREFETCH 8192
#endif
constexpr int RJ32_U = PYG_RJ32_U;  // probe words in flight per thread
// Words of the next item's probe chunk pulled into L2 ahead of use.
constexpr unsigned RJ32_PREFETCH = PYG_RJ32_PREFETCH;
constexpr unsigned long long kEmptyWord = ~0ULL;

// Slot of a key offset: the MurmurHash3 32-bit finaliser, then
// multiply-high into the table.
__device__ __forceinline__ unsigned rj32_slot(unsigned off)
{
    off ^= off >> 16;
    off *= 0x85ebca6bu;
    off ^= off >> 13;
    off *= 0xc2b2ae35u;
    off ^= off >> 16;
    return __umulhi(off, RJ32_SLOTS);
}

__global__ void __launch_bounds__(RJ32_THREADS, RJ32_BLOCKS) rj_join32_kernel(RJJoinArgs a)
{
    extern __shared__ __align__(16) unsigned long long rj32_table[];
    __shared__ long long item_cur, item_next;
    const unsigned long long* Rw = reinterpret_cast<const unsigned long long*>(a.R);
    const unsigned long long* Sw = reinterpret_cast<const unsigned long long*>(a.S);
    uint64_t cnt = 0, bsum = 0, psum = 0;  // matches, build and probe payload offsets
    bool dup = false;
    if (threadIdx.x == 0) item_next = (long long)atomicAdd(a.next, 1u);
    for (;;) {
        __syncthreads();  // previous item done with the table and item slots
        if (threadIdx.x == 0) {
            item_cur = item_next;
            if (item_cur < a.nitems) {
                item_next = (long long)atomicAdd(a.next, 1u);
                if (item_next < a.nitems) {
                    const RJItem nx = a.items[item_next];
                    rj_prefetch_l2(Rw + nx.r0, (unsigned long long)nx.rn * 8);
                    rj_prefetch_l2(Sw + nx.s0, (unsigned long long)min(nx.sn, RJ32_PREFETCH) * 8);
                }
            }
        }
        ulonglong2* T2 = reinterpret_cast<ulonglong2*>(rj32_table);
        for (unsigned i = threadIdx.x; i < RJ32_SLOTS / 2; i += RJ32_THREADS)
            T2[i] = make_ulonglong2(kEmptyWord, kEmptyWord);
        __syncthreads();
        const long long it = item_cur;
        if (it >= a.nitems) break;
        const RJItem item = a.items[it];
        // Build: one 64-bit CAS per word; a chunk fills at most half the
        // table, so a free slot always exists.
        for (unsigned i = threadIdx.x; i < item.rn; i += RJ32_THREADS) {
            const unsigned long long w = Rw[item.r0 + i];
            const unsigned off = (unsigned)w;
            unsigned pos = rj32_slot(off);
            for (unsigned steps = 0; steps < RJ32_SLOTS; ++steps) {
                const unsigned long long prev = atomicCAS(&rj32_table[pos], kEmptyWord, w);
                if (prev == kEmptyWord) break;
                if ((unsigned)prev == off) {  // a repeated build key: the counted join takes over
                    dup = true;
                    break;
                }
                pos = pos + 1 == RJ32_SLOTS ? 0 : pos + 1;
            }
        }
        __syncthreads();
        auto probe = [&](const unsigned long long w) {
            const unsigned off = (unsigned)w;
            unsigned pos = rj32_slot(off);
            for (unsigned steps = 0; steps < RJ32_SLOTS; ++steps) {
                const unsigned long long e = rj32_table[pos];
                if ((unsigned)e == off) {
                    cnt += 1;
                    bsum += e >> 32;
                    psum += w >> 32;
                    return;
                }
                if (e == kEmptyWord) return;
                pos = pos + 1 == RJ32_SLOTS ? 0 : pos + 1;
            }
        };
        const unsigned long long* S = Sw + item.s0;
        const unsigned sn = item.sn;
        unsigned i = threadIdx.x;
        for (; i + (RJ32_U - 1) * RJ32_THREADS < sn; i += RJ32_U * RJ32_THREADS) {
            unsigned long long w[RJ32_U];
#pragma unroll
            for (int u = 0; u < RJ32_U; ++u) w[u] = __ldcs(&S[i + u * RJ32_THREADS]);
#pragma unroll
            for (int u = 0; u < RJ32_U; ++u) probe(w[u]);
        }
        for (; i < sn; i += RJ32_THREADS) probe(__ldcs(&S[i]));
    }
    uint64_t b = cnt * a.rp + bsum, p = cnt * a.sp + psum;
    cnt = warp_sum_u64(cnt);
    b = warp_sum_u64(b);
    p = warp_sum_u64(p);
    if ((threadIdx.x & 31) == 0 && (cnt | b | p)) {
        atomicAdd(&a.acc[0], (unsigned long long)cnt);
        atomicAdd(&a.acc[1], (unsigned long long)b);
        atomicAdd(&a.acc[2], (unsigned long long)p);
    }
    if (__any_sync(0xffffffffu, dup) && (threadIdx.x & 31) == 0) atomicOr(a.dup, 1u);
}

// ---------------------------------------------------------------------------
// Host driver.

namespace {

struct RJEvents {
    // 0 start, 1 histograms, 2 / 3 build / probe passes done, 4 join done,
    // 5 / 6 build first pass begins / ends, 7 / 8 the same for the probe side,
    // 9 the join kernel begins.
    static constexpr int N = 10;
    cudaEvent_t ev[N] = {};
    bool on = false;
    void start(pyg_ctx* ctx, bool enable)
    {
        on = enable;
        if (!on) return;
        for (auto& e : ev) cudaEventCreate(&e);
        cudaEventRecord(ev[0], ctx->stream);
    }
    void mark(pyg_ctx* ctx, int i)
    {
        if (on) cudaEventRecord(ev[i], ctx->stream);
    }
    float ms(int a, int b)
    {
        float m = 0.f;
        cudaEventElapsedTime(&m, ev[a], ev[b]);
        return m;
    }
    ~RJEvents()
    {
        if (on)
            for (auto& e : ev) cudaEventDestroy(e);
    }
};

// Work items: every (build chunk, probe chunk) pair of every fine partition
// with both sides non-empty.
void make_items(const std::vector<unsigned long long>& hr, const std::vector<unsigned long long>& hs,
                const std::vector<unsigned long long>& rs, const std::vector<unsigned long long>& ss, unsigned rcap,
                std::vector<RJItem>& items)
{
    items.clear();
    const size_t F = hr.size();
    for (size_t f = 0; f < F; ++f) {
        const unsigned long long rn = hr[f], sn = hs[f];
        if (!rn || !sn) continue;
        for (unsigned long long r = 0; r < rn; r += rcap)
            for (unsigned long long s = 0; s < sn; s += RJ_SCHUNK) {
                RJItem it;
                it.r0 = rs[f] + r;
                it.s0 = ss[f] + s;
                it.rn = (unsigned)std::min<unsigned long long>(rcap, rn - r);
                it.sn = (unsigned)std::min<unsigned long long>(RJ_SCHUNK, sn - s);
                items.push_back(it);
            }
    }
}

// The join kernel for the partitions' formats (16-byte tuples or packed
// words on each side) and table kind.
template <bool UNIQUE>
void* join_fn(bool rp, bool sp)
{
    if (rp) return sp ? (void*)rj_join_kernel<UNIQUE, true, true> : (void*)rj_join_kernel<UNIQUE, true, false>;
    return sp ? (void*)rj_join_kernel<UNIQUE, false, true> : (void*)rj_join_kernel<UNIQUE, false, false>;
}

}  // namespace

int radix_join16(pyg_ctx* ctx, const void* Rv, int64_t nR, const void* Sv, int64_t nS, int fine_bits,
                 unsigned long long out[3], pyg_join_stats* stats)
{
    const longlong2* R = (const longlong2*)Rv;
    const longlong2* S = (const longlong2*)Sv;
    out[0] = out[1] = out[2] = 0;
    if (fine_bits <= 0) {
        // Partitions of about 0.7 x the table's build capacity.
        fine_bits = 1;
        while (fine_bits < RJ_MAX_FINE_BITS && (double)nR / (double)(1 << fine_bits) > 0.7 * RJ_RCAP_UNIQUE)
            ++fine_bits;
    }
    if (fine_bits < 1 || fine_bits > RJ_MAX_FINE_BITS) {
        set_error("pyg_hashjoin_agg: radix bits must be in [1, %d]", RJ_MAX_FINE_BITS);
        return PYG_ERR_ARG;
    }
    const int FB = fine_bits;
    const bool two = FB > RJ_MAX_LOCAL_BITS;
    const int F = 1 << FB;
    if (stats) {
        stats->algorithm = PYG_JOIN_RADIX;
        stats->radix_bits = FB;
    }
    if (nR == 0 || nS == 0) return PYG_OK;

    RJEvents tm;
    tm.start(ctx, stats != nullptr);
    void *R1 = nullptr, *R2 = nullptr, *S1 = nullptr, *S2 = nullptr;
    RJItem* ditems = nullptr;
    int rc = PYG_OK;
    do {
        // Words 224-227: per relation, [0] a bulk copy never landed, [1]
        // region overflow, [2] a tuple outside the packed frame, [3] unused.
        unsigned* flags = (unsigned*)(ctx->dcounters + 224);
        unsigned long long* h = (unsigned long long*)ctx->pinned;
        unsigned* hflags = (unsigned*)(h + 6);
        // 1-2. Partition both sides (histograms sampled for large inputs;
        // intermediates packed when the key and payload ranges allow).
        RPSide side[2];
        for (int s = 0; s < 2; ++s) {
            side[s].in = s ? S : R;
            side[s].n = s ? nS : nR;
            side[s].allow_pack = true;
            side[s].begin = tm.on ? tm.ev[5 + 2 * s] : nullptr;
            side[s].mid = tm.on ? tm.ev[6 + 2 * s] : nullptr;
            side[s].done = tm.on ? tm.ev[2 + s] : nullptr;
        }
        rc = rp_partition_sides(ctx, side, 2, FB, two, flags, hflags, tm.on ? tm.ev[1] : nullptr, true);
        R1 = side[0].P1;
        R2 = side[0].P2;
        S1 = side[1].P1;
        S2 = side[1].P2;
        if (rc) break;
        const RJLayout& LR = side[0].L;
        const RJLayout& LS = side[1].L;

        // 3. Join: distinct build keys first (16-byte slots); on a repeated
        // key, again with counted 32-byte slots and smaller build chunks.
        unsigned long long* acc = ctx->dcounters + 8;
        unsigned* next = (unsigned*)(ctx->dcounters + 200);  // word 200: queue head, word 201: dup flag
        unsigned* dupf = (unsigned*)(ctx->dcounters + 201);
        std::vector<unsigned long long> rstart(LR.fstart.begin(), LR.fstart.begin() + F);
        std::vector<unsigned long long> sstart(LS.fstart.begin(), LS.fstart.begin() + F);
        std::vector<RJItem> items;
        // Both relations packed in one key frame: the 32-bit-offset join
        // (distinct build keys; a repeated key falls back to the counted
        // join below, which decodes the words).
        const bool same_frame = LR.packed && LS.packed && LR.kbase == LS.kbase;
        for (int pass = 0; pass < 2; ++pass) {
            const bool unique = pass == 0;
            const bool j32 = unique && same_frame;
            make_items(LR.count, LS.count, rstart, sstart,
                       j32 ? RJ32_RCAP : (unique ? RJ_RCAP_UNIQUE : RJ_RCAP_COUNTED), items);
            if (items.empty()) break;
            dfree(ctx, ditems);
            ditems = nullptr;
            if ((rc = dalloc(ctx, (void**)&ditems, items.size() * sizeof(RJItem)))) break;
            if ((rc = stage_h2d(ctx, ditems, items.data(), items.size() * sizeof(RJItem)))) break;
            void* fn = j32 ? (void*)rj_join32_kernel
                           : (unique ? join_fn<true>(LR.packed, LS.packed) : join_fn<false>(LR.packed, LS.packed));
            const int smem = j32 ? RJ32_TABLE_BYTES : RJ_TABLE_BYTES;
            const int threads = j32 ? RJ32_THREADS : RJ_JOIN_THREADS;
            const int per_sm = j32 ? RJ32_BLOCKS : RJ_JOIN_BLOCKS;
            PYG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            PYG_CUDA(cudaMemsetAsync(acc, 0, 3 * 8, ctx->stream));
            PYG_CUDA(cudaMemsetAsync(next, 0, 16, ctx->stream));
            RJJoinArgs ja;
            ja.R = two ? R2 : R1;
            ja.S = two ? S2 : S1;
            ja.items = ditems;
            ja.nitems = (long long)items.size();
            ja.next = next;
            ja.fine_bits = FB;
            ja.acc = acc;
            ja.dup = dupf;
            ja.rk = LR.kbase;
            ja.rp = LR.pbase;
            ja.sk = LS.kbase;
            ja.sp = LS.pbase;
            const unsigned grid = (unsigned)std::min<long long>((long long)ctx->sm_count * per_sm, ja.nitems);
            if (unique) tm.mark(ctx, 9);
            void* args[] = {&ja};
            PYG_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(threads), args, smem, ctx->stream));
            PYG_LAUNCHED(ctx);
            PYG_CUDA(cudaMemcpyAsync(h, acc, 3 * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(h + 3, next, 16, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            out[0] = h[0];
            out[1] = h[1];
            out[2] = h[2];
            if (!unique || (unsigned)h[4] == 0) break;
        }
        if (rc) break;
        tm.mark(ctx, 4);
        if (stats) {
            cudaEventSynchronize(tm.ev[4]);
            // Histograms of both relations, then the build side's passes
            // (after the host round trip that lays out both), then the
            // probe side's passes.
            stats->histogram_ms = tm.ms(0, 1);
            stats->histogram_tuples = side[0].hist_tuples + side[1].hist_tuples;
            stats->build_partition_ms = tm.ms(1, 2);
            stats->build_ms = 0;
            stats->probe_partition_ms = tm.ms(2, 3);
            stats->probe_ms = tm.ms(3, 4);
            stats->join_kernel_ms = tm.ms(9, 4);
            for (int s = 0; s < 2; ++s) {
                double* pm = s ? stats->probe_pass_ms : stats->build_pass_ms;
                pm[0] = pm[1] = 0;
                if (!side[s].begin) continue;  // the relation was redone: no per-pass times
                if (two) {
                    pm[0] = tm.ms(5 + 2 * s, 6 + 2 * s);
                    pm[1] = tm.ms(6 + 2 * s, 2 + s);
                } else {
                    pm[0] = tm.ms(5 + 2 * s, 2 + s);
                }
            }
            stats->build_packed = LR.packed ? 1 : 0;
            stats->probe_packed = LS.packed ? 1 : 0;
            stats->padded_tuples = (int64_t)((LR.p2 + LS.p2) - (unsigned long long)(nR + nS));
            stats->overflow_tuples = (side[0].overflowed ? 1 : 0) + (side[1].overflowed ? 1 : 0);
        }
    } while (0);
    dfree(ctx, ditems);
    dfree(ctx, R1);
    dfree(ctx, R2);
    dfree(ctx, S1);
    dfree(ctx, S2);
    return rc;
}

}  // namespace pyg
