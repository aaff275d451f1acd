// Radix hash join + aggregation with shared-memory tables.
//
// Restates the reference's partitioned hash join (the `hashjoin` node over
// `partition` outputs, operators/hashjoin.cpp and operators/partition.cpp)
// for the 16-byte (int64 key, int64 payload) case, B200-first:
//
//   1. histogram  one read of each relation counts the top `fine_bits`
//                 bits of mix64(key) in a shared-memory histogram per CTA;
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
#include <vector>

#include "pyg_internal.cuh"
#include "radixjoin.cuh"
#include "bulk.cuh"

namespace pyg {

constexpr int RJ_TILE = 2048;        // tuples per partition tile
constexpr int RJ_PT_THREADS = 512;   // partition CTA
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
constexpr int RJ_MAX_LOCAL_BITS = 9;                   // bins of one partition pass
constexpr int RJ_LMAX = 1 << RJ_MAX_LOCAL_BITS;
#ifndef PYG_RJ_WARP_RANK
#define PYG_RJ_WARP_RANK 0
#endif
constexpr int RJ_STAGES = 2;                           // input tiles in flight per partition CTA
constexpr unsigned long long kBulkWaitNs = 2000000000ULL;  // 2 s

__device__ __forceinline__ unsigned rj_bin(uint64_t h, int shift, unsigned mask)
{
    return shift >= 64 ? 0u : (unsigned)(h >> shift) & mask;
}

// ---------------------------------------------------------------------------
// 1. Histogram of the top `bits` hash bits (bits <= 15: 128 KB of shared
// counters per CTA).

__global__ void __launch_bounds__(1024) rj_hist_kernel(const longlong2* __restrict__ in, int64_t n, int bits,
                                                       unsigned long long* __restrict__ hist)
{
    extern __shared__ unsigned rj_sh_hist[];
    const int P = 1 << bits;
    const int shift = 64 - bits;
    for (int b = threadIdx.x; b < P; b += blockDim.x) rj_sh_hist[b] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    constexpr int U = 8;
    for (; i + (U - 1) * stride < n; i += U * stride) {
        longlong2 t[U];
#pragma unroll
        for (int u = 0; u < U; ++u) t[u] = __ldcs(&in[i + u * stride]);
#pragma unroll
        for (int u = 0; u < U; ++u) atomicAdd(&rj_sh_hist[rj_bin(mix64((uint64_t)t[u].x), shift, P - 1)], 1u);
    }
    for (; i < n; i += stride) atomicAdd(&rj_sh_hist[rj_bin(mix64((uint64_t)__ldcs(&in[i]).x), shift, P - 1)], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < P; b += blockDim.x)
        if (rj_sh_hist[b]) atomicAdd(&hist[b], (unsigned long long)rj_sh_hist[b]);
}

// ---------------------------------------------------------------------------
// 2. Tile partition pass with exact offsets.  The input is a sequence of
// segments (one for the first pass; the coarse partitions for the second);
// tiles never straddle a segment.  Output bin of a tuple = (segment <<
// lbits) | ((mix64(key) >> shift) & mask).

struct RJPass {
    const longlong2* in;
    longlong2* out;
    const unsigned long long* seg_start;  // nseg + 1 exact segment bounds in `in`
    const unsigned long long* seg_tile0;  // nseg + 1 prefix of tiles per segment
    int nseg;
    int shift;
    unsigned mask;
    int lbits;
    const unsigned long long* bin_start;  // exact output start per output bin
    unsigned long long* cursor;           // per output bin, zeroed before the pass
    unsigned* err;                        // set if a tile's bulk copy never completed
};

struct RJTileRange {
    long long begin, end;
    int seg;
};

__device__ RJTileRange rj_tile_range(const RJPass& a, long long tile)
{
    int lo = 0, hi = a.nseg;  // seg_tile0[lo] <= tile < seg_tile0[hi]
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if ((long long)a.seg_tile0[mid] <= tile) lo = mid;
        else hi = mid;
    }
    RJTileRange r;
    r.seg = lo;
    r.begin = (long long)a.seg_start[lo] + (tile - (long long)a.seg_tile0[lo]) * RJ_TILE;
    r.end = min(r.begin + RJ_TILE, (long long)a.seg_start[lo + 1]);
    return r;
}

// Shared memory of one partition CTA: a ring of RJ_STAGES input tiles that
// bulk copies fill ahead of use, the grouped (staged) tile, and per-bin
// counters.
struct RJPartSmem {
    longlong2 in[RJ_STAGES][RJ_TILE];
    longlong2 stage[RJ_TILE];
    unsigned short stage_bin[RJ_TILE];
    unsigned hist[RJ_LMAX];
    unsigned loff[RJ_LMAX];
    unsigned long long gbase[RJ_LMAX];
    uint64_t bar[RJ_STAGES];
    RJTileRange info[RJ_STAGES];
    unsigned warp_tot[RJ_PT_THREADS / 32];
    int ok;
};

// Thread 0: starts the bulk copy of tile `tile` into ring slot `slot`.
__device__ __forceinline__ void rj_issue_tile(const RJPass& a, RJPartSmem& sm, int slot, long long tile)
{
    const RJTileRange r = rj_tile_range(a, tile);
    sm.info[slot] = r;
    const unsigned bytes = (unsigned)(r.end - r.begin) * 16u;
    mbar_arrive_expect_tx(&sm.bar[slot], bytes);
    bulk_load(sm.in[slot], a.in + r.begin, bytes, &sm.bar[slot]);
}

__global__ void __launch_bounds__(RJ_PT_THREADS, 2) rj_partition_kernel(RJPass a, long long ntiles)
{
    extern __shared__ __align__(128) unsigned char rj_pt_raw[];
    RJPartSmem& sm = *reinterpret_cast<RJPartSmem*>(rj_pt_raw);
    constexpr int PER = RJ_TILE / RJ_PT_THREADS;
    const int L = 1 << a.lbits;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    for (int b = tid; b < RJ_LMAX; b += RJ_PT_THREADS) sm.hist[b] = 0;
    if (tid == 0) {
        for (int s = 0; s < RJ_STAGES; ++s) mbar_init(&sm.bar[s], 1);
        mbar_fence_init();
        for (int s = 0; s < RJ_STAGES; ++s)
            if (blockIdx.x + (long long)s * gridDim.x < ntiles) rj_issue_tile(a, sm, s, blockIdx.x + (long long)s * gridDim.x);
        sm.ok = 1;
    }
    __syncthreads();
#if PYG_RJ_WARP_RANK
    const unsigned lt_mask = (1u << lane) - 1u;
#endif
    long long k = 0;
    for (long long tile = blockIdx.x; tile < ntiles; tile += gridDim.x, ++k) {
        const int slot = (int)(k % RJ_STAGES);
        const unsigned parity = (unsigned)((k / RJ_STAGES) & 1);
        // Every thread waits for the tile; a wait that runs out marks the
        // CTA failed and that thread's tuples are left out, so nothing is
        // written from memory the copy did not fill.
        const bool landed = mbar_wait(&sm.bar[slot], parity, kBulkWaitNs);
        if (!landed) sm.ok = 0;
        const RJTileRange cur = sm.info[slot];
        const unsigned n = (unsigned)(cur.end - cur.begin);
        // (1) Bin and rank every tuple; one shared atomic per (warp, bin).
        longlong2 t[PER];
        unsigned bin[PER], rank[PER];
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const unsigned i = j * RJ_PT_THREADS + tid;
            const bool valid = landed && i < n;
            bin[j] = 0xFFFFFFFFu;
            if (valid) {
                t[j] = sm.in[slot][i];
                bin[j] = rj_bin(mix64((uint64_t)t[j].x), a.shift, a.mask);
            }
#if PYG_RJ_WARP_RANK
            const unsigned peers = __match_any_sync(0xffffffffu, bin[j]);
            const int leader = __ffs(peers) - 1;
            unsigned base = 0;
            if (valid && lane == leader) base = atomicAdd(&sm.hist[bin[j]], (unsigned)__popc(peers));
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[j] = base + __popc(peers & lt_mask);
#else
            if (valid) rank[j] = atomicAdd(&sm.hist[bin[j]], 1u);
#endif
        }
        __syncthreads();  // A: histogram complete
        if (!sm.ok) break;
        // (2) Exclusive scan over bins (thread b owns bin b), reservation
        // of each non-empty bin's run, and reset of the counter.
        unsigned c = tid < L ? sm.hist[tid] : 0u;
        unsigned incl = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) sm.warp_tot[w] = incl;
        __syncthreads();  // B
        unsigned excl = incl - c, total = 0;
        for (int v = 0; v < RJ_PT_THREADS / 32; ++v) {
            if (v == w) excl += total;
            total += sm.warp_tot[v];
        }
        if (tid < L) {
            sm.loff[tid] = excl;
            if (c) {
                const unsigned ob = ((unsigned)cur.seg << a.lbits) | (unsigned)tid;
                sm.gbase[tid] = a.bin_start[ob] + atomicAdd(&a.cursor[ob], (unsigned long long)c);
            }
            sm.hist[tid] = 0;
        }
        __syncthreads();  // C: offsets ready
        // (3) Group the tile by bin in shared memory.
#pragma unroll
        for (int j = 0; j < PER; ++j)
            if (bin[j] != 0xFFFFFFFFu) {
                const unsigned s = sm.loff[bin[j]] + rank[j];
                sm.stage[s] = t[j];
                sm.stage_bin[s] = (unsigned short)bin[j];
            }
        __syncthreads();  // D: ring slot consumed, stage complete
        if (tid == 0) {
            const long long nt = tile + (long long)RJ_STAGES * gridDim.x;
            if (nt < ntiles) {
                fence_proxy_async_smem();
                rj_issue_tile(a, sm, slot, nt);
            }
        }
        // (4) Write each bin's run contiguously.
        for (unsigned i = tid; i < total; i += RJ_PT_THREADS) {
            const unsigned b = sm.stage_bin[i];
            __stcs(&a.out[sm.gbase[b] + (i - sm.loff[b])], sm.stage[i]);
        }
    }
    __syncthreads();
    if (tid == 0 && !sm.ok) atomicOr(a.err, 1u);
}

// ---------------------------------------------------------------------------
// 3. Join: persistent CTAs, one shared-memory table each.

struct RJItem {
    unsigned long long r0, s0;  // first build / probe tuple of the item
    unsigned rn, sn;            // build tuples (<= table capacity / 2), probe tuples
};

struct RJJoinArgs {
    const longlong2* R;
    const longlong2* S;
    const RJItem* items;
    long long nitems;
    unsigned* next;             // work queue head, zeroed
    int fine_bits;              // the table's slot uses the hash bits below these
    unsigned long long* acc;    // count, build sum, probe sum
    unsigned* dup;              // set when a build key repeats (UNIQUE)
};

// Slot of a key in a table of TS slots: multiply-high of the 32 hash bits
// below the fine partition bits (all keys of one partition share the top
// fine_bits bits).
__device__ __forceinline__ unsigned rj_slot(uint64_t h, int fb, unsigned TS)
{
    return __umulhi((unsigned)(h >> (32 - fb)), TS);
}

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

template <bool UNIQUE>
__global__ void __launch_bounds__(RJ_JOIN_THREADS, RJ_JOIN_BLOCKS) rj_join_kernel(RJJoinArgs a)
{
    extern __shared__ __align__(16) unsigned char rj_table[];
    constexpr unsigned TS = UNIQUE ? RJ_SLOTS_UNIQUE : RJ_SLOTS_COUNTED;
    constexpr int U = RJ_PROBE_UNROLL;
    __shared__ long long item_cur, item_next;
    __shared__ unsigned long long side_cnt, side_sum;
    ulonglong2* T2 = reinterpret_cast<ulonglong2*>(rj_table);  // UNIQUE slots
    ulonglong4* T4 = reinterpret_cast<ulonglong4*>(rj_table);  // counted slots
    uint64_t cnt = 0, bsum = 0, psum = 0;
    bool dup = false;
    const int fb = a.fine_bits;
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
                    rj_prefetch_l2(a.R + nx.r0, (unsigned long long)nx.rn * 16);
                    rj_prefetch_l2(a.S + nx.s0, (unsigned long long)min(nx.sn, 4096u) * 16);
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
            const longlong2 t = a.R[item.r0 + i];
            const uint64_t k = (uint64_t)t.x;
            if (k == kEmptyKey) {
                atomicAdd(&side_cnt, 1ULL);
                atomicAdd(&side_sum, (unsigned long long)t.y);
                continue;
            }
            unsigned pos = rj_slot(mix64(k), fb, TS);
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
            unsigned pos = rj_slot(mix64(k), fb, TS);
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
        const longlong2* S = a.S + item.s0;
        const unsigned sn = item.sn;
        unsigned i = threadIdx.x;
        for (; i + (U - 1) * RJ_JOIN_THREADS < sn; i += U * RJ_JOIN_THREADS) {
            longlong2 t[U];
#pragma unroll
            for (int u = 0; u < U; ++u) t[u] = __ldcs(&S[i + u * RJ_JOIN_THREADS]);
#pragma unroll
            for (int u = 0; u < U; ++u) probe(t[u]);
        }
        for (; i < sn; i += RJ_JOIN_THREADS) probe(__ldcs(&S[i]));
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
// Host driver.

namespace {

struct RJEvents {
    static constexpr int N = 5;
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

int launch_pass(pyg_ctx* ctx, const RJPass& p, long long ntiles)
{
    if (ntiles <= 0) return PYG_OK;
    const size_t smem = sizeof(RJPartSmem);
    PYG_CUDA(cudaFuncSetAttribute(rj_partition_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    PYG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, rj_partition_kernel, RJ_PT_THREADS, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = std::min<long long>(ntiles, (long long)ctx->sm_count * per_sm);
    rj_partition_kernel<<<(unsigned)grid, RJ_PT_THREADS, smem, ctx->stream>>>(p, ntiles);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

}  // namespace

int radix_join16(pyg_ctx* ctx, const void* Rv, int64_t nR, const void* Sv, int64_t nS, int fine_bits,
                 unsigned long long out[3], pyg_join_stats* stats)
{
    const longlong2* R = (const longlong2*)Rv;
    const longlong2* S = (const longlong2*)Sv;
    out[0] = out[1] = out[2] = 0;
    if (fine_bits <= 0) {
        // Fine partitions of about 0.7 x the table's build capacity.
        fine_bits = 1;
        while (fine_bits < RJ_MAX_FINE_BITS &&
               (double)nR / (double)(1 << fine_bits) > 0.7 * RJ_RCAP_UNIQUE)
            ++fine_bits;
    }
    if (fine_bits < 1 || fine_bits > RJ_MAX_FINE_BITS) {
        set_error("pyg_hashjoin_agg: radix bits must be in [1, %d]", RJ_MAX_FINE_BITS);
        return PYG_ERR_ARG;
    }
    const int FB = fine_bits;
    const bool two = FB > RJ_MAX_LOCAL_BITS;
    const int CB = two ? (FB + 1) / 2 : FB;
    const int F = 1 << FB, C = 1 << CB;
    if (stats) {
        stats->algorithm = PYG_JOIN_RADIX;
        stats->radix_bits = FB;
    }
    if (nR == 0 || nS == 0) return PYG_OK;

    RJEvents tm;
    tm.start(ctx, stats != nullptr);
    // Device metadata (u64 words):
    //   histR[F] histS[F] | fineR[F+1] fineS[F+1] | coarseR[C+1] coarseS[C+1]
    //   | tilesR[C+1] tilesS[C+1] | curR1[C] curS1[C] curR2[F] curS2[F]
    //   | whole[4] = {0, nR, 0, nS} | wtiles[4] = {0, tiles(R), 0, tiles(S)}
    const size_t nmeta = 2 * (size_t)F + 2 * (size_t)(F + 1) + 4 * (size_t)(C + 1) + 2 * (size_t)C + 2 * (size_t)F + 8;
    unsigned long long* meta = nullptr;
    void *R1 = nullptr, *R2 = nullptr, *S1 = nullptr, *S2 = nullptr;
    RJItem* ditems = nullptr;
    int rc = PYG_OK;
    do {
        if ((rc = dalloc(ctx, (void**)&meta, nmeta * 8))) break;
        unsigned long long* histR = meta;
        unsigned long long* histS = histR + F;
        unsigned long long* fineR = histS + F;
        unsigned long long* fineS = fineR + F + 1;
        unsigned long long* coarseR = fineS + F + 1;
        unsigned long long* coarseS = coarseR + C + 1;
        unsigned long long* tilesR = coarseS + C + 1;
        unsigned long long* tilesS = tilesR + C + 1;
        unsigned long long* curR1 = tilesS + C + 1;
        unsigned long long* curS1 = curR1 + C;
        unsigned long long* curR2 = curS1 + C;
        unsigned long long* curS2 = curR2 + F;
        unsigned long long* whole = curS2 + F;  // single-segment bounds of the unpartitioned inputs
        unsigned long long* wtiles = whole + 4;
        PYG_CUDA(cudaMemsetAsync(meta, 0, nmeta * 8, ctx->stream));
        unsigned* perr = (unsigned*)(ctx->dcounters + 202);  // partition passes: a bulk copy never landed
        PYG_CUDA(cudaMemsetAsync(perr, 0, 8, ctx->stream));

        // 1. Histograms.
        const size_t hsm = (size_t)F * 4;
        PYG_CUDA(cudaFuncSetAttribute(rj_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
        int hper = 0;
        PYG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&hper, rj_hist_kernel, 1024, hsm));
        if (hper < 1) hper = 1;
        rj_hist_kernel<<<ctx->sm_count * hper, 1024, hsm, ctx->stream>>>(R, nR, FB, histR);
        PYG_LAUNCHED(ctx);
        rj_hist_kernel<<<ctx->sm_count * hper, 1024, hsm, ctx->stream>>>(S, nS, FB, histS);
        PYG_LAUNCHED(ctx);
        std::vector<unsigned long long> hr(F), hs(F);
        PYG_CUDA(cudaMemcpyAsync(hr.data(), histR, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(hs.data(), histS, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));

        // Host: exact offsets, tile prefixes, work items.
        const int sub = FB - CB;
        std::vector<unsigned long long> up((size_t)2 * (F + 1) + 4 * (size_t)(C + 1));
        unsigned long long* fR = up.data();
        unsigned long long* fS = fR + F + 1;
        unsigned long long* cR = fS + F + 1;
        unsigned long long* cS = cR + C + 1;
        unsigned long long* tR = cS + C + 1;
        unsigned long long* tS = tR + C + 1;
        fR[0] = fS[0] = 0;
        for (int f = 0; f < F; ++f) {
            fR[f + 1] = fR[f] + hr[f];
            fS[f + 1] = fS[f] + hs[f];
        }
        if (fR[F] != (unsigned long long)nR || fS[F] != (unsigned long long)nS) {
            set_error("pyg_hashjoin_agg: partition histogram does not add up");
            rc = PYG_ERR_CUDA;
            break;
        }
        tR[0] = tS[0] = 0;
        for (int c = 0; c <= C; ++c) {
            cR[c] = fR[(size_t)c << sub];
            cS[c] = fS[(size_t)c << sub];
        }
        for (int c = 0; c < C; ++c) {
            tR[c + 1] = tR[c] + (cR[c + 1] - cR[c] + RJ_TILE - 1) / RJ_TILE;
            tS[c + 1] = tS[c] + (cS[c + 1] - cS[c] + RJ_TILE - 1) / RJ_TILE;
        }
        const long long ntR = (nR + RJ_TILE - 1) / RJ_TILE, ntS = (nS + RJ_TILE - 1) / RJ_TILE;
        const unsigned long long wh[8] = {0, (unsigned long long)nR, 0, (unsigned long long)nS,
                                          0, (unsigned long long)ntR, 0, (unsigned long long)ntS};
        std::vector<RJItem> items;
        std::vector<unsigned long long> rstart(fR, fR + F), sstart(fS, fS + F);
        make_items(hr, hs, rstart, sstart, RJ_RCAP_UNIQUE, items);
        PYG_CUDA(cudaMemcpyAsync(fineR, up.data(), up.size() * 8, cudaMemcpyHostToDevice, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(whole, wh, sizeof(wh), cudaMemcpyHostToDevice, ctx->stream));
        if (!items.empty()) {
            if ((rc = dalloc(ctx, (void**)&ditems, items.size() * sizeof(RJItem)))) break;
            PYG_CUDA(cudaMemcpyAsync(ditems, items.data(), items.size() * sizeof(RJItem), cudaMemcpyHostToDevice,
                                     ctx->stream));
        }
        tm.mark(ctx, 1);

        // 2. Partition passes.
        if ((rc = dalloc(ctx, &R1, (size_t)nR * 16)) || (rc = dalloc(ctx, &S1, (size_t)nS * 16))) break;
        if (two && ((rc = dalloc(ctx, &R2, (size_t)nR * 16)) || (rc = dalloc(ctx, &S2, (size_t)nS * 16)))) break;
        auto run_side = [&](const longlong2* in, const unsigned long long* seg, const unsigned long long* segt,
                            long long ntiles, unsigned long long* coarse, unsigned long long* cur1,
                            unsigned long long* fine, unsigned long long* cur2, unsigned long long* tiles, void* o1,
                            void* o2, long long ntiles2) -> int {
            RJPass p;
            p.in = in;
            p.out = (longlong2*)o1;
            p.seg_start = seg;
            p.seg_tile0 = segt;
            p.nseg = 1;
            p.shift = 64 - CB;
            p.mask = (unsigned)(C - 1);
            p.lbits = CB;
            p.bin_start = two ? coarse : fine;
            p.cursor = two ? cur1 : cur2;
            p.err = perr;
            int r = launch_pass(ctx, p, ntiles);
            if (r || !two) return r;
            p.in = (const longlong2*)o1;
            p.out = (longlong2*)o2;
            p.seg_start = coarse;
            p.seg_tile0 = tiles;
            p.nseg = C;
            p.shift = 64 - FB;
            p.mask = (unsigned)((1 << sub) - 1);
            p.lbits = sub;
            p.bin_start = fine;
            p.cursor = cur2;
            return launch_pass(ctx, p, ntiles2);
        };
        if ((rc = run_side(R, whole, wtiles, ntR, coarseR, curR1, fineR, curR2, tilesR, R1, R2, (long long)tR[C])))
            break;
        tm.mark(ctx, 2);
        if ((rc = run_side(S, whole + 2, wtiles + 2, ntS, coarseS, curS1, fineS, curS2, tilesS, S1, S2,
                           (long long)tS[C])))
            break;
        tm.mark(ctx, 3);

        // 3. Join: distinct build keys first (16-byte slots); on a repeated
        // key, again with counted 32-byte slots and smaller build chunks.
        const longlong2* Rf = (const longlong2*)(two ? R2 : R1);
        const longlong2* Sf = (const longlong2*)(two ? S2 : S1);
        unsigned long long* acc = ctx->dcounters + 8;
        unsigned* next = (unsigned*)(ctx->dcounters + 200);  // word 200: queue head, word 201: dup flag
        unsigned* dupf = (unsigned*)(ctx->dcounters + 201);
        unsigned long long* h = (unsigned long long*)ctx->pinned;
        for (int pass = 0; pass < 2 && !items.empty(); ++pass) {
            const bool unique = pass == 0;
            if (!unique) {
                make_items(hr, hs, rstart, sstart, RJ_RCAP_COUNTED, items);
                dfree(ctx, ditems);
                ditems = nullptr;
                if ((rc = dalloc(ctx, (void**)&ditems, items.size() * sizeof(RJItem)))) break;
                PYG_CUDA(cudaMemcpyAsync(ditems, items.data(), items.size() * sizeof(RJItem), cudaMemcpyHostToDevice,
                                         ctx->stream));
            }
            void* fn = unique ? (void*)rj_join_kernel<true> : (void*)rj_join_kernel<false>;
            PYG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, RJ_TABLE_BYTES));
            PYG_CUDA(cudaMemsetAsync(acc, 0, 3 * 8, ctx->stream));
            PYG_CUDA(cudaMemsetAsync(next, 0, 16, ctx->stream));
            RJJoinArgs ja;
            ja.R = Rf;
            ja.S = Sf;
            ja.items = ditems;
            ja.nitems = (long long)items.size();
            ja.next = next;
            ja.fine_bits = FB;
            ja.acc = acc;
            ja.dup = dupf;
            const unsigned grid = (unsigned)std::min<long long>((long long)ctx->sm_count * RJ_JOIN_BLOCKS, ja.nitems);
            if (unique) rj_join_kernel<true><<<grid, RJ_JOIN_THREADS, RJ_TABLE_BYTES, ctx->stream>>>(ja);
            else rj_join_kernel<false><<<grid, RJ_JOIN_THREADS, RJ_TABLE_BYTES, ctx->stream>>>(ja);
            PYG_LAUNCHED(ctx);
            PYG_CUDA(cudaMemcpyAsync(h, acc, 3 * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(h + 3, next, 24, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            if ((unsigned)h[5]) {
                set_error("pyg_hashjoin_agg: a partition tile copy did not complete in time");
                rc = PYG_ERR_TIMEOUT;
                break;
            }
            if (!unique || (unsigned)h[4] == 0) break;
        }
        if (rc) break;
        tm.mark(ctx, 4);
        if (!items.empty()) {
            out[0] = h[0];
            out[1] = h[1];
            out[2] = h[2];
        }
        if (stats) {
            cudaEventSynchronize(tm.ev[4]);
            stats->histogram_ms = tm.ms(0, 1);
            stats->build_partition_ms = tm.ms(1, 2);
            stats->build_ms = 0;
            stats->probe_partition_ms = tm.ms(2, 3);
            stats->probe_ms = tm.ms(3, 4);
        }
    } while (0);
    dfree(ctx, ditems);
    dfree(ctx, R1);
    dfree(ctx, R2);
    dfree(ctx, S1);
    dfree(ctx, S2);
    dfree(ctx, meta);
    return rc;
}

}  // namespace pyg
