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
#include <cmath>
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

__global__ void __launch_bounds__(1024) rj_hist_kernel(const longlong2* __restrict__ in, int64_t n, int64_t step,
                                                       int bits, unsigned long long* __restrict__ hist)
{
    // Counts in[0], in[step], in[2 step], ... (step 1: every tuple).
    extern __shared__ unsigned rj_sh_hist[];
    const int P = 1 << bits;
    const int shift = 64 - bits;
    const int64_t m = (n + step - 1) / step;
    for (int b = threadIdx.x; b < P; b += blockDim.x) rj_sh_hist[b] = 0;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    constexpr int U = 8;
    for (; i + (U - 1) * stride < m; i += U * stride) {
        longlong2 t[U];
#pragma unroll
        for (int u = 0; u < U; ++u) t[u] = __ldcs(&in[(i + u * stride) * step]);
#pragma unroll
        for (int u = 0; u < U; ++u) atomicAdd(&rj_sh_hist[rj_bin(mix64((uint64_t)t[u].x), shift, P - 1)], 1u);
    }
    for (; i < m; i += stride)
        atomicAdd(&rj_sh_hist[rj_bin(mix64((uint64_t)__ldcs(&in[i * step]).x), shift, P - 1)], 1u);
    __syncthreads();
    for (int b = threadIdx.x; b < P; b += blockDim.x)
        if (rj_sh_hist[b]) atomicAdd(&hist[b], (unsigned long long)rj_sh_hist[b]);
}

// Tiles per segment, as an exclusive prefix (one thread; at most 2^8
// segments): tiles[C] is the pass's tile count.  Counts are first clamped
// to their region's capacity, so a region that overflowed (its result is
// discarded and redone) is never read past its end.
__global__ void rj_tile_prefix_kernel(unsigned long long* __restrict__ count, const unsigned long long* __restrict__ cap,
                                      int C, unsigned long long* __restrict__ tiles)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long t = 0;
    tiles[0] = 0;
    for (int c = 0; c < C; ++c) {
        const unsigned long long n = count[c] < cap[c] ? count[c] : cap[c];
        count[c] = n;
        t += (n + RJ_TILE - 1) / RJ_TILE;
        tiles[c + 1] = t;
    }
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
    const unsigned long long* bin_start;  // output region start per output bin
    unsigned long long* cursor;           // per output bin, zeroed before the pass
    unsigned* err;                        // set if a tile's bulk copy never completed
    // Optional (null when offsets are exact):
    const unsigned long long* seg_count;  // tuples in each segment (segment end = start + count)
    const unsigned long long* bin_cap;    // region capacity per output bin
    unsigned* ovf;                        // set when a bin outgrows its region (the run is not written)
    const unsigned long long* ntiles_dev; // tile count read on the device
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
    const long long seg_end =
        a.seg_count ? (long long)a.seg_start[lo] + (long long)a.seg_count[lo] : (long long)a.seg_start[lo + 1];
    r.end = min(r.begin + RJ_TILE, seg_end);
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
    if (a.ntiles_dev) ntiles = (long long)*a.ntiles_dev;
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
        // The reservation's result (a global atomic, about a microsecond
        // away) is first needed after the tile is staged.
        unsigned long long resv = 0, bstart = 0, bcap = ~0ULL;
        if (tid < L) {
            sm.loff[tid] = excl;
            if (c) {
                const unsigned ob = ((unsigned)cur.seg << a.lbits) | (unsigned)tid;
                bstart = a.bin_start[ob];
                if (a.bin_cap) bcap = a.bin_cap[ob];
                resv = atomicAdd(&a.cursor[ob], (unsigned long long)c);
            }
            sm.hist[tid] = 0;
        }
        __syncthreads();  // C: in-tile offsets ready
        // (3) Group the tile by bin in shared memory.
#pragma unroll
        for (int j = 0; j < PER; ++j)
            if (bin[j] != 0xFFFFFFFFu) {
                const unsigned s = sm.loff[bin[j]] + rank[j];
                sm.stage[s] = t[j];
                sm.stage_bin[s] = (unsigned short)bin[j];
            }
        if (tid < L && c) {
            unsigned long long gb = bstart + resv;
            if (resv + c > bcap) {  // outgrew its region: not written; the host redoes the pass exactly
                atomicOr(a.ovf, 1u);
                gb = ~0ULL;
            }
            sm.gbase[tid] = gb;
        }
        __syncthreads();  // D: ring slot consumed, stage and global offsets complete
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
            const unsigned long long gb = sm.gbase[b];
            if (gb != ~0ULL) __stcs(&a.out[gb + (i - sm.loff[b])], sm.stage[i]);
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

// Host-side layout of one relation's partitions.  Exact layouts come from a
// full histogram (dense, contiguous partitions); sampled layouts size each
// partition's region from a strided sample with six standard deviations of
// slack, and the partition pass reports any region that overflows.
struct RJLayout {
    bool sampled = false;
    std::vector<unsigned long long> fstart;  // F + 1 fine region starts
    std::vector<unsigned long long> fcap;    // F fine region capacities (sampled)
    std::vector<unsigned long long> cstart;  // C + 1 coarse region starts
    std::vector<unsigned long long> ccap;    // C coarse region capacities (sampled)
    std::vector<unsigned long long> tiles2;  // C + 1 tile prefix of the second pass (exact)
    std::vector<unsigned long long> count;   // F tuples per fine partition, once known
    unsigned long long p1 = 0, p2 = 0;       // tuples in the pass-1 / pass-2 buffers
    unsigned long long tiles2_max = 0;       // upper bound of the second pass's tiles (sampled)
};

void layout_exact(const std::vector<unsigned long long>& h, int C, int sub, RJLayout& L)
{
    const size_t F = h.size();
    L.sampled = false;
    L.fstart.assign(F + 1, 0);
    for (size_t f = 0; f < F; ++f) L.fstart[f + 1] = L.fstart[f] + h[f];
    L.cstart.assign(C + 1, 0);
    for (int c = 0; c <= C; ++c) L.cstart[c] = L.fstart[(size_t)c << sub];
    L.tiles2.assign(C + 1, 0);
    for (int c = 0; c < C; ++c) L.tiles2[c + 1] = L.tiles2[c] + (L.cstart[c + 1] - L.cstart[c] + RJ_TILE - 1) / RJ_TILE;
    L.fcap.clear();
    L.ccap.clear();
    L.count = h;
    L.p1 = L.p2 = L.fstart[F];
    L.tiles2_max = L.tiles2[C];
}

unsigned long long sampled_cap(unsigned long long c, long long step, unsigned long long extra)
{
    const double x = (double)c;
    return (unsigned long long)std::ceil((x + 6.0 * std::sqrt(x) + 8.0) * (double)step) + extra;
}

void layout_sampled(const std::vector<unsigned long long>& sc, long long step, int C, int sub, RJLayout& L)
{
    const size_t F = sc.size();
    L.sampled = true;
    L.fcap.assign(F, 0);
    L.fstart.assign(F + 1, 0);
    for (size_t f = 0; f < F; ++f) {
        L.fcap[f] = sampled_cap(sc[f], step, 64);
        L.fstart[f + 1] = L.fstart[f] + L.fcap[f];
    }
    L.ccap.assign(C, 0);
    L.cstart.assign(C + 1, 0);
    L.tiles2_max = 0;
    for (int c = 0; c < C; ++c) {
        unsigned long long cc = 0;
        for (size_t f = (size_t)c << sub; f < (size_t)(c + 1) << sub; ++f) cc += sc[f];
        L.ccap[c] = sampled_cap(cc, step, 1024);
        L.cstart[c + 1] = L.cstart[c] + L.ccap[c];
        L.tiles2_max += (L.ccap[c] + RJ_TILE - 1) / RJ_TILE;
    }
    L.tiles2.clear();
    L.count.clear();
    L.p1 = L.cstart[C];
    L.p2 = L.fstart[F];
}

// Device copy of one relation's partition metadata (u64 words).
struct RJSideDev {
    unsigned long long *fstart, *fcap, *cstart, *ccap, *cur1, *cur2, *tiles2, *whole, *wtiles;
    static size_t words(int F, int C) { return (size_t)(F + 1) + F + (C + 1) + C + C + F + (C + 1) + 4; }
    void carve(unsigned long long* m, int F, int C)
    {
        fstart = m;
        fcap = fstart + F + 1;
        cstart = fcap + F;
        ccap = cstart + C + 1;
        cur1 = ccap + C;
        cur2 = cur1 + C;
        tiles2 = cur2 + F;
        whole = tiles2 + C + 1;
        wtiles = whole + 2;
    }
};

int upload_layout(pyg_ctx* ctx, const RJLayout& L, const RJSideDev& d, int F, int C, int64_t n)
{
    PYG_CUDA(cudaMemcpyAsync(d.fstart, L.fstart.data(), (size_t)(F + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    PYG_CUDA(cudaMemcpyAsync(d.cstart, L.cstart.data(), (size_t)(C + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    if (L.sampled) {
        PYG_CUDA(cudaMemcpyAsync(d.fcap, L.fcap.data(), (size_t)F * 8, cudaMemcpyHostToDevice, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(d.ccap, L.ccap.data(), (size_t)C * 8, cudaMemcpyHostToDevice, ctx->stream));
    } else {
        PYG_CUDA(cudaMemcpyAsync(d.tiles2, L.tiles2.data(), (size_t)(C + 1) * 8, cudaMemcpyHostToDevice, ctx->stream));
    }
    PYG_CUDA(cudaMemsetAsync(d.cur1, 0, (size_t)(C + F) * 8, ctx->stream));  // cur1 and cur2 are adjacent
    const unsigned long long w[4] = {0, (unsigned long long)n, 0, (unsigned long long)((n + RJ_TILE - 1) / RJ_TILE)};
    PYG_CUDA(cudaMemcpyAsync(d.whole, w, sizeof(w), cudaMemcpyHostToDevice, ctx->stream));
    return PYG_OK;
}

// Runs the partition pass(es) of one relation into P1 (and P2).
int run_passes(pyg_ctx* ctx, const longlong2* in, int64_t n, const RJLayout& L, const RJSideDev& d, bool two, int FB,
               int CB, void* P1, void* P2, unsigned* err, unsigned* ovf)
{
    const int C = 1 << CB, sub = FB - CB;
    RJPass p;
    memset(&p, 0, sizeof(p));
    p.in = in;
    p.out = (longlong2*)P1;
    p.seg_start = d.whole;
    p.seg_tile0 = d.wtiles;
    p.nseg = 1;
    p.shift = 64 - CB;
    p.mask = (unsigned)(C - 1);
    p.lbits = CB;
    p.bin_start = two ? d.cstart : d.fstart;
    p.bin_cap = L.sampled ? (two ? d.ccap : d.fcap) : nullptr;
    p.cursor = two ? d.cur1 : d.cur2;
    p.err = err;
    p.ovf = ovf;
    int rc = launch_pass(ctx, p, (n + RJ_TILE - 1) / RJ_TILE);
    if (rc || !two) return rc;
    long long ntiles2;
    if (L.sampled) {
        // Second-pass segments are the first pass's regions, filled to the
        // counts its cursors reached; the tile prefix is formed on the device.
        rj_tile_prefix_kernel<<<1, 32, 0, ctx->stream>>>(d.cur1, d.ccap, C, d.tiles2);
        PYG_LAUNCHED(ctx);
        p.seg_count = d.cur1;
        p.ntiles_dev = d.tiles2 + C;
        ntiles2 = (long long)L.tiles2_max;
    } else {
        ntiles2 = (long long)L.tiles2[C];
    }
    p.in = (const longlong2*)P1;
    p.out = (longlong2*)P2;
    p.seg_start = d.cstart;
    p.seg_tile0 = d.tiles2;
    p.nseg = C;
    p.shift = 64 - FB;
    p.mask = (unsigned)((1 << sub) - 1);
    p.lbits = sub;
    p.bin_start = d.fstart;
    p.bin_cap = L.sampled ? d.fcap : nullptr;
    p.cursor = d.cur2;
    return launch_pass(ctx, p, ntiles2);
}

int hist_launch(pyg_ctx* ctx, const longlong2* in, int64_t n, int64_t step, int FB, unsigned long long* hist)
{
    const size_t hsm = (size_t)4 << FB;
    PYG_CUDA(cudaFuncSetAttribute(rj_hist_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
    int per = 0;
    PYG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, rj_hist_kernel, 1024, hsm));
    if (per < 1) per = 1;
    const int64_t m = (n + step - 1) / step;
    const int64_t want = (m + 1024 * 8 - 1) / (1024 * 8);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->sm_count * per));
    PYG_CUDA(cudaMemsetAsync(hist, 0, (size_t)8 << FB, ctx->stream));
    rj_hist_kernel<<<grid, 1024, hsm, ctx->stream>>>(in, n, step, FB, hist);
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
        while (fine_bits < RJ_MAX_FINE_BITS && (double)nR / (double)(1 << fine_bits) > 0.7 * RJ_RCAP_UNIQUE)
            ++fine_bits;
    }
    if (fine_bits < 1 || fine_bits > RJ_MAX_FINE_BITS) {
        set_error("pyg_hashjoin_agg: radix bits must be in [1, %d]", RJ_MAX_FINE_BITS);
        return PYG_ERR_ARG;
    }
    const int FB = fine_bits;
    const bool two = FB > RJ_MAX_LOCAL_BITS;
    const int CB = two ? (FB + 1) / 2 : FB;
    const int F = 1 << FB, C = 1 << CB, sub = FB - CB;
    if (stats) {
        stats->algorithm = PYG_JOIN_RADIX;
        stats->radix_bits = FB;
    }
    if (nR == 0 || nS == 0) return PYG_OK;
    // The probe side of a two-pass join is laid out from a sample of about
    // 2^24 tuples instead of a full histogram read.
    const bool sample_s = two && nS >= ((int64_t)1 << 25);
    const int64_t sstep = sample_s ? std::max<int64_t>(1, nS >> 24) : 1;

    RJEvents tm;
    tm.start(ctx, stats != nullptr);
    const size_t side_words = RJSideDev::words(F, C);
    unsigned long long* meta = nullptr;
    void *R1 = nullptr, *R2 = nullptr, *S1 = nullptr, *S2 = nullptr;
    RJItem* ditems = nullptr;
    int rc = PYG_OK;
    do {
        if ((rc = dalloc(ctx, (void**)&meta, (2 * side_words + 2 * (size_t)F) * 8))) break;
        RJSideDev dR, dS;
        dR.carve(meta, F, C);
        dS.carve(meta + side_words, F, C);
        unsigned long long* histR = meta + 2 * side_words;
        unsigned long long* histS = histR + F;
        unsigned* flags = (unsigned*)(ctx->dcounters + 202);  // [0] a bulk copy never landed, [1] region overflow
        PYG_CUDA(cudaMemsetAsync(flags, 0, 8, ctx->stream));
        unsigned long long* h = (unsigned long long*)ctx->pinned;

        // 1. Histograms: exact for the build side, sampled or exact for the
        // probe side.
        if ((rc = hist_launch(ctx, R, nR, 1, FB, histR))) break;
        if ((rc = hist_launch(ctx, S, nS, sstep, FB, histS))) break;
        std::vector<unsigned long long> hr(F), hs(F);
        PYG_CUDA(cudaMemcpyAsync(hr.data(), histR, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaMemcpyAsync(hs.data(), histS, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        RJLayout LR, LS;
        layout_exact(hr, C, sub, LR);
        if (sample_s) layout_sampled(hs, sstep, C, sub, LS);
        else layout_exact(hs, C, sub, LS);
        if (LR.fstart[F] != (unsigned long long)nR || (!sample_s && LS.fstart[F] != (unsigned long long)nS)) {
            set_error("pyg_hashjoin_agg: partition histogram does not add up");
            rc = PYG_ERR_CUDA;
            break;
        }
        if ((rc = upload_layout(ctx, LR, dR, F, C, nR)) || (rc = upload_layout(ctx, LS, dS, F, C, nS))) break;
        tm.mark(ctx, 1);

        // 2. Partition passes.
        if ((rc = dalloc(ctx, &R1, (size_t)LR.p1 * 16))) break;
        if (two && (rc = dalloc(ctx, &R2, (size_t)LR.p2 * 16))) break;
        if ((rc = run_passes(ctx, R, nR, LR, dR, two, FB, CB, R1, R2, flags, flags + 1))) break;
        tm.mark(ctx, 2);
        for (int attempt = 0; attempt < 2; ++attempt) {
            dfree(ctx, S1);
            dfree(ctx, S2);
            S1 = S2 = nullptr;
            if ((rc = dalloc(ctx, &S1, (size_t)LS.p1 * 16))) break;
            if (two && (rc = dalloc(ctx, &S2, (size_t)LS.p2 * 16))) break;
            if ((rc = run_passes(ctx, S, nS, LS, dS, two, FB, CB, S1, S2, flags, flags + 1))) break;
            if (!LS.sampled) break;
            // Exact per-partition counts of the sampled layout (and whether
            // any region overflowed).
            LS.count.resize(F);
            PYG_CUDA(cudaMemcpyAsync(LS.count.data(), dS.cur2, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(h + 6, flags, 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            if (((unsigned*)(h + 6))[1] == 0) break;
            // A region overflowed (the sample misjudged a partition): redo the
            // probe side from an exact histogram.
            if ((rc = hist_launch(ctx, S, nS, 1, FB, histS))) break;
            PYG_CUDA(cudaMemcpyAsync(hs.data(), histS, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            layout_exact(hs, C, sub, LS);
            if ((rc = upload_layout(ctx, LS, dS, F, C, nS))) break;
            PYG_CUDA(cudaMemsetAsync(flags + 1, 0, 4, ctx->stream));
        }
        if (rc) break;
        if (stats) stats->overflow_tuples = LS.sampled ? 0 : (sample_s ? 1 : 0);
        tm.mark(ctx, 3);

        // 3. Join: distinct build keys first (16-byte slots); on a repeated
        // key, again with counted 32-byte slots and smaller build chunks.
        const longlong2* Rf = (const longlong2*)(two ? R2 : R1);
        const longlong2* Sf = (const longlong2*)(two ? S2 : S1);
        unsigned long long* acc = ctx->dcounters + 8;
        unsigned* next = (unsigned*)(ctx->dcounters + 200);  // word 200: queue head, word 201: dup flag
        unsigned* dupf = (unsigned*)(ctx->dcounters + 201);
        std::vector<unsigned long long> rstart(LR.fstart.begin(), LR.fstart.end() - 1);
        std::vector<unsigned long long> sstart(LS.fstart.begin(), LS.fstart.end() - 1);
        std::vector<RJItem> items;
        for (int pass = 0; pass < 2; ++pass) {
            const bool unique = pass == 0;
            make_items(LR.count, LS.count, rstart, sstart, unique ? RJ_RCAP_UNIQUE : RJ_RCAP_COUNTED, items);
            if (items.empty()) break;
            dfree(ctx, ditems);
            ditems = nullptr;
            if ((rc = dalloc(ctx, (void**)&ditems, items.size() * sizeof(RJItem)))) break;
            PYG_CUDA(cudaMemcpyAsync(ditems, items.data(), items.size() * sizeof(RJItem), cudaMemcpyHostToDevice,
                                     ctx->stream));
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
            PYG_CUDA(cudaMemcpyAsync(h + 3, next, 16, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaMemcpyAsync(h + 6, flags, 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            if (((unsigned*)(h + 6))[0]) {
                set_error("pyg_hashjoin_agg: a partition tile copy did not complete in time");
                rc = PYG_ERR_TIMEOUT;
                break;
            }
            if (((unsigned*)(h + 6))[1]) {
                set_error("pyg_hashjoin_agg: a partition outgrew its exact region");
                rc = PYG_ERR_CUDA;
                break;
            }
            out[0] = h[0];
            out[1] = h[1];
            out[2] = h[2];
            if (!unique || (unsigned)h[4] == 0) break;
        }
        if (rc) break;
        tm.mark(ctx, 4);
        if (stats) {
            cudaEventSynchronize(tm.ev[4]);
            stats->histogram_ms = tm.ms(0, 1);
            stats->build_partition_ms = tm.ms(1, 2);
            stats->build_ms = 0;
            stats->probe_partition_ms = tm.ms(2, 3);
            stats->probe_ms = tm.ms(3, 4);
            stats->padded_tuples = (int64_t)(LS.p2 - (unsigned long long)nS);
            stats->histogram_tuples = nR + (nS + sstep - 1) / sstep;
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
