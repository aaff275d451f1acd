// Hash partitioning shared by the radix operators: kernels and host
// helpers (declared in radixpart.cuh).
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <type_traits>
#include <vector>

#include "bulk.cuh"
#include "radixpart.cuh"

namespace pyg {

#ifndef PYG_RJ_PT_MINB
#define PYG_RJ_PT_MINB 2
#endif
#ifndef PYG_RJ_STAGES
#define PYG_RJ_STAGES 2
#endif
constexpr int RJ_STAGES = PYG_RJ_STAGES;                               // input tiles in flight per partition CTA
constexpr unsigned long long kBulkWaitNs = 2000000000ULL;  // 2 s
constexpr unsigned long long kSkipRun = 1ULL << 63;          // gdelta of a run that is not written

__device__ __forceinline__ unsigned rj_bin(uint64_t h, int shift, unsigned mask)
{
    return shift >= 64 ? 0u : (unsigned)(h >> shift) & mask;
}


// ---------------------------------------------------------------------------
// 1. Histogram of the top `bits` hash bits (bits <= 15: 128 KB of shared
// counters per CTA).

template <bool MODEL>
__global__ void __launch_bounds__(1024) rj_hist_kernel(const longlong2* __restrict__ in, int64_t n, int64_t step,
                                                       int bits, int base, int span, unsigned* __restrict__ part,
                                                       long long* __restrict__ mm, RJModel model)
{
    // Counts the bins [base, base + span) of in[0], in[step], in[2 step],
    // ... (step 1: every tuple); span 32-bit counters in shared memory,
    // stored to this CTA's row of part (rj_hist_sum_kernel adds the rows).
    // With mm: also the key and payload ranges of the tuples read.  MODEL:
    // the bins are the learned model's (rj_model_bin) instead of hash bits.
    extern __shared__ unsigned rj_sh_hist[];
    __shared__ long long sh_mm[4];
    const int P = 1 << bits;
    const int shift = 64 - bits;
    const int64_t m = (n + step - 1) / step;
    for (int b = threadIdx.x; b < span; b += blockDim.x) rj_sh_hist[b] = 0;
    if (threadIdx.x < 4) sh_mm[threadIdx.x] = (threadIdx.x & 1) ? LLONG_MIN : LLONG_MAX;
    __syncthreads();
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    long long kmin = LLONG_MAX, kmax = LLONG_MIN, pmin = LLONG_MAX, pmax = LLONG_MIN;
    auto count = [&](const longlong2 t) {
        const uint64_t code = MODEL ? rj_model_code(model, t.x) : rj_hash((uint64_t)t.x);
        const unsigned r = rj_bin(code, shift, P - 1) - (unsigned)base;
        if (r < (unsigned)span) atomicAdd(&rj_sh_hist[r], 1u);
        kmin = min(kmin, t.x);
        kmax = max(kmax, t.x);
        pmin = min(pmin, t.y);
        pmax = max(pmax, t.y);
    };
    constexpr int U = 8;
    for (; i + (U - 1) * stride < m; i += U * stride) {
        longlong2 t[U];
#pragma unroll
        for (int u = 0; u < U; ++u) t[u] = __ldcs(&in[(i + u * stride) * step]);
#pragma unroll
        for (int u = 0; u < U; ++u) count(t[u]);
    }
    for (; i < m; i += stride) count(__ldcs(&in[i * step]));
    if (mm) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            kmin = min(kmin, __shfl_xor_sync(0xffffffffu, kmin, o));
            kmax = max(kmax, __shfl_xor_sync(0xffffffffu, kmax, o));
            pmin = min(pmin, __shfl_xor_sync(0xffffffffu, pmin, o));
            pmax = max(pmax, __shfl_xor_sync(0xffffffffu, pmax, o));
        }
        if ((threadIdx.x & 31) == 0) {
            atomicMin(&sh_mm[0], kmin);
            atomicMax(&sh_mm[1], kmax);
            atomicMin(&sh_mm[2], pmin);
            atomicMax(&sh_mm[3], pmax);
        }
    }
    __syncthreads();
    unsigned* row = part + (size_t)blockIdx.x * span;
    for (int b = threadIdx.x; b < span; b += blockDim.x) row[b] = rj_sh_hist[b];
    if (mm && threadIdx.x == 0) {
        atomicMin(&mm[0], sh_mm[0]);
        atomicMax(&mm[1], sh_mm[1]);
        atomicMin(&mm[2], sh_mm[2]);
        atomicMax(&mm[3], sh_mm[3]);
    }
}

// mm = {LLONG_MAX, LLONG_MIN, LLONG_MAX, LLONG_MIN}: empty key / payload ranges.
__global__ void rj_mm_init_kernel(long long* mm)
{
    if (threadIdx.x < 4) mm[threadIdx.x] = (threadIdx.x & 1) ? LLONG_MIN : LLONG_MAX;
}

// hist[b] = sum over the nrow rows of part[row * span + b], b < span: the
// CTAs' shared-memory histograms added column by column (coalesced and in a
// fixed order) instead of by atomics from every CTA on each bin.
__global__ void rj_hist_sum_kernel(const unsigned* __restrict__ part, int nrow, int span,
                                   unsigned long long* __restrict__ hist)
{
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= span) return;
    unsigned long long sum = 0;
    for (int r = 0; r < nrow; ++r) sum += part[(size_t)r * span + b];
    hist[b] = sum;
}

// Tiles of `tile` elements per segment, as an exclusive prefix (one thread;
// at most 2^8 segments): tiles[C] is the pass's tile count.  Counts are
// first clamped to their region's capacity, so a region that overflowed
// (its result is discarded and redone) is never read past its end.
__global__ void rj_tile_prefix_kernel(unsigned long long* __restrict__ count, const unsigned long long* __restrict__ cap,
                                      int C, int tile, unsigned long long* __restrict__ tiles)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    unsigned long long t = 0;
    tiles[0] = 0;
    for (int c = 0; c < C; ++c) {
        const unsigned long long n = count[c] < cap[c] ? count[c] : cap[c];
        count[c] = n;
        t += (n + tile - 1) / tile;
        tiles[c + 1] = t;
    }
}

// ---------------------------------------------------------------------------
// 2. Tile partition pass with exact offsets.  The input is a sequence of
// segments (one for the first pass; the coarse partitions for the second);
// tiles never straddle a segment.  Output bin of a tuple = (segment <<
// lbits) | ((rj_hash(key) >> shift) & mask).

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
    // Range mode (nsplit > 0): bin = number of splitters <= key among the
    // segment's nsplit splitters, split + seg * 2^lbits (one segment: split).
    const long long* split;
    int nsplit;
    // Packed elements: frame of the 8-byte words, and the flag set when a
    // 16-byte input tuple falls outside it.
    unsigned long long kbase, pbase;
    unsigned* frame;
    // Model mode (the kernel's RJ_MODE_MODEL instances): the bin bits come
    // from the learned model's code (rj_model_code) instead of the key's hash.
    RJModel model;
};

// Element formats: a pass reads 16-byte tuples (the relation, or unpacked
// intermediates) or packed 8-byte words, and writes either.  Packed input
// tiles hold 4096 words (bins of at most 2^8, so the staged bin index is
// one byte); 16-byte tiles hold 2048 tuples.  Both fit two CTAs per SM.
template <bool IN8, bool OUT8>
struct RJFmt {
    using In = typename std::conditional<IN8, unsigned long long, longlong2>::type;
    using Out = typename std::conditional<OUT8, unsigned long long, longlong2>::type;
    using Bin = typename std::conditional<IN8, unsigned char, unsigned short>::type;
    static constexpr int TILE = IN8 ? RJ_TILE8 : RJ_TILE;
};

__device__ __forceinline__ long long rj_key(const longlong2& t, unsigned long long) { return t.x; }
__device__ __forceinline__ long long rj_key(unsigned long long w, unsigned long long kbase)
{
    return (long long)(kbase + (w & 0xFFFFFFFFULL));
}

struct RJTileRange {
    long long begin, end;
    int seg;
};

// The segment of the tiles one CTA issues, kept in the issuing thread's
// registers.  A CTA's tiles come in increasing order, so the segment only
// moves forward: most tiles stay in the current segment and need no global
// load; a tile past its end steps forward (over empty segments too) and
// loads the new segment's bounds.  Over a whole pass a CTA reads each
// segment's bounds at most once.
struct RJSegCursor {
    int seg;               // -1 before the first tile
    long long t0, t1;      // seg_tile0[seg], seg_tile0[seg + 1]
    long long start, end;  // the segment's elements in `in`
};

template <int TILE>
__device__ RJTileRange rj_tile_range(const RJPass& a, RJSegCursor& c, long long tile)
{
    if (tile >= c.t1) {
        int s = c.seg < 0 ? 0 : c.seg + 1;
        long long t1 = (long long)a.seg_tile0[s + 1];
        while (tile >= t1 && s + 1 < a.nseg) t1 = (long long)a.seg_tile0[++s + 1];
        c.seg = s;
        c.t0 = (long long)a.seg_tile0[s];
        c.t1 = t1;
        c.start = (long long)a.seg_start[s];
        c.end = a.seg_count ? c.start + (long long)a.seg_count[s] : (long long)a.seg_start[s + 1];
    }
    RJTileRange r;
    r.seg = c.seg;
    r.begin = c.start + (tile - c.t0) * TILE;
    r.end = min(r.begin + TILE, c.end);
    return r;
}

// Shared memory of one partition CTA: a ring of RJ_STAGES input tiles that
// bulk copies fill ahead of use, the grouped (staged) tile, and per-bin
// counters.
template <bool IN8, bool OUT8>
struct RJPartSmem {
    using F = RJFmt<IN8, OUT8>;
    typename F::In in[RJ_STAGES][F::TILE];
    typename F::Out stage[F::TILE];
    typename F::Bin stage_bin[F::TILE];
    unsigned hist[RJ_LMAX];
    unsigned loff[RJ_LMAX];
    unsigned long long gdelta[RJ_LMAX];  // output position of staged slot i = gdelta[bin] + i
    uint64_t bar[RJ_STAGES];
    RJTileRange info[RJ_STAGES];
    unsigned warp_tot[32];
    unsigned total;  // elements of the current tile (scan by warp 0)
    long long split[2][RJ_SPLIT_MAX];  // range mode: the splitters of this tile and the next
    int ok;
};
static_assert(2 * (sizeof(RJPartSmem<false, false>) + 1024) <= 233472, "two partition CTAs per SM");
static_assert(2 * (sizeof(RJPartSmem<false, true>) + 1024) <= 233472, "two partition CTAs per SM");
static_assert(2 * (sizeof(RJPartSmem<true, true>) + 1024) <= 233472, "two partition CTAs per SM");

__device__ __forceinline__ unsigned rj_range_bin(const long long* sp, int n, long long k)
{
    int lo = 0;
    while (n > 0) {
        const int half = n >> 1;
        if (k >= sp[lo + half]) {
            lo += half + 1;
            n -= half + 1;
        } else {
            n = half;
        }
    }
    return (unsigned)lo;
}

// All threads: the splitters of segment seg into dst.
template <int THREADS>
__device__ __forceinline__ void rj_load_split(const RJPass& a, long long* dst, int seg)
{
    const long long* src = a.split + (a.nseg > 1 ? ((long long)seg << a.lbits) : 0);
    for (int i = threadIdx.x; i < a.nsplit; i += THREADS) dst[i] = src[i];
}

// Histogram of range bins of in[0], in[step], ...: fine bin = coarse bin
// (among C - 1 coarse splitters held in shared memory) * 2^sub + bin among
// that coarse range's 2^sub - 1 fine splitters (read from global memory).
__global__ void __launch_bounds__(1024) rj_hist_range_kernel(const longlong2* __restrict__ in, int64_t n, int64_t step,
                                                             int CB, int sub, const long long* __restrict__ csplit,
                                                             const long long* __restrict__ fsplit,
                                                             unsigned* __restrict__ part)
{
    extern __shared__ __align__(16) unsigned char rj_hr_raw[];
    const int F = 1 << (CB + sub), C = 1 << CB, L = 1 << sub;
    long long* cs = (long long*)rj_hr_raw;
    unsigned* h = (unsigned*)(cs + RJ_SPLIT_MAX);
    for (int b = threadIdx.x; b < F; b += blockDim.x) h[b] = 0;
    for (int i = threadIdx.x; i < C - 1; i += blockDim.x) cs[i] = csplit[i];
    __syncthreads();
    const int64_t m = (n + step - 1) / step;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += stride) {
        const long long k = __ldcs(&in[i * step]).x;
        unsigned f = rj_range_bin(cs, C - 1, k);
        if (sub) f = (f << sub) | rj_range_bin(fsplit + ((long long)f << sub), L - 1, k);
        atomicAdd(&h[f], 1u);
    }
    __syncthreads();
    unsigned* row = part + (size_t)blockIdx.x * F;
    for (int b = threadIdx.x; b < F; b += blockDim.x) row[b] = h[b];
}

// Thread 0: starts the bulk copy of tile `tile` into ring slot `slot`.
// Packed tiles start at an even word (regions and tiles are even), and the
// copy is rounded up to 16 bytes: at most one word past the tile, inside
// the buffer's 16-byte tail, which is never used as data.
template <bool IN8, bool OUT8>
__device__ __forceinline__ void rj_issue_tile(const RJPass& a, RJPartSmem<IN8, OUT8>& sm, RJSegCursor& cur, int slot,
                                              long long tile)
{
    using F = RJFmt<IN8, OUT8>;
    const RJTileRange r = rj_tile_range<F::TILE>(a, cur, tile);
    sm.info[slot] = r;
    const unsigned bytes = ((unsigned)(r.end - r.begin) * (unsigned)sizeof(typename F::In) + 15u) & ~15u;
    mbar_arrive_expect_tx(&sm.bar[slot], bytes);
    bulk_load(sm.in[slot], reinterpret_cast<const typename F::In*>(a.in) + r.begin, bytes, &sm.bar[slot]);
}

// How a pass computes a tuple's bin, fixed per kernel instance so that no
// per-tuple branch chooses it.
enum RJMode { RJ_MODE_HASH = 0, RJ_MODE_MODEL = 1, RJ_MODE_RANGE = 2 };

// Threads of a partition CTA: 256 for hash bins of 16-byte tuples, 512
// otherwise.  The learned model's bins and splitter searches wait on loads
// (the key's leaf, the splitters) and measured faster with the larger CTA:
// MPSM partition phase at theta 1.0, 8.05 against 7.18 ms (model) and 10.59
// against 10.14 ms (sampled splitters) with 256 threads.
template <bool IN8, int MODE>
constexpr int rj_pt_threads()
{
    return (IN8 || MODE != RJ_MODE_HASH) ? RJ_PT_THREADS8 : RJ_PT_THREADS16;
}

template <bool IN8, bool OUT8, int MODE>
__global__ void __launch_bounds__(rj_pt_threads<IN8, MODE>(), PYG_RJ_PT_MINB) rj_partition_kernel(RJPass a, long long ntiles)
{
    using F = RJFmt<IN8, OUT8>;
    using Out = typename F::Out;
    if (a.ntiles_dev) ntiles = (long long)*a.ntiles_dev;
    extern __shared__ __align__(128) unsigned char rj_pt_raw[];
    RJPartSmem<IN8, OUT8>& sm = *reinterpret_cast<RJPartSmem<IN8, OUT8>*>(rj_pt_raw);
    constexpr int T = rj_pt_threads<IN8, MODE>();
    constexpr int PER = F::TILE / T;
    const int L = 1 << a.lbits;
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    Out* out = reinterpret_cast<Out*>(a.out);
    bool miss = false;  // a 16-byte tuple outside the packed frame
    RJSegCursor segc{-1, -1, -1, 0, 0};  // thread 0: segment of the tiles it issues
    for (int b = tid; b < RJ_LMAX; b += T) sm.hist[b] = 0;
    if (tid == 0) {
        for (int s = 0; s < RJ_STAGES; ++s) mbar_init(&sm.bar[s], 1);
        mbar_fence_init();
        for (int s = 0; s < RJ_STAGES; ++s)
            if (blockIdx.x + (long long)s * gridDim.x < ntiles)
                rj_issue_tile(a, sm, segc, s, blockIdx.x + (long long)s * gridDim.x);
        sm.ok = 1;
    }
    __syncthreads();
    if (a.nsplit) {
        rj_load_split<T>(a, sm.split[0], sm.info[0].seg);
        __syncthreads();
    }
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
        Out t[PER];
        unsigned bin[PER], rank[PER];
        auto bin_rank = [&](int j, bool valid) {
            const unsigned i = j * T + tid;
            bin[j] = 0xFFFFFFFFu;
            if (valid) {
                const typename F::In e = sm.in[slot][i];
                const long long key = rj_key(e, a.kbase);
                if constexpr (IN8 || !OUT8) {
                    t[j] = e;
                } else {
                    // Pack: (key - kbase) | (payload - pbase) << 32.
                    const unsigned long long dk = (unsigned long long)e.x - a.kbase;
                    const unsigned long long dp = (unsigned long long)e.y - a.pbase;
                    miss |= ((dk | dp) >> 32) != 0;
                    t[j] = (dk & 0xFFFFFFFFULL) | (dp << 32);
                }
                // 16-byte passes test nsplit at run time, the hash instance
                // too (it never has splitters): compiled without the test,
                // the first pass of the 2^30-tuple probe side measured 7.51
                // against 6.95 ms.
                if constexpr (MODE == RJ_MODE_MODEL)
                    bin[j] = rj_bin(rj_model_code(a.model, key), a.shift, a.mask);
                else if constexpr (!IN8)
                    bin[j] = a.nsplit ? rj_range_bin(sm.split[a.nseg > 1 ? (k & 1) : 0], a.nsplit, key)
                                      : rj_bin(rj_hash((uint64_t)key), a.shift, a.mask);
                else if constexpr (MODE == RJ_MODE_RANGE)
                    bin[j] = rj_range_bin(sm.split[a.nseg > 1 ? (k & 1) : 0], a.nsplit, key);
                else
                    bin[j] = rj_bin(rj_hash((uint64_t)key), a.shift, a.mask);
            }
            // Skewed keys put many lanes of a warp into one bin: when at
            // least 8 lanes share lane 0's bin, they take their ranks from
            // one atomic (lane order), the others one atomic each.
            const unsigned b0 = __shfl_sync(0xffffffffu, bin[j], 0);
            const unsigned m0 = __ballot_sync(0xffffffffu, valid && bin[j] == b0);
            if (__popc(m0) >= 8) {
                unsigned base = 0;
                if (lane == 0) base = atomicAdd(&sm.hist[b0], (unsigned)__popc(m0));
                base = __shfl_sync(0xffffffffu, base, 0);
                if ((m0 >> lane) & 1) rank[j] = base + __popc(m0 & ((1u << lane) - 1u));
                else if (valid) rank[j] = atomicAdd(&sm.hist[bin[j]], 1u);
            } else if (valid) {
                rank[j] = atomicAdd(&sm.hist[bin[j]], 1u);
            }
        };
        // Packed passes: full tiles (all but the last of each segment) skip
        // the per-tuple bounds test (second pass of the 2^30-tuple probe side
        // 4.94 -> 4.68 ms).  16-byte passes keep one loop: there the second
        // copy of the loop measured slower (7.03 -> 8.15 ms; 127 registers).
        if (IN8 && landed && n == (unsigned)F::TILE) {
#pragma unroll
            for (int j = 0; j < PER; ++j) bin_rank(j, true);
        } else {
#pragma unroll
            for (int j = 0; j < PER; ++j) bin_rank(j, landed && j * T + tid < n);
        }
        __syncthreads();  // A: histogram complete
        if (!sm.ok) break;
        // (2) In-tile offsets of the bins, reservation of each non-empty
        // bin's run (one global atomic) and reset of its counter.  Thread
        // tid handles bins tid + q x T.  With a thread per bin (packed
        // passes, 512 threads) the whole CTA scans; with fewer threads than
        // bins (16-byte passes, 256 threads) warp 0 scans alone and the
        // others go on to barrier C: measured 6.9 against 12.7 ms for the
        // 2^30-tuple probe side's first pass (one barrier fewer per tile,
        // where only 16 warps share an SM).
        constexpr int BPT = (RJ_LMAX + T - 1) / T;
        unsigned c[BPT], ex[BPT], total;
        // The reservation's result (a global atomic, about a microsecond
        // away) is first needed after the tile is staged.
        unsigned long long resv[BPT], bstart[BPT], bcap[BPT];
        auto reserve = [&](int q) {
            const int b = tid + q * T;
            resv[q] = 0;
            bstart[q] = 0;
            bcap[q] = ~0ULL;
            if (b < L) {
                if (c[q]) {
                    const unsigned ob = ((unsigned)cur.seg << a.lbits) | (unsigned)b;
                    bstart[q] = a.bin_start[ob];
                    if (a.bin_cap) bcap[q] = a.bin_cap[ob];
                    resv[q] = atomicAdd(&a.cursor[ob], (unsigned long long)c[q]);
                }
                sm.hist[b] = 0;
            }
        };
        if constexpr (BPT == 1) {
            c[0] = tid < L ? sm.hist[tid] : 0u;
            unsigned incl = c[0];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
                if (lane >= o) incl += v;
            }
            if (lane == 31) sm.warp_tot[w] = incl;
            __syncthreads();  // B
            // Prefix over the warp totals, by one more shuffle scan per warp.
            constexpr int NW = T / 32;
            const unsigned wt = lane < NW ? sm.warp_tot[lane] : 0u;
            unsigned wincl = wt;
#pragma unroll
            for (int o = 1; o < NW; o <<= 1) {
                const unsigned v = __shfl_up_sync(0xffffffffu, wincl, o);
                if (lane >= o) wincl += v;
            }
            ex[0] = incl - c[0] + __shfl_sync(0xffffffffu, wincl - wt, w);
            total = __shfl_sync(0xffffffffu, wincl, NW - 1);
            if (tid < L) sm.loff[tid] = ex[0];
            reserve(0);
            __syncthreads();  // C: in-tile offsets ready
        } else {
            // Lane l of warp 0 owns the PB consecutive bins from l x PB.
            if (w == 0) {
                const int PB = (L + 31) >> 5;
                const int b0 = lane * PB;
                unsigned sum = 0;
                for (int q = 0; q < PB; ++q)
                    if (b0 + q < L) sum += sm.hist[b0 + q];
                unsigned incl = sum;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const unsigned v = __shfl_up_sync(0xffffffffu, incl, o);
                    if (lane >= o) incl += v;
                }
                unsigned run = incl - sum;
                for (int q = 0; q < PB; ++q)
                    if (b0 + q < L) {
                        sm.loff[b0 + q] = run;
                        run += sm.hist[b0 + q];
                    }
                if (lane == 31) sm.total = incl;
            }
            __syncthreads();  // C: in-tile offsets ready
            total = sm.total;
#pragma unroll
            for (int q = 0; q < BPT; ++q) {
                const int b = tid + q * T;
                c[q] = b < L ? sm.hist[b] : 0u;
                ex[q] = b < L ? sm.loff[b] : 0u;
                reserve(q);
            }
        }
        // (3) Group the tile by bin in shared memory.
#pragma unroll
        for (int j = 0; j < PER; ++j)
            if (bin[j] != 0xFFFFFFFFu) {
                const unsigned s = sm.loff[bin[j]] + rank[j];
                sm.stage[s] = t[j];
                sm.stage_bin[s] = (typename F::Bin)bin[j];
            }
        // Range mode over several segments: the next tile's splitters
        // (its copy was issued a tile ago, so its segment is known).
        if (a.nsplit && a.nseg > 1 && tile + gridDim.x < ntiles)
            rj_load_split<T>(a, sm.split[(k + 1) & 1], sm.info[(k + 1) % RJ_STAGES].seg);
        // Per bin, the output position of staged slot i is gdelta + i.
#pragma unroll
        for (int q = 0; q < BPT; ++q) {
            const int b = tid + q * T;
            if (b < L && c[q]) {
                unsigned long long gd = bstart[q] + resv[q] - ex[q];
                if (resv[q] + c[q] > bcap[q]) {  // outgrew its region: not written; the host redoes the pass exactly
                    atomicOr(a.ovf, 1u);
                    gd = kSkipRun;
                }
                sm.gdelta[b] = gd;
            }
        }
        __syncthreads();  // D: ring slot consumed, stage and global offsets complete
        if (tid == 0) {
            const long long nt = tile + (long long)RJ_STAGES * gridDim.x;
            if (nt < ntiles) {
                fence_proxy_async_smem();
                rj_issue_tile(a, sm, segc, slot, nt);
            }
        }
        // (4) Write each bin's run contiguously (total <= PER x T: PER
        // unrolled steps cover the tile and their loads overlap).
#pragma unroll
        for (int j = 0; j < PER; ++j) {
            const unsigned i = j * T + tid;
            if (i < total) {
                const unsigned long long gd = sm.gdelta[sm.stage_bin[i]];
                if (gd != kSkipRun) __stcs(&out[gd + i], sm.stage[i]);
            }
        }
    }
    __syncthreads();
    if (tid == 0 && !sm.ok) atomicOr(a.err, 1u);
    if (miss) atomicOr(a.frame, 1u);
}


namespace {

template <bool IN8, bool OUT8, int MODE>
int launch_pass_t(pyg_ctx* ctx, const RJPass& p, long long ntiles)
{
    auto fn = rj_partition_kernel<IN8, OUT8, MODE>;
    const size_t smem = sizeof(RJPartSmem<IN8, OUT8>);
    PYG_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    constexpr int T = rj_pt_threads<IN8, MODE>();
    PYG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, T, smem));
    if (per_sm < 1) per_sm = 1;
    long long grid = std::min<long long>(ntiles, (long long)ctx->sm_count * per_sm);
    fn<<<(unsigned)grid, T, smem, ctx->stream>>>(p, ntiles);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

// One pass: 16-byte tuples in and out, 16-byte tuples in and packed words
// out (the first pass of a packed layout), or packed words in and out.
template <int MODE>
int launch_pass_m(pyg_ctx* ctx, const RJPass& p, long long ntiles, bool in8, bool out8)
{
    if (in8) return launch_pass_t<true, true, MODE>(ctx, p, ntiles);
    if (out8) return launch_pass_t<false, true, MODE>(ctx, p, ntiles);
    return launch_pass_t<false, false, MODE>(ctx, p, ntiles);
}

int launch_pass(pyg_ctx* ctx, const RJPass& p, long long ntiles, bool in8, bool out8)
{
    if (ntiles <= 0) return PYG_OK;
    if (p.model.leaf) return launch_pass_m<RJ_MODE_MODEL>(ctx, p, ntiles, in8, out8);
    if (p.nsplit) return launch_pass_m<RJ_MODE_RANGE>(ctx, p, ntiles, in8, out8);
    return launch_pass_m<RJ_MODE_HASH>(ctx, p, ntiles, in8, out8);
}

// Host-side layout of one relation's partitions.  Exact layouts come from a
// full histogram (dense, contiguous partitions); sampled layouts size each
// partition's region from a strided sample with six standard deviations of

}  // namespace

void layout_exact(const std::vector<unsigned long long>& h, int C, int sub, RJLayout& L, bool pack)
{
    const size_t F = h.size();
    L.sampled = false;
    L.packed = pack;
    // Packed regions are rounded up to an even number of words.
    auto sz = [&](unsigned long long c) { return pack ? (c + 1) & ~1ULL : c; };
    L.fstart.assign(F + 1, 0);
    for (size_t f = 0; f < F; ++f) L.fstart[f + 1] = L.fstart[f] + sz(h[f]);
    L.cstart.assign(C + 1, 0);
    for (int c = 0; c <= C; ++c) L.cstart[c] = L.fstart[(size_t)c << sub];
    L.fcap.clear();
    L.ccap.clear();
    L.tiles2.assign(C + 1, 0);
    if (pack) {
        // The second pass's tiles come from the first pass's cursors (the
        // exact counts), formed on the device as for sampled layouts; the
        // region sizes bound them.
        L.ccap.assign(C, 0);
        L.tiles2_max = 0;
        for (int c = 0; c < C; ++c) {
            L.ccap[c] = L.cstart[c + 1] - L.cstart[c];
            L.tiles2_max += (L.ccap[c] + RJ_TILE8 - 1) / RJ_TILE8;
        }
    } else {
        for (int c = 0; c < C; ++c)
            L.tiles2[c + 1] = L.tiles2[c] + (L.cstart[c + 1] - L.cstart[c] + RJ_TILE - 1) / RJ_TILE;
        L.tiles2_max = L.tiles2[C];
    }
    L.count = h;
    L.p1 = L.p2 = L.fstart[F];
}

unsigned long long sampled_cap(unsigned long long c, long long step, unsigned long long extra)
{
    const double x = (double)c;
    return (unsigned long long)std::ceil((x + 6.0 * std::sqrt(x) + 8.0) * (double)step) + extra;
}

void layout_sampled(const std::vector<unsigned long long>& sc, long long step, int C, int sub, RJLayout& L,
                    bool pack)
{
    const size_t F = sc.size();
    L.sampled = true;
    L.packed = pack;
    auto sz = [&](unsigned long long c) { return pack ? (c + 1) & ~1ULL : c; };
    const int tile2 = pack ? RJ_TILE8 : RJ_TILE;
    L.fcap.assign(F, 0);
    L.fstart.assign(F + 1, 0);
    for (size_t f = 0; f < F; ++f) {
        L.fcap[f] = sz(sampled_cap(sc[f], step, 64));
        L.fstart[f + 1] = L.fstart[f] + L.fcap[f];
    }
    L.ccap.assign(C, 0);
    L.cstart.assign(C + 1, 0);
    L.tiles2_max = 0;
    for (int c = 0; c < C; ++c) {
        unsigned long long cc = 0;
        for (size_t f = (size_t)c << sub; f < (size_t)(c + 1) << sub; ++f) cc += sc[f];
        L.ccap[c] = sz(sampled_cap(cc, step, 1024));
        L.cstart[c + 1] = L.cstart[c] + L.ccap[c];
        L.tiles2_max += (L.ccap[c] + tile2 - 1) / tile2;
    }
    L.tiles2.clear();
    L.count.clear();
    L.p1 = L.cstart[C];
    L.p2 = L.fstart[F];
}

// A window [base, base + 2^32 - 1) centred on [lo, hi] (offset 2^32 - 1 is
// never used, so a join can take it as its empty-slot marker); a sampled
// range must leave at least 2^30 of margin on each side.
static bool frame_fit(long long lo, long long hi, bool exact, unsigned long long& base)
{
    if (hi < lo) {  // nothing was read
        base = 0;
        return true;
    }
    const unsigned long long span = (unsigned long long)hi - (unsigned long long)lo;
    if (span > (exact ? 0xFFFFFFFEULL : (1ULL << 31))) return false;
    base = (unsigned long long)lo - (0xFFFFFFFEULL - span) / 2;
    return true;
}

bool pack_frame(long long kmin, long long kmax, long long pmin, long long pmax, bool exact, RJLayout& L,
                const unsigned long long* key_base)
{
    unsigned long long kb = 0, pb = 0;
    if (key_base) {
        kb = *key_base;  // a frame shared with another relation, fitted to both ranges
    } else if (!frame_fit(kmin, kmax, exact, kb)) {
        return false;
    }
    if (!frame_fit(pmin, pmax, exact, pb)) return false;
    L.kbase = kb;
    L.pbase = pb;
    return true;
}

bool common_key_frame(const long long* mm0, bool exact0, const long long* mm1, bool exact1, unsigned long long* base)
{
    if (mm0[1] < mm0[0] || mm1[1] < mm1[0]) return false;
    const long long lo = std::min(mm0[0], mm1[0]), hi = std::max(mm0[1], mm1[1]);
    return frame_fit(lo, hi, exact0 && exact1, *base);
}

int upload_layout(pyg_ctx* ctx, const RJLayout& L, const RJSideDev& d, int F, int C, int64_t n)
{
    int rc;
    if ((rc = stage_h2d(ctx, d.fstart, L.fstart.data(), (size_t)(F + 1) * 8))) return rc;
    if ((rc = stage_h2d(ctx, d.cstart, L.cstart.data(), (size_t)(C + 1) * 8))) return rc;
    if (L.sampled && (rc = stage_h2d(ctx, d.fcap, L.fcap.data(), (size_t)F * 8))) return rc;
    if (L.sampled || L.packed) {
        if ((rc = stage_h2d(ctx, d.ccap, L.ccap.data(), (size_t)C * 8))) return rc;
    } else if ((rc = stage_h2d(ctx, d.tiles2, L.tiles2.data(), (size_t)(C + 1) * 8))) {
        return rc;
    }
    PYG_CUDA(cudaMemsetAsync(d.cur1, 0, (size_t)(C + F) * 8, ctx->stream));  // cur1 and cur2 are adjacent
    const unsigned long long w[4] = {0, (unsigned long long)n, 0, (unsigned long long)((n + RJ_TILE - 1) / RJ_TILE)};
    return stage_h2d(ctx, d.whole, w, sizeof(w));
}

// Runs the partition pass(es) of one relation into P1 (and P2).
int run_passes(pyg_ctx* ctx, const longlong2* in, int64_t n, const RJLayout& L, const RJSideDev& d, bool two, int FB,
               int CB, void* P1, void* P2, unsigned* err, unsigned* ovf, const long long* csplit,
               const long long* fsplit, unsigned* frame, cudaEvent_t between, const RJModel* model)
{
    const int C = 1 << CB, sub = FB - CB;
    if (L.packed && (!frame || csplit || (two && sub > 8))) {
        set_error("partition: packed layouts need a frame flag, hash bins and at most 2^8 second-pass bins");
        return PYG_ERR_ARG;
    }
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
    p.kbase = L.kbase;
    p.pbase = L.pbase;
    p.frame = frame;
    if (model) p.model = *model;
    if (csplit) {
        p.split = csplit;
        p.nsplit = C - 1;
    }
    int rc = launch_pass(ctx, p, (n + RJ_TILE - 1) / RJ_TILE, false, L.packed);
    if (rc || !two) return rc;
    if (between) cudaEventRecord(between, ctx->stream);
    long long ntiles2;
    if (L.sampled || L.packed) {
        // Second-pass segments are the first pass's regions, filled to the
        // counts its cursors reached; the tile prefix is formed on the device.
        rj_tile_prefix_kernel<<<1, 32, 0, ctx->stream>>>(d.cur1, d.ccap, C, L.packed ? RJ_TILE8 : RJ_TILE,
                                                          d.tiles2);
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
    if (fsplit) {
        p.split = fsplit;
        p.nsplit = (1 << sub) - 1;
    }
    return launch_pass(ctx, p, ntiles2, L.packed, L.packed);
}

int hist_launch(pyg_ctx* ctx, const longlong2* in, int64_t n, int64_t step, int FB, unsigned long long* hist,
                long long* mm, const RJModel* model)
{
    // At most 2^15 counters (128 KB) per launch: 2^16 bins take two.
    const int F = 1 << FB, span = F < (1 << 15) ? F : (1 << 15);
    const size_t hsm = (size_t)4 * span;
    auto kern = model ? rj_hist_kernel<true> : rj_hist_kernel<false>;
    const RJModel none;
    PYG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
    int per = 0;
    PYG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kern, 1024, hsm));
    if (per < 1) per = 1;
    const int64_t m = (n + step - 1) / step;
    const int64_t want = (m + 1024 * 8 - 1) / (1024 * 8);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->sm_count * per));
    unsigned* part = nullptr;
    int rc;
    if ((rc = dalloc(ctx, (void**)&part, (size_t)grid * span * 4))) return rc;
    if (mm) {
        rj_mm_init_kernel<<<1, 32, 0, ctx->stream>>>(mm);
        PYG_LAUNCHED(ctx);
    }
    for (int base = 0; base < F; base += span) {
        // The key and payload ranges are taken in the first launch only.
        kern<<<grid, 1024, hsm, ctx->stream>>>(in, n, step, FB, base, span, part, base ? nullptr : mm,
                                                model ? *model : none);
        PYG_LAUNCHED(ctx);
        rj_hist_sum_kernel<<<(span + 255) / 256, 256, 0, ctx->stream>>>(part, grid, span, hist + base);
        PYG_LAUNCHED(ctx);
    }
    dfree(ctx, part);
    return PYG_OK;
}

int hist_launch_range(pyg_ctx* ctx, const longlong2* in, int64_t n, int64_t step, int CB, int sub,
                      const long long* csplit, const long long* fsplit, unsigned long long* hist)
{
    const int F = 1 << (CB + sub);
    const size_t hsm = (size_t)RJ_SPLIT_MAX * 8 + (size_t)4 * F;
    PYG_CUDA(cudaFuncSetAttribute(rj_hist_range_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsm));
    int per = 0;
    PYG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, rj_hist_range_kernel, 1024, hsm));
    if (per < 1) per = 1;
    const int64_t m = (n + step - 1) / step;
    const int64_t want = (m + 1024 * 8 - 1) / (1024 * 8);
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(want, (int64_t)ctx->sm_count * per));
    unsigned* part = nullptr;
    int rc;
    if ((rc = dalloc(ctx, (void**)&part, (size_t)grid * F * 4))) return rc;
    rj_hist_range_kernel<<<grid, 1024, hsm, ctx->stream>>>(in, n, step, CB, sub, csplit, fsplit, part);
    PYG_LAUNCHED(ctx);
    rj_hist_sum_kernel<<<(F + 255) / 256, 256, 0, ctx->stream>>>(part, grid, F, hist);
    PYG_LAUNCHED(ctx);
    dfree(ctx, part);
    return PYG_OK;
}

int rp_partition_sides(pyg_ctx* ctx, RPSide* sd, int ns, int FB, bool two, unsigned* flags, unsigned* hflags,
                       cudaEvent_t hist_done, bool share_key_frame)
{
    // Coarse bits of the first of two passes.  Unpacked layouts split FB
    // evenly (2048-tuple tiles); packed layouts keep the second pass at 2^8
    // bins, so that its 4096-word tiles use one-byte bin indexes and both
    // passes write runs of about 16 words.  The unpacked split has at least
    // as many coarse partitions, so its metadata size covers both.
    auto coarse_bits = [&](bool packed) { return !two ? FB : (packed ? std::max(1, FB - 8) : (FB + 1) / 2); };
    const int F = 1 << FB;
    const size_t side = RJSideDev::words(F, 1 << coarse_bits(false));
    const size_t per = side + F + 4;  // metadata, histogram, {kmin, kmax, pmin, pmax}
    if (ns < 1 || ns > 2 || (size_t)ns * (F + 4) * 8 > kPinnedStageBytes) {
        set_error("partition: %d relations of 2^%d partitions exceed the staging area", ns, FB);
        return PYG_ERR_ARG;
    }
    // Per-partition counts come back through pinned memory, so that both
    // relations' histograms cost one host round trip and both relations'
    // passes another.
    unsigned long long* hh = (unsigned long long*)((char*)ctx->pinned + kPinnedScalarBytes);
    unsigned long long* meta = nullptr;
    RJSideDev d[2];
    int CBs[2] = {FB, FB};
    bool sample[2] = {false, false};
    int rc = PYG_OK;
    for (int s = 0; s < ns; ++s) sd[s].P1 = sd[s].P2 = nullptr;
    auto hist_at = [&](int s) { return meta + (size_t)s * per + side; };
    auto hh_at = [&](int s) { return hh + (size_t)s * (F + 4); };
    auto hist_of = [&](int s, int64_t st) {
        if (sd[s].csplit) {
            const int cb = coarse_bits(false);
            return hist_launch_range(ctx, sd[s].in, sd[s].n, st, cb, FB - cb, sd[s].csplit, sd[s].fsplit, hist_at(s));
        }
        return hist_launch(ctx, sd[s].in, sd[s].n, st, FB, hist_at(s),
                           sd[s].allow_pack ? (long long*)(hist_at(s) + F) : nullptr, sd[s].model);
    };
    // Layout of relation s from host counts h (F counts, then the key and
    // payload ranges): packed when the caller allows it and a frame fits.
    auto form = [&](int s, const unsigned long long* h, int64_t st, bool exact, const unsigned long long* kb) {
        RJLayout& L = sd[s].L;
        const long long* mm = (const long long*)(h + F);
        const bool pack =
            sd[s].allow_pack && !sd[s].csplit && pack_frame(mm[0], mm[1], mm[2], mm[3], exact, L, kb);
        CBs[s] = coarse_bits(pack);
        const int C = 1 << CBs[s], sub = FB - CBs[s];
        std::vector<unsigned long long> hv(h, h + F);
        if (exact) layout_exact(hv, C, sub, L, pack);
        else layout_sampled(hv, st, C, sub, L, pack);
        d[s].carve(meta + (size_t)s * per, F, C);
    };
    auto launch = [&](int s) {
        const RJLayout& L = sd[s].L;
        int r;
        if ((r = upload_layout(ctx, L, d[s], F, 1 << CBs[s], sd[s].n))) return r;
        dfree(ctx, sd[s].P1);
        dfree(ctx, sd[s].P2);
        sd[s].P1 = sd[s].P2 = nullptr;
        if ((r = dalloc(ctx, &sd[s].P1, pass_bytes(L, L.p1)))) return r;
        if (two && (r = dalloc(ctx, &sd[s].P2, pass_bytes(L, L.p2)))) return r;
        if (sd[s].begin) cudaEventRecord(sd[s].begin, ctx->stream);
        if ((r = run_passes(ctx, sd[s].in, sd[s].n, L, d[s], two, FB, CBs[s], sd[s].P1, sd[s].P2, flags + 4 * s,
                            flags + 4 * s + 1, sd[s].csplit, sd[s].fsplit, flags + 4 * s + 2, sd[s].mid,
                            sd[s].model)))
            return r;
        if (sd[s].done) cudaEventRecord(sd[s].done, ctx->stream);
        return PYG_OK;
    };
    do {
        if ((rc = dalloc(ctx, (void**)&meta, per * 8 * ns))) break;
        PYG_CUDA(cudaMemsetAsync(flags, 0, (size_t)16 * ns, ctx->stream));
        int64_t step[2] = {1, 1};
        for (int s = 0; s < ns && !rc; ++s) {
            sample[s] = sd[s].allow_sample && two && sd[s].n >= ((int64_t)1 << 25);
            step[s] = sample[s] ? std::max<int64_t>(1, sd[s].n >> RJ_SAMPLE_LOG2) : 1;
            if ((rc = hist_of(s, step[s]))) break;
            sd[s].hist_tuples = (sd[s].n + step[s] - 1) / step[s];
        }
        if (rc) break;
        if (hist_done) cudaEventRecord(hist_done, ctx->stream);
        for (int s = 0; s < ns; ++s)
            PYG_CUDA(cudaMemcpyAsync(hh_at(s), hist_at(s), (size_t)(F + 4) * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        stage_reset(ctx);
        // One key frame for both relations when asked and both ranges fit
        // in it, so that their packed words compare by key offset.
        unsigned long long ckb = 0;
        const bool common = share_key_frame && ns == 2 && sd[0].allow_pack && sd[1].allow_pack && !sd[0].csplit &&
                            !sd[1].csplit &&
                            common_key_frame((const long long*)(hh_at(0) + F), !sample[0],
                                             (const long long*)(hh_at(1) + F), !sample[1], &ckb);
        // The second relation's layout is formed while the first one's
        // passes run.
        for (int s = 0; s < ns && !rc; ++s) {
            form(s, hh_at(s), step[s], !sample[s], common ? &ckb : nullptr);
            rc = launch(s);
        }
        if (rc) break;
        PYG_CUDA(cudaMemcpyAsync(hflags, flags, (size_t)16 * ns, cudaMemcpyDeviceToHost, ctx->stream));
        for (int s = 0; s < ns; ++s)
            if (sd[s].L.sampled)
                PYG_CUDA(cudaMemcpyAsync(hh_at(s), d[s].cur2, (size_t)F * 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        for (int s = 0; s < ns && !rc; ++s) {
            if (hflags[4 * s]) {
                set_error("partition: a tile copy did not complete in time");
                rc = PYG_ERR_TIMEOUT;
                break;
            }
            if (sd[s].L.sampled) sd[s].L.count.assign(hh_at(s), hh_at(s) + F);
            if (!hflags[4 * s + 1] && !hflags[4 * s + 2]) continue;
            // A sampled region overflowed, or a tuple fell outside a frame
            // taken from the sample: redo this relation from an exact
            // histogram, whose key and payload ranges are exact too (exact
            // regions cannot overflow, and an exact frame misses nothing).
            sd[s].overflowed = true;
            sd[s].done = sd[s].begin = sd[s].mid = nullptr;  // the redo's time is not attributed to the relation
            if ((rc = hist_of(s, 1))) break;
            PYG_CUDA(cudaMemcpyAsync(hh_at(s), hist_at(s), (size_t)(F + 4) * 8, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            form(s, hh_at(s), 1, true, nullptr);
            PYG_CUDA(cudaMemsetAsync(flags + 4 * s, 0, 16, ctx->stream));
            if ((rc = launch(s))) break;
            PYG_CUDA(cudaMemcpyAsync(hflags + 4 * s, flags + 4 * s, 16, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            if (hflags[4 * s]) {
                set_error("partition: a tile copy did not complete in time");
                rc = PYG_ERR_TIMEOUT;
            } else if (hflags[4 * s + 1] || hflags[4 * s + 2]) {
                set_error("partition: an exact layout overflowed a region or missed its frame");
                rc = PYG_ERR_CAPACITY;
            }
        }
    } while (0);
    dfree(ctx, meta);
    if (rc) {
        for (int s = 0; s < ns; ++s) {
            dfree(ctx, sd[s].P1);
            dfree(ctx, sd[s].P2);
            sd[s].P1 = sd[s].P2 = nullptr;
        }
    }
    return rc;
}

int rp_partition(pyg_ctx* ctx, const longlong2* in, int64_t n, int FB, bool two, bool allow_sample,
                 const long long* csplit, const long long* fsplit, RJLayout& L, void** P1, void** P2,
                 unsigned* flags, unsigned* hflags, float* hist_ms, int64_t* hist_tuples)
{
    RPSide s;
    s.in = in;
    s.n = n;
    s.allow_sample = allow_sample;
    s.csplit = csplit;
    s.fsplit = fsplit;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (hist_ms) {
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, ctx->stream);
    }
    const int rc = rp_partition_sides(ctx, &s, 1, FB, two, flags, hflags, e1);
    if (hist_ms) {
        *hist_ms = 0.f;
        if (!rc) cudaEventElapsedTime(hist_ms, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    if (hist_tuples) *hist_tuples = s.hist_tuples;
    L = std::move(s.L);
    *P1 = s.P1;
    *P2 = s.P2;
    return rc;
}

}  // namespace pyg
