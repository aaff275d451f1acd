// MPSM join + aggregation of 16-byte (int64 key, int64 payload) device
// relations: the aggregate sink of pyg_mpsm_join_agg on its common shape.
//
//   1. splitters   2^FB - 1 range splitters from the caller (equal-width,
//                  sample quantiles or the learned CDF model), chosen so a
//                  range holds a few thousand probe tuples.
//   2. partition   both relations range-partitioned by those splitters with
//                  the radix operators' bulk-copy partitioner (radixpart.cu,
//                  two passes above 2^8 ranges): splitter-search bins, or,
//                  for a learned model, the model's own bins (rj_model_bin,
//                  the same ranges without a search), whose intermediates
//                  are packed 8-byte words when the key and payload ranges
//                  allow; the merge decodes them on load.
//   3. sort+merge  persistent CTAs take (range, build chunk, probe chunk)
//                  items.  A range whose splitters bound it to at most
//                  MP16_DSPAN key values is sorted by counting: the build
//                  chunk (the whole range) is binned by key offset in shared
//                  memory, each bin holding its key's count and payload sum,
//                  and a probe tuple finds its key's run at its offset.  Any
//                  other range is sorted in chunks of <= 4096 by a bitonic
//                  network with a prefix sum of the payloads, and each probe
//                  tuple is merged into the run by a lower-bound search.
//                  Either way a probe tuple adds its key's run's count and
//                  payload sum.
// Build keys equal to INT64_MAX (the sort's padding value) are counted on
// the side per item, as are the probe tuples that match them.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "mpsm16.cuh"
#include "radixpart.cuh"

namespace pyg {

constexpr int MP16_THREADS = 512;          // two CTAs per SM: one sorts while the other merges
constexpr int MP16_RCHUNK = 4096;         // build tuples sorted per work item
constexpr int64_t MP16_SCHUNK = 1 << 16;  // probe tuples per work item
constexpr int MP16_SMEM = MP16_RCHUNK * 8 * 2 + (MP16_RCHUNK + 1) * 8;
constexpr long long kPadKey = 0x7FFFFFFFFFFFFFFFLL;
// Largest key span of a range sorted by counting: 4-byte counts and 8-byte
// sums per key value, 96 KB, inside the bitonic path's shared memory.
constexpr unsigned MP16_DSPAN = 8192;
static_assert(MP16_DSPAN * 12 <= MP16_SMEM, "counting bins fit the sort's shared memory");

struct Mp16Item {
    unsigned long long r0, s0;
    unsigned rn, sn;
    long long lo;   // counting sort: the range's first key value
    unsigned span;  // its number of key values (0: bitonic sort)
    unsigned pad;
};

struct Mp16Args {
    const void* R;  // 16-byte tuples, or packed 8-byte words (frame rk / rp, sk / sp)
    const void* S;
    unsigned long long rk, rp, sk, sp;
    const Mp16Item* items;
    long long nitems;
    unsigned* next;
    unsigned long long* acc;  // count, build sum, probe sum
    unsigned* bad;            // a key outside its range's span (never set by a correct partition)
};

// Element i of a partitioned relation: a 16-byte tuple, or a packed word
// (key - kb) | (payload - pb) << 32 decoded back to the tuple (exact).
// CS: a streamed read (evict first).
template <bool P, bool CS>
__device__ __forceinline__ longlong2 mp16_elem(const void* base, unsigned long long i, unsigned long long kb,
                                               unsigned long long pb)
{
    if constexpr (P) {
        const unsigned long long* q = reinterpret_cast<const unsigned long long*>(base) + i;
        const unsigned long long w = CS ? __ldcs(q) : *q;
        return make_longlong2((long long)(kb + (w & 0xFFFFFFFFULL)), (long long)(pb + (w >> 32)));
    } else {
        const longlong2* q = reinterpret_cast<const longlong2*>(base) + i;
        return CS ? __ldcs(q) : *q;
    }
}

template <bool RP, bool SP>
__global__ void __launch_bounds__(MP16_THREADS, 2) mp16_join_kernel(Mp16Args a)
{
    extern __shared__ __align__(16) unsigned char mp16_smem[];
    long long* keys = (long long*)mp16_smem;
    unsigned long long* pays = (unsigned long long*)(keys + MP16_RCHUNK);
    unsigned long long* pre = pays + MP16_RCHUNK;  // MP16_RCHUNK + 1 prefix sums
    __shared__ long long item;
    __shared__ unsigned long long side_cnt, side_sum;
    __shared__ unsigned long long warp_tot[MP16_THREADS / 32];
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    uint64_t cnt = 0, bsum = 0, psum = 0;
    for (;;) {
        if (tid == 0) {
            item = (long long)atomicAdd(a.next, 1u);
            side_cnt = side_sum = 0;
        }
        __syncthreads();
        const long long it = item;
        if (it >= a.nitems) break;
        const Mp16Item m = a.items[it];
        if (m.span) {
            // Counting sort of the whole range by key offset: bin o holds
            // the count and payload sum of key lo + o.
            unsigned* bc = (unsigned*)mp16_smem;
            unsigned long long* bs = (unsigned long long*)(mp16_smem + MP16_DSPAN * 4);
            for (unsigned i = tid; i < m.span; i += MP16_THREADS) {
                bc[i] = 0;
                bs[i] = 0;
            }
            __syncthreads();
            bool out_of_span = false;
            for (unsigned i = tid; i < m.rn; i += MP16_THREADS) {
                const longlong2 t = mp16_elem<RP, false>(a.R, m.r0 + i, a.rk, a.rp);
                const unsigned long long o = (unsigned long long)t.x - (unsigned long long)m.lo;
                if (o < m.span) {
                    atomicAdd(&bc[o], 1u);
                    atomicAdd(&bs[o], (unsigned long long)t.y);
                } else {
                    out_of_span = true;
                }
            }
            if (out_of_span) atomicOr(a.bad, 1u);
            __syncthreads();
            auto probe_bin = [&](const longlong2 t) {
                const unsigned long long o = (unsigned long long)t.x - (unsigned long long)m.lo;
                if (o >= m.span) return;
                const unsigned c = bc[o];
                if (c) {
                    cnt += c;
                    bsum += bs[o];
                    psum += (uint64_t)c * (uint64_t)t.y;
                }
            };
            constexpr int U = 8;
            unsigned i = tid;
            for (; i + (U - 1) * MP16_THREADS < m.sn; i += U * MP16_THREADS) {
                longlong2 t[U];
#pragma unroll
                for (int u = 0; u < U; ++u) t[u] = mp16_elem<SP, true>(a.S, m.s0 + i + u * MP16_THREADS, a.sk, a.sp);
#pragma unroll
                for (int u = 0; u < U; ++u) probe_bin(t[u]);
            }
            for (; i < m.sn; i += MP16_THREADS) probe_bin(mp16_elem<SP, true>(a.S, m.s0 + i, a.sk, a.sp));
            __syncthreads();  // the bins are reused by the next item
            continue;
        }
        int N = 32;
        while (N < (int)m.rn) N <<= 1;
        // Load the build chunk; INT64_MAX keys go to the side counters and
        // their slots become padding.
        for (int i = tid; i < N; i += MP16_THREADS) {
            long long k = kPadKey;
            unsigned long long p = 0;
            if (i < (int)m.rn) {
                const longlong2 t = mp16_elem<RP, false>(a.R, m.r0 + i, a.rk, a.rp);
                if (t.x == kPadKey) {
                    atomicAdd(&side_cnt, 1ULL);
                    atomicAdd(&side_sum, (unsigned long long)t.y);
                } else {
                    k = t.x;
                    p = (unsigned long long)t.y;
                }
            }
            keys[i] = k;
            pays[i] = p;
        }
        __syncthreads();
        // Bitonic sort of (key, payload) by key, ascending.  At stride
        // j <= 32 every compare-exchange a warp does stays inside that
        // warp's own 64-element blocks, so those stages need only a warp
        // barrier; a CTA barrier precedes every stage that follows or uses
        // a longer stride.
        bool wide = true;
        for (int kk = 2; kk <= N; kk <<= 1) {
            for (int j = kk >> 1; j > 0; j >>= 1) {
                if (wide || j >= 64) __syncthreads();
                else __syncwarp();
                wide = j >= 64;
                for (int i = tid; i < N / 2; i += MP16_THREADS) {
                    const int lo = 2 * i - (i & (j - 1));
                    const int hi = lo + j;
                    const bool up = (lo & kk) == 0;
                    const long long a0 = keys[lo], a1 = keys[hi];
                    if ((a0 > a1) == up) {
                        keys[lo] = a1;
                        keys[hi] = a0;
                        const unsigned long long p0 = pays[lo];
                        pays[lo] = pays[hi];
                        pays[hi] = p0;
                    }
                }
            }
        }
        __syncthreads();
        // Exclusive prefix sum of the sorted payloads: thread t owns a
        // contiguous run of N / MP16_THREADS (or one) entries.
        const int per = N >= MP16_THREADS ? N / MP16_THREADS : 1;
        const int b0 = tid * per;
        unsigned long long run = 0;
        if (b0 < N)
            for (int i = b0; i < b0 + per; ++i) run += pays[i];
        unsigned long long incl = run;
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (lane == 31) warp_tot[w] = incl;
        __syncthreads();
        unsigned long long base = incl - run;
        for (int v = 0; v < w; ++v) base += warp_tot[v];
        if (b0 < N) {
            for (int i = b0; i < b0 + per; ++i) {
                pre[i] = base;
                base += pays[i];
            }
            if (b0 + per == N) pre[N] = base;
        }
        __syncthreads();
        const int rv = (int)m.rn - (int)side_cnt;  // real (non-padding) keys, sorted first
        const uint64_t scnt = side_cnt, ssum = side_sum;
        // Merge the probe chunk into the sorted run.
        auto probe = [&](const longlong2 t) {
            if (t.x == kPadKey) {
                cnt += scnt;
                bsum += ssum;
                psum += scnt * (uint64_t)t.y;
                return;
            }
            int lo = 0, n = rv;
            while (n > 0) {
                const int half = n >> 1;
                if (keys[lo + half] < t.x) {
                    lo += half + 1;
                    n -= half + 1;
                } else {
                    n = half;
                }
            }
            if (lo >= rv || keys[lo] != t.x) return;
            int hi = lo + 1;
            if (hi < rv && keys[hi] == t.x) {  // repeated build key: upper bound by search
                int n2 = rv - hi;
                while (n2 > 0) {
                    const int half = n2 >> 1;
                    if (keys[hi + half] <= t.x) {
                        hi += half + 1;
                        n2 -= half + 1;
                    } else {
                        n2 = half;
                    }
                }
            }
            const uint64_t c = (uint64_t)(hi - lo);
            cnt += c;
            bsum += pre[hi] - pre[lo];
            psum += c * (uint64_t)t.y;
        };
        constexpr int U = 4;
        unsigned i = tid;
        for (; i + (U - 1) * MP16_THREADS < m.sn; i += U * MP16_THREADS) {
            longlong2 t[U];
#pragma unroll
            for (int u = 0; u < U; ++u) t[u] = mp16_elem<SP, true>(a.S, m.s0 + i + u * MP16_THREADS, a.sk, a.sp);
#pragma unroll
            for (int u = 0; u < U; ++u) probe(t[u]);
        }
        for (; i < m.sn; i += MP16_THREADS) probe(mp16_elem<SP, true>(a.S, m.s0 + i, a.sk, a.sp));
        __syncthreads();  // the run and the side counters are reused by the next item
    }
    cnt = warp_sum_u64(cnt);
    bsum = warp_sum_u64(bsum);
    psum = warp_sum_u64(psum);
    if (lane == 0 && (cnt | bsum | psum)) {
        atomicAdd(&a.acc[0], (unsigned long long)cnt);
        atomicAdd(&a.acc[1], (unsigned long long)bsum);
        atomicAdd(&a.acc[2], (unsigned long long)psum);
    }
}

int mpsm16_fine_bits(int64_t nR, int64_t nS)
{
    // Ranges of about 8K probe and at most ~3K build tuples on uniform data.
    int fb = 1;
    while (fb < RJ_MAX_RANGE_BITS && ((double)nS / (double)(1 << fb) > 8192.0 || (double)nR / (double)(1 << fb) > 3072.0))
        ++fb;
    return fb;
}

int mpsm16_agg(pyg_ctx* ctx, const void* Rv, int64_t nR, const void* Sv, int64_t nS, const int64_t* splitters, int FB,
               unsigned long long out[3], std::vector<unsigned long long>* sizes, float* part_ms, float* join_ms,
               const RJModel* model)
{
    const longlong2* R = (const longlong2*)Rv;
    const longlong2* S = (const longlong2*)Sv;
    out[0] = out[1] = out[2] = 0;
    const bool two = FB > 8;
    const int CB = two ? (FB + 1) / 2 : FB;
    const int F = 1 << FB, C = 1 << CB, L = 1 << (FB - CB);
    if (nR == 0 || nS == 0) return PYG_OK;
    cudaEvent_t ev[3];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], ctx->stream);
    long long* dsplit = nullptr;
    void *R1 = nullptr, *R2 = nullptr, *S1 = nullptr, *S2 = nullptr;
    Mp16Item* ditems = nullptr;
    int rc = PYG_OK;
    do {
        // Fine splitters, then the coarse ones (every L-th fine splitter).
        std::vector<long long> sp((size_t)(F - 1) + (C - 1));
        for (int i = 0; i < F - 1; ++i) sp[i] = (long long)splitters[i];
        for (int i = 0; i < C - 1; ++i) sp[F - 1 + i] = (long long)splitters[(size_t)(i + 1) * L - 1];
        if ((rc = dalloc(ctx, (void**)&dsplit, sp.size() * 8 + 8))) break;
        if ((rc = stage_h2d(ctx, dsplit, sp.data(), sp.size() * 8))) break;
        const long long* fs = dsplit;
        const long long* cs = two ? dsplit + (F - 1) : dsplit;
        unsigned* flags = (unsigned*)(ctx->dcounters + 208);
        unsigned* hflags = (unsigned*)ctx->pinned + 96;
        RJLayout LR, LS;
        if (model) {
            // Bins from the model: no splitter search in the histograms or
            // passes, and both relations' histograms in one round trip.
            RPSide sd[2];
            sd[0].in = R;
            sd[0].n = nR;
            sd[1].in = S;
            sd[1].n = nS;
            sd[0].model = sd[1].model = model;
            // One bin function for both passes: the intermediates can be
            // packed words whatever split of bits the passes take.
            sd[0].allow_pack = sd[1].allow_pack = true;
            rc = rp_partition_sides(ctx, sd, 2, FB, two, flags, hflags, nullptr);
            R1 = sd[0].P1;
            R2 = sd[0].P2;
            S1 = sd[1].P1;
            S2 = sd[1].P2;
            if (rc) break;
            LR = std::move(sd[0].L);
            LS = std::move(sd[1].L);
        } else {
            if ((rc = rp_partition(ctx, R, nR, FB, two, true, cs, fs, LR, &R1, &R2, flags, hflags))) break;
            if ((rc = rp_partition(ctx, S, nS, FB, two, true, cs, fs, LS, &S1, &S2, flags, hflags))) break;
        }
        cudaEventRecord(ev[1], ctx->stream);
        if (sizes) *sizes = LS.count;
        // Items: every (build chunk, probe chunk) pair of each range.  Range
        // f holds keys in [sp[f - 1], sp[f]); a bounded range of at most
        // MP16_DSPAN key values is one build chunk, sorted by counting.
        std::vector<Mp16Item> items;
        for (int f = 0; f < F; ++f) {
            const unsigned long long rn = LR.count[f], sn = LS.count[f];
            if (!rn || !sn) continue;
            long long lo = 0;
            unsigned span = 0;
            if (f > 0 && f < F - 1) {
                const __int128 w = (__int128)sp[f] - (__int128)sp[f - 1];
                if (w > 0 && w <= (__int128)MP16_DSPAN && rn <= 0xFFFFFFFFULL) {
                    lo = sp[f - 1];
                    span = (unsigned)w;
                }
            }
            const unsigned long long rchunk = span ? rn : (unsigned long long)MP16_RCHUNK;
            for (unsigned long long r = 0; r < rn; r += rchunk)
                for (unsigned long long s = 0; s < sn; s += MP16_SCHUNK) {
                    Mp16Item it;
                    it.r0 = LR.fstart[f] + r;
                    it.s0 = LS.fstart[f] + s;
                    it.rn = (unsigned)std::min<unsigned long long>(rchunk, rn - r);
                    it.sn = (unsigned)std::min<unsigned long long>(MP16_SCHUNK, sn - s);
                    it.lo = lo;
                    it.span = span;
                    it.pad = 0;
                    items.push_back(it);
                }
        }
        unsigned long long* acc = ctx->dcounters + 212;
        unsigned* next = (unsigned*)(ctx->dcounters + 215);  // word 215: queue head, then the bad-key flag
        unsigned* bad = next + 1;
        PYG_CUDA(cudaMemsetAsync(acc, 0, 32, ctx->stream));
        if (!items.empty()) {
            if ((rc = dalloc(ctx, (void**)&ditems, items.size() * sizeof(Mp16Item)))) break;
            if ((rc = stage_h2d(ctx, ditems, items.data(), items.size() * sizeof(Mp16Item)))) break;
            Mp16Args ja;
            ja.R = two ? R2 : R1;
            ja.S = two ? S2 : S1;
            ja.rk = LR.kbase;
            ja.rp = LR.pbase;
            ja.sk = LS.kbase;
            ja.sp = LS.pbase;
            ja.items = ditems;
            ja.nitems = (long long)items.size();
            ja.next = next;
            ja.acc = acc;
            ja.bad = bad;
            auto kern = LR.packed ? (LS.packed ? mp16_join_kernel<true, true> : mp16_join_kernel<true, false>)
                                  : (LS.packed ? mp16_join_kernel<false, true> : mp16_join_kernel<false, false>);
            PYG_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, MP16_SMEM));
            const unsigned grid = (unsigned)std::min<long long>(2LL * ctx->sm_count, ja.nitems);
            kern<<<grid, MP16_THREADS, MP16_SMEM, ctx->stream>>>(ja);
            PYG_LAUNCHED(ctx);
        }
        cudaEventRecord(ev[2], ctx->stream);
        unsigned long long* h = (unsigned long long*)ctx->pinned + 64;
        PYG_CUDA(cudaMemcpyAsync(h, acc, 32, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        if ((unsigned)(h[3] >> 32)) {
            set_error("pyg_mpsm_join_agg: a key fell outside its range's span");
            rc = PYG_ERR_CUDA;
            break;
        }
        out[0] = h[0];
        out[1] = h[1];
        out[2] = h[2];
        if (part_ms) cudaEventElapsedTime(part_ms, ev[0], ev[1]);
        if (join_ms) cudaEventElapsedTime(join_ms, ev[1], ev[2]);
    } while (0);
    dfree(ctx, ditems);
    dfree(ctx, R1);
    dfree(ctx, R2);
    dfree(ctx, S1);
    dfree(ctx, S2);
    dfree(ctx, dsplit);
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

}  // namespace pyg
