// MPSM sort-merge join on one B200.
//
// Pipeline (both sides carried as 16-byte items {int64 key, int64 val},
// val = the projected column or the input row number):
//   1. splitters: equal-width over [min, max] (the reference's
//      ExactRangeValueHasher), quantiles of a probe-key sample, or the
//      learned CDF model trained on that sample;
//   2. range partition both sides by the splitters (histogram / scan /
//      scatter partitioner);
//   3. sort every partition: 2048-item tiles (eight 4 KB pages of 256
//      items) bitonic-sorted in shared memory, then merge-path merge rounds
//      that split each merge across CTAs in 2048-item output tiles;
//   4. merge join: CTAs take (partition, probe chunk) work items; each
//      thread merges a run of sorted probe items against the partition's
//      sorted build run (binary search + forward scan) and either
//      accumulates count / sums (build sums from a prefix sum over the
//      sorted build vals) or writes the joined rows.
// A partition's build and probe items are sorted by (key, val), so the
// materialised output order is deterministic: key, probe row, build row.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "../../include/pyg_learned.h"
#include "../../include/pyg_mpsm.h"
#include "mpsm16.cuh"
#include "partition.cuh"
#include "primitives.cuh"
#include "radixpart.cuh"

namespace pyg {

constexpr int MP_TILE = 2048;        // items per shared-memory sorted tile
constexpr int MP_PAGE = 256;         // 4 KB page of 16-byte items
constexpr int MP_SORT_THREADS = 512;
constexpr int MP_MERGE_THREADS = 256;
constexpr int MP_MERGE_PER_THREAD = MP_TILE / MP_MERGE_THREADS;  // 8
constexpr int MP_JOIN_THREADS = 256;
constexpr int MP_JOIN_PER_THREAD = 32;
constexpr int64_t MP_JOIN_CHUNK = (int64_t)MP_JOIN_THREADS * MP_JOIN_PER_THREAD;

__device__ __forceinline__ bool item_le(const longlong2& a, const longlong2& b)
{
    return a.x < b.x || (a.x == b.x && a.y <= b.y);
}
__device__ __forceinline__ bool item_gt(long long ak, long long av, long long bk, long long bv)
{
    return ak > bk || (ak == bk && av > bv);
}

struct SpanWork {
    int64_t start;
    int32_t n;
    int32_t pad;
};

// Bitonic sort of each work tile (<= 2048 items) in shared memory.  The
// first eight levels of the network sort each 256-item (4 KB) page; the
// remaining levels merge the pages of the tile.
__global__ void __launch_bounds__(MP_SORT_THREADS) mp_tile_sort_kernel(longlong2* __restrict__ data,
                                                                       const SpanWork* __restrict__ work, int nwork)
{
    __shared__ long long sk[MP_TILE];
    __shared__ long long sv[MP_TILE];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const int64_t start = work[w].start;
        const int n = work[w].n;
        int m = 2;
        while (m < n) m <<= 1;
        for (int i = threadIdx.x; i < m; i += blockDim.x) {
            if (i < n) {
                longlong2 t = data[start + i];
                sk[i] = t.x;
                sv[i] = t.y;
            } else {
                sk[i] = 0x7fffffffffffffffLL;
                sv[i] = 0x7fffffffffffffffLL;
            }
        }
        __syncthreads();
        for (int k = 2; k <= m; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = threadIdx.x; i < (m >> 1); i += blockDim.x) {
                    int a = (i / j) * 2 * j + (i % j);
                    int b = a + j;
                    bool asc = (a & k) == 0;
                    long long ak = sk[a], av = sv[a], bk = sk[b], bv = sv[b];
                    bool swap = asc ? item_gt(ak, av, bk, bv) : item_gt(bk, bv, ak, av);
                    if (swap) {
                        sk[a] = bk;
                        sv[a] = bv;
                        sk[b] = ak;
                        sv[b] = av;
                    }
                }
                __syncthreads();
            }
        }
        for (int i = threadIdx.x; i < n; i += blockDim.x) data[start + i] = make_longlong2(sk[i], sv[i]);
        __syncthreads();
    }
}

struct MergeWork {
    int64_t a;      // first run [a, a + na) in src
    int64_t b;      // second run [b, b + nb) in src (b = a + na)
    int32_t na, nb;
    int64_t d;      // first output position handled (relative to a)
};

// Merge path: number of elements taken from A among the first d outputs
// (ties take A first, so the merge is stable).
__device__ __forceinline__ int merge_path(const longlong2* A, int na, const longlong2* B, int nb, int d)
{
    int lo = d > nb ? d - nb : 0, hi = d < na ? d : na;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (item_le(A[mid], B[d - 1 - mid])) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(MP_MERGE_THREADS) mp_merge_kernel(const longlong2* __restrict__ src,
                                                                    longlong2* __restrict__ dst,
                                                                    const MergeWork* __restrict__ work, int nwork)
{
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const MergeWork mw = work[w];
        const longlong2* A = src + mw.a;
        const longlong2* B = src + mw.b;
        int total = mw.na + mw.nb;
        int d = (int)mw.d + threadIdx.x * MP_MERGE_PER_THREAD;
        if (d >= total) continue;
        int cnt = total - d < MP_MERGE_PER_THREAD ? total - d : MP_MERGE_PER_THREAD;
        int i = merge_path(A, mw.na, B, mw.nb, d);
        int j = d - i;
        longlong2* out = dst + mw.a + d;
        for (int t = 0; t < cnt; ++t) {
            bool takeA = j >= mw.nb || (i < mw.na && item_le(A[i], B[j]));
            out[t] = takeA ? A[i++] : B[j++];
        }
    }
}

struct JoinWork {
    int32_t part;
    int32_t pad;
    int64_t s0;     // first probe item (absolute index in the probe array)
    int64_t s1;     // one past the last
};

struct JoinArgs {
    const longlong2* R;            // sorted build items (contiguous per partition)
    const unsigned long long* rpre;  // exclusive prefix sums of build vals (n_R + 1)
    const unsigned long long* roff;  // partition offsets into R
    const longlong2* S0;           // probe buffers (sorted result in S0 or S1 per partition)
    const longlong2* S1;
    const unsigned char* spar;     // per partition: 1 if the sorted probe run is in S1
    const JoinWork* work;
    int nwork;
    // materialise
    int mode;                      // 0 aggregate, 1 count matches, 2 write rows
    unsigned long long* counts;    // per probe item match count / output offset
    const uint8_t* rbase;          // original relations (row gather)
    const uint8_t* sbase;
    int32_t rtb, stb;
    int nproj;
    int32_t pside[PYG_MAX_COLS], poff[PYG_MAX_COLS], ptype[PYG_MAX_COLS], ooff[PYG_MAX_COLS];
    int32_t out_tb;
    uint8_t* out;
    int64_t out_cap;
    unsigned long long* acc;       // count, build sum, probe sum
};

__device__ __forceinline__ int64_t lower_bound_key(const longlong2* R, int64_t lo, int64_t hi, long long key)
{
    while (lo < hi) {
        int64_t mid = lo + ((hi - lo) >> 1);
        if (R[mid].x < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__global__ void __launch_bounds__(MP_JOIN_THREADS) mp_join_kernel(JoinArgs a)
{
    uint64_t cnt = 0, bsum = 0, psum = 0;
    for (int w = blockIdx.x; w < a.nwork; w += gridDim.x) {
        const JoinWork jw = a.work[w];
        const longlong2* S = a.spar[jw.part] ? a.S1 : a.S0;
        const int64_t rlo0 = (int64_t)a.roff[jw.part], rhi0 = (int64_t)a.roff[jw.part + 1];
        int64_t i0 = jw.s0 + (int64_t)threadIdx.x * MP_JOIN_PER_THREAD;
        int64_t i1 = i0 + MP_JOIN_PER_THREAD < jw.s1 ? i0 + MP_JOIN_PER_THREAD : jw.s1;
        int64_t lo = rlo0, hi = rlo0;
        long long cur = 0;
        bool have = false;
        for (int64_t i = i0; i < i1; ++i) {
            longlong2 s = S[i];
            if (!have || s.x != cur) {
                lo = lower_bound_key(a.R, have ? hi : rlo0, rhi0, s.x);
                hi = lo;
                while (hi < rhi0 && a.R[hi].x == s.x) ++hi;
                cur = s.x;
                have = true;
            }
            uint64_t c = (uint64_t)(hi - lo);
            if (a.mode == 0) {
                cnt += c;
                bsum += a.rpre[hi] - a.rpre[lo];
                psum += c * (uint64_t)s.y;
            } else if (a.mode == 1) {
                a.counts[i] = c;
            } else if (c) {
                int64_t pos = (int64_t)a.counts[i];
                const uint8_t* st = a.sbase + (int64_t)s.y * a.stb;
                for (int64_t r = lo; r < hi; ++r, ++pos) {
                    if (pos >= a.out_cap) break;
                    const uint8_t* rt = a.rbase + (int64_t)a.R[r].y * a.rtb;
                    uint8_t* dst = a.out + pos * (int64_t)a.out_tb;
                    for (int p = 0; p < a.nproj; ++p) {
                        store_col(dst, a.ooff[p], a.ptype[p],
                                  (uint64_t)load_col(a.pside[p] ? st : rt, a.poff[p], a.ptype[p]));
                    }
                }
            }
        }
    }
    if (a.mode == 0) {
        cnt = warp_sum_u64(cnt);
        bsum = warp_sum_u64(bsum);
        psum = warp_sum_u64(psum);
        if ((threadIdx.x & 31) == 0 && (cnt | bsum | psum)) {
            atomicAdd(&a.acc[0], (unsigned long long)cnt);
            atomicAdd(&a.acc[1], (unsigned long long)bsum);
            atomicAdd(&a.acc[2], (unsigned long long)psum);
        }
    }
}

__global__ void mp_extract_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb, int32_t koff, int32_t ktype,
                                  int32_t voff, int32_t vtype, int rowid, longlong2* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const uint8_t* t = base + i * (int64_t)tb;
        long long v = rowid ? (long long)i : (voff >= 0 ? (long long)load_col(t, voff, vtype) : 0);
        out[i] = make_longlong2((long long)load_col(t, koff, ktype), v);
    }
}

__global__ void mp_sample_kernel(const longlong2* __restrict__ items, int64_t n, int64_t stride, int64_t offset,
                                 int64_t ns, int64_t* __restrict__ out)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x) {
        int64_t i = j * stride + offset;
        out[j] = items[i < n ? i : n - 1].x;
    }
}

__global__ void mp_minmax_kernel(const longlong2* __restrict__ items, int64_t n, unsigned long long* mm)
{
    long long lo = 0x7fffffffffffffffLL, hi = (long long)0x8000000000000000ULL;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        long long k = items[i].x;
        lo = k < lo ? k : lo;
        hi = k > hi ? k : hi;
    }
    for (int o = 16; o > 0; o >>= 1) {
        long long a = __shfl_xor_sync(0xffffffffu, lo, o), b = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = a < lo ? a : lo;
        hi = b > hi ? b : hi;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin((unsigned long long*)&mm[0], to_sortable(lo));
        atomicMax((unsigned long long*)&mm[1], to_sortable(hi));
    }
}

__global__ void mp_vals_kernel(const longlong2* __restrict__ items, int64_t n, unsigned long long* __restrict__ vals)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        vals[i] = (unsigned long long)items[i].y;
    if (blockIdx.x == 0 && threadIdx.x == 0) vals[n] = 0;
}

// Host helper owning the device buffers of one MPSM run.
struct Mpsm {
    pyg_ctx* ctx;
    std::vector<void*> bufs;
    ~Mpsm()
    {
        for (void* p : bufs) dfree(ctx, p);
    }
    int alloc(void** p, size_t bytes)
    {
        int rc = dalloc(ctx, p, bytes);
        if (!rc) bufs.push_back(*p);
        return rc;
    }
};

// Sorts each partition of `data` (offsets `off`, host copy) in place or
// into `tmp`; par[p] = 1 when partition p's sorted result ends in tmp.
static int sort_partitions(pyg_ctx* ctx, Mpsm& M, longlong2* data, longlong2* tmp, const std::vector<int64_t>& off,
                           const std::vector<unsigned char>& single_key, std::vector<unsigned char>& par)
{
    const int F = (int)off.size() - 1;
    par.assign(F, 0);
    std::vector<SpanWork> tiles;
    int64_t maxn = 0;
    for (int p = 0; p < F; ++p) {
        int64_t n = off[p + 1] - off[p];
        maxn = std::max(maxn, n);
        if (n <= 1 || single_key[p]) continue;
        for (int64_t s = 0; s < n; s += MP_TILE)
            tiles.push_back({off[p] + s, (int32_t)std::min<int64_t>(MP_TILE, n - s), 0});
    }
    if (!tiles.empty()) {
        SpanWork* dw;
        int rc = M.alloc((void**)&dw, tiles.size() * sizeof(SpanWork));
        if (rc) return rc;
        PYG_CUDA(cudaMemcpyAsync(dw, tiles.data(), tiles.size() * sizeof(SpanWork), cudaMemcpyHostToDevice, ctx->stream));
        int grid = (int)std::min<size_t>(tiles.size(), (size_t)ctx->sm_count * 4);
        mp_tile_sort_kernel<<<grid, MP_SORT_THREADS, 0, ctx->stream>>>(data, dw, (int)tiles.size());
        PYG_LAUNCHED(ctx);
    }
    // Merge rounds: width w runs -> 2w runs, ping-pong between data and tmp.
    std::vector<MergeWork> mw;
    std::vector<int64_t> roundsize;
    longlong2* src = data;
    longlong2* dst = tmp;
    std::vector<unsigned char> cur(F, 0);
    for (int64_t w = MP_TILE; w < maxn; w *= 2) {
        mw.clear();
        for (int p = 0; p < F; ++p) {
            int64_t n = off[p + 1] - off[p];
            if (n <= w || single_key[p]) continue;
            // This partition's runs live in (cur[p] ? tmp : data); the
            // round writes the other buffer.
            for (int64_t s = 0; s < n; s += 2 * w) {
                int32_t na = (int32_t)std::min<int64_t>(w, n - s);
                int32_t nb = (int32_t)std::min<int64_t>(w, std::max<int64_t>(0, n - s - w));
                for (int64_t d = 0; d < na + nb; d += MP_TILE)
                    mw.push_back({off[p] + s, off[p] + s + na, na, nb, d});
            }
        }
        if (mw.empty()) break;
        // Partitions in this round all sit in the same buffer: every
        // partition with n > w has taken part in every earlier round.
        MergeWork* dw;
        int rc = M.alloc((void**)&dw, mw.size() * sizeof(MergeWork));
        if (rc) return rc;
        PYG_CUDA(cudaMemcpyAsync(dw, mw.data(), mw.size() * sizeof(MergeWork), cudaMemcpyHostToDevice, ctx->stream));
        int grid = (int)std::min<size_t>(mw.size(), (size_t)ctx->sm_count * 8);
        mp_merge_kernel<<<grid, MP_MERGE_THREADS, 0, ctx->stream>>>(src, dst, dw, (int)mw.size());
        PYG_LAUNCHED(ctx);
        for (int p = 0; p < F; ++p) {
            int64_t n = off[p + 1] - off[p];
            if (n > w && !single_key[p]) cur[p] ^= 1;
        }
        std::swap(src, dst);
    }
    par = cur;
    return PYG_OK;
}

struct Splits {
    std::vector<int64_t> spl;  // F - 1 splitters
};

static int mpsm_run(pyg_ctx* ctx, const pyg_rel* build, int32_t bkey, const pyg_rel* probe, int32_t pkey,
                    const pyg_proj* proj, int32_t nproj, const pyg_mpsm_opts* o, bool materialize, void* out,
                    int64_t out_cap, int64_t* out_count, pyg_join_result* res, pyg_mpsm_stats* stats)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_rel(build, "build")) || (rc = check_rel(probe, "probe"))) return rc;
    if (!o || o->fanout < 1 || o->fanout > (1 << 14) || (o->page_tuples != 0 && o->page_tuples != MP_PAGE) ||
        bkey < 0 || bkey >= build->ncols || pkey < 0 || pkey >= probe->ncols || nproj < 0 || nproj > PYG_MAX_COLS ||
        (nproj > 0 && !proj)) {
        set_error("mpsm: bad arguments (fan-out 1..2^14, page_tuples 256, key columns in range)");
        return PYG_ERR_ARG;
    }
    if (o->splitter_kind < PYG_MPSM_SPLIT_EXACTRANGE || o->splitter_kind > PYG_MPSM_SPLIT_LEARNED) {
        set_error("mpsm: unknown splitter kind %d", o->splitter_kind);
        return PYG_ERR_ARG;
    }
    // Value carried with each item: the projected column per side
    // (aggregate sink) or the row number (materialising sink).
    int bcol = -1, pcol = -1;
    for (int p = 0; p < nproj; ++p) {
        int& c = proj[p].side ? pcol : bcol;
        const pyg_rel* r = proj[p].side ? probe : build;
        if (proj[p].col < 0 || proj[p].col >= r->ncols) {
            set_error("mpsm: projected column %d out of range", proj[p].col);
            return PYG_ERR_ARG;
        }
        if (!materialize && c >= 0 && c != proj[p].col) {
            set_error("mpsm: the aggregate sink sums one column per side");
            return PYG_ERR_ARG;
        }
        c = proj[p].col;
    }
    if (!materialize && !res) {
        set_error("mpsm: null result");
        return PYG_ERR_ARG;
    }
    if (materialize && (!out_count || (out_cap > 0 && !out))) {
        set_error("mpsm: null output");
        return PYG_ERR_ARG;
    }
    const int F = o->fanout;
    const int64_t nR = build->ntuples, nS = probe->ntuples;
    Mpsm M{ctx, {}};
    cudaEvent_t ev[5];
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], ctx->stream);
    DevRel Rd, Sd;
    if ((rc = Rd.stage(ctx, build)) || (rc = Sd.stage(ctx, probe))) {
        Rd.release(ctx);
        Sd.release(ctx);
        for (auto& e : ev) cudaEventDestroy(e);
        return rc;
    }
    auto fail = [&](int code) {
        Rd.release(ctx);
        Sd.release(ctx);
        for (auto& e : ev) cudaEventDestroy(e);
        return code;
    };
    // 16-byte items {key, val}.
    auto items_of = [&](const pyg_rel* r, const pyg_rel& dev, int key, int col, int64_t n,
                        longlong2** items) -> int {
        bool direct = !materialize && r->tuple_bytes == 16 && r->col_offset[key] == 0 &&
                      r->col_type[key] == PYG_INT64 && (col < 0 || (r->col_offset[col] == 8 && r->col_type[col] == PYG_INT64)) &&
                      col >= 0 && (uintptr_t)dev.base % 16 == 0;
        if (direct) {
            *items = (longlong2*)dev.base;
            return PYG_OK;
        }
        int e = M.alloc((void**)items, (size_t)(n > 0 ? n : 1) * 16);
        if (e) return e;
        if (n > 0) {
            mp_extract_kernel<<<grid_for(ctx, n, 256, 4, 8), 256, 0, ctx->stream>>>(
                (const uint8_t*)dev.base, n, r->tuple_bytes, r->col_offset[key], r->col_type[key],
                col >= 0 ? r->col_offset[col] : -1, col >= 0 ? r->col_type[col] : PYG_INT64, materialize ? 1 : 0,
                *items);
            PYG_LAUNCHED(ctx);
        }
        return PYG_OK;
    };
    longlong2 *Ri, *Si;
    if ((rc = items_of(build, Rd.rel, bkey, bcol, nR, &Ri)) || (rc = items_of(probe, Sd.rel, pkey, pcol, nS, &Si)))
        return fail(rc);
    // Aggregate sink over 16-byte (int64 key, int64 payload) device tuples
    // summing column 1 of either side: range partitions small enough to be
    // sorted in shared memory (mpsm16.cu), with splitters of the same kind
    // at that finer fan-out.
    auto is16 = [](const pyg_rel* r, int key, int col) {
        return r->on_device && r->tuple_bytes == 16 && r->col_offset[key] == 0 && r->col_type[key] == PYG_INT64 &&
               (col < 0 || (col == 1 && r->col_offset[1] == 8 && r->col_type[1] == PYG_INT64)) &&
               (uintptr_t)r->base % 16 == 0;
    };
    const bool fast = !materialize && is16(build, bkey, bcol) && is16(probe, pkey, pcol) && nR > 0 && nS > 0;
    const int FBf = fast ? mpsm16_fine_bits(nR, nS) : 0;
    const int Fs = fast ? (1 << FBf) : F;

    // ---- 1. splitters
    std::vector<int64_t> spl(Fs > 1 ? Fs - 1 : 0);
    // Learned splitters on the 16-byte path: the model's own bins
    // (rj_model_bin) partition both relations, and its splitters (the first
    // key of each bin) bound the ranges; the model lives until the join.
    pyg_cdf* model = nullptr;
    RJModel bins;
    bool use_bins = false;
    auto done = [&](int code) {
        pyg_cdf_free(ctx, model);
        return fail(code);
    };
    unsigned long long* h = (unsigned long long*)ctx->pinned + 256;
    if (Fs > 1 && nR + nS > 0) {
        if (o->splitter_kind == PYG_MPSM_SPLIT_EXACTRANGE || nS == 0) {
            unsigned long long* mm = ctx->dcounters + 96;
            unsigned long long init[2] = {~0ULL, 0ULL};
            memcpy(h, init, 16);
            PYG_CUDA(cudaMemcpyAsync(mm, h, 16, cudaMemcpyHostToDevice, ctx->stream));
            if (nR) mp_minmax_kernel<<<grid_for(ctx, nR, 256, 8, 4), 256, 0, ctx->stream>>>(Ri, nR, mm);
            if (nS) mp_minmax_kernel<<<grid_for(ctx, nS, 256, 8, 4), 256, 0, ctx->stream>>>(Si, nS, mm);
            ctx->launches += (nR > 0) + (nS > 0);
            PYG_CUDA(cudaMemcpyAsync(h + 2, mm, 16, cudaMemcpyDeviceToHost, ctx->stream));
            PYG_CUDA(cudaStreamSynchronize(ctx->stream));
            int64_t mn = from_sortable(h[2]), mx = from_sortable(h[3]);
            // ExactRangeValueHasher(min, max, F) (hash.h:452-487): bucket
            // range br = (max - min + F) / F, bucket = (v - min) / br, i.e.
            // splitter j = min + j * br (clamped to the int64 range).
            __int128 br = ((__int128)mx - (__int128)mn + Fs) / Fs;
            for (int j = 1; j < Fs; ++j) {
                __int128 v = (__int128)mn + (__int128)j * br;
                spl[j - 1] = v > (__int128)INT64_MAX ? INT64_MAX : (int64_t)v;
            }
        } else {
            // The sample holds as many keys of each relation (each strided
            // over its own tuples), so that a range bounds its share of
            // both: splitters of the probe keys alone leave ranges whose
            // build side is many times the sort tile where the probe side
            // is skewed.  sample_rate sets the probe side's count; the
            // learned model needs far fewer keys than quantile splitters
            // (which want tens per range): its leaves are fitted lines, so at
            // most CDF_MPSM_SAMPLE keys (about 256 per leaf) are drawn for it.
            const double rate = o->sample_rate > 0 ? o->sample_rate : 0.01;
            int64_t want = (int64_t)llround((double)nS * rate);
            if (o->splitter_kind == PYG_MPSM_SPLIT_LEARNED) want = std::min<int64_t>(want, CDF_MPSM_SAMPLE / 2);
            want = std::max<int64_t>(want, 2);
            const int64_t nsS = std::min<int64_t>(want, nS), nsR = std::min<int64_t>(want, nR);
            const int64_t ns = nsS + nsR;
            const int64_t strideS = std::max<int64_t>(1, nS / nsS), strideR = nsR ? std::max<int64_t>(1, nR / nsR) : 1;
            int64_t* sample;
            if ((rc = M.alloc((void**)&sample, (size_t)ns * 8))) return fail(rc);
            mp_sample_kernel<<<grid_for(ctx, nsS, 256, 4, 4), 256, 0, ctx->stream>>>(
                Si, nS, strideS, (int64_t)(o->seed % (uint64_t)strideS), nsS, sample);
            PYG_LAUNCHED(ctx);
            if (nsR) {
                mp_sample_kernel<<<grid_for(ctx, nsR, 256, 4, 4), 256, 0, ctx->stream>>>(
                    Ri, nR, strideR, (int64_t)(o->seed % (uint64_t)strideR), nsR, sample + nsS);
                PYG_LAUNCHED(ctx);
            }
            if (o->splitter_kind == PYG_MPSM_SPLIT_SAMPLED || ns < 2) {
                if ((rc = pyg_sampled_splitters(ctx, sample, ns, Fs, spl.data()))) return fail(rc);
            } else {
                pyg_cdf_train_opts to;
                to.leaves = o->cdf_leaves > 0 ? o->cdf_leaves : 1024;
                // Least-squares start, then one fine-tuning epoch of the leaves.
                to.epochs = 1;
                to.lr = 0.002f;
                to.seed = o->seed;
                if ((rc = pyg_cdf_train(ctx, sample, ns, &to, &model))) return done(rc);
                if (fast) {
                    if ((rc = cdf_bin_model(ctx, model, FBf, &bins)) || (rc = model_splitters(ctx, bins, spl.data())))
                        return done(rc);
                    use_bins = true;
                } else {
                    rc = pyg_cdf_splitters(ctx, model, Fs, spl.data());
                    pyg_cdf_free(ctx, model);
                    model = nullptr;
                    if (rc) return fail(rc);
                }
            }
        }
    }
    cudaEventRecord(ev[1], ctx->stream);
    if (fast) {
        unsigned long long o3[3];
        std::vector<unsigned long long> sizes;
        float part_ms = 0.f, join_ms = 0.f;
        if ((rc = mpsm16_agg(ctx, Ri, nR, Si, nS, spl.data(), FBf, o3, &sizes, &part_ms, &join_ms,
                             use_bins ? &bins : nullptr)))
            return done(rc);
        memset(res, 0, sizeof(*res));
        res->count = (int64_t)o3[0];
        for (int p = 0; p < nproj; ++p) res->sums[p] = (int64_t)(proj[p].side ? o3[2] : o3[1]);
        if (stats) {
            // Imbalance over the caller's fan-out: its ranges are unions of
            // 2^FB / F consecutive fine ranges when F divides 2^FB.
            memset(stats, 0, sizeof(*stats));
            const int G = (Fs % F == 0) ? F : Fs;
            const int per = Fs / G;
            int64_t mx = 0;
            for (int g = 0; g < G; ++g) {
                int64_t t = 0;
                for (int q = 0; q < per; ++q) t += (int64_t)sizes[(size_t)g * per + q];
                mx = std::max(mx, t);
            }
            stats->max_partition = mx;
            stats->max_partition_imbalance = (double)mx / ((double)nS / G);
            float spl_ms = 0.f;
            cudaEventElapsedTime(&spl_ms, ev[0], ev[1]);
            stats->splitter_ms = spl_ms;
            stats->partition_ms = part_ms;
            stats->sort_ms = 0;  // the sort runs inside the merge kernel
            stats->merge_ms = join_ms;
        }
        return done(0);
    }

    // ---- 2. range partition both sides
    longlong2 *Rp, *Sp, *Rt, *St;
    unsigned long long *roff, *soff;
    if ((rc = M.alloc((void**)&Rp, (size_t)(nR > 0 ? nR : 1) * 16)) || (rc = M.alloc((void**)&Sp, (size_t)(nS > 0 ? nS : 1) * 16)) ||
        (rc = M.alloc((void**)&Rt, (size_t)(nR > 0 ? nR : 1) * 16)) || (rc = M.alloc((void**)&St, (size_t)(nS > 0 ? nS : 1) * 16)) ||
        (rc = M.alloc((void**)&roff, (size_t)(F + 1) * 8)) || (rc = M.alloc((void**)&soff, (size_t)(F + 1) * 8)))
        return fail(rc);
    pyg_splitter sp;
    sp.kind = PYG_SPLIT_SPLITTERS;
    sp.fanout = F;
    sp.range_min = sp.range_max = 0;
    sp.splitters = spl.data();
    BucketFn fn;
    int64_t* spl_dev = nullptr;
    if ((rc = make_bucket_fn(ctx, &sp, &fn, &spl_dev))) return fail(rc);
    if (spl_dev) M.bufs.push_back(spl_dev);
    pyg_rel irel;
    memset(&irel, 0, sizeof(irel));
    irel.tuple_bytes = 16;
    irel.ncols = 2;
    irel.col_offset[1] = 8;
    irel.col_type[0] = irel.col_type[1] = PYG_INT64;
    irel.on_device = 1;
    irel.base = Ri;
    irel.ntuples = nR;
    if ((rc = partition_device(ctx, &irel, 0, fn, Rp, roff))) return fail(rc);
    irel.base = Si;
    irel.ntuples = nS;
    if ((rc = partition_device(ctx, &irel, 0, fn, Sp, soff))) return fail(rc);
    std::vector<int64_t> ro(F + 1), so(F + 1);
    PYG_CUDA(cudaMemcpyAsync(ro.data(), roff, (size_t)(F + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    PYG_CUDA(cudaMemcpyAsync(so.data(), soff, (size_t)(F + 1) * 8, cudaMemcpyDeviceToHost, ctx->stream));
    cudaEventRecord(ev[2], ctx->stream);
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));

    // A partition whose splitter range holds one key value needs no sort
    // for the aggregate sink (the materialising sink still orders rows).
    std::vector<unsigned char> single(F, 0);
    if (!materialize)
        for (int p = 1; p + 1 < F; ++p) single[p] = spl[p] - spl[p - 1] == 1 ? 1 : 0;

    // ---- 3. sort partitions
    std::vector<unsigned char> rpar, spar;
    if ((rc = sort_partitions(ctx, M, Rp, Rt, ro, single, rpar))) return fail(rc);
    if ((rc = sort_partitions(ctx, M, Sp, St, so, single, spar))) return fail(rc);
    // Build side contiguous in Rp: copy partitions that ended in Rt back.
    {
        std::vector<MergeWork> back;
        for (int p = 0; p < F; ++p)
            if (rpar[p] && ro[p + 1] > ro[p])
                for (int64_t s0 = ro[p]; s0 < ro[p + 1]; s0 += MP_TILE)
                    back.push_back({s0, s0 + std::min<int64_t>(MP_TILE, ro[p + 1] - s0),
                                    (int32_t)std::min<int64_t>(MP_TILE, ro[p + 1] - s0), 0, 0});
        if (!back.empty()) {
            // A merge of one run with an empty one is a copy.
            MergeWork* dw;
            if ((rc = M.alloc((void**)&dw, back.size() * sizeof(MergeWork)))) return fail(rc);
            PYG_CUDA(cudaMemcpyAsync(dw, back.data(), back.size() * sizeof(MergeWork), cudaMemcpyHostToDevice,
                                     ctx->stream));
            mp_merge_kernel<<<(int)std::min<size_t>(back.size(), (size_t)ctx->sm_count * 8), MP_MERGE_THREADS, 0,
                              ctx->stream>>>(Rt, Rp, dw, (int)back.size());
            PYG_LAUNCHED(ctx);
        }
    }
    cudaEventRecord(ev[3], ctx->stream);

    // ---- 4. merge join
    unsigned long long* rpre;
    unsigned char* dspar;
    if ((rc = M.alloc((void**)&rpre, (size_t)(nR + 1) * 8)) || (rc = M.alloc((void**)&dspar, (size_t)F))) return fail(rc);
    mp_vals_kernel<<<grid_for(ctx, nR > 0 ? nR : 1, 256, 4, 8), 256, 0, ctx->stream>>>(Rp, nR, rpre);
    PYG_LAUNCHED(ctx);
    if ((rc = exclusive_scan_u64(ctx, rpre, rpre, nR + 1, nullptr))) return fail(rc);
    PYG_CUDA(cudaMemcpyAsync(dspar, spar.data(), (size_t)F, cudaMemcpyHostToDevice, ctx->stream));
    std::vector<JoinWork> jw;
    for (int p = 0; p < F; ++p) {
        if (ro[p + 1] == ro[p]) continue;
        for (int64_t s = so[p]; s < so[p + 1]; s += MP_JOIN_CHUNK)
            jw.push_back({p, 0, s, std::min<int64_t>(so[p + 1], s + MP_JOIN_CHUNK)});
    }
    JoinWork* djw = nullptr;
    if (!jw.empty()) {
        if ((rc = M.alloc((void**)&djw, jw.size() * sizeof(JoinWork)))) return fail(rc);
        PYG_CUDA(cudaMemcpyAsync(djw, jw.data(), jw.size() * sizeof(JoinWork), cudaMemcpyHostToDevice, ctx->stream));
    }
    JoinArgs ja;
    memset(&ja, 0, sizeof(ja));
    ja.R = Rp;
    ja.rpre = rpre;
    ja.roff = roff;
    ja.S0 = Sp;
    ja.S1 = St;
    ja.spar = dspar;
    ja.work = djw;
    ja.nwork = (int)jw.size();
    unsigned long long* acc = ctx->dcounters + 104;
    ja.acc = acc;
    PYG_CUDA(cudaMemsetAsync(acc, 0, 24, ctx->stream));
    int jgrid = (int)std::min<size_t>(jw.size() > 0 ? jw.size() : 1, (size_t)ctx->sm_count * 8);
    if (!materialize) {
        ja.mode = 0;
        if (!jw.empty()) {
            mp_join_kernel<<<jgrid, MP_JOIN_THREADS, 0, ctx->stream>>>(ja);
            PYG_LAUNCHED(ctx);
        }
        cudaEventRecord(ev[4], ctx->stream);
        PYG_CUDA(cudaMemcpyAsync(h, acc, 24, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        memset(res, 0, sizeof(*res));
        res->count = (int64_t)h[0];
        for (int p = 0; p < nproj; ++p) {
            uint64_t v = proj[p].side ? h[2] : h[1];
            int32_t t = (proj[p].side ? probe : build)->col_type[proj[p].col];
            res->sums[p] = t == PYG_INT32 ? (int64_t)(int32_t)(uint32_t)v : (int64_t)v;
        }
    } else {
        unsigned long long* counts;
        if ((rc = M.alloc((void**)&counts, (size_t)(nS + 1) * 8))) return fail(rc);
        PYG_CUDA(cudaMemsetAsync(counts, 0, (size_t)(nS + 1) * 8, ctx->stream));
        ja.counts = counts;
        ja.mode = 1;
        if (!jw.empty()) {
            mp_join_kernel<<<jgrid, MP_JOIN_THREADS, 0, ctx->stream>>>(ja);
            PYG_LAUNCHED(ctx);
        }
        unsigned long long* total = ctx->dcounters + 112;
        if ((rc = exclusive_scan_u64(ctx, counts, counts, nS + 1, total))) return fail(rc);
        PYG_CUDA(cudaMemcpyAsync(h, total, 8, cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        *out_count = (int64_t)h[0];
        ja.mode = 2;
        ja.rbase = (const uint8_t*)Rd.rel.base;
        ja.sbase = (const uint8_t*)Sd.rel.base;
        ja.rtb = build->tuple_bytes;
        ja.stb = probe->tuple_bytes;
        ja.nproj = nproj;
        int ob = 0;
        for (int p = 0; p < nproj; ++p) {
            const pyg_rel* r = proj[p].side ? probe : build;
            ja.pside[p] = proj[p].side ? 1 : 0;
            ja.poff[p] = r->col_offset[proj[p].col];
            ja.ptype[p] = r->col_type[proj[p].col];
            ja.ooff[p] = ob;
            ob += ja.ptype[p] == PYG_INT32 ? 4 : 8;
        }
        ja.out_tb = ob;
        ja.out = (uint8_t*)out;
        ja.out_cap = out_cap;
        if (!jw.empty() && out_cap > 0 && nproj > 0) {
            mp_join_kernel<<<jgrid, MP_JOIN_THREADS, 0, ctx->stream>>>(ja);
            PYG_LAUNCHED(ctx);
        }
        cudaEventRecord(ev[4], ctx->stream);
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    }
    if (stats) {
        memset(stats, 0, sizeof(*stats));
        int64_t mx = 0;
        for (int p = 0; p < F; ++p) mx = std::max(mx, so[p + 1] - so[p]);
        stats->max_partition = mx;
        stats->max_partition_imbalance = nS > 0 ? (double)mx / ((double)nS / F) : 0.0;
        float t[4];
        for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&t[i], ev[i], ev[i + 1]);
        stats->splitter_ms = t[0];
        stats->partition_ms = t[1];
        stats->sort_ms = t[2];
        stats->merge_ms = t[3];
    }
    fail(0);
    if (materialize && *out_count > out_cap) {
        set_error("mpsm: %lld joined rows exceed capacity %lld", (long long)*out_count, (long long)out_cap);
        return PYG_ERR_CAPACITY;
    }
    return PYG_OK;
}

}  // namespace pyg

using namespace pyg;

extern "C" {

int pyg_mpsm_join_agg(pyg_ctx* ctx, const pyg_rel* build, int32_t build_key, const pyg_rel* probe, int32_t probe_key,
                      const pyg_proj* proj, int32_t nproj, const pyg_mpsm_opts* opts, pyg_join_result* out,
                      pyg_mpsm_stats* stats)
{
    return mpsm_run(ctx, build, build_key, probe, probe_key, proj, nproj, opts, false, nullptr, 0, nullptr, out,
                    stats);
}

int pyg_mpsm_join_materialize(pyg_ctx* ctx, const pyg_rel* build, int32_t build_key, const pyg_rel* probe,
                              int32_t probe_key, const pyg_proj* proj, int32_t nproj, const pyg_mpsm_opts* opts,
                              void* out, int64_t out_capacity, int64_t* out_count)
{
    return mpsm_run(ctx, build, build_key, probe, probe_key, proj, nproj, opts, true, out, out_capacity, out_count,
                    nullptr, nullptr);
}

}  // extern "C"
