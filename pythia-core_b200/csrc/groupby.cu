// Group-by aggregation (sum and/or count) on one B200.
//
// Semantics follow GenericAggregate + AggregateSum / AggregateCount
// (operators/genericaggregate.cpp:247-494, aggregatesum.cpp:53-105,
// aggregatecount.cpp:44-52): one output tuple per distinct key with the
// wrapped sum of the sum column (its own width) and/or the int64 count.
//
// Kernel structure: lanes of a warp holding the same key are combined with
// __match_any_sync and __reduce_add_sync before any atomic; for low
// cardinality each CTA first folds into a shared-memory table and flushes
// it once; otherwise the combined values go straight to an open-addressing
// table of 32-byte slots {key, sum, count, -} in HBM (one sector per
// update).  The output is compacted from the table and, on request,
// ordered by key with the radix sort.
#include <string.h>

#include "primitives.cuh"
#include "gbradix.cuh"

namespace pyg {

constexpr int GB_THREADS = 256;
constexpr int GB_SMEM_SLOTS = 4096;     // shared table slots per CTA
constexpr int GB_SMEM_MAX_GROUPS = 2048;
constexpr uint64_t GB_PROBE_LIMIT = 4096;

struct GroupArgs {
    const uint8_t* base;
    int64_t n;
    int32_t tb;
    KeySpec ks;
    int32_t sum_off, sum_type;
    int32_t want_sum;
    ulonglong4* table;  // {key, sum, count, unused}
    uint64_t cap;
    unsigned long long* flags;  // [0] full, [1] groups, [2] sentinel sum, [3] sentinel count
};

// Sum of a 64-bit value over the lanes in `mask` (all of which call this
// with the same mask): four 16-bit slices so each 32-bit reduction is exact.
__device__ __forceinline__ uint64_t group_sum_u64(unsigned mask, uint64_t v)
{
    unsigned s0 = __reduce_add_sync(mask, (unsigned)(v & 0xFFFF));
    unsigned s1 = __reduce_add_sync(mask, (unsigned)((v >> 16) & 0xFFFF));
    unsigned s2 = __reduce_add_sync(mask, (unsigned)((v >> 32) & 0xFFFF));
    unsigned s3 = __reduce_add_sync(mask, (unsigned)(v >> 48));
    return (uint64_t)s0 + ((uint64_t)s1 << 16) + ((uint64_t)s2 << 32) + ((uint64_t)s3 << 48);
}

// Adds (sum, count) for key k to the global table.  Returns false if the
// probe limit was hit.
__device__ __forceinline__ bool global_insert(const GroupArgs& a, uint64_t k, uint64_t sum, uint64_t cnt,
                                              unsigned long long& fresh)
{
    uint64_t s = reduce_range(mix64(k), a.cap);
    for (uint64_t steps = 0; steps < GB_PROBE_LIMIT && steps < a.cap; ++steps) {
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

template <bool SMEM>
__global__ void __launch_bounds__(GB_THREADS) groupby_kernel(GroupArgs a)
{
    extern __shared__ unsigned long long sm[];
    unsigned long long* skey = sm;
    unsigned long long* ssum = sm + GB_SMEM_SLOTS;
    unsigned int* scnt = (unsigned int*)(sm + 2 * GB_SMEM_SLOTS);
    if (SMEM) {
        for (int i = threadIdx.x; i < GB_SMEM_SLOTS; i += blockDim.x) {
            skey[i] = kEmptyKey;
            ssum[i] = 0;
            scnt[i] = 0;
        }
        __syncthreads();
    }
    const unsigned lane = threadIdx.x & 31;
    unsigned long long fresh = 0;
    bool full = false;
    uint64_t sent_sum = 0, sent_cnt = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    const int64_t first = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u);
    for (int64_t wbase = first; wbase < a.n; wbase += stride) {
        int64_t i = wbase + lane;
        bool valid = i < a.n;
        unsigned active = __ballot_sync(0xffffffffu, valid);
        if (!valid) continue;
        const uint8_t* t = a.base + i * (int64_t)a.tb;
        uint64_t k = load_key(t, a.ks);
        uint64_t v = a.want_sum ? (uint64_t)load_col(t, a.sum_off, a.sum_type) : 0;
        unsigned mask = __match_any_sync(active, k);
        uint64_t gs = a.want_sum ? group_sum_u64(mask, v) : 0;
        unsigned gc = __popc(mask);
        if (lane != (unsigned)(__ffs(mask) - 1)) continue;
        if (k == kEmptyKey) {
            sent_sum += gs;
            sent_cnt += gc;
            continue;
        }
        if (SMEM) {
            unsigned s = (unsigned)reduce_range(mix64(k), GB_SMEM_SLOTS);
            bool done = false;
            for (int steps = 0; steps < GB_SMEM_SLOTS; ++steps) {
                unsigned long long prev = skey[s];
                if (prev == kEmptyKey) prev = atomicCAS(&skey[s], kEmptyKey, k);
                if (prev == kEmptyKey || prev == k) {
                    if (a.want_sum) atomicAdd(&ssum[s], (unsigned long long)gs);
                    atomicAdd(&scnt[s], gc);
                    done = true;
                    break;
                }
                s = (s + 1 == GB_SMEM_SLOTS) ? 0 : s + 1;
            }
            if (done) continue;
        }
        if (!global_insert(a, k, gs, gc, fresh)) full = true;
    }
    if (SMEM) {
        __syncthreads();
        for (int s = threadIdx.x; s < GB_SMEM_SLOTS; s += blockDim.x) {
            uint64_t k = skey[s];
            if (k == kEmptyKey) continue;
            if (!global_insert(a, k, ssum[s], scnt[s], fresh)) full = true;
        }
    }
    if (sent_cnt) {
        atomicAdd(&a.flags[2], (unsigned long long)sent_sum);
        atomicAdd(&a.flags[3], (unsigned long long)sent_cnt);
    }
    if (fresh) atomicAdd(&a.flags[1], fresh);
    if (full) a.flags[0] = 1;
}

__global__ void gb_init_kernel(ulonglong4* __restrict__ table, uint64_t cap)
{
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x)
        table[i] = make_ulonglong4(kEmptyKey, 0, 0, 0);
}

// No GROUP BY: one sum and count over the whole input.
__global__ void __launch_bounds__(GB_THREADS) reduce_all_kernel(const uint8_t* __restrict__ base, int64_t n, int32_t tb,
                                                                int32_t off, int32_t type, int want_sum,
                                                                unsigned long long* out)
{
    uint64_t s = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        if (want_sum) s += (uint64_t)load_col(base + i * (int64_t)tb, off, type);
    s = warp_sum_u64(s);
    if ((threadIdx.x & 31) == 0 && s) atomicAdd(&out[0], (unsigned long long)s);
}

struct OutSpec {
    int32_t nkeys;
    int32_t key_type0;     // single key type
    int32_t want_sum, sum_type, want_count;
    int32_t tb;            // output tuple bytes
    int32_t sum_off, cnt_off;
};

__device__ __forceinline__ void write_group(uint8_t* dst, const OutSpec& o, uint64_t k, uint64_t sum, uint64_t cnt)
{
    if (o.nkeys == 2) {
        store_col(dst, 0, PYG_INT32, k >> 32);
        store_col(dst, 4, PYG_INT32, k);
    } else if (o.nkeys == 1) {
        store_col(dst, 0, o.key_type0, k);
    }
    if (o.want_sum) store_col(dst, o.sum_off, o.sum_type, sum);
    if (o.want_count) store_col(dst, o.cnt_off, PYG_INT64, cnt);
}

// Compaction: occupied slots -> output rows (unordered), or -> (sortable
// key, slot) pairs for the ordered path.
__global__ void gb_compact_kernel(const ulonglong4* __restrict__ table, uint64_t cap, OutSpec o, uint8_t* out,
                                  int64_t out_cap, uint64_t* skeys, uint64_t* sidx, unsigned long long* cursor)
{
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t wb = blockIdx.x * (uint64_t)blockDim.x + (threadIdx.x & ~31u); wb < cap; wb += stride) {
        uint64_t s = wb + lane;
        ulonglong4 e = s < cap ? table[s] : make_ulonglong4(kEmptyKey, 0, 0, 0);
        bool occ = e.x != kEmptyKey;
        unsigned m = __ballot_sync(0xffffffffu, occ);
        if (!m) continue;
        unsigned long long base = 0;
        if (lane == 0) base = atomicAdd(cursor, (unsigned long long)__popc(m));
        base = __shfl_sync(0xffffffffu, base, 0);
        if (!occ) continue;
        int64_t p = (int64_t)(base + __popc(m & ((1u << lane) - 1)));
        if (skeys) {
            skeys[p] = packed_to_sortable(e.x, o.nkeys);
            sidx[p] = s;
        } else if (p < out_cap) {
            write_group(out + p * o.tb, o, e.x, e.y, e.z);
        }
    }
}

__global__ void gb_write_sorted_kernel(const ulonglong4* __restrict__ table, const uint64_t* __restrict__ sidx,
                                       int64_t n, int64_t sentinel_pos, OutSpec o, uint64_t sent_key,
                                       uint64_t sent_sum, uint64_t sent_cnt, uint8_t* out)
{
    // Rows before sentinel_pos come from sidx[i], the sentinel group (if any)
    // sits at sentinel_pos, the rest shift by one.
    int64_t total = n + (sentinel_pos >= 0 ? 1 : 0);
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < total; r += (int64_t)gridDim.x * blockDim.x) {
        if (r == sentinel_pos) {
            write_group(out + r * o.tb, o, sent_key, sent_sum, sent_cnt);
            continue;
        }
        int64_t i = (sentinel_pos >= 0 && r > sentinel_pos) ? r - 1 : r;
        ulonglong4 e = table[sidx[i]];
        write_group(out + r * o.tb, o, e.x, e.y, e.z);
    }
}

__global__ void count_below_kernel(const uint64_t* __restrict__ skeys, int64_t n, uint64_t pivot,
                                   unsigned long long* out)
{
    unsigned long long c = 0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        c += skeys[i] < pivot;
    c = warp_sum_u64(c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(out, c);
}

}  // namespace pyg

using namespace pyg;

extern "C" int pyg_groupby(pyg_ctx* ctx, const pyg_rel* in, const int32_t* key_cols, int32_t nkeys, int32_t flags,
                           int32_t sum_col, int32_t sort_by_key, int64_t expected_groups, void* out,
                           int64_t out_capacity, int64_t* out_groups)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if ((rc = check_rel(in, "group-by input"))) return rc;
    if (!out_groups || (flags & ~(PYG_AGG_SUM | PYG_AGG_COUNT)) || !flags || nkeys < 0 || nkeys > 2) {
        set_error("pyg_groupby: bad arguments (flags=%d nkeys=%d)", flags, nkeys);
        return PYG_ERR_ARG;
    }
    const int want_sum = (flags & PYG_AGG_SUM) != 0;
    if (want_sum && (sum_col < 0 || sum_col >= in->ncols)) {
        set_error("pyg_groupby: sum column %d out of range", sum_col);
        return PYG_ERR_ARG;
    }
    OutSpec o;
    memset(&o, 0, sizeof(o));
    o.nkeys = nkeys;
    o.want_sum = want_sum;
    o.want_count = (flags & PYG_AGG_COUNT) != 0;
    KeySpec ks;
    memset(&ks, 0, sizeof(ks));
    int kbytes = 0;
    if (nkeys > 0) {
        if ((rc = make_keyspec(in, key_cols, nkeys, &ks))) return rc;
        o.key_type0 = ks.type0;
        kbytes = nkeys == 2 ? 8 : (ks.type0 == PYG_INT32 ? 4 : 8);
    }
    o.sum_type = want_sum ? in->col_type[sum_col] : PYG_INT64;
    o.sum_off = kbytes;
    o.cnt_off = kbytes + (want_sum ? (o.sum_type == PYG_INT32 ? 4 : 8) : 0);
    o.tb = o.cnt_off + (o.want_count ? 8 : 0);

    *out_groups = 0;
    DevRel R;
    if ((rc = R.stage(ctx, in))) return rc;
    const int threads = GB_THREADS;
    unsigned long long* h = (unsigned long long*)ctx->pinned;

    if (nkeys == 0) {
        // No GROUP BY: a single group when the input is non-empty.
        unsigned long long* acc = ctx->dcounters + 40;
        PYG_CUDA(cudaMemsetAsync(acc, 0, 8, ctx->stream));
        if (in->ntuples > 0) {
            reduce_all_kernel<<<grid_for(ctx, in->ntuples, threads, 4, 8), threads, 0, ctx->stream>>>(
                (const uint8_t*)R.rel.base, in->ntuples, in->tuple_bytes, want_sum ? in->col_offset[sum_col] : 0,
                o.sum_type, want_sum, acc);
            PYG_LAUNCHED(ctx);
        }
        PYG_CUDA(cudaMemcpyAsync(h, acc, 8, cudaMemcpyDeviceToHost, ctx->stream));
        R.release(ctx);
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (in->ntuples == 0) return PYG_OK;
        *out_groups = 1;
        if (out_capacity < 1) {
            set_error("pyg_groupby: 1 group exceeds capacity %lld", (long long)out_capacity);
            return PYG_ERR_CAPACITY;
        }
        uint8_t row[24];
        uint64_t sum = h[0], cnt = (uint64_t)in->ntuples;
        if (want_sum) {
            if (o.sum_type == PYG_INT32) { uint32_t w = (uint32_t)sum; memcpy(row, &w, 4); }
            else memcpy(row, &sum, 8);
        }
        if (o.want_count) memcpy(row + o.cnt_off, &cnt, 8);
        PYG_CUDA(cudaMemcpyAsync(out, row, o.tb, cudaMemcpyHostToDevice, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        return PYG_OK;
    }

    // No group estimate from the caller (the plan's hash.buckets): on large
    // inputs the learned CDF model's distinct-key estimate from a key
    // sample stands in, so that tables are sized for the keys at hand and
    // 16-byte tuples take the shared-memory paths.  A wrong estimate costs
    // time only.
    if (expected_groups <= 0 && in->ntuples >= ((int64_t)1 << 20)) {
        int64_t est = 0;
        if ((rc = estimate_distinct_keys(ctx, (const uint8_t*)R.rel.base, in->ntuples, in->tuple_bytes, ks, &est))) {
            R.release(ctx);
            return rc;
        }
        expected_groups = est > 0 ? est : 0;
    }
    GroupArgs a;
    memset(&a, 0, sizeof(a));
    a.base = (const uint8_t*)R.rel.base;
    a.n = in->ntuples;
    a.tb = in->tuple_bytes;
    a.ks = ks;
    a.sum_off = want_sum ? in->col_offset[sum_col] : 0;
    a.sum_type = o.sum_type;
    a.want_sum = want_sum;
    a.flags = ctx->dcounters + 40;
    uint64_t guess = expected_groups > 0 ? (uint64_t)expected_groups
                                         : (uint64_t)(in->ntuples < (1 << 22) ? in->ntuples : (1 << 22));
    uint64_t cap = 2 * guess + 64;
    bool use_smem = expected_groups > 0 && expected_groups <= GB_SMEM_MAX_GROUPS;
    size_t smem = use_smem ? GB_SMEM_SLOTS * (2 * sizeof(unsigned long long) + sizeof(unsigned)) : 0;
    if (use_smem) PYG_CUDA(cudaFuncSetAttribute(groupby_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    // 16-byte (int64 key @0, int64 value @8) tuples with a group estimate
    // are aggregated in shared memory (gbradix.cu).
    const bool fast16 = a.tb == 16 && ks.nkeys == 1 && ks.off0 == 0 && ks.type0 == PYG_INT64 &&
                        (!want_sum || (a.sum_off == 8 && a.sum_type == PYG_INT64)) && (uintptr_t)a.base % 16 == 0 &&
                        groupby16_eligible(expected_groups);
    ulonglong4* table = nullptr;
    uint64_t groups = 0, sent_sum = 0, sent_cnt = 0;
    for (;;) {
        if ((rc = dalloc(ctx, (void**)&table, cap * sizeof(ulonglong4)))) break;
        gb_init_kernel<<<grid_for(ctx, (int64_t)cap, threads, 4, 8), threads, 0, ctx->stream>>>(table, cap);
        PYG_LAUNCHED(ctx);
        PYG_CUDA(cudaMemsetAsync(a.flags, 0, 4 * sizeof(unsigned long long), ctx->stream));
        a.table = table;
        a.cap = cap;
        if (a.n > 0 && fast16) {
            if ((rc = groupby16_fill(ctx, a.base, a.n, want_sum, expected_groups, table, cap, a.flags))) break;
        } else if (a.n > 0) {
            int grid = grid_for(ctx, a.n, threads, 16, use_smem ? 2 : 8);
            if (use_smem) groupby_kernel<true><<<grid, threads, smem, ctx->stream>>>(a);
            else groupby_kernel<false><<<grid, threads, 0, ctx->stream>>>(a);
            PYG_LAUNCHED(ctx);
        }
        PYG_CUDA(cudaMemcpyAsync(h, a.flags, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (!h[0]) {
            groups = h[1];
            sent_sum = h[2];
            sent_cnt = h[3];
            break;
        }
        // The group estimate was too small: double the table and redo.
        dfree(ctx, table);
        table = nullptr;
        if (cap > 4 * (uint64_t)in->ntuples + 4096) {
            set_error("pyg_groupby: table full at capacity %llu", (unsigned long long)cap);
            rc = PYG_ERR_TABLE_FULL;
            break;
        }
        cap *= 2;
    }
    if (rc) {
        R.release(ctx);
        return rc;
    }
    int64_t total = (int64_t)groups + (sent_cnt ? 1 : 0);
    *out_groups = total;
    if (total > out_capacity) {
        dfree(ctx, table);
        R.release(ctx);
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        set_error("pyg_groupby: %lld groups exceed capacity %lld", (long long)total, (long long)out_capacity);
        return PYG_ERR_CAPACITY;
    }
    unsigned long long* cursor = ctx->dcounters + 48;
    PYG_CUDA(cudaMemsetAsync(cursor, 0, 8, ctx->stream));
    int cgrid = grid_for(ctx, (int64_t)cap, threads, 4, 8);
    if (!sort_by_key) {
        gb_compact_kernel<<<cgrid, threads, 0, ctx->stream>>>(table, cap, o, (uint8_t*)out, out_capacity, nullptr,
                                                              nullptr, cursor);
        PYG_LAUNCHED(ctx);
        if (sent_cnt) {
            uint8_t row[24];
            uint8_t* dst = (uint8_t*)out + groups * o.tb;
            // Sentinel group written through a tiny host row.
            OutSpec oo = o;
            uint64_t k = kEmptyKey;
            memset(row, 0, sizeof(row));
            if (oo.nkeys == 2) { uint32_t x = (uint32_t)(k >> 32), y = (uint32_t)k; memcpy(row, &x, 4); memcpy(row + 4, &y, 4); }
            else memcpy(row, &k, 8);
            if (oo.want_sum) { if (oo.sum_type == PYG_INT32) { uint32_t w = (uint32_t)sent_sum; memcpy(row + oo.sum_off, &w, 4); } else memcpy(row + oo.sum_off, &sent_sum, 8); }
            if (oo.want_count) memcpy(row + oo.cnt_off, &sent_cnt, 8);
            memcpy(h + 16, row, oo.tb);
            PYG_CUDA(cudaMemcpyAsync(dst, h + 16, oo.tb, cudaMemcpyHostToDevice, ctx->stream));
        }
    } else {
        uint64_t* buf = nullptr;
        int64_t g = (int64_t)groups;
        if ((rc = dalloc(ctx, (void**)&buf, (size_t)4 * (g > 0 ? g : 1) * sizeof(uint64_t)))) {
            dfree(ctx, table);
            R.release(ctx);
            return rc;
        }
        uint64_t *k0 = buf, *v0 = buf + g, *k1 = buf + 2 * g, *v1 = buf + 3 * g;
        gb_compact_kernel<<<cgrid, threads, 0, ctx->stream>>>(table, cap, o, nullptr, 0, k0, v0, cursor);
        PYG_LAUNCHED(ctx);
        int b = 0, e = 0, alt = 0;
        rc = key_bit_range(ctx, k0, g, &b, &e);
        if (!rc) rc = radix_sort_pairs(ctx, k0, v0, k1, v1, g, b, e, &alt);
        int64_t sentinel_pos = -1;
        if (!rc && sent_cnt) {
            // Place the sentinel group: number of sorted keys below it.
            uint64_t pivot = packed_to_sortable(kEmptyKey, nkeys);
            unsigned long long* c = ctx->dcounters + 56;
            cudaMemsetAsync(c, 0, 8, ctx->stream);
            count_below_kernel<<<grid_for(ctx, g > 0 ? g : 1, threads, 4, 8), threads, 0, ctx->stream>>>(
                alt ? k1 : k0, g, pivot, c);
            PYG_LAUNCHED(ctx);
            cudaMemcpyAsync(h + 8, c, 8, cudaMemcpyDeviceToHost, ctx->stream);
            cudaStreamSynchronize(ctx->stream);
            sentinel_pos = (int64_t)h[8];
        }
        if (!rc && total > 0) {
            gb_write_sorted_kernel<<<grid_for(ctx, total, threads, 4, 8), threads, 0, ctx->stream>>>(
                table, alt ? v1 : v0, g, sentinel_pos, o, kEmptyKey, sent_sum, sent_cnt, (uint8_t*)out);
            PYG_LAUNCHED(ctx);
        }
        dfree(ctx, buf);
    }
    dfree(ctx, table);
    R.release(ctx);
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    return rc;
}
