// Hash join on one B200: open-addressing table in HBM, atomicCAS inserts,
// fused count/sum probe (16-byte vector loads, several independent probes
// in flight per thread), and a materialising probe with warp-aggregated
// output allocation.
//
// Semantics follow the reference's HashJoinOp (operators/join.cpp:367-903):
// every (build, probe) pair with equal keys is one output tuple made of the
// projected columns.  The bucket function of the reference only places
// tuples; the join result does not depend on it, so the tables here use
// their own hashes and linear probing: a 64-bit bijective mix with a
// multiply-high range reduction (general tables), or the top bits of the
// radix operators' hash over a power-of-two table (the one-shot direct
// join).
#include <string.h>

#include <algorithm>
#include <vector>

#include "pyg_internal.cuh"
#include "radixjoin.cuh"
#include "hashtable.cuh"
#include "partition.cuh"

namespace pyg {

// ---------------------------------------------------------------------------
// Kernels

__global__ void ht_init_kernel(uint64_t* __restrict__ slots, uint64_t cap, int W)
{
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    if (W == 2) {
        ulonglong2* s2 = reinterpret_cast<ulonglong2*>(slots);
        for (; i < cap; i += stride) s2[i] = make_ulonglong2(kEmptyKey, 0ULL);
        return;
    }
    uint64_t words = cap * (uint64_t)W;
    for (; i < words; i += stride) slots[i] = (i % W == 0) ? kEmptyKey : 0ULL;
}

struct BuildArgs {
    const uint8_t* base;
    int64_t n;
    int32_t tb;
    KeySpec ks;
    ColSpec pay;              // stored build columns
    uint64_t* slots;
    uint64_t cap;
    int W;
    int agg;                  // AGGREGATE mode
    uint64_t* side;           // entries whose key word equals kEmptyKey
    int64_t side_cap;
    unsigned long long* flags;  // [0] dup, [1] full, [2] side count, [3] new entries
};

__global__ void ht_build_kernel(BuildArgs a)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long fresh = 0, dup = 0, full = 0;
    for (; i < a.n; i += stride) {
        const uint8_t* t = a.base + i * (int64_t)a.tb;
        uint64_t k = load_key(t, a.ks);
        if (k == kEmptyKey) {
            unsigned long long e = atomicAdd(&a.flags[2], 1ULL);
            if ((int64_t)e < a.side_cap) {
                uint64_t* dst = a.side + e * a.W;
                dst[0] = k;
                for (int c = 0; c < a.pay.n; ++c) dst[1 + c] = (uint64_t)load_col(t, a.pay.off[c], a.pay.type[c]);
            }
            continue;
        }
        uint64_t s = reduce_range(mix64(k), a.cap);
        uint64_t steps = 0;
        for (;;) {
            uint64_t* slot = a.slots + s * a.W;
            unsigned long long prev = atomicCAS((unsigned long long*)slot, kEmptyKey, k);
            if (prev == kEmptyKey) {
                ++fresh;
                if (a.agg) {
                    for (int c = 0; c < a.pay.n; ++c)
                        atomicAdd((unsigned long long*)&slot[1 + c],
                                  (unsigned long long)load_col(t, a.pay.off[c], a.pay.type[c]));
                } else {
                    for (int c = 0; c < a.pay.n; ++c) slot[1 + c] = (uint64_t)load_col(t, a.pay.off[c], a.pay.type[c]);
                }
                break;
            }
            if (prev == k) {
                dup = 1;
                if (a.agg) {
                    for (int c = 0; c < a.pay.n; ++c)
                        atomicAdd((unsigned long long*)&slot[1 + c],
                                  (unsigned long long)load_col(t, a.pay.off[c], a.pay.type[c]));
                    break;
                }
            }
            if (++steps >= a.cap) {
                full = 1;
                break;
            }
            s = (s + 1 == a.cap) ? 0 : s + 1;
        }
    }
    // One atomic per warp for the counters.
    fresh = warp_sum_u64(fresh);
    dup = __any_sync(0xffffffffu, dup != 0);
    full = __any_sync(0xffffffffu, full != 0);
    if ((threadIdx.x & 31) == 0) {
        if (fresh) atomicAdd(&a.flags[3], fresh);
        if (dup) a.flags[0] = 1;
        if (full) a.flags[1] = 1;
    }
}

// Fast build for 16-byte (int64 key @0, int64 payload @8) tuples into a
// one-payload AGGREGATE table.  A fresh insert is one 16-byte CAS of the
// whole slot ({empty, 0} -> {key, payload}); only a duplicate key adds its
// payload with a second atomic.  Each thread keeps UNROLL independent
// insert chains in flight (loads, then the first CAS of every chain, then
// resolution).
__device__ __forceinline__ unsigned __int128 slot128(uint64_t key, uint64_t pay)
{
    return ((unsigned __int128)pay << 64) | (unsigned __int128)key;
}

template <int UNROLL>
__global__ void __launch_bounds__(256) ht_build16_kernel(BuildArgs a)
{
    const longlong2* R = reinterpret_cast<const longlong2*>(a.base);
    unsigned long long* slots = reinterpret_cast<unsigned long long*>(a.slots);
    unsigned __int128* slots128 = reinterpret_cast<unsigned __int128*>(a.slots);
    const unsigned __int128 empty = slot128(kEmptyKey, 0);
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    unsigned long long fresh = 0;
    bool dup = false, full = false;
    for (int64_t base = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; base < a.n; base += stride * UNROLL) {
        longlong2 t[UNROLL];
        uint64_t s[UNROLL];
        unsigned long long prev[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            int64_t i = base + u * stride;
            t[u] = i < a.n ? __ldcs(&R[i]) : make_longlong2((long long)kEmptyKey, 0);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            uint64_t k = (uint64_t)t[u].x;
            s[u] = reduce_range(mix64(k), a.cap);
            prev[u] = k == kEmptyKey
                          ? ~0ULL
                          : (unsigned long long)atomicCAS(&slots128[s[u]], empty, slot128(k, (uint64_t)t[u].y));
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            int64_t i = base + u * stride;
            if (i >= a.n) continue;
            uint64_t k = (uint64_t)t[u].x;
            if (k == kEmptyKey) {
                unsigned long long e = atomicAdd(&a.flags[2], 1ULL);
                if ((int64_t)e < a.side_cap) {
                    a.side[2 * e] = k;
                    a.side[2 * e + 1] = (uint64_t)t[u].y;
                }
                continue;
            }
            uint64_t ss = s[u];
            unsigned long long pv = prev[u];  // key word of the slot before the CAS
            uint64_t steps = 0;
            while (pv != kEmptyKey && pv != k) {
                if (++steps >= a.cap) {
                    full = true;
                    break;
                }
                ss = (ss + 1 == a.cap) ? 0 : ss + 1;
                pv = (unsigned long long)atomicCAS(&slots128[ss], empty, slot128(k, (uint64_t)t[u].y));
            }
            if (pv == kEmptyKey) {
                ++fresh;  // the CAS stored key and payload together
            } else if (pv == k) {
                dup = true;
                atomicAdd(&slots[2 * ss + 1], (unsigned long long)t[u].y);
            }
        }
    }
    fresh = warp_sum_u64(fresh);
    bool anydup = __any_sync(0xffffffffu, dup), anyfull = __any_sync(0xffffffffu, full);
    if ((threadIdx.x & 31) == 0) {
        if (fresh) atomicAdd(&a.flags[3], fresh);
        if (anydup) a.flags[0] = 1;
        if (anyfull) a.flags[1] = 1;
    }
}

// Duplicate counts for an AGGREGATE table (run only when duplicates exist).
__global__ void ht_count_kernel(BuildArgs a, unsigned long long* __restrict__ counts)
{
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < a.n; i += stride) {
        uint64_t k = load_key(a.base + i * (int64_t)a.tb, a.ks);
        if (k == kEmptyKey) continue;
        uint64_t s = reduce_range(mix64(k), a.cap);
        for (uint64_t steps = 0; steps < a.cap; ++steps) {
            uint64_t key = a.slots[s * a.W];
            if (key == k) {
                atomicAdd(&counts[s], 1ULL);
                break;
            }
            if (key == kEmptyKey) break;
            s = (s + 1 == a.cap) ? 0 : s + 1;
        }
    }
}

// Shared accumulation of probe results: [0] = count, [1 + p] = sum of
// projected column p.
__device__ __forceinline__ void block_flush(uint64_t* acc, int nacc, unsigned long long* out)
{
    __shared__ unsigned long long red[PYG_MAX_COLS + 1];
    if (threadIdx.x <= PYG_MAX_COLS) red[threadIdx.x] = 0;
    __syncthreads();
    for (int j = 0; j < nacc; ++j) {
        uint64_t v = warp_sum_u64(acc[j]);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&red[j], (unsigned long long)v);
    }
    __syncthreads();
    if (threadIdx.x < nacc && red[threadIdx.x]) atomicAdd(&out[threadIdx.x], red[threadIdx.x]);
}

// Fast path: 16-byte (int64 key, int64 value) probe tuples against a
// 16-byte-slot AGGREGATE table (one int64 build payload); accumulates the
// match count, the build-payload sum and the probe-value sum.  FILLERS:
// tuples whose key is the empty marker are padding (skipped) rather than
// real keys (matched against the side list).
#ifndef PYG_PROBE_UNROLL
#define PYG_PROBE_UNROLL 4
#endif
#ifndef PYG_PROBE_MIN_BLOCKS
#define PYG_PROBE_MIN_BLOCKS 4
#endif

template <int UNROLL, bool FILLERS>
__global__ void __launch_bounds__(256, PYG_PROBE_MIN_BLOCKS) probe_agg16_kernel(const longlong2* __restrict__ S, int64_t n,
                                                          const ulonglong2* __restrict__ slots, uint64_t cap,
                                                          const unsigned long long* __restrict__ counts,
                                                          const uint64_t* __restrict__ side, int64_t nside,
                                                          unsigned long long* __restrict__ out,
                                                          const unsigned long long* __restrict__ gate,
                                                          int64_t side_cap)
{
    // gate (optional): the build's flags, read here instead of on the host.
    // A build with repeated keys (no count array), a full table or more
    // empty-marker keys than the side list holds is probed again by the
    // general path, so this launch does nothing.
    if (gate) {
        const unsigned long long dup = gate[0], full = gate[1], ns = gate[2];
        if (dup | full || ns > (unsigned long long)side_cap) return;
        nside = (int64_t)ns;
    }
    uint64_t cnt = 0, bsum = 0, psum = 0;
    const int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t base = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    for (; base < n; base += stride * UNROLL) {
        longlong2 t[UNROLL];
        uint64_t s[UNROLL];
        ulonglong2 e[UNROLL];
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            int64_t idx = base + u * stride;
            t[u] = idx < n ? __ldcs(&S[idx]) : make_longlong2((long long)kEmptyKey, 0);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            s[u] = reduce_range(mix64((uint64_t)t[u].x), cap);
            e[u] = __ldg(&slots[s[u]]);
        }
#pragma unroll
        for (int u = 0; u < UNROLL; ++u) {
            int64_t idx = base + u * stride;
            if (idx >= n) continue;
            uint64_t k = (uint64_t)t[u].x;
            if (k == kEmptyKey) {
                if (FILLERS) continue;
                for (int64_t j = 0; j < nside; ++j)
                    if (side[2 * j] == k) {
                        ++cnt;
                        bsum += side[2 * j + 1];
                        psum += (uint64_t)t[u].y;
                    }
                continue;
            }
            uint64_t ss = s[u];
            ulonglong2 ee = e[u];
            uint64_t steps = 0;
            while (ee.x != k && ee.x != kEmptyKey && ++steps < cap) {
                ss = (ss + 1 == cap) ? 0 : ss + 1;
                ee = __ldg(&slots[ss]);
            }
            if (ee.x == k) {
                uint64_t c = counts ? (uint64_t)counts[ss] : 1ULL;
                cnt += c;
                bsum += ee.y;
                psum += c * (uint64_t)t[u].y;
            }
        }
    }
    uint64_t acc[3] = {cnt, bsum, psum};
    block_flush(acc, 3, out);
}

struct ProbeArgs {
    const uint8_t* base;
    int64_t n;
    int32_t tb;
    KeySpec ks;
    const uint64_t* slots;
    uint64_t cap;
    int W;
    int agg;
    const unsigned long long* counts;
    const uint64_t* side;
    int64_t nside;
    int nproj;
    int32_t pside[PYG_MAX_COLS];   // 0 build, 1 probe
    int32_t pidx[PYG_MAX_COLS];    // build: word index in slot (1..W-1); probe: unused
    int32_t poff[PYG_MAX_COLS];    // probe column offset / output offset
    int32_t ptype[PYG_MAX_COLS];   // column type
    int32_t outoff[PYG_MAX_COLS];  // byte offset in the output tuple
    int32_t out_tb;
};

// Generic fused count/sum probe (any layout, either table mode).
__global__ void __launch_bounds__(256) probe_agg_kernel(ProbeArgs a, unsigned long long* __restrict__ out)
{
    uint64_t acc[PYG_MAX_COLS + 1];
#pragma unroll
    for (int j = 0; j <= PYG_MAX_COLS; ++j) acc[j] = 0;
    int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    for (; i < a.n; i += stride) {
        const uint8_t* t = a.base + i * (int64_t)a.tb;
        uint64_t k = load_key(t, a.ks);
        uint64_t pv[PYG_MAX_COLS];
        for (int p = 0; p < a.nproj; ++p)
            pv[p] = a.pside[p] ? (uint64_t)load_col(t, a.poff[p], a.ptype[p]) : 0;
        if (k == kEmptyKey) {
            for (int64_t j = 0; j < a.nside; ++j) {
                const uint64_t* e = a.side + j * a.W;
                if (e[0] != k) continue;
                acc[0] += 1;
                for (int p = 0; p < a.nproj; ++p) acc[1 + p] += a.pside[p] ? pv[p] : e[a.pidx[p]];
            }
            continue;
        }
        uint64_t s = reduce_range(mix64(k), a.cap);
        for (uint64_t steps = 0; steps < a.cap; ++steps) {
            const uint64_t* e = a.slots + s * a.W;
            uint64_t key = e[0];
            if (key == kEmptyKey) break;
            if (key == k) {
                uint64_t c = a.counts ? (uint64_t)a.counts[s] : 1ULL;
                acc[0] += c;
                for (int p = 0; p < a.nproj; ++p) acc[1 + p] += a.pside[p] ? c * pv[p] : e[a.pidx[p]];
                if (a.agg) break;
            }
            s = (s + 1 == a.cap) ? 0 : s + 1;
        }
    }
    block_flush(acc, a.nproj + 1, out);
}


// Materialising probe.  Each lane first counts its matches, the warp
// reserves one contiguous output range with a single atomic, then every lane
// walks its chain again writing its pairs.  Pairs past the capacity are
// counted but not written.
__global__ void __launch_bounds__(256) probe_mat_kernel(ProbeArgs a, uint8_t* __restrict__ out, int64_t out_cap,
                                                        unsigned long long* __restrict__ cursor)
{
    const unsigned lane = threadIdx.x & 31;
    int64_t stride = (int64_t)gridDim.x * blockDim.x;
    int64_t first = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31u);
    // Whole warps iterate together so the warp-wide scan stays converged.
    for (int64_t wbase = first; wbase < a.n; wbase += stride) {
        int64_t i = wbase + lane;
        bool valid = i < a.n;
        const uint8_t* t = valid ? a.base + i * (int64_t)a.tb : nullptr;
        uint64_t k = valid ? load_key(t, a.ks) : 0;
        uint64_t s0 = valid ? reduce_range(mix64(k), a.cap) : 0;
        unsigned long long m = 0;
        if (valid) {
            if (k == kEmptyKey) {
                for (int64_t j = 0; j < a.nside; ++j) m += (a.side[j * a.W] == k);
            } else {
                uint64_t s = s0;
                for (uint64_t steps = 0; steps < a.cap; ++steps) {
                    uint64_t key = a.slots[s * a.W];
                    if (key == kEmptyKey) break;
                    m += (key == k);
                    s = (s + 1 == a.cap) ? 0 : s + 1;
                }
            }
        }
        // Warp-inclusive scan of match counts.
        unsigned long long incl = m;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            unsigned long long v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= (unsigned)o) incl += v;
        }
        unsigned long long total = __shfl_sync(0xffffffffu, incl, 31);
        unsigned long long wstart = 0;
        if (lane == 31 && total) wstart = atomicAdd(cursor, total);
        wstart = __shfl_sync(0xffffffffu, wstart, 31);
        if (!valid || m == 0) continue;
        int64_t pos = (int64_t)(wstart + incl - m);
        auto emit = [&](const uint64_t* e) {
            if (pos < out_cap) {
                uint8_t* dst = out + pos * (int64_t)a.out_tb;
                for (int p = 0; p < a.nproj; ++p) {
                    uint64_t v = a.pside[p] ? (uint64_t)load_col(t, a.poff[p], a.ptype[p]) : e[a.pidx[p]];
                    store_col(dst, a.outoff[p], a.ptype[p], v);
                }
            }
            ++pos;
        };
        if (k == kEmptyKey) {
            for (int64_t j = 0; j < a.nside; ++j)
                if (a.side[j * a.W] == k) emit(a.side + j * a.W);
        } else {
            uint64_t s = s0;
            for (uint64_t steps = 0; steps < a.cap; ++steps) {
                const uint64_t* e = a.slots + s * a.W;
                if (e[0] == kEmptyKey) break;
                if (e[0] == k) emit(e);
                s = (s + 1 == a.cap) ? 0 : s + 1;
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Host side

static int fill_probe_args(pyg_ctx* ctx, const pyg_hashtable* ht, const pyg_rel* S, const int32_t* key_cols,
                           const pyg_proj* proj, int32_t nproj, ProbeArgs* a)
{
    (void)ctx;
    memset(a, 0, sizeof(*a));
    if (nproj < 0 || nproj > PYG_MAX_COLS || (nproj > 0 && !proj)) {
        set_error("probe: nproj must be in [0, %d]", PYG_MAX_COLS);
        return PYG_ERR_ARG;
    }
    int rc = make_keyspec(S, key_cols, ht->nkeys, &a->ks);
    if (rc) return rc;
    if (a->ks.nkeys != ht->ks.nkeys) {
        set_error("probe: key arity differs from the build side");
        return PYG_ERR_ARG;
    }
    a->base = (const uint8_t*)S->base;
    a->n = S->ntuples;
    a->tb = S->tuple_bytes;
    a->slots = ht->slots;
    a->cap = ht->cap;
    a->W = ht->W;
    a->agg = ht->mode == PYG_HT_AGGREGATE;
    a->counts = ht->counts;
    a->side = ht->side;
    a->nside = ht->nside;
    a->nproj = nproj;
    int off = 0;
    for (int p = 0; p < nproj; ++p) {
        a->pside[p] = proj[p].side ? 1 : 0;
        if (proj[p].side) {
            if (proj[p].col < 0 || proj[p].col >= S->ncols) {
                set_error("probe: projection P$%d out of range", proj[p].col);
                return PYG_ERR_ARG;
            }
            a->poff[p] = S->col_offset[proj[p].col];
            a->ptype[p] = S->col_type[proj[p].col];
        } else {
            int w = -1;
            for (int c = 0; c < ht->npay; ++c)
                if (ht->pay_cols[c] == proj[p].col) w = c;
            if (w < 0) {
                set_error("probe: projection B$%d is not a stored build column", proj[p].col);
                return PYG_ERR_ARG;
            }
            a->pidx[p] = 1 + w;
            a->ptype[p] = ht->pay_types[w];
        }
        a->outoff[p] = off;
        off += a->ptype[p] == PYG_INT32 ? 4 : 8;
    }
    a->out_tb = off;
    return PYG_OK;
}


// 16-byte fast layout: (int64 key @0, int64 value @8) probe tuples, a
// one-payload AGGREGATE table, projection over {B$payload, P$1}.
static bool fast16_layout(const pyg_hashtable* ht, const ProbeArgs& a, const pyg_rel* probe, int nproj, int* fb,
                          int* fp)
{
    bool fast = a.agg && ht->W == 2 && probe->tuple_bytes == 16 && a.ks.nkeys == 1 && a.ks.off0 == 0 &&
                a.ks.type0 == PYG_INT64 && nproj <= 2 && ht->pay_types[0] == PYG_INT64;
    *fb = *fp = -1;
    for (int p = 0; fast && p < nproj; ++p) {
        if (a.pside[p] == 0 && a.ptype[p] == PYG_INT64 && *fb < 0) *fb = p;
        else if (a.pside[p] == 1 && a.poff[p] == 8 && a.ptype[p] == PYG_INT64 && *fp < 0) *fp = p;
        else fast = false;
    }
    return fast;
}

static void fill_result(pyg_join_result* out, const unsigned long long* h, const ProbeArgs& a, int nproj, bool fast,
                        int fb)
{
    memset(out, 0, sizeof(*out));
    out->count = (int64_t)h[0];
    for (int p = 0; p < nproj; ++p) {
        uint64_t v;
        if (fast) v = (p == fb) ? h[1] : h[2];
        else v = h[1 + p];
        out->sums[p] = a.ptype[p] == PYG_INT32 ? (int64_t)(int32_t)(uint32_t)v : (int64_t)v;
    }
}

static int launch_probe16(pyg_ctx* ctx, const pyg_hashtable* ht, const longlong2* S, int64_t n, bool fillers,
                          unsigned long long* acc)
{
    if (n <= 0) return PYG_OK;
    int threads = 256;
    constexpr int U = PYG_PROBE_UNROLL;
    int grid = grid_for(ctx, n, threads, U, 8);
    if (fillers)
        probe_agg16_kernel<U, true><<<grid, threads, 0, ctx->stream>>>(S, n, (const ulonglong2*)ht->slots, ht->cap,
                                                                       ht->counts, ht->side, ht->nside, acc, nullptr,
                                                                       0);
    else
        probe_agg16_kernel<U, false><<<grid, threads, 0, ctx->stream>>>(S, n, (const ulonglong2*)ht->slots, ht->cap,
                                                                        ht->counts, ht->side, ht->nside, acc, nullptr,
                                                                        0);
    PYG_LAUNCHED(ctx);
    return PYG_OK;
}

static int probe16_stream_host(pyg_ctx* ctx, const pyg_hashtable* ht, const longlong2* host, int64_t n,
                               unsigned long long* acc)
{
    const int64_t chunk = (int64_t)1 << 25;  // 512 MiB of tuples per buffer
    int64_t per = n < chunk ? n : chunk;
    longlong2* buf[2] = {nullptr, nullptr};
    int rc = dalloc(ctx, (void**)&buf[0], (size_t)per * 16);
    if (!rc) rc = dalloc(ctx, (void**)&buf[1], (size_t)per * 16);
    if (!rc) {
        // Buffers become usable on the copy stream once allocated.
        cudaEventRecord(ctx->consumed[0], ctx->stream);
        cudaEventRecord(ctx->consumed[1], ctx->stream);
        int64_t i = 0;
        for (int64_t off = 0; off < n && !rc; off += per, ++i) {
            int b = (int)(i & 1);
            int64_t len = n - off < per ? n - off : per;
            cudaStreamWaitEvent(ctx->copy_stream, ctx->consumed[b], 0);
            cudaError_t e = cudaMemcpyAsync(buf[b], host + off, (size_t)len * 16, cudaMemcpyHostToDevice,
                                            ctx->copy_stream);
            if (e != cudaSuccess) {
                rc = cuda_status(e, "probe chunk copy");
                break;
            }
            cudaEventRecord(ctx->copied[b], ctx->copy_stream);
            cudaStreamWaitEvent(ctx->stream, ctx->copied[b], 0);
            rc = launch_probe16(ctx, ht, buf[b], len, false, acc);
            cudaEventRecord(ctx->consumed[b], ctx->stream);
        }
    }
    dfree(ctx, buf[0]);
    dfree(ctx, buf[1]);
    return rc;
}

struct PhaseTimer {
    static constexpr int N = 5;
    cudaEvent_t ev[N] = {};
    bool on = false;
    void start(pyg_ctx* ctx, bool enable)
    {
        on = enable;
        if (!on) return;
        for (auto& e : ev) cudaEventCreate(&e);
        for (auto& e : ev) cudaEventRecord(e, ctx->stream);
    }
    void mark(pyg_ctx* ctx, int i)
    {
        if (on) cudaEventRecord(ev[i], ctx->stream);
    }
    // Phases between consecutive marks: build-side partition, build,
    // probe-side partition, probe.
    void finish(pyg_join_stats* st)
    {
        if (!on) return;
        cudaEventSynchronize(ev[N - 1]);
        float ms[N - 1];
        for (int i = 0; i + 1 < N; ++i) cudaEventElapsedTime(&ms[i], ev[i], ev[i + 1]);
        st->build_partition_ms = ms[0];
        st->build_ms = ms[1];
        st->probe_partition_ms = ms[2];
        st->probe_ms = ms[3];
        for (auto& e : ev) cudaEventDestroy(e);
    }
};

// ---------------------------------------------------------------------------
// One-shot direct join of 16-byte (int64 key @0, int64 payload @8) device
// relations.  The table is 2^b 16-byte slots {key, payload} (kEmptyKey marks
// a free slot), slot = the top b bits of the radix operators' hash (rj_hash:
// three xor-shifts, then a Fibonacci multiply), linear probing.  A block
// walks tiles of DJ_THREADS x DJ_U consecutive tuples, thread t taking
// tuples t, t + DJ_THREADS, ...: one 64-bit tile base per tile, constant
// offsets inside it, and DJ_U independent loads (and CASes / table reads)
// in flight per thread.  Build keys equal to kEmptyKey go to a side list;
// probe keys equal to it are matched against that list.

constexpr int DJ_THREADS = 256;
#ifndef PYG_DJ_UNROLL
#define PYG_DJ_UNROLL 4
#endif
constexpr int DJ_U = PYG_DJ_UNROLL;

__device__ __forceinline__ uint64_t dj_slot(uint64_t k, int shift) { return rj_hash(k) >> shift; }

// Empty table of cap 16-byte slots and nwords zeroed counter words.
__global__ void dj_clear_kernel(ulonglong2* __restrict__ slots, uint64_t cap, unsigned long long* __restrict__ words,
                                int nwords)
{
    uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (i < (uint64_t)nwords) words[i] = 0;
    for (; i < cap; i += (uint64_t)gridDim.x * blockDim.x) slots[i] = make_ulonglong2(kEmptyKey, 0ULL);
}

// Build: one 16-byte CAS stores key and payload together.  flags: [0] a
// repeated key, [1] no free slot found, [2] side-list entries.  The table
// has more slots than build tuples, so an insert always finds a free slot.
__global__ void __launch_bounds__(DJ_THREADS) dj_build_kernel(const longlong2* __restrict__ R, int64_t n,
                                                              ulonglong2* __restrict__ slots, uint64_t mask, int shift,
                                                              uint64_t* __restrict__ side, int64_t side_cap,
                                                              unsigned long long* __restrict__ flags)
{
    unsigned __int128* s128 = reinterpret_cast<unsigned __int128*>(slots);
    const unsigned __int128 empty = slot128(kEmptyKey, 0);
    const int64_t tile = (int64_t)DJ_THREADS * DJ_U;
    bool dup = false, full = false;
    for (int64_t t0 = (int64_t)blockIdx.x * tile; t0 < n; t0 += (int64_t)gridDim.x * tile) {
        const longlong2* p = R + t0 + threadIdx.x;
        const int64_t left = n - t0 - (int64_t)threadIdx.x;  // p[u * DJ_THREADS] exists iff u * DJ_THREADS < left
        longlong2 t[DJ_U];
        uint64_t s[DJ_U];
        unsigned long long prev[DJ_U];
#pragma unroll
        for (int u = 0; u < DJ_U; ++u)
            t[u] = u * DJ_THREADS < left ? __ldcs(p + u * DJ_THREADS) : make_longlong2((long long)kEmptyKey, 0);
#pragma unroll
        for (int u = 0; u < DJ_U; ++u) {
            const uint64_t k = (uint64_t)t[u].x;
            s[u] = dj_slot(k, shift);
            prev[u] = k == kEmptyKey
                          ? kEmptyKey
                          : (unsigned long long)atomicCAS(&s128[s[u]], empty, slot128(k, (uint64_t)t[u].y));
        }
#pragma unroll
        for (int u = 0; u < DJ_U; ++u) {
            if (u * DJ_THREADS >= left) continue;
            const uint64_t k = (uint64_t)t[u].x;
            if (k == kEmptyKey) {
                const unsigned long long e = atomicAdd(&flags[2], 1ULL);
                if ((int64_t)e < side_cap) {
                    side[2 * e] = k;
                    side[2 * e + 1] = (uint64_t)t[u].y;
                }
                continue;
            }
            uint64_t ss = s[u];
            unsigned long long pv = prev[u];  // key word of the slot before the CAS
            for (uint64_t steps = 0; pv != kEmptyKey && pv != k;) {
                if (++steps > mask) {
                    full = true;
                    break;
                }
                ss = (ss + 1) & mask;
                pv = (unsigned long long)atomicCAS(&s128[ss], empty, slot128(k, (uint64_t)t[u].y));
            }
            dup |= pv == k;
        }
    }
    const bool anydup = __any_sync(0xffffffffu, dup), anyfull = __any_sync(0xffffffffu, full);
    if ((threadIdx.x & 31) == 0) {
        if (anydup) flags[0] = 1;
        if (anyfull) flags[1] = 1;
    }
}

// Probe of one tuple whose home slot held e.
__device__ __forceinline__ void dj_match(const longlong2 t, ulonglong2 e, uint64_t s, const ulonglong2* __restrict__ slots,
                                         uint64_t mask, const uint64_t* __restrict__ side, int64_t nside,
                                         uint64_t& cnt, uint64_t& bsum, uint64_t& psum)
{
    const uint64_t k = (uint64_t)t.x;
    if (k == kEmptyKey) {
        for (int64_t j = 0; j < nside; ++j)
            if (side[2 * j] == k) {
                ++cnt;
                bsum += side[2 * j + 1];
                psum += (uint64_t)t.y;
            }
        return;
    }
    for (uint64_t steps = 0; e.x != k; ++steps) {
        if (e.x == kEmptyKey || steps > mask) return;
        s = (s + 1) & mask;
        e = __ldg(&slots[s]);
    }
    ++cnt;
    bsum += e.y;
    psum += (uint64_t)t.y;
}

// Probe with the fused count / sum sink: out[0] += matches, out[1] += build
// payloads, out[2] += probe payloads.  flags are the build's: a build that
// repeated a key or overfilled its side list is probed by the general path,
// so this launch then does nothing.
__global__ void __launch_bounds__(DJ_THREADS) dj_probe_kernel(const longlong2* __restrict__ S, int64_t n,
                                                              const ulonglong2* __restrict__ slots, uint64_t mask,
                                                              int shift, const uint64_t* __restrict__ side,
                                                              int64_t side_cap,
                                                              const unsigned long long* __restrict__ flags,
                                                              unsigned long long* __restrict__ out)
{
    const unsigned long long dup = flags[0], full = flags[1], ns = flags[2];
    if (dup | full || ns > (unsigned long long)side_cap) return;
    const int64_t nside = (int64_t)ns;
    uint64_t cnt = 0, bsum = 0, psum = 0;
    const int64_t tile = (int64_t)DJ_THREADS * DJ_U;
    for (int64_t t0 = (int64_t)blockIdx.x * tile; t0 < n; t0 += (int64_t)gridDim.x * tile) {
        const longlong2* p = S + t0 + threadIdx.x;
        const int64_t left = n - t0 - (int64_t)threadIdx.x;
        longlong2 t[DJ_U];
        ulonglong2 e[DJ_U];
        uint64_t s[DJ_U];
        if (left > (int64_t)(DJ_U - 1) * DJ_THREADS) {
#pragma unroll
            for (int u = 0; u < DJ_U; ++u) t[u] = __ldcs(p + u * DJ_THREADS);
#pragma unroll
            for (int u = 0; u < DJ_U; ++u) {
                s[u] = dj_slot((uint64_t)t[u].x, shift);
                e[u] = __ldg(&slots[s[u]]);
            }
#pragma unroll
            for (int u = 0; u < DJ_U; ++u) dj_match(t[u], e[u], s[u], slots, mask, side, nside, cnt, bsum, psum);
        } else {
            for (int u = 0; u * DJ_THREADS < left; ++u) {
                const longlong2 tu = __ldcs(p + u * DJ_THREADS);
                const uint64_t su = dj_slot((uint64_t)tu.x, shift);
                dj_match(tu, __ldg(&slots[su]), su, slots, mask, side, nside, cnt, bsum, psum);
            }
        }
    }
    uint64_t acc[3] = {cnt, bsum, psum};
    block_flush(acc, 3, out);
}

// Side-list capacity of the direct join (build keys equal to kEmptyKey).
static int64_t direct_side_cap(int64_t nR) { return nR < 1024 ? (nR > 0 ? nR : 1) : 1024; }

int direct_join16_enqueue(pyg_ctx* ctx, const void* Rv, int64_t nR, const void* Sv, int64_t nS, float lf,
                          unsigned long long* words, PhaseTimer* tm)
{
    const longlong2* R = (const longlong2*)Rv;
    const longlong2* S = (const longlong2*)Sv;
    // 2^bits slots, more than nR / lf (so at least one slot stays free).
    int bits = 6;
    while (bits < 62 && (double)((uint64_t)1 << bits) * (double)lf <= (double)nR) ++bits;
    const uint64_t cap = (uint64_t)1 << bits;
    const int64_t side_cap = direct_side_cap(nR);
    const size_t need = (size_t)cap * 16 + (size_t)side_cap * 16;
    if (ctx->join_arena_bytes < need) {
        // Stream-ordered: earlier joins on the stream finish with the old
        // arena before its memory is reused.
        dfree(ctx, ctx->join_arena);
        ctx->join_arena = nullptr;
        ctx->join_arena_bytes = 0;
        int rc = dalloc(ctx, &ctx->join_arena, need);
        if (rc) return rc;
        ctx->join_arena_bytes = need;
    }
    ulonglong2* slots = (ulonglong2*)ctx->join_arena;
    uint64_t* side = (uint64_t*)(slots + cap);
    dj_clear_kernel<<<grid_for(ctx, (int64_t)cap, 256, 4, 8), 256, 0, ctx->stream>>>(slots, cap, words, 11);
    PYG_LAUNCHED(ctx);
    if (tm) tm->mark(ctx, 1);
    if (nR > 0) {
        dj_build_kernel<<<grid_for(ctx, nR, DJ_THREADS, DJ_U, 8), DJ_THREADS, 0, ctx->stream>>>(
            R, nR, slots, cap - 1, 64 - bits, side, side_cap, words);
        PYG_LAUNCHED(ctx);
    }
    if (tm) {
        tm->mark(ctx, 2);
        tm->mark(ctx, 3);
    }
    if (nS > 0) {
        dj_probe_kernel<<<grid_for(ctx, nS, DJ_THREADS, DJ_U, 8), DJ_THREADS, 0, ctx->stream>>>(
            S, nS, slots, cap - 1, 64 - bits, side, side_cap, words, words + 8);
        PYG_LAUNCHED(ctx);
    }
    if (tm) tm->mark(ctx, 4);
    return PYG_OK;
}

bool direct_join16_result(const unsigned long long* w, int64_t nR, unsigned long long res[3])
{
    if (w[0] || w[1] || w[2] > (unsigned long long)direct_side_cap(nR)) return false;
    res[0] = w[8];
    res[1] = w[9];
    res[2] = w[10];
    return true;
}

// One-shot join + sum of 16-byte (int64 key @0, int64 payload @8) device
// relations through one table in HBM (L2-resident for build sides up to a
// few million tuples): clear, build, probe as three launches, one copy of
// the counter words and one host synchronisation.  The table and its side
// list live in the context's grow-only arena, so a call allocates nothing
// once the arena is large enough.  The probe reads the build's flags on
// the device; when the build side repeated a key or had more empty-marker
// keys than the side list holds, the probe does nothing, *fallback is set
// and the caller takes the general path.
// res = {count, build payload sum, probe payload sum}.
static int direct_join16(pyg_ctx* ctx, const longlong2* R, int64_t nR, const longlong2* S, int64_t nS, float lf,
                         unsigned long long res[3], bool* fallback, PhaseTimer* tm)
{
    unsigned long long* words = ctx->dcounters;  // [0..2] build flags, [8..10] probe sums
    int rc = direct_join16_enqueue(ctx, R, nR, S, nS, lf, words, tm);
    if (rc) return rc;
    unsigned long long* h = (unsigned long long*)ctx->pinned;
    PYG_CUDA(cudaMemcpyAsync(h, words, 11 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    *fallback = !direct_join16_result(h, nR, res);
    return PYG_OK;
}

}  // namespace pyg

using namespace pyg;

extern "C" {

int pyg_hashjoin_build(pyg_ctx* ctx, const pyg_rel* build, const int32_t* key_cols, int32_t nkeys,
                       const int32_t* payload_cols, int32_t npayload, int32_t mode, float load_factor,
                       pyg_hashtable** out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out) {
        set_error("pyg_hashjoin_build: null out");
        return PYG_ERR_ARG;
    }
    *out = nullptr;
    if ((rc = check_rel(build, "build"))) return rc;
    if (mode != PYG_HT_AGGREGATE && mode != PYG_HT_MATERIALIZE) {
        set_error("pyg_hashjoin_build: bad mode %d", mode);
        return PYG_ERR_ARG;
    }
    if (!(load_factor > 0.f && load_factor <= 0.95f)) {
        set_error("pyg_hashjoin_build: load factor %f outside (0, 0.95]", (double)load_factor);
        return PYG_ERR_ARG;
    }
    if (npayload < 0 || npayload > PYG_MAX_COLS - 1 || (npayload > 0 && !payload_cols)) {
        set_error("pyg_hashjoin_build: npayload must be in [0, %d]", PYG_MAX_COLS - 1);
        return PYG_ERR_ARG;
    }
    pyg_hashtable* ht = new pyg_hashtable();
    ht->mode = mode;
    ht->nkeys = nkeys;
    if ((rc = make_keyspec(build, key_cols, nkeys, &ht->ks))) {
        delete ht;
        return rc;
    }
    ht->npay = npayload;
    BuildArgs a;
    memset(&a, 0, sizeof(a));
    a.pay.n = npayload;
    for (int c = 0; c < npayload; ++c) {
        if (payload_cols[c] < 0 || payload_cols[c] >= build->ncols) {
            set_error("pyg_hashjoin_build: payload column %d out of range", payload_cols[c]);
            delete ht;
            return PYG_ERR_ARG;
        }
        ht->pay_cols[c] = payload_cols[c];
        ht->pay_types[c] = build->col_type[payload_cols[c]];
        a.pay.off[c] = build->col_offset[payload_cols[c]];
        a.pay.type[c] = build->col_type[payload_cols[c]];
    }
    ht->W = 1 + npayload;
    uint64_t cap = (uint64_t)((double)build->ntuples / (double)load_factor) + 1;
    if (cap < 64) cap = 64;
    ht->cap = cap;

    DevRel R;
    if ((rc = R.stage(ctx, build))) {
        delete ht;
        return rc;
    }
    int64_t side_cap = build->ntuples < 1024 ? (build->ntuples > 0 ? build->ntuples : 1) : 1024;
    for (int attempt = 0; attempt < 2; ++attempt) {
        if ((rc = dalloc(ctx, (void**)&ht->slots, cap * ht->W * sizeof(uint64_t)))) break;
        if ((rc = dalloc(ctx, (void**)&ht->side, side_cap * ht->W * sizeof(uint64_t)))) break;
        int threads = 256;
        int grid = grid_for(ctx, (int64_t)cap * (ht->W == 2 ? 1 : ht->W), threads, 4, 8);
        ht_init_kernel<<<grid, threads, 0, ctx->stream>>>(ht->slots, cap, ht->W);
        PYG_LAUNCHED(ctx);
        unsigned long long* flags = ctx->dcounters;
        PYG_CUDA(cudaMemsetAsync(flags, 0, 8 * sizeof(unsigned long long), ctx->stream));
        a.base = (const uint8_t*)R.rel.base;
        a.n = build->ntuples;
        a.tb = build->tuple_bytes;
        a.ks = ht->ks;
        a.slots = ht->slots;
        a.cap = cap;
        a.W = ht->W;
        a.agg = mode == PYG_HT_AGGREGATE;
        a.side = ht->side;
        a.side_cap = side_cap;
        a.flags = flags;
        if (a.n > 0) {
            bool fast = a.agg && a.W == 2 && a.tb == 16 && a.ks.nkeys == 1 && a.ks.off0 == 0 &&
                        a.ks.type0 == PYG_INT64 && a.pay.off[0] == 8 && a.pay.type[0] == PYG_INT64 &&
                        (uintptr_t)a.base % 16 == 0;
            if (fast) {
                grid = grid_for(ctx, a.n, threads, 4, 8);
                ht_build16_kernel<4><<<grid, threads, 0, ctx->stream>>>(a);
            } else {
                grid = grid_for(ctx, a.n, threads, 1, 8);
                ht_build_kernel<<<grid, threads, 0, ctx->stream>>>(a);
            }
            PYG_LAUNCHED(ctx);
        }
        unsigned long long* h = (unsigned long long*)ctx->pinned;
        PYG_CUDA(cudaMemcpyAsync(h, flags, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
        PYG_CUDA(cudaStreamSynchronize(ctx->stream));
        if (h[1]) {
            set_error("pyg_hashjoin_build: table full (capacity %llu)", (unsigned long long)cap);
            rc = PYG_ERR_TABLE_FULL;
            break;
        }
        ht->has_dups = h[0] ? 1 : 0;
        ht->entries = (int64_t)h[3];
        ht->nside = (int64_t)h[2];
        if (ht->nside > side_cap) {
            // More keys equal to the empty marker than the side list holds:
            // rebuild once with an exact side list.
            dfree(ctx, ht->slots);
            dfree(ctx, ht->side);
            ht->slots = nullptr;
            ht->side = nullptr;
            side_cap = ht->nside;
            continue;
        }
        ht->entries += ht->nside;  // side entries are kept per tuple
        if (ht->has_dups && mode == PYG_HT_AGGREGATE && a.n > 0) {
            if ((rc = dalloc(ctx, (void**)&ht->counts, cap * sizeof(unsigned long long)))) break;
            PYG_CUDA(cudaMemsetAsync(ht->counts, 0, cap * sizeof(unsigned long long), ctx->stream));
            grid = grid_for(ctx, a.n, threads, 1, 8);
            ht_count_kernel<<<grid, threads, 0, ctx->stream>>>(a, ht->counts);
            PYG_LAUNCHED(ctx);
        }
        rc = PYG_OK;
        break;
    }
    R.release(ctx);
    if (rc) {
        pyg_hashtable_free(ctx, ht);
        return rc;
    }
    *out = ht;
    return PYG_OK;
}

int pyg_hashtable_free(pyg_ctx* ctx, pyg_hashtable* ht)
{
    if (!ht) return PYG_OK;
    int rc = check_ctx(ctx);
    if (rc) return rc;
    dfree(ctx, ht->slots);
    dfree(ctx, ht->side);
    dfree(ctx, ht->counts);
    delete ht;
    return PYG_OK;
}

int pyg_hashtable_stats(pyg_ctx* ctx, const pyg_hashtable* ht, int64_t* entries, int64_t* capacity,
                        int32_t* has_duplicates)
{
    (void)ctx;
    if (!ht) {
        set_error("pyg_hashtable_stats: null table");
        return PYG_ERR_ARG;
    }
    if (entries) *entries = ht->entries;
    if (capacity) *capacity = (int64_t)ht->cap;
    if (has_duplicates) *has_duplicates = ht->has_dups;
    return PYG_OK;
}

int pyg_hashjoin_probe_agg(pyg_ctx* ctx, const pyg_hashtable* ht, const pyg_rel* probe, const int32_t* key_cols,
                           const pyg_proj* proj, int32_t nproj, pyg_join_result* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!ht || !out) {
        set_error("pyg_hashjoin_probe_agg: null table or out");
        return PYG_ERR_ARG;
    }
    if ((rc = check_rel(probe, "probe"))) return rc;
    ProbeArgs a;
    if ((rc = fill_probe_args(ctx, ht, probe, key_cols, proj, nproj, &a))) return rc;
    unsigned long long* acc = ctx->dcounters + 8;
    PYG_CUDA(cudaMemsetAsync(acc, 0, (PYG_MAX_COLS + 1) * sizeof(unsigned long long), ctx->stream));
    int fb = -1, fp = -1;
    bool fast = fast16_layout(ht, a, probe, nproj, &fb, &fp);
    if (fast && !probe->on_device && a.n > 0) {
        // Host probe relation: stream it through two device buffers, the
        // copy of chunk i+1 overlapping the probe of chunk i.
        if ((rc = probe16_stream_host(ctx, ht, (const longlong2*)probe->base, a.n, acc))) return rc;
    } else {
        DevRel S;
        if ((rc = S.stage(ctx, probe))) return rc;
        a.base = (const uint8_t*)S.rel.base;
        if (fast && (uintptr_t)a.base % 16) fast = false;
        if (a.n > 0) {
            if (fast) {
                if ((rc = launch_probe16(ctx, ht, (const longlong2*)a.base, a.n, false, acc))) {
                    S.release(ctx);
                    return rc;
                }
            } else {
                int threads = 256;
                int grid = grid_for(ctx, a.n, threads, 1, 8);
                probe_agg_kernel<<<grid, threads, 0, ctx->stream>>>(a, acc);
                PYG_LAUNCHED(ctx);
            }
        }
        S.release(ctx);
    }
    unsigned long long* h = (unsigned long long*)ctx->pinned;
    PYG_CUDA(cudaMemcpyAsync(h, acc, (PYG_MAX_COLS + 1) * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    fill_result(out, h, a, nproj, fast, fb);
    return PYG_OK;
}

int pyg_hashjoin_probe_materialize(pyg_ctx* ctx, const pyg_hashtable* ht, const pyg_rel* probe,
                                   const int32_t* key_cols, const pyg_proj* proj, int32_t nproj, void* out,
                                   int64_t out_capacity, int64_t* out_count)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!ht || !out_count || (out_capacity > 0 && !out)) {
        set_error("pyg_hashjoin_probe_materialize: null argument");
        return PYG_ERR_ARG;
    }
    if (ht->mode != PYG_HT_MATERIALIZE) {
        set_error("pyg_hashjoin_probe_materialize: table was built in AGGREGATE mode");
        return PYG_ERR_ARG;
    }
    if ((rc = check_rel(probe, "probe"))) return rc;
    ProbeArgs a;
    if ((rc = fill_probe_args(ctx, ht, probe, key_cols, proj, nproj, &a))) return rc;
    if (nproj < 1) {
        set_error("pyg_hashjoin_probe_materialize: empty projection");
        return PYG_ERR_ARG;
    }
    DevRel S;
    if ((rc = S.stage(ctx, probe))) return rc;
    a.base = (const uint8_t*)S.rel.base;
    unsigned long long* cursor = ctx->dcounters + 24;
    PYG_CUDA(cudaMemsetAsync(cursor, 0, sizeof(unsigned long long), ctx->stream));
    if (a.n > 0) {
        int threads = 256;
        int grid = grid_for(ctx, a.n, threads, 1, 8);
        probe_mat_kernel<<<grid, threads, 0, ctx->stream>>>(a, (uint8_t*)out, out_capacity, cursor);
        PYG_LAUNCHED(ctx);
    }
    unsigned long long* h = (unsigned long long*)ctx->pinned;
    PYG_CUDA(cudaMemcpyAsync(h, cursor, sizeof(unsigned long long), cudaMemcpyDeviceToHost, ctx->stream));
    S.release(ctx);
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    *out_count = (int64_t)h[0];
    if (*out_count > out_capacity) {
        set_error("pyg_hashjoin_probe_materialize: %lld pairs exceed capacity %lld", (long long)*out_count,
                  (long long)out_capacity);
        return PYG_ERR_CAPACITY;
    }
    return PYG_OK;
}

int pyg_hashjoin_agg(pyg_ctx* ctx, const pyg_rel* build, const int32_t* build_keys, const pyg_rel* probe,
                     const int32_t* probe_keys, int32_t nkeys, const pyg_proj* proj, int32_t nproj,
                     const pyg_join_opts* opts, pyg_join_result* out, pyg_join_stats* stats)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || (nproj > 0 && !proj) || nproj < 0 || nproj > PYG_MAX_COLS) {
        set_error("pyg_hashjoin_agg: bad arguments");
        return PYG_ERR_ARG;
    }
    if ((rc = check_rel(build, "build")) || (rc = check_rel(probe, "probe"))) return rc;
    int algorithm = opts ? opts->algorithm : PYG_JOIN_AUTO;
    float lf = (opts && opts->load_factor > 0) ? opts->load_factor : 0.5f;
    if (stats) memset(stats, 0, sizeof(*stats));
    // Build columns referenced by the projection.
    int32_t pay[PYG_MAX_COLS];
    int npay = 0;
    for (int p = 0; p < nproj; ++p) {
        if (proj[p].side) continue;
        bool seen = false;
        for (int c = 0; c < npay; ++c) seen |= pay[c] == proj[p].col;
        if (!seen) pay[npay++] = proj[p].col;
    }
    // The radix path covers 16-byte (int64 key @0, int64 payload @8)
    // device relations with a projection over {B$1, P$1}.
    auto is16 = [](const pyg_rel* r, const int32_t* k) {
        return r->on_device && r->tuple_bytes == 16 && r->ncols == 2 && k && k[0] == 0 && r->col_offset[0] == 0 &&
               r->col_type[0] == PYG_INT64 && r->col_offset[1] == 8 && r->col_type[1] == PYG_INT64 &&
               (uintptr_t)r->base % 16 == 0;
    };
    bool eligible = nkeys == 1 && is16(build, build_keys) && is16(probe, probe_keys) && nproj <= 2 && npay <= 1;
    for (int p = 0; eligible && p < nproj; ++p) eligible = proj[p].col == 1;
    if (eligible && nproj == 2) eligible = proj[0].side != proj[1].side;
    // AUTO: the direct join while its table (16 bytes per slot at load
    // factor lf) fits well inside the 126 MB L2, the radix join beyond.
    const double table_bytes = 16.0 * (double)build->ntuples / (double)lf;
    bool radix = eligible && (algorithm == PYG_JOIN_RADIX ||
                              (algorithm == PYG_JOIN_AUTO && table_bytes > 64.0 * 1024 * 1024 &&
                               probe->ntuples >= ((int64_t)1 << 22)));
    PhaseTimer tm;
    if (!radix && eligible) {
        // 16-byte device relations: the one-shot direct join (falls back
        // to the general path below on repeated build keys).
        tm.start(ctx, stats != nullptr);
        unsigned long long r3[3];
        bool fallback = false;
        if ((rc = direct_join16(ctx, (const longlong2*)build->base, build->ntuples, (const longlong2*)probe->base,
                                probe->ntuples, lf, r3, &fallback, &tm)))
            return rc;
        if (!fallback) {
            memset(out, 0, sizeof(*out));
            out->count = (int64_t)r3[0];
            for (int p = 0; p < nproj; ++p) out->sums[p] = (int64_t)(proj[p].side ? r3[2] : r3[1]);
            if (stats) {
                tm.finish(stats);
                stats->algorithm = PYG_JOIN_DIRECT;
            }
            return PYG_OK;
        }
        if (stats) tm.finish(stats);
        tm = PhaseTimer();
    }
    if (!radix) {
        tm.start(ctx, stats != nullptr);
        pyg_hashtable* ht = nullptr;
        if ((rc = pyg_hashjoin_build(ctx, build, build_keys, nkeys, pay, npay, PYG_HT_AGGREGATE, lf, &ht))) return rc;
        tm.mark(ctx, 2);
        tm.mark(ctx, 3);
        rc = pyg_hashjoin_probe_agg(ctx, ht, probe, probe_keys, proj, nproj, out);
        tm.mark(ctx, 4);
        pyg_hashtable_free(ctx, ht);
        if (stats) {
            tm.finish(stats);
            stats->algorithm = PYG_JOIN_DIRECT;
        }
        return rc;
    }
    // Radix path: exact two-level hash partitioning, then a join with one
    // shared-memory table per CTA (radixjoin.cu).
    unsigned long long r3[3];
    if ((rc = radix_join16(ctx, build->base, build->ntuples, probe->base, probe->ntuples, opts ? opts->radix_bits : 0,
                           r3, stats)))
        return rc;
    memset(out, 0, sizeof(*out));
    out->count = (int64_t)r3[0];
    for (int p = 0; p < nproj; ++p) out->sums[p] = (int64_t)(proj[p].side ? r3[2] : r3[1]);
    return PYG_OK;
}

}  // extern "C"
