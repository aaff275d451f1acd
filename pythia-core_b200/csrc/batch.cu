// Batched PK-FK join + sum fragments: one persistent kernel over a device
// work queue for the small and medium fragments, captured in a CUDA graph,
// then the large fragments as their own partitioned joins; the plain
// sequential baseline; and the autotuner that picks the persistent kernel's
// launch shape, the table load factor, the work-item grain and the size
// from which a fragment runs on its own.
#include <string.h>

#include <algorithm>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/pyg_batch.h"
#include "pyg_internal.cuh"
#include "radixjoin.cuh"

namespace pyg {

// A fragment's table: cap 16-byte slots {key, payload sum} (one 128-bit CAS
// stores a fresh key with its payload) and cap 32-bit counters of extra
// copies of a key, touched only by repeated build keys.  At the default
// load factor the largest fragment's slots stay inside L2.
struct FragDesc {
    const longlong2* build;
    int64_t nb;
    const longlong2* probe;
    int64_t np;
    ulonglong2* table;
    unsigned* extra;
    uint64_t cap;
    int32_t n_init, n_build, n_probe, pad;
};

struct WorkItem {
    int32_t frag;
    int32_t kind;  // 0 clear table slots, 1 build tuples, 2 probe tuples
    int64_t begin, end;
};

// Per-run state, zeroed by one memset node of the graph.
struct BatchState {
    unsigned long long next;       // work queue head
    unsigned long long t0;         // batch start (globaltimer, ns)
    unsigned int error;            // a bounded wait gave up
    unsigned int pad;
};

constexpr int RES_WORDS = 6;  // count, sum, then empty-marker key stats: build count/sum, probe count/sum
constexpr long long kWaitLimit = 1LL << 22;  // x ~256 ns sleeps, about one second
// Build tuples from which a fragment runs as its own join by default.  On
// a mix of 256 fragments with builds of 2^12..2^22 tuples, sending builds of
// 2^16 and more to their own calls measured fastest (58.4 ms against 61.0
// ms at 2^14 and 61.4-80.7 ms at 2^20 and above).
constexpr int64_t kLargeBuild = (int64_t)1 << 16;

struct BatchDev {
    const FragDesc* frags;
    const WorkItem* items;
    int64_t nitems;
    BatchState* st;
    unsigned int* init_done;
    unsigned int* build_done;
    unsigned int* probe_done;
    unsigned long long* res;     // RES_WORDS per fragment
    unsigned long long* t_done;  // per fragment completion time
    unsigned int* dup;           // per fragment: a build key repeated
};

constexpr int BATCH_U = 4;  // probe / build tuples in flight per thread

__device__ __forceinline__ unsigned __int128 bslot(uint64_t key, uint64_t pay)
{
    return ((unsigned __int128)pay << 64) | (unsigned __int128)key;
}

__device__ __forceinline__ unsigned long long gtimer()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Thread 0 waits until *ctr reaches target or the wait limit / an earlier
// timeout ends it.  Returns false on timeout.
__device__ bool wait_count(const unsigned int* ctr, unsigned int target, BatchState* st)
{
    volatile const unsigned int* c = ctr;
    volatile unsigned int* err = &st->error;
    for (long long i = 0; i < kWaitLimit; ++i) {
        if (*c >= target) return true;
        if (*err) return false;
        __nanosleep(256);
    }
    atomicOr(&st->error, 1u);
    return false;
}

__global__ void __launch_bounds__(1024) batch_kernel(BatchDev d)
{
    __shared__ long long item;
    __shared__ int ok, dupf;
    __shared__ unsigned long long red[RES_WORDS];
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicCAS(&d.st->t0, 0ULL, gtimer());
    const unsigned __int128 empty = bslot(kEmptyKey, 0);
    for (;;) {
        if (threadIdx.x == 0) item = (long long)atomicAdd(&d.st->next, 1ULL);
        __syncthreads();
        if (item >= d.nitems) break;
        const WorkItem w = d.items[item];
        const FragDesc f = d.frags[w.frag];
        if (threadIdx.x < RES_WORDS) red[threadIdx.x] = 0;
        if (threadIdx.x == 0) {
            ok = 1;
            if (w.kind == 1) ok = wait_count(&d.init_done[w.frag], (unsigned)f.n_init, d.st);
            if (w.kind == 2) ok = wait_count(&d.build_done[w.frag], (unsigned)f.n_build, d.st);
            __threadfence();
            dupf = w.kind == 2 ? (int)*(volatile unsigned*)&d.dup[w.frag] : 0;
        }
        __syncthreads();
        const int64_t stride = blockDim.x;
        if (w.kind == 0) {
            for (int64_t s = w.begin + threadIdx.x; s < w.end; s += stride) {
                f.table[s] = make_ulonglong2(kEmptyKey, 0);
                f.extra[s] = 0;
            }
        } else if (w.kind == 1 && ok) {
            // BATCH_U inserts in flight per thread: loads, the first 128-bit
            // CAS of each, then the chains.  A repeated key adds its payload
            // and one to the slot's extra-copies counter.
            uint64_t ec = 0, es = 0;
            bool dup = false;
            for (int64_t i0 = w.begin + threadIdx.x; i0 < w.end; i0 += stride * BATCH_U) {
                longlong2 t[BATCH_U];
                uint64_t s[BATCH_U];
                unsigned long long pv[BATCH_U];
#pragma unroll
                for (int u = 0; u < BATCH_U; ++u) {
                    const int64_t i = i0 + u * stride;
                    t[u] = i < w.end ? __ldcs(&f.build[i]) : make_longlong2((long long)kEmptyKey, 0);
                }
#pragma unroll
                for (int u = 0; u < BATCH_U; ++u) {
                    const uint64_t k = (uint64_t)t[u].x;
                    s[u] = reduce_range(mix64(k), f.cap);
                    pv[u] = k == kEmptyKey ? ~0ULL
                                           : (unsigned long long)atomicCAS((unsigned __int128*)&f.table[s[u]], empty,
                                                                           bslot(k, (uint64_t)t[u].y));
                }
#pragma unroll
                for (int u = 0; u < BATCH_U; ++u) {
                    if (i0 + u * stride >= w.end) continue;
                    const uint64_t k = (uint64_t)t[u].x;
                    if (k == kEmptyKey) {
                        ++ec;
                        es += (uint64_t)t[u].y;
                        continue;
                    }
                    uint64_t ss = s[u];
                    unsigned long long p = pv[u];
                    // cap > build tuples, so the chain ends at a free slot or the key.
                    for (uint64_t steps = 1; p != kEmptyKey && p != k && steps < f.cap; ++steps) {
                        ss = (ss + 1 == f.cap) ? 0 : ss + 1;
                        p = (unsigned long long)atomicCAS((unsigned __int128*)&f.table[ss], empty,
                                                          bslot(k, (uint64_t)t[u].y));
                    }
                    if (p == k) {
                        dup = true;
                        atomicAdd(&f.table[ss].y, (unsigned long long)t[u].y);
                        atomicAdd(&f.extra[ss], 1u);
                    }
                }
            }
            if (ec) {
                atomicAdd(&red[2], (unsigned long long)ec);
                atomicAdd(&red[3], (unsigned long long)es);
            }
            if (__any_sync(0xffffffffu, dup) && (threadIdx.x & 31) == 0) atomicOr(&d.dup[w.frag], 1u);
        } else if (w.kind == 2 && ok) {
            // BATCH_U independent lookups in flight per thread; the table
            // of the fragment being probed is L2-resident.
            uint64_t cnt = 0, sum = 0, ec = 0, es = 0;
            const bool dup = dupf != 0;
            for (int64_t i0 = w.begin + threadIdx.x; i0 < w.end; i0 += stride * BATCH_U) {
                longlong2 t[BATCH_U];
                uint64_t s[BATCH_U];
                ulonglong2 e[BATCH_U];
#pragma unroll
                for (int u = 0; u < BATCH_U; ++u) {
                    const int64_t i = i0 + u * stride;
                    t[u] = i < w.end ? __ldcs(&f.probe[i]) : make_longlong2((long long)kEmptyKey, 0);
                }
#pragma unroll
                for (int u = 0; u < BATCH_U; ++u) {
                    s[u] = reduce_range(mix64((uint64_t)t[u].x), f.cap);
                    e[u] = f.table[s[u]];
                }
#pragma unroll
                for (int u = 0; u < BATCH_U; ++u) {
                    if (i0 + u * stride >= w.end) continue;
                    const uint64_t k = (uint64_t)t[u].x;
                    if (k == kEmptyKey) {
                        ++ec;
                        es += (uint64_t)t[u].y;
                        continue;
                    }
                    uint64_t ss = s[u];
                    ulonglong2 ee = e[u];
                    for (uint64_t steps = 1; ee.x != k && ee.x != kEmptyKey && steps < f.cap; ++steps) {
                        ss = (ss + 1 == f.cap) ? 0 : ss + 1;
                        ee = f.table[ss];
                    }
                    if (ee.x == k) {
                        const uint64_t c = dup ? 1ULL + f.extra[ss] : 1ULL;
                        cnt += c;
                        sum += ee.y + c * (uint64_t)t[u].y;
                    }
                }
            }
            cnt = warp_sum_u64(cnt);
            sum = warp_sum_u64(sum);
            ec = warp_sum_u64(ec);
            es = warp_sum_u64(es);
            if ((threadIdx.x & 31) == 0) {
                if (cnt) atomicAdd(&red[0], (unsigned long long)cnt);
                if (sum) atomicAdd(&red[1], (unsigned long long)sum);
                if (ec) atomicAdd(&red[4], (unsigned long long)ec);
                if (es) atomicAdd(&red[5], (unsigned long long)es);
            }
        }
        __syncthreads();
        if (threadIdx.x < RES_WORDS && red[threadIdx.x])
            atomicAdd(&d.res[(int64_t)w.frag * RES_WORDS + threadIdx.x], red[threadIdx.x]);
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (w.kind == 0) {
                atomicAdd(&d.init_done[w.frag], 1u);
            } else if (w.kind == 1) {
                unsigned done = atomicAdd(&d.build_done[w.frag], 1u) + 1;
                if (f.n_probe == 0 && done == (unsigned)f.n_build) d.t_done[w.frag] = gtimer();
            } else {
                unsigned done = atomicAdd(&d.probe_done[w.frag], 1u) + 1;
                if (done == (unsigned)f.n_probe) d.t_done[w.frag] = gtimer();
            }
        }
        __syncthreads();
    }
}

}  // namespace pyg

struct pyg_batch {
    int32_t n = 0;
    pyg_tuning tuning;
    std::vector<void*> bufs;
    pyg::BatchDev dev;
    void* state = nullptr;       // BatchState + counters + results (one memset)
    size_t state_bytes = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<int32_t> order;  // fragments with no work item (empty) still report results
    std::vector<char> empty_frag;
    // Fragments run after the graph as their own joins: the direct join,
    // enqueued without waiting (its counters in 16 device words each of
    // large_words), or a partitioned join through pyg_hashjoin_agg.
    std::vector<int32_t> large;
    std::vector<pyg_fragment> large_frag;
    unsigned long long* large_words = nullptr;
};

namespace pyg {

static std::mutex g_tune_mu;
static std::map<std::string, pyg_tuning> g_tune_cache;

static pyg_tuning default_tuning()
{
    pyg_tuning t;
    t.block_threads = 512;
    t.blocks_per_sm = 2;
    t.load_factor = 0.5f;
    t.chunk_tuples = 4096;
    t.large_build = 0;
    return t;
}

static std::string signature(const pyg_fragment* fr, int n)
{
    double b = 0, p = 0;
    for (int i = 0; i < n; ++i) {
        b += (double)fr[i].nbuild;
        p += (double)fr[i].nprobe;
    }
    std::ostringstream os;
    os << "n" << n << "_b" << (int)(b > 0 ? log2(b) : 0) << "_p" << (int)(p > 0 ? log2(p) : 0);
    return os.str();
}

// The automatic algorithm's choice for a fragment (pyg_hashjoin_agg): the
// direct join while its table (16-byte slots at load factor 0.5) fits well
// inside L2 or the probe side is small, else the partitioned join.
static bool fragment_direct(const pyg_fragment& f)
{
    const double table_bytes = 16.0 * (double)f.nbuild / 0.5;
    return !(table_bytes > 64.0 * 1024 * 1024 && f.nprobe >= ((int64_t)1 << 22)) && (uintptr_t)f.build % 16 == 0 &&
           (uintptr_t)f.probe % 16 == 0;
}

// One fragment through pyg_hashjoin_agg with the automatic algorithm (the
// best single call): count and sum(build payload + probe value).
static int join_fragment(pyg_ctx* ctx, const pyg_fragment& f, int64_t* count, int64_t* sum)
{
    pyg_rel R, S;
    memset(&R, 0, sizeof(R));
    R.base = f.build;
    R.ntuples = f.nbuild;
    R.tuple_bytes = 16;
    R.ncols = 2;
    R.col_offset[1] = 8;
    R.col_type[0] = R.col_type[1] = PYG_INT64;
    R.on_device = 1;
    S = R;
    S.base = f.probe;
    S.ntuples = f.nprobe;
    int32_t k = 0;
    pyg_proj proj[2] = {{0, 1}, {1, 1}};
    pyg_join_opts o = {PYG_JOIN_AUTO, 0, 0.5f, 0};
    pyg_join_result r;
    int rc = pyg_hashjoin_agg(ctx, &R, &k, &S, &k, 1, proj, 2, &o, &r, nullptr);
    if (!rc) {
        *count = r.count;
        *sum = (int64_t)((uint64_t)r.sums[0] + (uint64_t)r.sums[1]);
    }
    return rc;
}

static int batch_alloc(pyg_ctx* ctx, pyg_batch* b, void** p, size_t bytes)
{
    int rc = dalloc(ctx, p, bytes);
    if (!rc) b->bufs.push_back(*p);
    return rc;
}

}  // namespace pyg

using namespace pyg;

extern "C" {

int pyg_batch_free(pyg_ctx* ctx, pyg_batch* b)
{
    if (!b) return PYG_OK;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    if (ctx) {
        cudaSetDevice(ctx->device);
        for (void* p : b->bufs) dfree(ctx, p);
        cudaStreamSynchronize(ctx->stream);
    }
    delete b;
    return PYG_OK;
}

int pyg_batch_create(pyg_ctx* ctx, const pyg_fragment* frags, int32_t n, const pyg_tuning* tuning, pyg_batch** out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!out || n < 1 || !frags) {
        set_error("pyg_batch_create: need >= 1 fragment");
        return PYG_ERR_ARG;
    }
    *out = nullptr;
    pyg_tuning t = default_tuning();
    if (tuning) {
        t = *tuning;
    } else {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(signature(frags, n));
        if (it != g_tune_cache.end()) t = it->second;
    }
    if (t.block_threads < 64 || t.block_threads > 1024 || (t.block_threads & 31) || t.blocks_per_sm < 1 ||
        t.blocks_per_sm > 16 || !(t.load_factor > 0 && t.load_factor <= 0.9f) || t.chunk_tuples < 256 ||
        t.large_build < 0) {
        set_error("pyg_batch_create: bad tuning");
        return PYG_ERR_ARG;
    }
    for (int i = 0; i < n; ++i)
        if (frags[i].nbuild < 0 || frags[i].nprobe < 0 || (frags[i].nbuild && !frags[i].build) ||
            (frags[i].nprobe && !frags[i].probe) || ((uintptr_t)frags[i].build % 16) || ((uintptr_t)frags[i].probe % 16)) {
            set_error("pyg_batch_create: fragment %d has a bad relation", i);
            return PYG_ERR_ARG;
        }
    pyg_batch* b = new pyg_batch();
    b->n = n;
    b->tuning = t;
    const int64_t large_build = t.large_build > 0 ? t.large_build : kLargeBuild;
    std::vector<char> is_large(n, 0);
    for (int i = 0; i < n; ++i)
        if (frags[i].nbuild >= large_build) {
            is_large[i] = 1;
            b->large.push_back(i);
            b->large_frag.push_back(frags[i]);
        }
    if (!b->large.empty()) {
        int rc = batch_alloc(ctx, b, (void**)&b->large_words, b->large.size() * 16 * sizeof(unsigned long long));
        if (rc) {
            pyg_batch_free(ctx, b);
            return rc;
        }
    }
    // Tables: one arena of 16-byte slots and one of extra-copy counters,
    // per-fragment capacity nbuild / load factor (queued fragments only).
    std::vector<FragDesc> fd(n);
    uint64_t total_slots = 0;
    for (int i = 0; i < n; ++i) {
        uint64_t cap = is_large[i] ? 0 : (uint64_t)((double)frags[i].nbuild / t.load_factor) + 64;
        fd[i].cap = cap;
        total_slots += cap;
    }
    ulonglong2* arena;
    unsigned* extra;
    if ((rc = batch_alloc(ctx, b, (void**)&arena, std::max<uint64_t>(total_slots, 1) * sizeof(ulonglong2))) ||
        (rc = batch_alloc(ctx, b, (void**)&extra, std::max<uint64_t>(total_slots, 1) * sizeof(unsigned)))) {
        pyg_batch_free(ctx, b);
        return rc;
    }
    // Work list: fragments in ascending size (shortest first), each as
    // clear, build, then probe items.
    std::vector<int32_t> order(n);
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
        return frags[a].nbuild + frags[a].nprobe < frags[c].nbuild + frags[c].nprobe;
    });
    std::vector<WorkItem> items;
    uint64_t off = 0;
    std::vector<uint64_t> toff(n);
    for (int i = 0; i < n; ++i) {
        toff[i] = off;
        off += fd[i].cap;
    }
    const int64_t grain = t.chunk_tuples;
    for (int i : order) {
        FragDesc& f = fd[i];
        f.build = (const longlong2*)frags[i].build;
        f.nb = is_large[i] ? 0 : frags[i].nbuild;
        f.probe = (const longlong2*)frags[i].probe;
        f.np = is_large[i] ? 0 : frags[i].nprobe;
        f.table = arena + toff[i];
        f.extra = extra + toff[i];
        f.n_init = f.n_build = f.n_probe = 0;
        for (uint64_t s = 0; s < f.cap; s += (uint64_t)grain * 2, ++f.n_init)
            items.push_back({i, 0, (int64_t)s, (int64_t)std::min<uint64_t>(f.cap, s + grain * 2)});
        for (int64_t s = 0; s < f.nb; s += grain, ++f.n_build)
            items.push_back({i, 1, s, std::min<int64_t>(f.nb, s + grain)});
        for (int64_t s = 0; s < f.np; s += grain, ++f.n_probe)
            items.push_back({i, 2, s, std::min<int64_t>(f.np, s + grain)});
    }
    b->empty_frag.assign(n, 0);
    for (int i = 0; i < n; ++i) b->empty_frag[i] = (fd[i].n_build == 0 && fd[i].n_probe == 0);
    FragDesc* dfd;
    WorkItem* ditems;
    b->state_bytes = sizeof(BatchState) + (size_t)n * (4 * sizeof(unsigned) + (RES_WORDS + 1) * 8) + 64;
    if ((rc = batch_alloc(ctx, b, (void**)&dfd, n * sizeof(FragDesc))) ||
        (rc = batch_alloc(ctx, b, (void**)&ditems, std::max<size_t>(items.size(), 1) * sizeof(WorkItem))) ||
        (rc = batch_alloc(ctx, b, &b->state, b->state_bytes))) {
        pyg_batch_free(ctx, b);
        return rc;
    }
    PYG_CUDA(cudaMemcpyAsync(dfd, fd.data(), n * sizeof(FragDesc), cudaMemcpyHostToDevice, ctx->stream));
    PYG_CUDA(cudaMemcpyAsync(ditems, items.data(), items.size() * sizeof(WorkItem), cudaMemcpyHostToDevice,
                             ctx->stream));
    PYG_CUDA(cudaStreamSynchronize(ctx->stream));
    char* sp = (char*)b->state;
    b->dev.frags = dfd;
    b->dev.items = ditems;
    b->dev.nitems = (int64_t)items.size();
    b->dev.st = (BatchState*)sp;
    sp += sizeof(BatchState);
    b->dev.res = (unsigned long long*)sp;
    sp += (size_t)n * RES_WORDS * 8;
    b->dev.t_done = (unsigned long long*)sp;
    sp += (size_t)n * 8;
    b->dev.init_done = (unsigned*)sp;
    b->dev.build_done = b->dev.init_done + n;
    b->dev.probe_done = b->dev.build_done + n;
    b->dev.dup = b->dev.probe_done + n;

    // Capture: reset the state, run the persistent kernel.
    int grid = ctx->sm_count * t.blocks_per_sm;
    cudaStream_t s = ctx->stream;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
        cudaMemsetAsync(b->state, 0, b->state_bytes, s);
        batch_kernel<<<grid, t.block_threads, 0, s>>>(b->dev);
        e = cudaStreamEndCapture(s, &b->graph);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    if (e != cudaSuccess) {
        rc = cuda_status(e, "batch graph capture");
        pyg_batch_free(ctx, b);
        return rc;
    }
    *out = b;
    return PYG_OK;
}

int pyg_batch_run(pyg_ctx* ctx, pyg_batch* b, int64_t* counts, int64_t* sums, double* latency_ms)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!b) {
        set_error("pyg_batch_run: null batch");
        return PYG_ERR_ARG;
    }
    // Queued fragments: the graph.  Large fragments: their own partitioned
    // joins, after it on the same stream; their latency is taken from
    // events against one recorded just before the graph.
    const size_t nl = b->large.size();
    std::vector<cudaEvent_t> ev(nl ? nl + 1 : 0);
    for (auto& e : ev) PYG_CUDA(cudaEventCreate(&e));
    if (nl) cudaEventRecord(ev[0], ctx->stream);
    PYG_CUDA(cudaGraphLaunch(b->exec, ctx->stream));
    ctx->launches += 1;
    std::vector<unsigned char> st(b->state_bytes);
    PYG_CUDA(cudaMemcpyAsync(st.data(), b->state, b->state_bytes, cudaMemcpyDeviceToHost, ctx->stream));
    std::vector<int64_t> lc(nl), ls(nl);
    // Direct joins first, one after another on the stream with no wait
    // between them; the partitioned joins after them.
    std::vector<char> direct(nl, 0);
    for (size_t j = 0; j < nl; ++j) direct[j] = fragment_direct(b->large_frag[j]) ? 1 : 0;
    for (int pass = 0; pass < 2 && !rc; ++pass)
        for (size_t j = 0; j < nl && !rc; ++j) {
            if (direct[j] != (pass == 0)) continue;
            const pyg_fragment& f = b->large_frag[j];
            if (direct[j]) rc = direct_join16_enqueue(ctx, f.build, f.nbuild, f.probe, f.nprobe, 0.5f,
                                                      b->large_words + 16 * j);
            else rc = join_fragment(ctx, f, &lc[j], &ls[j]);
            cudaEventRecord(ev[j + 1], ctx->stream);
        }
    std::vector<unsigned long long> lw(nl * 16);
    if (nl && !rc)
        PYG_CUDA(cudaMemcpyAsync(lw.data(), b->large_words, lw.size() * 8, cudaMemcpyDeviceToHost, ctx->stream));
    cudaError_t e = cudaStreamSynchronize(ctx->stream);
    // A direct join whose build repeated a key stood down: the general
    // path answers for it now.
    for (size_t j = 0; j < nl && !rc && e == cudaSuccess; ++j) {
        if (!direct[j]) continue;
        unsigned long long r3[3];
        if (direct_join16_result(lw.data() + 16 * j, b->large_frag[j].nbuild, r3)) {
            lc[j] = (int64_t)r3[0];
            ls[j] = (int64_t)(r3[1] + r3[2]);
        } else {
            rc = join_fragment(ctx, b->large_frag[j], &lc[j], &ls[j]);
        }
    }
    std::vector<float> lat_large(nl, 0.f);
    for (size_t j = 0; j < nl && !rc && e == cudaSuccess; ++j) cudaEventElapsedTime(&lat_large[j], ev[0], ev[j + 1]);
    for (auto& x : ev) cudaEventDestroy(x);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_status(e, "pyg_batch_run");
    const BatchState* bs = (const BatchState*)st.data();
    if (bs->error) {
        set_error("pyg_batch_run: a bounded wait for a fragment's build gave up");
        return PYG_ERR_TIMEOUT;
    }
    const int n = b->n;
    const unsigned long long* res = (const unsigned long long*)(st.data() + sizeof(BatchState));
    const unsigned long long* td = res + (size_t)n * RES_WORDS;
    for (int i = 0; i < n; ++i) {
        const unsigned long long* r = res + (size_t)i * RES_WORDS;
        // Keys equal to the empty marker join among themselves.
        uint64_t cnt = r[0] + r[2] * r[4];
        uint64_t sum = r[1] + r[3] * r[4] + r[2] * r[5];
        if (counts) counts[i] = (int64_t)cnt;
        if (sums) sums[i] = (int64_t)sum;
        if (latency_ms) latency_ms[i] = td[i] > bs->t0 ? (double)(td[i] - bs->t0) / 1e6 : 0.0;
    }
    for (size_t j = 0; j < nl; ++j) {
        const int i = b->large[j];
        if (counts) counts[i] = lc[j];
        if (sums) sums[i] = ls[j];
        if (latency_ms) latency_ms[i] = lat_large[j];
    }
    return PYG_OK;
}

int pyg_batch_run_plain(pyg_ctx* ctx, const pyg_fragment* frags, int32_t n, int64_t* counts, int64_t* sums,
                        double* latency_ms)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!frags || n < 1) {
        set_error("pyg_batch_run_plain: need >= 1 fragment");
        return PYG_ERR_ARG;
    }
    std::vector<cudaEvent_t> ev(n + 1);
    for (auto& e : ev) cudaEventCreate(&e);
    cudaEventRecord(ev[0], ctx->stream);
    for (int i = 0; i < n && !rc; ++i) {
        int64_t c = 0, sm = 0;
        rc = join_fragment(ctx, frags[i], &c, &sm);
        cudaEventRecord(ev[i + 1], ctx->stream);
        if (!rc) {
            if (counts) counts[i] = c;
            if (sums) sums[i] = sm;
        }
    }
    cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < n && latency_ms; ++i) {
        float ms = 0;
        cudaEventElapsedTime(&ms, ev[0], ev[i + 1]);
        latency_ms[i] = ms;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    return rc;
}

int pyg_batch_inject_stall(pyg_ctx* ctx, pyg_batch* b, int32_t frag)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!b || frag < 0 || frag >= b->n ||
        std::find(b->large.begin(), b->large.end(), frag) != b->large.end()) {
        set_error("pyg_batch_inject_stall: not a queued fragment");
        return PYG_ERR_ARG;
    }
    // Raise the fragment's expected build-item count by one: its probe
    // items then wait for a build item that never exists.
    FragDesc f;
    PYG_CUDA(cudaMemcpy(&f, b->dev.frags + frag, sizeof(f), cudaMemcpyDeviceToHost));
    f.n_build += 1;
    PYG_CUDA(cudaMemcpy((void*)(b->dev.frags + frag), &f, sizeof(f), cudaMemcpyHostToDevice));
    return PYG_OK;
}

int pyg_autotune(pyg_ctx* ctx, const pyg_fragment* frags, int32_t n, const char* cache_path, pyg_tuning* out)
{
    int rc = check_ctx(ctx);
    if (rc) return rc;
    if (!frags || n < 1 || !out) {
        set_error("pyg_autotune: bad arguments");
        return PYG_ERR_ARG;
    }
    const std::string sig = signature(frags, n);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        auto it = g_tune_cache.find(sig);
        if (it != g_tune_cache.end()) {
            *out = it->second;
            return PYG_OK;
        }
    }
    if (cache_path) {
        std::ifstream in(cache_path);
        std::string s;
        pyg_tuning t;
        while (in >> s >> t.block_threads >> t.blocks_per_sm >> t.load_factor >> t.chunk_tuples >> t.large_build) {
            if (s == sig) {
                std::lock_guard<std::mutex> g(g_tune_mu);
                g_tune_cache[sig] = t;
                *out = t;
                return PYG_OK;
            }
        }
    }
    // First the size from which fragments run as their own joins, timed on
    // whole runs with the default kernel shape; then the persistent
    // kernel's candidate grid (block shape x occupancy x load factor x
    // grain) for the fragments that stay queued, timed on the graph alone.
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    auto time_tuning = [&](const pyg_tuning& t, bool whole, int reps) -> float {
        pyg_batch* b = nullptr;
        if (pyg_batch_create(ctx, frags, n, &t, &b)) return 1e30f;
        float ms = 1e30f;
        bool good = pyg_batch_run(ctx, b, nullptr, nullptr, nullptr) == PYG_OK;
        for (int rep = 0; rep < reps && good; ++rep) {
            cudaEventRecord(e0, ctx->stream);
            if (whole) good = pyg_batch_run(ctx, b, nullptr, nullptr, nullptr) == PYG_OK;
            else cudaGraphLaunch(b->exec, ctx->stream);
            cudaEventRecord(e1, ctx->stream);
            cudaEventSynchronize(e1);
            float x = 0;
            cudaEventElapsedTime(&x, e0, e1);
            ms = std::min(ms, x);
        }
        pyg_batch_free(ctx, b);
        return good ? ms : 1e30f;
    };
    pyg_tuning best_t = default_tuning();
    float best = 1e30f;
    {
        const int32_t larges[] = {1 << 14, 1 << 16, 1 << 18, 1 << 20};
        const pyg_tuning base = best_t;
        for (int32_t lb : larges) {
            pyg_tuning t = base;
            t.large_build = lb;
            const float ms = time_tuning(t, true, 2);
            if (ms < best) {
                best = ms;
                best_t = t;
            }
        }
    }
    const int bts[] = {256, 512, 1024};
    const int bps[] = {1, 2, 4};
    const float lfs[] = {0.5f, 0.7f};
    const int chunks[] = {4096, 16384, 65536};
    const int32_t lb = best_t.large_build;
    best = 1e30f;
    for (int bt : bts)
        for (int bp : bps) {
            if (bt * bp > 2048) continue;
            for (float lf : lfs)
                for (int ch : chunks) {
                    const pyg_tuning t = {bt, bp, lf, ch, lb};
                    const float ms = time_tuning(t, false, 3);
                    if (ms < best) {
                        best = ms;
                        best_t = t;
                    }
                }
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> g(g_tune_mu);
        g_tune_cache[sig] = best_t;
    }
    if (cache_path) {
        std::ofstream o(cache_path, std::ios::app);
        o << sig << " " << best_t.block_threads << " " << best_t.blocks_per_sm << " " << best_t.load_factor << " "
          << best_t.chunk_tuples << " " << best_t.large_build << "\n";
    }
    *out = best_t;
    return PYG_OK;
}

}  // extern "C"
