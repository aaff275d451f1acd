/*
 * pyg_batch.h - batched query fragments of the B200 engine (libpyg.so).
 *
 * Replaces drivers/executemultiplequery.cpp:134-282, which forks one
 * process per plan fragment (at most 32) and runs each through its own
 * thread pool.  Here many PK-FK hash join + sum fragments of uneven size
 * run as one persistent kernel over a shared device work queue: per
 * fragment, table-clear items, then build items, then probe items, queued
 * shortest fragment first.  A probe item waits (with a bounded spin that
 * reports PYG_ERR_TIMEOUT instead of hanging) only for build items of its
 * own fragment that other CTAs already dequeued.  The queue reset and the
 * kernel are captured once in a CUDA graph and replayed per run.
 *
 * Fragments whose build side has at least `large_build` tuples are not
 * queued: their tables would not stay in L2 beside the others', and their
 * work dwarfs a call's fixed cost, so after the graph they run one by one
 * with the algorithm pyg_hashjoin_agg would pick.  Those that take the
 * direct join are enqueued back to back with no host synchronisation
 * between them (their counters stay on the device until the run's single
 * synchronisation; a build side with a repeated key is answered by the
 * general path after it); the partitioned joins follow.  The persistent
 * kernel takes the many small and medium fragments, whose separate calls
 * would be dominated by launches and host synchronisations.
 */
#ifndef PYG_BATCH_H
#define PYG_BATCH_H

#include "pyg.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pyg_batch pyg_batch;

/* One fragment: build (key, payload) and probe (fk, value) relations of
 * 16-byte (int64, int64) device tuples.  Result: count and
 * sum(build payload + probe value) over the joined pairs (wrapping). */
typedef struct pyg_fragment {
    const void* build;
    int64_t nbuild;
    const void* probe;
    int64_t nprobe;
} pyg_fragment;

typedef struct pyg_tuning {
    int32_t block_threads;       /* threads per CTA of the persistent kernel */
    int32_t blocks_per_sm;       /* resident CTAs per SM                     */
    float load_factor;           /* per-fragment table load factor           */
    int32_t chunk_tuples;        /* work-item grain in tuples                */
    int32_t large_build;         /* build tuples from which a fragment runs
                                    as its own join (0: 2^16)             */
} pyg_tuning;

/* Plans n fragments (tuning NULL: the autotuner's cached choice, else
 * defaults) and captures the execution in a CUDA graph. */
int pyg_batch_create(pyg_ctx* ctx, const pyg_fragment* frags, int32_t n, const pyg_tuning* tuning,
                     pyg_batch** out);
/* Replays the graph once.  counts / sums: host arrays of n (optional);
 * latency_ms: host array of n (optional), device-clock time from batch
 * start to each fragment's completion. */
int pyg_batch_run(pyg_ctx* ctx, pyg_batch* b, int64_t* counts, int64_t* sums, double* latency_ms);
int pyg_batch_free(pyg_ctx* ctx, pyg_batch* b);
/* Failure-detection test hook (host-side injection): makes fragment frag's
 * probe items wait for one build item more than exists, so the next run's
 * bounded device wait gives up (about one second) and pyg_batch_run
 * returns PYG_ERR_TIMEOUT with the context still usable. */
int pyg_batch_inject_stall(pyg_ctx* ctx, pyg_batch* b, int32_t frag);
/* The same fragments one after another through pyg_hashjoin_agg (the
 * plain GPU path the batch is measured against). */
int pyg_batch_run_plain(pyg_ctx* ctx, const pyg_fragment* frags, int32_t n, int64_t* counts,
                        int64_t* sums, double* latency_ms);
/* Times candidate tunings (block shape, occupancy, load factor, grain) on
 * the fragments and returns the fastest; cached per workload signature in
 * memory and, if cache_path is not NULL, in a text file. */
int pyg_autotune(pyg_ctx* ctx, const pyg_fragment* frags, int32_t n, const char* cache_path,
                 pyg_tuning* out);

#ifdef __cplusplus
}
#endif
#endif /* PYG_BATCH_H */
