/*
 * pyg_mpsm.h - MPSM sort-merge join of the B200 engine (libpyg.so).
 *
 * Replaces SortMergeJoinOp / OldMPSMJoinOp (operators/join.cpp:905-1617,
 * plan types sortmergejoin / mpsmjoin) together with the range partition
 * that feeds them (PartitionOp with exactrange, operators/partition.cpp,
 * and the buildprepartitioned option, join.cpp:1002-1009, :1266-1283).
 *
 * Both inputs are range-partitioned by the same splitters (equal-width as
 * the reference's ExactRangeValueHasher, quantiles of a key sample, or the
 * learned CDF model), each partition is sorted (4 KB pages bitonic-sorted
 * in shared memory, then merge-path merge rounds), and matching partitions
 * are merge-joined.  Single join key column per side (int32 or int64).
 */
#ifndef PYG_MPSM_H
#define PYG_MPSM_H

#include "pyg.h"

#ifdef __cplusplus
extern "C" {
#endif

#define PYG_MPSM_SPLIT_EXACTRANGE 0  /* equal-width ranges (reference)  */
#define PYG_MPSM_SPLIT_SAMPLED    1  /* quantiles of a key sample        */
#define PYG_MPSM_SPLIT_LEARNED    2  /* trained piecewise-linear CDF     */

typedef struct pyg_mpsm_opts {
    int32_t splitter_kind;       /* PYG_MPSM_SPLIT_*                     */
    int32_t fanout;              /* range partitions (<= 2^14)           */
    double sample_rate;          /* fraction of probe keys sampled       */
    int32_t cdf_leaves;          /* learned model leaves (e.g. 1024)     */
    int32_t page_tuples;         /* bitonic page size in tuples: 256 = 4 KB of 16-byte items */
    uint64_t seed;
} pyg_mpsm_opts;

typedef struct pyg_mpsm_stats {
    double max_partition_imbalance;  /* max / mean probe partition size */
    int64_t max_partition;           /* largest probe partition          */
    double splitter_ms;
    double partition_ms;
    double sort_ms;
    double merge_ms;
} pyg_mpsm_stats;

/* Aggregate sink: count + wrapped sums of the projected columns (each side
 * may project any of its columns). */
int pyg_mpsm_join_agg(pyg_ctx* ctx, const pyg_rel* build, int32_t build_key, const pyg_rel* probe,
                      int32_t probe_key, const pyg_proj* proj, int32_t nproj,
                      const pyg_mpsm_opts* opts, pyg_join_result* out, pyg_mpsm_stats* stats);

/* Materialising variant into a device buffer of out_capacity tuples
 * (projected columns packed).  Output order: ascending key, then probe
 * input position, then build input position.  PYG_ERR_CAPACITY (with
 * *out_count set) when the result does not fit. */
int pyg_mpsm_join_materialize(pyg_ctx* ctx, const pyg_rel* build, int32_t build_key,
                              const pyg_rel* probe, int32_t probe_key, const pyg_proj* proj,
                              int32_t nproj, const pyg_mpsm_opts* opts, void* out,
                              int64_t out_capacity, int64_t* out_count);

#ifdef __cplusplus
}
#endif
#endif /* PYG_MPSM_H */
