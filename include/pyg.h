/*
 * pyg.h - C ABI of the B200 join / aggregation engine (libpyg.so).
 *
 * Plain pointers and sizes only.  Every function returns an int status
 * (PYG_OK == 0, negative on failure; pyg_last_error() gives the message of
 * the calling thread's last failure).  A context binds one CUDA device and
 * one stream; calls on a context are stream-ordered and a context is used
 * by one host thread at a time.  The caller owns every buffer it passes in;
 * the library owns hash tables, CDF models and batch plans until their
 * *_free call.
 *
 * Each entry point names the reference interface it replaces
 * (damodar123/pythia-core, paths relative to that project).
 */
#ifndef PYG_H
#define PYG_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------- */
#define PYG_OK               0
#define PYG_ERR_ARG         -1  /* bad argument / unsupported schema      */
#define PYG_ERR_OOM         -2  /* device or host allocation failed       */
#define PYG_ERR_CUDA        -3  /* CUDA runtime error                     */
#define PYG_ERR_TABLE_FULL  -4  /* open-addressing probe limit exceeded   */
#define PYG_ERR_TIMEOUT     -5  /* a bounded device-side wait gave up     */
#define PYG_ERR_CAPACITY    -6  /* caller's output buffer too small       */
#define PYG_ERR_NO_DEVICE   -7  /* no CUDA device / extension unusable    */

/* ---- column types (reference CT_INTEGER / CT_LONG, schema.h) --------- */
#define PYG_INT32 1
#define PYG_INT64 2
#define PYG_MAX_COLS 8

/* A relation: packed row-major fixed-width tuples, the layout of a
 * reference TupleBuffer page for schema ("long","long",...)
 * (util/buffer.h:134-357; columns packed back to back by Schema::add,
 * schema.cpp).  base is device memory of the context's device when
 * on_device != 0, else (pinned or pageable) host memory. */
typedef struct pyg_rel {
    const void* base;
    int64_t ntuples;
    int32_t tuple_bytes;
    int32_t ncols;
    int32_t col_offset[PYG_MAX_COLS];
    int32_t col_type[PYG_MAX_COLS];
    int32_t on_device;
    int32_t reserved;
} pyg_rel;

/* One projected output column: side 0 = build ("B$col"), 1 = probe
 * ("P$col"); the reference's projection list (operators/join.cpp:142-183). */
typedef struct pyg_proj {
    int32_t side;
    int32_t col;
} pyg_proj;

/* ---- context -------------------------------------------------------- */
typedef struct pyg_ctx pyg_ctx;

/* Replaces the per-thread setup of MergeOp::threadInit
 * (operators/merge.cpp:304-353): binds a device and a stream. */
int pyg_ctx_create(int device, pyg_ctx** out);
int pyg_ctx_destroy(pyg_ctx* ctx);
/* Use a caller-owned cudaStream_t (passed as void*); NULL restores the
 * context's own stream. */
int pyg_ctx_set_stream(pyg_ctx* ctx, void* cuda_stream);
void* pyg_ctx_stream(pyg_ctx* ctx);
int pyg_ctx_sync(pyg_ctx* ctx);
/* Number of kernels this context has launched so far. */
int64_t pyg_ctx_kernel_launches(pyg_ctx* ctx);
const char* pyg_last_error(void);
const char* pyg_version(void);

/* Stream-ordered device allocation (replaces numaallocate_local /
 * numaallocate_onnode, util/numaallocate.h:35-39). */
int pyg_alloc(pyg_ctx* ctx, size_t bytes, void** out);
int pyg_free(pyg_ctx* ctx, void* ptr);
int pyg_host_alloc(size_t bytes, void** out);   /* pinned host memory */
int pyg_host_free(void* ptr);
int pyg_memcpy_h2d(pyg_ctx* ctx, void* dst, const void* src, size_t bytes);
int pyg_memcpy_d2h(pyg_ctx* ctx, void* dst, const void* src, size_t bytes);
int pyg_memcpy_d2d(pyg_ctx* ctx, void* dst, const void* src, size_t bytes);

/* ---- overlapped ingest ---------------------------------------------- */
/* A host byte stream uploaded into one device buffer through a ring of
 * pinned staging slots: while slot i's copy runs on the context's copy
 * stream, the caller fills slot i+1 (reads a file chunk, parses text).
 * Replaces the scan's whole-file load into memory followed by a separate
 * copy (ParallelScanOp::scanStart / MemMappedTable::load,
 * operators/parallelscan.cpp:176-190, operators/loaders/table.cpp:198-348).
 *
 *   pyg_upload_open   device buffer of `capacity` bytes (grown on demand),
 *                     `slots` staging buffers of `slot_bytes` each.
 *   pyg_upload_slot   the next staging buffer (waits for its last copy).
 *   pyg_upload_commit queues the copy of its first `bytes` to the end of
 *                     the uploaded data (`bytes` <= slot_bytes).
 *   pyg_upload_finish waits for every copy; hands over the device buffer
 *                     (owned by the caller, pyg_free) and the byte count,
 *                     and frees the staging slots.
 *   pyg_upload_abort  frees everything (after an error). */
typedef struct pyg_upload pyg_upload;
int pyg_upload_open(pyg_ctx* ctx, size_t capacity, size_t slot_bytes, int32_t slots, pyg_upload** out);
int pyg_upload_slot(pyg_ctx* ctx, pyg_upload* up, void** buf, size_t* bytes);
int pyg_upload_commit(pyg_ctx* ctx, pyg_upload* up, size_t bytes);
int pyg_upload_finish(pyg_ctx* ctx, pyg_upload* up, void** device_buffer, size_t* total_bytes);
int pyg_upload_abort(pyg_ctx* ctx, pyg_upload* up);

/* ---- hash join ------------------------------------------------------ */
/* Table modes.  AGGREGATE keeps one entry per distinct key with the
 * duplicate count and the wrapped sums of the stored build columns (all a
 * fused count/sum probe needs); MATERIALIZE keeps every build tuple so a
 * probe can emit each joined pair. */
#define PYG_HT_AGGREGATE    1
#define PYG_HT_MATERIALIZE  2

typedef struct pyg_hashtable pyg_hashtable;

typedef struct pyg_join_result {
    int64_t count;                 /* number of joined pairs             */
    int64_t sums[PYG_MAX_COLS];    /* wrapped sum of each projected col  */
} pyg_join_result;

/* Build: replaces HashJoinOp::threadInit + scanStart/buildFromPage
 * (operators/join.cpp:520-637, :838-884) and HashTable::init/allocate
 * (util/hashtable.cpp:57-89, :254-292).  key_cols: 1 or 2 columns whose
 * widths total at most 8 bytes (int64, int32, or int32+int32).
 * payload_cols: build columns kept in the table (those a projection may
 * reference as B$col).  load_factor in (0, 0.95]. */
int pyg_hashjoin_build(pyg_ctx* ctx, const pyg_rel* build, const int32_t* key_cols, int32_t nkeys,
                       const int32_t* payload_cols, int32_t npayload, int32_t mode,
                       float load_factor, pyg_hashtable** out);
int pyg_hashtable_free(pyg_ctx* ctx, pyg_hashtable* ht);
/* Distinct keys (AGGREGATE) or stored tuples (MATERIALIZE); 1 if any build
 * key occurred more than once. */
int pyg_hashtable_stats(pyg_ctx* ctx, const pyg_hashtable* ht, int64_t* entries, int64_t* capacity,
                        int32_t* has_duplicates);

/* Probe with a fused aggregate sink: replaces HashJoinOp::getNext
 * (operators/join.cpp:681-757) feeding printer_tuplecount and
 * aggregate_sum(fields=[]) over each projected column
 * (operators/genericaggregate.cpp:247-289, aggregatesum.cpp:81-105).
 * Result written to host memory *out after the stream is synchronised. */
int pyg_hashjoin_probe_agg(pyg_ctx* ctx, const pyg_hashtable* ht, const pyg_rel* probe,
                           const int32_t* key_cols, const pyg_proj* proj, int32_t nproj,
                           pyg_join_result* out);

/* Probe materialising joined tuples (projected columns packed in
 * projection order, HashJoinOp::constructOutputTuple, operators/
 * join.cpp:648-679) into device buffer out.  Requires a MATERIALIZE table.
 * *out_count receives the number of pairs; PYG_ERR_CAPACITY if it exceeds
 * out_capacity (nothing past out_capacity is written). */
int pyg_hashjoin_probe_materialize(pyg_ctx* ctx, const pyg_hashtable* ht, const pyg_rel* probe,
                                   const int32_t* key_cols, const pyg_proj* proj, int32_t nproj,
                                   void* out, int64_t out_capacity, int64_t* out_count);

/* One-shot join + aggregate (build and probe in one call), the plan
 * hashjoin -> aggregate_sum of the reference (HashJoinOp::scanStart +
 * getNext, operators/join.cpp:548-757, feeding GenericAggregate).
 * PYG_JOIN_DIRECT: one table in HBM, probed in input order; for 16-byte
 * device relations a three-launch call with one host synchronisation whose
 * table lives in a buffer the context keeps between calls.
 * PYG_JOIN_RADIX: both sides partitioned by the top radix_bits bits of the
 * key hash first, then joined partition by partition with shared-memory
 * tables (16-byte (int64, int64) device relations, projection over
 * {B$1, P$1}; other shapes use DIRECT).  PYG_JOIN_AUTO picks RADIX for
 * eligible inputs whose direct table would exceed 64 MB (so not stay in
 * L2) and whose probe side has at least 2^22 tuples.  stats (optional)
 * receives phase timings. */
#define PYG_JOIN_AUTO   0
#define PYG_JOIN_DIRECT 1
#define PYG_JOIN_RADIX  2

typedef struct pyg_join_opts {
    int32_t algorithm;     /* PYG_JOIN_*                               */
    int32_t radix_bits;    /* log2 partition fan-out (0 = automatic)   */
    float load_factor;     /* table load factor (0 = 0.5)              */
    int32_t reserved;
} pyg_join_opts;

typedef struct pyg_join_stats {
    int32_t algorithm;
    int32_t radix_bits;
    double build_partition_ms;  /* build side partition passes (RADIX)  */
    double build_ms;            /* table init + inserts                 */
    double probe_partition_ms;  /* probe side partition passes (RADIX)  */
    double probe_ms;            /* probes + fused aggregation           */
    int64_t overflow_tuples;
    int64_t padded_tuples;
    double histogram_ms;        /* both relations' histograms (RADIX)   */
    int64_t histogram_tuples;   /* tuples the histograms read (RADIX)   */
    /* RADIX: each partition pass on its own (pass 2 is 0 with one pass);
     * build_partition_ms / probe_partition_ms also hold the host round
     * trip that lays the relation out. */
    double build_pass_ms[2];
    double probe_pass_ms[2];
    int32_t build_packed;       /* 8-byte packed intermediates (RADIX)  */
    int32_t probe_packed;
    /* RADIX: the join kernel alone; probe_ms also holds the host round trip
     * that reads the partition counts and uploads the work items. */
    double join_kernel_ms;
} pyg_join_stats;

int pyg_hashjoin_agg(pyg_ctx* ctx, const pyg_rel* build, const int32_t* build_keys,
                     const pyg_rel* probe, const int32_t* probe_keys, int32_t nkeys,
                     const pyg_proj* proj, int32_t nproj, const pyg_join_opts* opts,
                     pyg_join_result* out, pyg_join_stats* stats);

/* Hash join + sum that allocates nothing.  No counterpart in the
 * reference: it is for callers that cannot call cudaMalloc where they
 * join, such as an engine whose device memory all belongs to another
 * allocator (a framework's caching pool, a query runtime's arena) that a
 * library must not bypass, or a latency-critical path where an allocation
 * could block on the device.  The table lives in a fixed device array
 * inside the library (about 16 MiB held on every GPU that loads the
 * library until the process exits), so the build side is limited to
 * PYG_NOALLOC_MAX_BUILD tuples; larger inputs are rejected with
 * PYG_ERR_ARG.  Inputs: 16-byte (int64 key, int64 payload) device tuples.
 * Output: out_dev[0..2] (device) = match count, wrapped sum of build
 * payloads, wrapped sum of probe payloads over the joined pairs.  Kernels
 * are only enqueued on `stream` (a cudaStream_t, NULL = legacy default
 * stream) on the current device; nothing is synchronised.  The first call
 * on a device looks up the array's device address once (make that first
 * call before any stream capture); a device reset (cudaDeviceReset)
 * invalidates the address, so reload the library after one.  Calls share
 * the array (each clears it first), so calls that overlap on the GPU
 * race: order them on one stream.  A CUDA error still pending from an
 * earlier, unrelated call is reported (and left pending) before anything
 * is enqueued. */
#define PYG_NOALLOC_MAX_BUILD (1 << 18)
int pyg_hashjoin_agg_noalloc(const void* build, int64_t nbuild, const void* probe, int64_t nprobe,
                             int64_t* out_dev, void* stream);

/* ---- group-by aggregation ------------------------------------------ */
#define PYG_AGG_SUM    1
#define PYG_AGG_COUNT  2

/* Replaces GenericAggregate::scanStart/remember/getNext with AggregateSum
 * and AggregateCount folds (operators/genericaggregate.cpp:247-494,
 * aggregatesum.cpp:53-105, aggregatecount.cpp:44-52).  Output tuples (device
 * buffer): key columns packed, then the sum (type of sum_col) if
 * PYG_AGG_SUM, then the int64 count if PYG_AGG_COUNT.  nkeys == 0 is the
 * no-GROUP-BY case.  sort_by_key != 0 orders groups by key (signed,
 * lexicographic over key columns). */
int pyg_groupby(pyg_ctx* ctx, const pyg_rel* in, const int32_t* key_cols, int32_t nkeys,
                int32_t flags, int32_t sum_col, int32_t sort_by_key, int64_t expected_groups,
                void* out, int64_t out_capacity, int64_t* out_groups);

/* ---- partition ------------------------------------------------------ */
#define PYG_SPLIT_EXACTRANGE 0   /* ExactRangeValueHasher(min,max,fanout) */
#define PYG_SPLIT_SPLITTERS  1   /* fanout-1 ascending splitters          */
#define PYG_SPLIT_RADIX      2   /* low log2(fanout) bits of the key      */
#define PYG_SPLIT_HASH       3   /* high bits of a 64-bit mix of the key  */

typedef struct pyg_splitter {
    int32_t kind;
    int32_t fanout;
    int64_t range_min;           /* EXACTRANGE                           */
    int64_t range_max;
    const int64_t* splitters;    /* SPLITTERS: host array, fanout-1 long */
} pyg_splitter;

/* Replaces PartitionOp::scanStart (operators/partition.cpp:272-359):
 * histogram, exclusive prefix, scatter.  out: device buffer of
 * in->ntuples tuples; offsets: host array of fanout+1 entries.
 * Fails with PYG_ERR_ARG if an EXACTRANGE key falls outside the range. */
int pyg_partition(pyg_ctx* ctx, const pyg_rel* in, int32_t key_col, const pyg_splitter* spl,
                  void* out, int64_t* offsets);

/* ---- sort ----------------------------------------------------------- */
/* Replaces SortOp / TupleBuffer::sort<KeyT> (operators/sort.cpp:87-311,
 * util/buffer.inl:119-452): orders tuples by the signed key column.
 * Stable.  out may not alias in. */
int pyg_sort(pyg_ctx* ctx, const pyg_rel* in, int32_t key_col, void* out);

/* Replaces SortLimit (operators/sortlimit.cpp:32-262, plan node
 * `sortlimit`): the first min(limit, n) tuples of the relation in the
 * order of the key columns (1 or 2 columns of at most 8 bytes together,
 * lexicographic, signed), ascending when asc != 0 else descending, ties
 * kept in input order, written to device buffer out.  *out_n receives the
 * count; PYG_ERR_CAPACITY if it exceeds out_capacity. */
int pyg_sortlimit(pyg_ctx* ctx, const pyg_rel* in, const int32_t* key_cols, int32_t nkeys, int32_t asc,
                  int64_t limit, void* out, int64_t out_capacity, int64_t* out_n);

/* Replaces TupleBuffer::bitonicsort (util/buffer.cpp:97-110) and its SIMD
 * merge sort (util/bitonicsort.cpp:59-74, 371-443): sorts n 8-byte records
 * {int32 rid; int32 key} of device buffer `records` in place by the signed
 * key.  4096-record pages are bitonic-sorted in shared memory (each page
 * brought in by one bulk copy), then merged.  Equal keys end in rid order
 * (the reference leaves it open).  The reference requires n = 2^k > 4096;
 * any n works here.  records must be 16-byte aligned. */
int pyg_bitonic_sort(pyg_ctx* ctx, void* records, int64_t n);

/* Replaces TupleBuffer::findsmallest<KeyT> (util/buffer.inl:~300-452):
 * for each of nq query keys (device array), the index of the first tuple
 * of the sorted relation whose key is >= the query. */
int pyg_lower_bound(pyg_ctx* ctx, const pyg_rel* sorted, int32_t key_col, const int64_t* queries,
                    int64_t nq, int64_t* out_idx);

/* ---- seeded synthetic data (bench / tests) -------------------------- */
/* keys = 1 + seeded permutation of [0, n) (bijective hash of the index),
 * payload = key * payload_mul.  16-byte (int64, int64) tuples. */
int pyg_gen_pk(pyg_ctx* ctx, void* out, int64_t n, int64_t payload_mul, uint64_t seed);
/* fk ~ Zipf(theta) over ranks 1..nkeys mapped through the same
 * permutation as pyg_gen_pk(seed_keys) (theta == 0: uniform);
 * value ~ U[0, vmax). */
int pyg_gen_fk(pyg_ctx* ctx, void* out, int64_t n, int64_t nkeys, double theta, uint64_t seed_keys,
               int64_t vmax, uint64_t seed);

#ifdef __cplusplus
}
#endif
#endif /* PYG_H */
