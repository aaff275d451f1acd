// Radix hash join + aggregation with shared-memory tables (radixjoin.cu).
#pragma once
#include <stdint.h>

#include "pyg.h"
#include "radixpart.cuh"

struct pyg_ctx;

namespace pyg {

struct PhaseTimer;

// The one-shot direct join of 16-byte (int64 key, int64 payload) device
// relations (hashjoin.cu), enqueued on ctx->stream without waiting: clear,
// build and probe through the context's table arena, with the counters in
// 11 device words (`words`; the build's flags in [0..2], the sums in
// [8..10]).  Joins enqueued one after another on the stream reuse the
// arena in stream order.  tm (optional) records the phase events.
int direct_join16_enqueue(pyg_ctx* ctx, const void* R, int64_t nR, const void* S, int64_t nS, float lf,
                          unsigned long long* words, PhaseTimer* tm = nullptr);
// The result from a host copy of those words: false when the build side
// repeated a key or overfilled its side list (the probe stood down and
// the general path must answer), else res = {count, build payload sum,
// probe payload sum}.
bool direct_join16_result(const unsigned long long* words, int64_t nR, unsigned long long res[3]);

// Joins 16-byte (int64 key, int64 payload) device relations R and S on the
// key and returns out = {match count, wrapped sum of R payloads, wrapped sum
// of S payloads} over the joined pairs.  fine_bits <= 0 picks the partition
// count from |R|.  Fills the timing fields of stats when it is not null.
int radix_join16(pyg_ctx* ctx, const void* R, int64_t nR, const void* S, int64_t nS, int fine_bits,
                 unsigned long long out[3], pyg_join_stats* stats);

}  // namespace pyg
