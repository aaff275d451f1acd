// Radix hash join + aggregation with shared-memory tables (radixjoin.cu).
#pragma once
#include <stdint.h>

#include "pyg.h"
#include "radixpart.cuh"

struct pyg_ctx;

namespace pyg {





// Joins 16-byte (int64 key, int64 payload) device relations R and S on the
// key and returns out = {match count, wrapped sum of R payloads, wrapped sum
// of S payloads} over the joined pairs.  fine_bits <= 0 picks the partition
// count from |R|.  Fills the timing fields of stats when it is not null.
int radix_join16(pyg_ctx* ctx, const void* R, int64_t nR, const void* S, int64_t nS, int fine_bits,
                 unsigned long long out[3], pyg_join_stats* stats);

}  // namespace pyg
