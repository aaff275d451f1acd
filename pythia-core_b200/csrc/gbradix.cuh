// Group-by of 16-byte (int64 key, int64 value) device tuples aggregated in
// shared memory (gbradix.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "pyg_internal.cuh"

namespace pyg {

// The shared-memory path needs a group estimate (the plan's bucket count or
// the caller's expected_groups).
bool groupby16_eligible(int64_t expected_groups);

// Fills the group-by result table (cap 32-byte slots {key, sum, count, -},
// already initialised empty) and flags {full, groups, INT64_MIN sum,
// INT64_MIN count} from n tuples at `in` (16-byte aligned).  Enqueued on
// the context's stream.
int groupby16_fill(pyg_ctx* ctx, const void* in, int64_t n, int want_sum, int64_t expected_groups, ulonglong4* table,
                   uint64_t cap, unsigned long long* flags);

}  // namespace pyg
