// The device hash table shared by the hash join entry points.
#pragma once

#include "pyg_internal.cuh"

// Open-addressing table of cap slots, W 64-bit words per slot: word 0 is
// the packed key (kEmptyKey marks a free slot), words 1..W-1 hold the
// stored build columns (MATERIALIZE: one slot per build tuple) or their
// wrapped per-key sums (AGGREGATE: one slot per distinct key).  Build
// tuples whose key word equals kEmptyKey live in a small side list.
struct pyg_hashtable {
    int32_t mode;
    int32_t nkeys;
    pyg::KeySpec ks;
    int32_t npay;
    int32_t pay_cols[PYG_MAX_COLS];
    int32_t pay_types[PYG_MAX_COLS];
    int32_t W;
    uint64_t cap;
    uint64_t* slots = nullptr;
    uint64_t* side = nullptr;
    int64_t nside = 0;
    unsigned long long* counts = nullptr;  // AGGREGATE with duplicate keys
    int32_t has_dups = 0;
    int64_t entries = 0;
};
