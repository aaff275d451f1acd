// MPSM join + aggregation of 16-byte (int64 key, int64 payload) device
// relations (mpsm16.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "pyg_internal.cuh"

namespace pyg {

// log2 of the range count mpsm16_agg wants for these relation sizes.
int mpsm16_fine_bits(int64_t nR, int64_t nS);

struct RJModel;

// Range-partitions R and S by the 2^FB - 1 ascending splitters, sorts each
// range's build tuples in shared memory and merges the probe tuples into
// them.  out = {match count, wrapped sum of R payloads, wrapped sum of S
// payloads}.  sizes (optional) receives the probe tuples per range.
// model (optional): the bins come from the learned model (rj_model_bin,
// model->fbits == FB) instead of a splitter search, and `splitters` must
// be that model's splitters (model_splitters), which bound the ranges.
int mpsm16_agg(pyg_ctx* ctx, const void* R, int64_t nR, const void* S, int64_t nS, const int64_t* splitters, int FB,
               unsigned long long out[3], std::vector<unsigned long long>* sizes, float* part_ms, float* join_ms,
               const RJModel* model = nullptr);

}  // namespace pyg
