// codes.h -- 4-bit code rows of a flat index and the exact re-rank that follows a search
// over them.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/pgb.h"

namespace pgb {

// Re-ranks each query's first R candidates (cand: nq x R ids, padded with 0xFFFFFFFF) by
// the exact distance to the index's vector rows, ties by id, and writes the k best
// (ids / dists: nq x k, padded with PGB_NO_NEIGHBOR / INT32_MAX).
pgb_status rerank_launch(const pgb_index* ix, const void* queries, uint32_t nq,
                         uint32_t query_stride, const uint32_t* cand, uint32_t R, uint32_t k,
                         uint32_t* ids, int32_t* dists, cudaStream_t stream);

// Host restatement of the quantizer choice from per-dimension histograms (hist: dim x 256
// counts of value - lo, lo = -128 for int8 and 0 for uint8): the step in 1..17 and, per
// dimension, the offset that minimise the total squared reconstruction error (ties: the
// smaller step, then the smaller offset), with every reconstructed value inside the
// element's range.
void choose_codes(const uint64_t* hist, uint32_t dim, bool is_signed, int32_t* step,
                  int32_t* offsets);

}  // namespace pgb
