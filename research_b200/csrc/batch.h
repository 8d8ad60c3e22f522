// Stacking of many independent products into one block-diagonal product
// (implemented in batch.cu).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "ocean_internal.cuh"

namespace ocean {

// One product of a batch, with its place in the stacked inputs.
struct BatchProblem {
  const void* a_rp;
  const uint32_t* a_col;
  const double* a_val;
  const void* b_rp;
  const uint32_t* b_col;
  const double* b_val;
  uint64_t nnz0, brow0, bnnz0;  // first entry of A_p, first row and entry of B_p in the stacked arrays
  uint32_t a_bits, b_bits;      // row-pointer widths of A_p and B_p
};

// Stacked row pointers (rows + 1 values; the last is total_nnz) of A (of_b
// false) or B. row_prefix: n + 1 first-row offsets of the problems.
template <typename RPO>
void launch_batch_rowptr(const BatchProblem* probs, const uint64_t* row_prefix, uint32_t n, uint64_t rows,
                         uint64_t total_nnz, bool of_b, RPO* out, cudaStream_t s);

// Stacked column ids (A's shifted by brow0) and values (skipped if val_out is null).
void launch_batch_entries(const BatchProblem* probs, const uint64_t* nnz_prefix, uint32_t n, uint64_t total,
                          bool of_b, uint32_t* col_out, double* val_out, cudaStream_t s);

// Per-problem row pointers of the stacked C: out[out_prefix[p] + r] =
// big[row_prefix[p] + r] - big[row_prefix[p]] for r in [0, rows_p];
// out_prefix[p] = row_prefix[p] + p, total = rows + n.
template <typename RPI, typename RPO>
void launch_batch_rebase(const RPI* big, const uint64_t* row_prefix, const uint64_t* out_prefix, uint32_t n,
                         uint64_t total, RPO* out, cudaStream_t s);

// Capacity guard of a batch run (one thread): if *total > cap, the planned
// buffers are too small for this run's structure: set DEV_BATCH_MISMATCH in
// ctr->status and empty the numeric and overflow row queues, so no later
// kernel writes past the buffers.
void launch_batch_guard(DevCounters* ctr, const unsigned long long* total, unsigned long long cap, cudaStream_t s);

// out[p] = big[row_prefix[p]] for p in [0, n].
template <typename RPI>
void launch_batch_bounds(const RPI* big, const uint64_t* row_prefix, uint32_t n, uint64_t* out, cudaStream_t s);

}  // namespace ocean
