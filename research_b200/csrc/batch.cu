// Batched execution: many independent products C_p = A_p * B_p run as one
// block-diagonal product. The rows of every A_p are stacked into one A (their
// column ids shifted by the first row of B_p in the stacked B), the rows of
// every B_p into one B (column ids unchanged), so row g of the stacked C is
// row g - row0_p of C_p with C_p's own column ids, and every class kernel
// handles the rows of all problems in one persistent launch. These kernels
// build the stacked inputs and split the stacked C's row pointers back into
// one row-pointer array per problem.
#include "batch.h"

namespace ocean {
namespace {

// Largest p < n with prefix[p] <= g (prefix: n + 1 ascending offsets).
__device__ __forceinline__ uint32_t find_problem(const uint64_t* __restrict__ prefix, uint32_t n, uint64_t g) {
  uint32_t lo = 0, hi = n;  // answer in [lo, hi)
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (prefix[mid] <= g) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <typename RPO>
__global__ void __launch_bounds__(256) k_batch_rowptr(const BatchProblem* __restrict__ probs,
                                                      const uint64_t* __restrict__ row_prefix, uint32_t n,
                                                      uint64_t rows, uint64_t total_nnz, bool of_b,
                                                      RPO* __restrict__ out) {
  for (uint64_t g = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; g <= rows;
       g += (uint64_t)gridDim.x * blockDim.x) {
    if (g == rows) {
      out[g] = (RPO)total_nnz;
      continue;
    }
    const uint32_t p = find_problem(row_prefix, n, g);
    const BatchProblem& q = probs[p];
    const uint64_t r = g - row_prefix[p];
    const void* rp = of_b ? q.b_rp : q.a_rp;
    const uint32_t bits = of_b ? q.b_bits : q.a_bits;
    const uint64_t v = bits == 32 ? (uint64_t)((const uint32_t*)rp)[r] : ((const uint64_t*)rp)[r];
    out[g] = (RPO)((of_b ? q.bnnz0 : q.nnz0) + v);
  }
}

__global__ void __launch_bounds__(256) k_batch_entries(const BatchProblem* __restrict__ probs,
                                                       const uint64_t* __restrict__ nnz_prefix, uint32_t n,
                                                       uint64_t total, bool of_b, uint32_t* __restrict__ col_out,
                                                       double* __restrict__ val_out) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = find_problem(nnz_prefix, n, e);
    const BatchProblem& q = probs[p];
    const uint64_t k = e - nnz_prefix[p];
    if (of_b) {
      col_out[e] = q.b_col[k];
      if (val_out) val_out[e] = q.b_val[k];
    } else {
      col_out[e] = q.a_col[k] + (uint32_t)q.brow0;  // A's column ids index the stacked B's rows
      if (val_out) val_out[e] = q.a_val[k];
    }
  }
}

// out[out_prefix[p] + r] = big[row_prefix[p] + r] - big[row_prefix[p]], r in [0, rows_p].
template <typename RPI, typename RPO>
__global__ void __launch_bounds__(256) k_batch_rebase(const RPI* __restrict__ big,
                                                      const uint64_t* __restrict__ row_prefix,
                                                      const uint64_t* __restrict__ out_prefix, uint32_t n,
                                                      uint64_t total, RPO* __restrict__ out) {
  for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = find_problem(out_prefix, n, e);
    const uint64_t r = e - out_prefix[p];
    const uint64_t base = row_prefix[p];
    out[e] = (RPO)((uint64_t)big[base + r] - (uint64_t)big[base]);
  }
}

// Start of every problem's entries in the stacked C (n + 1 values).
template <typename RPI>
__global__ void k_batch_bounds(const RPI* __restrict__ big, const uint64_t* __restrict__ row_prefix, uint32_t n,
                               uint64_t* __restrict__ out) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p <= n) out[p] = (uint64_t)big[row_prefix[p]];
}

__global__ void k_batch_guard(DevCounters* __restrict__ ctr, const unsigned long long* __restrict__ total,
                              unsigned long long cap) {
  if (*total <= cap) return;
  atomicOr(&ctr->status, (unsigned)DEV_BATCH_MISMATCH);
  for (int c = 0; c < NB_COUNT; ++c) ctr->num_count[c] = 0;
  ctr->overflow_n = 0;
}

unsigned grid_for(uint64_t n) {
  const uint64_t b = (n + 255) / 256;
  return (unsigned)(b < 148ull * 32 ? (b ? b : 1) : 148ull * 32);
}

}  // namespace

template <typename RPO>
void launch_batch_rowptr(const BatchProblem* probs, const uint64_t* row_prefix, uint32_t n, uint64_t rows,
                         uint64_t total_nnz, bool of_b, RPO* out, cudaStream_t s) {
  k_batch_rowptr<RPO><<<grid_for(rows + 1), 256, 0, s>>>(probs, row_prefix, n, rows, total_nnz, of_b, out);
}

void launch_batch_entries(const BatchProblem* probs, const uint64_t* nnz_prefix, uint32_t n, uint64_t total,
                          bool of_b, uint32_t* col_out, double* val_out, cudaStream_t s) {
  if (total == 0) return;
  k_batch_entries<<<grid_for(total), 256, 0, s>>>(probs, nnz_prefix, n, total, of_b, col_out, val_out);
}

template <typename RPI, typename RPO>
void launch_batch_rebase(const RPI* big, const uint64_t* row_prefix, const uint64_t* out_prefix, uint32_t n,
                         uint64_t total, RPO* out, cudaStream_t s) {
  if (total == 0) return;
  k_batch_rebase<RPI, RPO><<<grid_for(total), 256, 0, s>>>(big, row_prefix, out_prefix, n, total, out);
}

void launch_batch_guard(DevCounters* ctr, const unsigned long long* total, unsigned long long cap, cudaStream_t s) {
  k_batch_guard<<<1, 1, 0, s>>>(ctr, total, cap);
}

template <typename RPI>
void launch_batch_bounds(const RPI* big, const uint64_t* row_prefix, uint32_t n, uint64_t* out, cudaStream_t s) {
  k_batch_bounds<RPI><<<(n + 1 + 255) / 256, 256, 0, s>>>(big, row_prefix, n, out);
}

template void launch_batch_rowptr<uint32_t>(const BatchProblem*, const uint64_t*, uint32_t, uint64_t, uint64_t, bool,
                                            uint32_t*, cudaStream_t);
template void launch_batch_rowptr<uint64_t>(const BatchProblem*, const uint64_t*, uint32_t, uint64_t, uint64_t, bool,
                                            uint64_t*, cudaStream_t);
template void launch_batch_rebase<uint32_t, uint32_t>(const uint32_t*, const uint64_t*, const uint64_t*, uint32_t,
                                                      uint64_t, uint32_t*, cudaStream_t);
template void launch_batch_rebase<uint64_t, uint64_t>(const uint64_t*, const uint64_t*, const uint64_t*, uint32_t,
                                                      uint64_t, uint64_t*, cudaStream_t);
template void launch_batch_rebase<uint64_t, uint32_t>(const uint64_t*, const uint64_t*, const uint64_t*, uint32_t,
                                                      uint64_t, uint32_t*, cudaStream_t);
template void launch_batch_bounds<uint32_t>(const uint32_t*, const uint64_t*, uint32_t, uint64_t*, cudaStream_t);
template void launch_batch_bounds<uint64_t>(const uint64_t*, const uint64_t*, uint32_t, uint64_t*, cudaStream_t);

}  // namespace ocean
