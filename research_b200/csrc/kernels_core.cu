// SpGEMM kernels for sm_100a: row analysis, symbolic and numeric accumulators, scan.
//
// Reference counterparts (paths inside the reference project):
//   row analysis            kernels/Analysis.cuh:31-105   (analysisKernel)
//   row binning             kernels/Analysis.cuh:110-303  (binning / numericBinning)
//   ESC accumulator         kernels/AccumulatorESC.cuh:12-166
//   hash accumulators       kernels/AccumulatorHash.cuh:11-755, kernels/Hashmap.cuh:14-281
//   dense accumulators      kernels/AccumulatorDense.cuh:43-893
//   row-pointer scan        cub::DeviceScan::ExclusiveSum at kernels/SpGEMM.cuh:1147,1221,1622
//   column sort             kernels/Epilogue.cuh:68-222 (CUB BlockRadixSort)
//
// Design: every row class runs as a persistent kernel whose blocks pull rows
// from a device-side class list, so the kernels need no bin count from the
// host. The host reads back the class sizes after the analysis (large inputs
// only, to size the grids and the bitmap cache) and the total output count
// (to allocate C).
// Numeric kernels write each row already sorted straight into its final place
// in C, so there is no temporary output buffer and no separate sort/copy pass.
#include <algorithm>
#include <cstdio>
#include <mutex>
#include "kernels.h"

namespace ocean {

// ---------------------------------------------------------------- helpers
__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
  return v;
}

// Block-wide sum; `scratch` holds 33 entries. All threads get the result.
template <int NT>
__device__ __forceinline__ unsigned long long block_sum_u64(unsigned long long v,
                                                            unsigned long long* scratch) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  v = warp_sum_u64(v);
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  if (warp == 0) {
    unsigned long long t = lane < NT / 32 ? scratch[lane] : 0ull;
    t = warp_sum_u64(t);
    if (lane == 0) scratch[32] = t;
  }
  __syncthreads();
  const unsigned long long r = scratch[32];
  __syncthreads();
  return r;
}

// Block-wide exclusive scan; `scratch` holds 33 entries; *total gets the sum.
template <int NT, typename T>
__device__ __forceinline__ T block_excl_scan(T v, T* scratch, T* total) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  T x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const T y = __shfl_up_sync(kFull, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) scratch[warp] = x;
  __syncthreads();
  if (warp == 0) {
    const T s = lane < NT / 32 ? scratch[lane] : T(0);
    T incl = s;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const T y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane < NT / 32) scratch[lane] = incl - s;
    if (lane == 31) scratch[32] = incl;
  }
  __syncthreads();
  const T r = scratch[warp] + x - v;
  *total = scratch[32];
  __syncthreads();
  return r;
}

__device__ __forceinline__ void raise_status(DevCounters* ctr, unsigned bit, uint32_t row) {
  const unsigned old = atomicOr(&ctr->status, bit);
  if (old == 0) ctr->err_row = row;
}

// One thread per row, once the row's true count n is known: exact mode checks
// n against the expected count; estimation mode records n and appends the row
// to the overflow list when it does not fit its slots. Returns whether to write.
__device__ __forceinline__ bool out_accept(const OutSpec& o, DevCounters* ctr, uint32_t row, uint32_t n,
                                           uint32_t cap) {
  if (!o.count) {
    if (n != cap) raise_status(ctr, DEV_COUNT_MISMATCH, row);
    return true;
  }
  o.count[row] = n;
  if (n <= cap) return true;
  const unsigned i = atomicAdd(o.overflow_n, 1u);
  o.overflow[i] = row;
  return false;
}


// Visiting order of a class queue: position i -> list entry (i * stride) mod
// count, with stride ~ 0.618 * count and coprime with it (a golden-ratio
// sequence, a permutation of the list). Lists are filled in row order, so rows
// of similar size sit together; this order spreads them evenly over a
// persistent kernel's run.
__device__ __forceinline__ uint32_t spread_stride(uint32_t count) {
  if (count < 3) return 1u;
  uint32_t st = (uint32_t)((double)count * 0.6180339887498949) | 1u;
  while (st < count) {
    uint32_t a = st, b = count;
    while (b) {
      const uint32_t t = a % b;
      a = b;
      b = t;
    }
    if (a == 1u) return st;
    st += 2u;
  }
  return 1u;
}

__device__ __forceinline__ uint32_t spread_index(uint32_t idx, uint32_t count, uint32_t stride) {
  return (uint32_t)(((uint64_t)idx * stride) % count);
}

// ---------------------------------------------------------------- analysis
// Row table of B for the analysis: first column, last column and length of
// every row in one 16-byte entry, so an A entry costs one load of a table
// that stays in L2 instead of its B row's pointers and two column loads.
template <typename RP>
__global__ void __launch_bounds__(256) k_brow_table(Csr<RP> B, uint4* __restrict__ tab) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < B.rows;
       r += (uint64_t)gridDim.x * blockDim.x) {
    const uint64_t b0 = B.row_begin(r), b1 = B.row_end(r);
    const uint64_t len = b1 - b0;
    tab[r] = make_uint4(len ? B.col[b0] : kEmpty, len ? B.col[b1 - 1] : 0u, (uint32_t)len, (uint32_t)(len >> 32));
  }
}

// Products, smallest first column, largest last column and longest B row
// over A entries k0, k0 + G, k0 + 2G, ... below k1, accumulated into p, mn,
// mx, lb. Four entries per pass have their dependent loads in flight together;
// with the row table of B (btab) each entry is one table load, two per pass.
template <int G, typename RP>
__device__ __forceinline__ void span_part(const Csr<RP>& A, const Csr<RP>& B, const uint4* __restrict__ btab,
                                          uint64_t k0, uint64_t k1, unsigned long long& p, uint32_t& mn,
                                          uint32_t& mx, uint32_t& lb) {
  if (btab) {
    // two table loads in flight: with 32 registers k_analysis keeps 8 blocks
    // per SM (6 with 64-bit row pointers), which hides the block barriers'
    // wait for each block's slowest row (held-out R-MAT 2^21 learned sizing
    // 2.77 -> 2.34 ms against 4 entries in flight at 61 registers)
    for (; k0 < k1; k0 += 2 * G) {
      uint4 t[2];
#pragma unroll
      for (int u = 0; u < 2; ++u)
        t[u] = k0 + (uint64_t)u * G < k1 ? btab[A.col[k0 + (uint64_t)u * G]] : make_uint4(kEmpty, 0u, 0u, 0u);
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint64_t len = (uint64_t)t[u].z | ((uint64_t)t[u].w << 32);
        if (len) {
          p += len;
          mn = min(mn, t[u].x);
          mx = max(mx, t[u].y);
          lb = max(lb, (uint32_t)min(len, (uint64_t)0xFFFFFFFFu));
        }
      }
    }
    return;
  }
  for (; k0 < k1; k0 += 4 * G) {
    uint32_t j[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) j[u] = k0 + (uint64_t)u * G < k1 ? A.col[k0 + (uint64_t)u * G] : kEmpty;
    uint64_t b0[4], b1[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      b0[u] = b1[u] = 0;
      if (j[u] != kEmpty) {
        b0[u] = B.row_begin(j[u]);
        b1[u] = B.row_end(j[u]);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      if (b1[u] > b0[u]) {
        p += b1[u] - b0[u];
        mn = min(mn, B.col[b0[u]]);
        mx = max(mx, B.col[b1[u] - 1]);
        lb = max(lb, (uint32_t)min(b1[u] - b0[u], (uint64_t)0xFFFFFFFFu));
      }
    }
  }
}

// The analysis results of one row: per-row arrays, and whether and where it
// joins a symbolic class (-1: no product, no class).
__device__ __forceinline__ int analysis_write(uint64_t row, uint64_t a_len, unsigned long long p, uint32_t mn,
                                              uint32_t mx, uint32_t lb, uint32_t* __restrict__ prod,
                                              uint32_t* __restrict__ lo, uint32_t* __restrict__ hi,
                                              uint32_t* __restrict__ anz, uint32_t* __restrict__ maxb,
                                              uint32_t* __restrict__ row_nnz, uint64_t* __restrict__ bm_off,
                                              const SymPolicySet& pols, const uint8_t* __restrict__ row_pol) {
  prod[row] = p > 0xFFFFFFFFull ? 0xFFFFFFFFu : (uint32_t)p;
  lo[row] = mn;
  hi[row] = mx;
  anz[row] = (uint32_t)a_len;
  maxb[row] = lb;
  bm_off[row] = ~0ull;
  if (p == 0) {
    row_nnz[row] = 0;
    return -1;
  }
  return sym_bin_for(p, (uint64_t)mx - mn + 1, pols.p[row_pol ? row_pol[row] : 0]);
}

// One group of G lanes per row of A: products, output column span; then the
// row is appended to its symbolic class list (rows with no product get
// row_nnz = 0 here and no class). A block covers 256 / G consecutive rows; its
// class-list append and totals cost one global atomic per class and block.
// Rows longer than kLongRowEntries are only listed here (when the list
// exists) and summarised by k_analysis_long.
template <typename RP, int G>
__global__ void __launch_bounds__(256, sizeof(RP) == 4 ? 8 : 6) k_analysis(Csr<RP> A, Csr<RP> B, uint32_t* __restrict__ prod,
                                                  uint32_t* __restrict__ lo, uint32_t* __restrict__ hi,
                                                  uint32_t* __restrict__ anz, uint32_t* __restrict__ maxb,
                                                  uint32_t* __restrict__ row_nnz, uint64_t* __restrict__ bm_off,
                                                  uint32_t* __restrict__ sym_bins,
                                                  DevCounters* __restrict__ ctr, SymPolicySet pols,
                                                  const uint8_t* __restrict__ row_pol,
                                                  uint32_t* __restrict__ long_rows,
                                                  LongRowAcc* __restrict__ long_acc, uint32_t long_cap,
                                                  uint32_t* __restrict__ long_chunk_row, uint32_t chunk_cap,
                                                  const uint4* __restrict__ btab) {
  __shared__ unsigned long long s_anz[SB_COUNT], s_prod[SB_COUNT], s_words, s_tot;
  __shared__ unsigned s_maxp, s_maxa, s_cnt[SB_COUNT];
  if (threadIdx.x < SB_COUNT) {
    s_anz[threadIdx.x] = 0ull;
    s_prod[threadIdx.x] = 0ull;
    s_cnt[threadIdx.x] = 0u;
  }
  if (threadIdx.x == 0) {
    s_words = 0ull;
    s_tot = 0ull;
    s_maxp = 0u;
    s_maxa = 0u;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int sl = lane & (G - 1);
  const uint64_t row = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) / G;
  const bool valid = row < A.rows;
  uint64_t a0 = 0, a1 = 0;
  if (valid) {
    a0 = A.row_begin(row);
    a1 = A.row_end(row);
  }
  const bool is_long = long_acc != nullptr && a1 - a0 > kLongRowEntries;  // uniform in the group
  unsigned long long p = 0;
  uint32_t mn = kEmpty, mx = 0, lb = 0;
  if (!is_long) span_part<G>(A, B, btab, a0 + sl, a1, p, mn, mx, lb);
#pragma unroll
  for (int o = G / 2; o > 0; o >>= 1) {
    p += __shfl_xor_sync(kFull, p, o);
    mn = min(mn, __shfl_xor_sync(kFull, mn, o));
    mx = max(mx, __shfl_xor_sync(kFull, mx, o));
    lb = max(lb, __shfl_xor_sync(kFull, lb, o));
  }
  int b = -1;
  const bool leader = valid && sl == 0;
  if (leader) {
    if (a1 > a0) atomicMax(&s_maxa, (unsigned)(a1 - a0));
    if (is_long) {
      // list the row and give it its chunk ids (the list holds nnz(A) / 512 + 1
      // rows and the map nnz(A) / 256 + that many chunks, so both always fit)
      const uint32_t nch = (uint32_t)((a1 - a0 + kLongChunk - 1) / kLongChunk);
      const unsigned i = atomicAdd(&ctr->num_long, 1u);
      const unsigned base = i < long_cap ? atomicAdd(&ctr->long_chunks, nch) : 0u;
      if (i < long_cap && (uint64_t)base + nch <= chunk_cap) {
        long_rows[i] = (uint32_t)row;
        LongRowAcc& L = long_acc[i];
        L.prod = 0ull;
        L.lo = kEmpty;
        L.hi = 0u;
        L.maxb = 0u;
        L.done = 0u;
        L.hdone = 0u;
        L.base = base;
        for (int r = 0; r < 64; ++r) L.reg[r] = 0u;
        for (uint32_t c = 0; c < nch; ++c) long_chunk_row[base + c] = i;
      } else {
        raise_status(ctr, DEV_BIN_OVERFLOW, (uint32_t)row);
      }
    } else {
      b = analysis_write(row, a1 - a0, p, mn, mx, lb, prod, lo, hi, anz, maxb, row_nnz, bm_off, pols, row_pol);
      // totals for stats and the workflow decision
      if (p) {
        atomicAdd(&s_tot, p);
        atomicMax(&s_maxp, p > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned)p);
      }
    }
  }
  {
    // per-class sums: shared atomics of the leaders (G = 32: one row per
    // warp), or one per warp and class present in the warp
    const unsigned long long my_anz = (b >= 0) ? (unsigned long long)(a1 - a0) : 0ull;
    const unsigned long long my_p = (b >= 0) ? p : 0ull;
    const uint64_t span = (uint64_t)mx - mn + 1;
    const unsigned long long my_w = (b == SB_BITMAP && span <= kBitmapBits) ? ((span + 63) >> 6) : 0ull;
    if (G == 32) {
      if (b >= 0) {
        atomicAdd(&s_anz[b], my_anz);
        atomicAdd(&s_prod[b], my_p);
        if (my_w) atomicAdd(&s_words, my_w);
      }
    } else {
      unsigned present = __reduce_or_sync(kFull, b >= 0 ? 1u << b : 0u);
      while (present) {
        const int c = __ffs(present) - 1;
        present &= present - 1;
        const unsigned long long sa = warp_sum_u64(b == c ? my_anz : 0ull);
        const unsigned long long sp = warp_sum_u64(b == c ? my_p : 0ull);
        if (lane == 0 && sp) {
          atomicAdd(&s_anz[c], sa);
          atomicAdd(&s_prod[c], sp);
        }
      }
      if (__any_sync(kFull, my_w != 0)) {
        const unsigned long long sw = warp_sum_u64(my_w);
        if (lane == 0 && sw) atomicAdd(&s_words, sw);
      }
    }
  }
  {
    const int bq[1] = {b};
    const uint32_t rq[1] = {(uint32_t)row};
    const int sq[1] = {0};
    block_bin_append<1>(bq, sq, rq, s_cnt, SB_COUNT, 1, nullptr, ctr->sym_count, nullptr, sym_bins, A.rows);
  }
  if (threadIdx.x < SB_COUNT) {
    if (s_anz[threadIdx.x]) atomicAdd(&ctr->sym_anz[threadIdx.x], s_anz[threadIdx.x]);
    if (s_prod[threadIdx.x]) atomicAdd(&ctr->sym_prod[threadIdx.x], s_prod[threadIdx.x]);
  }
  if (threadIdx.x == 32) {
    if (s_words) atomicAdd(&ctr->sym_words, s_words);
    if (s_tot) atomicAdd(&ctr->total_products, s_tot);
    if (s_maxp) atomicMax(&ctr->max_products, s_maxp);
    if (s_maxa) atomicMax(&ctr->max_a_nnz, s_maxa);
  }
}

// Grid of the long-row kernels: 8 blocks of 256 per SM (32 registers), so
// enough chunks are in flight to hide their atomics and fences.
constexpr unsigned kLongGrid = 8 * 148;

// The analysis of the listed long rows: the warps of the grid stride over the
// chunk ids, merge each chunk's partial sums into its row's accumulator with
// atomics, and the warp that finishes a row's last chunk writes the row's
// results, appends it to its class and adds its totals.
template <typename RP>
__global__ void __launch_bounds__(256, 8) k_analysis_long(Csr<RP> A, Csr<RP> B, uint32_t* __restrict__ prod,
                                                       uint32_t* __restrict__ lo, uint32_t* __restrict__ hi,
                                                       uint32_t* __restrict__ anz, uint32_t* __restrict__ maxb,
                                                       uint32_t* __restrict__ row_nnz,
                                                       uint64_t* __restrict__ bm_off, uint32_t* __restrict__ sym_bins,
                                                       DevCounters* __restrict__ ctr, SymPolicySet pols,
                                                       const uint8_t* __restrict__ row_pol,
                                                       const uint32_t* __restrict__ long_rows,
                                                       LongRowAcc* __restrict__ long_acc, uint32_t long_cap,
                                                       const uint32_t* __restrict__ long_chunk_row,
                                                       uint32_t chunk_cap, const uint4* __restrict__ btab) {
  const uint32_t total = min(ctr->long_chunks, chunk_cap);
  const uint32_t nl = min(ctr->num_long, long_cap);
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < total; c += nw) {
    const uint32_t i = long_chunk_row[c];
    if (i >= nl) continue;  // (a row that did not fit the map: flagged by the analysis)
    LongRowAcc& L = long_acc[i];
    const uint32_t row = long_rows[i];
    const uint64_t a0 = A.row_begin(row), a1 = A.row_end(row);
    const uint32_t nch = (uint32_t)((a1 - a0 + kLongChunk - 1) / kLongChunk);
    if (c - L.base >= nch) continue;
    const uint64_t c0 = a0 + (uint64_t)(c - L.base) * kLongChunk;
    unsigned long long p = 0;
    uint32_t mn = kEmpty, mx = 0, lb = 0;
    span_part<32>(A, B, btab, c0 + lane, min(a1, c0 + kLongChunk), p, mn, mx, lb);
    p = warp_sum_u64(p);
    mn = __reduce_min_sync(kFull, mn);
    mx = __reduce_max_sync(kFull, mx);
    lb = __reduce_max_sync(kFull, lb);
    if (lane == 0) {
      if (p) atomicAdd(&L.prod, p);
      atomicMin(&L.lo, mn);
      atomicMax(&L.hi, mx);
      atomicMax(&L.maxb, lb);
      __threadfence();
      if (atomicAdd(&L.done, 1u) == nch - 1) {
        __threadfence();
        const unsigned long long tp = atomicAdd(&L.prod, 0ull);
        const uint32_t tmn = atomicOr(&L.lo, 0u), tmx = atomicOr(&L.hi, 0u), tlb = atomicOr(&L.maxb, 0u);
        const int b = analysis_write(row, a1 - a0, tp, tmn, tmx, tlb, prod, lo, hi, anz, maxb, row_nnz, bm_off,
                                     pols, row_pol);
        if (b >= 0) {
          const unsigned pos = atomicAdd(&ctr->sym_count[b], 1u);
          sym_bins[(uint64_t)b * A.rows + pos] = row;
          atomicAdd(&ctr->sym_anz[b], (unsigned long long)(a1 - a0));
          atomicAdd(&ctr->sym_prod[b], tp);
          const uint64_t span = (uint64_t)tmx - tmn + 1;
          if (b == SB_BITMAP && span <= kBitmapBits) atomicAdd(&ctr->sym_words, (unsigned long long)((span + 63) >> 6));
          atomicAdd(&ctr->total_products, tp);
          atomicMax(&ctr->max_products, tp > 0xFFFFFFFFull ? 0xFFFFFFFFu : (unsigned)tp);
        }
      }
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- ESC (<= 32K products)
// Expand-sort-compress in the registers of one warp: a row's (<= 32K)
// products are listed, held K per lane, bitonic-sorted by column across the
// warp into blocked order (lane l ends with sorted elements l*K .. l*K+K-1;
// register swaps for partners in the same lane, shuffles for the others), then
// equal columns are merged by suffix sums inside each lane and one segmented
// scan across lanes. The output is the row, sorted, with no shared-memory
// table and no block barrier. The symbolic variant sorts keys only and counts
// run heads.

// Lists the (<= CAP) products of `row` in warp order: src[i] = index into B,
// aidx[i] = index into A. Returns the product count (> CAP means overflow).
template <int CAP, typename RP>
__device__ __forceinline__ uint32_t gather_products(const Csr<RP>& A, const Csr<RP>& B, uint32_t row,
                                                    uint64_t* src, uint64_t* aidx) {
  const int lane = threadIdx.x & 31;
  const uint64_t a0 = A.row_begin(row), a1 = A.row_end(row);
  uint32_t base = 0;
  for (uint64_t k0 = a0; k0 < a1 && base <= CAP; k0 += 32) {
    const uint64_t k = k0 + lane;
    uint64_t b0 = 0;
    uint32_t len = 0;
    if (k < a1) {
      const uint32_t j = A.col[k];
      b0 = B.row_begin(j);
      const uint64_t l = B.row_end(j) - b0;
      len = l > CAP + 1 ? CAP + 1u : (uint32_t)l;
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += y;
    }
    const uint32_t excl = base + incl - len;
    for (uint32_t t = 0; t < len && excl + t < CAP; ++t) {
      src[excl + t] = b0 + t;
      if (aidx) aidx[excl + t] = k;
    }
    base += __shfl_sync(kFull, incl, 31);
  }
  __syncwarp();
  return base;
}

// Bitonic sort of the warp's 32K (key, value) elements into blocked order:
// afterwards lane l holds sorted elements l*K .. l*K + K - 1 in registers
// 0 .. K - 1 (element L = lane*K + e). Stages whose partner element lies in
// the same lane (j < K) swap registers; the others exchange one register with
// lane ^ (j / K). Against the strided layout this moves log2(K) stages of
// every merge into registers and lets the merge that follows scan each lane's
// run locally before one scan across lanes.
template <int K, bool VALS>
__device__ __forceinline__ void warp_sort_blocked(uint32_t (&key)[K], double (&val)[K]) {
  const int lane = threadIdx.x & 31;
  constexpr int N = 32 * K;
#pragma unroll
  for (int k = 2; k <= N; k <<= 1) {
#pragma unroll
    for (int j = k >> 1; j > 0; j >>= 1) {
      if (j < K) {
#pragma unroll
        for (int e = 0; e < K; ++e) {
          if ((e & j) == 0) {
            const int e2 = e | j;
            const bool asc = ((lane * K + e) & k) == 0;
            if (!VALS) {
              const uint32_t a = key[e], b = key[e2];
              key[e] = asc ? min(a, b) : max(a, b);
              key[e2] = asc ? max(a, b) : min(a, b);
            } else if ((key[e] > key[e2]) == asc) {
              const uint32_t tk = key[e];
              key[e] = key[e2];
              key[e2] = tk;
              const double tv = val[e];
              val[e] = val[e2];
              val[e2] = tv;
            }
          }
        }
      } else {
        const int lj = j / K;
        const bool asc = ((lane * K) & k) == 0;  // k > j >= K: the register index does not reach bit k
        const bool low = (lane & lj) == 0;
        const bool keep_min = low == asc;  // this lane keeps the smaller key of the pair
#pragma unroll
        for (int e = 0; e < K; ++e) {
          const uint32_t ok = __shfl_xor_sync(kFull, key[e], lj);
          if (!VALS) {
            // keys only: one predicated min/max per element (equal keys are
            // interchangeable)
            key[e] = keep_min ? min(key[e], ok) : max(key[e], ok);
          } else {
            // with values the strict test keeps both lanes of a tie on their
            // own element
            const double ov = __shfl_xor_sync(kFull, val[e], lj);
            if (keep_min ? (ok < key[e]) : (ok > key[e])) {
              key[e] = ok;
              val[e] = ov;
            }
          }
        }
      }
    }
  }
}

// Run heads of blocked-sorted keys (kEmpty last): head[e] if the key is real
// and differs from the element before it. Returns the warp's number of runs;
// `before` = runs that start in lanes below this one.
template <int K>
__device__ __forceinline__ uint32_t warp_heads_blocked(const uint32_t (&key)[K], bool (&head)[K],
                                                       uint32_t& before) {
  const int lane = threadIdx.x & 31;
  const uint32_t prev_last = __shfl_up_sync(kFull, key[K - 1], 1);
  const unsigned lt = lanemask_lt();
  uint32_t n = 0;
  before = 0;
#pragma unroll
  for (int e = 0; e < K; ++e) {
    const uint32_t prev = e > 0 ? key[e - 1] : prev_last;
    head[e] = key[e] != kEmpty && ((e == 0 && lane == 0) || prev != key[e]);
    const unsigned hb = __ballot_sync(kFull, head[e]);
    n += __popc(hb);
    before += __popc(hb & lt);
  }
  return n;
}

// Segmented sums of blocked-sorted (key, val): afterwards the first element
// of every run of equal keys holds the run's sum. Suffix sums inside each
// lane, then one segmented suffix scan across lanes of each lane's first-run
// sum (keys are sorted, so a lane whose first key equals a later lane's first
// key holds that key only, and key equality alone delimits the segments),
// then the lane's last run takes the sum of its continuation in the lanes
// above.
template <int K>
__device__ __forceinline__ void warp_merge_blocked(const uint32_t (&key)[K], double (&val)[K]) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int e = K - 2; e >= 0; --e)
    if (key[e] == key[e + 1]) val[e] += val[e + 1];
  const uint32_t kf = key[0];
  double acc = val[0];
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t ck = __shfl_down_sync(kFull, kf, d);
    const double cv = __shfl_down_sync(kFull, acc, d);
    if (lane + d < 32 && ck == kf) acc += cv;
  }
  const uint32_t nk = __shfl_down_sync(kFull, kf, 1);
  const double nacc = __shfl_down_sync(kFull, acc, 1);
  const uint32_t kl = key[K - 1];
  if (lane < 31 && nk == kl) {
#pragma unroll
    for (int e = 0; e < K; ++e)
      if (key[e] == kl) val[e] += nacc;
  }
}

template <typename RP, int K>
__global__ void __launch_bounds__(256) k_sym_esc(Csr<RP> A, Csr<RP> B, RowQueue q, DevCounters* __restrict__ ctr,
                                                 uint32_t* __restrict__ row_nnz) {
  constexpr int CAP = 32 * K;
  __shared__ uint64_t s_src[8][CAP];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t count = *q.count;
  const uint32_t* list = q.rows;
  for (uint64_t idx = (uint64_t)blockIdx.x * 8 + warp; idx < count; idx += (uint64_t)gridDim.x * 8) {
    const uint32_t row = list[idx];
    const uint32_t np = gather_products<CAP>(A, B, row, s_src[warp], nullptr);
    if (np > CAP && lane == 0) raise_status(ctr, DEV_BIN_OVERFLOW, row);
    uint32_t key[K];
    double val[K];
#pragma unroll
    for (int e = 0; e < K; ++e) {
      const uint32_t i = (uint32_t)(e << 5) | lane;
      key[e] = i < np && i < (uint32_t)CAP ? B.col[s_src[warp][i]] : kEmpty;
      val[e] = 0.0;
    }
    uint32_t n;
    if (K == 1) {
      // one product per lane: distinct count without sorting
      const unsigned peers = __match_any_sync(kFull, key[0]);
      const bool first = key[0] != kEmpty && (__ffs(peers) - 1 == lane);
      n = __popc(__ballot_sync(kFull, first));
    } else {
      warp_sort_blocked<K, false>(key, val);
      bool head[K];
      uint32_t before;
      n = warp_heads_blocked<K>(key, head, before);
    }
    if (lane == 0) row_nnz[row] = n;
    __syncwarp();
  }
}

template <typename RP, int K>
__global__ void __launch_bounds__(256) k_num_esc(Csr<RP> A, Csr<RP> B, RowQueue q, OutSpec o,
                                                 DevCounters* __restrict__ ctr, uint32_t* __restrict__ c_col,
                                                 double* __restrict__ c_val) {
  constexpr int CAP = 32 * K;
  constexpr int LOGN = K == 1 ? 5 : (K == 2 ? 6 : 7);  // bits of a product's position in the warp
  __shared__ uint64_t s_src[8][CAP];
  __shared__ uint64_t s_aidx[8][CAP];
  __shared__ double s_pval[8][CAP];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t count = *q.count;
  const uint32_t* list = q.rows;
  for (uint64_t idx = (uint64_t)blockIdx.x * 8 + warp; idx < count; idx += (uint64_t)gridDim.x * 8) {
    const uint32_t row = list[idx];
    const uint32_t np = gather_products<CAP>(A, B, row, s_src[warp], s_aidx[warp]);
    if (np > CAP && lane == 0) raise_status(ctr, DEV_BIN_OVERFLOW, row);
    uint32_t key[K];
    double val[K];
#pragma unroll
    for (int e = 0; e < K; ++e) {
      const uint32_t i = (uint32_t)(e << 5) | lane;
      key[e] = kEmpty;
      val[e] = 0.0;
      if (i < np && i < (uint32_t)CAP) {
        const uint64_t sidx = s_src[warp][i];
        key[e] = B.col[sidx];
        val[e] = A.val[s_aidx[warp][i]] * B.val[sidx];
      }
    }
    // when the row's columns span less than 2^(32 - LOGN), the sort runs on
    // one 32-bit word per product, (column - lo) << LOGN | position, and the
    // values are fetched from shared memory by position afterwards: a third of
    // the shuffles of sorting (column, value) pairs
    uint32_t kmin = kEmpty, kmax = 0;
#pragma unroll
    for (int e = 0; e < K; ++e) {
      kmin = min(kmin, key[e]);
      if (key[e] != kEmpty) kmax = max(kmax, key[e]);
    }
    kmin = __reduce_min_sync(kFull, kmin);
    kmax = __reduce_max_sync(kFull, kmax);
    if (kmin == kEmpty || kmax - kmin < (1u << (32 - LOGN)) - 1u) {
      uint32_t pk[K];
#pragma unroll
      for (int e = 0; e < K; ++e) {
        const uint32_t pos = (uint32_t)(e << 5) | lane;
        s_pval[warp][pos] = val[e];
        pk[e] = key[e] == kEmpty ? kEmpty : ((key[e] - kmin) << LOGN) | pos;
      }
      __syncwarp();
      warp_sort_blocked<K, false>(pk, val);
#pragma unroll
      for (int e = 0; e < K; ++e) {
        if (pk[e] == kEmpty) {
          key[e] = kEmpty;
          val[e] = 0.0;
        } else {
          key[e] = (pk[e] >> LOGN) + kmin;
          val[e] = s_pval[warp][pk[e] & (CAP - 1)];
        }
      }
      __syncwarp();
    } else {
      warp_sort_blocked<K, true>(key, val);
    }
    // lane l now holds sorted elements l*K .. l*K + K - 1: run sums, heads
    warp_merge_blocked<K>(key, val);
    bool head[K];
    uint32_t before;
    const uint32_t n = warp_heads_blocked<K>(key, head, before);
    const uint32_t cap = o.cap[row];
    int accept = 0;
    if (lane == 0) accept = out_accept(o, ctr, row, n, cap);
    accept = __shfl_sync(kFull, accept, 0);
    const uint32_t lim = accept ? min(n, cap) : 0u;
    const uint64_t off = o.off[row];
#pragma unroll
    for (int e = 0; e < K; ++e) {
      if (head[e] && before < lim) {
        c_col[off + before] = key[e];
        c_val[off + before] = val[e];
      }
      before += head[e] ? 1u : 0u;
    }
    __syncwarp();
  }
}

// ---------------------------------------------------------------- fused ultra-sparse multiply
// One launch for an input whose every row has at most 256 products (the
// ultra-sparse workflow's inputs): each warp merges one row of C in registers
// (the ESC classes' register sort and segmented sums; rows of 129-256 products
// sort one packed 64-bit key per product in shared memory first) and stages
// it in shared memory; a block's 8 rows form a tile whose output offset comes
// from a decoupled look-back over the preceding tiles' published counts
// (tile ids are taken in launch order, so every tile waits only on tiles that
// already run); then the rows are written at their final place in C and the
// row pointers with them. No temporary output, no separate scan, no copy.
// The look-back's wait is bounded: after kUspSpinLimit polls the block flags
// DEV_SCAN_TIMEOUT and continues with a smaller prefix, which keeps every
// write inside C's capacity (the sum of the products).
constexpr int kUspWarps = 8;     // rows per tile, one per warp
constexpr int kUspCap = 256;     // products per row
constexpr unsigned long long kTileAgg = 1ull << 62, kTileIncl = 2ull << 62, kTileVal = (1ull << 62) - 1;
constexpr int kUspSpinLimit = 1 << 20;

struct UspSmem {
  uint64_t src[kUspWarps][kUspCap];   // gathered B indices; packed sort keys of the largest rows
  uint64_t aidx[kUspWarps][kUspCap];  // gathered A indices
  uint32_t okey[kUspWarps][kUspCap];  // merged row: column ids
  double oval[kUspWarps][kUspCap];    // merged row: values (scratch of the packed sorts before)
  uint32_t cnt[kUspWarps];
  uint32_t np[kUspWarps];
  unsigned long long prefix;
  uint32_t tile;
};

// Segmented sums of the blocked-sorted (key, val) of one row (kEmpty keys
// last), then the distinct columns and their sums written compactly to
// okey/oval. Returns the row's output count. Warp-collective.
template <int K>
__device__ __forceinline__ uint32_t usp_merge_stage(uint32_t (&key)[K], double (&val)[K], uint32_t* okey,
                                                    double* oval) {
  warp_merge_blocked<K>(key, val);
  bool head[K];
  uint32_t before;
  const uint32_t n = warp_heads_blocked<K>(key, head, before);
#pragma unroll
  for (int e = 0; e < K; ++e) {
    if (head[e]) {
      okey[before] = key[e];
      oval[before] = val[e];
      ++before;
    }
  }
  __syncwarp();
  return n;
}

// Register ESC of a row of np <= 32K products gathered in src/aidx; the
// merged row goes to okey/oval. Returns the output count.
template <int K, typename RP>
__device__ __forceinline__ uint32_t usp_row_regs(const Csr<RP>& A, const Csr<RP>& B, uint32_t np,
                                                 const uint64_t* src, const uint64_t* aidx, uint32_t* okey,
                                                 double* oval) {
  constexpr int LOGN = K == 1 ? 5 : (K == 2 ? 6 : 7);
  const int lane = threadIdx.x & 31;
  uint32_t key[K];
  double val[K];
#pragma unroll
  for (int e = 0; e < K; ++e) {
    const uint32_t i = (uint32_t)(e << 5) | lane;
    key[e] = kEmpty;
    val[e] = 0.0;
    if (i < np) {
      const uint64_t sidx = src[i];
      key[e] = B.col[sidx];
      val[e] = A.val[aidx[i]] * B.val[sidx];
    }
  }
  uint32_t kmin = kEmpty, kmax = 0;
#pragma unroll
  for (int e = 0; e < K; ++e) {
    kmin = min(kmin, key[e]);
    if (key[e] != kEmpty) kmax = max(kmax, key[e]);
  }
  kmin = __reduce_min_sync(kFull, kmin);
  kmax = __reduce_max_sync(kFull, kmax);
  if (kmin == kEmpty || kmax - kmin < (1u << (32 - LOGN)) - 1u) {
    uint32_t pk[K];
#pragma unroll
    for (int e = 0; e < K; ++e) {
      const uint32_t pos = (uint32_t)(e << 5) | lane;
      oval[pos] = val[e];
      pk[e] = key[e] == kEmpty ? kEmpty : ((key[e] - kmin) << LOGN) | pos;
    }
    __syncwarp();
    warp_sort_blocked<K, false>(pk, val);
#pragma unroll
    for (int e = 0; e < K; ++e) {
      if (pk[e] == kEmpty) {
        key[e] = kEmpty;
        val[e] = 0.0;
      } else {
        key[e] = (pk[e] >> LOGN) + kmin;
        val[e] = oval[pk[e] & (32 * K - 1)];
      }
    }
    __syncwarp();
  } else {
    warp_sort_blocked<K, true>(key, val);
  }
  return usp_merge_stage<K>(key, val, okey, oval);
}

// A row of 129-256 products: one 64-bit key (column << 8 | position) per
// product bitonic-sorted in shared memory, then merged in registers.
template <typename RP>
__device__ __forceinline__ uint32_t usp_row_smem(const Csr<RP>& A, const Csr<RP>& B, uint32_t np, uint64_t* src,
                                                 const uint64_t* aidx, uint32_t* okey, double* oval) {
  const int lane = threadIdx.x & 31;
  for (uint32_t i = lane; i < (uint32_t)kUspCap; i += 32) {
    uint64_t kk = ~0ull;
    if (i < np) {
      const uint64_t sidx = src[i];
      kk = ((uint64_t)B.col[sidx] << 8) | i;
      oval[i] = A.val[aidx[i]] * B.val[sidx];
    }
    src[i] = kk;
  }
  __syncwarp();
  for (int k = 2; k <= kUspCap; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int t = lane; t < kUspCap / 2; t += 32) {
        const int i = ((t & ~(j - 1)) << 1) | (t & (j - 1));
        const int l = i + j;
        const bool asc = (i & k) == 0;
        const uint64_t a = src[i], b = src[l];
        if ((a > b) == asc) {
          src[i] = b;
          src[l] = a;
        }
      }
      __syncwarp();
    }
  }
  uint32_t key[8];
  double val[8];
#pragma unroll
  for (int e = 0; e < 8; ++e) {
    const uint64_t kk = src[(lane << 3) | e];  // blocked order: lane l takes sorted elements 8l .. 8l + 7
    key[e] = kk == ~0ull ? kEmpty : (uint32_t)(kk >> 8);
    val[e] = kk == ~0ull ? 0.0 : oval[kk & 255];
  }
  __syncwarp();
  return usp_merge_stage<8>(key, val, okey, oval);
}

__device__ __forceinline__ unsigned long long ld_volatile_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.volatile.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

template <typename RP>
__global__ void __launch_bounds__(256) k_usp_fused(Csr<RP> A, Csr<RP> B, unsigned long long* __restrict__ tiles,
                                                   DevCounters* __restrict__ ctr, uint64_t cap,
                                                   uint64_t* __restrict__ rowptr64, uint32_t* __restrict__ rowptr32,
                                                   uint32_t* __restrict__ c_col, double* __restrict__ c_val) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  UspSmem& S = *reinterpret_cast<UspSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  if (tid == 0) S.tile = atomicAdd(&ctr->usp_tile, 1u);
  __syncthreads();
  const uint32_t t = S.tile;
  const uint64_t row = (uint64_t)t * kUspWarps + warp;
  uint32_t n = 0, np_row = 0;
  if (row < A.rows) {
    const uint32_t np = gather_products<kUspCap>(A, B, (uint32_t)row, S.src[warp], S.aidx[warp]);
    np_row = np;
    if (np > (uint32_t)kUspCap) {
      if (lane == 0) raise_status(ctr, DEV_BIN_OVERFLOW, (uint32_t)row);
    } else if (np > 128) {
      n = usp_row_smem(A, B, np, S.src[warp], S.aidx[warp], S.okey[warp], S.oval[warp]);
    } else if (np > 64) {
      n = usp_row_regs<4>(A, B, np, S.src[warp], S.aidx[warp], S.okey[warp], S.oval[warp]);
    } else if (np > 32) {
      n = usp_row_regs<2>(A, B, np, S.src[warp], S.aidx[warp], S.okey[warp], S.oval[warp]);
    } else if (np > 0) {
      n = usp_row_regs<1>(A, B, np, S.src[warp], S.aidx[warp], S.okey[warp], S.oval[warp]);
    }
  }
  if (lane == 0) {
    S.cnt[warp] = n;
    S.np[warp] = np_row;
  }
  __syncthreads();
  // warp 0: the tile's aggregate, then a look-back over the preceding tiles,
  // 32 tiles per read: the nearest tile with an inclusive prefix ends it,
  // the aggregates of the tiles after it are added; a tile that has not
  // published yet is polled (bounded)
  if (warp == 0) {
    unsigned long long agg = 0;
    for (int w = 0; w < kUspWarps; ++w) agg += S.cnt[w];
    unsigned long long prefix = 0;
    if (t > 0) {
      if (lane == 0) atomicExch(&tiles[t], kTileAgg | agg);
      int64_t top = (int64_t)t - 1;  // nearest tile not yet summed
      int spins = 0;
      while (top >= 0) {
        const int64_t j = top - lane;
        const unsigned long long v = j >= 0 ? ld_volatile_u64(&tiles[j]) : kTileIncl;  // before tile 0: prefix 0
        const unsigned ready = __ballot_sync(kFull, (v & (kTileAgg | kTileIncl)) != 0);
        const unsigned incl = __ballot_sync(kFull, (v & kTileIncl) != 0);
        // lanes up to the nearest inclusive one must all have published
        const unsigned need = incl ? ((incl & (0u - incl)) << 1) - 1u : kFull;
        if ((ready & need) != need) {
          if (++spins > kUspSpinLimit) {
            if (lane == 0) raise_status(ctr, DEV_SCAN_TIMEOUT, t);
            break;
          }
          __nanosleep(32);
          continue;
        }
        const unsigned long long part = (need >> lane) & 1u ? (v & kTileVal) : 0ull;
        prefix += warp_sum_u64(part);
        if (incl) break;
        top -= 32;
      }
    }
    if (lane == 0) {
      atomicExch(&tiles[t], kTileIncl | (prefix + agg));
      S.prefix = prefix;
      const uint64_t last_row = (uint64_t)t * kUspWarps + kUspWarps;
      if (last_row >= A.rows) {
        rowptr64[A.rows] = prefix + agg;
        if (rowptr32) rowptr32[A.rows] = (uint32_t)(prefix + agg);
        ctr->total_nnz = prefix + agg;
      }
      // class accounting of the tile's rows (stats): ESC1/2/4 by products,
      // rows of 129-256 products under the small-hash class
      for (int w = 0; w < kUspWarps; ++w) {
        if (S.cnt[w] == 0) continue;
        const uint32_t q = S.np[w];
        const int c = q <= 32 ? NB_ESC1 : (q <= 64 ? NB_ESC2 : (q <= 128 ? NB_ESC4 : NB_HASH_S));
        atomicAdd(&ctr->num_count[c], 1u);
        atomicAdd(&ctr->num_nnz[c], (unsigned long long)S.cnt[w]);
        atomicAdd(&ctr->num_prod[c], (unsigned long long)q);
      }
    }
  }
  __syncthreads();
  if (row < A.rows) {
    uint64_t off = S.prefix;
    for (int w = 0; w < warp; ++w) off += S.cnt[w];
    if (lane == 0) {
      rowptr64[row] = off;
      if (rowptr32) rowptr32[row] = (uint32_t)off;
    }
    for (uint32_t j = lane; j < n; j += 32) {
      if (off + j < cap) {
        c_col[off + j] = S.okey[warp][j];
        c_val[off + j] = S.oval[warp][j];
      }
    }
  }
}

// ---------------------------------------------------------------- product enumeration
// Block-wide, load-balanced enumeration of the products of one row of A.
//
// The row's A entries are taken in chunks of NT. Each chunk is compacted to its
// non-empty B rows (one packed block scan gives both the compacted rank and the
// running product offset), so the chunk's products form one contiguous range
// [0, total). Every warp takes an equal contiguous slice of that range, 32
// products per step, lane l handling product base + l. The owning B row of each
// lane is found without searching: each lane of a 32-row window publishes the
// bit (incl - base - 1) when its row ends inside the step, one __reduce_or_sync
// collects the bits, and popc(bits below the lane) is the lane's row offset.
// UNROLL steps are resolved first and their loads issued together, so every
// thread keeps UNROLL gathers of B in flight whatever the B-row lengths are.
template <int NT>
struct EnumSmem {
  unsigned long long incl[NT];   // inclusive product offset of each non-empty row
  unsigned long long bbase[NT];  // B index of the row start minus its product offset
  double av[NT];                 // A value of the row
  unsigned long long scan[33];
  unsigned long long total;      // products of the loaded chunk
  uint32_t nrows;                // non-empty rows of the loaded chunk
};

#ifndef OCEAN_UNROLL
#define OCEAN_UNROLL 4
#endif
constexpr int kUnroll = OCEAN_UNROLL;  // gathers in flight per thread in the product enumeration

// Packs one B-row range per thread (start bs, length len, A value av) into E,
// compacted to the non-empty ranges.
template <int NT, bool VALS>
__device__ __forceinline__ void block_pack_chunk(unsigned long long bs, unsigned long long len, double av,
                                                 EnumSmem<NT>& E) {
  const int tid = threadIdx.x;
  // packed scan: high 16 bits count non-empty rows, low 48 bits sum products
  const unsigned long long packed = len ? ((1ull << 48) | len) : 0ull;
  unsigned long long tot;
  const unsigned long long ex = block_excl_scan<NT, unsigned long long>(packed, E.scan, &tot);
  constexpr unsigned long long kLow = (1ull << 48) - 1;
  if (len) {
    const uint32_t r = (uint32_t)(ex >> 48);
    const unsigned long long off = ex & kLow;
    E.incl[r] = off + len;
    E.bbase[r] = bs - off;
    if (VALS) E.av[r] = av;
  }
  if (tid == 0) {
    E.nrows = (uint32_t)(tot >> 48);
    E.total = tot & kLow;
  }
  __syncthreads();
}

// Loads A entries [c0, min(c0 + NT, a1)) into E (compacted to non-empty B rows).
template <int NT, bool VALS, typename RP>
__device__ __forceinline__ void block_load_chunk(const Csr<RP>& A, const Csr<RP>& B, uint64_t c0, uint64_t a1,
                                                 EnumSmem<NT>& E) {
  const uint64_t k = c0 + threadIdx.x;
  unsigned long long len = 0, bs = 0;
  double av = 0.0;
  if (k < a1) {
    const uint32_t j = A.col[k];
    bs = B.row_begin(j);
    len = B.row_end(j) - bs;
    if (VALS) av = A.val[k];
  }
  block_pack_chunk<NT, VALS>(bs, len, av, E);
}

// Enumerates the products of the chunk held in E. `op(col, value, ok)` is
// called by all 32 lanes of a warp together (ok = false for idle lanes).
// Fast path: while the warp's next kUnroll steps all lie inside one B row, the
// lanes issue plain strided gathers of that row (no owner search).
template <int NT, bool VALS, typename RP, typename Op>
__device__ __forceinline__ void block_run_chunk(const Csr<RP>& B, EnumSmem<NT>& E, Op&& op) {
  constexpr int NW = NT / 32;
  constexpr unsigned long long kSpan = 32ull * kUnroll;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const uint32_t nrows = E.nrows;
  const unsigned long long total = E.total;
  const unsigned long long slice = (((total + NW - 1) / NW) + 31) & ~31ull;
  unsigned long long base = (unsigned long long)warp * slice;
  const unsigned long long end = min(base + slice, total);
  if (base < end) {
    // owner row of product `base`: first row whose inclusive offset exceeds it
    uint32_t lo = 0, hi = nrows;
    while (lo < hi) {
      const uint32_t mid = (lo + hi) >> 1;
      if (E.incl[mid] <= base) lo = mid + 1; else hi = mid;
    }
    uint32_t r_cur = lo;
    const unsigned lt = lanemask_lt();
    while (base < end) {
      while (E.incl[r_cur] <= base) ++r_cur;
      if (E.incl[r_cur] >= base + kSpan && end >= base + kSpan) {
        const unsigned long long b0 = E.bbase[r_cur] + base + lane;
        const double av = VALS ? E.av[r_cur] : 0.0;
        uint32_t c[kUnroll];
        double bv[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
          c[u] = B.col[b0 + 32 * u];
          if (VALS) bv[u] = B.val[b0 + 32 * u];
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) op(c[u], VALS ? av * bv[u] : 0.0, true);
        base += kSpan;
        continue;
      }
      unsigned long long bi[kUnroll];
      uint32_t rr[kUnroll];
      bool ok[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        const unsigned long long sb = base + (unsigned long long)u * 32;
        const uint32_t w = r_cur + lane;
        const unsigned long long inc = w < nrows ? E.incl[w] : ~0ull;
        const unsigned long long d = inc - sb - 1;
        const unsigned bit = d < 32 ? (1u << d) : 0u;
        const unsigned m = __reduce_or_sync(kFull, bit);
        rr[u] = r_cur + __popc(m & lt);
        ok[u] = sb + lane < end;
        bi[u] = ok[u] ? E.bbase[rr[u]] + sb + lane : 0ull;
        r_cur += __popc(m);
      }
      uint32_t c[kUnroll];
      double bv[kUnroll];
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) {
        c[u] = kEmpty;
        bv[u] = 0.0;
        if (ok[u]) {
          c[u] = B.col[bi[u]];
          if (VALS) bv[u] = B.val[bi[u]];
        }
      }
#pragma unroll
      for (int u = 0; u < kUnroll; ++u) op(c[u], (VALS && ok[u]) ? E.av[rr[u]] * bv[u] : 0.0, ok[u]);
      base += kSpan;
    }
  }
  __syncthreads();
}

// Enumerates every product of A entries [a0, a1) (all chunks).
template <int NT, bool VALS, typename RP, typename Op>
__device__ __forceinline__ void block_for_each_product(const Csr<RP>& A, const Csr<RP>& B, uint64_t a0,
                                                       uint64_t a1, EnumSmem<NT>& E, Op&& op) {
  for (uint64_t c0 = a0; c0 < a1; c0 += NT) {
    block_load_chunk<NT, VALS>(A, B, c0, a1, E);
    block_run_chunk<NT, VALS>(B, E, op);
  }
}

// Sets the bit of column c of the window [w0, w1) (`single`: the window
// holds the whole row, no range test). The word is read first and only
// written by an atomic when the bit is still clear, so hot columns that are
// already marked cost one shared-memory load.
__device__ __forceinline__ void mark_bit(unsigned long long* bits, uint32_t c, bool ok, bool single, uint64_t w0,
                                         uint64_t w1) {
  if (ok && (single || (c >= w0 && c < w1))) {
    const uint32_t d = (uint32_t)(c - w0);
    // through a 32-bit view of the (little-endian) 64-bit words: 32-bit
    // shared-memory atomics are the fast ones (R-MAT 2^20 symbolic bitmap
    // 76.5 -> 34.4 ms against 64-bit atomicOr)
    unsigned int* b32 = reinterpret_cast<unsigned int*>(bits);
    const unsigned int m = 1u << (d & 31);
    if (!(b32[d >> 5] & m)) atomicOr(&b32[d >> 5], m);
  }
}

// ---------------------------------------------------------------- hash accumulators
// Symbolic: one block per row, open-addressing set of column ids in shared memory
// (linear probing, bounded by the table size).
template <int NT, int LOG2T>
struct SymHashSmem {
  uint32_t keys[1 << LOG2T];
  EnumSmem<NT> e;
  unsigned long long red[33];
  uint32_t s_idx;
};

template <typename RP, int NT, int LOG2T>
__global__ void __launch_bounds__(NT) k_sym_hash(Csr<RP> A, Csr<RP> B, RowQueue q, DevCounters* __restrict__ ctr,
                                                 const uint32_t* __restrict__ prod, const uint32_t* __restrict__ lo,
                                                 const uint32_t* __restrict__ hi, uint32_t* __restrict__ row_nnz) {
  constexpr int T = 1 << LOG2T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  SymHashSmem<NT, LOG2T>& S = *reinterpret_cast<SymHashSmem<NT, LOG2T>*>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < T; i += NT) S.keys[i] = kEmpty;
  const uint32_t count = *q.count;
  const uint32_t* list = q.rows;
  for (;;) {
    if (tid == 0) S.s_idx = atomicAdd(q.cursor, 1u);
    __syncthreads();
    const uint32_t idx = S.s_idx;
    if (idx >= count) break;
    const uint32_t row = list[idx];
    // a row whose column span fits the table addresses it directly: slot = column - lo
    const uint32_t rlo = lo[row];
    const bool direct = hi[row] - rlo < (uint32_t)T;
    unsigned cnt = 0;
    bool full = false;
    block_for_each_product<NT, false>(A, B, A.row_begin(row), A.row_end(row), S.e, [&](uint32_t c, double, bool ok) {
      if (!ok) return;
      uint32_t h = direct ? c - rlo : hash_slot(c, LOG2T);
      int probe = 0;
      for (; probe < T; ++probe) {
        const uint32_t cur = S.keys[h];
        if (cur == c) break;
        if (cur == kEmpty) {
          const uint32_t prev = atomicCAS(&S.keys[h], kEmpty, c);
          if (prev == kEmpty) {
            ++cnt;
            break;
          }
          if (prev == c) break;
        }
        h = (h + 1) & (T - 1);
      }
      full |= probe == T;
    });
    if (full) raise_status(ctr, DEV_TABLE_FULL, row);
    const unsigned long long total = block_sum_u64<NT>(cnt, S.red);
    if (tid == 0) row_nnz[row] = (uint32_t)total;
    for (int i = tid; i < T; i += NT) S.keys[i] = kEmpty;
  }
}

// Numeric: hash-accumulate FP64 values in shared memory, then write the row in
// column order directly into C: rows whose span fits the table were addressed
// directly and are compacted in slot order; the others are radix-sorted on
// packed (column offset, dense index) words, or, when the span is too wide for
// the packing, bitonic-sorted as (column << 32 | slot) keys.
template <int NT, int LOG2T>
struct NumHashSmem {
  double vals[1 << LOG2T];
  uint32_t keys[1 << LOG2T];  // reused as (1 << LOG2T) / 2 sort keys of 64 bits, or two radix buffers
  EnumSmem<NT> e;  // after the products: radix digit counts and dense-to-slot map
  uint32_t s_idx, s_n, s_acc;
};

template <typename RP, int NT, int LOG2T>
__global__ void __launch_bounds__(NT) k_num_hash(Csr<RP> A, Csr<RP> B, RowQueue q, OutSpec o,
                                                 DevCounters* __restrict__ ctr, const uint32_t* __restrict__ prod,
                                                 const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi,
                                                 uint32_t* __restrict__ c_col, double* __restrict__ c_val) {
  constexpr int T = 1 << LOG2T;
  constexpr int PER = T / NT;
  constexpr int CAP = T / 2;  // sort capacity (entries) in the reused key area
  extern __shared__ __align__(16) unsigned char smem_raw[];
  NumHashSmem<NT, LOG2T>& S = *reinterpret_cast<NumHashSmem<NT, LOG2T>*>(smem_raw);
  unsigned long long* sortbuf = reinterpret_cast<unsigned long long*>(S.keys);
  const int tid = threadIdx.x;
  for (int i = tid; i < T; i += NT) {
    S.keys[i] = kEmpty;
    S.vals[i] = 0.0;
  }
  const uint32_t count = *q.count;
  const uint32_t* list = q.rows;
  for (;;) {
    if (tid == 0) {
      S.s_idx = atomicAdd(q.cursor, 1u);
      S.s_n = 0;
    }
    __syncthreads();
    const uint32_t idx = S.s_idx;
    if (idx >= count) break;
    const uint32_t row = list[idx];
    // a row whose column span fits the table addresses it directly (slot =
    // column - lo): no probing, and the slots are already in column order
    const uint32_t rlo = lo[row];
    const bool direct = hi[row] - rlo < (uint32_t)T;
    bool full = false;
    block_for_each_product<NT, true>(A, B, A.row_begin(row), A.row_end(row), S.e, [&](uint32_t c, double v, bool ok) {
      if (!ok) return;
      uint32_t h = direct ? c - rlo : hash_slot(c, LOG2T);
      int probe = 0;
      for (; probe < T; ++probe) {
        const uint32_t cur = S.keys[h];
        if (cur == c) {
          atomicAdd(&S.vals[h], v);
          break;
        }
        if (cur == kEmpty) {
          const uint32_t prev = atomicCAS(&S.keys[h], kEmpty, c);
          if (prev == kEmpty || prev == c) {
            atomicAdd(&S.vals[h], v);
            break;
          }
        }
        h = (h + 1) & (T - 1);
      }
      full |= probe == T;
    });
    // a full table cannot count the row: an error in exact mode, an overflow
    // with unknown count in estimation mode
    const int any_full = __syncthreads_or(full);
    if (any_full && tid == 0 && !o.count) raise_status(ctr, DEV_TABLE_FULL, row);
    if (direct) {
      // ordered compaction: thread t owns slots [t * PER, t * PER + PER); a
      // block scan of the occupied counts gives each thread its output position
      unsigned cnt = 0;
#pragma unroll
      for (int i = 0; i < PER; ++i) cnt += S.keys[tid * PER + i] != kEmpty;
      unsigned long long n64;
      const unsigned long long pos0 = block_excl_scan<NT, unsigned long long>(cnt, S.e.scan, &n64);
      const uint32_t n = (uint32_t)n64;
      const uint32_t cap = o.cap[row];
      if (tid == 0) S.s_acc = out_accept(o, ctr, row, n, cap);
      __syncthreads();
      const uint32_t wn = S.s_acc ? min(n, cap) : 0u;
      const uint64_t off = o.off[row];
      uint32_t w = (uint32_t)pos0;
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        const uint32_t sl = tid * PER + i;
        const uint32_t key = S.keys[sl];
        if (key != kEmpty) {
          if (w < wn) {
            c_col[off + w] = key;
            c_val[off + w] = S.vals[sl];
          }
          ++w;
          S.keys[sl] = kEmpty;
          S.vals[sl] = 0.0;
        }
      }
      __syncthreads();
      continue;
    }
    // Rows whose span fits 32 - IB bits (the common case) are sorted by an LSD
    // radix sort of one packed word per entry, (column - lo) << IB | dense
    // index, 7 bits a pass (3 passes for a 2^20-column span, ~15 barriers
    // instead of the bitonic network's 78 for 4096 entries). The digit counts
    // and the dense-index-to-slot map live in the product enumerator's arrays,
    // free by now (8 NT + T bytes <= 24 NT bytes for every class); values
    // stay in their slots.
    constexpr int IB = LOG2T - 1;  // bits of a dense index below CAP = T / 2
    constexpr int NW = NT / 32;
    constexpr int RB = 128;        // buckets of a 7-bit digit
    static_assert(2 * RB * NW + 2 * CAP <= (int)(3 * sizeof(unsigned long long) * NT), "radix scratch");
    const int warp = tid >> 5, lane = tid & 31;
    const uint32_t span1 = hi[row] - rlo;
    if (!any_full && span1 < (1u << (32 - IB))) {
      uint16_t* hist = reinterpret_cast<uint16_t*>(S.e.incl);  // [RB][NW]
      uint16_t* dslot = hist + RB * NW;                         // [CAP]
      uint32_t kk[PER];
      unsigned cnt = 0;
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        kk[i] = S.keys[tid * PER + i];
        cnt += kk[i] != kEmpty;
      }
      unsigned long long n64;
      const uint32_t pos0 = (uint32_t)block_excl_scan<NT, unsigned long long>(cnt, S.e.scan, &n64);
      const uint32_t n = (uint32_t)n64;
      uint32_t* kin = S.keys;
      uint32_t* kout = S.keys + CAP;
      if (n <= CAP) {
        // every key was read before the scan's barriers: the writes are safe
        uint32_t w = pos0;
#pragma unroll
        for (int i = 0; i < PER; ++i) {
          if (kk[i] != kEmpty) {
            kin[w] = ((kk[i] - rlo) << IB) | w;
            dslot[w] = (uint16_t)(tid * PER + i);
            ++w;
          }
        }
      }
      __syncthreads();
      if (n <= CAP) {
        constexpr int E = RB * NW / NT;  // offsets per thread in the scan (4)
        const uint32_t kb = span1 ? 32u - (uint32_t)__clz(span1) : 0u;
        const uint32_t i0 = (uint32_t)((uint64_t)n * warp / NW), i1 = (uint32_t)((uint64_t)n * (warp + 1) / NW);
        for (uint32_t sh = IB; sh < IB + kb; sh += 7) {
          for (int i = tid; i < RB * NW; i += NT) hist[i] = 0;
          __syncthreads();
          // digit counts of this warp's contiguous item range
          for (uint32_t b = i0; b < i1; b += 32) {
            const uint32_t it = b + lane;
            const bool act = it < i1;
            const uint32_t d = act ? (kin[it] >> sh) & (RB - 1) : RB + lane;
            const unsigned peers = __match_any_sync(kFull, d);
            if (act && lane == __ffs(peers) - 1) hist[d * NW + warp] += (uint16_t)__popc(peers);
          }
          __syncthreads();
          // exclusive offsets in (digit, warp) order: a stable pass
          uint32_t loc[E], sum = 0;
#pragma unroll
          for (int e = 0; e < E; ++e) {
            loc[e] = hist[tid * E + e];
            sum += loc[e];
          }
          unsigned long long tot;
          uint32_t run = (uint32_t)block_excl_scan<NT, unsigned long long>(sum, S.e.scan, &tot);
#pragma unroll
          for (int e = 0; e < E; ++e) {
            hist[tid * E + e] = (uint16_t)run;
            run += loc[e];
          }
          __syncthreads();
          // scatter in item order: rank among equal digits of a 32-item step
          for (uint32_t b = i0; b < i1; b += 32) {
            const uint32_t it = b + lane;
            const bool act = it < i1;
            const uint32_t key = act ? kin[it] : 0u;
            const uint32_t d = act ? (key >> sh) & (RB - 1) : RB + lane;
            const unsigned peers = __match_any_sync(kFull, d);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (act && lane == leader) base = hist[d * NW + warp];
            base = __shfl_sync(kFull, base, leader);
            if (act) kout[base + __popc(peers & lanemask_lt())] = key;
            if (act && lane == leader) hist[d * NW + warp] = (uint16_t)(base + __popc(peers));
            __syncwarp();
          }
          __syncthreads();
          uint32_t* t = kin;
          kin = kout;
          kout = t;
        }
      }
      const uint32_t cap = o.cap[row];
      if (tid == 0) {
        const bool acc = out_accept(o, ctr, row, n, cap);
        if (!o.count && n > CAP) raise_status(ctr, DEV_COUNT_MISMATCH, row);
        S.s_acc = acc && n <= CAP;
      }
      __syncthreads();
      const uint32_t wn = S.s_acc ? min(n, cap) : 0u;
      const uint64_t off = o.off[row];
      for (uint32_t i = tid; i < wn; i += NT) {
        const uint32_t key = kin[i];
        c_col[off + i] = (key >> IB) + rlo;
        c_val[off + i] = S.vals[dslot[key & ((1u << IB) - 1u)]];
      }
      __syncthreads();
      for (int i = tid; i < T; i += NT) {
        S.keys[i] = kEmpty;
        S.vals[i] = 0.0;
      }
      continue;
    }
    // compaction: read this thread's slots, then rewrite the key area as sort keys
    uint32_t mine[PER];
    unsigned cnt = 0;
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      mine[i] = S.keys[tid + i * NT];
      cnt += mine[i] != kEmpty;
    }
    const unsigned base = cnt ? atomicAdd(&S.s_n, cnt) : 0u;
    __syncthreads();
    const uint32_t n = S.s_n;
    if (n <= CAP) {
      unsigned w = base;
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        if (mine[i] != kEmpty)
          sortbuf[w++] = ((unsigned long long)mine[i] << 32) | (unsigned)(tid + i * NT);
      }
    }
    uint32_t np2 = 1;
    while (np2 < n) np2 <<= 1;
    if (np2 > CAP) np2 = CAP;
    for (uint32_t i = n + tid; i < np2; i += NT) sortbuf[i] = ~0ull;
    __syncthreads();
    // bitonic sort of np2 keys
    for (uint32_t k = 2; k <= np2; k <<= 1) {
      for (uint32_t j = k >> 1; j > 0; j >>= 1) {
        for (uint32_t i = tid; i < np2 / 2; i += NT) {
          const uint32_t l = ((i & ~(j - 1)) << 1) | (i & (j - 1));
          const uint32_t r = l + j;
          const unsigned long long x = sortbuf[l], y = sortbuf[r];
          const bool asc = (l & k) == 0;
          if ((x > y) == asc) {
            sortbuf[l] = y;
            sortbuf[r] = x;
          }
        }
        __syncthreads();
      }
    }
    const uint32_t cap = o.cap[row];
    if (tid == 0) {
      const uint32_t nn = any_full ? kUnknownCount : n;
      bool acc = out_accept(o, ctr, row, nn, cap);
      if (!o.count && n > CAP) raise_status(ctr, DEV_COUNT_MISMATCH, row);
      S.s_acc = acc && n <= CAP && !any_full;
    }
    __syncthreads();
    // rows that overflowed the sort capacity or their slots are not written
    const uint32_t wn = S.s_acc ? min(n, cap) : 0u;
    const uint64_t off = o.off[row];
    for (uint32_t i = tid; i < wn; i += NT) {
      const unsigned long long e = sortbuf[i];
      c_col[off + i] = (uint32_t)(e >> 32);
      c_val[off + i] = S.vals[(uint32_t)e];
    }
    __syncthreads();
    for (int i = tid; i < T; i += NT) {
      S.keys[i] = kEmpty;
      S.vals[i] = 0.0;
    }
  }
}

// Emits the set bits of one 64-bit word per lane (a warp's group of 32
// consecutive bitmap words) in rank order: emit(j, b) for the group's j-th set
// bit, at bit offset b from the group's first bit. Sparse groups (at most
// kSparseBits bits in every word) are written by a per-lane loop over each
// word's bits (lanes write nearly consecutive entries); denser groups entry by
// entry, lane l taking entries l, l + 32, ..., the owner word found by a
// binary search over the lanes' exclusive counts and the bit by a 6-step
// select. Warp-collective; emit runs on the lanes that own an entry.
constexpr uint32_t kSparseBits = 8;
template <typename Emit>
__device__ __forceinline__ void warp_emit_group(unsigned long long word, int lane, Emit&& emit,
                                                uint32_t jlo = 0u, uint32_t jhi = 0xFFFFFFFFu) {
  const uint32_t cnt = (uint32_t)__popcll(word);
  uint32_t incl = cnt;
#pragma unroll
  for (int sh = 1; sh < 32; sh <<= 1) {
    const uint32_t y = __shfl_up_sync(kFull, incl, sh);
    if (lane >= sh) incl += y;
  }
  const uint32_t excl = incl - cnt;
  const uint32_t total = __shfl_sync(kFull, incl, 31);
  jhi = min(jhi, total);
  if (jlo >= jhi) return;
  if (__reduce_max_sync(kFull, cnt) <= kSparseBits) {
    uint32_t j = excl;
    unsigned long long x = word;
    while (x) {
      const uint32_t b = (uint32_t)(__ffsll((long long)x) - 1);
      x &= x - 1ull;
      if (j >= jlo && j < jhi) emit(j, (uint32_t)lane * 64u + b);
      ++j;
    }
    return;
  }
  const uint32_t rounds = (jhi - jlo + 31) >> 5;
  for (uint32_t rd = 0; rd < rounds; ++rd) {
    const uint32_t j = jlo + rd * 32 + lane;
    uint32_t k = 0;
#pragma unroll
    for (int step = 16; step > 0; step >>= 1) {
      const uint32_t e = __shfl_sync(kFull, excl, k + step);
      if (e <= j) k += step;
    }
    unsigned long long x = __shfl_sync(kFull, word, k);
    uint32_t r = j - __shfl_sync(kFull, excl, k);
    if (j < jhi) {
      uint32_t pos = 0;
#pragma unroll
      for (int sb = 32; sb > 0; sb >>= 1) {
        const uint32_t c = (uint32_t)__popcll(x & ((1ull << sb) - 1ull));
        if (r >= c) {
          r -= c;
          x >>= sb;
          pos += sb;
        }
      }
      emit(j, k * 64u + pos);
    }
  }
}

// ---------------------------------------------------------------- bitmap accumulators
// Symbolic: a bitmap over (a window of) the row's output column span; the count
// is the popcount. Windows of 2^20 columns sweep wider spans.
struct BitmapSymSmem {
  unsigned long long bits[kBitmapWords];
  EnumSmem<kBitmapThreads> e;
  unsigned long long red[33];
  unsigned long long slot;
  uint32_t s_idx;
};

template <typename RP>
__global__ void __launch_bounds__(kBitmapThreads, 1)
    k_sym_bitmap(Csr<RP> A, Csr<RP> B, RowQueue q, DevCounters* __restrict__ ctr,
                 const uint32_t* __restrict__ prod, const uint32_t* __restrict__ lo,
                 const uint32_t* __restrict__ hi, uint32_t* __restrict__ row_nnz, uint64_t* __restrict__ bm_off,
                 unsigned long long* __restrict__ cache, uint64_t cache_words, bool unknown_only) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BitmapSymSmem& S = *reinterpret_cast<BitmapSymSmem*>(smem_raw);
  const int tid = threadIdx.x;
  for (int i = tid; i < kBitmapWords; i += kBitmapThreads) S.bits[i] = 0ull;
  const uint32_t count = *q.count;
  const uint32_t* list = q.rows;
  for (;;) {
    if (tid == 0) S.s_idx = atomicAdd(q.cursor, 1u);
    __syncthreads();
    const uint32_t idx = S.s_idx;
    if (idx >= count) break;
    const uint32_t row = list[idx];
    if (unknown_only && row_nnz[row] != kUnknownCount) {  // count already known (uniform over the block)
      __syncthreads();
      continue;
    }
    const uint64_t a0 = A.row_begin(row), a1 = A.row_end(row);
    const uint64_t rlo = lo[row], rhi = hi[row];
    unsigned long long total = 0;
    for (uint64_t w0 = rlo; w0 <= rhi; w0 += kBitmapBits) {
      const uint64_t w1 = min(rhi + 1, w0 + kBitmapBits);
      const uint32_t nwords = (uint32_t)((w1 - w0 + 63) >> 6);
      const bool single = w0 == rlo && rhi < w0 + kBitmapBits;
      block_for_each_product<kBitmapThreads, false>(A, B, a0, a1, S.e, [&](uint32_t c, double, bool ok) {
        mark_bit(S.bits, c, ok, single, w0, w1);
      });
      // a single-window row's exact bitmap is saved for the numeric pass when room is left
      if (tid == 0) {
        unsigned long long slot = ~0ull;
        if (single && cache_words) {
          const unsigned long long at = atomicAdd(&ctr->cache_cursor, (unsigned long long)nwords);
          if (at + nwords <= cache_words) slot = at;
        }
        S.slot = slot;
        if (single) bm_off[row] = slot;
      }
      __syncthreads();
      const unsigned long long slot = S.slot;
      unsigned long long cnt = 0;
      for (uint32_t w = tid; w < nwords; w += kBitmapThreads) {
        const unsigned long long word = S.bits[w];
        cnt += __popcll(word);
        if (slot != ~0ull) cache[slot + w] = word;
        S.bits[w] = 0ull;
      }
      total += block_sum_u64<kBitmapThreads>(cnt, S.red);
    }
    if (tid == 0) row_nnz[row] = (uint32_t)total;
  }
}

// Numeric: bitmap-rank accumulator. The row's output columns are marked in a
// bitmap (pass 1, or reloaded from the copy the symbolic pass saved); a block
// scan turns it into a rank table (u16 exclusive popcount of every 64-bit word
// inside its 1024-word superblock plus u32 superblock offsets);
// the sorted column ids are written from the bitmap, and the values are
// accumulated straight into C at position rank(column) with FP64 reductions in
// L2 (pass 2). Output is sorted by construction: no hash collisions, no sort.
struct BitmapNumSmem {
  unsigned long long bits[kBitmapWords];
  uint16_t wpre[kBitmapWords];        // popcount of the words before each word, within its 1024-word superblock
  uint32_t spre[kBitmapWords / 1024];  // popcount of the superblocks before each superblock
  uint32_t scan[33];
  EnumSmem<kBitmapThreads> e;
  uint32_t s_idx, s_acc;
};

template <typename RP>
__global__ void __launch_bounds__(kBitmapThreads, 1)
    k_num_bitmap(Csr<RP> A, Csr<RP> B, RowQueue q, OutSpec o, DevCounters* __restrict__ ctr,
                 const uint32_t* __restrict__ prod, const uint32_t* __restrict__ lo,
                 const uint32_t* __restrict__ hi, const uint64_t* __restrict__ bm_off,
                 const unsigned long long* __restrict__ cache, uint32_t* __restrict__ c_col,
                 double* __restrict__ c_val, bool wide_only) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  BitmapNumSmem& S = *reinterpret_cast<BitmapNumSmem*>(smem_raw);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kBitmapWords; i += kBitmapThreads) S.bits[i] = 0ull;
  const uint32_t count = *q.count;
  const uint32_t* list = q.rows;
  // Rows are visited in a spread order: on power-law inputs the heaviest rows
  // sit together in the list (low row ids), and taking them all at once puts
  // ~one heavy row per SM in flight, whose C values (zeroed, then reduced
  // into) overflow L2 and make the round trip through DRAM in between.
  // Spread, few heavy rows run together (R-MAT 2^20: 280 -> 225 ms).
  const uint32_t stride = spread_stride(count);
  for (;;) {
    __syncthreads();  // every thread has read the previous row index
    if (tid == 0) S.s_idx = atomicAdd(q.cursor, 1u);
    __syncthreads();
    const uint32_t idx = S.s_idx;
    if (idx >= count) break;
    const uint32_t row = list[spread_index(idx, count, stride)];
    const uint64_t a0 = A.row_begin(row), a1 = A.row_end(row);
    const uint64_t rlo = lo[row], rhi = hi[row];
    if (wide_only && rhi - rlo + 1 <= kBitmapBits) continue;  // k_num_window's rows
    const uint64_t row_off = o.off[row];
    const uint32_t expect = o.cap[row];
    const uint64_t row_lim = row_off + expect;
    // estimation mode counts a row before writing it; a row wider than one
    // window is not counted here and goes to the overflow list
    if (o.count && rhi - rlo + 1 > kBitmapBits) {
      if (tid == 0) out_accept(o, ctr, row, kUnknownCount, expect);
      continue;
    }
    const uint64_t slot = cache ? bm_off[row] : ~0ull;
    uint64_t off = row_off;
    // a row whose A entries fit one chunk is loaded once for both passes
    const bool one_chunk = a1 - a0 <= (uint64_t)kBitmapThreads;
    if (one_chunk) block_load_chunk<kBitmapThreads, true>(A, B, a0, a1, S.e);
    for (uint64_t w0 = rlo; w0 <= rhi; w0 += kBitmapBits) {
      const uint64_t w1 = min(rhi + 1, w0 + kBitmapBits);
      const uint32_t nwords = (uint32_t)((w1 - w0 + 63) >> 6);
      const bool single = w0 == rlo && rhi < w0 + kBitmapBits;
      if (single && slot != ~0ull) {
        // reload the exact bitmap saved by the symbolic pass
        for (uint32_t w = tid; w < nwords; w += kBitmapThreads) S.bits[w] = cache[slot + w];
        __syncthreads();
      } else {
        // pass 1: mark columns
        auto mark = [&](uint32_t c, double, bool ok) { mark_bit(S.bits, c, ok, single, w0, w1); };
        if (one_chunk) block_run_chunk<kBitmapThreads, false>(B, S.e, mark);
        else block_for_each_product<kBitmapThreads, false>(A, B, a0, a1, S.e, mark);
      }
      // rank table, warp-major so shared-memory reads do not collide: warp w
      // covers words [512w, 512w + 512), lane l reads words 512w + 32i + l
      const uint32_t wbase = (uint32_t)warp * 512u;
      uint32_t local = 0;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const uint32_t w = wbase + 32u * i + lane;
        local += (w < nwords) ? __popcll(S.bits[w]) : 0u;
      }
#pragma unroll
      for (int sh = 16; sh > 0; sh >>= 1) local += __shfl_xor_sync(kFull, local, sh);
      uint32_t nw_total;
      const uint32_t warp_base =
          __shfl_sync(kFull, block_excl_scan<kBitmapThreads, uint32_t>(lane == 0 ? local : 0u, S.scan, &nw_total), 0);
      if (o.count) {
        // estimation mode (single window): the count is known now; a row that
        // does not fit its slots is listed and skipped
        if (tid == 0) S.s_acc = out_accept(o, ctr, row, nw_total, expect);
        __syncthreads();
        if (!S.s_acc) {
          for (uint32_t w = tid; w < nwords; w += kBitmapThreads) S.bits[w] = 0ull;
          __syncthreads();
          off = row_lim;
          break;
        }
      }
      // superblock k (words [1024k, 1024k + 1024)) starts with warp 2k
      if (lane == 0 && (warp & 1) == 0) S.spre[warp >> 1] = warp_base;
      __syncthreads();
      uint32_t run = warp_base - S.spre[warp >> 1];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const uint32_t w = wbase + 32u * i + lane;
        const uint32_t pc = (w < nwords) ? (uint32_t)__popcll(S.bits[w]) : 0u;
        uint32_t x = pc;
#pragma unroll
        for (int sh = 1; sh < 32; sh <<= 1) {
          const uint32_t y = __shfl_up_sync(kFull, x, sh);
          if (lane >= sh) x += y;
        }
        if (w < nwords) S.wpre[w] = (uint16_t)(run + x - pc);
        run += __shfl_sync(kFull, x, 31);
      }
      __syncthreads();
      // ordered output of the column ids (and zeroed values): warp w writes
      // the window's entries [w n / 32, (w + 1) n / 32), starting at the word
      // that holds its first entry, 32 words at a time. Split by entries, not
      // by words: the dense words of a power-law row's hub columns would
      // otherwise all fall to the first few warps.
      {
        const uint32_t e0 = (uint32_t)(((uint64_t)warp * nw_total) >> 5);
        const uint32_t e1 = (uint32_t)(((uint64_t)(warp + 1) * nw_total) >> 5);
        if (e0 < e1) {
          // last word whose prefix is <= e0
          uint32_t lo_w = 0, hi_w = nwords;  // prefix(lo_w) <= e0 < prefix(hi_w) (prefix(nwords) = total)
          while (hi_w - lo_w > 1) {
            const uint32_t mid = (lo_w + hi_w) >> 1;
            if (S.spre[mid >> 10] + (uint32_t)S.wpre[mid] <= e0) lo_w = mid; else hi_w = mid;
          }
          for (uint32_t wb = lo_w; wb < nwords; wb += 32u) {
            const uint32_t gpre = S.spre[wb >> 10] + S.wpre[wb];
            if (gpre >= e1) break;
            const uint32_t w = wb + lane;
            const uint64_t gout = off + gpre;
            const uint64_t gcol = w0 + (uint64_t)wb * 64;
            warp_emit_group(w < nwords ? S.bits[w] : 0ull, lane, [&](uint32_t j, uint32_t b) {
              const uint64_t o = gout + j;
              if (o < row_lim) {
                c_col[o] = (uint32_t)(gcol + b);
                c_val[o] = 0.0;
              }
            }, e0 > gpre ? e0 - gpre : 0u, e1 - gpre);
          }
        }
      }
      __syncthreads();
      // pass 2: accumulate values at their ranks
      auto accumulate = [&](uint32_t c, double v, bool ok) {
        if (ok && (single || (c >= w0 && c < w1))) {
          const uint32_t d = (uint32_t)(c - w0);
          const uint32_t w = d >> 6;
          const uint32_t r = S.spre[w >> 10] + S.wpre[w] + __popcll(S.bits[w] & ((1ull << (d & 63)) - 1ull));
          if (off + r < row_lim) atomicAdd(&c_val[off + r], v);
        }
      };
      if (one_chunk) block_run_chunk<kBitmapThreads, true>(B, S.e, accumulate);
      else block_for_each_product<kBitmapThreads, true>(A, B, a0, a1, S.e, accumulate);
      for (uint32_t w = tid; w < nwords; w += kBitmapThreads) S.bits[w] = 0ull;
      off += nw_total;
      __syncthreads();
    }
    if (tid == 0 && !o.count && off != row_lim) raise_status(ctr, DEV_COUNT_MISMATCH, row);
  }
}

// ---------------------------------------------------------------- windowed numeric accumulator
// Exact-mode numeric kernel of the bitmap class, for rows whose column span
// fits one 2^20-bit bitmap. The row's exact output bitmap (saved by the
// symbolic pass, or marked here into a per-block scratch copy) is swept in
// windows of whole words holding at most kWinV output entries and kWinWords
// words. For each window the block loads the window's bitmap words and their
// exclusive popcounts into shared memory, finds every A entry's run of its
// sorted B row inside the window's column range (a resume cursor per A entry
// marks where the previous window stopped, so every B entry of the row is
// enumerated once over the whole sweep), accumulates the products into FP64
// slots in shared memory at the window-local rank of their column, and writes
// the window's column ids and values to C once, in order. There is no global
// atomic and no zero-fill of C; the reference's denseNumericIterKernel
// (kernels/AccumulatorDense.cuh:610-806) sweeps column windows the same way
// with dense per-column slots, which this kernel replaces by bitmap ranks so
// that sparse wide rows take few windows.
constexpr int kWinV = 12288;     // output entries per window (FP64 slots in shared memory)
constexpr int kWinWords = 8192;  // bitmap words per window (512K columns)
static_assert(kWinV + kWinWords >= kBitmapWords, "the marking bitmap overlays the slots and window words");
static_assert(kWinV < 65536, "window-local ranks are 16-bit");

struct WinNumSmem {
  unsigned long long area[kWinV + kWinWords];  // FP64 slots, then the window's words; marking: the row bitmap
  uint16_t wpre[kWinWords];                    // exclusive popcount of the window's words before each word
  EnumSmem<kBitmapThreads> e;
  unsigned long long seg_pos[64], seg_end[64];  // few-entry chunks: B-run starts / row ends, then run ends
  uint32_t scan[33];
  uint32_t s_idx, s_we, s_nwin;
};

// First index p in [lo, hi) with col[p] >= cb (hi when there is none); col is
// sorted on [lo, hi). Warp-collective: the first round checks the first 32
// entries, later rounds probe 32 evenly spaced entries of the remaining range.
__device__ __forceinline__ uint64_t warp_run_end(const uint32_t* __restrict__ col, uint64_t lo, uint64_t hi,
                                                 uint32_t cb) {
  const int lane = threadIdx.x & 31;
  for (int round = 0; round < 24 && lo < hi; ++round) {
    const uint64_t n = hi - lo;
    if (round == 0 || n <= 32) {
      const uint64_t p = lo + lane;
      const bool ge = p < hi && col[p] >= cb;
      const unsigned m = __ballot_sync(kFull, ge);
      if (m) return lo + (uint64_t)(__ffs(m) - 1);
      if (n <= 32) return hi;
      lo += 32;
      continue;
    }
    const uint64_t step = (n + 31) / 32;
    const uint64_t q = lo + (uint64_t)(lane + 1) * step - 1;
    const bool ge = q < hi ? col[q] >= cb : true;
    const unsigned m = __ballot_sync(kFull, ge);
    const int f = __ffs(m) - 1;  // lane 31 probes at or past hi - 1: m == 0 only if col[hi - 1] < cb
    if (f < 0) return hi;
    const uint64_t nhi = min(lo + (uint64_t)(f + 1) * step - 1, hi);
    lo = lo + (uint64_t)f * step;
    hi = nhi;
  }
  return hi;
}

// The same search by one thread: galloping from lo, then bisection.
__device__ __forceinline__ uint64_t thread_run_end(const uint32_t* __restrict__ col, uint64_t lo, uint64_t hi,
                                                   uint32_t cb) {
  if (lo >= hi || col[lo] >= cb) return lo;
  uint64_t good = lo, step = 1;  // col[good] < cb
  for (int i = 0; i < 64; ++i) {
    const uint64_t p = good + step;
    if (p >= hi) break;
    if (col[p] >= cb) {
      hi = p;
      break;
    }
    good = p;
    step <<= 1;
  }
  uint64_t a = good + 1, b = hi;
  while (a < b) {
    const uint64_t m = a + ((b - a) >> 1);
    if (col[m] >= cb) b = m; else a = m + 1;
  }
  return a;
}

template <typename RP>
__global__ void __launch_bounds__(kBitmapThreads, 1)
    k_num_window(Csr<RP> A, Csr<RP> B, RowQueue q, OutSpec o, DevCounters* __restrict__ ctr,
                 const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi,
                 const uint64_t* __restrict__ bm_off, const unsigned long long* __restrict__ cache,
                 unsigned long long* __restrict__ scratch, uint32_t* __restrict__ cursor,
                 uint32_t* __restrict__ c_col, double* __restrict__ c_val) {
  constexpr int NT = kBitmapThreads;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  WinNumSmem& S = *reinterpret_cast<WinNumSmem*>(smem_raw);
  double* vals = reinterpret_cast<double*>(S.area);
  unsigned long long* wbits = S.area + kWinV;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < kWinV; i += NT) vals[i] = 0.0;
  unsigned long long* my_scratch = scratch + (uint64_t)blockIdx.x * kBitmapWords;
  const uint32_t count = *q.count;
  const uint32_t stride = spread_stride(count);
  for (;;) {
    __syncthreads();  // every thread has read the previous row index
    if (tid == 0) S.s_idx = atomicAdd(q.cursor, 1u);
    __syncthreads();
    const uint32_t idx = S.s_idx;
    if (idx >= count) break;
    const uint32_t row = q.rows[spread_index(idx, count, stride)];
    const uint64_t rlo = lo[row], rhi = hi[row];
    if (rhi - rlo + 1 > kBitmapBits) continue;  // wider rows: k_num_bitmap
    const uint64_t a0 = A.row_begin(row), a1 = A.row_end(row);
    const uint64_t row_off = o.off[row];
    const uint32_t expect = o.cap[row];
    const uint32_t nw = (uint32_t)((rhi - rlo + 64) >> 6);
    const uint64_t slot = cache ? bm_off[row] : ~0ull;
    const unsigned long long* gbits;
    if (slot != ~0ull) {
      gbits = cache + slot;
    } else {
      // mark the row's bitmap over the slot area, keep a copy in this block's scratch
      for (uint32_t w = tid; w < nw; w += NT) S.area[w] = 0ull;
      __syncthreads();
      block_for_each_product<NT, false>(A, B, a0, a1, S.e, [&](uint32_t c, double, bool ok) {
        mark_bit(S.area, c, ok, true, rlo, rhi + 1);
      });
      for (uint32_t w = tid; w < nw; w += NT) my_scratch[w] = S.area[w];
      __syncthreads();
      for (int i = tid; i < kWinV; i += NT) vals[i] = 0.0;
      __syncthreads();
      gbits = my_scratch;
    }
    // resume cursors (offsets into each A entry's B row): registers when the
    // row's A entries fit one chunk, else the per-entry array
    const bool one_chunk = a1 - a0 <= (uint64_t)NT;
    uint32_t my_cur = 0;
    if (!one_chunk)
      for (uint64_t k = a0 + tid; k < a1; k += NT) cursor[k] = 0u;
    uint64_t r0 = 0;  // rank of the window's first entry within the row
    for (uint32_t ws = 0; ws < nw;) {
      const uint32_t wl = min(nw - ws, (uint32_t)kWinWords);
      if (tid == 0) S.s_we = wl;
      // window words and their popcounts, warp-major (warp w: words [256w, 256w + 256))
      const uint32_t wbase = (uint32_t)warp * (kWinWords / 32);
      uint32_t local = 0;
#pragma unroll
      for (int i = 0; i < kWinWords / 1024; ++i) {
        const uint32_t w = wbase + 32u * i + lane;
        const unsigned long long x = w < wl ? gbits[ws + w] : 0ull;
        wbits[w] = x;
        local += __popcll(x);
      }
#pragma unroll
      for (int sh = 16; sh > 0; sh >>= 1) local += __shfl_xor_sync(kFull, local, sh);
      uint32_t wtotal;
      const uint32_t warp_base =
          __shfl_sync(kFull, block_excl_scan<NT, uint32_t>(lane == 0 ? local : 0u, S.scan, &wtotal), 0);
      uint32_t run = warp_base;
#pragma unroll
      for (int i = 0; i < kWinWords / 1024; ++i) {
        const uint32_t w = wbase + 32u * i + lane;
        const uint32_t pc = (uint32_t)__popcll(wbits[w]);
        uint32_t x = pc;
#pragma unroll
        for (int sh = 1; sh < 32; sh <<= 1) {
          const uint32_t y = __shfl_up_sync(kFull, x, sh);
          if (lane >= sh) x += y;
        }
        const uint32_t ex = run + x - pc;
        S.wpre[w] = (uint16_t)ex;  // exact below the window's end (<= kWinV)
        // the word that takes the count past kWinV ends the window
        if (w < wl && ex <= (uint32_t)kWinV && ex + pc > (uint32_t)kWinV) {
          S.s_we = w;
          S.s_nwin = ex;
        }
        run += __shfl_sync(kFull, x, 31);
      }
      __syncthreads();
      const uint32_t we = S.s_we;
      const uint32_t nwin = we == wl ? wtotal : S.s_nwin;
      const uint64_t ca = rlo + 64ull * ws;
      const uint32_t cb = (uint32_t)min((uint64_t)(rlo + 64ull * (ws + we)), (uint64_t)(rhi + 1));
      // products whose column lies in [ca, cb), accumulated at their window rank
      auto accumulate = [&](uint32_t c, double v, bool ok) {
        if (ok) {
          const uint32_t d = c - (uint32_t)ca;
          const uint32_t w = d >> 6;
          const uint32_t r = S.wpre[w] + (uint32_t)__popcll(wbits[w] & ((1ull << (d & 63)) - 1ull));
          if (r < (uint32_t)kWinV) atomicAdd(&vals[r], v);
        }
      };
      for (uint64_t c0 = a0; c0 < a1; c0 += NT) {
        const uint32_t na = (uint32_t)min(a1 - c0, (uint64_t)NT);
        const uint64_t k = c0 + tid;
        unsigned long long bs = 0, be = 0, pos = 0;
        double av = 0.0;
        if (tid < (int)na) {
          const uint32_t j = A.col[k];
          bs = B.row_begin(j);
          be = B.row_end(j);
          pos = bs + (one_chunk ? my_cur : cursor[k]);
          av = A.val[k];
        }
        unsigned long long end = pos;
        if (na <= 64) {
          // few entries: one warp searches each run
          if (tid < (int)na) {
            S.seg_pos[tid] = pos;
            S.seg_end[tid] = be;
          }
          __syncthreads();
          for (uint32_t e = warp; e < na; e += NT / 32) {
            const uint64_t r = warp_run_end(B.col, S.seg_pos[e], S.seg_end[e], cb);
            __syncwarp();
            if (lane == 0) S.seg_end[e] = r;
          }
          __syncthreads();
          if (tid < (int)na) end = S.seg_end[tid];
        } else if (tid < (int)na) {
          end = thread_run_end(B.col, pos, be, cb);
        }
        if (tid < (int)na) {
          if (one_chunk) my_cur = (uint32_t)(end - bs);
          else cursor[k] = (uint32_t)(end - bs);
        }
        block_pack_chunk<NT, true>(pos, end - pos, av, S.e);
        block_run_chunk<NT, true>(B, S.e, accumulate);
      }
      // the window's entries in rank order: column ids from the bitmap, values
      // from the slots (which are cleared for the next window)
      const uint64_t wout = row_off + r0;
      const uint64_t row_lim = row_off + expect;
      // split by entries across the warps (dense hub words would otherwise
      // all fall to the first warps), 32 words at a time from the word that
      // holds each warp's first entry
      const uint32_t e0 = (uint32_t)(((uint64_t)warp * nwin) / (NT / 32));
      const uint32_t e1 = (uint32_t)(((uint64_t)(warp + 1) * nwin) / (NT / 32));
      if (e0 < e1) {
        uint32_t lo_w = 0, hi_w = we;  // prefix(lo_w) <= e0 < prefix(hi_w) (prefix(we) = nwin)
        while (hi_w - lo_w > 1) {
          const uint32_t mid = (lo_w + hi_w) >> 1;
          if ((uint32_t)S.wpre[mid] <= e0) lo_w = mid; else hi_w = mid;
        }
        for (uint32_t wb = lo_w; wb < we; wb += 32u) {
          const uint32_t gpre = S.wpre[wb];
          if (gpre >= e1) break;
          const uint32_t w = wb + lane;
          const uint64_t gcol = ca + (uint64_t)wb * 64;
          warp_emit_group(w < we ? wbits[w] : 0ull, lane, [&](uint32_t j, uint32_t b) {
            const uint32_t lr = gpre + j;
            const uint64_t at = wout + lr;
            const double v = vals[lr];
            vals[lr] = 0.0;
            if (at < row_lim) {
              c_col[at] = (uint32_t)(gcol + b);
              c_val[at] = v;
            }
          }, e0 > gpre ? e0 - gpre : 0u, e1 - gpre);
        }
      }
      __syncthreads();
      r0 += nwin;
      ws += we;
    }
    if (tid == 0 && r0 != expect) raise_status(ctr, DEV_COUNT_MISMATCH, row);
  }
}

// ---------------------------------------------------------------- segment dispatch
// Writes each row's dispatch slot: block i paints rows [iv[3i], iv[3i+1]) with
// slot iv[3i+2]. Intervals are disjoint; unpainted rows keep slot 0.
__global__ void __launch_bounds__(256) k_paint_rows(const uint32_t* __restrict__ iv, uint8_t* __restrict__ row_pol) {
  const uint32_t r0 = iv[3 * blockIdx.x], r1 = iv[3 * blockIdx.x + 1];
  const uint8_t slot = (uint8_t)iv[3 * blockIdx.x + 2];
  for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) row_pol[r] = slot;
}

void launch_paint_rows(const uint32_t* iv, uint32_t n, uint8_t* row_pol, uint64_t rows, cudaStream_t s) {
  cudaMemsetAsync(row_pol, 0, rows, s);
  if (n) k_paint_rows<<<n, 256, 0, s>>>(iv, row_pol);
}

// ---------------------------------------------------------------- scan
__global__ void __launch_bounds__(1024) k_scan_reduce(const uint32_t* __restrict__ in, uint64_t n,
                                                      unsigned long long* __restrict__ tile_sums) {
  __shared__ unsigned long long red[33];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile;
  unsigned long long s = 0;
#pragma unroll
  for (int q = 0; q < kScanTile / 1024; ++q) {
    const uint64_t i = base + (uint64_t)q * 1024 + threadIdx.x;
    if (i < n) s += in[i];
  }
  s = block_sum_u64<1024>(s, red);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_scan_tiles(unsigned long long* __restrict__ tile_sums,
                                                     uint64_t ntiles, unsigned long long* __restrict__ total_out,
                                                     uint64_t* __restrict__ rowptr64,
                                                     uint32_t* __restrict__ rowptr32, uint64_t rows) {
  __shared__ unsigned long long scr[33];
  const uint64_t per = (ntiles + 1023) / 1024;
  const uint64_t b = (uint64_t)threadIdx.x * per;
  unsigned long long s = 0;
  for (uint64_t i = 0; i < per; ++i)
    if (b + i < ntiles) s += tile_sums[b + i];
  unsigned long long total;
  unsigned long long run = block_excl_scan<1024, unsigned long long>(s, scr, &total);
  for (uint64_t i = 0; i < per; ++i) {
    if (b + i < ntiles) {
      const unsigned long long t = tile_sums[b + i];
      tile_sums[b + i] = run;
      run += t;
    }
  }
  if (threadIdx.x == 0) {
    *total_out = total;
    rowptr64[rows] = total;
    if (rowptr32) rowptr32[rows] = (uint32_t)total;
  }
}

// Per tile (256 threads x 4 rows): local exclusive scan + tile offset -> row
// pointers; each row is also appended to its numeric class list.
constexpr int kScanApplyThreads = kScanTile / 4;
static_assert(NB_COUNT * kMaxChunks <= kScanApplyThreads, "one thread per class-list counter");
__global__ void __launch_bounds__(kScanApplyThreads) k_scan_apply(const uint32_t* __restrict__ in, uint64_t n,
                                                     const unsigned long long* __restrict__ tile_offs,
                                                     uint64_t* __restrict__ rowptr64,
                                                     uint32_t* __restrict__ rowptr32,
                                                     const uint32_t* __restrict__ prod,
                                                     const uint32_t* __restrict__ lo,
                                                     const uint32_t* __restrict__ hi,
                                                     const uint32_t* __restrict__ anz,
                                                     const uint64_t* __restrict__ bm_off,
                                                     uint32_t* __restrict__ num_bins,
                                                     DevCounters* __restrict__ ctr, NumPolicySet pols,
                                                     const uint8_t* __restrict__ row_pol, int bin_rows, int chunks,
                                                     const uint32_t* __restrict__ chunk_bound,
                                                     unsigned* __restrict__ chunk_count) {
  __shared__ unsigned long long scr[33];
  __shared__ unsigned long long s_cls[3][NB_COUNT];
  __shared__ unsigned s_cnt[NB_COUNT * kMaxChunks];
  __shared__ uint32_t s_bound[kMaxChunks + 1];
  const int nseg = chunks > 1 ? chunks : 1;
  if (threadIdx.x < 3 * NB_COUNT) (&s_cls[0][0])[threadIdx.x] = 0ull;
  if (threadIdx.x < NB_COUNT * kMaxChunks) s_cnt[threadIdx.x] = 0u;
  if (nseg > 1 && (int)threadIdx.x <= nseg) s_bound[threadIdx.x] = chunk_bound[threadIdx.x];
  const uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * 4;
  uint32_t v[4];
  unsigned long long s = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    v[q] = (base + q < n) ? in[base + q] : 0u;
    s += v[q];
  }
  unsigned long long total;
  unsigned long long run =
      block_excl_scan<kScanApplyThreads, unsigned long long>(s, scr, &total) + tile_offs[blockIdx.x];
  int bq[4], sq[4];
  uint32_t rq[4], aq[4], pq[4];
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const uint64_t i = base + q;
    int b = -1;
    if (i < n) {
      rowptr64[i] = run;
      if (rowptr32) rowptr32[i] = (uint32_t)run;
      run += v[q];
    }
    if (i < n && bin_rows) {
      const uint32_t p = prod[i];
      const NumPolicy& pol = pols.p[row_pol ? row_pol[i] : 0];
      b = num_bin_for(v[q], p, (uint64_t)hi[i] - lo[i] + 1, pol);
      if (b >= 0 && pol.force_bin < 0 && bm_off[i] != ~0ull) b = NB_BITMAP;  // reuse the saved bitmap
      if (b == NB_BITMAP && (uint64_t)hi[i] - lo[i] + 1 > kBitmapBits) atomicAdd(&ctr->num_wide, 1u);
      aq[q] = anz[i];
      pq[q] = p;
    }
    bq[q] = b;
    rq[q] = (uint32_t)i;
    // row chunk of the row: the last chunk whose first row is <= i (the
    // bounds are visible after the block scan's barriers)
    int g = 0;
    if (nseg > 1 && b >= 0)
      while (g + 1 < nseg && s_bound[g + 1] <= i) ++g;
    sq[q] = g;
  }
  if (!bin_rows) return;
  block_bin_append<4>(bq, sq, rq, s_cnt, NB_COUNT, nseg, s_bound, nseg > 1 ? chunk_count : ctr->num_count,
                      ctr->num_count, num_bins, n);
  // per-class sums (nnz, A entries, products) of the classes present in the
  // warp: warp sums, then one shared atomic per warp and class
  const int lane = threadIdx.x & 31;
  unsigned present = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) present |= bq[q] >= 0 ? 1u << bq[q] : 0u;
  present = __reduce_or_sync(kFull, present);
  while (present) {
    const int c = __ffs(present) - 1;
    present &= present - 1;
    unsigned long long a = 0, b2 = 0, d = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      if (bq[q] == c) {
        a += v[q];
        b2 += aq[q];
        d += pq[q];
      }
    }
    a = warp_sum_u64(a);
    b2 = warp_sum_u64(b2);
    d = warp_sum_u64(d);
    if (lane == 0 && a) {
      atomicAdd(&s_cls[0][c], a);
      atomicAdd(&s_cls[1][c], b2);
      atomicAdd(&s_cls[2][c], d);
    }
  }
  __syncthreads();
  if (threadIdx.x < NB_COUNT && s_cls[0][threadIdx.x]) {
    atomicAdd(&ctr->num_nnz[threadIdx.x], s_cls[0][threadIdx.x]);
    atomicAdd(&ctr->num_anz[threadIdx.x], s_cls[1][threadIdx.x]);
    atomicAdd(&ctr->num_prod[threadIdx.x], s_cls[2][threadIdx.x]);
  }
}

// ---------------------------------------------------------------- murmur3
// 32-bit MurmurHash3 of one 4-byte little-endian key (public-domain algorithm by
// Austin Appleby; reference: kernels/MurmurHash.cuh:44-98).
__device__ __forceinline__ uint32_t murmur3_u32(uint32_t key, uint32_t seed) {
  uint32_t k = key * 0xcc9e2d51u;
  k = (k << 15) | (k >> 17);
  k *= 0x1b873593u;
  uint32_t h = seed ^ k;
  h = (h << 13) | (h >> 19);
  h = h * 5u + 0xe6546b64u;
  h ^= 4u;
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

__global__ void k_murmur3(const uint32_t* __restrict__ keys, uint32_t* __restrict__ out, uint64_t n,
                          uint32_t seed) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = murmur3_u32(keys[i], seed);
}

// ---------------------------------------------------------------- HyperLogLog
// Row-size estimates (reference: kernels/HLL.cuh:11-357). A B row's sketch has
// 2^P one-byte registers: register (h & (2^P-1)) keeps the largest
// clz(h) + 1 (capped at 32 - P + 1) over the MurmurHash3 values h of the row's
// column ids (seed 1234). The sketch of an A row's output is the register-wise
// maximum over the sketches of the B rows it references; the estimate is
// E = alpha_P * m^2 / sum 2^-M[i], replaced by m * ln(m / V) when V registers
// are empty and E < 2.5 m.
constexpr uint32_t kMurmurSeed = 1234;

template <typename RP, int LOGP>
__global__ void __launch_bounds__(256) k_hll_sketch(Csr<RP> B, uint8_t* __restrict__ sk) {
  constexpr int M = 1 << LOGP;
  __shared__ unsigned regs[8][M];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t r = (uint64_t)blockIdx.x * 8 + warp; r < B.rows; r += (uint64_t)gridDim.x * 8) {
    for (int i = lane; i < M; i += 32) regs[warp][i] = 0u;
    __syncwarp();
    const uint64_t b1 = B.row_end(r);
    for (uint64_t q = B.row_begin(r) + lane; q < b1; q += 32) {
      const uint32_t h = murmur3_u32(B.col[q], kMurmurSeed);
      unsigned v = (unsigned)__clz(h) + 1u;
      if (v > 32u - LOGP + 1u) v = 32u - LOGP + 1u;
      atomicMax(&regs[warp][h & (M - 1)], v);
    }
    __syncwarp();
    for (int i = lane; i < M; i += 32) sk[r * M + i] = (uint8_t)regs[warp][i];
    __syncwarp();
  }
}

// HLL sketch union over A entries [k0, k1) (warp-collective): lane l merges
// word (l % W) of the sketches of every (32 / W)-th entry with a packed
// per-byte maximum, four entries' loads in flight per pass. The lane's word
// is returned unreduced across the lanes that share it.
template <typename RP, int LOGP>
__device__ __forceinline__ unsigned hll_merge_part(const Csr<RP>& A, const uint8_t* __restrict__ sk, uint64_t k0,
                                                   uint64_t k1) {
  constexpr int M = 1 << LOGP;
  constexpr int W = M / 4;   // 32-bit words per sketch
  constexpr int G = 32 / W;  // A entries merged per step
  const int lane = threadIdx.x & 31;
  unsigned acc = 0u;
  for (uint64_t k = k0 + lane / W; k < k1; k += 4 * G) {
    uint32_t j[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) j[u] = k + (uint64_t)u * G < k1 ? A.col[k + (uint64_t)u * G] : kEmpty;
#pragma unroll
    for (int u = 0; u < 4; ++u)
      if (j[u] != kEmpty) acc = __vmaxu4(acc, reinterpret_cast<const unsigned*>(sk + (uint64_t)j[u] * M)[lane % W]);
  }
  return acc;
}

// Raw HLL estimate from the lanes' words (warp-collective; every lane gets the
// result): xor shuffles finish the union, the harmonic sum runs over the lanes
// that own a word, with the small-range correction.
template <int LOGP>
__device__ __forceinline__ int hll_finish(unsigned acc) {
  constexpr int M = 1 << LOGP;
  constexpr int W = M / 4;
  constexpr double kAlpha = LOGP == 4 ? 0.673 : (LOGP == 5 ? 0.697 : (LOGP == 6 ? 0.709 : 0.715));
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = W; o < 32; o <<= 1) acc = __vmaxu4(acc, __shfl_xor_sync(kFull, acc, o));
  double z = 0.0;
  int zeros = 0;
  if (lane < W) {
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int v = (acc >> (8 * b)) & 0xFF;
      z += ldexp(1.0, -v);
      zeros += v == 0;
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    z += __shfl_xor_sync(kFull, z, o);
    zeros += __shfl_xor_sync(kFull, zeros, o);
  }
  int result = (int)(kAlpha * M * M / z);
  if (zeros != 0 && result < 2.5 * M) result = (int)(M * log((double)M / (double)zeros));
  return result;
}

// Raw HLL estimate of the output size of A row `row` (warp-collective; every
// lane gets the result).
template <typename RP, int LOGP>
__device__ __forceinline__ int hll_row_estimate(const Csr<RP>& A, const uint8_t* __restrict__ sk, uint64_t row) {
  return hll_finish<LOGP>(hll_merge_part<RP, LOGP>(A, sk, A.row_begin(row), A.row_end(row)));
}

// A row's sizing value from its raw HLL estimate: raw_only, the raw value;
// otherwise raw x expansion, at least 1 and at most min(products, column span).
__device__ __forceinline__ uint32_t hll_value(int raw, uint32_t p, uint32_t lo, uint32_t hi, double expansion,
                                              int raw_only) {
  if (raw_only) return raw > 0 ? (uint32_t)raw : 0u;
  const uint64_t span = (uint64_t)hi - lo + 1;
  double e = ceil((double)raw * expansion);
  if (e < 1.0) e = 1.0;
  uint64_t v = (uint64_t)e;
  v = v < p ? v : p;
  v = v < span ? v : span;
  return (uint32_t)v;
}

// Estimated output count of every A row for the estimation workflow: rows of at
// most esc_max products get their product count (an exact upper bound, they run
// in the register classes); others the HLL estimate times `expansion`, at least
// 1 and at most min(products, column span), or (raw_only) the raw HLL
// estimate. Rows that the analysis listed as long (long_acc set) are left to
// k_hll_estimate_long.
template <typename RP, int LOGP>
__global__ void __launch_bounds__(256) k_hll_estimate(Csr<RP> A, const uint8_t* __restrict__ sk,
                                                      const uint32_t* __restrict__ prod,
                                                      const uint32_t* __restrict__ lo,
                                                      const uint32_t* __restrict__ hi, uint32_t* __restrict__ est,
                                                      double expansion, uint32_t esc_max, int raw_only,
                                                      const LongRowAcc* __restrict__ long_acc) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t r = (uint64_t)blockIdx.x * 8 + warp; r < A.rows; r += (uint64_t)gridDim.x * 8) {
    const uint32_t p = prod[r];
    if (p <= esc_max) {  // warp-uniform
      if (lane == 0) est[r] = p;
      continue;
    }
    if (long_acc && A.row_end(r) - A.row_begin(r) > kLongRowEntries) continue;
    const int raw = hll_row_estimate<RP, LOGP>(A, sk, r);
    if (lane == 0) est[r] = hll_value(raw, p, lo[r], hi[r], expansion, raw_only);
  }
}

// HLL estimates of the listed long rows: the warps of the grid stride over
// the chunk ids (as in k_analysis_long), merge each chunk's union into the
// row's registers with per-register atomicMax, and the warp that finishes the
// row's last chunk computes the row's estimate.
template <typename RP, int LOGP>
__global__ void __launch_bounds__(256, 8) k_hll_estimate_long(Csr<RP> A, const uint8_t* __restrict__ sk,
                                                           const uint32_t* __restrict__ prod,
                                                           const uint32_t* __restrict__ lo,
                                                           const uint32_t* __restrict__ hi,
                                                           uint32_t* __restrict__ est, double expansion,
                                                           uint32_t esc_max, int raw_only,
                                                           const DevCounters* __restrict__ ctr,
                                                           const uint32_t* __restrict__ long_rows,
                                                           LongRowAcc* __restrict__ long_acc, uint32_t long_cap,
                                                           const uint32_t* __restrict__ long_chunk_row,
                                                           uint32_t chunk_cap) {
  constexpr int W = (1 << LOGP) / 4;
  const uint32_t total = min(ctr->long_chunks, chunk_cap);
  const uint32_t nl = min(ctr->num_long, long_cap);
  const int lane = threadIdx.x & 31;
  const uint32_t nw = gridDim.x * (blockDim.x >> 5);
  for (uint32_t c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < total; c += nw) {
    const uint32_t i = long_chunk_row[c];
    if (i >= nl) continue;  // (a row that did not fit the map: flagged by the analysis)
    LongRowAcc& L = long_acc[i];
    const uint32_t row = long_rows[i];
    const uint32_t p = prod[row];
    if (p <= esc_max) continue;  // sized by k_hll_estimate
    const uint64_t a0 = A.row_begin(row), a1 = A.row_end(row);
    const uint32_t nch = (uint32_t)((a1 - a0 + kLongChunk - 1) / kLongChunk);
    if (c - L.base >= nch) continue;
    const uint64_t c0 = a0 + (uint64_t)(c - L.base) * kLongChunk;
    unsigned acc = hll_merge_part<RP, LOGP>(A, sk, c0, min(a1, c0 + kLongChunk));
#pragma unroll
    for (int o = W; o < 32; o <<= 1) acc = __vmaxu4(acc, __shfl_xor_sync(kFull, acc, o));
    if (lane < W) {
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const unsigned v = (acc >> (8 * b)) & 0xFFu;
        if (v) atomicMax(&L.reg[lane * 4 + b], v);
      }
    }
    __threadfence();
    __syncwarp();
    unsigned last = 0;
    if (lane == 0) last = atomicAdd(&L.hdone, 1u) == nch - 1;
    last = __shfl_sync(kFull, last, 0);
    if (last) {
      // every chunk of the row is merged: read the registers and leave them
      // (and the counter) zeroed for a later estimate after the same analysis
      __threadfence();
      unsigned word = 0u;
      if (lane < W) {
#pragma unroll
        for (int b = 0; b < 4; ++b) word |= (atomicExch(&L.reg[lane * 4 + b], 0u) & 0xFFu) << (8 * b);
      }
      const int raw = hll_finish<LOGP>(word);
      if (lane == 0) {
        est[row] = hll_value(raw, p, lo[row], hi[row], expansion, raw_only);
        atomicExch(&L.hdone, 0u);
      }
    }
  }
}

// Compaction statistics of the LCG-sampled rows (reference: kernels/HLL.cuh:239-357;
// sample i takes row ((1664525 x + 1013904223) mod 2^32) mod rows with
// x = 112233 + i * 2654435761). Rows without products or with a zero estimate
// are skipped (their ratio is undefined).
template <typename RP, int LOGP>
__global__ void __launch_bounds__(256) k_hll_sample(Csr<RP> A, const uint8_t* __restrict__ sk,
                                                    const uint32_t* __restrict__ prod, unsigned samples,
                                                    DevCounters* __restrict__ ctr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (uint64_t i = (uint64_t)blockIdx.x * 8 + warp; i < samples; i += (uint64_t)gridDim.x * 8) {
    uint64_t x = 112233ull + i * 2654435761ull;
    x = (1664525ull * x + 1013904223ull) % (1ull << 32);
    const uint64_t row = x % A.rows;
    const uint32_t p = prod[row];
    if (p == 0) continue;
    const int raw = hll_row_estimate<RP, LOGP>(A, sk, row);
    if (lane == 0 && raw > 0) {
      atomicAdd(&ctr->sample_rows, 1u);
      atomicAdd(&ctr->sample_products, (unsigned long long)p);
      atomicAdd(&ctr->sample_est, (double)raw);
      atomicAdd(&ctr->sample_compaction, (double)p / (double)raw);
    }
  }
}

// Estimation-workflow epilogue: rows that fit their estimate are copied from
// the temporary output (slots at src_off) to C (dst_off). A block takes 256
// consecutive rows, scans their counts and deals the tile's entries out to its
// threads in order, each finding its row by a search of the tile's inclusive
// offsets in shared memory: loads and stores stay coalesced across row ends
// and the work per thread does not depend on the row lengths (rows of a few
// dozen entries left most lanes of a warp-per-row copy idle).
__global__ void __launch_bounds__(256) k_copy_rows(uint64_t rows, const uint64_t* __restrict__ src_off,
                                                   const uint32_t* __restrict__ cap,
                                                   const uint32_t* __restrict__ cnt,
                                                   const uint64_t* __restrict__ dst_off,
                                                   const uint32_t* __restrict__ t_col,
                                                   const double* __restrict__ t_val, uint32_t* __restrict__ c_col,
                                                   double* __restrict__ c_val, const unsigned* __restrict__ stop) {
  if (stop && (*stop & DEV_BATCH_MISMATCH)) return;
  __shared__ unsigned long long s_incl[256];
  __shared__ uint64_t s_src[256], s_dst[256];
  __shared__ unsigned long long scr[33];
  const int tid = threadIdx.x;
  for (uint64_t r0 = (uint64_t)blockIdx.x * 256; r0 < rows; r0 += (uint64_t)gridDim.x * 256) {
    const uint64_t r = r0 + tid;
    uint32_t n = 0;
    if (r < rows) {
      n = cnt[r];
      if (n == kUnknownCount || n > cap[r]) n = 0;
    }
    s_src[tid] = n ? src_off[r] : 0ull;
    s_dst[tid] = n ? dst_off[r] : 0ull;
    unsigned long long total;
    const unsigned long long ex = block_excl_scan<256, unsigned long long>(n, scr, &total);
    s_incl[tid] = ex + n;
    __syncthreads();
    int t = 0;  // row of the previous entry: entries ascend, so rows do too
    for (unsigned long long e = tid; e < total; e += 256) {
      int lo = t, hi = 255;  // first row whose inclusive offset exceeds e
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (s_incl[mid] <= e) lo = mid + 1;
        else hi = mid;
      }
      t = lo;
      const unsigned long long k = e - (t ? s_incl[t - 1] : 0ull);
      c_col[s_dst[t] + k] = t_col[s_src[t] + k];
      c_val[s_dst[t] + k] = t_val[s_src[t] + k];
    }
    __syncthreads();
  }
}

// out[r] = min(products, column span) of row r: an exact upper bound of its
// output count (0 for rows without products).
__global__ void __launch_bounds__(256) k_row_bounds(uint64_t rows, const uint32_t* __restrict__ prod,
                                                    const uint32_t* __restrict__ lo,
                                                    const uint32_t* __restrict__ hi, uint32_t* __restrict__ out) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t p = prod[r];
    const uint64_t span = p ? (uint64_t)hi[r] - lo[r] + 1 : 0;
    out[r] = (uint32_t)(p < span ? p : span);
  }
}

// ---------------------------------------------------------------- launchers
namespace {
constexpr size_t kNumBitmapSmem = sizeof(BitmapNumSmem);
constexpr size_t kWinNumSmem = sizeof(WinNumSmem);
constexpr size_t kSymBitmapSmem = sizeof(BitmapSymSmem);
template <int NT, int LOG2T>
constexpr size_t num_hash_smem() { return sizeof(NumHashSmem<NT, LOG2T>); }
template <int NT, int LOG2T>
constexpr size_t sym_hash_smem() { return sizeof(SymHashSmem<NT, LOG2T>); }

int g_occ[24];  // resident blocks per SM of each persistent kernel (same order as kinds)
enum Kind { K_SYM_ESC1, K_SYM_ESC2, K_SYM_ESC4, K_SYM_S, K_SYM_M, K_SYM_L, K_SYM_BM,
            K_NUM_ESC1, K_NUM_ESC2, K_NUM_ESC4, K_NUM_S, K_NUM_M, K_NUM_L, K_NUM_BM, K_NUM_WIN };

template <typename F>
int occ_of(F f, int threads, size_t smem) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, f, threads, smem) != cudaSuccess || n < 1) n = 1;
  return n;
}

template <typename K>
void allow_smem(K k, size_t bytes) {
  cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <typename RP>
void set_attrs() {
  allow_smem(k_sym_bitmap<RP>, kSymBitmapSmem);
  allow_smem(k_num_bitmap<RP>, kNumBitmapSmem);
  allow_smem(k_num_window<RP>, kWinNumSmem);
  allow_smem(k_usp_fused<RP>, sizeof(UspSmem));
  allow_smem(k_sym_hash<RP, 128, 11>, sym_hash_smem<128, 11>());
  allow_smem(k_sym_hash<RP, 256, 13>, sym_hash_smem<256, 13>());
  allow_smem(k_sym_hash<RP, 512, 15>, sym_hash_smem<512, 15>());
  allow_smem(k_num_hash<RP, 128, 10>, num_hash_smem<128, 10>());
  allow_smem(k_num_hash<RP, 256, 12>, num_hash_smem<256, 12>());
  allow_smem(k_num_hash<RP, 512, 13>, num_hash_smem<512, 13>());
}
}  // namespace

void configure_kernel_attributes() {
  set_attrs<uint32_t>();
  set_attrs<uint64_t>();
  g_occ[K_SYM_ESC1] = occ_of(k_sym_esc<uint32_t, 1>, 256, 0);
  g_occ[K_SYM_ESC2] = occ_of(k_sym_esc<uint32_t, 2>, 256, 0);
  g_occ[K_SYM_ESC4] = occ_of(k_sym_esc<uint32_t, 4>, 256, 0);
  g_occ[K_SYM_S] = occ_of(k_sym_hash<uint32_t, 128, 11>, 128, sym_hash_smem<128, 11>());
  g_occ[K_SYM_M] = occ_of(k_sym_hash<uint32_t, 256, 13>, 256, sym_hash_smem<256, 13>());
  g_occ[K_SYM_L] = occ_of(k_sym_hash<uint32_t, 512, 15>, 512, sym_hash_smem<512, 15>());
  g_occ[K_SYM_BM] = occ_of(k_sym_bitmap<uint32_t>, kBitmapThreads, kSymBitmapSmem);
  g_occ[K_NUM_ESC1] = occ_of(k_num_esc<uint32_t, 1>, 256, 0);
  g_occ[K_NUM_ESC2] = occ_of(k_num_esc<uint32_t, 2>, 256, 0);
  g_occ[K_NUM_ESC4] = occ_of(k_num_esc<uint32_t, 4>, 256, 0);
  g_occ[K_NUM_S] = occ_of(k_num_hash<uint32_t, 128, 10>, 128, num_hash_smem<128, 10>());
  g_occ[K_NUM_M] = occ_of(k_num_hash<uint32_t, 256, 12>, 256, num_hash_smem<256, 12>());
  g_occ[K_NUM_L] = occ_of(k_num_hash<uint32_t, 512, 13>, 512, num_hash_smem<512, 13>());
  g_occ[K_NUM_BM] = occ_of(k_num_bitmap<uint32_t>, kBitmapThreads, kNumBitmapSmem);
  g_occ[K_NUM_WIN] = occ_of(k_num_window<uint32_t>, kBitmapThreads, kWinNumSmem);
}

namespace {
std::mutex g_attr_mutex;
bool g_attr_done[64] = {false};
}  // namespace

bool ensure_kernel_attributes(int dev) {
  std::lock_guard<std::mutex> lock(g_attr_mutex);
  if (dev < 0 || dev >= 64) return false;
  if (!g_attr_done[dev]) {
    configure_kernel_attributes();
    g_attr_done[dev] = true;
  }
  return true;
}

size_t window_scratch_words(int num_sms) { return (size_t)num_sms * (size_t)g_occ[K_NUM_WIN] * kBitmapWords; }

template <typename RP>
int launch_analysis(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, const SymPolicy& pol,
                    cudaStream_t s, const SymPolicy* seg) {
  if (A.rows == 0) return 0;
  SymPolicySet pols;
  for (int i = 0; i < kPolicySlots; ++i) pols.p[i] = (i > 0 && seg) ? seg[i - 1] : pol;
  const uint8_t* row_pol = seg ? w.row_pol : nullptr;
  // lanes per row: the smallest power of two (at least 4) whose pass of 4
  // entries per lane covers the mean row length; one row per 4 lanes measured
  // fastest on short rows (fewer threads, less per-row overhead)
  const double avg = (double)A.nnz / (double)A.rows;
  const int g = avg <= 16.0 ? 4 : avg <= 32.0 ? 8 : avg <= 64.0 ? 16 : 32;
  const uint64_t per_block = 256 / g;
  const unsigned blocks = (unsigned)((A.rows + per_block - 1) / per_block);
  int launched = 0;
  // the row table of B pays from about a million entries of B (on the 256x256
  // Laplacian, 0.33 M entries, its extra launch costs more than it saves)
  const uint4* btab = (w.btab && B.nnz >= (1ull << 20)) ? w.btab : nullptr;
  if (btab) {
    k_brow_table<RP><<<(unsigned)std::min<uint64_t>((B.rows + 255) / 256, 148ull * 16), 256, 0, s>>>(B, w.btab);
    ++launched;
  }
#define OCEAN_ANALYSIS(G)                                                                                          \
  k_analysis<RP, G><<<blocks, 256, 0, s>>>(A, B, w.prod, w.lo, w.hi, w.anz, w.maxb, w.row_nnz, w.bm_off, w.sym_bins, \
                                           w.ctr, pols, row_pol, w.long_rows, w.long_acc, w.long_cap, w.long_chunk_row, \
                                           w.long_chunk_cap, btab)
  if (g == 32) OCEAN_ANALYSIS(32);
  else if (g == 16) OCEAN_ANALYSIS(16);
  else if (g == 8) OCEAN_ANALYSIS(8);
  else OCEAN_ANALYSIS(4);
#undef OCEAN_ANALYSIS
  ++launched;
  if (w.long_acc) {
    k_analysis_long<RP><<<kLongGrid, 256, 0, s>>>(A, B, w.prod, w.lo, w.hi, w.anz, w.maxb, w.row_nnz, w.bm_off,
                                                w.sym_bins, w.ctr, pols, row_pol, w.long_rows, w.long_acc, w.long_cap,
                                                w.long_chunk_row, w.long_chunk_cap, btab);
    ++launched;
  }
  return launched;
}

// Grid of a persistent class kernel: resident blocks on all SMs, capped by
// the class's work items (rows, or warps of rows for warp kernels).
inline unsigned class_grid(int num_sms, int occ, const unsigned* counts, int cls, unsigned rows_per_block) {
  const unsigned full = (unsigned)(num_sms * occ);
  if (!counts) return full;
  const unsigned need = (counts[cls] + rows_per_block - 1) / rows_per_block;
  return need < full ? need : full;
}

template <typename RP>
int launch_symbolic(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, int num_sms, cudaStream_t s,
                    cudaEvent_t* ev, const unsigned* counts) {
  if (A.rows == 0) return 0;
  int launched = 0;
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], s);
  };
  auto grid = [&](int kind, int cls, unsigned per_block) {
    return class_grid(num_sms, g_occ[kind], counts, cls, per_block);
  };
  auto queue = [&](int c) {
    return RowQueue{w.sym_bins + (uint64_t)c * A.rows, w.ctr->sym_count + c, w.ctr->sym_cursor + c};
  };
  unsigned gsz;
  mark(SB_ESC1);
  if ((gsz = grid(K_SYM_ESC1, SB_ESC1, 8)) && ++launched)
    k_sym_esc<RP, 1><<<gsz, 256, 0, s>>>(A, B, queue(SB_ESC1), w.ctr, w.row_nnz);
  mark(SB_ESC2);
  if ((gsz = grid(K_SYM_ESC2, SB_ESC2, 8)) && ++launched)
    k_sym_esc<RP, 2><<<gsz, 256, 0, s>>>(A, B, queue(SB_ESC2), w.ctr, w.row_nnz);
  mark(SB_ESC4);
  if ((gsz = grid(K_SYM_ESC4, SB_ESC4, 8)) && ++launched)
    k_sym_esc<RP, 4><<<gsz, 256, 0, s>>>(A, B, queue(SB_ESC4), w.ctr, w.row_nnz);
  mark(SB_HASH_S);
  if ((gsz = grid(K_SYM_S, SB_HASH_S, 1)) && ++launched)
    k_sym_hash<RP, 128, 11><<<gsz, 128, sym_hash_smem<128, 11>(), s>>>(A, B, queue(SB_HASH_S), w.ctr, w.prod,
                                                                       w.lo, w.hi, w.row_nnz);
  mark(SB_HASH_M);
  if ((gsz = grid(K_SYM_M, SB_HASH_M, 1)) && ++launched)
    k_sym_hash<RP, 256, 13><<<gsz, 256, sym_hash_smem<256, 13>(), s>>>(A, B, queue(SB_HASH_M), w.ctr, w.prod,
                                                                       w.lo, w.hi, w.row_nnz);
  mark(SB_HASH_L);
  if ((gsz = grid(K_SYM_L, SB_HASH_L, 1)) && ++launched)
    k_sym_hash<RP, 512, 15><<<gsz, 512, sym_hash_smem<512, 15>(), s>>>(A, B, queue(SB_HASH_L), w.ctr, w.prod,
                                                                       w.lo, w.hi, w.row_nnz);
  mark(SB_BITMAP);
  if ((gsz = grid(K_SYM_BM, SB_BITMAP, 1)) && ++launched)
    k_sym_bitmap<RP><<<gsz, kBitmapThreads, kSymBitmapSmem, s>>>(A, B, queue(SB_BITMAP), w.ctr, w.prod, w.lo, w.hi,
                                                                 w.row_nnz, w.bm_off, w.bm_cache, w.bm_cache_words,
                                                                 false);
  mark(SB_COUNT);
  return launched;
}

int launch_scan(const DevWork& w, const uint32_t* in, uint64_t* out64, uint32_t* out32,
                unsigned long long* total, bool bin_rows, const NumPolicy& pol, cudaStream_t s,
                const NumPolicy* seg) {
  const uint64_t nt = scan_tiles(w.rows);
  if (w.rows == 0) return 0;
  NumPolicySet pols;
  for (int i = 0; i < kPolicySlots; ++i) pols.p[i] = (i > 0 && seg) ? seg[i - 1] : pol;
  const uint8_t* row_pol = seg ? w.row_pol : nullptr;
  k_scan_reduce<<<(unsigned)nt, 1024, 0, s>>>(in, w.rows, w.tile_sums);
  k_scan_tiles<<<1, 1024, 0, s>>>(w.tile_sums, nt, total, out64, out32, w.rows);
  const int chunks = bin_rows ? w.chunks : 0;
  k_scan_apply<<<(unsigned)nt, kScanApplyThreads, 0, s>>>(in, w.rows, w.tile_sums, out64, out32, w.prod, w.lo, w.hi, w.anz,
                                             w.bm_off, w.num_bins, w.ctr, pols, row_pol, bin_rows ? 1 : 0, chunks,
                                             w.chunk_bound, w.chunk_count);
  return 3;
}

// bound[k] = first row r with prefix[r] >= ceil(k * total / chunks), by binary
// search; bound[0] = 0, bound[chunks] = rows. One thread per bound.
__global__ void k_chunk_bounds(const uint64_t* __restrict__ prefix, uint64_t rows, int chunks,
                               uint32_t* __restrict__ bound) {
  const int k = threadIdx.x;
  if (k > chunks) return;
  const uint64_t total = prefix[rows];
  if (k == 0 || k == chunks) {
    bound[k] = k == 0 ? 0u : (uint32_t)rows;
    return;
  }
  const uint64_t target = (total * (uint64_t)k + chunks - 1) / chunks;
  uint64_t lo = 0, hi = rows;  // first r in [0, rows] with prefix[r] >= target
  while (lo < hi) {
    const uint64_t mid = (lo + hi) >> 1;
    if (prefix[mid] < target) lo = mid + 1;
    else hi = mid;
  }
  bound[k] = (uint32_t)lo;
}

void launch_chunk_bounds(const DevWork& w, const uint64_t* prefix, int chunks, cudaStream_t s) {
  k_chunk_bounds<<<1, 32, 0, s>>>(prefix, w.rows, chunks, w.chunk_bound);
}

template <typename RP>
int launch_numeric(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, const OutSpec& o, uint32_t* c_col,
                   double* c_val, int num_sms, cudaStream_t s, cudaEvent_t* ev, const unsigned* counts, int chunk,
                   uint32_t row_base) {
  if (A.rows == 0) return 0;
  int launched = 0;
  auto mark = [&](int i) {
    if (ev) cudaEventRecord(ev[i], s);
  };
  auto grid = [&](int kind, int cls, unsigned per_block) {
    return class_grid(num_sms, g_occ[kind], counts, cls, per_block);
  };
  const bool chunked = chunk >= 0 && w.chunks > 1;
  auto queue = [&](int c) {
    if (chunked) {
      const int slot = c * w.chunks + chunk;
      return RowQueue{w.num_bins + (uint64_t)c * A.rows + row_base, w.chunk_count + slot, w.chunk_cursor + slot};
    }
    return RowQueue{w.num_bins + (uint64_t)c * A.rows, w.ctr->num_count + c, w.ctr->num_cursor + c};
  };
  unsigned gsz;
  mark(NB_ESC1);
  if ((gsz = grid(K_NUM_ESC1, NB_ESC1, 8)) && ++launched)
    k_num_esc<RP, 1><<<gsz, 256, 0, s>>>(A, B, queue(NB_ESC1), o, w.ctr, c_col, c_val);
  mark(NB_ESC2);
  if ((gsz = grid(K_NUM_ESC2, NB_ESC2, 8)) && ++launched)
    k_num_esc<RP, 2><<<gsz, 256, 0, s>>>(A, B, queue(NB_ESC2), o, w.ctr, c_col, c_val);
  mark(NB_ESC4);
  if ((gsz = grid(K_NUM_ESC4, NB_ESC4, 8)) && ++launched)
    k_num_esc<RP, 4><<<gsz, 256, 0, s>>>(A, B, queue(NB_ESC4), o, w.ctr, c_col, c_val);
  mark(NB_HASH_S);
  if ((gsz = grid(K_NUM_S, NB_HASH_S, 1)) && ++launched)
    k_num_hash<RP, 128, 10><<<gsz, 128, num_hash_smem<128, 10>(), s>>>(A, B, queue(NB_HASH_S), o, w.ctr, w.prod,
                                                                       w.lo, w.hi, c_col, c_val);
  mark(NB_HASH_M);
  if ((gsz = grid(K_NUM_M, NB_HASH_M, 1)) && ++launched)
    k_num_hash<RP, 256, 12><<<gsz, 256, num_hash_smem<256, 12>(), s>>>(A, B, queue(NB_HASH_M), o, w.ctr, w.prod,
                                                                       w.lo, w.hi, c_col, c_val);
  mark(NB_HASH_L);
  if ((gsz = grid(K_NUM_L, NB_HASH_L, 1)) && ++launched)
    k_num_hash<RP, 512, 13><<<gsz, 512, num_hash_smem<512, 13>(), s>>>(A, B, queue(NB_HASH_L), o, w.ctr, w.prod,
                                                                       w.lo, w.hi, c_col, c_val);
  mark(NB_BITMAP);
  const bool windowed = !o.count && w.win_cursor && w.win_scratch;
  if (windowed) {
    // rows up to 2^20 columns wide in the windowed kernel, wider ones in
    // k_num_bitmap (own queue cursor), launched only when there are any
    if ((gsz = grid(K_NUM_WIN, NB_BITMAP, 1)) && ++launched)
      k_num_window<RP><<<gsz, kBitmapThreads, kWinNumSmem, s>>>(A, B, queue(NB_BITMAP), o, w.ctr, w.lo, w.hi,
                                                                w.bm_off, w.bm_cache, w.win_scratch, w.win_cursor,
                                                                c_col, c_val);
    if (w.wide_rows && (gsz = grid(K_NUM_BM, NB_BITMAP, 1)) && ++launched) {
      const RowQueue wq{w.num_bins + (uint64_t)NB_BITMAP * A.rows, w.ctr->num_count + NB_BITMAP,
                        &w.ctr->wide_cursor};
      k_num_bitmap<RP><<<gsz, kBitmapThreads, kNumBitmapSmem, s>>>(A, B, wq, o, w.ctr, w.prod, w.lo, w.hi,
                                                                   w.bm_off, w.bm_cache, c_col, c_val, true);
    }
  } else if ((gsz = grid(K_NUM_BM, NB_BITMAP, 1)) && ++launched) {
    k_num_bitmap<RP><<<gsz, kBitmapThreads, kNumBitmapSmem, s>>>(A, B, queue(NB_BITMAP), o, w.ctr, w.prod, w.lo,
                                                                 w.hi, w.bm_off, w.bm_cache, c_col, c_val, false);
  }
  mark(NB_COUNT);
  return launched;
}

template <typename RP>
int launch_usp_fused(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, unsigned long long* tiles, uint64_t cap,
                     bool rowptr32, uint32_t* c_col, double* c_val, cudaStream_t s) {
  if (A.rows == 0) return 0;
  const uint64_t ntiles = (A.rows + kUspWarps - 1) / kUspWarps;
  cudaMemsetAsync(tiles, 0, ntiles * sizeof(unsigned long long), s);
  k_usp_fused<RP><<<(unsigned)ntiles, kUspWarps * 32, sizeof(UspSmem), s>>>(
      A, B, tiles, w.ctr, cap, w.rowptr64, rowptr32 ? w.rowptr32 : nullptr, c_col, c_val);
  return 1;
}

uint64_t usp_tiles(uint64_t rows) { return (rows + kUspWarps - 1) / kUspWarps; }

int launch_row_bounds(const DevWork& w, uint32_t* out, cudaStream_t s) {
  if (w.rows == 0) return 0;
  const uint64_t blocks = std::min<uint64_t>((w.rows + 255) / 256, 148ull * 16);
  k_row_bounds<<<(unsigned)blocks, 256, 0, s>>>(w.rows, w.prod, w.lo, w.hi, out);
  return 1;
}

void launch_murmur3(const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t seed, cudaStream_t s) {
  if (n == 0) return;
  const uint64_t blocks = (n + 255) / 256;
  k_murmur3<<<(unsigned)(blocks > 4096 ? 4096 : blocks), 256, 0, s>>>(keys, out, n, seed);
}

template <typename RP>
int launch_hll_sketch_sample(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, int log2p, unsigned sample_rows,
                             uint8_t* sketch, cudaStream_t s) {
  if (A.rows == 0) return 0;
  const unsigned gb = (unsigned)std::min<uint64_t>((B.rows + 7) / 8, 65535u * 8);
  const unsigned gs = (sample_rows + 7) / 8;
  int n = 0;
  if (log2p == 5) {
    if (B.rows) k_hll_sketch<RP, 5><<<gb, 256, 0, s>>>(B, sketch), ++n;
    if (gs) k_hll_sample<RP, 5><<<gs, 256, 0, s>>>(A, sketch, w.prod, sample_rows, w.ctr), ++n;
  } else {
    if (B.rows) k_hll_sketch<RP, 6><<<gb, 256, 0, s>>>(B, sketch), ++n;
    if (gs) k_hll_sample<RP, 6><<<gs, 256, 0, s>>>(A, sketch, w.prod, sample_rows, w.ctr), ++n;
  }
  return n;
}

template <typename RP>
int launch_hll_rows(const Csr<RP>& A, const DevWork& w, int log2p, double expansion, uint32_t esc_max, bool raw,
                    const uint8_t* sketch, uint32_t* out, cudaStream_t s) {
  if (A.rows == 0) return 0;
  const unsigned ga = (unsigned)std::min<uint64_t>((A.rows + 7) / 8, 65535u * 8);
  const int ro = raw ? 1 : 0;
  if (log2p == 5)
    k_hll_estimate<RP, 5><<<ga, 256, 0, s>>>(A, sketch, w.prod, w.lo, w.hi, out, expansion, esc_max, ro, w.long_acc);
  else
    k_hll_estimate<RP, 6><<<ga, 256, 0, s>>>(A, sketch, w.prod, w.lo, w.hi, out, expansion, esc_max, ro, w.long_acc);
  if (!w.long_acc) return 1;
  if (log2p == 5)
    k_hll_estimate_long<RP, 5><<<kLongGrid, 256, 0, s>>>(A, sketch, w.prod, w.lo, w.hi, out, expansion, esc_max, ro,
                                                       w.ctr, w.long_rows, w.long_acc, w.long_cap,
                                                       w.long_chunk_row, w.long_chunk_cap);
  else
    k_hll_estimate_long<RP, 6><<<kLongGrid, 256, 0, s>>>(A, sketch, w.prod, w.lo, w.hi, out, expansion, esc_max, ro,
                                                       w.ctr, w.long_rows, w.long_acc, w.long_cap,
                                                       w.long_chunk_row, w.long_chunk_cap);
  return 2;
}

void launch_copy_rows(const DevWork& w, const uint32_t* t_col, const double* t_val, uint32_t* c_col, double* c_val,
                      cudaStream_t s, const unsigned* stop) {
  if (w.rows == 0) return;
  const unsigned g = (unsigned)std::min<uint64_t>((w.rows + 255) / 256, 148u * 8u);
  k_copy_rows<<<g, 256, 0, s>>>(w.rows, w.est_off, w.est, w.cnt, w.rowptr64, t_col, t_val, c_col, c_val, stop);
}

template <typename RP>
int launch_overflow(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, bool numeric, uint32_t* c_col,
                    double* c_val, int num_sms, cudaStream_t s) {
  const RowQueue q{w.ovf, &w.ctr->overflow_n, w.ctr->overflow_cursor + (numeric ? 1 : 0)};
  if (!numeric) {
    k_sym_bitmap<RP><<<num_sms, kBitmapThreads, kSymBitmapSmem, s>>>(A, B, q, w.ctr, w.prod, w.lo, w.hi, w.cnt,
                                                                     w.bm_off, nullptr, 0, true);
  } else {
    const OutSpec o{w.rowptr64, w.cnt, nullptr, nullptr, nullptr};
    k_num_bitmap<RP><<<num_sms, kBitmapThreads, kNumBitmapSmem, s>>>(A, B, q, o, w.ctr, w.prod, w.lo, w.hi, w.bm_off,
                                                                     nullptr, c_col, c_val, false);
  }
  return 1;
}

template int launch_hll_sketch_sample<uint32_t>(const Csr<uint32_t>&, const Csr<uint32_t>&, const DevWork&, int,
                                                unsigned, uint8_t*, cudaStream_t);
template int launch_hll_sketch_sample<uint64_t>(const Csr<uint64_t>&, const Csr<uint64_t>&, const DevWork&, int,
                                                unsigned, uint8_t*, cudaStream_t);
template int launch_hll_rows<uint32_t>(const Csr<uint32_t>&, const DevWork&, int, double, uint32_t, bool,
                                       const uint8_t*, uint32_t*, cudaStream_t);
template int launch_hll_rows<uint64_t>(const Csr<uint64_t>&, const DevWork&, int, double, uint32_t, bool,
                                       const uint8_t*, uint32_t*, cudaStream_t);
template int launch_usp_fused<uint32_t>(const Csr<uint32_t>&, const Csr<uint32_t>&, const DevWork&,
                                        unsigned long long*, uint64_t, bool, uint32_t*, double*, cudaStream_t);
template int launch_usp_fused<uint64_t>(const Csr<uint64_t>&, const Csr<uint64_t>&, const DevWork&,
                                        unsigned long long*, uint64_t, bool, uint32_t*, double*, cudaStream_t);
template int launch_overflow<uint32_t>(const Csr<uint32_t>&, const Csr<uint32_t>&, const DevWork&, bool, uint32_t*,
                                       double*, int, cudaStream_t);
template int launch_overflow<uint64_t>(const Csr<uint64_t>&, const Csr<uint64_t>&, const DevWork&, bool, uint32_t*,
                                       double*, int, cudaStream_t);
template int launch_analysis<uint32_t>(const Csr<uint32_t>&, const Csr<uint32_t>&, const DevWork&,
                                        const SymPolicy&, cudaStream_t, const SymPolicy*);
template int launch_analysis<uint64_t>(const Csr<uint64_t>&, const Csr<uint64_t>&, const DevWork&,
                                        const SymPolicy&, cudaStream_t, const SymPolicy*);
template int launch_symbolic<uint32_t>(const Csr<uint32_t>&, const Csr<uint32_t>&, const DevWork&, int,
                                        cudaStream_t, cudaEvent_t*, const unsigned*);
template int launch_symbolic<uint64_t>(const Csr<uint64_t>&, const Csr<uint64_t>&, const DevWork&, int,
                                        cudaStream_t, cudaEvent_t*, const unsigned*);
template int launch_numeric<uint32_t>(const Csr<uint32_t>&, const Csr<uint32_t>&, const DevWork&, const OutSpec&,
                                      uint32_t*, double*, int, cudaStream_t, cudaEvent_t*, const unsigned*, int,
                                      uint32_t);
template int launch_numeric<uint64_t>(const Csr<uint64_t>&, const Csr<uint64_t>&, const DevWork&, const OutSpec&,
                                      uint32_t*, double*, int, cudaStream_t, cudaEvent_t*, const unsigned*, int,
                                      uint32_t);

}  // namespace ocean
