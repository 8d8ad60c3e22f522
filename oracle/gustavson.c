/*
 * CPU oracle for the SpGEMM path — TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference
 * arm may load this code, and only as the checker or as the reported CPU
 * baseline, never as the thing measured or shipped.
 *
 * It restates the reference's output semantics for C = A·B on CSR/FP64
 * (the reference itself has no CPU implementation):
 *  - row i of C holds the union of the columns of B.row(k) over k in A.row(i),
 *    including structural zeros and products that cancel to exactly 0, like the
 *    reference's dense compaction (kernels/AccumulatorDense.cuh:208-219) and hash
 *    compaction (kernels/AccumulatorHash.cuh:462-466), which emit every touched
 *    column whatever its value;
 *  - columns are sorted ascending in each row (kernels/Epilogue.cuh:68-222);
 *  - empty B rows contribute nothing (kernels/Analysis.cuh:73);
 *  - the end of the last row is `nnz`, not rowptr[rows] (src/CSR.cpp:54);
 *  - values are sums of a_ik*b_kj in FP64, accumulated here in A-row order.
 * Row pointers are passed as uint64 (callers widen 32-bit ones).
 *
 * MurmurHash3 (32-bit, one 4-byte key) restates kernels/MurmurHash.cuh:44-98;
 * the HyperLogLog register rule and estimate restate kernels/HLL.cuh:11-24 and
 * kernels/HLL.cuh:107-236 (precision constants include/Common.h:51).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ROW_END(rp, r, rows, nnz) ((r) + 1 == (rows) ? (nnz) : (rp)[(r) + 1])

/* --------------------------------------------------------------- sorting */
static void sort_u32(uint32_t* a, uint32_t* tmp, uint64_t n, uint32_t maxv) {
  if (n < 48) {
    for (uint64_t i = 1; i < n; ++i) {
      uint32_t x = a[i];
      uint64_t j = i;
      while (j > 0 && a[j - 1] > x) {
        a[j] = a[j - 1];
        --j;
      }
      a[j] = x;
    }
    return;
  }
  int bits = 0;
  while (bits < 32 && (maxv >> bits)) ++bits;
  uint32_t* src = a;
  uint32_t* dst = tmp;
  for (int shift = 0; shift < bits; shift += 11) {
    uint64_t cnt[2048];
    memset(cnt, 0, sizeof cnt);
    for (uint64_t i = 0; i < n; ++i) cnt[(src[i] >> shift) & 2047]++;
    uint64_t run = 0;
    for (int d = 0; d < 2048; ++d) {
      uint64_t c = cnt[d];
      cnt[d] = run;
      run += c;
    }
    for (uint64_t i = 0; i < n; ++i) dst[cnt[(src[i] >> shift) & 2047]++] = src[i];
    uint32_t* t = src;
    src = dst;
    dst = t;
  }
  if (src != a) memcpy(a, src, n * sizeof(uint32_t));
}

/* --------------------------------------------------------------- row stats */
/* products per row, smallest and largest output column (UINT32_MAX / 0 if none) */
int oracle_row_stats(uint64_t a_rows, uint64_t a_nnz, const uint64_t* ap, const uint32_t* aj,
                     uint64_t b_rows, uint64_t b_nnz, const uint64_t* bp, const uint32_t* bj,
                     uint64_t* prod, uint32_t* lo, uint32_t* hi, int nthreads) {
#pragma omp parallel for schedule(dynamic, 256) num_threads(nthreads)
  for (uint64_t i = 0; i < a_rows; ++i) {
    uint64_t p = 0;
    uint32_t mn = 0xFFFFFFFFu, mx = 0;
    const uint64_t e = ROW_END(ap, i, a_rows, a_nnz);
    for (uint64_t k = ap[i]; k < e; ++k) {
      const uint32_t j = aj[k];
      const uint64_t b0 = bp[j], b1 = ROW_END(bp, j, b_rows, b_nnz);
      if (b1 > b0) {
        p += b1 - b0;
        if (bj[b0] < mn) mn = bj[b0];
        if (bj[b1 - 1] > mx) mx = bj[b1 - 1];
      }
    }
    prod[i] = p;
    lo[i] = mn;
    hi[i] = mx;
  }
  return 0;
}

/* --------------------------------------------------------------- symbolic */
/* exact output count of rows [r0, r1) into row_nnz[i - r0] */
int oracle_symbolic(uint64_t a_rows, uint64_t a_nnz, const uint64_t* ap, const uint32_t* aj,
                    uint64_t b_rows, uint64_t b_nnz, const uint64_t* bp, const uint32_t* bj, uint64_t b_cols,
                    uint64_t r0, uint64_t r1, uint64_t* row_nnz, int nthreads) {
  int err = 0;
#pragma omp parallel num_threads(nthreads)
  {
    uint64_t* mark = (uint64_t*)malloc((b_cols ? b_cols : 1) * sizeof(uint64_t));
    if (!mark) {
#pragma omp atomic write
      err = 1;
    } else {
      memset(mark, 0, (b_cols ? b_cols : 1) * sizeof(uint64_t));
#pragma omp for schedule(dynamic, 64)
      for (uint64_t i = r0; i < r1; ++i) {
        uint64_t n = 0;
        const uint64_t e = ROW_END(ap, i, a_rows, a_nnz);
        for (uint64_t k = ap[i]; k < e; ++k) {
          const uint32_t j = aj[k];
          const uint64_t b1 = ROW_END(bp, j, b_rows, b_nnz);
          for (uint64_t q = bp[j]; q < b1; ++q) {
            const uint32_t c = bj[q];
            if (mark[c] != i + 1) {
              mark[c] = i + 1;
              ++n;
            }
          }
        }
        row_nnz[i - r0] = n;
      }
      free(mark);
    }
  }
  return err;
}

/* --------------------------------------------------------------- numeric */
/* C rows [r0, r1): cp[i - r0] is the offset of row i inside cj/cx (cp has
 * r1 - r0 + 1 entries). cabs (optional) receives sum |a_ik * b_kj| per entry,
 * the scale of the value tolerance. Returns 1 on allocation failure, 2 when a
 * row's count disagrees with cp. */
int oracle_numeric(uint64_t a_rows, uint64_t a_nnz, const uint64_t* ap, const uint32_t* aj, const double* ax,
                   uint64_t b_rows, uint64_t b_nnz, const uint64_t* bp, const uint32_t* bj, const double* bx,
                   uint64_t b_cols, uint64_t r0, uint64_t r1, const uint64_t* cp, uint32_t* cj, double* cx,
                   double* cabs, int nthreads) {
  int err = 0;
#pragma omp parallel num_threads(nthreads)
  {
    const uint64_t nc = b_cols ? b_cols : 1;
    uint64_t* mark = (uint64_t*)calloc(nc, sizeof(uint64_t));
    double* acc = (double*)malloc(nc * sizeof(double));
    double* aacc = (double*)malloc(nc * sizeof(double));
    uint32_t* list = (uint32_t*)malloc(nc * sizeof(uint32_t));
    uint32_t* tmp = (uint32_t*)malloc(nc * sizeof(uint32_t));
    if (!mark || !acc || !aacc || !list || !tmp) {
#pragma omp atomic write
      err = 1;
    } else {
#pragma omp for schedule(dynamic, 64)
      for (uint64_t i = r0; i < r1; ++i) {
        uint64_t n = 0;
        uint32_t mx = 0;
        const uint64_t e = ROW_END(ap, i, a_rows, a_nnz);
        for (uint64_t k = ap[i]; k < e; ++k) {
          const uint32_t j = aj[k];
          const double a = ax[k];
          const uint64_t b1 = ROW_END(bp, j, b_rows, b_nnz);
          for (uint64_t q = bp[j]; q < b1; ++q) {
            const uint32_t c = bj[q];
            const double v = a * bx[q];
            if (mark[c] != i + 1) {
              mark[c] = i + 1;
              acc[c] = 0.0;
              aacc[c] = 0.0;
              list[n++] = c;
              if (c > mx) mx = c;
            }
            acc[c] += v;
            aacc[c] += fabs(v);
          }
        }
        const uint64_t off = cp[i - r0];
        if (cp[i - r0 + 1] - off != n) {
#pragma omp atomic write
          err = 2;
          continue;
        }
        sort_u32(list, tmp, n, mx);
        for (uint64_t t = 0; t < n; ++t) {
          const uint32_t c = list[t];
          cj[off + t] = c;
          cx[off + t] = acc[c];
          if (cabs) cabs[off + t] = aacc[c];
        }
      }
    }
    free(mark);
    free(acc);
    free(aacc);
    free(list);
    free(tmp);
  }
  return err;
}

/* --------------------------------------------------------------- MurmurHash3 */
static uint32_t rotl32(uint32_t x, int r) { return (x << r) | (x >> (32 - r)); }

/* 32-bit MurmurHash3 (Austin Appleby, public domain) of one 4-byte little-endian key. */
uint32_t oracle_murmur3_u32(uint32_t key, uint32_t seed) {
  uint32_t h = seed;
  uint32_t k = key * 0xcc9e2d51u;
  k = rotl32(k, 15);
  k *= 0x1b873593u;
  h ^= k;
  h = rotl32(h, 13);
  h = h * 5u + 0xe6546b64u;
  h ^= 4u; /* length in bytes */
  h ^= h >> 16;
  h *= 0x85ebca6bu;
  h ^= h >> 13;
  h *= 0xc2b2ae35u;
  h ^= h >> 16;
  return h;
}

void oracle_murmur3_batch(const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t seed) {
  for (uint64_t i = 0; i < n; ++i) out[i] = oracle_murmur3_u32(keys[i], seed);
}

/* --------------------------------------------------------------- HyperLogLog */
/* Register index = low log2p bits of the hash; register value = number of
 * leading zeros of the 32-bit hash + 1, capped at 32 - log2p + 1
 * (kernels/HLL.cuh:11-24). Sketch of every B row: out[r * 2^log2p + idx]. */
void oracle_hll_sketch_rows(uint64_t rows, uint64_t nnz, const uint64_t* rp, const uint32_t* col, int log2p,
                            uint32_t seed, uint8_t* out) {
  const uint32_t m = 1u << log2p;
  const uint32_t cap = 32u - (uint32_t)log2p + 1u;
  memset(out, 0, rows * m);
  for (uint64_t r = 0; r < rows; ++r) {
    const uint64_t e = ROW_END(rp, r, rows, nnz);
    for (uint64_t q = rp[r]; q < e; ++q) {
      const uint32_t h = oracle_murmur3_u32(col[q], seed);
      const uint32_t idx = h & (m - 1);
      uint32_t v = (h == 0 ? 32u : (uint32_t)__builtin_clz(h)) + 1u;
      if (v > cap) v = cap;
      if (out[r * m + idx] < v) out[r * m + idx] = (uint8_t)v;
    }
  }
}

/* Raw HLL cardinality estimate of the union of the B-row sketches selected by
 * one A row (kernels/HLL.cuh:161-219): E = alpha*m^2 / sum 2^-M[i], replaced by
 * m*ln(m/V) when some registers are empty and E < 2.5m. The reference takes
 * that log of a float quotient with -use_fast_math, so its integer estimate can
 * differ from this double-precision one by one; estimates only size buffers. */
int64_t oracle_hll_estimate_union(const uint8_t* sketches, int log2p, const uint32_t* rows, uint64_t nrows) {
  static const double kAlpha[8] = {0.0, 0.0, 0.0, 0.0, 0.673, 0.697, 0.709, 0.715};
  const uint32_t m = 1u << log2p;
  uint8_t reg[128];
  memset(reg, 0, sizeof reg);
  for (uint64_t t = 0; t < nrows; ++t)
    for (uint32_t i = 0; i < m; ++i) {
      const uint8_t v = sketches[(uint64_t)rows[t] * m + i];
      if (v > reg[i]) reg[i] = v;
    }
  double z = 0.0;
  int empty = 0;
  for (uint32_t i = 0; i < m; ++i) {
    z += 1.0 / (double)(1ull << reg[i]);
    empty += reg[i] == 0;
  }
  int64_t result = (int64_t)(kAlpha[log2p] * m * m / z);
  if (empty != 0 && result < 2.5 * m) result = (int64_t)(m * log((double)m / (double)empty));
  return result;
}
