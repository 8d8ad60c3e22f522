// Internal types and device helpers shared by the SpGEMM kernels.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ocean {

constexpr uint32_t kEmpty = 0xFFFFFFFFu;
constexpr unsigned kFull = 0xFFFFFFFFu;

// Bitmap accumulator window: 2^20 columns per pass (128 KB of bits in shared
// memory). A row whose output column span is wider is swept in several windows.
constexpr int kBitmapLog2 = 20;
constexpr uint64_t kBitmapBits = 1ull << kBitmapLog2;
constexpr int kBitmapWords = 1 << (kBitmapLog2 - 6);   // 64-bit words
constexpr int kBitmapThreads = 1024;
constexpr int kWordsPerThread = kBitmapWords / kBitmapThreads;  // 16
constexpr int kSuperWords = 1024;                       // words per rank superblock
constexpr int kSupers = kBitmapWords / kSuperWords;     // 16

// Row classes ("bins"). Symbolic classes are chosen from the product count and
// the column span, numeric classes from the exact output count.
enum SymBin : int {
  SB_ESC1 = 0,     // <= 32 products: one warp, 1 product per lane, register sort + distinct count
  SB_ESC2 = 1,     // <= 64 products: one warp, 2 per lane
  SB_ESC4 = 2,     // <= 128 products: one warp, 4 per lane
  SB_HASH_S = 3,   // hash set, 128 threads, 2048 slots
  SB_HASH_M = 4,   // hash set, 256 threads, 8192 slots
  SB_HASH_L = 5,   // hash set, 512 threads, 32768 slots
  SB_BITMAP = 6,   // bitmap over the column span, 1024 threads
  SB_COUNT = 7
};
enum NumBin : int {
  NB_ESC1 = 0,     // <= 32 products: one warp, register sort + segmented sum
  NB_ESC2 = 1,     // <= 64 products
  NB_ESC4 = 2,     // <= 128 products
  NB_HASH_S = 3,   // hash accumulate + sort, 128 threads, 1024 slots (<= 512 out)
  NB_HASH_M = 4,   // 256 threads, 4096 slots (<= 2048 out)
  NB_HASH_L = 5,   // 512 threads, 8192 slots (<= 4096 out)
  NB_BITMAP = 6,   // bitmap-rank accumulator, any size
  NB_COUNT = 7
};

// Device-side counters of one multiply (zeroed at the start of each call).
struct DevCounters {
  unsigned long long total_products;
  unsigned long long total_nnz;
  unsigned int max_products;
  unsigned int max_a_nnz;
  unsigned int sym_count[SB_COUNT];
  unsigned int sym_cursor[SB_COUNT];
  unsigned int num_count[NB_COUNT];
  unsigned int num_cursor[NB_COUNT];
  unsigned long long num_nnz[NB_COUNT];   // output entries per numeric class
  unsigned long long num_anz[NB_COUNT];   // A entries of the rows of each numeric class
  unsigned long long num_prod[NB_COUNT];  // products of the rows of each numeric class
  unsigned long long sym_anz[SB_COUNT];   // A entries of the rows of each symbolic class
  unsigned long long sym_prod[SB_COUNT];  // products of the rows of each symbolic class
  unsigned long long sym_words;           // bitmap words of single-window bitmap-class rows
  unsigned long long cache_cursor;        // words handed out from the bitmap cache
  unsigned long long total_est;           // estimation workflow: sum of the row-size estimates
  unsigned int overflow_n;                // estimation workflow: rows that did not fit their estimate
  unsigned int overflow_cursor[2];        // queue cursors of the overflow recount and rerun
  unsigned int sample_rows;               // HLL sampling: rows sampled
  unsigned long long sample_products;     // HLL sampling: products of the sampled rows
  double sample_est;                      // HLL sampling: raw estimates of the sampled rows
  double sample_compaction;               // HLL sampling: sum of products / estimate over samples
  unsigned int status;     // OR of DevError bits
  unsigned int err_row;
  unsigned int num_wide;     // numeric bitmap-class rows whose column span exceeds one 2^20-bit bitmap
  unsigned int wide_cursor;  // queue cursor of those rows' kernel (k_num_bitmap beside k_num_window)
  unsigned int usp_tile;     // fused ultra-sparse multiply: tiles handed out
  unsigned int num_long;     // rows of A listed as long (more than kLongRowEntries entries)
  unsigned int long_chunks;  // chunks of kLongChunk A entries of the listed rows
  unsigned int pad[1];
};

// Rows of A with more than kLongRowEntries entries are not summarised by one
// lane group in the analysis, nor merged by one warp in the HLL row estimate:
// one such row would keep its group busy long after every other row is done.
// The analysis lists them and gives each a contiguous range of chunk ids (one
// chunk = kLongChunk A entries) with a chunk -> row map; second kernels stride
// over the chunk ids with all warps, merge the chunks' partial results into
// the row's accumulator with atomics, and the warp that finishes a row's last
// chunk writes the row's result.
constexpr uint32_t kLongRowEntries = 512;
constexpr uint32_t kLongChunk = 256;
struct LongRowAcc {
  unsigned long long prod;  // sum of the referenced B-row lengths
  unsigned int lo, hi;      // smallest first column, largest last column
  unsigned int maxb;        // longest referenced B row
  unsigned int done;        // analysis chunks finished
  unsigned int hdone;       // HLL chunks finished
  unsigned int base;        // first chunk id of the row
  unsigned int reg[64];     // HLL registers (one per word), max-merged
};

enum DevError : unsigned int {
  DEV_TABLE_FULL = 1u,     // an open-addressing probe exceeded the table size
  DEV_BIN_OVERFLOW = 2u,   // a row did not fit the class it was placed in
  DEV_COUNT_MISMATCH = 4u,  // numeric output count differs from the symbolic count
  DEV_TC_TIMEOUT = 8u,      // a tensor-core completion wait gave up (bounded spin)
  DEV_BATCH_MISMATCH = 16u, // a batch run needed more room than its plan holds; writes were skipped
  DEV_SCAN_TIMEOUT = 32u    // a look-back wait for a preceding tile gave up (bounded spin)
};

constexpr uint32_t kUnknownCount = 0xFFFFFFFFu;

// A device-side list of rows rows[0 .. *count), taken one by one through *cursor.
struct RowQueue {
  const uint32_t* rows;
  const unsigned int* count;
  unsigned int* cursor;
};

// Where a numeric kernel writes each row. Exact mode (count == nullptr): row r
// has exactly cap[r] entries starting at off[r]. Estimation mode: row r has
// cap[r] slots at off[r]; its true count is stored in count[r] (kUnknownCount
// when it could not be counted) and a row that does not fit is appended to
// overflow[] and not written.
struct OutSpec {
  const uint64_t* off;
  const uint32_t* cap;
  uint32_t* count;
  uint32_t* overflow;
  unsigned int* overflow_n;
};

// CSR view used by kernels. RP is the row-pointer type (uint32_t or uint64_t).
template <typename RP>
struct Csr {
  uint64_t rows, cols, nnz;
  const RP* rp;
  const uint32_t* col;
  const double* val;
  __device__ __forceinline__ uint64_t row_begin(uint64_t r) const { return (uint64_t)rp[r]; }
  __device__ __forceinline__ uint64_t row_end(uint64_t r) const {
    return (r + 1 == rows) ? nnz : (uint64_t)rp[r + 1];
  }
};

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Block-aggregated append to class lists: every thread of the block calls it
// with R rows (b[q] < 0: no append), each in list segment seg[q] (one segment
// per row chunk; 0 when the lists are not split). Offsets inside the block
// come from shared counters (one shared atomic per warp, class, segment and
// q), then one global atomic per class, segment and block reserves the
// block's slots: same-address global atomics drop from one per warp and class
// to one per block and class, which is what limits these kernels on inputs of
// many short rows. Segment g of class c starts at bins[c * stride +
// seg_base[g]] and counts into counts[c * nseg + g]; with nseg > 1 the class
// totals also go to totals[c]. s_cnt holds ncls * nseg zeroed counters,
// visible to the block before the call; ncls * nseg <= blockDim.x.
// Block-collective (two __syncthreads).
template <int R>
__device__ __forceinline__ void block_bin_append(const int (&b)[R], const int (&seg)[R], const uint32_t (&row)[R],
                                                 unsigned* s_cnt, int ncls, int nseg, const uint32_t* seg_base,
                                                 unsigned int* counts, unsigned int* totals, uint32_t* bins,
                                                 uint64_t stride) {
  const int lane = threadIdx.x & 31;
  unsigned off[R];
#pragma unroll
  for (int q = 0; q < R; ++q) {
    const int slot = b[q] >= 0 ? b[q] * nseg + seg[q] : -1;
    const unsigned peers = __match_any_sync(kFull, slot);
    const int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (lane == leader && slot >= 0) base = atomicAdd(&s_cnt[slot], (unsigned)__popc(peers));
    off[q] = __shfl_sync(kFull, base, leader) + __popc(peers & lanemask_lt());
  }
  __syncthreads();
  const int nslot = ncls * nseg;
  if ((int)threadIdx.x < nslot) {
    const unsigned c = s_cnt[threadIdx.x];
    if (c && nseg > 1) atomicAdd(&totals[threadIdx.x / nseg], c);
    s_cnt[threadIdx.x] = c ? atomicAdd(&counts[threadIdx.x], c) : 0u;
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < R; ++q)
    if (b[q] >= 0)
      bins[(uint64_t)b[q] * stride + (nseg > 1 ? seg_base[seg[q]] : 0u) + s_cnt[b[q] * nseg + seg[q]] + off[q]] =
          row[q];
}

// Group size (lanes per A element) for a row: enough lanes to cover the mean
// B-row length, a power of two in [1, 32].
__device__ __forceinline__ int group_size_for(uint64_t products, uint64_t a_nnz) {
  if (a_nnz == 0) return 32;
  const uint64_t avg = (products + a_nnz - 1) / a_nnz;
  int g = 1;
  while (g < 32 && (uint64_t)g < avg) g <<= 1;
  return g;
}

// Multiplicative hash of a column id into [0, 2^log2).
__device__ __forceinline__ uint32_t hash_slot(uint32_t c, int log2) {
  return (c * 0x9E3779B1u) >> (32 - log2);
}

}  // namespace ocean
