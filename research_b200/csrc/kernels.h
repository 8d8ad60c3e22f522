// Host-side launchers of the SpGEMM kernels (implemented in kernels_core.cu).
#pragma once
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
#include "ocean_internal.cuh"

namespace ocean {

// Device buffers of one multiply, sized for `rows` rows of A.
struct DevWork {
  uint64_t rows = 0;
  uint32_t* prod = nullptr;      // products per row (saturated to u32)
  uint32_t* lo = nullptr;        // smallest output column per row (kEmpty if none)
  uint32_t* hi = nullptr;        // largest output column per row
  uint32_t* anz = nullptr;       // entries per row of A
  uint32_t* maxb = nullptr;      // longest referenced B row per row of A
  uint32_t* row_nnz = nullptr;   // exact output count per row
  uint32_t* sym_bins = nullptr;  // [SB_COUNT][rows] row ids per symbolic class
  uint32_t* num_bins = nullptr;  // [NB_COUNT][rows] row ids per numeric class
  unsigned long long* tile_sums = nullptr;
  uint64_t* rowptr64 = nullptr;  // rows+1 exclusive scan of row_nnz
  uint32_t* rowptr32 = nullptr;  // same, truncated to 32 bits
  uint64_t* bm_off = nullptr;    // per row: word offset of its cached bitmap, or ~0
  uint32_t* est = nullptr;       // estimation workflow: estimated output count per row
  uint64_t* est_off = nullptr;   // estimation workflow: exclusive scan of est (slots in the temporary output)
  uint32_t* cnt = nullptr;       // estimation workflow: true output count per row
  uint32_t* ovf = nullptr;       // estimation workflow: rows that overflowed their estimate
  unsigned long long* bm_cache = nullptr;  // exact column bitmaps saved by the symbolic pass
  uint64_t bm_cache_words = 0;   // capacity of bm_cache (0: no cache)
  DevCounters* ctr = nullptr;
  // exact-mode numeric bitmap class (k_num_window): resume cursor per A entry
  // (capacity >= nnz(A) when some row of the class has more than 1024 A
  // entries), a 2^20-bit bitmap per block for rows without a saved bitmap, and
  // the host's count of the class's rows wider than 2^20 columns (kUnknownCount:
  // not known, the kernel for them is launched anyway). Null buffers: the class
  // runs in k_num_bitmap alone.
  uint32_t* win_cursor = nullptr;
  unsigned long long* win_scratch = nullptr;
  uint32_t wide_rows = 0xFFFFFFFFu;
  // rows of A with more than kLongRowEntries entries: listed by the analysis
  // and summarised (and HLL-merged) by all warps together; null: each row is
  // handled by its own lane group
  uint32_t* long_rows = nullptr;
  LongRowAcc* long_acc = nullptr;
  uint32_t long_cap = 0;
  uint32_t* long_chunk_row = nullptr;  // chunk id -> index in long_rows
  uint32_t long_chunk_cap = 0;
  // per row of B: first column, last column, length (low, high word); built
  // at the start of each analysis (null: the analysis reads B itself)
  uint4* btab = nullptr;
  uint64_t btab_cap = 0;
  // numeric class lists split into row chunks (0: one list per class): rows
  // of chunk k are [chunk_bound[k], chunk_bound[k + 1]); class c's list of
  // chunk k starts at num_bins[c * rows + chunk_bound[k]] with its own count
  // and cursor (chunk_count / chunk_cursor[c * chunks + k])
  int chunks = 0;
  uint32_t* chunk_bound = nullptr;
  unsigned* chunk_count = nullptr;
  unsigned* chunk_cursor = nullptr;
  // segment-driven dispatch: per-row policy slot (0: the call's policy,
  // 1 + SegClass: that segment class's policy); null: slot 0 for every row
  const uint8_t* row_pol = nullptr;
};

constexpr int kScanTile = 1024;  // rows per scan tile: 1024 threads of k_scan_reduce, 256 x 4 of k_scan_apply
inline uint64_t scan_tiles(uint64_t n) { return (n + kScanTile - 1) / kScanTile; }

// Class choice of a row (tunable: the batched autotuner searches these).
// Capacities of the fixed shared-memory tables bound the hash limits from above.
struct SymPolicy {
  uint32_t esc_max_products = 128;  // at most 128 (ESC4: 32 lanes x 4)
  int force_bin = -1;               // >= 0: every non-empty row goes to this class (tests)
  uint32_t hash_s_max = 1024;       // products of a small-hash row (table of 2048 slots)
  uint32_t bm_words_m = 2048;       // 4096-product rows: bitmap when the span needs at most this many words
  uint32_t bm_words_l = 8192;       // larger rows up to 16384 products: same rule
  uint32_t direct = 1;              // mid rows whose span fits a hash table take it (direct slots), not a bitmap
};
struct NumPolicy {
  uint32_t esc_max_products = 128;
  int force_bin = -1;
  uint32_t hash_s_max = 512;        // outputs of a small-hash row (table of 1024 slots)
  uint32_t bm_words_m = 1024;
  uint32_t bm_words_l = 4096;
  uint32_t direct = 1;
};

// Policies of the dispatch slots (slot 0: the call's policy; 1..4: the
// policies of the segment classes when segment-driven dispatch is on).
constexpr int kPolicySlots = 5;
struct SymPolicySet {
  SymPolicy p[kPolicySlots];
};
struct NumPolicySet {
  NumPolicy p[kPolicySlots];
};

// Symbolic class of a row from its product count and output column span.
__device__ __forceinline__ int sym_bin_for(uint64_t p, uint64_t span, const SymPolicy& pol) {
  if (pol.force_bin >= 0) return pol.force_bin;
  if (p <= pol.esc_max_products) return p <= 32 ? SB_ESC1 : (p <= 64 ? SB_ESC2 : SB_ESC4);
  const uint64_t words = (span + 63) >> 6;
  if (p > 16384) return SB_BITMAP;
  if (p <= pol.hash_s_max) return SB_HASH_S;
  if (p <= 4096) return ((pol.direct && span <= 8192) || words > pol.bm_words_m) ? SB_HASH_M : SB_BITMAP;
  return ((pol.direct && span <= 32768) || words > pol.bm_words_l) ? SB_HASH_L : SB_BITMAP;
}

// Numeric class of a row from its exact output count.
__device__ __forceinline__ int num_bin_for(uint32_t n, uint64_t p, uint64_t span,
                                           const NumPolicy& pol) {
  if (n == 0) return -1;
  if (pol.force_bin >= 0) return pol.force_bin;
  if (p <= pol.esc_max_products) return p <= 32 ? NB_ESC1 : (p <= 64 ? NB_ESC2 : NB_ESC4);
  const uint64_t words = (span + 63) >> 6;
  if (n <= pol.hash_s_max) return NB_HASH_S;
  if (n <= 2048) return ((pol.direct && span <= 4096) || words > pol.bm_words_m) ? NB_HASH_M : NB_BITMAP;
  if (n <= 4096) return ((pol.direct && span <= 8192) || words > pol.bm_words_l) ? NB_HASH_L : NB_BITMAP;
  return NB_BITMAP;
}

template <typename RP>
int launch_analysis(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, const SymPolicy& pol,
                     cudaStream_t s, const SymPolicy* seg = nullptr);
// seg (optional): policies of the 4 segment classes, applied through w.row_pol.

// bin_events (optional): SB_COUNT + 1 events recorded around the class kernels.
// counts (optional): host copy of the rows per class; empty classes are not
// launched and grids are capped by the class size.
// Each launcher returns the number of kernels it launched.
template <typename RP>
int launch_symbolic(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, int num_sms,
                    cudaStream_t s, cudaEvent_t* bin_events, const unsigned* counts = nullptr);

// Exclusive scan of in[w.rows] into out64 (and out32 if given), total into
// *total and out[rows]; with bin_rows, also appends every row to its numeric
// class (chosen from in[] as the output count).
int launch_scan(const DevWork& w, const uint32_t* in, uint64_t* out64, uint32_t* out32,
                unsigned long long* total, bool bin_rows, const NumPolicy& pol, cudaStream_t s,
                const NumPolicy* seg = nullptr);
// Dispatch slots of the rows: 0 everywhere, then iv (n triples start, end,
// slot of disjoint row intervals, device memory) painted over.
void launch_paint_rows(const uint32_t* iv, uint32_t n, uint8_t* row_pol, uint64_t rows, cudaStream_t s);

// HLL (estimation workflow): sketches of B's rows (2^log2p one-byte registers
// each, into `sketch`) and the compaction statistics of the LCG-sampled rows
// of A (into the counters).
template <typename RP>
int launch_hll_sketch_sample(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, int log2p, unsigned sample_rows,
                             uint8_t* sketch, cudaStream_t s);

// Per-row output-size estimates into out[A.rows]: raw HLL union estimates, or
// (raw = false) the estimate times `expansion`, at least 1 and at most
// min(products, column span), with the product count for rows of at most
// esc_max products.
template <typename RP>
int launch_hll_rows(const Csr<RP>& A, const DevWork& w, int log2p, double expansion, uint32_t esc_max, bool raw,
                    const uint8_t* sketch, uint32_t* out, cudaStream_t s);

// Estimation workflow epilogue: copy the rows that fit their estimate from the
// temporary output into C. stop (optional): the kernel does nothing if
// DEV_BATCH_MISMATCH is set there.
void launch_copy_rows(const DevWork& w, const uint32_t* t_col, const double* t_val, uint32_t* c_col,
                      double* c_val, cudaStream_t s, const unsigned* stop = nullptr);

// Exact counts (bitmap symbolic kernel) and exact numeric output (bitmap
// numeric kernel) for the rows of the overflow queue.
template <typename RP>
int launch_overflow(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, bool numeric, uint32_t* c_col,
                    double* c_val, int num_sms, cudaStream_t s);

// chunk >= 0 (w.chunks > 0): only the rows of that row chunk, from its
// per-chunk class lists (row_base = its first row); counts are then the
// chunk's class sizes.
template <typename RP>
int launch_numeric(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, const OutSpec& out, uint32_t* c_col,
                    double* c_val, int num_sms, cudaStream_t s, cudaEvent_t* bin_events,
                    const unsigned* counts = nullptr, int chunk = -1, uint32_t row_base = 0);

// Row chunks of equal products for a chunked numeric phase: with prefix[] the
// exclusive scan of the per-row products (rows + 1 values), w.chunk_bound[k] =
// the first row whose prefix reaches k/chunks of the total (k = 0 .. chunks).
constexpr int kMaxChunks = 16;
void launch_chunk_bounds(const DevWork& w, const uint64_t* prefix, int chunks, cudaStream_t s);

void launch_murmur3(const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t seed, cudaStream_t s);

// Fused ultra-sparse multiply (every row at most 256 products): C's column
// ids and values (capacity `cap` >= the sum of the products) and the row
// pointers w.rowptr64 (and w.rowptr32 when rowptr32) in one launch, nnz(C) into
// w.ctr->total_nnz. `tiles` holds usp_tiles(A.rows) words.
template <typename RP>
int launch_usp_fused(const Csr<RP>& A, const Csr<RP>& B, const DevWork& w, unsigned long long* tiles, uint64_t cap,
                     bool rowptr32, uint32_t* c_col, double* c_val, cudaStream_t s);
uint64_t usp_tiles(uint64_t rows);
constexpr uint32_t kUspMaxProducts = 256;

// out[r] = min(products, column span) for every row of the last analysis.
int launch_row_bounds(const DevWork& w, uint32_t* out, cudaStream_t s);

// Per-kernel dynamic shared memory opt-in and occupancy table; call once per
// device, with it current (ensure_kernel_attributes does so under a lock, for
// every entry point that may be first on a device; false: bad ordinal).
void configure_kernel_attributes();
bool ensure_kernel_attributes(int dev);

// Words of DevWork::win_scratch for a device with num_sms SMs (one 2^20-bit
// bitmap per resident block of k_num_window); valid after configure_kernel_attributes.
size_t window_scratch_words(int num_sms);

// Stores the calling thread's error message returned by ocean_last_error().
void set_last_error(const char* msg);

// ---------------------------------------------------------------- segmentation
// Spy-plot segmentation of A (reference: kernels/Segmentation.cuh:34-73).
enum SegClass : uint32_t { SEG_SPARSE_UNIFORM = 0, SEG_DENSE = 1, SEG_POWER_LAW = 2, SEG_BANDED = 3 };

struct SegRecord {
  uint32_t row_start, row_end, row_count;
  uint32_t col_left, col_right;  // union of the rows' output column spans
  uint32_t cls;                  // SegClass
  unsigned long long sum_products, sum_a_nnz;
  uint32_t max_b_row_len, max_a_row_len;
  double mean_row_len;  // mean products per row
  double var_row_len;   // population variance of products per row
  double local_er;      // sum_products / sum_a_nnz
};

struct SegmentationResult {
  std::vector<SegRecord> segments;
  uint32_t grid_h = 0, grid_w = 0, tile_rows = 0, tile_cols = 0;
  uint32_t num_components = 0;
  double density_mean = 0.0, density_stddev = 0.0;
  float time_density_ms = 0.f, time_threshold_ms = 0.f, time_cc_ms = 0.f, time_classify_ms = 0.f;
  int cc_iterations = 0;
};

// Needs the analysis outputs w.prod, w.anz, w.maxb, w.lo, w.hi of A * B.
template <typename RP>
cudaError_t run_segmentation(const Csr<RP>& A, uint64_t b_cols, const DevWork& w, int grid_max, double hot_k,
                             int min_segment_rows, int cc_max_iters, int expansion_threshold, cudaStream_t s,
                             SegmentationResult* out);
const char* segment_class_name(uint32_t cls);

}  // namespace ocean
