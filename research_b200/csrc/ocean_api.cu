// C ABI and host orchestration of one SpGEMM (C = A·B).
//
// Replaces somespgemm::SpGEMM::run (kernels/SpGEMM.cuh:213-338). The reference
// runs one of four workflows with ~18 blocking read-backs and 20 streams; this
// orchestration runs analysis -> symbolic -> scan -> (one read-back of nnz(C)
// to allocate C) -> numeric, with every row class handled by a persistent
// kernel that reads its row list and count from device memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <fstream>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

#include "config.h"
#include "batch.h"
#include "kernels.h"
#include "mlp.h"
#include "ocean.h"

#include "mlp_weights.inc"

using namespace ocean;

namespace {

thread_local std::string g_last_error;

struct OceanError {
  int code;
  std::string msg;
};

#define OCEAN_CUDA(call)                                                                          \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) {                                                                      \
      throw OceanError{e_ == cudaErrorMemoryAllocation ? (int)OCEAN_ERR_OOM : (int)OCEAN_ERR_CUDA, \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};                       \
    }                                                                                             \
  } while (0)

#define OCEAN_CHECK(cond, code, msg)        \
  do {                                      \
    if (!(cond)) throw OceanError{code, msg}; \
  } while (0)

// Allocation record of a result (C->_owner).
struct CResult {
  int location;  // 0 device (owned), 1 host (lent by the handle)
  void* rowptr = nullptr;
  uint32_t* col = nullptr;
  double* val = nullptr;
  int refs = 1;  // results of one batched call share one allocation
  bool plain_alloc = false;  // allocated with cudaMalloc (freed with cudaFree)
};

enum Ev {
  EV_START = 0,
  EV_ANALYSIS,
  EV_SYM0,  // EV_SYM0 .. EV_SYM0+5: symbolic class boundaries
  EV_SYMBOLIC = EV_SYM0 + SB_COUNT,
  EV_SCAN,
  EV_NUM0,  // EV_NUM0 .. EV_NUM0+5: numeric class boundaries
  EV_NUM_END = EV_NUM0 + NB_COUNT,
  EV_END,
  EV_COUNT
};

const char* const kSymNames[SB_COUNT] = {"esc1", "esc2", "esc4", "hash_s", "hash_m", "hash_l", "bitmap"};
const char* const kNumNames[NB_COUNT] = {"esc1", "esc2", "esc4", "hash_s", "hash_m", "hash_l", "bitmap"};

struct Stats {
  uint64_t a_rows = 0, a_cols = 0, a_nnz = 0, b_rows = 0, b_cols = 0, b_nnz = 0;
  uint64_t c_rows = 0, c_cols = 0, c_nnz = 0;
  uint64_t total_products = 0;
  uint32_t max_products = 0, max_a_nnz = 0;
  uint32_t sym_bins[SB_COUNT] = {0};
  uint32_t num_bins[NB_COUNT] = {0};
  uint64_t num_nnz[NB_COUNT] = {0};
  uint64_t num_anz[NB_COUNT] = {0};
  uint64_t num_prod[NB_COUNT] = {0};
  uint64_t sym_anz[SB_COUNT] = {0};
  uint64_t sym_prod[SB_COUNT] = {0};
  uint64_t cache_words = 0, cache_used = 0;
  bool cache_dropped = false;
  int bm_kernel = 0;  // numeric bitmap class: 0 no rows, 1 k_num_bitmap (rank + FP64 red), 2 k_num_window
  int host_chunks = 0;  // host-buffer multiply: row chunks whose copies overlapped the numeric phase (0: none)
  bool fused = false;  // ultra-sparse workflow in one fused launch
  int launches = 0;  // kernels launched by the last call
  uint64_t total_est = 0, overflow_rows = 0;
  int hll_log2p = 0;
  double hll_expansion = 0.0, compaction1 = 0.0, compaction2 = 0.0;
  bool sampled = false;
  int workflow = 0;  // 0 = precise (symbolic + numeric)
  int rowptr_bits = 32;
  bool valid = false;
  double host_ms = 0.0;
  // host clock at the steps of the last multiply (ms since its start): where a
  // call that is short on the device spends its time between read-backs
  std::vector<std::pair<const char*, double>> host_marks;
  // estimation workflows: which estimator sized the rows, and (estimator_metrics)
  // its error against the exact counts: mean relative row-size error and share
  // of rows whose numeric class differs, with and without the safety margin
  int estimator = 0;  // 0 none, 1 HLL, 2 learned
  bool metrics = false;
  double mre = 0.0, misbinned = 0.0, mre_raw = 0.0, misbinned_raw = 0.0;
  uint64_t metric_rows = 0;
};

__global__ void k_widen_rowptr(const uint32_t* __restrict__ in, uint64_t* __restrict__ out, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    out[i] = in[i];
}

template <typename T>
void grow(T*& p, uint64_t& cap, uint64_t need) {
  if (need <= cap && p) return;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  const uint64_t n = std::max<uint64_t>(need, 1);
  OCEAN_CUDA(cudaMalloc((void**)&p, n * sizeof(T)));
  cap = n;
}

template <typename T>
void grow_host(T*& p, uint64_t& cap, uint64_t need) {
  if (need <= cap && p) return;
  if (p) cudaFreeHost(p);
  p = nullptr;
  cap = 0;
  const uint64_t n = std::max<uint64_t>(need, 1);
  OCEAN_CUDA(cudaHostAlloc((void**)&p, n * sizeof(T), cudaHostAllocDefault));
  cap = n;
}

}  // namespace

struct ocean_handle {
  Config cfg;
  int device = 0;
  int num_sms = 148;
  uint64_t device_bytes = 0;  // total device memory (read once at creation)
  DevWork w;
  uint64_t cap_rows = 0;
  DevCounters* h_ctr = nullptr;  // pinned
  cudaEvent_t ev[EV_COUNT];
  uint64_t ev_mask = 0;  // events recorded during the last call
  bool ev_recorded = false;
  bool tracked = false;
  Stats st;
  // learned estimator: device blob (parameters | mu | inv_sd), margin
  float* mlp_dev = nullptr;
  float mlp_margin = 0.f;
  bool mlp_ready = false;
  uint32_t* raw_est = nullptr;  // estimator_metrics: estimates without the margin
  uint64_t raw_est_cap = 0;
  double* metrics_dev = nullptr;  // 2 x 4 sums of launch_est_metrics
  // spy-plot segmentation of the last multiply (use_segmented_workflow)
  SegmentationResult seg;
  bool seg_ran = false;
  // segment-driven dispatch of the last multiply: per-row slots, the
  // segment-class policies, and the rows each slot received
  uint8_t* row_pol = nullptr;
  uint64_t row_pol_cap = 0;
  uint32_t* seg_iv = nullptr;
  uint64_t seg_iv_cap = 0;
  SymPolicy seg_sp[4];
  NumPolicy seg_np[4];
  bool seg_dispatch = false;   // in force for the call under way (reset by every analysis)
  bool seg_dispatched = false; // the last multiply was dispatched by segments (stats)
  uint64_t seg_rows[kPolicySlots] = {0};
  // widened row pointers for mixed 32/64-bit inputs
  uint64_t* wide_a = nullptr;
  uint64_t wide_a_cap = 0;
  uint64_t* wide_b = nullptr;
  uint64_t wide_b_cap = 0;
  // device copies of host inputs (ocean_spgemm_host)
  unsigned char* in_rp[2] = {nullptr, nullptr};
  uint64_t in_rp_cap[2] = {0, 0};
  uint32_t* in_col[2] = {nullptr, nullptr};
  uint64_t in_col_cap[2] = {0, 0};
  double* in_val[2] = {nullptr, nullptr};
  uint64_t in_val_cap[2] = {0, 0};
  // pinned host output (ocean_spgemm_host)
  unsigned char* out_rp = nullptr;
  uint64_t out_rp_cap = 0;
  uint32_t* out_col = nullptr;
  uint64_t out_col_cap = 0;
  double* out_val = nullptr;
  uint64_t out_val_cap = 0;
  CResult host_owner{1};
  // saved row bitmaps of the symbolic pass (grow-only, kept across calls)
  unsigned long long* cache_buf = nullptr;
  uint64_t cache_cap_words = 0;
  // fused ultra-sparse multiply: look-back state per tile (grow-only)
  unsigned long long* usp_tiles_buf = nullptr;
  uint64_t usp_tiles_cap = 0;
  // k_num_window: resume cursors per A entry and per-block bitmaps (grow-only)
  uint32_t* win_cursor = nullptr;
  uint64_t win_cursor_cap = 0;
  unsigned long long* win_scratch = nullptr;
  uint64_t win_scratch_cap = 0;
  // host-buffer multiply (ocean_spgemm_host) under way: the precise workflow
  // may run its numeric phase in row chunks and copy each finished chunk of C
  // to the pinned host buffers on copy_stream (sink_filled: it did)
  bool sink_active = false;
  bool sink_filled = false;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t chunk_ev[kMaxChunks + 1] = {};
  uint32_t* chunk_dev = nullptr;  // bounds (kMaxChunks + 1), counts and cursors (NB_COUNT x kMaxChunks each)
  uint32_t* chunk_host = nullptr; // pinned: bounds and counts read back

  void free_all() {
    DevWork& x = w;
    void* ps[] = {x.prod, x.lo, x.hi, x.anz, x.maxb, x.row_nnz, x.sym_bins, x.num_bins, x.tile_sums, x.rowptr64,
                  x.rowptr32, x.bm_off, x.est, x.est_off, x.cnt, x.ovf, x.long_rows, x.long_acc, x.long_chunk_row,
                  x.btab, x.ctr, wide_a,
                  wide_b, in_rp[0], in_rp[1], in_col[0], in_col[1], in_val[0], in_val[1]};
    for (void* p : ps)
      if (p) cudaFree(p);
    if (h_ctr) cudaFreeHost(h_ctr);
    if (out_rp) cudaFreeHost(out_rp);
    if (out_col) cudaFreeHost(out_col);
    if (out_val) cudaFreeHost(out_val);
    if (cache_buf) cudaFree(cache_buf);
    if (usp_tiles_buf) cudaFree(usp_tiles_buf);
    if (win_cursor) cudaFree(win_cursor);
    if (win_scratch) cudaFree(win_scratch);
    if (chunk_dev) cudaFree(chunk_dev);
    if (chunk_host) cudaFreeHost(chunk_host);
    if (copy_stream) cudaStreamDestroy(copy_stream);
    for (auto& e : chunk_ev)
      if (e) cudaEventDestroy(e);
    if (mlp_dev) cudaFree(mlp_dev);
    if (raw_est) cudaFree(raw_est);
    if (row_pol) cudaFree(row_pol);
    if (seg_iv) cudaFree(seg_iv);
    if (metrics_dev) cudaFree(metrics_dev);
    for (auto& e : ev) cudaEventDestroy(e);
  }
};

namespace {

void init_handle(ocean_handle* h, const std::string& json) {
  h->cfg = Config::from_json_text(json);
  OCEAN_CUDA(cudaGetDevice(&h->device));
  OCEAN_CUDA(cudaDeviceGetAttribute(&h->num_sms, cudaDevAttrMultiProcessorCount, h->device));
  {
    size_t free_b = 0, total_b = 0;
    OCEAN_CUDA(cudaMemGetInfo(&free_b, &total_b));
    h->device_bytes = total_b;
  }
  // Stream-ordered allocations come from the device's default pool, which is told
  // to keep freed memory (as the reference does, kernels/SpGEMM.cuh:219-223).
  cudaMemPool_t pool;
  OCEAN_CUDA(cudaDeviceGetDefaultMemPool(&pool, h->device));
  uint64_t threshold = UINT64_MAX;
  OCEAN_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &threshold));
  static std::mutex mlp_mutex;
  static bool mlp_configured[64] = {false};
  OCEAN_CHECK(ensure_kernel_attributes(h->device), OCEAN_ERR_INVALID, "device ordinal out of range (64 devices)");
  {
    std::lock_guard<std::mutex> lock(mlp_mutex);
    if (!mlp_configured[h->device]) {
      configure_mlp_attributes();
      mlp_configured[h->device] = true;
    }
  }
  OCEAN_CUDA(cudaGetLastError());
  for (auto& e : h->ev) OCEAN_CUDA(cudaEventCreate(&e));
  OCEAN_CUDA(cudaHostAlloc((void**)&h->h_ctr, sizeof(DevCounters), cudaHostAllocDefault));
  OCEAN_CUDA(cudaMalloc((void**)&h->w.ctr, sizeof(DevCounters)));
}

// Frees the per-row arrays of a DevWork (not its counters).
void free_work_rows(DevWork& x) {
  void* ps[] = {x.prod, x.lo, x.hi, x.anz, x.maxb, x.row_nnz, x.sym_bins, x.num_bins, x.tile_sums, x.rowptr64,
                x.rowptr32, x.bm_off, x.est, x.est_off, x.cnt, x.ovf, x.long_rows, x.long_acc, x.long_chunk_row,
                x.btab};
  for (void* p : ps)
    if (p) cudaFree(p);
  DevCounters* keep = x.ctr;
  x = DevWork();
  x.ctr = keep;
}

// Per-row arrays of a DevWork for `rows` rows of A (about 100 B per row).
void alloc_work_rows(DevWork& x, uint64_t rows) {
  free_work_rows(x);
  const uint64_t r = std::max<uint64_t>(rows, 1);
  OCEAN_CUDA(cudaMalloc((void**)&x.prod, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.anz, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.maxb, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.lo, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.hi, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.row_nnz, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.sym_bins, r * 4 * SB_COUNT));
  OCEAN_CUDA(cudaMalloc((void**)&x.num_bins, r * 4 * NB_COUNT));
  OCEAN_CUDA(cudaMalloc((void**)&x.tile_sums, scan_tiles(r) * 8 + 8));
  OCEAN_CUDA(cudaMalloc((void**)&x.rowptr64, (r + 1) * 8));
  OCEAN_CUDA(cudaMalloc((void**)&x.rowptr32, (r + 1) * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.bm_off, r * 8));
  OCEAN_CUDA(cudaMalloc((void**)&x.est, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.est_off, (r + 1) * 8));
  OCEAN_CUDA(cudaMalloc((void**)&x.cnt, r * 4));
  OCEAN_CUDA(cudaMalloc((void**)&x.ovf, r * 4));
  x.rows = rows;
}

// The long-row list, its accumulators and the chunk -> row map for an A of
// `rows` rows and `nnz` entries (at most nnz / kLongRowEntries rows are long,
// and they have at most nnz / kLongChunk + that many chunks). Without them
// (allocation failed) every row is summarised by its own lane group.
void ensure_long_rows(DevWork& x, uint64_t nnz, uint64_t rows) {
  const uint64_t need = std::max<uint64_t>(std::min<uint64_t>(rows, nnz / kLongRowEntries + 1), 1);
  const uint64_t chunks = nnz / kLongChunk + need + 1;
  if (x.long_acc && x.long_cap >= need && x.long_chunk_cap >= chunks) return;
  void* old[] = {x.long_rows, x.long_acc, x.long_chunk_row};
  for (void* q : old)
    if (q) cudaFree(q);
  x.long_rows = nullptr;
  x.long_acc = nullptr;
  x.long_chunk_row = nullptr;
  x.long_cap = 0;
  x.long_chunk_cap = 0;
  if (chunks > 0xFFFFFFFFull) return;
  if (cudaMalloc((void**)&x.long_rows, need * 4) != cudaSuccess ||
      cudaMalloc((void**)&x.long_acc, need * sizeof(LongRowAcc)) != cudaSuccess ||
      cudaMalloc((void**)&x.long_chunk_row, chunks * 4) != cudaSuccess) {
    (void)cudaGetLastError();
    void* got[] = {x.long_rows, x.long_acc, x.long_chunk_row};
    for (void* q : got)
      if (q) cudaFree(q);
    x.long_rows = nullptr;
    x.long_acc = nullptr;
    x.long_chunk_row = nullptr;
    return;
  }
  x.long_cap = (uint32_t)need;
  x.long_chunk_cap = (uint32_t)chunks;
}

// The row table of B (16 B per row of B, grow-only). Without it (allocation
// failed) the analysis reads B's rows itself.
void ensure_btab(DevWork& x, uint64_t b_rows) {
  const uint64_t need = std::max<uint64_t>(b_rows, 1);
  if (x.btab && x.btab_cap >= need) return;
  if (x.btab) cudaFree(x.btab);
  x.btab = nullptr;
  x.btab_cap = 0;
  if (cudaMalloc((void**)&x.btab, need * sizeof(uint4)) != cudaSuccess) {
    (void)cudaGetLastError();
    x.btab = nullptr;
    return;
  }
  x.btab_cap = need;
}

void ensure_rows(ocean_handle* h, uint64_t rows) {
  if (rows <= h->cap_rows && h->w.prod) {
    h->w.rows = rows;
    return;
  }
  h->cap_rows = 0;
  alloc_work_rows(h->w, rows);
  h->cap_rows = std::max<uint64_t>(rows, 1);
}

void validate_view(const ocean_csr_view* m, const char* name) {
  OCEAN_CHECK(m != nullptr, OCEAN_ERR_INVALID, std::string(name) + " is NULL");
  OCEAN_CHECK(m->rowptr_bits == 32 || m->rowptr_bits == 64, OCEAN_ERR_INVALID,
              std::string(name) + ".rowptr_bits must be 32 or 64");
  OCEAN_CHECK(m->rows == 0 || m->rowptr != nullptr, OCEAN_ERR_INVALID, std::string(name) + ".rowptr is NULL");
  OCEAN_CHECK(m->nnz == 0 || (m->col != nullptr && m->val != nullptr), OCEAN_ERR_INVALID,
              std::string(name) + ".col/.val is NULL");
  OCEAN_CHECK(m->rows < 0xFFFFFFFFull, OCEAN_ERR_INVALID, std::string(name) + " has too many rows (>= 2^32-1)");
  OCEAN_CHECK(m->cols <= 0xFFFFFFFFull, OCEAN_ERR_INVALID, std::string(name) + " has too many columns (> 2^32-1)");
  OCEAN_CHECK(m->rowptr_bits == 64 || m->nnz <= 0xFFFFFFFFull, OCEAN_ERR_INVALID,
              std::string(name) + " has nnz >= 2^32 with 32-bit row pointers");
}

void record(ocean_handle* h, int i, cudaStream_t s) {
  cudaEventRecord(h->ev[i], s);
  h->ev_mask |= 1ull << i;
}

// Waits for `s` by polling for a short, bounded time before falling back to a
// blocking synchronize: the mid-call read-backs are tens of microseconds apart
// on small problems, where a sleeping wait adds scheduler wake-up jitter.
cudaError_t wait_stream(cudaStream_t s, int spin_us) {
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaStreamQuery(s);
    if (e != cudaErrorNotReady) return e;
    if (std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - t0).count() > spin_us)
      return cudaStreamSynchronize(s);
  }
}

const char* status_text(unsigned st) {
  if (st & DEV_TABLE_FULL) return "a shared-memory hash table ran full (probe limit reached)";
  if (st & DEV_BIN_OVERFLOW) return "a row exceeded the capacity of its accumulator class";
  if (st & DEV_COUNT_MISMATCH) return "numeric output count differs from the symbolic count";
  if (st & DEV_TC_TIMEOUT) return "a tensor-core completion wait timed out";
  if (st & DEV_SCAN_TIMEOUT) return "a look-back wait for a preceding tile timed out";
  return "device error";
}

void check_device_status(ocean_handle* h) {
  if (h->h_ctr->status) {
    char buf[256];
    snprintf(buf, sizeof buf, "%s (status 0x%x, first row %u)", status_text(h->h_ctr->status), h->h_ctr->status,
             h->h_ctr->err_row);
    const unsigned st = h->h_ctr->status;
    throw OceanError{(st & DEV_COUNT_MISMATCH) ? (int)OCEAN_ERR_INTERNAL
                                               : (st & (DEV_TC_TIMEOUT | DEV_SCAN_TIMEOUT)) ? (int)OCEAN_ERR_TIMEOUT
                                                                                            : (int)OCEAN_ERR_CAPACITY,
                     buf};
  }
}

template <typename RP>
Csr<RP> to_csr(const ocean_csr_view* m, const RP* rp) {
  Csr<RP> c;
  c.rows = m->rows;
  c.cols = m->cols;
  c.nnz = m->nnz;
  c.rp = rp;
  c.col = m->col;
  c.val = m->val;
  return c;
}

// Bytes the device could still hand out: free memory plus what the stream-ordered
// pool holds in reserve.
uint64_t available_device_bytes(int device) {
  size_t free_b = 0, total_b = 0;
  if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
  cudaMemPool_t pool;
  uint64_t reserved = 0, used = 0;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved);
    cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used);
  }
  return (uint64_t)free_b + (reserved > used ? reserved - used : 0);
}

// Whether `bytes` fit in `frac` of the memory the device can still give.
// Needs below 1% of the device's memory are taken to fit without asking: the
// driver query costs tens of microseconds, as much as the whole analysis of
// a problem that small, and an allocation that fails still raises an error.
bool fits_device(const ocean_handle* h, double bytes, double frac) {
  if (bytes < 0.01 * (double)h->device_bytes) return true;
  return bytes < frac * (double)available_device_bytes(h->device);
}

// Policies of the class choice from the config.
void make_policies(const Config& c, SymPolicy* sp, NumPolicy* np) {
  OCEAN_CHECK(c.esc_max_products >= 0 && c.esc_max_products <= 128, OCEAN_ERR_INVALID,
              "esc_max_products must be in [0, 128]");
  OCEAN_CHECK(c.hash_s_max_scale > 0.0 && c.hash_s_max_scale <= 1.0, OCEAN_ERR_INVALID,
              "hash_s_max_scale must be in (0, 1]");
  OCEAN_CHECK(c.bitmap_words_scale > 0.0 && c.bitmap_words_scale <= 64.0, OCEAN_ERR_INVALID,
              "bitmap_words_scale must be in (0, 64]");
  *sp = SymPolicy();
  *np = NumPolicy();
  sp->esc_max_products = (uint32_t)c.esc_max_products;
  sp->force_bin = c.force_sym_bin;
  np->esc_max_products = (uint32_t)c.esc_max_products;
  np->force_bin = c.force_num_bin;
  sp->hash_s_max = std::max<uint32_t>(1, (uint32_t)(sp->hash_s_max * c.hash_s_max_scale));
  np->hash_s_max = std::max<uint32_t>(1, (uint32_t)(np->hash_s_max * c.hash_s_max_scale));
  sp->bm_words_m = (uint32_t)(sp->bm_words_m * c.bitmap_words_scale);
  sp->bm_words_l = (uint32_t)(sp->bm_words_l * c.bitmap_words_scale);
  np->bm_words_m = (uint32_t)(np->bm_words_m * c.bitmap_words_scale);
  np->bm_words_l = (uint32_t)(np->bm_words_l * c.bitmap_words_scale);
  sp->direct = np->direct = c.prefer_direct_hash ? 1u : 0u;
  OCEAN_CHECK(sp->force_bin < SB_COUNT && np->force_bin < NB_COUNT, OCEAN_ERR_INVALID, "forced class out of range");
}

// Policies of the segment classes (SegClass order): the call's policies with
// the class's configured fields in place of the global ones.
void make_segment_policies(const Config& c, const SymPolicy& sp, const NumPolicy& np, SymPolicy* ssp,
                           NumPolicy* snp) {
  for (int k = 0; k < 4; ++k) {
    Config ck = c;
    if (c.seg_esc_max_products[k] >= 0) ck.esc_max_products = c.seg_esc_max_products[k];
    if (c.seg_hash_s_max_scale[k] > 0.0) ck.hash_s_max_scale = c.seg_hash_s_max_scale[k];
    if (c.seg_bitmap_words_scale[k] > 0.0) ck.bitmap_words_scale = c.seg_bitmap_words_scale[k];
    if (c.seg_prefer_direct_hash[k] >= 0) ck.prefer_direct_hash = c.seg_prefer_direct_hash[k] > 0;
    if (c.seg_force_sym_bin[k] >= -1) ck.force_sym_bin = c.seg_force_sym_bin[k];
    if (c.seg_force_num_bin[k] >= -1) ck.force_num_bin = c.seg_force_num_bin[k];
    make_policies(ck, &ssp[k], &snp[k]);
  }
  (void)sp;
  (void)np;
}

// The segment policies in force for this call (null: no segment dispatch).
const SymPolicy* seg_sym(const ocean_handle* h) { return h->seg_dispatch ? h->seg_sp : nullptr; }
const NumPolicy* seg_num(const ocean_handle* h) { return h->seg_dispatch ? h->seg_np : nullptr; }

// Phase 1: row analysis. Large inputs read the counters back (class sizes,
// product totals); small inputs skip the read-back. Returns whether it read back.
template <typename RP>
bool run_analysis(ocean_handle* h, const Csr<RP>& A, const Csr<RP>& B, cudaStream_t s) {
  h->ev_recorded = false;  // the stats describe a completed multiply only
  h->ev_mask = 0;
  h->seg_dispatch = false;  // a call dispatches by segments only after its own segmentation
  h->w.row_pol = nullptr;
  ensure_rows(h, A.rows);
  ensure_long_rows(h->w, A.nnz, A.rows);
  ensure_btab(h->w, B.rows);
  OCEAN_CUDA(cudaMemsetAsync(h->w.ctr, 0, sizeof(DevCounters), s));
  SymPolicy sp;
  NumPolicy np;
  make_policies(h->cfg, &sp, &np);
  h->w.bm_cache = nullptr;
  h->w.bm_cache_words = 0;
  record(h, EV_START, s);
  h->st.launches = launch_analysis(A, B, h->w, sp, s);
  OCEAN_CUDA(cudaGetLastError());
  if (h->cfg.track_stage_times) record(h, EV_ANALYSIS, s);
  const bool readback = A.nnz > (uint64_t)h->cfg.small_problem_nnz;
  if (readback) {
    OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
  }
  return readback;
}

// Segment-driven dispatch: the segments' row bands become per-row policy
// slots (slot 1 + SegClass; a row inside several bands takes the first band
// listed; rows in no band keep slot 0, the call's policy); then the analysis
// classes every row again under its slot's policy and, for inputs that read
// back, the counters are read back again.
template <typename RP>
void dispatch_segments(ocean_handle* h, const Csr<RP>& A, const Csr<RP>& B, cudaStream_t s, bool readback) {
  SymPolicy sp;
  NumPolicy np;
  make_policies(h->cfg, &sp, &np);
  make_segment_policies(h->cfg, sp, np, h->seg_sp, h->seg_np);
  std::vector<uint32_t> iv;                               // start, end, slot triples
  std::vector<std::pair<uint32_t, uint32_t>> taken;       // covered bands, sorted, disjoint
  for (uint64_t i = 0; i < kPolicySlots; ++i) h->seg_rows[i] = 0;
  for (const SegRecord& r : h->seg.segments) {
    const uint32_t a = r.row_start;
    const uint32_t b = (uint32_t)std::min<uint64_t>(r.row_end, A.rows);
    if (a >= b || r.cls > SEG_BANDED) continue;
    const uint32_t slot = 1 + r.cls;
    uint32_t cur = a;
    for (const auto& t : taken) {
      if (t.second <= cur) continue;
      if (t.first >= b) break;
      if (t.first > cur) {
        iv.insert(iv.end(), {cur, t.first, slot});
        h->seg_rows[slot] += t.first - cur;
      }
      cur = std::max(cur, t.second);
      if (cur >= b) break;
    }
    if (cur < b) {
      iv.insert(iv.end(), {cur, b, slot});
      h->seg_rows[slot] += b - cur;
    }
    taken.emplace_back(a, b);
    std::sort(taken.begin(), taken.end());
    std::vector<std::pair<uint32_t, uint32_t>> merged;
    for (const auto& t : taken) {
      if (!merged.empty() && t.first <= merged.back().second) merged.back().second = std::max(merged.back().second, t.second);
      else merged.push_back(t);
    }
    taken.swap(merged);
  }
  uint64_t painted = 0;
  for (int i = 1; i < kPolicySlots; ++i) painted += h->seg_rows[i];
  h->seg_rows[0] = A.rows - painted;
  const uint32_t n = (uint32_t)(iv.size() / 3);
  grow(h->row_pol, h->row_pol_cap, A.rows);
  if (n) {
    grow(h->seg_iv, h->seg_iv_cap, iv.size());
    // from pageable memory: the call returns once the triples are staged
    OCEAN_CUDA(cudaMemcpyAsync(h->seg_iv, iv.data(), iv.size() * 4, cudaMemcpyHostToDevice, s));
  }
  launch_paint_rows(h->seg_iv, n, h->row_pol, A.rows, s);
  h->w.row_pol = h->row_pol;
  h->seg_dispatch = true;
  h->seg_dispatched = true;
  OCEAN_CUDA(cudaMemsetAsync(h->w.ctr, 0, sizeof(DevCounters), s));
  h->st.launches += (n ? 1 : 0) + launch_analysis(A, B, h->w, sp, s, h->seg_sp);
  OCEAN_CUDA(cudaGetLastError());
  if (readback) {
    OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
  }
}

// Buffers of the windowed exact numeric kernel for the bitmap class: cursors
// for nnz(A) entries when a row of A has more than one chunk (1024) of
// entries, and one 2^20-bit bitmap per resident block. If they cannot be
// allocated, the class runs in k_num_bitmap alone (no error).
void prepare_windows(ocean_handle* h, uint64_t a_nnz, unsigned bitmap_rows) {
  h->w.win_cursor = nullptr;
  h->w.win_scratch = nullptr;
  h->w.wide_rows = h->h_ctr->num_wide;
  h->st.bm_kernel = bitmap_rows ? 1 : 0;
  if (!h->cfg.numeric_windows || bitmap_rows == 0) return;
  const uint64_t need_cur = h->h_ctr->max_a_nnz > (unsigned)kBitmapThreads ? a_nnz : 1;
  const uint64_t need_scr = window_scratch_words(h->num_sms);
  auto try_grow = [](auto*& p, uint64_t& cap, uint64_t need, size_t elem) {
    if (p && cap >= need) return true;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    if (cudaMalloc((void**)&p, need * elem) != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      return false;
    }
    cap = need;
    return true;
  };
  if (!try_grow(h->win_cursor, h->win_cursor_cap, need_cur, sizeof(uint32_t))) return;
  if (!try_grow(h->win_scratch, h->win_scratch_cap, need_scr, sizeof(unsigned long long))) return;
  h->w.win_cursor = h->win_cursor;
  h->w.win_scratch = h->win_scratch;
  h->st.bm_kernel = 2;
}

// Phase 2 of the precise workflow: symbolic class kernels (exact counts into
// w.row_nnz) and, with_scan, the row-pointer scan and numeric class lists; the
// counters are read back at the end. With allow_cache (and the class sizes of
// a read-back), bitmap-class rows save their bitmaps into h->w.bm_cache, whose
// size comes from the analysis and is capped by bitmap_cache_fraction of free memory.
template <typename RP>
void run_symbolic(ocean_handle* h, const Csr<RP>& A, const Csr<RP>& B, cudaStream_t s, bool readback,
                  bool with_scan, bool allow_cache) {
  SymPolicy sp;
  NumPolicy np;
  make_policies(h->cfg, &sp, &np);
  unsigned sym_counts[SB_COUNT];
  for (int i = 0; i < SB_COUNT; ++i) sym_counts[i] = h->h_ctr->sym_count[i];
  if (readback && allow_cache && h->cfg.bitmap_cache_fraction > 0.0) {
    const uint64_t want = h->h_ctr->sym_words;
    const uint64_t budget =
        want >= 1024 ? (uint64_t)(h->cfg.bitmap_cache_fraction * (double)available_device_bytes(h->device)) / 8 : 0;
    const uint64_t words = std::min(want, budget);
    if (words >= 1024) {
      if (h->cache_cap_words < words) {
        if (h->cache_buf) cudaFree(h->cache_buf);
        h->cache_buf = nullptr;
        h->cache_cap_words = 0;
        const uint64_t grow_to = std::min(budget, words + words / 8);
        if (cudaMalloc((void**)&h->cache_buf, grow_to * 8) == cudaSuccess) {
          h->cache_cap_words = grow_to;
        } else {
          cudaGetLastError();
        }
      }
      if (h->cache_buf) {
        h->w.bm_cache = h->cache_buf;
        h->w.bm_cache_words = std::min(words, h->cache_cap_words);
      }
    }
  }
  // per-class boundary events only when stage timing is asked for (each record costs device time)
  const bool track = h->cfg.track_stage_times;
  h->st.launches += launch_symbolic(A, B, h->w, h->num_sms, s, track ? h->ev + EV_SYM0 : nullptr,
                                    readback ? sym_counts : nullptr);
  if (track && A.rows) h->ev_mask |= ((1ull << (SB_COUNT + 1)) - 1) << EV_SYM0;
  OCEAN_CUDA(cudaGetLastError());
  if (with_scan) {
    h->st.launches += launch_scan(h->w, h->w.row_nnz, h->w.rowptr64, h->w.rowptr32, &h->w.ctr->total_nnz, true, np, s,
                                  seg_num(h));
    OCEAN_CUDA(cudaGetLastError());
  }
  if (track) record(h, EV_SCAN, s);
  OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
  OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
  check_device_status(h);
}

// Analysis + symbolic + scan (ocean_symbolic and the precise workflow).
template <typename RP>
void run_front(ocean_handle* h, const Csr<RP>& A, const Csr<RP>& B, cudaStream_t s, bool with_scan,
               bool allow_cache) {
  const bool readback = run_analysis(h, A, B, s);
  run_symbolic(h, A, B, s, readback, with_scan, allow_cache);
}

// Stops using the saved bitmaps for this call (the buffer stays with the handle).
void release_cache(ocean_handle* h, cudaStream_t) {
  h->w.bm_cache = nullptr;
  h->w.bm_cache_words = 0;
}

// Frees the saved-bitmap buffer (when C needs the memory).
void drop_cache_buffer(ocean_handle* h, cudaStream_t s) {
  release_cache(h, s);
  if (h->cache_buf) {
    cudaStreamSynchronize(s);
    cudaFree(h->cache_buf);
  }
  h->cache_buf = nullptr;
  h->cache_cap_words = 0;
}

// Loads the estimator network once: from learned_estimator_weights (text:
// the tag "ocean-mlp-v1", then kMlpBlob numbers) or the built-in one.
void load_model(ocean_handle* h) {
  if (h->mlp_ready) return;
  std::vector<float> blob(kMlpBlob);
  const std::string& path = h->cfg.learned_estimator_weights;
  if (!path.empty()) {
    std::ifstream f(path);
    OCEAN_CHECK(f.good(), OCEAN_ERR_INVALID, "cannot open learned_estimator_weights file");
    std::string tag;
    f >> tag;
    OCEAN_CHECK(tag == "ocean-mlp-v1", OCEAN_ERR_INVALID, "learned_estimator_weights: not an ocean-mlp-v1 file");
    for (auto& x : blob) f >> x;
    OCEAN_CHECK(!f.fail(), OCEAN_ERR_INVALID, "learned_estimator_weights: expected 5346 numbers");
  } else {
    OCEAN_CHECK(kMlpBuiltinTrained != 0, OCEAN_ERR_INVALID,
                "no trained estimator is built in; set learned_estimator_weights");
    std::copy(kMlpBuiltin, kMlpBuiltin + kMlpBlob, blob.begin());
  }
  if (!h->mlp_dev) OCEAN_CUDA(cudaMalloc((void**)&h->mlp_dev, kMlpBlob * sizeof(float)));
  OCEAN_CUDA(cudaMemcpy(h->mlp_dev, blob.data(), kMlpBlob * sizeof(float), cudaMemcpyHostToDevice));
  h->mlp_margin = blob[kMlpBlob - 1];
  h->mlp_ready = true;
}

MlpModel model_of(const ocean_handle* h) {
  MlpModel m;
  m.params = h->mlp_dev;
  m.mu = h->mlp_dev + kMlpParams;
  m.inv_sd = m.mu + kMlpF;
  m.margin = h->mlp_margin * (float)h->cfg.learned_margin_scale;
  return m;
}

// The estimator's per-row inputs: the analysis arrays, the raw HLL estimates
// in w.est, and two scalars of B.
template <typename RP>
MlpRowInputs row_inputs(const DevWork& w, const Csr<RP>& B) {
  MlpRowInputs in;
  in.anz = w.anz;
  in.prod = w.prod;
  in.lo = w.lo;
  in.hi = w.hi;
  in.maxb = w.maxb;
  in.hll = w.est;
  in.log_b_cols = log2f(1.f + (float)B.cols);
  in.log_b_avg = log2f(1.f + (B.rows ? (float)((double)B.nnz / (double)B.rows) : 0.f));
  return in;
}

// Log2 precision of the HLL sketch the learned estimator's features use.
constexpr int kLearnedLog2p = 5;

// Workflow ids as reported in the stats (reference: kernels/SpGEMM.cuh:1807-1817).
// Output columns below which the FAT workflow applies: the reference's largest
// dense numeric bin, 64 KB / 9 B - 4 (include/Common.h:78-110,261-269).
constexpr uint64_t kFatMaxCols = 7277;
enum Workflow { WF_PRECISE = 0, WF_ESTIMATION = 1, WF_ULTRASPARSE = 2, WF_FAT = 3 };

// Chooses the workflow after the analysis (reference rules,
// kernels/SpGEMM.cuh:456-540 and kernels/Analysis.cuh:10-29):
//  * ultra-sparse when the mean row has at most usparse_avg_product_threshold
//    products: every row's estimate is its product count (never overflows);
//  * estimation when products / nnz(A) reaches estimation_input_expansion_threshold
//    and the HLL-sampled compaction (products per estimated output) reaches
//    estimation_output_compaction_threshold twice (sum ratio and mean ratio);
//  * precise otherwise, for small inputs (no read-back), or when the temporary
//    output of an estimated workflow would not fit in memory.
// For the estimation workflow the HLL estimates are left in w.est.
template <typename RP>
int choose_workflow(ocean_handle* h, const Csr<RP>& A, const Csr<RP>& B, cudaStream_t s, bool readback) {
  const Config& c = h->cfg;
  // short, fat A times tall, skinny B with few output columns
  // (kernels/SpGEMM.cuh:456-466): every row gets its exact upper bound
  // min(products, span) <= B.cols as its slots, so nothing overflows
  const bool fat = c.use_fat_workflow && c.fat_ratio > 0 && A.cols / (uint64_t)c.fat_ratio > A.rows &&
                   B.rows / (uint64_t)c.fat_ratio > B.cols && B.cols < kFatMaxCols;
  if (c.force_workflow == WF_FAT || (c.force_workflow < 0 && fat)) {
    h->st.launches += launch_row_bounds(h->w, h->w.est, s);
    h->st.estimator = 3;
    return WF_FAT;
  }
  if (c.force_workflow == WF_PRECISE || (!readback && c.force_workflow < 0)) return WF_PRECISE;
  const DevCounters& k = *h->h_ctr;
  const uint64_t products = readback ? k.total_products : 0;
  if (c.force_workflow == WF_ULTRASPARSE ||
      (c.force_workflow < 0 && c.use_ultrasparse_workflow && A.rows &&
       (double)products / (double)A.rows <= c.usparse_avg_product_threshold &&
       fits_device(h, 12.0 * (double)products, 0.4))) {
    OCEAN_CUDA(cudaMemcpyAsync(h->w.est, h->w.prod, A.rows * 4, cudaMemcpyDeviceToDevice, s));
    return WF_ULTRASPARSE;
  }
  if (c.force_workflow < 0) {
    if (!c.use_estimation_workflow) return WF_PRECISE;
    if (A.nnz == 0 || products / A.nnz < (uint64_t)c.estimation_input_expansion_threshold) return WF_PRECISE;
  }
  // HLL estimates and sampled compaction
  const uint64_t ratio = A.nnz ? products / A.nnz : 0;
  const bool learned = c.use_learned_estimator;
  if (learned) load_model(h);
  const int log2p = learned ? kLearnedLog2p
                            : (readback && ratio >= (uint64_t)c.hll_higher_precision_expansion_threshold) ? 6 : 5;
  const double expansion = (log2p == 5 ? 2.0 : 1.5) * c.estimate_scale;
  int samples = (int)(A.rows * c.hll_sample_rate);
  samples = std::max(samples, c.hll_sample_min_rows);
  samples = std::min(samples, c.hll_sample_max_rows);
  void* sk = nullptr;
  OCEAN_CUDA(cudaMallocAsync(&sk, std::max<uint64_t>(B.rows, 1) << log2p, s));
  int wf = WF_ESTIMATION;
  try {
    h->st.launches += launch_hll_sketch_sample(A, B, h->w, log2p, (unsigned)samples, (uint8_t*)sk, s);
    OCEAN_CUDA(cudaGetLastError());
    OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(wait_stream(s, c.spin_wait_us));
    h->st.hll_log2p = log2p;
    h->st.hll_expansion = expansion;
    const unsigned n = h->h_ctr->sample_rows;
    h->st.compaction1 = n && h->h_ctr->sample_est > 0 ? (double)h->h_ctr->sample_products / h->h_ctr->sample_est : 0.0;
    h->st.compaction2 = n ? h->h_ctr->sample_compaction / n : 0.0;
    h->st.sampled = true;
    if (c.force_workflow != WF_ESTIMATION && (h->st.compaction1 < c.estimation_output_compaction_threshold ||
                                              h->st.compaction2 < c.estimation_output_compaction_threshold))
      wf = WF_PRECISE;
    if (wf == WF_ESTIMATION) {
      uint32_t* raw = nullptr;
      if (c.estimator_metrics) {
        grow(h->raw_est, h->raw_est_cap, A.rows);
        raw = h->raw_est;
      }
      if (learned) {
        // raw HLL estimates become a feature; the network then writes the estimates over them
        // (rows of at most esc_max products take their product count and need no HLL)
        h->st.launches += launch_hll_rows(A, h->w, log2p, 1.0, (uint32_t)c.esc_max_products, true,
                                          (const uint8_t*)sk, h->w.est, s);
        h->st.launches += launch_mlp_estimate(model_of(h), row_inputs(h->w, B), A.rows, (uint32_t)c.esc_max_products,
                                              h->w.est, raw, &h->w.ctr->status, h->num_sms, s);
        h->st.estimator = 2;
      } else {
        if (raw) h->st.launches += launch_hll_rows(A, h->w, log2p, 1.0, (uint32_t)c.esc_max_products, false,
                                                   (const uint8_t*)sk, raw, s);
        h->st.launches += launch_hll_rows(A, h->w, log2p, expansion, (uint32_t)c.esc_max_products, false,
                                          (const uint8_t*)sk, h->w.est, s);
        h->st.estimator = 1;
      }
      OCEAN_CUDA(cudaGetLastError());
    }
  } catch (...) {
    cudaFreeAsync(sk, s);
    throw;
  }
  cudaFreeAsync(sk, s);
  return wf;
}

// estimator_metrics: error of the preallocated estimates (w.est) and of the
// estimates without margin/expansion (raw_est) against the exact counts (w.cnt).
template <typename RP>
void measure_estimates(ocean_handle* h, const Csr<RP>& B, const NumPolicy& np, cudaStream_t s) {
  if (!h->metrics_dev) OCEAN_CUDA(cudaMalloc((void**)&h->metrics_dev, 8 * sizeof(double)));
  OCEAN_CUDA(cudaMemsetAsync(h->metrics_dev, 0, 8 * sizeof(double), s));
  const MlpRowInputs in = row_inputs(h->w, B);
  launch_est_metrics(h->w.est, h->w.cnt, in, h->w.rows, np, 0u, h->metrics_dev, s);
  launch_est_metrics(h->raw_est, h->w.cnt, in, h->w.rows, np, 0u, h->metrics_dev + 4, s);
  h->st.launches += 2;
  double m[8];
  OCEAN_CUDA(cudaMemcpyAsync(m, h->metrics_dev, sizeof m, cudaMemcpyDeviceToHost, s));
  OCEAN_CUDA(cudaStreamSynchronize(s));
  Stats& st = h->st;
  st.metrics = true;
  st.metric_rows = (uint64_t)m[1];
  st.mre = m[1] > 0 ? m[0] / m[1] : 0.0;
  st.mre_raw = m[5] > 0 ? m[4] / m[5] : 0.0;
  st.misbinned = m[1] > 0 ? 100.0 * m[2] / m[1] : 0.0;
  st.misbinned_raw = m[5] > 0 ? 100.0 * m[6] / m[5] : 0.0;
}

// C's buffers; if they do not fit and bitmaps are saved, the bitmaps are
// dropped (the numeric pass then marks its columns itself) and C retried.
void alloc_c(ocean_handle* h, CResult* owner, uint64_t rows, uint64_t nnz, int bits, cudaStream_t s) {
  auto attempt = [&]() -> cudaError_t {
    cudaError_t e = cudaMallocAsync(&owner->rowptr, (rows + 1) * (bits / 8), s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&owner->col, std::max<uint64_t>(nnz, 1) * 4, s);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&owner->val, std::max<uint64_t>(nnz, 1) * 8, s);
    return e;
  };
  cudaError_t e = attempt();
  if (e != cudaSuccess && h->w.bm_cache) {
    cudaGetLastError();
    for (void** p : {&owner->rowptr, (void**)&owner->col, (void**)&owner->val}) {
      if (*p) cudaFreeAsync(*p, s);
      *p = nullptr;
    }
    drop_cache_buffer(h, s);
    h->st.cache_dropped = true;
    e = attempt();
  }
  OCEAN_CUDA(e);
}

// The chunked numeric phase of a host-buffer multiply (h->w.chunks > 0, the
// chunk bounds and class sizes read back into h->chunk_host): C's row
// pointers go to the pinned host buffer first; then for every row chunk its
// numeric class kernels run on s, and an event lets copy_stream copy the
// chunk's column ids and values (contiguous in C) to the host while the
// following chunks compute. s waits for the copies at the end, so the caller's
// stream order covers them. Returns the kernels launched.
template <typename RP>
int pipeline_numeric(ocean_handle* h, const Csr<RP>& A, const Csr<RP>& B, const OutSpec& exact, CResult* owner,
                     uint64_t nnz, int bits, cudaStream_t s) {
  const int k = h->w.chunks;
  const uint32_t* bound = h->chunk_host;
  const uint32_t* counts = h->chunk_host + (kMaxChunks + 1);
  const uint64_t rpb = (A.rows + 1) * (uint64_t)(bits / 8);
  grow_host(h->out_rp, h->out_rp_cap, rpb);
  grow_host(h->out_col, h->out_col_cap, nnz);
  grow_host(h->out_val, h->out_val_cap, nnz);
  OCEAN_CUDA(cudaMemcpyAsync(h->out_rp, bits == 64 ? (void*)h->w.rowptr64 : (void*)h->w.rowptr32, rpb,
                             cudaMemcpyDeviceToHost, s));
  OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
  auto offset = [&](uint32_t r) -> uint64_t {
    return bits == 64 ? ((const uint64_t*)h->out_rp)[r] : (uint64_t)((const uint32_t*)h->out_rp)[r];
  };
  int launched = 0;
  for (int c = 0; c < k; ++c) {
    const uint32_t r0 = bound[c], r1 = bound[c + 1];
    if (r1 <= r0) continue;
    unsigned cc[NB_COUNT];
    for (int i = 0; i < NB_COUNT; ++i) cc[i] = counts[i * k + c];
    launched += launch_numeric(A, B, h->w, exact, owner->col, owner->val, h->num_sms, s, nullptr, cc, c, r0);
    OCEAN_CUDA(cudaEventRecord(h->chunk_ev[c], s));
    OCEAN_CUDA(cudaStreamWaitEvent(h->copy_stream, h->chunk_ev[c], 0));
    const uint64_t o0 = offset(r0), o1 = offset(r1);
    if (o1 > o0) {
      OCEAN_CUDA(cudaMemcpyAsync(h->out_col + o0, owner->col + o0, (o1 - o0) * 4, cudaMemcpyDeviceToHost,
                                 h->copy_stream));
      OCEAN_CUDA(cudaMemcpyAsync(h->out_val + o0, owner->val + o0, (o1 - o0) * 8, cudaMemcpyDeviceToHost,
                                 h->copy_stream));
    }
  }
  OCEAN_CUDA(cudaEventRecord(h->chunk_ev[kMaxChunks], h->copy_stream));
  OCEAN_CUDA(cudaStreamWaitEvent(s, h->chunk_ev[kMaxChunks], 0));
  h->st.host_chunks = k;
  h->w.chunks = 0;
  h->sink_filled = true;
  return launched;
}

template <typename RP>
void run_spgemm(ocean_handle* h, const ocean_csr_view* Av, const ocean_csr_view* Bv, const RP* arp,
                const RP* brp, ocean_csr* C, cudaStream_t s) {
  const auto t0 = std::chrono::steady_clock::now();
  const Csr<RP> A = to_csr<RP>(Av, arp);
  const Csr<RP> B = to_csr<RP>(Bv, brp);
  Stats& st = h->st;
  st = Stats();
  auto mark = [&](const char* what) {
    st.host_marks.emplace_back(what, std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
  };
  st.a_rows = A.rows, st.a_cols = A.cols, st.a_nnz = A.nnz;
  st.b_rows = B.rows, st.b_cols = B.cols, st.b_nnz = B.nnz;
  h->ev_recorded = false;
  h->ev_mask = 0;
  h->seg_ran = false;
  h->seg_dispatched = false;
  const bool track = h->cfg.track_stage_times;
  NumPolicy np;
  {
    SymPolicy sp;
    make_policies(h->cfg, &sp, &np);
  }

  uint64_t nnz = 0;
  int wf = WF_PRECISE;
  void* t_col = nullptr;  // temporary output of the estimated workflows
  void* t_val = nullptr;
  CResult* owner = new CResult{0};
  try {
    if (A.rows > 0) {
      const bool readback = run_analysis(h, A, B, s);
      mark("analysis");
      if (h->cfg.use_segmented_workflow || h->cfg.use_segment_dispatch) {
        // spy-plot segmentation; its records go to the stats (reference:
        // kernels/SpGEMM.cuh:240-259, where it is analysis-only)
        const Config& c = h->cfg;
        OCEAN_CUDA(run_segmentation(A, B.cols, h->w, c.segmentation_grid_max, c.segmentation_hot_threshold_k,
                                    c.segmentation_min_segment_rows, c.segmentation_cc_max_iters,
                                    c.estimation_input_expansion_threshold, s, &h->seg));
        h->seg_ran = true;
        if (c.use_segment_dispatch) {
          // segment-driven dispatch (the reference's listed follow-up,
          // kernels/SpGEMM.cuh:241-244): every row of a segment takes its
          // class's policy, and the rows are classed again with them
          dispatch_segments(h, A, B, s, readback);
          mark("segment_dispatch");
        }
      }
      wf = choose_workflow(h, A, B, s, readback);
      mark("workflow");
      // numeric class sizes on the host (grids capped by class size); without
      // them every class is launched at full grid
      bool class_counts = true;
      // ultra-sparse rows of at most 256 products: one fused launch writes C
      // in place (capacity: the product count, read back by the analysis).
      // Small inputs skip the analysis read-back on the precise path; here
      // the counters are read back once to see whether the fused path applies.
      const Config& cf = h->cfg;
      const bool fusable_cfg = cf.fused_ultrasparse && !cf.estimator_metrics && !cf.use_segment_dispatch &&
                               (cf.force_workflow == WF_ULTRASPARSE ||
                                (cf.force_workflow < 0 && cf.use_ultrasparse_workflow));
      bool fresh = readback;  // h_ctr holds this call's analysis counters
      if (!readback && fusable_cfg && (wf == WF_PRECISE || wf == WF_ULTRASPARSE)) {
        OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
        OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
        fresh = true;
        mark("fused_probe");
      }
      const DevCounters& kc = *h->h_ctr;
      const bool fits = fresh && kc.max_products <= kUspMaxProducts && kc.total_products < (1ull << 32);
      if (fits && wf == WF_PRECISE && !readback && cf.force_workflow < 0 &&
          (double)kc.total_products <= cf.usparse_avg_product_threshold * (double)A.rows)
        wf = WF_ULTRASPARSE;
      st.fused = fits && fusable_cfg && wf == WF_ULTRASPARSE;
      if (st.fused) {
        nnz = h->h_ctr->total_products;  // C's capacity until the kernel has counted
        st.total_est = nnz;
      } else if (wf == WF_ULTRASPARSE && readback) {
        // the estimates are the product counts, whose total the analysis read
        // back and choose_workflow checked against free memory: no read-back
        st.launches += launch_scan(h->w, h->w.est, h->w.est_off, nullptr, &h->w.ctr->total_est, true, np, s,
                                   seg_num(h));
        st.total_est = h->h_ctr->total_products;
        class_counts = false;
      } else if (wf == WF_ESTIMATION || wf == WF_ULTRASPARSE || wf == WF_FAT) {
        // scan of the estimates: temporary slots per row, numeric classes by estimate
        st.launches += launch_scan(h->w, h->w.est, h->w.est_off, nullptr, &h->w.ctr->total_est, true, np, s,
                                   seg_num(h));
        OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
        OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
        st.total_est = h->h_ctr->total_est;
        if (!fits_device(h, 12.0 * (double)st.total_est, 0.45)) {
          wf = WF_PRECISE;  // the temporary output would not fit: count exactly instead
          OCEAN_CUDA(cudaMemsetAsync(h->w.ctr->num_count, 0, sizeof(unsigned) * NB_COUNT * 2, s));
        }
      }
      // host-buffer multiplies of many products: the numeric phase runs in
      // row chunks of equal products (the scan splits the class lists by
      // chunk) so that each chunk's copy to the host overlaps the next ones
      h->w.chunks = 0;
      if (h->sink_active && wf == WF_PRECISE && readback && !st.fused && !cf.numeric_windows && !track &&
          cf.host_pipeline_chunks > 1 && (double)h->h_ctr->total_products >= cf.host_pipeline_min_products) {
        const int k = std::min(cf.host_pipeline_chunks, kMaxChunks);
        const size_t words = (kMaxChunks + 1) + 2 * NB_COUNT * kMaxChunks;
        if (!h->chunk_dev) {
          OCEAN_CUDA(cudaMalloc((void**)&h->chunk_dev, words * 4));
          OCEAN_CUDA(cudaHostAlloc((void**)&h->chunk_host, words * 4, cudaHostAllocDefault));
        }
        if (!h->copy_stream) {
          OCEAN_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
          for (auto& e : h->chunk_ev) OCEAN_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        }
        h->w.chunks = k;
        h->w.chunk_bound = h->chunk_dev;
        h->w.chunk_count = h->chunk_dev + (kMaxChunks + 1);
        h->w.chunk_cursor = h->w.chunk_count + NB_COUNT * kMaxChunks;
        OCEAN_CUDA(cudaMemsetAsync(h->w.chunk_count, 0, 2 * NB_COUNT * kMaxChunks * 4, s));
        // exclusive scan of the products (into est_off, unused by this workflow), then the bounds
        st.launches += launch_scan(h->w, h->w.prod, h->w.est_off, nullptr, &h->w.ctr->total_est, false, np, s);
        launch_chunk_bounds(h->w, h->w.est_off, k, s);
        st.launches += 1;
      }
      if (st.fused) {
      } else if (wf == WF_PRECISE) {
        run_symbolic(h, A, B, s, readback, true, true);
        mark("symbolic");
        nnz = h->h_ctr->total_nnz;
        if (h->w.chunks) {
          OCEAN_CUDA(cudaMemcpyAsync(h->chunk_host, h->chunk_dev, ((kMaxChunks + 1) + NB_COUNT * kMaxChunks) * 4,
                                     cudaMemcpyDeviceToHost, s));
          OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
        }
      } else {
        OCEAN_CUDA(cudaMallocAsync(&t_col, std::max<uint64_t>(st.total_est, 1) * 4, s));
        OCEAN_CUDA(cudaMallocAsync(&t_val, std::max<uint64_t>(st.total_est, 1) * 8, s));
        OCEAN_CUDA(cudaMemsetAsync(h->w.cnt, 0, A.rows * 4, s));
        unsigned num_counts[NB_COUNT];
        for (int i = 0; i < NB_COUNT; ++i) num_counts[i] = h->h_ctr->num_count[i];
        const OutSpec est_out{h->w.est_off, h->w.est, h->w.cnt, h->w.ovf, &h->w.ctr->overflow_n};
        st.bm_kernel = num_counts[NB_BITMAP] ? 1 : 0;
        st.launches += launch_numeric(A, B, h->w, est_out, (uint32_t*)t_col, (double*)t_val, h->num_sms, s,
                                      track ? h->ev + EV_NUM0 : nullptr, class_counts ? num_counts : nullptr);
        if (track) h->ev_mask |= ((1ull << (NB_COUNT + 1)) - 1) << EV_NUM0;
        // rows that did not fit their estimate: exact counts, then the row pointers
        st.launches += launch_overflow(A, B, h->w, false, nullptr, nullptr, h->num_sms, s);
        st.launches += launch_scan(h->w, h->w.cnt, h->w.rowptr64, h->w.rowptr32, &h->w.ctr->total_nnz, false, np, s);
        OCEAN_CUDA(cudaGetLastError());
        OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
        OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
        check_device_status(h);
        mark("estimated_numeric");
        nnz = h->h_ctr->total_nnz;
        st.overflow_rows = h->h_ctr->overflow_n;
        if (h->cfg.estimator_metrics && st.estimator != 0) measure_estimates(h, B, np, s);
      }
    } else {
      std::memset(h->h_ctr, 0, sizeof(DevCounters));
    }
    const int bits = h->cfg.output_rowptr_bits ? h->cfg.output_rowptr_bits : (nnz >= (1ull << 32) ? 64 : 32);
    OCEAN_CHECK(!(bits == 32 && nnz >= (1ull << 32)), OCEAN_ERR_INVALID,
                "nnz(C) >= 2^32 does not fit 32-bit row pointers (output_rowptr_bits=32)");
    st.rowptr_bits = bits;
    st.cache_words = h->w.bm_cache_words;
    st.cache_used = std::min<uint64_t>(h->h_ctr->cache_cursor, h->w.bm_cache_words);
    alloc_c(h, owner, A.rows, nnz, bits, s);
    mark("alloc_c");
    if (A.rows > 0) {
      if (st.fused) {
        grow(h->usp_tiles_buf, h->usp_tiles_cap, usp_tiles(A.rows));
        // stage events: the fused kernel is reported as the numeric ESC1 stage
        if (track) record(h, EV_NUM0, s);
        st.launches += launch_usp_fused(A, B, h->w, h->usp_tiles_buf, nnz, bits == 32, owner->col, owner->val, s);
        if (track) {
          for (int i = EV_NUM0 + 1; i <= EV_NUM0 + NB_COUNT; ++i) record(h, i, s);
          h->ev_mask |= ((1ull << (NB_COUNT + 1)) - 1) << EV_NUM0;
        }
      } else if (wf == WF_PRECISE) {
        unsigned num_counts[NB_COUNT];
        for (int i = 0; i < NB_COUNT; ++i) num_counts[i] = h->h_ctr->num_count[i];
        prepare_windows(h, A.nnz, num_counts[NB_BITMAP]);
        const OutSpec exact{h->w.rowptr64, h->w.row_nnz, nullptr, nullptr, nullptr};
        if (h->w.chunks) {
          st.launches += pipeline_numeric(h, A, B, exact, owner, nnz, bits, s);
        } else {
          st.launches += launch_numeric(A, B, h->w, exact, owner->col, owner->val, h->num_sms, s,
                                        track ? h->ev + EV_NUM0 : nullptr, num_counts);
        }
        if (track) h->ev_mask |= ((1ull << (NB_COUNT + 1)) - 1) << EV_NUM0;
      } else {
        launch_copy_rows(h->w, (const uint32_t*)t_col, (const double*)t_val, owner->col, owner->val, s);
        st.launches += 1;
        if (st.overflow_rows) st.launches += launch_overflow(A, B, h->w, true, owner->col, owner->val, h->num_sms, s);
        cudaFreeAsync(t_col, s);
        cudaFreeAsync(t_val, s);
        t_col = t_val = nullptr;
      }
      OCEAN_CUDA(cudaGetLastError());
      OCEAN_CUDA(cudaMemcpyAsync(owner->rowptr, bits == 64 ? (void*)h->w.rowptr64 : (void*)h->w.rowptr32,
                                 (A.rows + 1) * (bits / 8), cudaMemcpyDeviceToDevice, s));
    } else {
      OCEAN_CUDA(cudaMemsetAsync(owner->rowptr, 0, bits / 8, s));
      for (int i = EV_START; i < EV_END; ++i) record(h, i, s);
    }
    release_cache(h, s);
    record(h, EV_END, s);
    h->ev_recorded = true;
    h->tracked = track;
    mark("launched");
    if ((h->cfg.sync_on_return || st.fused) && A.rows > 0) {
      // (the fused path needs the count the kernel wrote: it always waits)
      OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
      OCEAN_CUDA(wait_stream(s, h->cfg.spin_wait_us));
      check_device_status(h);
      if (st.fused) nnz = h->h_ctr->total_nnz;
      mark("synced");
    }
  } catch (...) {
    h->w.chunks = 0;
    if (h->copy_stream) cudaStreamSynchronize(h->copy_stream);  // no copy may still read C
    release_cache(h, s);
    if (t_col) cudaFreeAsync(t_col, s);
    if (t_val) cudaFreeAsync(t_val, s);
    if (owner->rowptr) cudaFreeAsync(owner->rowptr, s);
    if (owner->col) cudaFreeAsync(owner->col, s);
    if (owner->val) cudaFreeAsync(owner->val, s);
    delete owner;
    throw;
  }
  C->rows = A.rows;
  C->cols = B.cols;
  C->nnz = nnz;
  C->rowptr = owner->rowptr;
  C->rowptr_bits = st.rowptr_bits;
  C->col = owner->col;
  C->val = owner->val;
  C->location = 0;
  C->_owner = owner;

  st.c_rows = A.rows, st.c_cols = B.cols, st.c_nnz = nnz;
  st.total_products = h->h_ctr->total_products;
  st.max_products = h->h_ctr->max_products;
  st.max_a_nnz = h->h_ctr->max_a_nnz;
  for (int i = 0; i < SB_COUNT; ++i) st.sym_bins[i] = h->h_ctr->sym_count[i];
  for (int i = 0; i < NB_COUNT; ++i) st.num_bins[i] = h->h_ctr->num_count[i];
  for (int i = 0; i < NB_COUNT; ++i) {
    st.num_nnz[i] = h->h_ctr->num_nnz[i];
    st.num_anz[i] = h->h_ctr->num_anz[i];
    st.num_prod[i] = h->h_ctr->num_prod[i];
  }
  for (int i = 0; i < SB_COUNT; ++i) {
    st.sym_anz[i] = h->h_ctr->sym_anz[i];
    st.sym_prod[i] = h->h_ctr->sym_prod[i];
  }
  st.workflow = wf;
  st.valid = true;
  st.host_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// Dispatch on row-pointer widths (mixed widths are widened to 64 bits).
void dispatch_spgemm(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, ocean_csr* C,
                     cudaStream_t s) {
  validate_view(A, "A");
  validate_view(B, "B");
  OCEAN_CHECK(A->cols == B->rows, OCEAN_ERR_INVALID, "Incompatible matrix dimensions (A.cols != B.rows)");
  OCEAN_CHECK(C != nullptr, OCEAN_ERR_INVALID, "C is NULL");
  OCEAN_CHECK(!(h->cfg.use_hybrid_accumulator && !h->cfg.use_indirect_sort), OCEAN_ERR_INVALID,
              "Invalid configuration: use_hybrid_accumulator requires use_indirect_sort");
  if (A->rowptr_bits == 32 && B->rowptr_bits == 32) {
    run_spgemm<uint32_t>(h, A, B, (const uint32_t*)A->rowptr, (const uint32_t*)B->rowptr, C, s);
    return;
  }
  const uint64_t* arp = (const uint64_t*)A->rowptr;
  const uint64_t* brp = (const uint64_t*)B->rowptr;
  if (A->rowptr_bits == 32 && A->rows) {
    grow(h->wide_a, h->wide_a_cap, A->rows + 1);
    k_widen_rowptr<<<256, 256, 0, s>>>((const uint32_t*)A->rowptr, h->wide_a, A->rows);
    arp = h->wide_a;
  }
  if (B->rowptr_bits == 32 && B->rows) {
    grow(h->wide_b, h->wide_b_cap, B->rows + 1);
    k_widen_rowptr<<<256, 256, 0, s>>>((const uint32_t*)B->rowptr, h->wide_b, B->rows);
    brp = h->wide_b;
  }
  OCEAN_CUDA(cudaGetLastError());
  run_spgemm<uint64_t>(h, A, B, arp, brp, C, s);
}

// Milliseconds between two events of the last call; -1 when either was not
// recorded. A failed query does not leave an error behind for the caller.
double ev_ms(ocean_handle* h, int a, int b) {
  if (!h->ev_recorded || !((h->ev_mask >> a) & 1) || !((h->ev_mask >> b) & 1)) return -1.0;
  float ms = 0.f;
  if (cudaEventSynchronize(h->ev[b]) != cudaSuccess || cudaEventElapsedTime(&ms, h->ev[a], h->ev[b]) != cudaSuccess) {
    cudaGetLastError();
    return -1.0;
  }
  return ms;
}

std::string stats_json(ocean_handle* h) {
  const Stats& st = h->st;
  std::ostringstream o;
  o.precision(17);
  auto dims = [&](const char* n, uint64_t r, uint64_t c, uint64_t z) {
    o << "\"" << n << "\": {\"rows\": " << r << ", \"cols\": " << c << ", \"nnz\": " << z << "}, ";
  };
  o << "{";
  dims("A", st.a_rows, st.a_cols, st.a_nnz);
  dims("B", st.b_rows, st.b_cols, st.b_nnz);
  dims("C", st.c_rows, st.c_cols, st.c_nnz);
  const double avg = st.a_rows ? (double)st.total_products / (double)st.a_rows : 0.0;
  const double ie = st.a_nnz ? (double)st.total_products / (double)st.a_nnz : 0.0;
  const double oc = st.c_nnz ? (double)st.total_products / (double)st.c_nnz : 0.0;
  o << "\"stats\": {\"intermediate_product\": " << st.total_products
    << ", \"intermediate_product_max\": " << st.max_products << ", \"intermediate_product_avg\": " << avg
    << ", \"input_expansion\": " << ie << ", \"output_compression\": " << oc
    << ", \"max_a_row_nnz\": " << st.max_a_nnz << "}, ";
  o << "\"decision\": {\"workflow\": " << st.workflow << ", \"rowptr_bits\": " << st.rowptr_bits
    << ", \"bitmap_cache_bytes\": " << 8 * st.cache_words << ", \"bitmap_cache_used_bytes\": " << 8 * st.cache_used
    << ", \"bitmap_cache_dropped\": " << (st.cache_dropped ? "true" : "false")
    << ", \"fused_ultrasparse\": " << (st.fused ? "true" : "false")
    << ", \"numeric_bitmap_kernel\": \"" << (st.bm_kernel == 2 ? "window" : st.bm_kernel == 1 ? "rank" : "none")
    << "\", \"host_pipeline_chunks\": " << st.host_chunks << ", \"kernel_launches\": " << st.launches << "}, ";
  if (st.sampled)
    o << "\"sampling\": {\"compaction_1\": " << st.compaction1 << ", \"compaction_2\": " << st.compaction2
      << "}, ";
  if (st.workflow == 1 || st.workflow == 2 || st.workflow == 3) {
    o << "\"estimation\": {\"overflow_rows\": " << st.overflow_rows << ", \"log2_precision\": " << st.hll_log2p
      << ", \"total_est\": " << st.total_est << ", \"expansion\": " << st.hll_expansion << ", \"estimator\": \""
      << (st.estimator == 3 ? "bound" : st.estimator == 2 ? "learned" : st.estimator == 1 ? "hll" : "products")
      << "\"";
    if (st.metrics)
      o << ", \"metrics\": {\"rows\": " << st.metric_rows << ", \"mean_rel_error\": " << st.mre
        << ", \"misbinned_pct\": " << st.misbinned << ", \"mean_rel_error_raw\": " << st.mre_raw
        << ", \"misbinned_pct_raw\": " << st.misbinned_raw << "}";
    o << "}, ";
  }
  if (h->seg_ran) {
    // reference: kernels/SpGEMM.cuh:1851-1886
    const SegmentationResult& g = h->seg;
    o << "\"segmentation\": {\"grid_h\": " << g.grid_h << ", \"grid_w\": " << g.grid_w
      << ", \"tile_rows\": " << g.tile_rows << ", \"tile_cols\": " << g.tile_cols
      << ", \"density_mean\": " << g.density_mean << ", \"density_stddev\": " << g.density_stddev
      << ", \"num_components\": " << g.num_components << ", \"cc_iterations\": " << g.cc_iterations
      << ", \"time_density_ms\": " << g.time_density_ms << ", \"time_threshold_ms\": " << g.time_threshold_ms
      << ", \"time_cc_ms\": " << g.time_cc_ms << ", \"time_classify_ms\": " << g.time_classify_ms
      << ", \"segments\": [";
    for (size_t i = 0; i < g.segments.size(); ++i) {
      const SegRecord& r = g.segments[i];
      o << (i ? ", " : "") << "{\"row_start\": " << r.row_start << ", \"row_end\": " << r.row_end
        << ", \"row_count\": " << r.row_count << ", \"col_left\": " << r.col_left
        << ", \"col_right\": " << r.col_right << ", \"class\": \"" << segment_class_name(r.cls)
        << "\", \"sum_products\": " << r.sum_products << ", \"sum_a_nnz\": " << r.sum_a_nnz
        << ", \"mean_row_len\": " << r.mean_row_len << ", \"var_row_len\": " << r.var_row_len
        << ", \"local_er\": " << r.local_er << ", \"max_b_row_len\": " << r.max_b_row_len
        << ", \"max_a_row_len\": " << r.max_a_row_len << "}";
    }
    o << "]}, ";
  }
  if (h->seg_dispatched) {
    // rows per dispatch slot: outside every segment, then per segment class
    o << "\"segment_dispatch\": {\"rows\": {\"unsegmented\": " << h->seg_rows[0];
    static const char* kSegKey[4] = {"sparse_uniform", "dense", "power_law", "banded"};
    for (int k = 0; k < 4; ++k) o << ", \"" << kSegKey[k] << "\": " << h->seg_rows[1 + k];
    o << "}}, ";
  }
  o << "\"binning_1\": [";
  for (int i = 0; i < SB_COUNT; ++i) o << (i ? ", " : "") << st.sym_bins[i];
  o << "], \"binning_2\": [";
  for (int i = 0; i < NB_COUNT; ++i) o << (i ? ", " : "") << st.num_bins[i];
  o << "], \"classes\": {\"symbolic\": {";
  for (int i = 0; i < SB_COUNT; ++i)
    o << (i ? ", " : "") << "\"" << kSymNames[i] << "\": {\"rows\": " << st.sym_bins[i]
      << ", \"a_nnz\": " << st.sym_anz[i] << ", \"products\": " << st.sym_prod[i] << "}";
  o << "}, \"numeric\": {";
  for (int i = 0; i < NB_COUNT; ++i)
    o << (i ? ", " : "") << "\"" << kNumNames[i] << "\": {\"rows\": " << st.num_bins[i]
      << ", \"nnz\": " << st.num_nnz[i] << ", \"a_nnz\": " << st.num_anz[i]
      << ", \"products\": " << st.num_prod[i] << "}";
  o << "}}, ";
  const double total = ev_ms(h, EV_START, EV_END);
  if (h->tracked) {
    o << "\"timing\": {\"analysis\": " << ev_ms(h, EV_START, EV_ANALYSIS)
      << ", \"symbolic\": " << ev_ms(h, EV_SYM0, EV_SYMBOLIC) << ", \"scan\": " << ev_ms(h, EV_SYMBOLIC, EV_SCAN)
      << ", \"numeric\": " << ev_ms(h, EV_NUM0, EV_NUM_END);
    for (int i = 0; i < SB_COUNT; ++i)
      o << ", \"symbolic_" << kSymNames[i] << "\": " << ev_ms(h, EV_SYM0 + i, EV_SYM0 + i + 1);
    for (int i = 0; i < NB_COUNT; ++i)
      o << ", \"numeric_" << kNumNames[i] << "\": " << ev_ms(h, EV_NUM0 + i, EV_NUM0 + i + 1);
    o << ", \"host_ms\": " << st.host_ms << "}, ";
  }
  o << "\"host_timeline_ms\": {";
  for (size_t i = 0; i < st.host_marks.size(); ++i)
    o << (i ? ", " : "") << "\"" << st.host_marks[i].first << "\": " << st.host_marks[i].second;
  o << "}, ";
  o << "\"total_time\": " << total << ", \"gflops\": "
    << (total > 0 ? 2.0 * (double)st.total_products / total / 1e6 : 0.0) << "}";
  return o.str();
}

template <typename F>
int guarded(F&& f) {
  try {
    f();
    return OCEAN_OK;
  } catch (const OceanError& e) {
    g_last_error = e.msg;
    return e.code;
  } catch (const std::invalid_argument& e) {
    g_last_error = e.what();
    return OCEAN_ERR_INVALID;
  } catch (const std::bad_alloc&) {
    g_last_error = "host allocation failed";
    return OCEAN_ERR_OOM;
  } catch (const std::exception& e) {
    g_last_error = e.what();
    return OCEAN_ERR_INTERNAL;
  }
}

}  // namespace

namespace ocean {
void set_last_error(const char* msg) { g_last_error = msg ? msg : ""; }
}  // namespace ocean

namespace {
MlpModel model_from(const ocean_mlp_model* m) {
  OCEAN_CHECK(m != nullptr && m->params && m->mu && m->inv_sd, OCEAN_ERR_INVALID, "model pointers are NULL");
  MlpModel x;
  x.params = m->params;
  x.mu = m->mu;
  x.inv_sd = m->inv_sd;
  x.margin = m->margin;
  return x;
}

// Runs one MLP launch with the handle's status word and reports a timeout.
template <typename F>
void with_status(ocean_handle* h, cudaStream_t s, F&& launch) {
  OCEAN_CUDA(cudaMemsetAsync(&h->w.ctr->status, 0, sizeof(unsigned), s));
  launch(&h->w.ctr->status);
  OCEAN_CUDA(cudaGetLastError());
  OCEAN_CUDA(cudaMemcpyAsync(&h->h_ctr->status, &h->w.ctr->status, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
  OCEAN_CUDA(cudaStreamSynchronize(s));
  h->h_ctr->err_row = 0;
  check_device_status(h);
}
}  // namespace

// ---------------------------------------------------------------- batches
// A batch plan: many independent products C_p = A_p * B_p run as one
// block-diagonal product (see batch.cu). Planning stacks the inputs, runs the
// whole pipeline once with read-backs to learn the class sizes, the
// temporary and output sizes, and captures the same pipeline, without any
// read-back or allocation, into a CUDA graph; every run is then one graph
// launch. The plan owns its per-row arrays and counters, so calls on the
// handle in between do not disturb it; the handle (and the inputs' device
// buffers) must outlive the plan. The inputs' values (and columns) may change
// between runs; a run whose structure no longer matches the plan fails.
struct ocean_batch {
  ocean_handle* h = nullptr;
  Config cfg;  // the handle's config plus the tuned class policy
  uint32_t n = 0;
  bool same_b = false;  // every B_p is A_p: the stacked B shares A's row pointers and values
  int bits = 32;        // stacked input row-pointer width
  uint64_t rows = 0, nnz = 0, brows = 0, bnnz = 0, bcols = 0;
  std::vector<uint64_t> row0, nnz0, brow0, bnnz0;  // n + 1 prefixes
  std::vector<uint64_t> a_rows, b_cols;
  BatchProblem* d_probs = nullptr;
  uint64_t* d_pref = nullptr;  // row0 | nnz0 | brow0 | bnnz0 | out0 (n + 1 each)
  uint32_t* d_row_problem = nullptr;  // problem of every stacked row (learned estimator features)
  float2* d_ctx = nullptr;            // per problem: log2(1 + B.cols), log2(1 + nnz(B) / B.rows)
  void* a_rp = nullptr;
  uint32_t* a_col = nullptr;
  double* a_val = nullptr;
  void* b_rp = nullptr;
  uint32_t* b_col = nullptr;
  double* b_val = nullptr;
  DevWork w;
  int wf = 0;         // Workflow
  int estimator = 0;  // 0 products, 1 HLL, 2 learned
  int log2p = 5;
  double expansion = 1.0;
  uint8_t* sketch = nullptr;
  unsigned sym_counts[SB_COUNT] = {0};
  unsigned num_counts[NB_COUNT] = {0};
  uint64_t total_est = 0, c_nnz = 0, products = 0;
  int out_bits = 32;
  uint32_t* t_col = nullptr;
  double* t_val = nullptr;
  uint32_t* c_col = nullptr;
  double* c_val = nullptr;
  void* c_rp = nullptr;  // rows + n per-problem row pointers
  std::vector<uint64_t> c_off;  // n + 1 starts in the stacked C
  uint64_t* d_bounds = nullptr;  // the same, written by every run
  std::vector<uint64_t> h_bounds;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int launches = 0;  // kernels per run
  double tuned_ms = 0.0;
  std::string tuning;  // description of the tuned policy
  std::string tune_key;     // the batch's autotuning cache key
  bool tune_cached = false; // the knobs came from the autotuning cache
  DevCounters* h_ctr = nullptr;

  uint64_t* pref(int i) const { return d_pref + (uint64_t)i * (n + 1); }
  void drop_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }
  void free_arenas() {
    for (void* p : {(void*)t_col, (void*)t_val, (void*)c_col, (void*)c_val, (void*)c_rp})
      if (p) cudaFree(p);
    t_col = nullptr, t_val = nullptr, c_col = nullptr, c_val = nullptr, c_rp = nullptr;
  }
  ~ocean_batch() {
    drop_graph();
    free_arenas();
    free_work_rows(w);
    for (void* p : {(void*)w.ctr, (void*)d_probs, (void*)d_pref, a_rp, (void*)a_col, (void*)a_val, (void*)sketch,
                    (void*)d_bounds, (void*)d_row_problem, (void*)d_ctx})
      if (p) cudaFree(p);
    if (!same_b)
      for (void* p : {b_rp, (void*)b_col, (void*)b_val})
        if (p) cudaFree(p);
    else if (b_col)
      cudaFree(b_col);
    if (h_ctr) cudaFreeHost(h_ctr);
  }
};

namespace {

void batch_readback(ocean_batch* b, cudaStream_t s) {
  OCEAN_CUDA(cudaMemcpyAsync(b->h_ctr, b->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
  OCEAN_CUDA(cudaStreamSynchronize(s));
  if (b->h_ctr->status) {
    char buf[160];
    snprintf(buf, sizeof buf, "%s (status 0x%x, batched)", status_text(b->h_ctr->status), b->h_ctr->status);
    throw OceanError{(b->h_ctr->status & DEV_TC_TIMEOUT) ? (int)OCEAN_ERR_TIMEOUT : (int)OCEAN_ERR_CAPACITY, buf};
  }
}

// The whole batched pipeline on stream s. plan = true: with read-backs that
// fix the workflow, class sizes and buffer sizes (and allocate the arenas);
// plan = false: the same launches with those values, nothing else (capturable).
template <typename RP>
void batch_pipeline(ocean_batch* b, cudaStream_t s, bool plan) {
  ocean_handle* h = b->h;
  DevWork& w = b->w;
  const uint32_t n = b->n;
  SymPolicy sp;
  NumPolicy np;
  make_policies(b->cfg, &sp, &np);
  int launched = 0;
  // 1. stacked inputs
  launch_batch_rowptr<RP>(b->d_probs, b->pref(0), n, b->rows, b->nnz, false, (RP*)b->a_rp, s);
  launch_batch_entries(b->d_probs, b->pref(1), n, b->nnz, false, b->a_col, b->a_val, s);
  launched += 2;
  if (b->same_b) {
    launch_batch_entries(b->d_probs, b->pref(1), n, b->nnz, true, b->b_col, nullptr, s);
    launched += 1;
  } else {
    launch_batch_rowptr<RP>(b->d_probs, b->pref(2), n, b->brows, b->bnnz, true, (RP*)b->b_rp, s);
    launch_batch_entries(b->d_probs, b->pref(3), n, b->bnnz, true, b->b_col, b->b_val, s);
    launched += 2;
  }
  Csr<RP> A, B;
  A.rows = b->rows, A.cols = b->brows, A.nnz = b->nnz, A.rp = (const RP*)b->a_rp, A.col = b->a_col, A.val = b->a_val;
  B.rows = b->brows, B.cols = b->bcols, B.nnz = b->bnnz, B.rp = (const RP*)b->b_rp, B.col = b->b_col,
  B.val = b->b_val;
  // 2. analysis
  w.bm_cache = nullptr;
  w.bm_cache_words = 0;
  OCEAN_CUDA(cudaMemsetAsync(w.ctr, 0, sizeof(DevCounters), s));
  launched += launch_analysis(A, B, w, sp, s);
  if (plan) {
    batch_readback(b, s);
    const DevCounters& k = *b->h_ctr;
    for (int i = 0; i < SB_COUNT; ++i) b->sym_counts[i] = k.sym_count[i];
    b->products = k.total_products;
    const Config& c = b->cfg;
    const double avg = A.rows ? (double)k.total_products / (double)A.rows : 0.0;
    // as for one product: ultra-sparse inputs are sized by their product
    // counts (already exact upper bounds) before any estimator is asked
    if (c.force_workflow == WF_PRECISE) b->wf = WF_PRECISE;
    else if (c.force_workflow == WF_ESTIMATION) b->wf = WF_ESTIMATION;
    else if (c.force_workflow == WF_ULTRASPARSE || (c.use_ultrasparse_workflow && avg <= c.usparse_avg_product_threshold))
      b->wf = WF_ULTRASPARSE;
    else if (c.use_learned_estimator) b->wf = WF_ESTIMATION;
    else b->wf = WF_PRECISE;
    b->estimator = b->wf == WF_ESTIMATION ? (c.use_learned_estimator ? 2 : 1) : 0;
    if (b->estimator == 2) load_model(h);
    const uint64_t ratio = A.nnz ? k.total_products / A.nnz : 0;
    b->log2p = b->estimator == 2 ? kLearnedLog2p : (ratio >= (uint64_t)c.hll_higher_precision_expansion_threshold ? 6 : 5);
    b->expansion = (b->log2p == 5 ? 2.0 : 1.5) * c.estimate_scale;
    if (b->estimator && !b->sketch) OCEAN_CUDA(cudaMalloc((void**)&b->sketch, std::max<uint64_t>(B.rows, 1) << 6));
  }
  if (b->wf == WF_PRECISE) {
    launched += launch_symbolic(A, B, w, h->num_sms, s, nullptr, b->sym_counts);
    launched += launch_scan(w, w.row_nnz, w.rowptr64, w.rowptr32, &w.ctr->total_nnz, true, np, s);
    if (plan) {
      batch_readback(b, s);
      b->c_nnz = b->h_ctr->total_nnz;
      for (int i = 0; i < NB_COUNT; ++i) b->num_counts[i] = b->h_ctr->num_count[i];
    } else {
      launch_batch_guard(w.ctr, &w.ctr->total_nnz, b->c_nnz, s);
      launched += 1;
    }
  } else {
    if (b->wf == WF_ULTRASPARSE) {
      OCEAN_CUDA(cudaMemcpyAsync(w.est, w.prod, A.rows * 4, cudaMemcpyDeviceToDevice, s));
    } else {
      launched += launch_hll_sketch_sample(A, B, w, b->log2p, 0u, b->sketch, s);
      if (b->estimator == 2) {
        launched += launch_hll_rows(A, w, b->log2p, 1.0, sp.esc_max_products, true, b->sketch, w.est, s);
        MlpRowInputs in = row_inputs(w, B);
        in.row_problem = b->d_row_problem;
        in.problem_ctx = b->d_ctx;
        launched += launch_mlp_estimate(model_of(h), in, A.rows, sp.esc_max_products, w.est, nullptr,
                                        &w.ctr->status, h->num_sms, s);
      } else {
        launched += launch_hll_rows(A, w, b->log2p, b->expansion, sp.esc_max_products, false, b->sketch, w.est, s);
      }
    }
    launched += launch_scan(w, w.est, w.est_off, nullptr, &w.ctr->total_est, true, np, s);
    if (plan) {
      batch_readback(b, s);
      b->total_est = b->h_ctr->total_est;
      for (int i = 0; i < NB_COUNT; ++i) b->num_counts[i] = b->h_ctr->num_count[i];
      OCEAN_CUDA(cudaMalloc((void**)&b->t_col, std::max<uint64_t>(b->total_est, 1) * 4));
      OCEAN_CUDA(cudaMalloc((void**)&b->t_val, std::max<uint64_t>(b->total_est, 1) * 8));
    } else {
      launch_batch_guard(w.ctr, &w.ctr->total_est, b->total_est, s);
      launched += 1;
    }
    OCEAN_CUDA(cudaMemsetAsync(w.cnt, 0, A.rows * 4, s));
    const OutSpec est_out{w.est_off, w.est, w.cnt, w.ovf, &w.ctr->overflow_n};
    launched += launch_numeric(A, B, w, est_out, b->t_col, b->t_val, h->num_sms, s, nullptr, b->num_counts);
    launched += launch_overflow(A, B, w, false, nullptr, nullptr, h->num_sms, s);
    launched += launch_scan(w, w.cnt, w.rowptr64, w.rowptr32, &w.ctr->total_nnz, false, np, s);
    if (plan) {
      batch_readback(b, s);
      b->c_nnz = b->h_ctr->total_nnz;
    } else {
      launch_batch_guard(w.ctr, &w.ctr->total_nnz, b->c_nnz, s);
      launched += 1;
    }
  }
  if (plan) {
    b->out_bits = b->c_nnz >= (1ull << 32) ? 64 : 32;
    OCEAN_CUDA(cudaMalloc((void**)&b->c_col, std::max<uint64_t>(b->c_nnz, 1) * 4));
    OCEAN_CUDA(cudaMalloc((void**)&b->c_val, std::max<uint64_t>(b->c_nnz, 1) * 8));
    OCEAN_CUDA(cudaMalloc(&b->c_rp, (b->rows + n) * (b->out_bits / 8)));
  }
  if (b->wf == WF_PRECISE) {
    const OutSpec exact{w.rowptr64, w.row_nnz, nullptr, nullptr, nullptr};
    launched += launch_numeric(A, B, w, exact, b->c_col, b->c_val, h->num_sms, s, nullptr, b->num_counts);
  } else {
    launch_copy_rows(w, b->t_col, b->t_val, b->c_col, b->c_val, s, &w.ctr->status);
    launched += 1;
    launched += launch_overflow(A, B, w, true, b->c_col, b->c_val, h->num_sms, s);
  }
  // 3. one row-pointer array per problem
  if (b->out_bits == 64) launch_batch_rebase<uint64_t, uint64_t>(w.rowptr64, b->pref(0), b->pref(4), n, b->rows + n,
                                                                 (uint64_t*)b->c_rp, s);
  else launch_batch_rebase<uint64_t, uint32_t>(w.rowptr64, b->pref(0), b->pref(4), n, b->rows + n,
                                               (uint32_t*)b->c_rp, s);
  launch_batch_bounds<uint64_t>(w.rowptr64, b->pref(0), n, b->d_bounds, s);
  launched += 2;
  OCEAN_CUDA(cudaGetLastError());
  if (plan) {
    b->c_off.assign(n + 1, 0);
    OCEAN_CUDA(cudaMemcpyAsync(b->c_off.data(), b->d_bounds, (n + 1) * 8, cudaMemcpyDeviceToHost, s));
    batch_readback(b, s);
    b->launches = launched + (b->wf == WF_PRECISE ? 1 : 2);  // the capacity guards of a captured run
  }
}

void batch_run_pipeline(ocean_batch* b, cudaStream_t s, bool plan) {
  if (b->bits == 32) batch_pipeline<uint32_t>(b, s, plan);
  else batch_pipeline<uint64_t>(b, s, plan);
}

// Plans (eager run), then captures the pipeline into a graph.
void batch_plan_and_capture(ocean_batch* b, cudaStream_t s) {
  b->drop_graph();
  b->free_arenas();
  if (b->rows == 0) {  // every problem is empty: row pointers of zeros
    b->out_bits = 32;
    b->c_nnz = 0;
    b->c_off.assign(b->n + 1, 0);
    OCEAN_CUDA(cudaMalloc(&b->c_rp, b->n * 4ull));
    OCEAN_CUDA(cudaMemset(b->c_rp, 0, b->n * 4ull));
    return;
  }
  batch_run_pipeline(b, s, true);
  cudaStream_t cs;
  OCEAN_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    try {
      batch_run_pipeline(b, cs, false);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(cs, &g);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(cs);
      throw;
    }
    e = cudaStreamEndCapture(cs, &b->graph);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  cudaStreamDestroy(cs);
  OCEAN_CUDA(e);
}

// One graph launch; with check, waits and verifies the structure still matches.
void batch_launch(ocean_batch* b, cudaStream_t s, bool check) {
  if (!b->exec) return;
  OCEAN_CUDA(cudaGraphLaunch(b->exec, s));
  if (check) {
    b->h_bounds.resize(b->n + 1);
    OCEAN_CUDA(cudaMemcpyAsync(b->h_bounds.data(), b->d_bounds, (b->n + 1) * 8, cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(cudaMemcpyAsync(b->h_ctr, b->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(cudaStreamSynchronize(s));
    const unsigned st = b->h_ctr->status;
    OCEAN_CHECK(!(st & DEV_BATCH_MISMATCH) && b->h_bounds == b->c_off &&
                    (b->wf == WF_PRECISE || b->h_ctr->total_est == b->total_est),
                OCEAN_ERR_INVALID, "batch structure changed since the plan was made (re-plan it)");
    batch_readback(b, s);
  }
}

// Coordinate search over the class policy on the batch itself: each candidate
// is planned, captured and timed over `reps` graph launches (CUDA events);
// the fastest is kept.
// Key of a batch in the autotuning cache: the GPU's name and SM count, the
// batch's size and its rows and entries (log2 buckets of the totals and of the
// means per problem and per row), and the workflow options that change which
// kernels run.
std::string autotune_key(const ocean_batch* b) {
  cudaDeviceProp prop;
  std::string gpu = "unknown";
  if (cudaGetDeviceProperties(&prop, b->h->device) == cudaSuccess) gpu = prop.name;
  for (char& c : gpu)
    if (c == '"' || c == '\\' || c == '\t') c = ' ';
  auto lg = [](double x) { return x > 0 ? (int)std::floor(std::log2(x) * 2.0) : -1; };  // half-octave buckets
  const double rows = (double)b->rows, nnz = (double)b->nnz, n = (double)b->n;
  char buf[256];
  snprintf(buf, sizeof buf, "%s|sm%d|n%d|rows%d|nnz%d|rpp%d|npr%d|learned%d|wf%d", gpu.c_str(), b->h->num_sms, lg(n),
           lg(rows), lg(nnz), lg(rows / n), lg(rows > 0 ? nnz / rows : 0.0), b->cfg.use_learned_estimator ? 1 : 0,
           b->cfg.force_workflow);
  return buf;
}

// Tuned knobs of a batch as one flat JSON object (a line of the cache file).
std::string autotune_line(const std::string& key, const Config& c, double ms) {
  std::ostringstream o;
  o.precision(17);
  o << "{\"key\": \"" << key << "\", \"esc_max_products\": " << c.esc_max_products
    << ", \"hash_s_max_scale\": " << c.hash_s_max_scale << ", \"bitmap_words_scale\": " << c.bitmap_words_scale
    << ", \"prefer_direct_hash\": " << (c.prefer_direct_hash ? "true" : "false")
    << ", \"numeric_windows\": " << (c.numeric_windows ? "true" : "false") << ", \"tuned_ms\": " << ms << "}";
  return o.str();
}

// Looks the key up in the cache file; on a hit the knobs go into c.
bool autotune_lookup(const std::string& path, const std::string& key, Config* c, double* ms) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  bool hit = false;
  while (std::getline(f, line)) {
    if (line.empty()) continue;
    std::map<std::string, JsonScalar> m;
    try {
      m = FlatJson::parse(line);
    } catch (const std::exception&) {
      continue;  // a damaged line is skipped
    }
    auto it = m.find("key");
    if (it == m.end() || it->second.kind != JsonScalar::kString || it->second.str != key) continue;
    auto num = [&](const char* k, double d) {
      auto j = m.find(k);
      return j != m.end() && j->second.kind == JsonScalar::kNumber ? j->second.num : d;
    };
    auto flag = [&](const char* k, bool d) {
      auto j = m.find(k);
      return j != m.end() && j->second.kind == JsonScalar::kBool ? j->second.b : d;
    };
    c->esc_max_products = (int)num("esc_max_products", c->esc_max_products);
    c->hash_s_max_scale = num("hash_s_max_scale", c->hash_s_max_scale);
    c->bitmap_words_scale = num("bitmap_words_scale", c->bitmap_words_scale);
    c->prefer_direct_hash = flag("prefer_direct_hash", c->prefer_direct_hash);
    c->numeric_windows = flag("numeric_windows", c->numeric_windows);
    *ms = num("tuned_ms", 0.0);
    hit = true;  // the last matching line wins
  }
  return hit;
}

// Coordinate search of the class policy on the batch itself: each knob in
// turn takes every listed value while the others keep their best, each
// candidate planned, captured and timed over `reps` graph launches; the
// fastest is kept and captured. With autotune_cache_file, a batch whose key
// is in the cache takes the cached knobs without searching, and a search
// appends its result.
void batch_autotune(ocean_batch* b, cudaStream_t s, int reps) {
  const std::string cache = b->cfg.autotune_cache_file;
  const std::string key = autotune_key(b);
  b->tune_key = key;
  double cached_ms = 0.0;
  if (!cache.empty() && autotune_lookup(cache, key, &b->cfg, &cached_ms)) {
    batch_plan_and_capture(b, s);
    b->tuned_ms = cached_ms;
    b->tune_cached = true;
  } else {
    struct Knob {
      const char* name;
      std::vector<double> values;
    };
    std::vector<Knob> knobs = {{"esc_max_products", {128, 64, 32}},
                               {"hash_s_max_scale", {1.0, 0.75, 0.5}},
                               {"bitmap_words_scale", {1.0, 0.5, 2.0, 4.0}},
                               {"prefer_direct_hash", {1, 0}},
                               {"numeric_windows", {0, 1}}};
    cudaEvent_t e0, e1;
    OCEAN_CUDA(cudaEventCreate(&e0));
    OCEAN_CUDA(cudaEventCreate(&e1));
    auto set = [&](const char* k, double v) {
      if (!strcmp(k, "esc_max_products")) b->cfg.esc_max_products = (int)v;
      else if (!strcmp(k, "hash_s_max_scale")) b->cfg.hash_s_max_scale = v;
      else if (!strcmp(k, "bitmap_words_scale")) b->cfg.bitmap_words_scale = v;
      else if (!strcmp(k, "prefer_direct_hash")) b->cfg.prefer_direct_hash = v != 0.0;
      else b->cfg.numeric_windows = v != 0.0;
    };
    auto get = [&](const char* k) -> double {
      if (!strcmp(k, "esc_max_products")) return b->cfg.esc_max_products;
      if (!strcmp(k, "hash_s_max_scale")) return b->cfg.hash_s_max_scale;
      if (!strcmp(k, "bitmap_words_scale")) return b->cfg.bitmap_words_scale;
      if (!strcmp(k, "prefer_direct_hash")) return b->cfg.prefer_direct_hash ? 1.0 : 0.0;
      return b->cfg.numeric_windows ? 1.0 : 0.0;
    };
    auto measure = [&]() -> double {
      batch_plan_and_capture(b, s);
      batch_launch(b, s, true);  // warm-up and structure check
      OCEAN_CUDA(cudaEventRecord(e0, s));
      for (int i = 0; i < reps; ++i) OCEAN_CUDA(cudaGraphLaunch(b->exec, s));
      OCEAN_CUDA(cudaEventRecord(e1, s));
      OCEAN_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      OCEAN_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      return ms / reps;
    };
    double best = measure();
    for (const Knob& k : knobs) {
      double keep = get(k.name);
      for (double v : k.values) {
        if (v == keep) continue;
        set(k.name, v);
        const double t = measure();
        if (t < best) best = t, keep = v;
      }
      set(k.name, keep);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    batch_plan_and_capture(b, s);
    b->tuned_ms = best;
    if (!cache.empty()) {
      std::ofstream f(cache, std::ios::app);
      if (f) f << autotune_line(key, b->cfg, best) << "\n";
    }
  }
  char buf[200];
  snprintf(buf, sizeof buf, "esc_max_products=%d hash_s_max_scale=%g bitmap_words_scale=%g prefer_direct_hash=%d "
           "numeric_windows=%d%s", b->cfg.esc_max_products, b->cfg.hash_s_max_scale, b->cfg.bitmap_words_scale,
           b->cfg.prefer_direct_hash ? 1 : 0, b->cfg.numeric_windows ? 1 : 0, b->tune_cached ? " (cached)" : "");
  b->tuning = buf;
}

// Stacks the problems' geometry and copies the problem table to the device.
void batch_setup(ocean_batch* b, uint64_t n, const ocean_csr_view* A, const ocean_csr_view* B) {
  OCEAN_CHECK(n > 0 && n < 0xFFFFFFFFull, OCEAN_ERR_INVALID, "batch size must be in [1, 2^32)");
  OCEAN_CHECK(A != nullptr, OCEAN_ERR_INVALID, "A is NULL");
  b->n = (uint32_t)n;
  b->same_b = true;
  for (uint64_t p = 0; p < n; ++p) {
    validate_view(&A[p], "A[p]");
    if (B) {
      validate_view(&B[p], "B[p]");
      OCEAN_CHECK(A[p].cols == B[p].rows, OCEAN_ERR_INVALID, "Incompatible matrix dimensions (A[p].cols != B[p].rows)");
      if (memcmp(&A[p], &B[p], sizeof(ocean_csr_view)) != 0) b->same_b = false;
    } else {
      OCEAN_CHECK(A[p].cols == A[p].rows, OCEAN_ERR_INVALID, "B = NULL needs square A[p] (C = A[p] * A[p])");
    }
  }
  b->row0.assign(n + 1, 0), b->nnz0.assign(n + 1, 0), b->brow0.assign(n + 1, 0), b->bnnz0.assign(n + 1, 0);
  b->a_rows.resize(n), b->b_cols.resize(n);
  std::vector<BatchProblem> probs(n);
  for (uint64_t p = 0; p < n; ++p) {
    const ocean_csr_view& a = A[p];
    const ocean_csr_view& bb = B ? B[p] : A[p];
    b->row0[p + 1] = b->row0[p] + a.rows;
    b->nnz0[p + 1] = b->nnz0[p] + a.nnz;
    b->brow0[p + 1] = b->brow0[p] + bb.rows;
    b->bnnz0[p + 1] = b->bnnz0[p] + bb.nnz;
    b->a_rows[p] = a.rows;
    b->b_cols[p] = bb.cols;
    b->bcols = std::max<uint64_t>(b->bcols, bb.cols);
    BatchProblem& q = probs[p];
    q.a_rp = a.rowptr, q.a_col = a.col, q.a_val = a.val, q.a_bits = (uint32_t)a.rowptr_bits;
    q.b_rp = bb.rowptr, q.b_col = bb.col, q.b_val = bb.val, q.b_bits = (uint32_t)bb.rowptr_bits;
    q.nnz0 = b->nnz0[p], q.brow0 = b->brow0[p], q.bnnz0 = b->bnnz0[p];
  }
  b->rows = b->row0[n], b->nnz = b->nnz0[n], b->brows = b->brow0[n], b->bnnz = b->bnnz0[n];
  OCEAN_CHECK(b->rows < 0xFFFFFFFFull && b->brows < 0xFFFFFFFFull, OCEAN_ERR_INVALID,
              "the stacked batch has 2^32 - 1 or more rows");
  b->bits = (b->nnz >= (1ull << 32) || b->bnnz >= (1ull << 32)) ? 64 : 32;
  const int rb = b->bits / 8;
  OCEAN_CUDA(cudaMalloc((void**)&b->d_probs, n * sizeof(BatchProblem)));
  OCEAN_CUDA(cudaMemcpy(b->d_probs, probs.data(), n * sizeof(BatchProblem), cudaMemcpyHostToDevice));
  std::vector<uint64_t> pref(5 * (n + 1));
  for (uint64_t p = 0; p <= n; ++p) {
    pref[p] = b->row0[p];
    pref[(n + 1) + p] = b->nnz0[p];
    pref[2 * (n + 1) + p] = b->brow0[p];
    pref[3 * (n + 1) + p] = b->bnnz0[p];
    pref[4 * (n + 1) + p] = b->row0[p] + p;
  }
  OCEAN_CUDA(cudaMalloc((void**)&b->d_pref, pref.size() * 8));
  OCEAN_CUDA(cudaMemcpy(b->d_pref, pref.data(), pref.size() * 8, cudaMemcpyHostToDevice));
  OCEAN_CUDA(cudaMalloc(&b->a_rp, (b->rows + 1) * rb));
  OCEAN_CUDA(cudaMalloc((void**)&b->a_col, std::max<uint64_t>(b->nnz, 1) * 4));
  OCEAN_CUDA(cudaMalloc((void**)&b->a_val, std::max<uint64_t>(b->nnz, 1) * 8));
  if (b->same_b) {
    b->b_rp = b->a_rp;
    b->b_val = b->a_val;
    OCEAN_CUDA(cudaMalloc((void**)&b->b_col, std::max<uint64_t>(b->nnz, 1) * 4));
  } else {
    OCEAN_CUDA(cudaMalloc(&b->b_rp, (b->brows + 1) * rb));
    OCEAN_CUDA(cudaMalloc((void**)&b->b_col, std::max<uint64_t>(b->bnnz, 1) * 4));
    OCEAN_CUDA(cudaMalloc((void**)&b->b_val, std::max<uint64_t>(b->bnnz, 1) * 8));
  }
  {
    // per-row problem ids and per-problem B scalars (the learned estimator's context features)
    std::vector<uint32_t> rp(std::max<uint64_t>(b->rows, 1));
    std::vector<float2> ctx(n);
    for (uint64_t p = 0; p < n; ++p) {
      for (uint64_t r = b->row0[p]; r < b->row0[p + 1]; ++r) rp[r] = (uint32_t)p;
      const ocean_csr_view& bb = B ? B[p] : A[p];
      ctx[p].x = log2f(1.f + (float)bb.cols);
      ctx[p].y = log2f(1.f + (bb.rows ? (float)((double)bb.nnz / (double)bb.rows) : 0.f));
    }
    OCEAN_CUDA(cudaMalloc((void**)&b->d_row_problem, rp.size() * 4));
    OCEAN_CUDA(cudaMemcpy(b->d_row_problem, rp.data(), rp.size() * 4, cudaMemcpyHostToDevice));
    OCEAN_CUDA(cudaMalloc((void**)&b->d_ctx, n * sizeof(float2)));
    OCEAN_CUDA(cudaMemcpy(b->d_ctx, ctx.data(), n * sizeof(float2), cudaMemcpyHostToDevice));
  }
  OCEAN_CUDA(cudaMalloc((void**)&b->w.ctr, sizeof(DevCounters)));
  OCEAN_CUDA(cudaMalloc((void**)&b->d_bounds, (n + 1) * 8));
  OCEAN_CUDA(cudaHostAlloc((void**)&b->h_ctr, sizeof(DevCounters), cudaHostAllocDefault));
  alloc_work_rows(b->w, b->rows);
  ensure_long_rows(b->w, b->nnz, b->rows);
  ensure_btab(b->w, b->brows);
}

// The n results as views into the plan's arena (location 2: lent by the plan).
void batch_outputs(const ocean_batch* b, ocean_csr* C) {
  for (uint32_t p = 0; p < b->n; ++p) {
    ocean_csr& c = C[p];
    std::memset(&c, 0, sizeof c);
    c.rows = b->a_rows[p];
    c.cols = b->b_cols[p];
    c.rowptr_bits = b->out_bits;
    c.location = 2;
    c.rowptr = (char*)b->c_rp + (b->row0[p] + p) * (uint64_t)(b->out_bits / 8);
    c.nnz = b->c_off[p + 1] - b->c_off[p];
    if (c.nnz) {
      c.col = b->c_col + b->c_off[p];
      c.val = b->c_val + b->c_off[p];
    }
  }
}

}  // namespace

namespace {
// Queues the copies of a batch's results into host buffers on s.
void batch_download(ocean_batch* b, void* rowptrs, uint32_t* col, double* val, cudaStream_t s) {
  OCEAN_CHECK(b != nullptr && rowptrs != nullptr, OCEAN_ERR_INVALID, "batch or rowptrs is NULL");
  OCEAN_CHECK(b->c_nnz == 0 || (col && val), OCEAN_ERR_INVALID, "col or val is NULL");
  OCEAN_CUDA(cudaMemcpyAsync(rowptrs, b->c_rp, (b->rows + b->n) * (uint64_t)(b->out_bits / 8),
                             cudaMemcpyDeviceToHost, s));
  if (b->c_nnz) {
    OCEAN_CUDA(cudaMemcpyAsync(col, b->c_col, b->c_nnz * 4, cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(cudaMemcpyAsync(val, b->c_val, b->c_nnz * 8, cudaMemcpyDeviceToHost, s));
  }
}
}  // namespace

extern "C" {

int ocean_create(ocean_handle** out, const char* json_config) {
  return guarded([&] {
    OCEAN_CHECK(out != nullptr, OCEAN_ERR_INVALID, "out is NULL");
    *out = nullptr;
    ocean_handle* h = new ocean_handle();
    try {
      init_handle(h, json_config ? std::string(json_config) : std::string());
    } catch (...) {
      h->free_all();
      delete h;
      throw;
    }
    *out = h;
  });
}

int ocean_create_from_file(ocean_handle** out, const char* json_path) {
  return guarded([&] {
    OCEAN_CHECK(json_path != nullptr, OCEAN_ERR_INVALID, "json_path is NULL");
    std::ifstream f(json_path);
    OCEAN_CHECK(f.good(), OCEAN_ERR_INVALID, std::string("cannot open config file ") + json_path);
    std::stringstream ss;
    ss << f.rdbuf();
    const std::string text = ss.str();
    const int rc = ocean_create(out, text.c_str());
    if (rc != OCEAN_OK) throw OceanError{rc, g_last_error};
  });
}

void ocean_destroy(ocean_handle* h) {
  if (!h) return;
  h->free_all();
  delete h;
}

int ocean_spgemm(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, ocean_csr* C, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    dispatch_spgemm(h, A, B, C, (cudaStream_t)stream);
  });
}

int ocean_spgemm_host(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, ocean_csr* C,
                      void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    validate_view(A, "A");
    validate_view(B, "B");
    OCEAN_CHECK(C != nullptr, OCEAN_ERR_INVALID, "C is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    ocean_csr_view dv[2];
    const ocean_csr_view* src[2] = {A, B};
    const bool same = A->rowptr == B->rowptr && A->col == B->col && A->val == B->val && A->rows == B->rows &&
                      A->nnz == B->nnz && A->rowptr_bits == B->rowptr_bits;
    for (int m = 0; m < (same ? 1 : 2); ++m) {
      const ocean_csr_view* v = src[m];
      const uint64_t rpb = (v->rows + 1) * (uint64_t)(v->rowptr_bits / 8);
      grow(h->in_rp[m], h->in_rp_cap[m], rpb);
      grow(h->in_col[m], h->in_col_cap[m], v->nnz);
      grow(h->in_val[m], h->in_val_cap[m], v->nnz);
      if (v->rows) OCEAN_CUDA(cudaMemcpyAsync(h->in_rp[m], v->rowptr, rpb, cudaMemcpyHostToDevice, s));
      if (v->nnz) {
        OCEAN_CUDA(cudaMemcpyAsync(h->in_col[m], v->col, v->nnz * 4, cudaMemcpyHostToDevice, s));
        OCEAN_CUDA(cudaMemcpyAsync(h->in_val[m], v->val, v->nnz * 8, cudaMemcpyHostToDevice, s));
      }
      dv[m] = *v;
      dv[m].rowptr = h->in_rp[m];
      dv[m].col = h->in_col[m];
      dv[m].val = h->in_val[m];
    }
    if (same) dv[1] = dv[0];
    ocean_csr dc;
    const auto t_in = std::chrono::steady_clock::now();
    // large precise multiplies copy C to the pinned host buffers chunk by
    // chunk from inside the numeric phase (pipeline_numeric)
    h->sink_active = true;
    h->sink_filled = false;
    try {
      dispatch_spgemm(h, &dv[0], &dv[1], &dc, s);
    } catch (...) {
      h->sink_active = false;
      throw;
    }
    h->sink_active = false;
    const uint64_t rpb = (dc.rows + 1) * (uint64_t)(dc.rowptr_bits / 8);
    CResult* dev_owner = (CResult*)dc._owner;
    try {
      if (!h->sink_filled) {
        grow_host(h->out_rp, h->out_rp_cap, rpb);
        grow_host(h->out_col, h->out_col_cap, dc.nnz);
        grow_host(h->out_val, h->out_val_cap, dc.nnz);
        OCEAN_CUDA(cudaMemcpyAsync(h->out_rp, dc.rowptr, rpb, cudaMemcpyDeviceToHost, s));
        if (dc.nnz) {
          OCEAN_CUDA(cudaMemcpyAsync(h->out_col, dc.col, dc.nnz * 4, cudaMemcpyDeviceToHost, s));
          OCEAN_CUDA(cudaMemcpyAsync(h->out_val, dc.val, dc.nnz * 8, cudaMemcpyDeviceToHost, s));
        }
      }
    } catch (...) {
      cudaFreeAsync(dev_owner->rowptr, s);
      cudaFreeAsync(dev_owner->col, s);
      cudaFreeAsync(dev_owner->val, s);
      delete dev_owner;
      throw;
    }
    OCEAN_CUDA(cudaFreeAsync(dev_owner->rowptr, s));
    OCEAN_CUDA(cudaFreeAsync(dev_owner->col, s));
    OCEAN_CUDA(cudaFreeAsync(dev_owner->val, s));
    delete dev_owner;
    OCEAN_CUDA(cudaStreamSynchronize(s));
    // the copy-back on the multiply's host timeline (which starts at t_in)
    h->st.host_marks.emplace_back(
        "host_output_copied", std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_in).count());
    *C = dc;
    C->rowptr = h->out_rp;
    C->col = h->out_col;
    C->val = h->out_val;
    C->location = 1;
    C->_owner = &h->host_owner;
  });
}

int ocean_csr_free(ocean_csr* C, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(C != nullptr, OCEAN_ERR_INVALID, "C is NULL");
    CResult* o = (CResult*)C->_owner;
    if (o && o->location == 0 && --o->refs == 0) {
      cudaStream_t s = (cudaStream_t)stream;
      for (void* p : {o->rowptr, (void*)o->col, (void*)o->val}) {
        if (!p) continue;
        if (o->plain_alloc) OCEAN_CUDA(cudaFree(p));
        else OCEAN_CUDA(cudaFreeAsync(p, s));
      }
      delete o;
    }
    std::memset(C, 0, sizeof(*C));
  });
}

int ocean_csr_download(const ocean_csr* C, void* rowptr, uint32_t* col, double* val, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(C != nullptr, OCEAN_ERR_INVALID, "C is NULL");
    OCEAN_CHECK(rowptr != nullptr && (C->nnz == 0 || (col && val)), OCEAN_ERR_INVALID, "output buffer is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    const cudaMemcpyKind kind = C->location == 1 ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost;
    OCEAN_CUDA(cudaMemcpyAsync(rowptr, C->rowptr, (C->rows + 1) * (uint64_t)(C->rowptr_bits / 8), kind, s));
    if (C->nnz) {
      OCEAN_CUDA(cudaMemcpyAsync(col, C->col, C->nnz * 4, kind, s));
      OCEAN_CUDA(cudaMemcpyAsync(val, C->val, C->nnz * 8, kind, s));
    }
    OCEAN_CUDA(cudaStreamSynchronize(s));
  });
}

int ocean_csr_download_rows(const ocean_csr* C, uint64_t r0, uint64_t r1, uint64_t* rowptr, uint32_t* col,
                            double* val, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(C != nullptr && rowptr != nullptr, OCEAN_ERR_INVALID, "NULL argument");
    OCEAN_CHECK(r0 <= r1 && r1 <= C->rows, OCEAN_ERR_INVALID, "row range outside C");
    cudaStream_t s = (cudaStream_t)stream;
    const cudaMemcpyKind kind = C->location == 1 ? cudaMemcpyHostToHost : cudaMemcpyDeviceToHost;
    const uint64_t n = r1 - r0 + 1;
    if (C->rowptr_bits == 64) {
      OCEAN_CUDA(cudaMemcpyAsync(rowptr, (const uint64_t*)C->rowptr + r0, n * 8, kind, s));
      OCEAN_CUDA(cudaStreamSynchronize(s));
    } else {
      std::vector<uint32_t> tmp(n);
      OCEAN_CUDA(cudaMemcpyAsync(tmp.data(), (const uint32_t*)C->rowptr + r0, n * 4, kind, s));
      OCEAN_CUDA(cudaStreamSynchronize(s));
      for (uint64_t i = 0; i < n; ++i) rowptr[i] = tmp[i];
    }
    if (r1 == C->rows) rowptr[n - 1] = C->nnz;
    const uint64_t b = rowptr[0], e = rowptr[n - 1];
    OCEAN_CHECK(b <= e && e <= C->nnz, OCEAN_ERR_INTERNAL, "row pointers out of range");
    if (e > b && col != nullptr && val != nullptr) {
      OCEAN_CUDA(cudaMemcpyAsync(col, C->col + b, (e - b) * 4, kind, s));
      OCEAN_CUDA(cudaMemcpyAsync(val, C->val + b, (e - b) * 8, kind, s));
    }
    OCEAN_CUDA(cudaStreamSynchronize(s));
  });
}

int ocean_symbolic(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, uint32_t* row_nnz,
                   void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    validate_view(A, "A");
    validate_view(B, "B");
    OCEAN_CHECK(A->cols == B->rows, OCEAN_ERR_INVALID, "Incompatible matrix dimensions (A.cols != B.rows)");
    OCEAN_CHECK(A->rows == 0 || row_nnz != nullptr, OCEAN_ERR_INVALID, "row_nnz is NULL");
    OCEAN_CHECK(A->rowptr_bits == B->rowptr_bits, OCEAN_ERR_INVALID,
                "ocean_symbolic needs equal row-pointer widths for A and B");
    if (A->rows == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    if (A->rowptr_bits == 32) {
      run_front(h, to_csr<uint32_t>(A, (const uint32_t*)A->rowptr), to_csr<uint32_t>(B, (const uint32_t*)B->rowptr),
                s, false, false);
    } else {
      run_front(h, to_csr<uint64_t>(A, (const uint64_t*)A->rowptr), to_csr<uint64_t>(B, (const uint64_t*)B->rowptr),
                s, false, false);
    }
    OCEAN_CUDA(cudaMemcpyAsync(row_nnz, h->w.row_nnz, A->rows * 4, cudaMemcpyDeviceToDevice, s));
    OCEAN_CUDA(cudaStreamSynchronize(s));
  });
}

int ocean_row_estimates(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, int log2p,
                        uint32_t* est, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    validate_view(A, "A");
    validate_view(B, "B");
    OCEAN_CHECK(A->cols == B->rows, OCEAN_ERR_INVALID, "Incompatible matrix dimensions (A.cols != B.rows)");
    OCEAN_CHECK(A->rowptr_bits == B->rowptr_bits, OCEAN_ERR_INVALID,
                "ocean_row_estimates needs equal row-pointer widths for A and B");
    OCEAN_CHECK(log2p == 5 || log2p == 6, OCEAN_ERR_INVALID, "log2p must be 5 or 6");
    OCEAN_CHECK(A->rows == 0 || est != nullptr, OCEAN_ERR_INVALID, "est is NULL");
    if (A->rows == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    auto go = [&](auto rp_tag) {
      using RP = decltype(rp_tag);
      const Csr<RP> a = to_csr<RP>(A, (const RP*)A->rowptr), b = to_csr<RP>(B, (const RP*)B->rowptr);
      run_analysis(h, a, b, s);
      void* sk = nullptr;
      OCEAN_CUDA(cudaMallocAsync(&sk, std::max<uint64_t>(B->rows, 1) << log2p, s));
      launch_hll_sketch_sample(a, b, h->w, log2p, 0u, (uint8_t*)sk, s);
      launch_hll_rows(a, h->w, log2p, 1.0, 0u, true, (const uint8_t*)sk, est, s);
      const cudaError_t e = cudaGetLastError();
      cudaFreeAsync(sk, s);
      OCEAN_CUDA(e);
      OCEAN_CUDA(cudaStreamSynchronize(s));
    };
    if (A->rowptr_bits == 32) go(uint32_t{});
    else go(uint64_t{});
  });
}

int ocean_mlp_features(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, float* feat,
                       void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    validate_view(A, "A");
    validate_view(B, "B");
    OCEAN_CHECK(A->cols == B->rows, OCEAN_ERR_INVALID, "Incompatible matrix dimensions (A.cols != B.rows)");
    OCEAN_CHECK(A->rowptr_bits == B->rowptr_bits, OCEAN_ERR_INVALID,
                "ocean_mlp_features needs equal row-pointer widths for A and B");
    OCEAN_CHECK(A->rows == 0 || feat != nullptr, OCEAN_ERR_INVALID, "feat is NULL");
    if (A->rows == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    auto go = [&](auto rp_tag) {
      using RP = decltype(rp_tag);
      const Csr<RP> a = to_csr<RP>(A, (const RP*)A->rowptr), b = to_csr<RP>(B, (const RP*)B->rowptr);
      run_analysis(h, a, b, s);
      void* sk = nullptr;
      OCEAN_CUDA(cudaMallocAsync(&sk, std::max<uint64_t>(B->rows, 1) << kLearnedLog2p, s));
      launch_hll_sketch_sample(a, b, h->w, kLearnedLog2p, 0u, (uint8_t*)sk, s);
      launch_hll_rows(a, h->w, kLearnedLog2p, 1.0, 0u, true, (const uint8_t*)sk, h->w.est, s);
      launch_mlp_features(row_inputs(h->w, b), a.rows, feat, s);
      const cudaError_t e = cudaGetLastError();
      cudaFreeAsync(sk, s);
      OCEAN_CUDA(e);
      OCEAN_CUDA(cudaStreamSynchronize(s));
    };
    if (A->rowptr_bits == 32) go(uint32_t{});
    else go(uint64_t{});
  });
}


int ocean_mlp_forward(ocean_handle* h, const ocean_mlp_model* m, const float* feat, uint64_t n, float* pred,
                      void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    const MlpModel mm = model_from(m);
    OCEAN_CHECK(n == 0 || (feat && pred), OCEAN_ERR_INVALID, "feat or pred is NULL");
    OCEAN_CHECK(((uintptr_t)feat & 15) == 0, OCEAN_ERR_INVALID, "feat must be 16-byte aligned");
    if (n == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    with_status(h, s, [&](unsigned* st) { launch_mlp_forward(mm, feat, n, pred, st, h->num_sms, s); });
  });
}

int ocean_mlp_grad(ocean_handle* h, const ocean_mlp_model* m, const float* feat, const float* target, uint64_t n,
                   float batch, float* grad, float* loss, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    const MlpModel mm = model_from(m);
    OCEAN_CHECK(n == 0 || (feat && target && grad && loss), OCEAN_ERR_INVALID, "an array pointer is NULL");
    OCEAN_CHECK(((uintptr_t)feat & 15) == 0, OCEAN_ERR_INVALID, "feat must be 16-byte aligned");
    OCEAN_CHECK(batch > 0.f, OCEAN_ERR_INVALID, "batch must be positive");
    if (n == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    with_status(h, s,
                [&](unsigned* st) { launch_mlp_grad(mm, feat, target, n, batch, grad, loss, st, h->num_sms, s); });
  });
}

int ocean_mlp_adam(ocean_handle* h, float* params, float* m1, float* m2, float* grad, int step, float lr,
                   float beta1, float beta2, float eps, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    OCEAN_CHECK(params && m1 && m2 && grad, OCEAN_ERR_INVALID, "an array pointer is NULL");
    OCEAN_CHECK(step >= 1, OCEAN_ERR_INVALID, "step must be >= 1");
    launch_mlp_adam(params, m1, m2, grad, step, lr, beta1, beta2, eps, (cudaStream_t)stream);
    OCEAN_CUDA(cudaGetLastError());
  });
}

int ocean_mlp_builtin(float* blob, size_t n) {
  return guarded([&] {
    OCEAN_CHECK(kMlpBuiltinTrained != 0, OCEAN_ERR_INVALID, "no trained estimator is built in");
    OCEAN_CHECK(blob != nullptr && n >= (size_t)kMlpBlob, OCEAN_ERR_INVALID, "blob too small");
    std::memcpy(blob, kMlpBuiltin, kMlpBlob * sizeof(float));
  });
}

int ocean_estimate(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, int estimator,
                   int with_margin, uint32_t* est, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    validate_view(A, "A");
    validate_view(B, "B");
    OCEAN_CHECK(A->cols == B->rows, OCEAN_ERR_INVALID, "Incompatible matrix dimensions (A.cols != B.rows)");
    OCEAN_CHECK(A->rowptr_bits == B->rowptr_bits, OCEAN_ERR_INVALID,
                "ocean_estimate needs equal row-pointer widths for A and B");
    OCEAN_CHECK(estimator == 1 || estimator == 2, OCEAN_ERR_INVALID, "estimator must be 1 (HLL) or 2 (learned)");
    OCEAN_CHECK(A->rows == 0 || est != nullptr, OCEAN_ERR_INVALID, "est is NULL");
    if (A->rows == 0) return;
    cudaStream_t s = (cudaStream_t)stream;
    const Config& c = h->cfg;
    auto go = [&](auto rp_tag) {
      using RP = decltype(rp_tag);
      const Csr<RP> a = to_csr<RP>(A, (const RP*)A->rowptr), b = to_csr<RP>(B, (const RP*)B->rowptr);
      run_analysis(h, a, b, s);
      OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
      OCEAN_CUDA(cudaStreamSynchronize(s));
      const uint64_t ratio = a.nnz ? h->h_ctr->total_products / a.nnz : 0;
      const bool learned = estimator == 2;
      if (learned) load_model(h);
      const int log2p = learned ? kLearnedLog2p
                                : (ratio >= (uint64_t)c.hll_higher_precision_expansion_threshold ? 6 : 5);
      void* sk = nullptr;
      OCEAN_CUDA(cudaMallocAsync(&sk, std::max<uint64_t>(B->rows, 1) << log2p, s));
      launch_hll_sketch_sample(a, b, h->w, log2p, 0u, (uint8_t*)sk, s);
      if (learned) {
        launch_hll_rows(a, h->w, log2p, 1.0, (uint32_t)c.esc_max_products, true, (const uint8_t*)sk, h->w.est, s);
        MlpModel m = model_of(h);
        if (!with_margin) m.margin = 0.f;
        launch_mlp_estimate(m, row_inputs(h->w, b), a.rows, (uint32_t)c.esc_max_products, est, nullptr,
                            &h->w.ctr->status, h->num_sms, s);
      } else {
        const double expansion = with_margin ? (log2p == 5 ? 2.0 : 1.5) * c.estimate_scale : 1.0;
        launch_hll_rows(a, h->w, log2p, expansion, (uint32_t)c.esc_max_products, false, (const uint8_t*)sk, est, s);
      }
      const cudaError_t e = cudaGetLastError();
      cudaFreeAsync(sk, s);
      OCEAN_CUDA(e);
      OCEAN_CUDA(cudaMemcpyAsync(h->h_ctr, h->w.ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost, s));
      OCEAN_CUDA(cudaStreamSynchronize(s));
      check_device_status(h);
    };
    if (A->rowptr_bits == 32) go(uint32_t{});
    else go(uint64_t{});
  });
}

int ocean_estimate_metrics(ocean_handle* h, const uint32_t* est, const uint32_t* truth, uint32_t min_products,
                           double* out, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    OCEAN_CHECK(out != nullptr, OCEAN_ERR_INVALID, "out is NULL");
    const uint64_t n = h->w.rows;
    OCEAN_CHECK(n == 0 || (est && truth), OCEAN_ERR_INVALID, "est or truth is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    if (!h->metrics_dev) OCEAN_CUDA(cudaMalloc((void**)&h->metrics_dev, 8 * sizeof(double)));
    OCEAN_CUDA(cudaMemsetAsync(h->metrics_dev, 0, 4 * sizeof(double), s));
    SymPolicy sp;
    NumPolicy np;
    make_policies(h->cfg, &sp, &np);
    MlpRowInputs in;
    in.prod = h->w.prod;
    in.lo = h->w.lo;
    in.hi = h->w.hi;
    launch_est_metrics(est, truth, in, n, np, min_products, h->metrics_dev, s);
    double m[4];
    OCEAN_CUDA(cudaMemcpyAsync(m, h->metrics_dev, sizeof m, cudaMemcpyDeviceToHost, s));
    OCEAN_CUDA(cudaStreamSynchronize(s));
    out[0] = m[1] > 0 ? m[0] / m[1] : 0.0;
    out[1] = m[1] > 0 ? 100.0 * m[2] / m[1] : 0.0;
    out[2] = m[1];
    out[3] = m[3];
  });
}

int ocean_batch_create(ocean_handle* h, uint64_t n, const ocean_csr_view* A, const ocean_csr_view* B,
                       ocean_batch** out, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr && out != nullptr, OCEAN_ERR_INVALID, "handle or out is NULL");
    *out = nullptr;
    std::unique_ptr<ocean_batch> b(new ocean_batch());
    b->h = h;
    b->cfg = h->cfg;
    batch_setup(b.get(), n, A, B);
    cudaStream_t s = (cudaStream_t)stream;
    if (b->cfg.batch_autotune && b->rows) batch_autotune(b.get(), s, 5);
    else batch_plan_and_capture(b.get(), s);
    *out = b.release();
  });
}

int ocean_batch_launch(ocean_batch* b, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(b != nullptr, OCEAN_ERR_INVALID, "batch is NULL");
    batch_launch(b, (cudaStream_t)stream, false);
  });
}

int ocean_batch_run(ocean_batch* b, ocean_csr* C, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(b != nullptr && C != nullptr, OCEAN_ERR_INVALID, "batch or C is NULL");
    batch_launch(b, (cudaStream_t)stream, true);
    batch_outputs(b, C);
  });
}

int ocean_batch_results(ocean_batch* b, ocean_csr* C) {
  return guarded([&] {
    OCEAN_CHECK(b != nullptr && C != nullptr, OCEAN_ERR_INVALID, "batch or C is NULL");
    batch_outputs(b, C);
  });
}

int ocean_batch_info_json(ocean_batch* b, char* buf, size_t cap, size_t* needed) {
  return guarded([&] {
    OCEAN_CHECK(b != nullptr, OCEAN_ERR_INVALID, "batch is NULL");
    std::ostringstream o;
    o.precision(17);
    o << "{\"problems\": " << b->n << ", \"rows\": " << b->rows << ", \"nnz_a\": " << b->nnz
      << ", \"nnz_b\": " << b->bnnz << ", \"nnz_c\": " << b->c_nnz << ", \"products\": " << b->products
      << ", \"rowptr_bits\": " << b->out_bits
      << ", \"workflow\": " << b->wf
      << ", \"estimator\": \"" << (b->estimator == 2 ? "learned" : b->estimator == 1 ? "hll" : "none")
      << "\", \"total_est\": " << b->total_est << ", \"kernel_launches\": " << b->launches
      << ", \"graph\": " << (b->exec ? "true" : "false") << ", \"tuned_ms\": " << b->tuned_ms
      << ", \"tune_cached\": " << (b->tune_cached ? "true" : "false") << ", \"tune_key\": \"" << b->tune_key << "\""
      << ", \"prefer_direct_hash\": " << (b->cfg.prefer_direct_hash ? "true" : "false")
      << ", \"numeric_windows\": " << (b->cfg.numeric_windows ? "true" : "false")
      << ", \"esc_max_products\": " << b->cfg.esc_max_products << ", \"hash_s_max_scale\": "
      << b->cfg.hash_s_max_scale << ", \"bitmap_words_scale\": " << b->cfg.bitmap_words_scale
      << ", \"tuning\": \"" << b->tuning << "\"}";
    const std::string js = o.str();
    if (needed) *needed = js.size() + 1;
    OCEAN_CHECK(buf == nullptr || cap >= js.size() + 1, OCEAN_ERR_CAPACITY, "buffer too small");
    if (buf) std::memcpy(buf, js.c_str(), js.size() + 1);
  });
}


int ocean_batch_download(ocean_batch* b, void* rowptrs, uint32_t* col, double* val, void* stream) {
  return guarded([&] {
    batch_download(b, rowptrs, col, val, (cudaStream_t)stream);
    OCEAN_CUDA(cudaStreamSynchronize((cudaStream_t)stream));
  });
}

int ocean_batch_download_async(ocean_batch* b, void* rowptrs, uint32_t* col, double* val, void* stream) {
  return guarded([&] { batch_download(b, rowptrs, col, val, (cudaStream_t)stream); });
}

int ocean_batch_destroy(ocean_batch* b) {
  return guarded([&] { delete b; });
}

int ocean_spgemm_batched(ocean_handle* h, uint64_t n, const ocean_csr_view* A, const ocean_csr_view* B,
                         ocean_csr* C, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr && C != nullptr, OCEAN_ERR_INVALID, "handle or C is NULL");
    std::unique_ptr<ocean_batch> b(new ocean_batch());
    b->h = h;
    b->cfg = h->cfg;
    batch_setup(b.get(), n, A, B);
    cudaStream_t s = (cudaStream_t)stream;
    if (b->rows == 0) {
      b->out_bits = 32;
      b->c_off.assign(b->n + 1, 0);
      OCEAN_CUDA(cudaMalloc(&b->c_rp, b->n * 4ull));
      OCEAN_CUDA(cudaMemset(b->c_rp, 0, b->n * 4ull));
    } else {
      batch_run_pipeline(b.get(), s, true);
    }
    batch_outputs(b.get(), C);
    CResult* o = new CResult{0};
    o->rowptr = b->c_rp;
    o->col = b->c_col;
    o->val = b->c_val;
    o->refs = (int)b->n;
    o->plain_alloc = true;
    b->c_rp = nullptr, b->c_col = nullptr, b->c_val = nullptr;  // now owned by the results
    for (uint32_t p = 0; p < b->n; ++p) {
      C[p].location = 0;
      C[p]._owner = o;
    }
  });
}

int ocean_stats_json(ocean_handle* h, char* buf, size_t cap, size_t* needed) {
  return guarded([&] {
    OCEAN_CHECK(h != nullptr, OCEAN_ERR_INVALID, "handle is NULL");
    const std::string js = stats_json(h);
    if (needed) *needed = js.size() + 1;
    OCEAN_CHECK(buf == nullptr || cap >= js.size() + 1, OCEAN_ERR_CAPACITY, "stats buffer too small");
    if (buf) std::memcpy(buf, js.c_str(), js.size() + 1);
  });
}

double ocean_stage_ms(ocean_handle* h, const char* stage) {
  if (!h || !stage || !h->ev_recorded) return -1.0;
  const std::string s(stage);
  if (s == "total") return ev_ms(h, EV_START, EV_END);
  if (!h->tracked) return -1.0;
  if (s == "analysis") return ev_ms(h, EV_START, EV_ANALYSIS);
  if (s == "symbolic") return ev_ms(h, EV_SYM0, EV_SYMBOLIC);
  if (s == "scan") return ev_ms(h, EV_SYMBOLIC, EV_SCAN);
  if (s == "numeric") return ev_ms(h, EV_NUM0, EV_NUM_END);
  for (int i = 0; i < SB_COUNT; ++i)
    if (s == std::string("symbolic_") + kSymNames[i]) return ev_ms(h, EV_SYM0 + i, EV_SYM0 + i + 1);
  for (int i = 0; i < NB_COUNT; ++i)
    if (s == std::string("numeric_") + kNumNames[i]) return ev_ms(h, EV_NUM0 + i, EV_NUM0 + i + 1);
  return -1.0;
}

int ocean_murmur3_u32(const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t seed, void* stream) {
  return guarded([&] {
    OCEAN_CHECK(n == 0 || (keys && out), OCEAN_ERR_INVALID, "keys/out is NULL");
    launch_murmur3(keys, out, n, seed, (cudaStream_t)stream);
    OCEAN_CUDA(cudaGetLastError());
  });
}

const char* ocean_last_error(void) { return g_last_error.c_str(); }
const char* ocean_version(void) { return "ocean-b200 0.1.0"; }

}  // extern "C"
