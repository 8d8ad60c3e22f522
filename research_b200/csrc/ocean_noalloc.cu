// ocean_symbolic_noalloc: the symbolic phase (exact output count of every row
// of C = A·B) without any allocation by the library.
//
// Who needs it: callers that cannot let a library allocate device memory on
// their path. Examples are applications whose device memory is owned by their
// own arena or caching allocator (a cudaMalloc from a library then fails or
// fragments the arena), and latency-bound services that forbid allocation in
// steady state because cudaMalloc/cudaFree can synchronize the device and take
// unbounded time. The regular entry points (ocean_create, ocean_symbolic) grow
// per-handle workspaces and a pinned read-back buffer, so they allocate.
//
// How: all scratch of the analysis and symbolic kernels (per-row products,
// column spans, A-row lengths, class lists and the device counters) lives in
// one file-scope device array of fixed size, kNoAllocScratchBytes (about 7.3 MB),
// which every GPU that loads this library holds until the process exits. It
// bounds A to kNoAllocMaxRows rows; larger inputs are rejected with
// OCEAN_ERR_INVALID before any work. Inputs and the output array row_nnz are
// the caller's. Every class kernel is launched with its full persistent grid
// (no read-back of class sizes), and the row bitmaps are not saved.
//
// Set-up: the first call on a device, with that device current, resolves the
// array's device address with cudaGetSymbolAddress and sets the kernels'
// shared-memory limits; make that first call before any stream capture. The
// address is kept for the life of the process: a cudaDeviceReset after the
// first call is not supported (the module, and with it the array, is reloaded
// at another address).
// All calls share the one array and it keeps the last call's contents: each
// call clears the counters it relies on (a stream-ordered memset), and calls
// that overlap on the GPU (different streams, no ordering between them) race on
// the array, so callers must order them (one stream, or events).
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdio>
#include <mutex>

#include "kernels.h"
#include "ocean.h"

namespace ocean {
namespace {

constexpr uint64_t kNoAllocMaxRows = 131072;
constexpr uint64_t kCountersBytes = 1024;
constexpr uint64_t kNoAllocScratchBytes =
    kCountersBytes + kNoAllocMaxRows * (4 /*prod*/ + 4 /*lo*/ + 4 /*hi*/ + 4 /*anz*/ + 4 /*maxb*/ + 8 /*bm_off*/ +
                                        4 * (uint64_t)SB_COUNT /*class lists*/);
static_assert(sizeof(DevCounters) <= kCountersBytes, "counters do not fit their slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mutex;
void* g_scratch_addr[64] = {nullptr};
int g_num_sms[64] = {0};

// Resolves the scratch array's device address on the current device (once).
bool setup_device(int dev, void** addr, int* sms, char* err, size_t errlen) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (dev < 0 || dev >= 64) {
    snprintf(err, errlen, "device ordinal %d out of range", dev);
    return false;
  }
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) {
      snprintf(err, errlen, "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return false;
    }
    int n = 0;
    const cudaError_t e2 = cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    if (e2 != cudaSuccess) {
      snprintf(err, errlen, "cudaDeviceGetAttribute: %s", cudaGetErrorString(e2));
      return false;
    }
    if (!ensure_kernel_attributes(dev)) {
      snprintf(err, errlen, "device ordinal %d out of range", dev);
      return false;
    }
    g_num_sms[dev] = n;
    g_scratch_addr[dev] = p;
  }
  *addr = g_scratch_addr[dev];
  *sms = g_num_sms[dev];
  return true;
}

template <typename RP>
int run_noalloc(const ocean_csr_view* A, const ocean_csr_view* B, uint32_t* row_nnz, cudaStream_t s,
                unsigned char* scratch, int sms) {
  DevWork w;
  w.rows = A->rows;
  const uint64_t R = kNoAllocMaxRows;
  w.ctr = reinterpret_cast<DevCounters*>(scratch);
  unsigned char* p = scratch + kCountersBytes;
  w.bm_off = reinterpret_cast<uint64_t*>(p);
  p += R * 8;
  w.prod = reinterpret_cast<uint32_t*>(p);
  p += R * 4;
  w.lo = reinterpret_cast<uint32_t*>(p);
  p += R * 4;
  w.hi = reinterpret_cast<uint32_t*>(p);
  p += R * 4;
  w.anz = reinterpret_cast<uint32_t*>(p);
  p += R * 4;
  w.maxb = reinterpret_cast<uint32_t*>(p);
  p += R * 4;
  w.sym_bins = reinterpret_cast<uint32_t*>(p);  // class lists are strided by A->rows (<= R)
  w.row_nnz = row_nnz;
  w.bm_cache = nullptr;
  w.bm_cache_words = 0;

  Csr<RP> a, b;
  a.rows = A->rows, a.cols = A->cols, a.nnz = A->nnz, a.rp = (const RP*)A->rowptr, a.col = A->col, a.val = A->val;
  b.rows = B->rows, b.cols = B->cols, b.nnz = B->nnz, b.rp = (const RP*)B->rowptr, b.col = B->col, b.val = B->val;

  // the counters (class sizes, row cursors, status) must start at zero
  cudaError_t e = cudaMemsetAsync(w.ctr, 0, sizeof(DevCounters), s);
  if (e == cudaSuccess) {
    SymPolicy pol;
    launch_analysis(a, b, w, pol, s);
    launch_symbolic(a, b, w, sms, s, nullptr, nullptr);
    e = cudaGetLastError();
  }
  // status and err_row are adjacent in the counters: one read-back of both
  static_assert(offsetof(DevCounters, err_row) == offsetof(DevCounters, status) + sizeof(unsigned),
                "status and err_row must be adjacent");
  unsigned st[2] = {0, 0};
  if (e == cudaSuccess) e = cudaMemcpyAsync(st, &w.ctr->status, sizeof(st), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e));
    return OCEAN_ERR_CUDA;
  }
  if (st[0]) {
    char msg[256];
    const char* what = (st[0] & DEV_TABLE_FULL)     ? "a shared-memory hash table ran full (probe limit reached)"
                       : (st[0] & DEV_BIN_OVERFLOW) ? "a row exceeded the capacity of its accumulator class"
                                                    : "device error";
    snprintf(msg, sizeof msg, "ocean_symbolic_noalloc: %s (status 0x%x, first row %u)", what, st[0], st[1]);
    set_last_error(msg);
    return OCEAN_ERR_CAPACITY;
  }
  return OCEAN_OK;
}

}  // namespace
}  // namespace ocean

extern "C" int ocean_symbolic_noalloc(const ocean_csr_view* A, const ocean_csr_view* B, uint32_t* row_nnz,
                                      void* stream) {
  using namespace ocean;
  if (!A || !B || (A->rows && !row_nnz)) {
    set_last_error("ocean_symbolic_noalloc: NULL argument");
    return OCEAN_ERR_INVALID;
  }
  if (A->rowptr_bits != B->rowptr_bits || (A->rowptr_bits != 32 && A->rowptr_bits != 64)) {
    set_last_error("ocean_symbolic_noalloc: A and B need the same row-pointer width (32 or 64)");
    return OCEAN_ERR_INVALID;
  }
  if (A->cols != B->rows) {
    set_last_error("ocean_symbolic_noalloc: Incompatible matrix dimensions (A.cols != B.rows)");
    return OCEAN_ERR_INVALID;
  }
  if (A->rows > kNoAllocMaxRows) {
    char msg[160];
    snprintf(msg, sizeof msg, "ocean_symbolic_noalloc: A has %llu rows, more than the fixed scratch allows (%llu)",
             (unsigned long long)A->rows, (unsigned long long)kNoAllocMaxRows);
    set_last_error(msg);
    return OCEAN_ERR_INVALID;
  }
  if ((A->rows && !A->rowptr) || (A->nnz && (!A->col || !A->val)) || (B->rows && !B->rowptr) ||
      (B->nnz && (!B->col || !B->val)) || B->cols > 0xFFFFFFFFull) {
    set_last_error("ocean_symbolic_noalloc: invalid matrix view");
    return OCEAN_ERR_INVALID;
  }
  if (A->rows == 0) return OCEAN_OK;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    set_last_error(cudaGetErrorString(e));
    return OCEAN_ERR_CUDA;
  }
  void* scratch = nullptr;
  int sms = 0;
  char err[200];
  if (!setup_device(dev, &scratch, &sms, err, sizeof err)) {
    set_last_error(err);
    return OCEAN_ERR_CUDA;
  }
  if (A->rowptr_bits == 32)
    return run_noalloc<uint32_t>(A, B, row_nnz, (cudaStream_t)stream, (unsigned char*)scratch, sms);
  return run_noalloc<uint64_t>(A, B, row_nnz, (cudaStream_t)stream, (unsigned char*)scratch, sms);
}
