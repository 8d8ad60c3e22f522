/*
 * ocean.h — C ABI of the B200-native estimation-based SpGEMM (C = A·B, CSR, FP64).
 *
 * Every entry point is plain C: pointers, sizes and status codes, no C++ or torch
 * types. Device pointers are CUDA device addresses on the current device; a
 * `stream` argument is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - somespgemm::SpGEMM::SpGEMM(const Config&)          kernels/SpGEMM.cuh:211
 *   - somespgemm::SpGEMM::run(shared_ptr<cuCSR>, ...)    kernels/SpGEMM.cuh:213-338
 *   - somespgemm::SpGEMM::get_stats()                    kernels/SpGEMM.cuh:340-342
 *   - somespgemm::from_json(const json&, Config&)        src/Utils.cpp:8-37
 *   - somespgemm::cuCSR / convert(cuCSR&, const CSR&)    include/CSR.h:35-51, src/CSR.cpp:226-250
 *   - somespgemm::loadCSR(const char*)                   src/CSR.cpp:119-152
 * Errors: the reference exits the process on CUDA errors (include/Common.h:296-310)
 * and throws on capacity/config problems; here every call returns an ocean_status
 * and ocean_last_error() gives the message of the calling thread's last failure.
 */
#ifndef OCEAN_H_
#define OCEAN_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  OCEAN_OK = 0,
  OCEAN_ERR_CUDA = 1,      /* a CUDA runtime call or kernel launch failed */
  OCEAN_ERR_CAPACITY = 2,  /* a bounded device structure (table, window, buffer) ran full */
  OCEAN_ERR_TIMEOUT = 3,   /* a bounded device-side wait gave up */
  OCEAN_ERR_INVALID = 4,   /* bad argument, dimension mismatch, bad config or file */
  OCEAN_ERR_OOM = 5,       /* device or pinned host allocation failed */
  OCEAN_ERR_INTERNAL = 6   /* an internal consistency check failed */
} ocean_status;

/* Read-only CSR view. `rowptr_bits` is 32 or 64. As in the reference
 * (src/CSR.cpp:54), the end of the last row is taken from `nnz`, so
 * rowptr[rows] is never read. Column ids are uint32, values double. */
typedef struct {
  uint64_t rows, cols, nnz;
  const void* rowptr;
  int32_t rowptr_bits;
  const uint32_t* col;
  const double* val;
} ocean_csr_view;

/* Owning CSR result. rowptr has rows+1 entries and rowptr[rows] == nnz (a
 * superset of the reference's contract, which leaves the last offset unspecified).
 * `rowptr_bits` is 32 when nnz < 2^32 (unless the config asks for 64), else 64.
 * `location` is 0 for device memory (free with ocean_csr_free), 1 for pinned
 * host memory lent by the handle (valid until the next call on that handle) and
 * 2 for device memory lent by a batch plan (valid until its next run). */
typedef struct {
  uint64_t rows, cols, nnz;
  void* rowptr;
  int32_t rowptr_bits;
  uint32_t* col;
  double* val;
  int32_t location;
  void* _owner; /* internal: allocation record */
} ocean_csr;

typedef struct ocean_handle ocean_handle;

/* Create a handle from JSON config text (NULL or "" = defaults). Accepts every
 * key of the reference's from_json (src/Utils.cpp:9-36, e.g. "track_stage_time",
 * "use_estimation_workflow", "hll_numeric_malloc_expansion_coe",
 * "segmentation_grid_max") with the same meaning, ignores unknown keys, and adds
 * optional keys of its own ("output_rowptr_bits", "estimator", ...). */
int ocean_create(ocean_handle** out, const char* json_config);
/* Same, reading the JSON config from a file path (reference: src/main.cu:53-59). */
int ocean_create_from_file(ocean_handle** out, const char* json_path);
void ocean_destroy(ocean_handle* h);

/* C = A·B with A, B in device memory. Allocates C on `stream` (stream-ordered
 * pool) and returns with C complete on `stream`. Replaces SpGEMM::run. */
int ocean_spgemm(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B,
                 ocean_csr* C, void* stream);

/* C = A·B with A, B in HOST memory (pinned or pageable). The call copies A and
 * B to the device, multiplies, and copies C back into pinned host buffers owned
 * by the handle (C->location == 1, reused by the next call). Replaces the
 * reference driver's cuCSR(H2D) → run → CSR(D2H) sequence (src/main.cu:61-67). */
int ocean_spgemm_host(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B,
                      ocean_csr* C, void* stream);

/* Release a device result of ocean_spgemm (stream-ordered on `stream`). */
int ocean_csr_free(ocean_csr* C, void* stream);

/* Copy a result into caller host buffers (rowptr: rows+1 entries of
 * C->rowptr_bits, col/val: nnz entries) and wait for the copy. Replaces
 * convert(CSR&, const cuCSR&) (src/CSR.cpp:243-250). */
int ocean_csr_download(const ocean_csr* C, void* rowptr, uint32_t* col, double* val, void* stream);

/* Copy rows [r0, r1) of a result into host buffers: rowptr receives r1-r0+1
 * absolute offsets (uint64), col/val the entries between them (pass NULL for
 * both to fetch the row pointers only). Lets a caller inspect part of a result
 * too large for host memory. */
int ocean_csr_download_rows(const ocean_csr* C, uint64_t r0, uint64_t r1, uint64_t* rowptr,
                            uint32_t* col, double* val, void* stream);

/* Exact per-row output counts of A·B (the symbolic phase alone) into the
 * device array row_nnz[A.rows]. Replaces the symbolic kernels' result
 * d_num_outputs_row (kernels/SpGEMM.cuh:759-923). */
int ocean_symbolic(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B,
                   uint32_t* row_nnz, void* stream);

/* Raw HyperLogLog estimate of every row's output count into the device array
 * est[A.rows]: register-wise maximum of the 2^log2p-register sketches
 * (log2p 5 or 6, MurmurHash3 seed 1234) of the B rows each A row references,
 * then the harmonic-mean estimate with small-range correction. Replaces
 * hllConstruct + hllMerge (kernels/HLL.cuh:28-236) without the expansion and
 * bin rounding. */
int ocean_row_estimates(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, int log2p,
                        uint32_t* est, void* stream);

/* ocean_symbolic without any allocation by the library, for callers that
 * cannot let a library allocate device memory (an application-owned arena or
 * caching allocator holds the device memory; or a service forbids cudaMalloc in
 * steady state because it can synchronize the device). No handle: the scratch
 * of the analysis and symbolic kernels is one fixed device array inside the
 * library (about 7.3 MB, held by every GPU that loads the library until exit),
 * so A may have at most 131072 rows (larger A: OCEAN_ERR_INVALID). A and B need
 * the same row-pointer width; row_nnz[A.rows] is the caller's device array. The
 * first call on a device resolves the array's address and must come before any
 * stream capture; the address is kept, so a cudaDeviceReset after that first
 * call is not supported. Calls share the array: calls that overlap on the GPU
 * race and must be ordered by the caller. Waits for the result before returning.
 * No counterpart in the reference (which allocates on every run). */
int ocean_symbolic_noalloc(const ocean_csr_view* A, const ocean_csr_view* B, uint32_t* row_nnz,
                           void* stream);

/* ---- Learned row-size estimator -------------------------------------------
 * A 3-layer perceptron (16 features -> 64 -> 64 -> 1, ReLU) predicting
 * t = log2(1 + nnz of an output row). Its GEMMs run on the tensor cores with
 * BF16 weights/activations and FP32 accumulation. With the config key
 * "use_learned_estimator" it replaces the HLL estimate that sizes each row in
 * the estimation workflow (the reference's estimator: kernels/HLL.cuh:107-236
 * feeding kernels/SpGEMM.cuh:1395-1480); rows that outgrow the estimate are
 * counted and recomputed exactly, so C is unchanged. No counterpart in the
 * reference. The entry points below train and check the network; all pointers
 * except `blob` are device pointers. */
#define OCEAN_MLP_FEATURES 16
#define OCEAN_MLP_PARAMS 5313 /* W1[64][16], b1[64], W2[64][64], b2[64], w3[64], b3 */
#define OCEAN_MLP_BLOB 5346   /* params, mu[16], inv_sd[16], margin */

typedef struct {
  const float* params; /* OCEAN_MLP_PARAMS floats; weights are rounded to BF16 on use */
  const float* mu;     /* feature means (16) */
  const float* inv_sd; /* inverse feature standard deviations (16) */
  float margin;        /* log2 margin added before an estimate sizes a row */
} ocean_mlp_model;

/* Raw features of every row of A·B into feat[A.rows][16] (row analysis plus
 * the raw 32-register HLL union estimate). Waits for the result. */
int ocean_mlp_features(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, float* feat,
                       void* stream);
/* pred[i] = network output for feat[i] (i < n). Waits for the result. */
int ocean_mlp_forward(ocean_handle* h, const ocean_mlp_model* m, const float* feat, uint64_t n, float* pred,
                      void* stream);
/* Forward and backward pass of L = sum_i (pred_i - target_i)^2 / batch over
 * the n rows: dL/dparams is ADDED to grad[OCEAN_MLP_PARAMS] and the sum of
 * squared errors to *loss. Waits for the result. */
int ocean_mlp_grad(ocean_handle* h, const ocean_mlp_model* m, const float* feat, const float* target, uint64_t n,
                   float batch, float* grad, float* loss, void* stream);
/* One Adam step (bias-corrected, step >= 1) on params; zeroes grad. */
int ocean_mlp_adam(ocean_handle* h, float* params, float* m1, float* m2, float* grad, int step, float lr,
                   float beta1, float beta2, float eps, void* stream);
/* Copies the built-in trained network (OCEAN_MLP_BLOB floats) to host `blob`. */
int ocean_mlp_builtin(float* blob, size_t n);

/* Per-row output-size estimates of A·B into est[A.rows], made as the
 * estimation workflow makes them. estimator 1 = HLL (kernels/HLL.cuh:107-236:
 * log2 precision 5 or 6 by the reference's rule; with_margin: times the
 * expansion 2.0 / 1.5, else the union estimate itself; clamped to
 * [1, min(products, span)]); 2 = the learned network (with_margin: plus its
 * log2 margin; clamped to [max(1, longest B row), min(products, span)]).
 * Rows of at most esc_max_products products get their product count. */
int ocean_estimate(ocean_handle* h, const ocean_csr_view* A, const ocean_csr_view* B, int estimator,
                   int with_margin, uint32_t* est, void* stream);
/* Quality of est[] against exact counts truth[] (device arrays) for the rows
 * of the handle's last analysed A·B (ocean_estimate or ocean_symbolic with
 * the same A and B) that have more than min_products products (0: all rows
 * with output): out[0] mean |est - truth| / truth; out[1] percent of them
 * whose numeric class differs; out[2] their number; out[3] rows with
 * est < truth (they would be rerun). */
int ocean_estimate_metrics(ocean_handle* h, const uint32_t* est, const uint32_t* truth, uint32_t min_products,
                           double* out, void* stream);

/* ---- Batches ---------------------------------------------------------------
 * Many independent products C[p] = A[p]·B[p] (B == NULL: C[p] = A[p]·A[p])
 * computed as one block-diagonal product: the rows of all A[p] are stacked
 * (their column ids shifted to the stacked B's rows), so every accumulator
 * class runs once, as one persistent launch over the rows of all problems.
 * No counterpart in the reference (one SpGEMM::run per product). */
typedef struct ocean_batch ocean_batch;

/* Plans a batch: stacks the problems, runs the pipeline once to size the
 * class lists and buffers, and captures the pipeline (input stacking,
 * analysis, estimation or exact counting, accumulators, row-pointer split)
 * into a CUDA graph with no host synchronisation inside. With the config key
 * "batch_autotune" the class policy (ESC limit, small-hash fill limit, bitmap
 * span limits) is first searched on the batch by timing graph launches. The
 * input device buffers and the handle must outlive the plan; their values may
 * change between runs, their structure may not. */
int ocean_batch_create(ocean_handle* h, uint64_t n, const ocean_csr_view* A, const ocean_csr_view* B,
                       ocean_batch** out, void* stream);
/* One run: a single graph launch on `stream`, then a wait and a check that the
 * structure still matches the plan; C[0..n) receive views of the results
 * (location 2: lent by the plan until its next run or destruction;
 * ocean_csr_free on them only clears the struct). */
int ocean_batch_run(ocean_batch* b, ocean_csr* C, void* stream);
/* The graph launch alone, without waiting or checking. */
int ocean_batch_launch(ocean_batch* b, void* stream);
/* Views of the results of the last completed run (as ocean_batch_run). */
int ocean_batch_results(ocean_batch* b, ocean_csr* C);
/* All results of the last completed run into host buffers and wait: rowptrs
 * receives every problem's row pointers one after another (A[p].rows + 1
 * values each, of the width in the results' rowptr_bits), col and val the
 * problems' entries one after another (the sum of their nnz). */
int ocean_batch_download(ocean_batch* b, void* rowptrs, uint32_t* col, double* val, void* stream);
/* The same copies, queued on `stream` without waiting, so that a pipeline of
 * several plans can copy one plan's results back while another computes (the
 * host buffers should be pinned; the caller synchronizes the stream). No
 * counterpart in the reference. */
int ocean_batch_download_async(ocean_batch* b, void* rowptrs, uint32_t* col, double* val, void* stream);
/* Plan facts as JSON: sizes, workflow, estimator, kernels per run, tuned policy. */
int ocean_batch_info_json(ocean_batch* b, char* buf, size_t cap, size_t* needed);
int ocean_batch_destroy(ocean_batch* b);
/* One-shot batch without a graph: C[p] are owned results that share one
 * allocation, released when every C[p] has been passed to ocean_csr_free. */
int ocean_spgemm_batched(ocean_handle* h, uint64_t n, const ocean_csr_view* A, const ocean_csr_view* B,
                         ocean_csr* C, void* stream);

/* Stats of the last multiply as JSON text, with the reference's keys
 * (kernels/SpGEMM.cuh:1788-1890: "A","B","C","stats","decision","timing",
 * "total_time","gflops", ...). If cap is too small, *needed gets the size. */
int ocean_stats_json(ocean_handle* h, char* buf, size_t cap, size_t* needed);

/* Device time in milliseconds of the last call's named stage ("analysis",
 * "symbolic", "scan", "numeric", "numeric_bitmap", ...), measured with CUDA
 * events on the launching stream when "track_stage_time" is on; -1 if absent. */
double ocean_stage_ms(ocean_handle* h, const char* stage);

/* 32-bit MurmurHash3 of each uint32 key with the given seed, on the device
 * (reference: kernels/MurmurHash.cuh:44-98, seed 1234 at include/Common.h:73). */
int ocean_murmur3_u32(const uint32_t* keys, uint32_t* out, uint64_t n, uint32_t seed,
                      void* stream);

/* Message of the calling thread's last failed call ("" if none). */
const char* ocean_last_error(void);
/* Library version string. */
const char* ocean_version(void);

#ifdef __cplusplus
}
#endif

#endif /* OCEAN_H_ */
