// Learned row-size estimator: a 3-layer perceptron (16 features -> 64 -> 64 ->
// 1, ReLU) whose GEMMs run on the tensor cores with BF16 operands and FP32
// accumulation (tcgen05, accumulators in TMEM). It predicts
// t = log2(1 + nnz of the output row) from per-row features of A * B.
// The reference has no counterpart; its estimator is HLL (kernels/HLL.cuh).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace ocean {

constexpr int kMlpF = 16;    // features (padded)
constexpr int kMlpH = 64;    // hidden width
constexpr int kMlpTile = 128;  // rows per tile (one thread per row)

// Offsets in the flat FP32 parameter vector (weights rounded to BF16 when a
// kernel stages them; biases stay FP32).
constexpr int kMlpOffW1 = 0;                            // [64][16]
constexpr int kMlpOffB1 = kMlpOffW1 + kMlpH * kMlpF;    // [64]
constexpr int kMlpOffW2 = kMlpOffB1 + kMlpH;            // [64][64]  (out, in)
constexpr int kMlpOffB2 = kMlpOffW2 + kMlpH * kMlpH;    // [64]
constexpr int kMlpOffW3 = kMlpOffB2 + kMlpH;            // [64]
constexpr int kMlpOffB3 = kMlpOffW3 + kMlpH;            // [1]
constexpr int kMlpParams = kMlpOffB3 + 1;               // 5313
// A stored network: parameters, feature means, inverse deviations, margin.
constexpr int kMlpBlob = kMlpParams + 2 * kMlpF + 1;    // 5346

// Model as the kernels see it: parameters plus the feature normalisation
// x = (f - mu) * inv_sd, and the log2 margin added before an estimate is
// turned into a preallocation.
struct MlpModel {
  const float* params = nullptr;  // kMlpParams
  const float* mu = nullptr;      // kMlpF
  const float* inv_sd = nullptr;  // kMlpF
  float margin = 0.f;
};

// Per-row quantities the features are made of (device arrays of A.rows).
struct MlpRowInputs {
  const uint32_t* anz = nullptr;
  const uint32_t* prod = nullptr;
  const uint32_t* lo = nullptr;
  const uint32_t* hi = nullptr;
  const uint32_t* maxb = nullptr;
  const uint32_t* hll = nullptr;  // raw HLL union estimate per row
  float log_b_cols = 0.f;         // log2(1 + B.cols)
  float log_b_avg = 0.f;          // log2(1 + nnz(B) / B.rows)
  // stacked batches: the two B scalars of each row's own problem
  // (ctx[row_problem[row]] = {log_b_cols, log_b_avg}) instead of the above
  const uint32_t* row_problem = nullptr;
  const float2* problem_ctx = nullptr;
};

// Raw (unnormalised) features of rows [0, n) into feat[n][16].
void launch_mlp_features(const MlpRowInputs& in, uint64_t n, float* feat, cudaStream_t s);

// Inference from stored features: pred[i] = predicted log2(1 + nnz).
// status: device word; DEV_TC_TIMEOUT is OR-ed in if a tensor-core wait timed out.
int launch_mlp_forward(const MlpModel& m, const float* feat, uint64_t n, float* pred, unsigned* status,
                       int num_sms, cudaStream_t s);

// Fused estimate for the estimation workflow: features from `in`, network,
// est[i] = clamp(ceil(2^(pred + margin) - 1), max(1, longest B row), min(products, span)),
// and est[i] = products for rows of at most esc_max products; est_raw
// (optional) the same without the margin. est may alias in.hll.
int launch_mlp_estimate(const MlpModel& m, const MlpRowInputs& in, uint64_t n, uint32_t esc_max, uint32_t* est,
                        uint32_t* est_raw, unsigned* status, int num_sms, cudaStream_t s);

// Forward + backward of the squared log2 error over rows [0, n), mean over
// `batch` rows: gradients are ADDED to grad[kMlpParams] and the summed squared
// error to *loss.
int launch_mlp_grad(const MlpModel& m, const float* feat, const float* target, uint64_t n, float batch,
                    float* grad, float* loss, unsigned* status, int num_sms, cudaStream_t s);

// Adam step on the FP32 parameters; zeroes grad.
void launch_mlp_adam(float* params, float* m1, float* m2, float* grad, int step, float lr, float beta1, float beta2,
                     float eps, cudaStream_t s);

// Estimate-quality metrics against exact counts: adds to acc[0] the sum of
// |est - true| / true over rows with true > 0, to acc[1] the number of those
// rows, to acc[2] the number of rows whose numeric class (from products, span
// and the count) differs between est and true, and to acc[3] the number of
// rows with est < true; only rows with more than min_products products count
// (min_products = 0: every row).
void launch_est_metrics(const uint32_t* est, const uint32_t* truth, const MlpRowInputs& in, uint64_t n,
                        const NumPolicy& pol, uint32_t min_products, double* acc, cudaStream_t s);

void configure_mlp_attributes();

}  // namespace ocean
