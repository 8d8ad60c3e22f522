// Learned row-size estimator kernels (tcgen05 BF16 x BF16 -> FP32 in TMEM).
//
// One CTA = 4 warps = 128 threads; a tile is 128 rows of the batch, thread t
// owns row t of the tile, which is also TMEM lane t (warp w reads lanes
// 32w..32w+31). Per tile:
//   layer 1  D1[128 x 64]  = X[128 x 16]  * W1^T        (1 MMA,  K = 16)
//   layer 2  D2[128 x 64]  = H1[128 x 64] * W2^T        (4 MMAs, K = 64)
//   layer 3  D3[128 x 16]  = H2[128 x 64] * W3pad^T     (4 MMAs; row 0 of W3pad is w3)
// and, for training,
//   dH1      D4[128 x 64]  = dZ2[128 x 64] * W2         (4 MMAs; B operand W2^T)
//   weights  DW[128 x 80] += [dZ2^T; dZ1^T][128 x 128] * [H1^T; X^T]^T   (8 MMAs, K = 128 rows)
// where DW rows 0-63 x cols 0-63 are dW2 and rows 64-127 x cols 64-79 are dW1
// (the off-diagonal blocks are unused). DW stays in TMEM across all tiles a CTA
// processes and is added to the global gradient once. Epilogues (bias, ReLU,
// masks, BF16 rounding) run on the CUDA cores between the MMAs.
#include <cmath>

#include "mlp.h"
#include "tc05.cuh"

namespace ocean {
namespace {

using namespace tc05;

constexpr uint32_t kWaitTries = 1u << 24;
constexpr int kF32Floats = 228;

// ---- shared memory of the inference kernel (bytes)
constexpr uint32_t kFX = 0;               // X   [128][16]  K-major
constexpr uint32_t kFW1 = kFX + 4096;     // W1  [64][16]
constexpr uint32_t kFH = kFW1 + 2048;     // H1, then H2 [128][64]
constexpr uint32_t kFW2 = kFH + 16384;    // W2  [64][64]
constexpr uint32_t kFW3 = kFW2 + 8192;    // W3pad [16][64]
constexpr uint32_t kFF32 = kFW3 + 2048;   // b1[64] b2[64] b3[4] mu[16] inv_sd[16] w3[64]
constexpr uint32_t kFUsed = kFF32 + kF32Floats * 4;
// 56 KB per CTA keeps at most 4 CTAs on an SM, so 4 x 128 TMEM columns fit.
constexpr uint32_t kFwdSmem = 56 * 1024;
constexpr uint32_t kFwdTmemCols = 128;

// ---- shared memory of the training kernel (bytes)
constexpr uint32_t kGX = 0;               // X   [128][16]
constexpr uint32_t kGW1 = kGX + 4096;     // W1  [64][16]
constexpr uint32_t kGH = kGW1 + 2048;     // H1, then H2, then dZ2 [128][64]
constexpr uint32_t kGW2 = kGH + 16384;    // W2  [64][64]
constexpr uint32_t kGW3 = kGW2 + 8192;    // W3pad [16][64]
constexpr uint32_t kGW2T = kGW3 + 2048;   // W2^T [64][64]
constexpr uint32_t kGEA = kGW2T + 8192;   // [dZ2^T; dZ1^T] [128 rows][128 K]
constexpr uint32_t kGEB = kGEA + 32768;   // [H1^T; X^T]    [80 rows][128 K]
constexpr uint32_t kGF32 = kGEB + 20480;  // b1 b2 b3[4] mu inv_sd w3
constexpr uint32_t kGAcc = kGF32 + kF32Floats * 4;  // dW3[64] db1[64] db2[64] db3 loss (+2 pad)
constexpr uint32_t kGUsed = kGAcc + 196 * 4;
// 96 KB per CTA keeps at most 2 CTAs on an SM, so 2 x 256 TMEM columns fit.
constexpr uint32_t kGradSmem = 96 * 1024;
constexpr uint32_t kGradTmemCols = 256;
static_assert(kFUsed <= kFwdSmem && kGUsed <= kGradSmem, "shared memory layout");

// F32 region offsets (floats); w3 holds the BF16-rounded layer-3 weights
constexpr int kB1 = 0, kB2 = 64, kB3 = 128, kMu = 132, kIsd = 148, kW3 = 164;
// accumulator offsets (floats)
constexpr int kAW3 = 0, kAB1 = 64, kAB2 = 128, kAB3 = 192, kALoss = 193;

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// Stages W1, W2, W3pad (and W2^T) as BF16 K-major tiles, biases and the
// normalisation as FP32.
__device__ void stage_model(const MlpModel& m, unsigned char* sm, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t w2t,
                            float* f32) {
  const float* P = m.params;
  for (int u = threadIdx.x; u < 64 * 2; u += blockDim.x) {
    const int o = u >> 1, c = u & 1;
    float f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = P[kMlpOffW1 + o * kMlpF + c * 8 + i];
    *reinterpret_cast<uint4*>(sm + w1 + kmajor_offset(o, c * 8, 64)) = pack8_bf16(f);
  }
  for (int u = threadIdx.x; u < 64 * 8; u += blockDim.x) {
    const int o = u >> 3, c = u & 7;
    float f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = P[kMlpOffW2 + o * kMlpH + c * 8 + i];
    *reinterpret_cast<uint4*>(sm + w2 + kmajor_offset(o, c * 8, 64)) = pack8_bf16(f);
    if (w2t != ~0u) {
      // W2^T row i = o here, column chunk c: W2[c*8 + j][o]
#pragma unroll
      for (int j = 0; j < 8; ++j) f[j] = P[kMlpOffW2 + (c * 8 + j) * kMlpH + o];
      *reinterpret_cast<uint4*>(sm + w2t + kmajor_offset(o, c * 8, 64)) = pack8_bf16(f);
    }
  }
  for (int u = threadIdx.x; u < 16 * 8; u += blockDim.x) {
    const int n = u >> 3, c = u & 7;
    float f[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = n == 0 ? P[kMlpOffW3 + c * 8 + i] : 0.f;
    *reinterpret_cast<uint4*>(sm + w3 + kmajor_offset(n, c * 8, 16)) = pack8_bf16(f);
  }
  for (int i = threadIdx.x; i < 64; i += blockDim.x) {
    f32[kB1 + i] = P[kMlpOffB1 + i];
    f32[kB2 + i] = P[kMlpOffB2 + i];
    f32[kW3 + i] = bf16_round(P[kMlpOffW3 + i]);
  }
  if (threadIdx.x < 16) {
    f32[kMu + threadIdx.x] = m.mu[threadIdx.x];
    f32[kIsd + threadIdx.x] = m.inv_sd[threadIdx.x];
  }
  if (threadIdx.x == 0) f32[kB3] = P[kMlpOffB3];
}

// Raw features of one row (the network's input before normalisation).
__device__ __forceinline__ void row_features(const MlpRowInputs& in, uint64_t row, float (&f)[kMlpF]) {
  const float anz = (float)in.anz[row];
  const uint32_t p = in.prod[row];
  const uint64_t span = p ? (uint64_t)in.hi[row] - in.lo[row] + 1 : 0;
  const uint64_t ub = p < span ? p : span;
  f[0] = log2f(1.f + anz);
  f[1] = log2f(1.f + (float)p);
  f[2] = log2f(1.f + (float)span);
  f[3] = log2f(1.f + (float)in.maxb[row]);
  f[4] = log2f(1.f + (float)ub);
  f[5] = log2f(1.f + (float)in.hll[row]);
  f[6] = f[1] - f[0];
  f[7] = f[5] - f[4];
  if (in.row_problem) {
    const float2 c = in.problem_ctx[in.row_problem[row]];
    f[8] = c.x;
    f[9] = c.y;
  } else {
    f[8] = in.log_b_cols;
    f[9] = in.log_b_avg;
  }
  f[10] = f[3] - f[4];
#pragma unroll
  for (int i = 11; i < kMlpF; ++i) f[i] = 0.f;
}

__global__ void __launch_bounds__(256) k_mlp_features(MlpRowInputs in, uint64_t n, float* __restrict__ feat) {
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    float f[kMlpF];
    row_features(in, r, f);
    float4* o = reinterpret_cast<float4*>(feat + r * kMlpF);
#pragma unroll
    for (int i = 0; i < kMlpF / 4; ++i) o[i] = make_float4(f[4 * i], f[4 * i + 1], f[4 * i + 2], f[4 * i + 3]);
  }
}

// Writes this thread's normalised feature row as BF16 into the X tile.
__device__ __forceinline__ void put_x(unsigned char* sm, uint32_t xoff, const float* f32, const float (&f)[kMlpF],
                                     bool valid, float (&xr)[kMlpF]) {
#pragma unroll
  for (int i = 0; i < kMlpF; ++i) xr[i] = valid ? bf16_round((f[i] - f32[kMu + i]) * f32[kIsd + i]) : 0.f;
  *reinterpret_cast<uint4*>(sm + xoff + kmajor_offset(threadIdx.x, 0, 128)) = pack8_bf16(xr);
  *reinterpret_cast<uint4*>(sm + xoff + kmajor_offset(threadIdx.x, 8, 128)) = pack8_bf16(xr + 8);
}

// bias + ReLU of 64 accumulator columns -> BF16 row of a [128][64] tile;
// returns the ReLU mask (bit j: z_j > 0).
__device__ __forceinline__ unsigned long long relu_layer(uint32_t taddr, const float* bias, unsigned char* sm,
                                                         uint32_t hoff, float* keep /* 64 or null */) {
  unsigned long long mask = 0;
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    float v[16];
    tmem_ld16(taddr + q * 16, v);
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      const float z = v[i] + bias[q * 16 + i];
      mask |= (unsigned long long)(z > 0.f) << (q * 16 + i);
      v[i] = z > 0.f ? z : 0.f;
    }
    *reinterpret_cast<uint4*>(sm + hoff + kmajor_offset(threadIdx.x, q * 16, 128)) = pack8_bf16(v);
    *reinterpret_cast<uint4*>(sm + hoff + kmajor_offset(threadIdx.x, q * 16 + 8, 128)) = pack8_bf16(v + 8);
    if (keep) {
#pragma unroll
      for (int i = 0; i < 16; ++i) keep[q * 16 + i] = bf16_round(v[i]);
    }
  }
  return mask;
}

// Thread 0: the MMAs of one K-major product, then the commit.
__device__ __forceinline__ void issue(uint32_t d_tmem, uint32_t a_saddr, uint32_t a_lbo, uint32_t b_saddr,
                                      uint32_t b_lbo, int n, int ksteps, bool accumulate_first, uint64_t* mbar) {
  fence_after_sync();
  const uint32_t idesc = idesc_bf16_f32(128, n);
  for (int s = 0; s < ksteps; ++s) {
    const uint64_t a = smem_desc(a_saddr + s * 2 * a_lbo, a_lbo, 128);
    const uint64_t b = smem_desc(b_saddr + s * 2 * b_lbo, b_lbo, 128);
    mma_bf16(d_tmem, a, b, idesc, accumulate_first || s > 0);
  }
  commit(mbar);
}

// All threads: shared-memory writes done -> visible to the tensor cores.
__device__ __forceinline__ void publish() {
  fence_smem_to_async();
  fence_before_sync();
  __syncthreads();
}

// All threads: waits for the commit of the current phase; false (for every
// thread) if any thread gave up.
__device__ __forceinline__ bool await(uint64_t* mbar, uint32_t& phase) {
  const bool ok = mbar_wait(mbar, phase, kWaitTries);
  phase ^= 1u;
  const int bad = __syncthreads_or(!ok);
  fence_after_sync();
  return bad == 0;
}

// Preallocation of one row from the prediction y = log2(1 + nnz): rows of at
// most esc_max products get their product count; others 2^(y + margin) - 1,
// rounded up and clamped to [max(1, longest B row), min(products, span)].
__device__ __forceinline__ uint32_t estimate_from_pred(const MlpRowInputs& in, uint64_t row, float y, float margin,
                                                       uint32_t esc_max) {
  const uint32_t p = in.prod[row];
  if (p == 0) return 0;
  if (p <= esc_max) return p;
  const uint64_t span = (uint64_t)in.hi[row] - in.lo[row] + 1;
  const double ub = (double)(p < span ? p : span);
  double lb = (double)in.maxb[row];
  lb = lb < 1.0 ? 1.0 : lb;
  double x = exp2((double)y + (double)margin) - 1.0;
  if (!(x >= lb)) x = lb;
  if (x > ub) x = ub;
  return (uint32_t)ceil(x);
}

// Inference. FromWork: features computed from the analysis arrays and the
// estimate written; otherwise features read from feat[n][16].
template <bool FromWork>
__global__ void __launch_bounds__(128) k_mlp_infer(MlpModel m, MlpRowInputs in, const float* __restrict__ feat,
                                                   uint64_t n, uint32_t esc_max, uint32_t* __restrict__ est,
                                                   uint32_t* __restrict__ est_raw, float* __restrict__ pred,
                                                   unsigned* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  float* f32 = reinterpret_cast<float*>(sm + kFF32);
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tmem_alloc(&tmem_slot, kFwdTmemCols);
  if (threadIdx.x == 0) mbar_init(&mbar, 1);
  stage_model(m, sm, kFW1, kFW2, kFW3, ~0u, f32);
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t sbase = smem_u32(sm);
  uint32_t phase = 0;
  bool ok = true;
  const uint64_t tiles = (n + kMlpTile - 1) / kMlpTile;
  for (uint64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const uint64_t row = t * kMlpTile + threadIdx.x;
    const bool valid = row < n;
    float f[kMlpF], xr[kMlpF];
    if (valid) {
      if (FromWork) {
        row_features(in, row, f);
      } else {
        const float4* src = reinterpret_cast<const float4*>(feat + row * kMlpF);
#pragma unroll
        for (int i = 0; i < kMlpF / 4; ++i) {
          const float4 q = src[i];
          f[4 * i] = q.x, f[4 * i + 1] = q.y, f[4 * i + 2] = q.z, f[4 * i + 3] = q.w;
        }
      }
    }
    put_x(sm, kFX, f32, f, valid, xr);
    publish();
    if (threadIdx.x == 0) issue(tmem, sbase + kFX, 2048, sbase + kFW1, 1024, 64, 1, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    relu_layer(lane_addr, f32 + kB1, sm, kFH, nullptr);
    publish();
    if (threadIdx.x == 0) issue(tmem + 64, sbase + kFH, 2048, sbase + kFW2, 1024, 64, 4, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    relu_layer(lane_addr + 64, f32 + kB2, sm, kFH, nullptr);
    publish();
    if (threadIdx.x == 0) issue(tmem, sbase + kFH, 2048, sbase + kFW3, 256, 16, 4, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    float v[16];
    tmem_ld16(lane_addr, v);
    const float y = v[0] + f32[kB3];
    if (valid) {
      if (pred) pred[row] = y;
      if (FromWork) {
        est[row] = estimate_from_pred(in, row, y, m.margin, esc_max);
        if (est_raw) est_raw[row] = estimate_from_pred(in, row, y, 0.f, esc_max);
      }
    }
    fence_before_sync();
    __syncthreads();
  }
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(status, (unsigned)DEV_TC_TIMEOUT);
    mbar_wait(&mbar, phase, kWaitTries);  // the MMAs in flight, if any
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, kFwdTmemCols);
}

// Sum over the warp, lane 0 adds it to *dst (shared).
__device__ __forceinline__ void warp_add(float v, float* dst) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(dst, v);
}

__global__ void __launch_bounds__(128) k_mlp_grad(MlpModel m, const float* __restrict__ feat,
                                                  const float* __restrict__ target, uint64_t n, float inv_batch,
                                                  float* __restrict__ grad, float* __restrict__ loss,
                                                  unsigned* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char sm[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  float* f32 = reinterpret_cast<float*>(sm + kGF32);
  float* acc = reinterpret_cast<float*>(sm + kGAcc);
  const int warp = threadIdx.x >> 5;
  if (warp == 0) tmem_alloc(&tmem_slot, kGradTmemCols);
  if (threadIdx.x == 0) mbar_init(&mbar, 1);
  stage_model(m, sm, kGW1, kGW2, kGW3, kGW2T, f32);
  for (int i = threadIdx.x; i < 196; i += blockDim.x) acc[i] = 0.f;
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  const uint32_t tmem = tmem_slot;
  const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
  const uint32_t sbase = smem_u32(sm);
  const uint32_t r = threadIdx.x;
  const float* w3 = f32 + kW3;
  uint32_t phase = 0;
  bool ok = true;
  int done_tiles = 0;
  const uint64_t tiles = (n + kMlpTile - 1) / kMlpTile;
  for (uint64_t t = blockIdx.x; t < tiles && ok; t += gridDim.x) {
    const uint64_t row = t * kMlpTile + r;
    const bool valid = row < n;
    float f[kMlpF], xr[kMlpF];
    if (valid) {
      const float4* src = reinterpret_cast<const float4*>(feat + row * kMlpF);
#pragma unroll
      for (int i = 0; i < kMlpF / 4; ++i) {
        const float4 q = src[i];
        f[4 * i] = q.x, f[4 * i + 1] = q.y, f[4 * i + 2] = q.z, f[4 * i + 3] = q.w;
      }
    }
    put_x(sm, kGX, f32, f, valid, xr);
#pragma unroll
    for (int i = 0; i < kMlpF; ++i)  // X^T into rows 64..79 of EB
      *reinterpret_cast<__nv_bfloat16*>(sm + kGEB + kmajor_offset(64 + i, r, 80)) = __float2bfloat16_rn(xr[i]);
    publish();
    if (r == 0) issue(tmem, sbase + kGX, 2048, sbase + kGW1, 1024, 64, 1, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    float keep[kMlpH];
    const unsigned long long mask1 = relu_layer(lane_addr, f32 + kB1, sm, kGH, keep);
#pragma unroll
    for (int i = 0; i < kMlpH; ++i)  // H1^T into rows 0..63 of EB
      *reinterpret_cast<__nv_bfloat16*>(sm + kGEB + kmajor_offset(i, r, 80)) = __float2bfloat16_rn(keep[i]);
    publish();
    if (r == 0) issue(tmem + 64, sbase + kGH, 2048, sbase + kGW2, 1024, 64, 4, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    const unsigned long long mask2 = relu_layer(lane_addr + 64, f32 + kB2, sm, kGH, keep);  // keep = bf16 h2
    publish();
    if (r == 0) issue(tmem, sbase + kGH, 2048, sbase + kGW3, 256, 16, 4, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    float v[16];
    tmem_ld16(lane_addr, v);
    const float y = v[0] + f32[kB3];
    const float diff = valid ? y - target[row] : 0.f;
    const float dy = 2.f * diff * inv_batch;
    warp_add(diff * diff, acc + kALoss);
    warp_add(dy, acc + kAB3);
    // layer 3 weights; then dZ2 (into the H region, this thread's own row, and EA rows 0..63)
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) warp_add(dy * keep[j], acc + kAW3 + j);
    float dz[kMlpH];
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) dz[j] = ((mask2 >> j) & 1ull) ? dy * w3[j] : 0.f;
#pragma unroll
    for (int j = 0; j < kMlpH; ++j) warp_add(dz[j], acc + kAB2 + j);
#pragma unroll
    for (int q = 0; q < 8; ++q)
      *reinterpret_cast<uint4*>(sm + kGH + kmajor_offset(r, q * 8, 128)) = pack8_bf16(dz + q * 8);
#pragma unroll
    for (int j = 0; j < kMlpH; ++j)
      *reinterpret_cast<__nv_bfloat16*>(sm + kGEA + kmajor_offset(j, r, 128)) = __float2bfloat16_rn(dz[j]);
    publish();
    if (r == 0) issue(tmem + 64, sbase + kGH, 2048, sbase + kGW2T, 1024, 64, 4, false, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    // dZ1 = dH1 * mask1 -> EA rows 64..127
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      tmem_ld16(lane_addr + 64 + q * 16, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int o = q * 16 + i;
        const float d = ((mask1 >> o) & 1ull) ? v[i] : 0.f;
        warp_add(d, acc + kAB1 + o);
        *reinterpret_cast<__nv_bfloat16*>(sm + kGEA + kmajor_offset(64 + o, r, 128)) = __float2bfloat16_rn(d);
      }
    }
    publish();
    if (r == 0) issue(tmem + 128, sbase + kGEA, 2048, sbase + kGEB, 1280, 80, 8, done_tiles > 0, &mbar);
    if (!(ok = await(&mbar, phase))) break;
    ++done_tiles;
  }
  if (!ok) {
    if (threadIdx.x == 0) atomicOr(status, (unsigned)DEV_TC_TIMEOUT);
    mbar_wait(&mbar, phase, kWaitTries);
  } else if (done_tiles > 0) {
    // DW: rows 0..63 cols 0..63 = dW2, rows 64..127 cols 64..79 = dW1
    float v[16];
    if (r < 64) {  // warps 0 and 1
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        tmem_ld16(lane_addr + 128 + q * 16, v);
#pragma unroll
        for (int i = 0; i < 16; ++i) atomicAdd(grad + kMlpOffW2 + r * kMlpH + q * 16 + i, v[i]);
      }
    } else {  // warps 2 and 3
      tmem_ld16(lane_addr + 128 + 64, v);
#pragma unroll
      for (int i = 0; i < 16; ++i) atomicAdd(grad + kMlpOffW1 + (r - 64) * kMlpF + i, v[i]);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < 64; i += blockDim.x) {
      atomicAdd(grad + kMlpOffW3 + i, acc[kAW3 + i]);
      atomicAdd(grad + kMlpOffB1 + i, acc[kAB1 + i]);
      atomicAdd(grad + kMlpOffB2 + i, acc[kAB2 + i]);
    }
    if (threadIdx.x == 0) {
      atomicAdd(grad + kMlpOffB3, acc[kAB3]);
      atomicAdd(loss, acc[kALoss]);
    }
  }
  fence_before_sync();
  __syncthreads();
  fence_after_sync();
  if (warp == 0) tmem_dealloc(tmem, kGradTmemCols);
}

__global__ void k_mlp_adam(float* __restrict__ w, float* __restrict__ m1, float* __restrict__ m2,
                           float* __restrict__ g, float lr, float beta1, float beta2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kMlpParams) return;
  const float gi = g[i];
  const float a = beta1 * m1[i] + (1.f - beta1) * gi;
  const float b = beta2 * m2[i] + (1.f - beta2) * gi * gi;
  m1[i] = a;
  m2[i] = b;
  w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  g[i] = 0.f;
}

__global__ void __launch_bounds__(256) k_est_metrics(const uint32_t* __restrict__ est,
                                                     const uint32_t* __restrict__ truth, MlpRowInputs in, uint64_t n,
                                                     NumPolicy pol, uint32_t min_products, double* __restrict__ acc) {
  double rel = 0.0, cnt = 0.0, mis = 0.0, under = 0.0;
  for (uint64_t r = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t t = truth[r], e = est[r], p = in.prod[r];
    if (p <= min_products && min_products != 0) continue;
    if (t > 0) {
      rel += fabs((double)e - (double)t) / (double)t;
      cnt += 1.0;
    }
    under += e < t ? 1.0 : 0.0;
    const uint64_t span = p ? (uint64_t)in.hi[r] - in.lo[r] + 1 : 0;
    mis += num_bin_for(e, p, span, pol) != num_bin_for(t, p, span, pol) ? 1.0 : 0.0;
  }
  for (int o = 16; o > 0; o >>= 1) {
    rel += __shfl_xor_sync(0xFFFFFFFFu, rel, o);
    cnt += __shfl_xor_sync(0xFFFFFFFFu, cnt, o);
    mis += __shfl_xor_sync(0xFFFFFFFFu, mis, o);
    under += __shfl_xor_sync(0xFFFFFFFFu, under, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(acc, rel);
    atomicAdd(acc + 1, cnt);
    atomicAdd(acc + 2, mis);
    atomicAdd(acc + 3, under);
  }
}

int persistent_grid(uint64_t n, int per_sm, int num_sms) {
  const uint64_t tiles = (n + kMlpTile - 1) / kMlpTile;
  const uint64_t cap = (uint64_t)per_sm * (uint64_t)num_sms;
  return (int)(tiles < cap ? (tiles ? tiles : 1) : cap);
}

}  // namespace

void configure_mlp_attributes() {
  cudaFuncSetAttribute(k_mlp_infer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
  cudaFuncSetAttribute(k_mlp_infer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kFwdSmem);
  cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, kGradSmem);
}

void launch_mlp_features(const MlpRowInputs& in, uint64_t n, float* feat, cudaStream_t s) {
  if (n == 0) return;
  const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148ull * 16);
  k_mlp_features<<<(unsigned)blocks, 256, 0, s>>>(in, n, feat);
}

int launch_mlp_forward(const MlpModel& m, const float* feat, uint64_t n, float* pred, unsigned* status, int num_sms,
                       cudaStream_t s) {
  if (n == 0) return 0;
  k_mlp_infer<false><<<persistent_grid(n, 4, num_sms), 128, kFwdSmem, s>>>(m, MlpRowInputs(), feat, n, 0, nullptr,
                                                                           nullptr, pred, status);
  return 1;
}

int launch_mlp_estimate(const MlpModel& m, const MlpRowInputs& in, uint64_t n, uint32_t esc_max, uint32_t* est,
                        uint32_t* est_raw, unsigned* status, int num_sms, cudaStream_t s) {
  if (n == 0) return 0;
  k_mlp_infer<true><<<persistent_grid(n, 4, num_sms), 128, kFwdSmem, s>>>(m, in, nullptr, n, esc_max, est, est_raw,
                                                                          nullptr, status);
  return 1;
}

int launch_mlp_grad(const MlpModel& m, const float* feat, const float* target, uint64_t n, float batch, float* grad,
                    float* loss, unsigned* status, int num_sms, cudaStream_t s) {
  if (n == 0) return 0;
  k_mlp_grad<<<persistent_grid(n, 2, num_sms), 128, kGradSmem, s>>>(m, feat, target, n, 1.f / batch, grad, loss,
                                                                    status);
  return 1;
}

void launch_mlp_adam(float* params, float* m1, float* m2, float* grad, int step, float lr, float beta1, float beta2,
                     float eps, cudaStream_t s) {
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  k_mlp_adam<<<(kMlpParams + 255) / 256, 256, 0, s>>>(params, m1, m2, grad, lr, beta1, beta2, eps, c1, c2);
}

void launch_est_metrics(const uint32_t* est, const uint32_t* truth, const MlpRowInputs& in, uint64_t n,
                        const NumPolicy& pol, uint32_t min_products, double* acc, cudaStream_t s) {
  if (n == 0) return;
  const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, 148ull * 8);
  k_est_metrics<<<(unsigned)blocks, 256, 0, s>>>(est, truth, in, n, pol, min_products, acc);
}

}  // namespace ocean
