// Spy-plot segmentation of A (analysis only; its records go to the stats).
//
// Reference: kernels/Segmentation.cuh:75-683. Steps: tile-count density map of
// A's pattern (at most grid_max x grid_max tiles), hot tiles = density at least
// mean + k * stddev, 4-connected components of the hot tiles (label = smallest
// tile index of the component), the dominant label of every grid row, row bands
// by run-length encoding those labels (bands shorter than min_segment_rows join
// the previous band), then per band: products, A entries, row-length mean and
// variance, column span, longest rows, and a class (BANDED > DENSE >
// POWER_LAW > SPARSE_UNIFORM).
//
// B200 layout: the density map is counted in shared memory by one block per
// grid row; the threshold, all component iterations and the pointer jumping run
// inside single-block kernels (the reference syncs the host after every
// iteration). Component labels are updated Jacobi style (two label buffers),
// so the labels and the iteration count do not depend on thread timing; after
// convergence they equal the reference's (smallest tile index of the
// component). Ties of the dominant label go to the label whose slot
// (label * 2654435761 mod grid_w) comes first, then to the smaller label: the
// reference's table order when no two labels of the grid row share a slot.
// All floating-point formulas round every operation (no fused multiply-add),
// so a CPU restatement reproduces them bit for bit.
#include <algorithm>
#include <cmath>
#include <vector>

#include "kernels.h"

namespace ocean {
namespace {

constexpr uint32_t kNone = 0xFFFFFFFFu;

template <typename RP>
__global__ void __launch_bounds__(256) k_seg_density(Csr<RP> A, uint32_t grid_h, uint32_t grid_w, uint32_t tile_rows,
                                                     uint32_t tile_cols, uint32_t* __restrict__ density) {
  extern __shared__ unsigned hist[];
  const uint32_t tr = blockIdx.x;
  for (uint32_t i = threadIdx.x; i < grid_w; i += blockDim.x) hist[i] = 0u;
  __syncthreads();
  const uint64_t r0 = (uint64_t)tr * tile_rows;
  uint64_t r1 = r0 + tile_rows;
  if (tr == grid_h - 1 || r1 > A.rows) r1 = A.rows;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
  for (uint64_t r = r0 + warp; r < r1; r += nw) {
    const uint64_t e = A.row_end(r);
    for (uint64_t k = A.row_begin(r) + lane; k < e; k += 32) {
      uint32_t tc = A.col[k] / tile_cols;
      if (tc >= grid_w) tc = grid_w - 1;
      atomicAdd(&hist[tc], 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < grid_w; i += blockDim.x) density[(uint64_t)tr * grid_w + i] = hist[i];
}

// One block: mean and standard deviation of the tile counts, then the labels
// (hot tile: its own index; cold tile: none).
__global__ void __launch_bounds__(1024) k_seg_threshold(const uint32_t* __restrict__ density, uint32_t tiles,
                                                        double k, uint32_t* __restrict__ labels,
                                                        double* __restrict__ stats) {
  __shared__ unsigned long long s1[32], s2[32];
  __shared__ double s_thresh;
  unsigned long long a = 0, b = 0;
  for (uint32_t i = threadIdx.x; i < tiles; i += blockDim.x) {
    const unsigned long long d = density[i];
    a += d;
    b += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(kFull, a, o);
    b += __shfl_xor_sync(kFull, b, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s1[threadIdx.x >> 5] = a;
    s2[threadIdx.x >> 5] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long sa = 0, sb = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) sa += s1[i], sb += s2[i];
    const double mean = (double)sa / (double)tiles;
    double var = __dsub_rn((double)sb / (double)tiles, __dmul_rn(mean, mean));
    if (var < 0.0) var = 0.0;
    const double sd = sqrt(var);
    stats[0] = mean;
    stats[1] = sd;
    s_thresh = __dadd_rn(mean, __dmul_rn(k, sd));
  }
  __syncthreads();
  const double thresh = s_thresh;
  for (uint32_t i = threadIdx.x; i < tiles; i += blockDim.x)
    labels[i] = ((double)density[i] >= thresh && density[i] > 0u) ? i : kNone;
}

// One block: min-label propagation over 4-neighbours, Jacobi style (reads
// cur, writes nxt) until nothing changes or max_iters rounds, then up to 8
// pointer-jumping rounds (label <- label[label]). The result ends in `a`.
__global__ void __launch_bounds__(1024) k_seg_cc(uint32_t* __restrict__ a, uint32_t* __restrict__ b, uint32_t grid_h,
                                                 uint32_t grid_w, int max_iters, int* __restrict__ iters_out) {
  const uint32_t tiles = grid_h * grid_w;
  uint32_t* cur = a;
  uint32_t* nxt = b;
  int it = 0;
  for (; it < max_iters; ++it) {
    int changed = 0;
    for (uint32_t idx = threadIdx.x; idx < tiles; idx += blockDim.x) {
      const uint32_t my = cur[idx];
      uint32_t best = my;
      if (my != kNone) {
        const uint32_t x = idx % grid_w, y = idx / grid_w;
        if (x > 0) best = min(best, cur[idx - 1]);
        if (x + 1 < grid_w) best = min(best, cur[idx + 1]);
        if (y > 0) best = min(best, cur[idx - grid_w]);
        if (y + 1 < grid_h) best = min(best, cur[idx + grid_w]);
        changed |= best < my;
      }
      nxt[idx] = best;
    }
    const int any = __syncthreads_or(changed);
    uint32_t* t = cur;
    cur = nxt;
    nxt = t;
    if (!any) break;
  }
  for (int pj = 0; pj < 8; ++pj) {
    int changed = 0;
    for (uint32_t idx = threadIdx.x; idx < tiles; idx += blockDim.x) {
      const uint32_t l = cur[idx];
      const uint32_t p = l == kNone ? kNone : cur[l];
      changed |= p != l;
      nxt[idx] = p;
    }
    const int any = __syncthreads_or(changed);
    uint32_t* t = cur;
    cur = nxt;
    nxt = t;
    if (!any) break;
  }
  if (cur != a) {
    for (uint32_t idx = threadIdx.x; idx < tiles; idx += blockDim.x) a[idx] = cur[idx];
  }
  if (threadIdx.x == 0) *iters_out = it;
}

// One block per grid row: the most frequent hot label and the number of hot
// tiles. Order of the vote: count, then earlier slot, then smaller label.
__global__ void __launch_bounds__(256) k_seg_rowband(const uint32_t* __restrict__ labels, uint32_t grid_w,
                                                     uint32_t* __restrict__ band_label, uint32_t* __restrict__ band_hot) {
  extern __shared__ uint32_t row[];
  __shared__ unsigned long long s_best[8];
  __shared__ unsigned s_hot[8];
  const uint32_t y = blockIdx.x;
  for (uint32_t x = threadIdx.x; x < grid_w; x += blockDim.x) row[x] = labels[(uint64_t)y * grid_w + x];
  __syncthreads();
  unsigned long long best = 0;  // count << 45 | (4095 - slot) << 32 | (~label)
  unsigned hot = 0;
  for (uint32_t x = threadIdx.x; x < grid_w; x += blockDim.x) {
    const uint32_t l = row[x];
    if (l == kNone) continue;
    ++hot;
    unsigned c = 0;
    for (uint32_t z = 0; z < grid_w; ++z) c += row[z] == l;
    const uint32_t slot = (l * 2654435761u) % grid_w;
    const unsigned long long key =
        ((unsigned long long)c << 45) | ((unsigned long long)(4095u - slot) << 32) | (0xFFFFFFFFu - l);
    if (key > best) best = key;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long ob = __shfl_xor_sync(kFull, best, o);
    best = ob > best ? ob : best;
    hot += __shfl_xor_sync(kFull, hot, o);
  }
  if ((threadIdx.x & 31) == 0) {
    s_best[threadIdx.x >> 5] = best;
    s_hot[threadIdx.x >> 5] = hot;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long bk = 0;
    unsigned h = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
      bk = s_best[i] > bk ? s_best[i] : bk;
      h += s_hot[i];
    }
    band_label[y] = bk ? 0xFFFFFFFFu - (uint32_t)(bk & 0xFFFFFFFFull) : kNone;
    band_hot[y] = h;
  }
}

// One block per segment: reductions over its rows, then the class, in the
// reference's priority BANDED > DENSE > POWER_LAW > SPARSE_UNIFORM:
// banded if the column span is < 5% of B's columns and products / A entries
// >= the input-expansion threshold; dense if the mean products per row fill
// >= 25% of the span; power-law if the coefficient of variation of products
// per row is >= 1.5. Rows without products carry span (~0, 0) and so add
// nothing to it.
__global__ void __launch_bounds__(128) k_seg_classify(const uint32_t* __restrict__ seg_start,
                                                      const uint32_t* __restrict__ seg_end,
                                                      const uint32_t* __restrict__ prod,
                                                      const uint32_t* __restrict__ anz,
                                                      const uint32_t* __restrict__ maxb,
                                                      const uint32_t* __restrict__ lo, const uint32_t* __restrict__ hi,
                                                      uint32_t b_cols, int expansion_threshold,
                                                      SegRecord* __restrict__ out) {
  const uint32_t r0 = seg_start[blockIdx.x], r1 = seg_end[blockIdx.x];
  unsigned long long sp = 0, sa = 0, sq = 0;
  uint32_t mb = 0, ma = 0, cl = kNone, cr = 0;
  for (uint32_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) {
    const unsigned long long p = prod[r];
    sp += p;
    sq += p * p;
    sa += anz[r];
    ma = max(ma, anz[r]);
    mb = max(mb, maxb[r]);
    cl = min(cl, lo[r]);
    cr = max(cr, hi[r]);
  }
  __shared__ unsigned long long s_sp[4], s_sa[4], s_sq[4];
  __shared__ uint32_t s_mb[4], s_ma[4], s_cl[4], s_cr[4];
  for (int o = 16; o > 0; o >>= 1) {
    sp += __shfl_xor_sync(kFull, sp, o);
    sa += __shfl_xor_sync(kFull, sa, o);
    sq += __shfl_xor_sync(kFull, sq, o);
    mb = max(mb, __shfl_xor_sync(kFull, mb, o));
    ma = max(ma, __shfl_xor_sync(kFull, ma, o));
    cl = min(cl, __shfl_xor_sync(kFull, cl, o));
    cr = max(cr, __shfl_xor_sync(kFull, cr, o));
  }
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    s_sp[w] = sp, s_sa[w] = sa, s_sq[w] = sq, s_mb[w] = mb, s_ma[w] = ma, s_cl[w] = cl, s_cr[w] = cr;
  }
  __syncthreads();
  if (threadIdx.x != 0) return;
  for (int i = 1; i < 4; ++i) {
    sp += s_sp[i], sa += s_sa[i], sq += s_sq[i];
    mb = max(mb, s_mb[i]), ma = max(ma, s_ma[i]), cl = min(cl, s_cl[i]), cr = max(cr, s_cr[i]);
  }
  SegRecord rec;
  rec.row_start = r0;
  rec.row_end = r1;
  rec.row_count = r1 - r0;
  rec.col_left = cl == kNone ? 0u : cl;
  rec.col_right = cr;
  rec.sum_products = sp;
  rec.sum_a_nnz = sa;
  rec.max_b_row_len = mb;
  rec.max_a_row_len = ma;
  const double n = (double)rec.row_count;
  const double mean = rec.row_count > 0 ? (double)sp / n : 0.0;
  double var = 0.0;
  if (rec.row_count > 0) var = __dsub_rn((double)sq / n, __dmul_rn(mean, mean));
  if (var < 0.0) var = 0.0;
  const double cv = mean > 0.0 ? sqrt(var) / mean : 0.0;
  const double er = sa > 0 ? (double)sp / (double)sa : 0.0;
  const double span_ratio = b_cols > 0 ? (double)(rec.col_right + 1u - rec.col_left) / (double)b_cols : 0.0;
  const double density = span_ratio > 0.0 ? mean / __dmul_rn((double)b_cols, span_ratio) : 0.0;
  rec.mean_row_len = mean;
  rec.var_row_len = var;
  rec.local_er = er;
  uint32_t cls = SEG_SPARSE_UNIFORM;
  if (span_ratio > 0.0 && span_ratio < 0.05 && mean > 0.0 && er >= (double)expansion_threshold) cls = SEG_BANDED;
  else if (density >= 0.25) cls = SEG_DENSE;
  else if (cv >= 1.5) cls = SEG_POWER_LAW;
  rec.cls = cls;
  out[blockIdx.x] = rec;
}

}  // namespace

// Host driver (reference: kernels/Segmentation.cuh:386-673). Grid: at most
// grid_max (8..4096) tiles per side, tile_rows = ceil(rows / grid_h),
// tile_cols = ceil(B.cols / grid_w); A's column ids are binned by tile_cols
// like the reference does (clamped to the last tile column). Row bands are
// run-length encoded on the host; a band shorter than min_segment_rows joins
// the previous one. Synchronises `s` twice (bands, records).
template <typename RP>
cudaError_t run_segmentation(const Csr<RP>& A, uint64_t b_cols, const DevWork& w, int grid_max, double hot_k,
                             int min_segment_rows, int cc_max_iters, int expansion_threshold, cudaStream_t s,
                             SegmentationResult* out) {
  *out = SegmentationResult();
  if (A.rows == 0 || b_cols == 0) return cudaSuccess;
  const uint32_t gmax = (uint32_t)std::min(std::max(8, grid_max), 4096);
  const uint32_t grid_h = (uint32_t)std::min<uint64_t>(gmax, A.rows);
  const uint32_t grid_w = (uint32_t)std::min<uint64_t>(gmax, b_cols);
  const uint32_t tile_rows = (uint32_t)((A.rows + grid_h - 1) / grid_h);
  const uint32_t tile_cols = (uint32_t)((b_cols + grid_w - 1) / grid_w);
  const uint32_t tiles = grid_h * grid_w;
  out->grid_h = grid_h, out->grid_w = grid_w, out->tile_rows = tile_rows, out->tile_cols = tile_cols;

  // one scratch block: density, two label buffers, band labels/hot counts, stats, iterations
  const size_t off_lab = tiles * 4ull, off_lab2 = off_lab * 2, off_band = off_lab * 3,
               off_hot = off_band + grid_h * 4ull, off_stats = (off_hot + grid_h * 4ull + 15) & ~size_t(15),
               off_iter = off_stats + 16, bytes = off_iter + 16;
  char* scratch = nullptr;
  cudaError_t e = cudaMallocAsync((void**)&scratch, bytes, s);
  if (e != cudaSuccess) return e;
  uint32_t* density = (uint32_t*)scratch;
  uint32_t* labels = (uint32_t*)(scratch + off_lab);
  uint32_t* labels2 = (uint32_t*)(scratch + off_lab2);
  uint32_t* band_label = (uint32_t*)(scratch + off_band);
  uint32_t* band_hot = (uint32_t*)(scratch + off_hot);
  double* stats = (double*)(scratch + off_stats);
  int* iters = (int*)(scratch + off_iter);

  cudaEvent_t ev[5];
  for (auto& x : ev) cudaEventCreate(&x);
  cudaEventRecord(ev[0], s);
  k_seg_density<RP><<<grid_h, 256, grid_w * 4, s>>>(A, grid_h, grid_w, tile_rows, tile_cols, density);
  cudaEventRecord(ev[1], s);
  k_seg_threshold<<<1, 1024, 0, s>>>(density, tiles, hot_k, labels, stats);
  cudaEventRecord(ev[2], s);
  k_seg_cc<<<1, 1024, 0, s>>>(labels, labels2, grid_h, grid_w, std::max(0, cc_max_iters), iters);
  k_seg_rowband<<<grid_h, 256, grid_w * 4, s>>>(labels, grid_w, band_label, band_hot);
  cudaEventRecord(ev[3], s);
  std::vector<uint32_t> h_band(grid_h);
  double h_stats[2] = {0, 0};
  int h_iters = 0;
  cudaMemcpyAsync(h_band.data(), band_label, grid_h * 4ull, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(h_stats, stats, 16, cudaMemcpyDeviceToHost, s);
  cudaMemcpyAsync(&h_iters, iters, 4, cudaMemcpyDeviceToHost, s);
  e = cudaStreamSynchronize(s);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFreeAsync(scratch, s);
    for (auto& x : ev) cudaEventDestroy(x);
    return e;
  }
  out->density_mean = h_stats[0];
  out->density_stddev = h_stats[1];
  out->cc_iterations = h_iters;

  // row bands by run-length encoding of the grid-row labels (reference: kernels/Segmentation.cuh:527-563)
  struct Band {
    uint32_t start, end, label;
  };
  std::vector<Band> bands;
  uint32_t cur = h_band[0], cur_start = 0;
  for (uint32_t g = 1; g < grid_h; ++g) {
    if (h_band[g] != cur) {
      const Band b{cur_start * tile_rows, (uint32_t)std::min<uint64_t>(A.rows, (uint64_t)g * tile_rows), cur};
      if (b.end > b.start) bands.push_back(b);
      cur = h_band[g];
      cur_start = g;
    }
  }
  {
    const Band b{cur_start * tile_rows, (uint32_t)A.rows, cur};
    if (b.end > b.start) bands.push_back(b);
  }
  std::vector<Band> merged;
  const uint32_t min_rows = (uint32_t)std::max(1, min_segment_rows);
  for (const auto& b : bands) {
    if (!merged.empty() && b.end - b.start < min_rows) merged.back().end = b.end;
    else merged.push_back(b);
  }
  std::vector<uint32_t> uniq;
  for (const auto& b : merged)
    if (b.label != kNone && std::find(uniq.begin(), uniq.end(), b.label) == uniq.end()) uniq.push_back(b.label);
  out->num_components = (uint32_t)uniq.size();
  if (merged.empty()) merged.push_back(Band{0, (uint32_t)A.rows, kNone});

  const uint32_t nseg = (uint32_t)merged.size();
  std::vector<uint32_t> h_se(2 * (size_t)nseg);
  for (uint32_t i = 0; i < nseg; ++i) h_se[i] = merged[i].start, h_se[nseg + i] = merged[i].end;
  char* seg = nullptr;
  const size_t rec_off = (8ull * nseg + 15) & ~size_t(15);
  e = cudaMallocAsync((void**)&seg, rec_off + nseg * sizeof(SegRecord), s);
  if (e == cudaSuccess) {
    uint32_t* d_se = (uint32_t*)seg;
    SegRecord* d_rec = (SegRecord*)(seg + rec_off);
    cudaMemcpyAsync(d_se, h_se.data(), 8ull * nseg, cudaMemcpyHostToDevice, s);
    k_seg_classify<<<nseg, 128, 0, s>>>(d_se, d_se + nseg, w.prod, w.anz, w.maxb, w.lo, w.hi, (uint32_t)b_cols,
                                        expansion_threshold, d_rec);
    cudaEventRecord(ev[4], s);
    out->segments.resize(nseg);
    cudaMemcpyAsync(out->segments.data(), d_rec, nseg * sizeof(SegRecord), cudaMemcpyDeviceToHost, s);
    e = cudaStreamSynchronize(s);
    if (e == cudaSuccess) e = cudaGetLastError();
    cudaFreeAsync(seg, s);
  }
  if (e == cudaSuccess) {
    cudaEventElapsedTime(&out->time_density_ms, ev[0], ev[1]);
    cudaEventElapsedTime(&out->time_threshold_ms, ev[1], ev[2]);
    cudaEventElapsedTime(&out->time_cc_ms, ev[2], ev[3]);
    cudaEventElapsedTime(&out->time_classify_ms, ev[3], ev[4]);
  }
  cudaFreeAsync(scratch, s);
  for (auto& x : ev) cudaEventDestroy(x);
  return e;
}

template cudaError_t run_segmentation<uint32_t>(const Csr<uint32_t>&, uint64_t, const DevWork&, int, double, int, int,
                                                int, cudaStream_t, SegmentationResult*);
template cudaError_t run_segmentation<uint64_t>(const Csr<uint64_t>&, uint64_t, const DevWork&, int, double, int, int,
                                                int, cudaStream_t, SegmentationResult*);

const char* segment_class_name(uint32_t cls) {
  switch (cls) {
    case SEG_SPARSE_UNIFORM: return "SPARSE_UNIFORM";
    case SEG_DENSE: return "DENSE";
    case SEG_POWER_LAW: return "POWER_LAW";
    case SEG_BANDED: return "BANDED";
    default: return "UNKNOWN";
  }
}

}  // namespace ocean
