// ocean_spgemm.hpp — C++ compatibility layer with the reference's class names,
// implemented over the C ABI in ocean.h.
//
// Mirrors (paths inside the reference project):
//   somespgemm::Config            include/Utils.h:17-108  (public fields, same names/defaults)
//   somespgemm::CSR / cuCSR       include/CSR.h:16-51     (rows, cols, nnz, data, row_offsets, col_ids)
//   somespgemm::SpGEMM            kernels/SpGEMM.cuh:209-343 (SpGEMM(const Config&), run(A, B), get_stats())
//   somespgemm::loadCSR           src/CSR.cpp:119-152     (binary .hicsr reader)
//   somespgemm::compare           src/CSR.cpp:252-335     (exact structure, relative value error)
// Differences: get_stats() returns the JSON text instead of an nlohmann::json
// object; results whose nnz needs 64-bit row offsets carry them in
// cuCSR::row_offsets64 (the reference's uint32 offsets cannot hold them); errors
// are thrown as std::runtime_error carrying ocean_last_error().
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "ocean.h"

namespace somespgemm {

typedef uint32_t index_t;
typedef double data_t;

struct Config {
  bool use_estimation_workflow = true;
  bool use_ultrasparse_workflow = true;
  bool use_fat_workflow = true;
  bool use_assist_information = true;
  bool use_hybrid_accumulator = true;
  bool use_indirect_sort = true;
  bool use_segmented_workflow = false;
  int segmentation_grid_max = 256;
  double segmentation_hot_threshold_k = 2.0;
  int segmentation_min_segment_rows = 1024;
  int segmentation_cc_max_iters = 32;
  int estimation_input_expansion_threshold = 8;
  int estimation_output_compaction_threshold = 8;
  double hll_numeric_malloc_expansion_coe = 1.3;
  bool track_stage_times = false;
  bool check_correctness = false;
  bool output_stats = false;
  double compare_relative_error = 1e-6;
  double compare_autofail_relative_error = 1e-4;
  std::string ground_truth_file;
  std::string stats_output_file;
  int warmup_iters = 10, bench_iters = 10;
  bool print_info = false;
  bool print_memory = false;
  std::string extra_json;  // further keys of this library, e.g. "\"output_rowptr_bits\": 64"

  std::string to_json() const {
    std::ostringstream o;
    o.precision(17);
    auto b = [](bool x) { return x ? "true" : "false"; };
    o << "{\"use_estimation_workflow\": " << b(use_estimation_workflow)
      << ", \"use_ultrasparse_workflow\": " << b(use_ultrasparse_workflow)
      << ", \"use_fat_workflow\": " << b(use_fat_workflow)
      << ", \"use_assist_information\": " << b(use_assist_information)
      << ", \"use_hybrid_accumulator\": " << b(use_hybrid_accumulator)
      << ", \"use_indirect_sort\": " << b(use_indirect_sort)
      << ", \"use_segmented_workflow\": " << b(use_segmented_workflow)
      << ", \"segmentation_grid_max\": " << segmentation_grid_max
      << ", \"segmentation_hot_threshold_k\": " << segmentation_hot_threshold_k
      << ", \"segmentation_min_segment_rows\": " << segmentation_min_segment_rows
      << ", \"segmentation_cc_max_iters\": " << segmentation_cc_max_iters
      << ", \"estimation_input_expansion_threshold\": " << estimation_input_expansion_threshold
      << ", \"estimation_output_compaction_threshold\": " << estimation_output_compaction_threshold
      << ", \"hll_numeric_malloc_expansion_coe\": " << hll_numeric_malloc_expansion_coe
      << ", \"track_stage_time\": " << b(track_stage_times) << ", \"warmup_iters\": " << warmup_iters
      << ", \"bench_iters\": " << bench_iters;
    if (!extra_json.empty()) o << ", " << extra_json;
    o << "}";
    return o.str();
  }
};

struct CSR {
  size_t rows = 0, cols = 0, nnz = 0;
  std::vector<data_t> data;
  std::vector<index_t> row_offsets;
  std::vector<uint64_t> row_offsets64;  // filled instead of row_offsets when nnz >= 2^32
  std::vector<index_t> col_ids;
};

// Device CSR. Inputs: caller-owned device pointers (owned=false). Results of
// SpGEMM::run own their memory and release it in the destructor, like the
// reference's cuCSR (src/CSR.cpp:211-214).
struct cuCSR {
  size_t rows = 0, cols = 0, nnz = 0;
  data_t* data = nullptr;
  index_t* row_offsets = nullptr;
  uint64_t* row_offsets64 = nullptr;
  index_t* col_ids = nullptr;
  ocean_csr result{};
  bool owned = false;

  cuCSR() = default;
  explicit cuCSR(const CSR& h) { upload(h); }
  cuCSR(const cuCSR&) = delete;
  cuCSR& operator=(const cuCSR&) = delete;
  ~cuCSR() { reset(); }

  void upload(const CSR& h) {
    reset();
    rows = h.rows, cols = h.cols, nnz = h.nnz;
    if (!h.row_offsets64.empty()) {
      cudaMalloc((void**)&row_offsets64, (rows + 1) * 8);
      cudaMemcpy(row_offsets64, h.row_offsets64.data(), (rows + 1) * 8, cudaMemcpyHostToDevice);
    } else {
      cudaMalloc((void**)&row_offsets, (rows + 1) * 4);
      cudaMemcpy(row_offsets, h.row_offsets.data(), (rows + 1) * 4, cudaMemcpyHostToDevice);
    }
    cudaMalloc((void**)&col_ids, (nnz ? nnz : 1) * 4);
    cudaMalloc((void**)&data, (nnz ? nnz : 1) * 8);
    if (nnz) {
      cudaMemcpy(col_ids, h.col_ids.data(), nnz * 4, cudaMemcpyHostToDevice);
      cudaMemcpy(data, h.data.data(), nnz * 8, cudaMemcpyHostToDevice);
    }
    owned = false;
    uploaded_ = true;
  }

  void reset() {
    if (owned) ocean_csr_free(&result, nullptr);
    if (uploaded_) {
      cudaFree(row_offsets);
      cudaFree(row_offsets64);
      cudaFree(col_ids);
      cudaFree(data);
    }
    owned = uploaded_ = false;
    data = nullptr;
    row_offsets = nullptr;
    row_offsets64 = nullptr;
    col_ids = nullptr;
    rows = cols = nnz = 0;
  }

  ocean_csr_view view() const {
    ocean_csr_view v;
    v.rows = rows, v.cols = cols, v.nnz = nnz;
    v.rowptr = row_offsets64 ? (const void*)row_offsets64 : (const void*)row_offsets;
    v.rowptr_bits = row_offsets64 ? 64 : 32;
    v.col = col_ids;
    v.val = data;
    return v;
  }

  // Copies to host (reference: convert(CSR&, const cuCSR&), src/CSR.cpp:243-250).
  CSR download() const {
    CSR h;
    h.rows = rows, h.cols = cols, h.nnz = nnz;
    h.col_ids.resize(nnz);
    h.data.resize(nnz);
    if (row_offsets64) {
      h.row_offsets64.resize(rows + 1);
      cudaMemcpy(h.row_offsets64.data(), row_offsets64, (rows + 1) * 8, cudaMemcpyDeviceToHost);
    } else {
      h.row_offsets.resize(rows + 1);
      cudaMemcpy(h.row_offsets.data(), row_offsets, (rows + 1) * 4, cudaMemcpyDeviceToHost);
    }
    if (nnz) {
      cudaMemcpy(h.col_ids.data(), col_ids, nnz * 4, cudaMemcpyDeviceToHost);
      cudaMemcpy(h.data.data(), data, nnz * 8, cudaMemcpyDeviceToHost);
    }
    return h;
  }

 private:
  bool uploaded_ = false;
};

class SpGEMM {
 public:
  explicit SpGEMM(const Config& config) : config_(config) {
    if (ocean_create(&h_, config.to_json().c_str()) != OCEAN_OK)
      throw std::runtime_error(std::string("ocean_create: ") + ocean_last_error());
  }
  SpGEMM(const SpGEMM&) = delete;
  SpGEMM& operator=(const SpGEMM&) = delete;
  ~SpGEMM() { ocean_destroy(h_); }

  // warmup_iters + bench_iters multiplies, like the reference's run()
  // (kernels/SpGEMM.cuh:226-320); returns the last C, owned by the result.
  std::shared_ptr<cuCSR> run(std::shared_ptr<cuCSR> A, std::shared_ptr<cuCSR> B) {
    const ocean_csr_view av = A->view(), bv = B->view();
    auto C = std::make_shared<cuCSR>();
    double total_ms = 0.0;
    const int iters = config_.warmup_iters + config_.bench_iters;
    for (int i = 0; i < (iters > 0 ? iters : 1); ++i) {
      C->reset();
      ocean_csr out{};
      if (ocean_spgemm(h_, &av, &bv, &out, nullptr) != OCEAN_OK)
        throw std::runtime_error(std::string("ocean_spgemm: ") + ocean_last_error());
      C->result = out;
      C->owned = true;
      C->rows = out.rows, C->cols = out.cols, C->nnz = out.nnz;
      C->data = out.val;
      C->col_ids = out.col;
      if (out.rowptr_bits == 64) C->row_offsets64 = (uint64_t*)out.rowptr;
      else C->row_offsets = (index_t*)out.rowptr;
      if (i >= config_.warmup_iters) total_ms += ocean_stage_ms(h_, "total");
    }
    last_avg_ms_ = config_.bench_iters > 0 ? total_ms / config_.bench_iters : 0.0;
    return C;
  }

  // Stats of the last multiply as JSON text (reference keys).
  std::string get_stats() const {
    size_t need = 0;
    ocean_stats_json(h_, nullptr, 0, &need);
    std::string s(need, '\0');
    ocean_stats_json(h_, &s[0], need, &need);
    if (!s.empty() && s.back() == '\0') s.pop_back();
    return s;
  }

  double average_ms() const { return last_avg_ms_; }

 private:
  Config config_;
  ocean_handle* h_ = nullptr;
  double last_avg_ms_ = 0.0;
};

// Binary .hicsr reader (reference: loadCSR, src/CSR.cpp:119-152).
inline std::shared_ptr<CSR> loadCSR(const char* file) {
  std::ifstream f(file, std::ios::binary);
  if (!f.is_open()) throw std::runtime_error(std::string("could not open \"") + file + "\"");
  char header[80];
  f.read(header, sizeof header);
  if (!f.good()) throw std::runtime_error("Could not read CSR header");
  static const char magic[9] = {'H', 'i', 1, 'C', 'o', 'm', 'p', 's', 'd'};
  for (int i = 0; i < 9; ++i)
    if (header[i] != magic[i]) throw std::runtime_error("File does not appear to be a CSR Matrix");
  uint64_t fields[8];
  std::memcpy(fields, header + 16, sizeof fields);
  char state[16];
  f.read(state, sizeof state);
  if (!f.good()) throw std::runtime_error("Could not read CompressedMatrix state");
  if (fields[0] != sizeof(data_t)) throw std::runtime_error("File does not contain a CSR matrix with matching type");
  auto m = std::make_shared<CSR>();
  m->rows = fields[5], m->cols = fields[6], m->nnz = fields[7];
  m->data.resize(m->nnz);
  m->col_ids.resize(m->nnz);
  m->row_offsets.resize(m->rows + 1);
  f.read(reinterpret_cast<char*>(m->data.data()), m->nnz * sizeof(data_t));
  f.read(reinterpret_cast<char*>(m->col_ids.data()), m->nnz * sizeof(index_t));
  f.read(reinterpret_cast<char*>(m->row_offsets.data()), (m->rows + 1) * sizeof(index_t));
  if (!f.good()) throw std::runtime_error("Could not read CSR matrix data");
  return m;
}

// Reference comparison semantics (src/CSR.cpp:252-335): dimensions, row
// offsets [0, rows) and column ids exact; values by relative error, counted
// above `rel` and fatal above `fatal`. Returns the count above `rel`.
inline size_t compare(const CSR& a, const CSR& b, double rel = 1e-6, double fatal = 1e-4) {
  if (a.rows != b.rows || a.cols != b.cols || a.nnz != b.nnz)
    throw std::runtime_error("Matrices have different dimensions");
  auto off = [](const CSR& m, size_t i) -> uint64_t {
    return m.row_offsets64.empty() ? (uint64_t)m.row_offsets[i] : m.row_offsets64[i];
  };
  for (size_t i = 0; i < a.rows; ++i)
    if (off(a, i) != off(b, i)) throw std::runtime_error("Matrices have different row offsets");
  for (size_t i = 0; i < a.nnz; ++i)
    if (a.col_ids[i] != b.col_ids[i]) throw std::runtime_error("Matrices have different column IDs");
  size_t errors = 0;
  for (size_t i = 0; i < a.nnz; ++i) {
    const double x = a.data[i], y = b.data[i];
    const double d = std::fabs(x - y), m = std::fmax(std::fabs(x), std::fabs(y));
    const double r = m > 0 ? d / m : 0.0;
    if (r > rel) ++errors;
    if (r > fatal) throw std::runtime_error("Matrices have different data");
  }
  return errors;
}

}  // namespace somespgemm
