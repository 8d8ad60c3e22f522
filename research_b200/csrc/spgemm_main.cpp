// `spgemm` driver with the reference's command line (src/main.cu:11-83):
//   spgemm <A.hicsr> [B.hicsr] [config.json]
// A second argument ending in ".mtxd_.hicsr" or not ending in ".json" is B;
// without B, C = A·A. The config file takes the reference's JSON keys. Runs
// warmup_iters + bench_iters multiplies, copies C to the host, optionally
// compares with `ground_truth_file` (reference compare semantics) and writes the
// stats JSON to `stats_output_file` when `output_stats` is set.
#include <cstdio>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>

#include "config.h"
#include "ocean_spgemm.hpp"

static bool ends_with(const std::string& s, const std::string& suf) {
  return s.size() >= suf.size() && s.compare(s.size() - suf.size(), suf.size(), suf) == 0;
}

int main(int argc, char** argv) {
  if (argc < 2 || argc > 4) {
    std::cerr << "Usage: " << argv[0] << " <matrix_file> [matrix_b_file] [config_file]" << std::endl;
    std::cerr << "Matrices should end with .mtxd_.hicsr, and config should end with .json." << std::endl;
    return 1;
  }
  std::string a_file = argv[1], b_file = argv[1], cfg_file;
  if (argc == 3) {
    const std::string arg2 = argv[2];
    if (ends_with(arg2, ".mtxd_.hicsr")) b_file = arg2;
    else if (ends_with(arg2, ".json")) cfg_file = arg2;
    else b_file = arg2;
  } else if (argc == 4) {
    b_file = argv[2];
    cfg_file = argv[3];
  }
  try {
    std::string cfg_text;
    if (!cfg_file.empty()) {
      std::ifstream f(cfg_file);
      if (!f.good()) {
        std::cerr << "could not open config file " << cfg_file << std::endl;
        return 1;
      }
      std::stringstream ss;
      ss << f.rdbuf();
      cfg_text = ss.str();
    }
    const ocean::Config c = ocean::Config::from_json_text(cfg_text);
    std::cout << "trying to load csr file \"" << a_file << "\"\n";
    auto A = somespgemm::loadCSR(a_file.c_str());
    std::cout << "successfully loaded: \"" << a_file << "\"\n";
    auto B = A;
    if (b_file != a_file) {
      std::cout << "trying to load csr file \"" << b_file << "\"\n";
      B = somespgemm::loadCSR(b_file.c_str());
      std::cout << "successfully loaded: \"" << b_file << "\"\n";
    }
    if (A->cols != B->rows) {
      std::cerr << "Incompatible matrix dimensions!" << std::endl;
      return 1;
    }
    somespgemm::Config cfg;
    cfg.warmup_iters = c.warmup_iters;
    cfg.bench_iters = c.bench_iters;
    cfg.track_stage_times = c.track_stage_times;
    cfg.use_estimation_workflow = c.use_estimation_workflow;
    cfg.use_ultrasparse_workflow = c.use_ultrasparse_workflow;
    cfg.use_assist_information = c.use_assist_information;
    cfg.use_hybrid_accumulator = c.use_hybrid_accumulator;
    cfg.use_indirect_sort = c.use_indirect_sort;
    cfg.use_fat_workflow = c.use_fat_workflow;
    cfg.hll_numeric_malloc_expansion_coe = c.hll_numeric_malloc_expansion_coe;
    cfg.estimation_input_expansion_threshold = c.estimation_input_expansion_threshold;
    cfg.estimation_output_compaction_threshold = c.estimation_output_compaction_threshold;
    cfg.use_segmented_workflow = c.use_segmented_workflow;
    cfg.segmentation_grid_max = c.segmentation_grid_max;
    cfg.segmentation_hot_threshold_k = c.segmentation_hot_threshold_k;
    cfg.segmentation_min_segment_rows = c.segmentation_min_segment_rows;
    cfg.segmentation_cc_max_iters = c.segmentation_cc_max_iters;
    // keys of this library pass through unchanged
    if (!cfg_text.empty()) {
      const size_t lb = cfg_text.find('{'), rb = cfg_text.rfind('}');
      if (lb != std::string::npos && rb != std::string::npos && rb > lb + 1) {
        std::string inner = cfg_text.substr(lb + 1, rb - lb - 1);
        if (inner.find_first_not_of(" \t\r\n") != std::string::npos) cfg.extra_json = inner;
      }
    }
    somespgemm::SpGEMM spgemm(cfg);
    auto dA = std::make_shared<somespgemm::cuCSR>(*A);
    auto dB = (B == A) ? dA : std::make_shared<somespgemm::cuCSR>(*B);
    auto result = spgemm.run(dA, dB);
    std::cout << "Average SpGEMM time over " << c.bench_iters << " iters: " << spgemm.average_ms() << " ms\n";
    somespgemm::CSR host = result->download();
    if (c.check_correctness) {
      auto truth = somespgemm::loadCSR(c.ground_truth_file.c_str());
      const size_t n = somespgemm::compare(host, *truth, c.compare_relative_error, c.compare_autofail_relative_error);
      std::cout << n << " / " << host.nnz << " elements have relative error greater than " << c.compare_relative_error
                << "\nComparison completed" << std::endl;
    }
    if (c.output_stats) {
      std::cout << "Writing to " << c.stats_output_file << std::endl;
      std::ofstream o(c.stats_output_file);
      o << spgemm.get_stats() << "\n";
    }
  } catch (const std::exception& e) {
    std::cerr << "error: " << e.what() << std::endl;
    return 1;
  }
  return 0;
}
