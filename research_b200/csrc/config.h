// Runtime configuration: the reference's JSON keys with the reference's defaults
// (include/Utils.h:17-108, src/Utils.cpp:8-37), plus this library's own keys.
// A small JSON reader is included; it keeps the top-level scalar members of an
// object and skips nested values and unknown keys, like the reference's
// assign_if_present (include/Utils.h:111-115).
#pragma once
#include <cctype>
#include <cstdlib>
#include <map>
#include <stdexcept>
#include <string>

namespace ocean {

struct JsonScalar {
  enum Kind { kNull, kBool, kNumber, kString } kind = kNull;
  bool b = false;
  double num = 0.0;
  std::string str;
};

class FlatJson {
 public:
  // Parses `text`; throws std::invalid_argument on malformed input.
  static std::map<std::string, JsonScalar> parse(const std::string& text) {
    FlatJson p(text);
    std::map<std::string, JsonScalar> out;
    p.ws();
    if (p.i_ == p.s_.size()) return out;  // empty document = defaults
    p.expect('{');
    p.ws();
    if (p.peek() == '}') {
      ++p.i_;
      return out;
    }
    for (;;) {
      p.ws();
      std::string key = p.string_lit();
      p.ws();
      p.expect(':');
      p.ws();
      JsonScalar v;
      if (p.value(&v)) out[key] = v;
      p.ws();
      const char c = p.next();
      if (c == '}') break;
      if (c != ',') throw std::invalid_argument("config JSON: expected ',' or '}'");
    }
    return out;
  }

 private:
  explicit FlatJson(const std::string& s) : s_(s) {}
  const std::string& s_;
  size_t i_ = 0;
  char peek() const { return i_ < s_.size() ? s_[i_] : '\0'; }
  char next() {
    if (i_ >= s_.size()) throw std::invalid_argument("config JSON: unexpected end");
    return s_[i_++];
  }
  void ws() {
    while (i_ < s_.size() && std::isspace((unsigned char)s_[i_])) ++i_;
  }
  void expect(char c) {
    if (next() != c) throw std::invalid_argument(std::string("config JSON: expected '") + c + "'");
  }
  std::string string_lit() {
    expect('"');
    std::string r;
    for (;;) {
      char c = next();
      if (c == '"') break;
      if (c == '\\') {
        char e = next();
        switch (e) {
          case 'n': r += '\n'; break;
          case 't': r += '\t'; break;
          case 'r': r += '\r'; break;
          case 'b': r += '\b'; break;
          case 'f': r += '\f'; break;
          case 'u': {
            unsigned code = 0;
            for (int k = 0; k < 4; ++k) {
              const char h = next();
              code = code * 16 + (std::isdigit((unsigned char)h) ? h - '0' : (std::tolower(h) - 'a' + 10));
            }
            r += code < 128 ? (char)code : '?';
            break;
          }
          default: r += e;
        }
      } else {
        r += c;
      }
    }
    return r;
  }
  // Returns true for a scalar, false for a nested object/array (skipped).
  bool value(JsonScalar* v) {
    const char c = peek();
    if (c == '"') {
      v->kind = JsonScalar::kString;
      v->str = string_lit();
      return true;
    }
    if (c == '{' || c == '[') {
      skip_nested();
      return false;
    }
    if (s_.compare(i_, 4, "true") == 0) {
      i_ += 4;
      v->kind = JsonScalar::kBool;
      v->b = true;
      return true;
    }
    if (s_.compare(i_, 5, "false") == 0) {
      i_ += 5;
      v->kind = JsonScalar::kBool;
      v->b = false;
      return true;
    }
    if (s_.compare(i_, 4, "null") == 0) {
      i_ += 4;
      v->kind = JsonScalar::kNull;
      return true;
    }
    const char* start = s_.c_str() + i_;
    char* end = nullptr;
    const double d = std::strtod(start, &end);
    if (end == start) throw std::invalid_argument("config JSON: bad value");
    i_ += (size_t)(end - start);
    v->kind = JsonScalar::kNumber;
    v->num = d;
    return true;
  }
  void skip_nested() {
    int depth = 0;
    do {
      const char c = next();
      if (c == '"') {
        --i_;
        string_lit();
        continue;
      }
      if (c == '{' || c == '[') ++depth;
      if (c == '}' || c == ']') --depth;
    } while (depth > 0);
  }
};

struct Config {
  // reference keys (src/Utils.cpp:9-36) with reference defaults (include/Utils.h)
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
  bool use_estimation_workflow = true;
  bool use_ultrasparse_workflow = true;
  bool use_assist_information = true;
  bool use_hybrid_accumulator = true;
  bool use_indirect_sort = true;
  bool use_fat_workflow = true;
  double hll_numeric_malloc_expansion_coe = 1.3;
  int estimation_input_expansion_threshold = 8;
  int estimation_output_compaction_threshold = 8;
  bool use_segmented_workflow = false;
  int segmentation_grid_max = 256;
  double segmentation_hot_threshold_k = 2.0;
  int segmentation_min_segment_rows = 1024;
  int segmentation_cc_max_iters = 32;
  // code-only reference defaults (include/Utils.h:36-60)
  int usparse_avg_product_threshold = 64;
  double hll_sample_rate = 0.03;
  int hll_sample_min_rows = 648;
  int hll_sample_max_rows = 10800;
  int hll_higher_precision_expansion_threshold = 48;
  int fat_ratio = 100;
  // this library's keys
  int output_rowptr_bits = 0;     // 0: 32 when nnz(C) < 2^32, else 64
  int esc_max_products = 128;     // rows with at most this many products use the register ESC classes
  int force_sym_bin = -1;         // testing: put every non-empty row in one symbolic class
  int force_num_bin = -1;         // testing: put every non-empty row in one numeric class
  bool sync_on_return = true;     // check device status before returning
  double bitmap_cache_fraction = 0.25;  // share of free device memory the saved row bitmaps may use
  int small_problem_nnz = 1 << 20;      // A with at most this many entries: no read-back after analysis
  int spin_wait_us = 2000;              // poll the stream this long before a blocking synchronize
  int force_workflow = -1;              // -1 auto; 0 precise, 1 estimation (HLL), 2 ultra-sparse, 3 fat
  double estimate_scale = 1.0;          // multiplies the HLL expansion (testing: < 1 forces overflows)
  bool use_learned_estimator = false;   // estimation workflow: per-row sizes from the MLP instead of HLL
  std::string learned_estimator_weights;  // weights file; empty: the built-in trained network
  double learned_margin_scale = 1.0;    // multiplies the network's log2 preallocation margin
  bool estimator_metrics = false;       // after an estimated multiply: error of the estimates vs exact counts
  double hash_s_max_scale = 1.0;        // (0, 1]: fill limit of the small hash tables relative to the default
  double bitmap_words_scale = 1.0;      // > 0: scales the column-span limits under which mid rows use bitmaps
  bool prefer_direct_hash = true;       // mid rows whose column span fits a hash table use it (direct slots)
  bool numeric_windows = false;         // exact numeric bitmap class: shared-memory value windows (k_num_window)
  bool fused_ultrasparse = false;       // ultra-sparse inputs (<= 256 products per row): one fused launch
  // host-buffer multiplies (ocean_spgemm_host) of at least this many products
  // run the numeric phase in row chunks of equal products and copy each
  // finished chunk of C to the host while the next one computes (0: off)
  int host_pipeline_chunks = 8;
  double host_pipeline_min_products = 67108864.0;
  bool batch_autotune = false;          // batched plans: search the class policy on the batch before capturing
  std::string autotune_cache_file;      // JSON-lines cache of tuned policies (key: GPU name + batch features); "" off
  // segment-driven dispatch: rows of each spy-plot segment class take that
  // class's policy (index = SegClass: sparse_uniform, dense, power_law, banded);
  // unset fields inherit the global policy above
  bool use_segment_dispatch = false;
  int seg_esc_max_products[4] = {-1, -1, -1, -1};
  double seg_hash_s_max_scale[4] = {0, 0, 0, 0};
  double seg_bitmap_words_scale[4] = {0, 0, 0, 0};
  int seg_prefer_direct_hash[4] = {-1, -1, -1, -1};
  int seg_force_sym_bin[4] = {-2, -2, -2, -2};
  int seg_force_num_bin[4] = {-2, -2, -2, -2};

  static Config from_json_text(const std::string& text) {
    Config c;
    const auto m = FlatJson::parse(text);
    auto getb = [&](const char* k, bool& f) {
      auto it = m.find(k);
      if (it == m.end()) return;
      if (it->second.kind == JsonScalar::kBool) f = it->second.b;
      else if (it->second.kind == JsonScalar::kNumber) f = it->second.num != 0.0;
      else throw std::invalid_argument(std::string("config key '") + k + "' must be a boolean");
    };
    auto getd = [&](const char* k, double& f) {
      auto it = m.find(k);
      if (it == m.end()) return;
      if (it->second.kind != JsonScalar::kNumber)
        throw std::invalid_argument(std::string("config key '") + k + "' must be a number");
      f = it->second.num;
    };
    auto geti = [&](const char* k, int& f) {
      double d = f;
      getd(k, d);
      f = (int)d;
    };
    auto gets = [&](const char* k, std::string& f) {
      auto it = m.find(k);
      if (it == m.end()) return;
      if (it->second.kind != JsonScalar::kString)
        throw std::invalid_argument(std::string("config key '") + k + "' must be a string");
      f = it->second.str;
    };
    getb("track_stage_time", c.track_stage_times);
    getb("check_correctness", c.check_correctness);
    getb("output_stats", c.output_stats);
    getd("compare_relative_error", c.compare_relative_error);
    getd("compare_autofail_relative_error", c.compare_autofail_relative_error);
    gets("ground_truth_file", c.ground_truth_file);
    gets("stats_output_file", c.stats_output_file);
    geti("warmup_iters", c.warmup_iters);
    geti("bench_iters", c.bench_iters);
    getb("print_info", c.print_info);
    getb("print_memory", c.print_memory);
    getb("use_estimation_workflow", c.use_estimation_workflow);
    getb("use_ultrasparse_workflow", c.use_ultrasparse_workflow);
    getb("use_assist_information", c.use_assist_information);
    getb("use_hybrid_accumulator", c.use_hybrid_accumulator);
    getb("use_indirect_sort", c.use_indirect_sort);
    getb("use_fat_workflow", c.use_fat_workflow);
    getd("hll_numeric_malloc_expansion_coe", c.hll_numeric_malloc_expansion_coe);
    geti("estimation_input_expansion_threshold", c.estimation_input_expansion_threshold);
    geti("estimation_output_compaction_threshold", c.estimation_output_compaction_threshold);
    getb("use_segmented_workflow", c.use_segmented_workflow);
    geti("segmentation_grid_max", c.segmentation_grid_max);
    getd("segmentation_hot_threshold_k", c.segmentation_hot_threshold_k);
    geti("segmentation_min_segment_rows", c.segmentation_min_segment_rows);
    geti("segmentation_cc_max_iters", c.segmentation_cc_max_iters);
    geti("output_rowptr_bits", c.output_rowptr_bits);
    geti("esc_max_products", c.esc_max_products);
    geti("force_sym_bin", c.force_sym_bin);
    geti("force_num_bin", c.force_num_bin);
    getb("sync_on_return", c.sync_on_return);
    getd("bitmap_cache_fraction", c.bitmap_cache_fraction);
    geti("small_problem_nnz", c.small_problem_nnz);
    geti("spin_wait_us", c.spin_wait_us);
    geti("force_workflow", c.force_workflow);
    geti("fat_ratio", c.fat_ratio);
    getd("estimate_scale", c.estimate_scale);
    getb("use_learned_estimator", c.use_learned_estimator);
    gets("learned_estimator_weights", c.learned_estimator_weights);
    getd("learned_margin_scale", c.learned_margin_scale);
    getb("estimator_metrics", c.estimator_metrics);
    getd("hash_s_max_scale", c.hash_s_max_scale);
    getd("bitmap_words_scale", c.bitmap_words_scale);
    getb("prefer_direct_hash", c.prefer_direct_hash);
    getb("numeric_windows", c.numeric_windows);
    getb("fused_ultrasparse", c.fused_ultrasparse);
    geti("host_pipeline_chunks", c.host_pipeline_chunks);
    getd("host_pipeline_min_products", c.host_pipeline_min_products);
    getb("batch_autotune", c.batch_autotune);
    gets("autotune_cache_file", c.autotune_cache_file);
    getb("use_segment_dispatch", c.use_segment_dispatch);
    static const char* kSegKey[4] = {"sparse_uniform", "dense", "power_law", "banded"};
    for (int k = 0; k < 4; ++k) {
      const std::string p = std::string("segment_") + kSegKey[k] + "_";
      geti((p + "esc_max_products").c_str(), c.seg_esc_max_products[k]);
      getd((p + "hash_s_max_scale").c_str(), c.seg_hash_s_max_scale[k]);
      getd((p + "bitmap_words_scale").c_str(), c.seg_bitmap_words_scale[k]);
      bool direct = c.seg_prefer_direct_hash[k] > 0;
      const bool had = m.count(p + "prefer_direct_hash") > 0;
      getb((p + "prefer_direct_hash").c_str(), direct);
      if (had) c.seg_prefer_direct_hash[k] = direct ? 1 : 0;
      geti((p + "force_sym_bin").c_str(), c.seg_force_sym_bin[k]);
      geti((p + "force_num_bin").c_str(), c.seg_force_num_bin[k]);
      if (c.seg_esc_max_products[k] < -1 || c.seg_esc_max_products[k] > 128)
        throw std::invalid_argument(p + "esc_max_products must be in [0, 128]");
      if (c.seg_hash_s_max_scale[k] < 0.0 || c.seg_hash_s_max_scale[k] > 1.0)
        throw std::invalid_argument(p + "hash_s_max_scale must be in (0, 1]");
      if (c.seg_bitmap_words_scale[k] < 0.0 || c.seg_bitmap_words_scale[k] > 64.0)
        throw std::invalid_argument(p + "bitmap_words_scale must be in (0, 64]");
      if (c.seg_force_sym_bin[k] < -2 || c.seg_force_sym_bin[k] > 6 || c.seg_force_num_bin[k] < -2 ||
          c.seg_force_num_bin[k] > 6)
        throw std::invalid_argument(p + "force_sym_bin / force_num_bin must be in [-1, 6]");
    }
    if (c.output_rowptr_bits != 0 && c.output_rowptr_bits != 32 && c.output_rowptr_bits != 64)
      throw std::invalid_argument("output_rowptr_bits must be 0, 32 or 64");
    if (c.force_workflow < -1 || c.force_workflow > 3)
      throw std::invalid_argument("force_workflow must be -1, 0, 1, 2 or 3");
    if (c.estimate_scale <= 0.0) throw std::invalid_argument("estimate_scale must be positive");
    if (c.bitmap_cache_fraction < 0.0 || c.bitmap_cache_fraction > 0.9)
      throw std::invalid_argument("bitmap_cache_fraction must be in [0, 0.9]");
    if (c.esc_max_products < 0 || c.esc_max_products > 128)
      throw std::invalid_argument("esc_max_products must be in [0, 128]");
    return c;
  }
};

}  // namespace ocean
