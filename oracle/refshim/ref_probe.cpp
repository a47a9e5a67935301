// Probe harness around the reference's own C++ objects (test infrastructure
// only; linked with the reference's sources by oracle/ref.mk into
// oracle/_ref/libtcref.so).  It drives the reference through its public C++
// API -- Dataset::from_dense / compute_bins (src/core/dataset.cpp:50,176),
// Booster::train (src/boosting/booster.cpp:47), SymmetricTree::build
// (src/tree/symmetric_tree.cpp:34), Booster::save_binary
// (src/boosting/booster.cpp:1049) and the predict family
// (src/boosting/booster.cpp:899-945) -- and exposes plain C entry points so
// the tests and the CPU baseline can call it through ctypes.
//
// Nothing here changes the reference's arithmetic: every number it returns is
// computed by the reference's own code.
#include <chrono>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <exception>
#include <algorithm>
#include <memory>
#include <numeric>
#include <sstream>
#include <string>
#include <vector>

#include "turbocat/turbocat.hpp"

using namespace turbocat;

namespace {

thread_local std::string g_err;

struct Params {
  int32_t loss;            // 0 logloss, 1 mse, 2 focal, 3 softmax cross-entropy
  int32_t n_classes;       // 2 for binary / regression
  int32_t n_estimators;
  int32_t max_depth;
  int32_t max_bins;
  int32_t min_samples_leaf;
  float learning_rate;
  float lambda_l2;
  float lambda_l1;
  float min_child_weight;
  float min_split_gain;
  float max_delta_step;
  int32_t regular;         // 1: regular (depth-wise) trees instead of symmetric ones
};

Config make_config(const Params& p) {
  Config cfg;
  if (p.loss == 1) {
    cfg = Config::regression();
  } else if (p.loss == 3) {
    cfg = Config::multiclass_classification(static_cast<uint32_t>(p.n_classes));
  } else {
    cfg = Config::binary_classification();
    if (p.loss == 2) cfg.loss.loss_type = LossType::RobustFocal;
  }
  cfg.boosting.n_estimators = static_cast<uint32_t>(p.n_estimators);
  cfg.boosting.learning_rate = p.learning_rate;
  cfg.boosting.subsample = 1.0f;
  cfg.boosting.colsample_bytree = 1.0f;
  cfg.boosting.use_goss = false;
  cfg.tree.max_depth = static_cast<uint16_t>(p.max_depth);
  cfg.tree.max_bins = static_cast<uint16_t>(p.max_bins);
  cfg.tree.lambda_l2 = p.lambda_l2;
  cfg.tree.lambda_l1 = p.lambda_l1;
  cfg.tree.min_child_weight = p.min_child_weight;
  cfg.tree.min_samples_leaf = static_cast<uint32_t>(p.min_samples_leaf);
  cfg.tree.min_split_gain = p.min_split_gain;
  cfg.tree.max_delta_step = p.max_delta_step;
  cfg.tree.use_symmetric = p.regular == 0;
  cfg.verbosity = 0;
  return cfg;
}

void copy_bins(const Dataset& ds, uint8_t* bins_out, float* edges_out, uint16_t* n_edges_out) {
  const Index n = ds.n_samples();
  const FeatureIndex f = ds.n_features();
  if (bins_out) {
    for (FeatureIndex j = 0; j < f; ++j) {
      std::memcpy(bins_out + static_cast<size_t>(j) * n, ds.binned().column(j), n);
    }
  }
  if (edges_out || n_edges_out) {
    const auto& edges = ds.bin_edges();
    for (FeatureIndex j = 0; j < f; ++j) {
      const size_t m = edges[j].size();
      if (n_edges_out) n_edges_out[j] = static_cast<uint16_t>(m);
      if (edges_out) {
        for (size_t k = 0; k < m && k < 255; ++k) edges_out[static_cast<size_t>(j) * 255 + k] = edges[j][k];
      }
    }
  }
}

int fail(const std::exception& e) {
  g_err = e.what();
  return -1;
}

}  // namespace

extern "C" {

const char* tcref_last_error() { return g_err.c_str(); }

void tcref_free(void* p) { std::free(p); }

// Quantile binning only (Dataset::from_dense + compute_bins).
int tcref_bin(const float* X, uint32_t n, uint16_t f, int32_t max_bins, uint8_t* bins_out,
              float* edges_out, uint16_t* n_edges_out) {
  try {
    Dataset ds;
    ds.from_dense(X, n, f, nullptr);
    Config cfg;
    cfg.tree.max_bins = static_cast<uint16_t>(max_bins);
    ds.compute_bins(cfg);
    copy_bins(ds, bins_out, edges_out, n_edges_out);
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Full reference fit (binary / regression: Booster::train with symmetric
// trees).  Optionally records the per-iteration gradients and hessians the
// reference used (read from the Dataset in the training callback, after the
// iteration's tree was built) and returns the TCAT v3 model bytes.
int tcref_fit(const float* X, uint32_t n, uint16_t f, const float* y, const Params* p,
              uint8_t* bins_out, float* edges_out, uint16_t* n_edges_out, float* grad_trace,
              float* hess_trace, float* train_pred_out, char** model_bytes, size_t* model_len) {
  try {
    Config cfg = make_config(*p);
    Dataset ds;
    ds.from_dense(X, n, f, y);
    ds.compute_bins(cfg);
    copy_bins(ds, bins_out, edges_out, n_edges_out);
    Booster booster(cfg);
    TrainingCallback cb = nullptr;
    if (grad_trace || hess_trace) {
      cb = [&](const TrainingInfo& info) {
        const size_t off = static_cast<size_t>(info.iteration) * n;
        if (grad_trace) std::memcpy(grad_trace + off, ds.gradients(), n * sizeof(float));
        if (hess_trace) std::memcpy(hess_trace + off, ds.hessians(), n * sizeof(float));
        return true;
      };
    }
    booster.train(ds, nullptr, cb);
    if (train_pred_out) {
      booster.predict_raw_nobinning_fast(X, n, f, train_pred_out);
    }
    std::ostringstream os;
    booster.save_binary(os);
    const std::string s = os.str();
    *model_len = s.size();
    *model_bytes = static_cast<char*>(std::malloc(s.size()));
    std::memcpy(*model_bytes, s.data(), s.size());
    return static_cast<int>(booster.n_trees());
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Load TCAT bytes with Booster::load_binary and predict through the
// reference's no-binning fast path.  kind: 0 raw, 1 probability (sigmoid).
int tcref_predict(const char* model_bytes, size_t model_len, const float* X, uint32_t n, uint16_t f,
                  int32_t kind, float* out) {
  try {
    std::istringstream is(std::string(model_bytes, model_len));
    Booster b = Booster::load_binary(is);
    if (kind == 1) {
      b.predict_proba_nobinning_fast(X, n, f, out);
    } else {
      b.predict_raw_nobinning_fast(X, n, f, out);
    }
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// One SymmetricTree::build on caller-given gradients / hessians (teacher
// forcing).  Outputs splits (feature, bin, float threshold, gain) per level
// and 2^depth leaf values; returns the depth.
int tcref_build_tree(const float* X, uint32_t n, uint16_t f, const float* grad, const float* hess,
                     const Params* p, uint16_t* split_feature, uint8_t* split_bin,
                     float* split_threshold, float* split_gain, float* leaf_values) {
  try {
    Config cfg = make_config(*p);
    Dataset ds;
    ds.from_dense(X, n, f, nullptr);
    ds.compute_bins(cfg);
    ds.set_gradients_copy(grad, hess, n);
    std::vector<Index> rows(n);
    std::iota(rows.begin(), rows.end(), 0u);
    auto hb = HistogramBuilder::create(cfg.device);
    SymmetricTree tree(cfg.tree);
    tree.build(ds, rows, *hb);
    const auto& sp = tree.splits();
    for (size_t d = 0; d < sp.size(); ++d) {
      split_feature[d] = sp[d].feature;
      split_bin[d] = sp[d].threshold;
      split_threshold[d] = sp[d].float_threshold;
      split_gain[d] = sp[d].gain;
    }
    const auto& lv = tree.leaf_values();
    std::memcpy(leaf_values, lv.data(), lv.size() * sizeof(float));
    return static_cast<int>(tree.depth());
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Composed symmetric multiclass fit.  The reference's own multiclass loop
// (Booster::train_multiclass, src/boosting/booster.cpp:1263-1395) builds
// regular Trees, and its symmetric multiclass predict reads an empty
// ensemble; this harness keeps that loop's structure -- softmax gradients for
// all classes (CrossEntropyLoss::compute_multiclass_gradients), then one tree
// per class on that class's gradient column, prediction update
// preds[:,k] += lr * tree -- with SymmetricTree substituted for Tree.
// Outputs per tree (iteration-major, class-minor): depth, splits, leaves
// (padded to 2^max_depth) and the final raw train predictions [n x K].
int tcref_fit_multiclass(const float* X, uint32_t n, uint16_t f, const float* y, const Params* p,
                         int32_t* depth_out, uint16_t* split_feature, uint8_t* split_bin,
                         float* split_threshold, float* leaf_values, float* train_pred_out) {
  try {
    Config cfg = make_config(*p);
    const uint32_t K = static_cast<uint32_t>(p->n_classes);
    const uint32_t D = static_cast<uint32_t>(p->max_depth);
    Dataset ds;
    ds.from_dense(X, n, f, y);
    ds.compute_bins(cfg);
    CrossEntropyLoss ce(K);
    std::vector<Float> preds(static_cast<size_t>(n) * K, 0.0f);
    std::vector<Float> g(static_cast<size_t>(n) * K), h(static_cast<size_t>(n) * K);
    std::vector<Index> rows(n);
    std::iota(rows.begin(), rows.end(), 0u);
    auto hb = HistogramBuilder::create(cfg.device);
    const Float lr = cfg.boosting.learning_rate;
    std::vector<Float> tree_out(n);
    size_t t = 0;
    for (int it = 0; it < p->n_estimators; ++it) {
      ce.compute_multiclass_gradients(ds.labels().data(), preds.data(), g.data(), h.data(), n);
      for (uint32_t k = 0; k < K; ++k, ++t) {
        AlignedVector<Float> cg(n), ch(n);
        for (Index i = 0; i < n; ++i) {
          cg[i] = g[static_cast<size_t>(i) * K + k];
          ch[i] = h[static_cast<size_t>(i) * K + k];
        }
        ds.set_gradients(std::move(cg), std::move(ch));
        SymmetricTree tree(cfg.tree);
        tree.build(ds, rows, *hb);
        tree.predict_batch(ds, tree_out.data());
        for (Index i = 0; i < n; ++i) preds[static_cast<size_t>(i) * K + k] += lr * tree_out[i];
        depth_out[t] = tree.depth();
        const auto& sp = tree.splits();
        for (size_t d = 0; d < sp.size(); ++d) {
          split_feature[t * D + d] = sp[d].feature;
          split_bin[t * D + d] = sp[d].threshold;
          split_threshold[t * D + d] = sp[d].float_threshold;
        }
        const auto& lv = tree.leaf_values();
        for (size_t l = 0; l < lv.size(); ++l) leaf_values[t * (size_t(1) << D) + l] = lv[l];
      }
    }
    if (train_pred_out) std::memcpy(train_pred_out, preds.data(), preds.size() * sizeof(Float));
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Timed reference fit for the CPU baseline: Dataset::from_dense +
// compute_bins, then Booster::train with the configuration's n_estimators,
// stopped through the training callback (which the reference's loop honours
// with a break, src/boosting/booster.cpp:393-406) after `max_trees` trees or
// once `max_seconds` have passed.  setup_s[0] = seconds of from_dense +
// compute_bins; tree_end_s[i] = seconds from the start to the end of tree i
// (Booster::train's own set-up falls inside tree 0).  Returns the number of
// trees built.
int tcref_fit_timed(const float* X, uint32_t n, uint16_t f, const float* y, const Params* p, int32_t max_trees,
                    double max_seconds, double* setup_s, double* tree_end_s) {
  try {
    using clk = std::chrono::steady_clock;
    const auto t0 = clk::now();
    Config cfg = make_config(*p);
    Dataset ds;
    ds.from_dense(X, n, f, y);
    ds.compute_bins(cfg);
    setup_s[0] = std::chrono::duration<double>(clk::now() - t0).count();
    Booster booster(cfg);
    int32_t done = 0;
    TrainingCallback cb = [&](const TrainingInfo&) {
      const double t = std::chrono::duration<double>(clk::now() - t0).count();
      if (done < max_trees) tree_end_s[done] = t;
      ++done;
      return done < max_trees && t < max_seconds;
    };
    booster.train(ds, nullptr, cb);
    return done < max_trees ? done : max_trees;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Categorical target statistics (Dataset::from_dense with cat_features,
// compute_target_statistics, compute_bins; python/bindings.cpp:207-224).
// method: 0 ordered, 1 cross-validated.  enc_out [n_cat][n] = the per-row
// encodings the reference drew (get_sample_categorical_encoding), bins /
// edges as tcref_bin, and per categorical feature its global table
// (target_stats) sorted by category: tab_len[c] entries at tab_keys /
// tab_vals + c * tab_cap.  With fit != 0 it then trains on those bins
// (Booster::train, symmetric trees) and returns the TCAT bytes.
int tcref_cat_ts(const float* X, uint32_t n, uint16_t f, const float* y, const uint16_t* cats, int32_t n_cat,
                 int32_t method, const Params* p, int32_t fit, float* enc_out, uint8_t* bins_out,
                 float* edges_out, uint16_t* n_edges_out, uint32_t* tab_keys, float* tab_vals, uint32_t* tab_len,
                 uint32_t tab_cap, char** model_bytes, size_t* model_len) {
  try {
    Config cfg = make_config(*p);
    cfg.categorical.method = method == 1 ? CategoricalConfig::EncodingMethod::CrossValidatedTS
                                         : CategoricalConfig::EncodingMethod::TargetStatistics;
    std::vector<FeatureIndex> cf(cats, cats + n_cat);
    Dataset ds;
    ds.from_dense(X, n, f, y, nullptr, cf);
    ds.compute_target_statistics(cfg);
    for (int32_t c = 0; c < n_cat; ++c) {
      for (uint32_t i = 0; i < n; ++i)
        enc_out[static_cast<size_t>(c) * n + i] = ds.get_sample_categorical_encoding(cats[c], i);
      std::vector<std::pair<Index, Float>> t(ds.target_stats()[cats[c]].begin(), ds.target_stats()[cats[c]].end());
      std::sort(t.begin(), t.end());
      tab_len[c] = static_cast<uint32_t>(t.size());
      for (size_t k = 0; k < t.size() && k < tab_cap; ++k) {
        tab_keys[static_cast<size_t>(c) * tab_cap + k] = t[k].first;
        tab_vals[static_cast<size_t>(c) * tab_cap + k] = t[k].second;
      }
    }
    ds.compute_bins(cfg);
    copy_bins(ds, bins_out, edges_out, n_edges_out);
    if (!fit) return 0;
    Booster booster(cfg);
    booster.train(ds, nullptr, nullptr);
    std::ostringstream os;
    booster.save_binary(os);
    const std::string s = os.str();
    *model_len = s.size();
    *model_bytes = static_cast<char*>(std::malloc(s.size()));
    std::memcpy(*model_bytes, s.data(), s.size());
    return static_cast<int>(booster.n_trees());
  } catch (const std::exception& e) {
    return fail(e);
  }
}

// Seconds of the reference's compute_target_statistics alone on one dataset
// (from_dense with the categorical features first, untimed); the CPU
// baseline of the categorical encoding.
int tcref_cat_ts_timed(const float* X, uint32_t n, uint16_t f, const float* y, const uint16_t* cats,
                       int32_t n_cat, int32_t method, double* seconds) {
  try {
    Config cfg = Config::binary_classification();
    cfg.categorical.method = method == 1 ? CategoricalConfig::EncodingMethod::CrossValidatedTS
                                         : CategoricalConfig::EncodingMethod::TargetStatistics;
    std::vector<FeatureIndex> cf(cats, cats + n_cat);
    Dataset ds;
    ds.from_dense(X, n, f, y, nullptr, cf);
    const auto t0 = std::chrono::steady_clock::now();
    ds.compute_target_statistics(cfg);
    *seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return 0;
  } catch (const std::exception& e) {
    return fail(e);
  }
}

}  // extern "C"
