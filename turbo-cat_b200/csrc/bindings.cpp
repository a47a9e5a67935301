// pybind11 module `_turbocat`: the reference's Python-facing surface
// (python/bindings.cpp:37-1131 -- class names, constructor arguments with
// their defaults, method names, return types and error texts), with the
// implementation swapped for the device engine behind include/tcgpu.h.
//
// C++ host side: GpuBooster owns the device dataset and model and calls the
// C ABI; there is no CPU fallback -- without a usable sm_100 device every
// fit/predict raises.
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "tcgpu.h"

namespace py = pybind11;

namespace {

using FArray = py::array_t<float, py::array::c_style | py::array::forcecast>;

tc_ctx* g_ctx = nullptr;
std::mutex g_ctx_mu;

tc_ctx* device_context() {
  std::lock_guard<std::mutex> g(g_ctx_mu);
  if (!g_ctx) {
    int dev = 0;
    if (const char* e = std::getenv("TURBOCAT_DEVICE")) dev = std::atoi(e);
    const tc_status s = tc_ctx_create(dev, 0, &g_ctx);
    if (s != TC_OK) {
      g_ctx = nullptr;
      throw std::runtime_error("TurboCat B200 engine: no usable sm_100 CUDA device " + std::to_string(dev) +
                               " (status " + std::to_string((int)s) + ")");
    }
  }
  return g_ctx;
}

void check(tc_status s, tc_ctx* ctx) {
  if (s == TC_OK) return;
  const std::string msg = tc_last_error(ctx);
  if (s == TC_ERR_INVALID_ARG) throw std::invalid_argument(msg);
  throw std::runtime_error(msg);
}

struct ModelPtr {
  tc_model* m = nullptr;
  ~ModelPtr() { tc_model_destroy(m); }
};

struct DatasetPtr {
  tc_dataset* d = nullptr;
  ~DatasetPtr() { tc_dataset_destroy(d); }
};

// Categorical features of a fit and their encoding (python/bindings.cpp:106-116, 201-224).
struct CatSpec {
  std::vector<uint16_t> features;
  tc_cat_params params{TC_CAT_ORDERED, 1.0f, 5, 0};
};

// Host-side booster: the counterpart of turbocat::Booster for the symmetric path.
class GpuBooster {
 public:
  std::unique_ptr<ModelPtr> model;
  tc_model_info info{};
  tc_train_stats stats{};

  // With a validation set (Xv, yv, nv > 0) the fit follows Booster::train's
  // valid_data branch: validation loss every iteration, early stopping after
  // `es_rounds` iterations without improvement (src/boosting/booster.cpp:255-371).
  // With categorical features the training set's categorical columns are
  // replaced by their target statistics before binning (compute_target_statistics
  // before compute_bins, python/bindings.cpp:218-224); the training set is
  // kept, as the reference keeps train_data_, to encode the validation set and
  // the rows of the binned predict path (Dataset::apply_bins).
  std::unique_ptr<DatasetPtr> train_set;

  void fit(const float* X, uint32_t n, uint16_t f, const float* y, const tc_train_params& p,
           const float* Xv = nullptr, const float* yv = nullptr, uint32_t nv = 0, int es_rounds = 50,
           const CatSpec* cats = nullptr, bool regular = false) {
    tc_ctx* ctx = device_context();
    tc_dataset* ds = nullptr;
    tc_dataset* vds = nullptr;
    check(tc_dataset_upload(ctx, X, n, f, y, &ds), ctx);
    const bool keep = cats && !cats->features.empty();
    tc_status s = TC_OK;
    if (keep) s = tc_encode_categorical(ds, cats->features.data(), (uint16_t)cats->features.size(), &cats->params,
                                        nullptr);
    if (s == TC_OK) s = tc_quantize(ds, (uint16_t)p.max_bins, 1, nullptr, nullptr);
    tc_model* m = nullptr;
    if (s == TC_OK && nv == 0) s = regular ? tc_train_regular(ctx, ds, &p, &m, &stats) : tc_train(ctx, ds, &p, &m, &stats);
    if (s == TC_OK && nv > 0) {
      tc_trainer* tr = nullptr;
      s = tc_dataset_upload(ctx, Xv, nv, f, yv, &vds);
      if (s == TC_OK && keep) s = tc_apply_bins(vds, ds);  // valid_data->apply_bins(*train_data_)
      if (s == TC_OK) s = tc_trainer_create(ctx, ds, &p, &tr);
      if (s == TC_OK) s = tc_trainer_set_validation(tr, vds, es_rounds);
      if (s == TC_OK) s = tc_trainer_step(tr, p.n_estimators, 1);
      if (s == TC_OK) s = tc_trainer_model(tr, &m);
      if (s == TC_OK) s = tc_trainer_stats(tr, &stats);
      if (tr) tc_trainer_destroy(tr);
    }
    if (vds) tc_dataset_destroy(vds);
    if (keep && s == TC_OK) {
      train_set.reset(new DatasetPtr());
      train_set->d = ds;
    } else {
      tc_dataset_destroy(ds);
    }
    check(s, ctx);
    model.reset(new ModelPtr());
    model->m = m;
    tc_model_info_get(m, &info);
  }

  std::vector<float> predict(const float* X, uint32_t n, uint16_t f, int transform) const {
    tc_ctx* ctx = device_context();
    std::vector<float> out((size_t)n * info.n_classes);
    check(tc_predict(ctx, model->m, X, n, f, transform, out.data()), ctx);
    return out;
  }

  // The reference's binned predict path (Dataset::apply_bins against the
  // training set, then the tree walk; python/bindings.cpp:311-334): rows'
  // categorical columns take the training set's global encodings.
  std::vector<float> predict_binned(const float* X, uint32_t n, uint16_t f, int transform) const {
    if (!train_set) return predict(X, n, f, transform);
    tc_ctx* ctx = device_context();
    std::vector<float> out((size_t)n * info.n_classes);
    DatasetPtr t;
    check(tc_dataset_upload(ctx, X, n, f, nullptr, &t.d), ctx);
    check(tc_apply_bins(t.d, train_set->d), ctx);
    check(tc_predict_dataset(ctx, model->m, t.d, transform, out.data()), ctx);
    return out;
  }

  void save(const std::string& path) const {
    tc_ctx* ctx = device_context();
    size_t len = 0;
    check(tc_model_save_tcat(model->m, nullptr, &len), ctx);
    std::vector<uint8_t> buf(len);
    check(tc_model_save_tcat(model->m, buf.data(), &len), ctx);
    std::ofstream os(path, std::ios::binary);
    if (!os) throw std::runtime_error("Cannot open file for writing: " + path);
    os.write(reinterpret_cast<const char*>(buf.data()), (std::streamsize)len);
  }

  void load(const std::string& path) {
    tc_ctx* ctx = device_context();
    std::ifstream is(path, std::ios::binary);
    if (!is) throw std::runtime_error("Cannot open file for reading: " + path);
    std::vector<uint8_t> buf((std::istreambuf_iterator<char>(is)), std::istreambuf_iterator<char>());
    tc_model* m = nullptr;
    check(tc_model_load_tcat(ctx, buf.data(), buf.size(), &m), ctx);
    model.reset(new ModelPtr());
    model->m = m;
    tc_model_info_get(m, &info);
  }

  // SymmetricEnsemble::feature_importance + Booster::feature_importance
  // (src/tree/symmetric_tree.cpp:1175-1193, src/boosting/booster.cpp:951-974).
  void importance(std::vector<float>& gain, std::vector<float>& norm) const {
    const int T = info.n_trees, D = info.max_depth;
    std::vector<int32_t> depth(T);
    std::vector<uint16_t> feat((size_t)T * D);
    std::vector<float> g((size_t)T * D);
    tc_model_export(model->m, depth.data(), feat.data(), nullptr, nullptr, g.data(), nullptr, nullptr, nullptr,
                    nullptr);
    const size_t nf = std::max<size_t>(256, (size_t)info.n_features);
    gain.assign(nf, 0.0f);
    for (int t = 0; t < T; ++t) {
      std::vector<float> tree(nf, 0.0f);
      for (int d = 0; d < depth[t]; ++d) tree[feat[(size_t)t * D + d]] += g[(size_t)t * D + d];
      for (size_t i = 0; i < nf; ++i) gain[i] += tree[i];
    }
    float sum = 0.0f;
    for (float v : gain) sum += v;
    if (sum > 0) for (float& v : gain) v /= sum;
    norm.assign(nf, 0.0f);
    float s2 = 0.0f;
    for (float v : gain) s2 += v;
    if (s2 > 0) for (size_t i = 0; i < nf; ++i) norm[i] = gain[i] / s2;
  }

  // Per-tree summary (python/bindings.cpp:804-830): node and leaf counts,
  // the FP32 sum of the leaf values in leaf order and whether the tree is a
  // single leaf.  A symmetric tree of depth d has 2^d - 1 split nodes and 2^d
  // leaves.
  py::list tree_info() const {
    py::list trees;
    if (!model) return trees;
    const int T = info.n_trees, D = info.max_depth, L = 1 << D;
    std::vector<int32_t> depth(T);
    std::vector<float> lv((size_t)T * L);
    tc_model_export(model->m, depth.data(), nullptr, nullptr, nullptr, nullptr, lv.data(), nullptr, nullptr,
                    nullptr);
    for (int t = 0; t < T; ++t) {
      const int nl = 1 << depth[t];
      float sum = 0.0f;
      for (int l = 0; l < nl; ++l) sum += lv[(size_t)t * L + l];
      py::dict d;
      d["n_nodes"] = (size_t)(2 * nl - 1);
      d["n_leaves"] = (size_t)nl;
      d["leaf_sum"] = sum;
      d["is_single_leaf"] = depth[t] == 0;
      trees.append(d);
    }
    return trees;
  }

  // The model's bin edges (the training set's), for Dataset::apply_bins-style
  // host binning: bin = number of edges <= x (std::upper_bound), NaN -> 255
  // (src/core/dataset.cpp:336-379).
  void edges(std::vector<float>& e, std::vector<uint16_t>& ne) const {
    e.assign((size_t)info.n_features * 255, 0.0f);
    ne.assign(info.n_features, 0);
    tc_model_export(model->m, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, e.data(), ne.data());
  }
  static int host_bin(float x, const float* e, int m) {
    if (std::isnan(x)) return 255;
    return (int)(std::upper_bound(e, e + m, x) - e);
  }

  py::list dump() const {
    const int T = info.n_trees, D = info.max_depth, L = 1 << D;
    std::vector<int32_t> depth(T);
    std::vector<uint16_t> feat((size_t)T * D);
    std::vector<uint8_t> bin((size_t)T * D);
    std::vector<float> thr((size_t)T * D), g((size_t)T * D), lv((size_t)T * L), w(T);
    tc_model_export(model->m, depth.data(), feat.data(), bin.data(), thr.data(), g.data(), lv.data(), w.data(),
                    nullptr, nullptr);
    py::list trees;
    for (int t = 0; t < T; ++t) {
      py::dict d;
      d["weight"] = w[t];
      d["depth"] = depth[t];
      d["class"] = t % std::max(1, info.n_classes);
      py::list splits;
      for (int k = 0; k < depth[t]; ++k) {
        py::dict s;
        s["feature"] = (int)feat[(size_t)t * D + k];
        s["threshold"] = (int)bin[(size_t)t * D + k];
        s["float_threshold"] = thr[(size_t)t * D + k];
        s["gain"] = g[(size_t)t * D + k];
        splits.append(s);
      }
      d["splits"] = splits;
      d["leaf_values"] = std::vector<float>(lv.begin() + (size_t)t * L, lv.begin() + (size_t)t * L + (1 << depth[t]));
      trees.append(d);
    }
    return trees;
  }
};

tc_train_params base_params() {
  tc_train_params p{};
  p.loss = TC_LOSS_LOGLOSS;
  p.n_classes = 1;
  p.n_estimators = 500;
  p.max_depth = 6;
  p.max_bins = 255;
  p.min_samples_leaf = 1;
  p.learning_rate = 0.2f;
  p.lambda_l2 = 1.0f;
  p.min_child_weight = 1.0f;
  p.focal_gamma = 2.0f;   // LossConfig defaults, include/turbocat/config.hpp:108-110
  p.focal_alpha = 0.25f;
  p.batched = 1;
  return p;
}

void warn(const std::string& msg) {
  py::module_::import("warnings").attr("warn")(msg, py::module_::import("builtins").attr("UserWarning"), 2);
}

void check_2d(const FArray& X, const char* what) {
  if (X.ndim() != 2) throw std::runtime_error(std::string(what) + " must be 2-dimensional");
}

// ------------------------------------------------------------------ classifier

class TurboCatClassifier {
 public:
  TurboCatClassifier(int n_estimators, float learning_rate, int max_depth, int max_bins, float subsample,
                     float colsample_bytree, float min_child_weight, float lambda_l2, const std::string& loss,
                     bool use_goss, float goss_top_rate, float goss_other_rate, bool use_gradtree, bool use_symmetric,
                     bool use_ordered_boosting, const std::string& grow_policy, const std::string& mode,
                     int early_stopping_rounds, const std::string& early_stopping_metric,
                     const std::string& cat_encoding, bool auto_interactions, int max_interactions,
                     const std::string& interaction_method, int n_threads, int seed, int verbosity)
      : loss_(loss), mode_(mode), subsample_(subsample), colsample_(colsample_bytree), use_goss_(use_goss),
        use_gradtree_(use_gradtree), use_ordered_(use_ordered_boosting), auto_interactions_(auto_interactions),
        verbosity_(verbosity) {
    p_ = base_params();
    p_.n_estimators = n_estimators;
    p_.learning_rate = learning_rate;
    p_.max_depth = max_depth;
    p_.max_bins = max_bins;
    p_.min_child_weight = min_child_weight;
    p_.lambda_l2 = lambda_l2;
    (void)use_symmetric; (void)grow_policy;
    p_.use_goss = use_goss ? 1 : 0;  // python/bindings.cpp:76-78
    p_.goss_top_rate = goss_top_rate;
    p_.goss_other_rate = goss_other_rate;
    p_.subsample = subsample;
    p_.colsample_bytree = colsample_bytree;
    p_.seed = (uint64_t)(int64_t)seed;
    es_rounds_ = early_stopping_rounds;
    if (early_stopping_metric != "loss" && early_stopping_metric != "logloss")
      warn("early_stopping_metric '" + early_stopping_metric + "' is not on the device path; the validation "
           "loss is used (the reference's fallback for metrics it does not know)");
    // python/bindings.cpp:106-116: "cv" / "cross_validated", "onehot" / "one_hot", else ordered
    if (cat_encoding == "cv" || cat_encoding == "cross_validated") cat_.params.method = TC_CAT_CV;
    else if (cat_encoding == "onehot" || cat_encoding == "one_hot") onehot_ = true;
    cat_.params.seed = p_.seed;  // the reference draws the order from std::random_device
    (void)max_interactions;
    (void)interaction_method; (void)n_threads;
  }

  void fit(FArray X, FArray y, FArray X_val, FArray y_val, std::vector<int> cat_features) {
    check_2d(X, "X");
    if (y.ndim() != 1) throw std::runtime_error("y must be 1-dimensional");
    const uint32_t n = (uint32_t)X.shape(0);
    const uint16_t f = (uint16_t)X.shape(1);
    if ((size_t)y.shape(0) != n) throw std::runtime_error("X and y have different numbers of rows");
    if (colsample_ < 1.0f && verbosity_ > 1) warn("colsample_bytree has no effect on symmetric trees");
    if (use_gradtree_ || use_ordered_ || auto_interactions_)
      warn("use_gradtree / use_ordered_boosting / auto_interactions are not on the device path and are ignored");
    CatSpec cats = cat_;
    for (int c : cat_features) {
      if (c < 0 || c >= (int)f) throw std::invalid_argument("cat_features index out of range");
      cats.features.push_back((uint16_t)c);
    }
    if (!cats.features.empty() && onehot_)
      throw std::invalid_argument("cat_encoding='onehot' is not on the device path (target statistics: 'ordered', 'cv')");
    const bool has_val = X_val.size() > 0 && y_val.size() > 0;
    if (has_val) {
      check_2d(X_val, "X_val");
      if (X_val.shape(1) != X.shape(1)) throw std::invalid_argument("X_val must have as many features as X");
      if ((size_t)y_val.size() != (size_t)X_val.shape(0)) throw std::invalid_argument("y_val does not match X_val");
    }
    const float* yp = y.data();
    float mx = 0.0f;
    for (uint32_t i = 0; i < n; ++i) mx = std::max(mx, yp[i]);
    n_classes_ = (uint32_t)mx + 1;  // python/bindings.cpp:161-167
    tc_train_params p = p_;
    if (n_classes_ <= 2) {
      if (loss_ == "auto" || loss_ == "logloss" || loss_ == "binary_crossentropy") p.loss = TC_LOSS_LOGLOSS;
      else if (loss_ == "focal" || loss_ == "robust_focal") p.loss = TC_LOSS_FOCAL;
      else throw std::invalid_argument("loss '" + loss_ + "' is not on the device path (logloss, focal)");
      p.n_classes = 1;
    } else {
      p.loss = TC_LOSS_SOFTMAX;
      p.n_classes = (int)n_classes_;
    }
    // mode="small": regular (depth-wise) trees where the device builds them --
    // binary logloss on every row without a validation set or categorical
    // columns (tc_train_regular); otherwise symmetric trees
    bool regular = false;
    if (mode_ == "small") {
      regular = n_classes_ <= 2 && p.loss == TC_LOSS_LOGLOSS && p.subsample >= 1.0f && !p.use_goss && !has_val &&
                cats.features.empty();
      if (!regular)
        warn("mode='small' (regular trees) is on the device path for binary logloss with subsample=1.0, no GOSS, "
             "no validation set and no cat_features; building symmetric trees");
    }
    {
      py::gil_scoped_release nogil;
      booster_.reset(new GpuBooster());
      if (has_val)
        booster_->fit(X.data(), n, f, yp, p, X_val.data(), y_val.data(), (uint32_t)X_val.shape(0), es_rounds_,
                      &cats);
      else
        booster_->fit(X.data(), n, f, yp, p, nullptr, nullptr, 0, 50, &cats, regular);
    }
    n_features_ = f;
    is_fitted_ = true;
    if (verbosity_ > 0)
      py::print("[TurboCat-B200] trained", booster_->info.n_trees, "trees in", booster_->stats.seconds, "s (device)");
  }

  py::array_t<float> predict_proba(FArray X) {
    if (!is_fitted_) throw std::runtime_error("Model not fitted. Call fit() first.");
    check_2d(X, "X");
    const uint32_t n = (uint32_t)X.shape(0);
    const uint16_t f = (uint16_t)X.shape(1);
    const int K = booster_->info.n_classes;
    std::vector<float> out;
    {
      py::gil_scoped_release nogil;
      // binary: the no-binning path on the raw rows (categorical columns
      // compared as given); multiclass: the binned path, which encodes them
      // (python/bindings.cpp:297-334)
      out = K > 1 ? booster_->predict_binned(X.data(), n, f, TC_TRANSFORM_SOFTMAX)
                  : booster_->predict(X.data(), n, f, TC_TRANSFORM_SIGMOID);
    }
    if (K > 1) {
      py::array_t<float> r({(py::ssize_t)n, (py::ssize_t)K});
      std::memcpy(r.mutable_data(), out.data(), out.size() * sizeof(float));
      return r;
    }
    py::array_t<float> r({(py::ssize_t)n, (py::ssize_t)2});
    float* q = r.mutable_data();
    for (uint32_t i = 0; i < n; ++i) {
      q[2 * i] = 1.0f - out[i];  // python/bindings.cpp:377-381
      q[2 * i + 1] = out[i];
    }
    return r;
  }

  py::array_t<float> predict_proba_nobinning_fast(FArray X) { return predict_proba(X); }

  py::array_t<int> predict(FArray X) {
    auto proba = predict_proba(X);
    const py::ssize_t n = proba.shape(0), k = proba.shape(1);
    const float* p = proba.data();
    py::array_t<int> r(n);
    int* q = r.mutable_data();
    for (py::ssize_t i = 0; i < n; ++i) {
      if (k > 2) {
        int best = 0;
        float bp = p[i * k];
        for (py::ssize_t c = 1; c < k; ++c)
          if (p[i * k + c] > bp) { bp = p[i * k + c]; best = (int)c; }
        q[i] = best;
      } else {
        q[i] = p[i * 2 + 1] >= 0.5f ? 1 : 0;
      }
    }
    return r;
  }

  py::dict feature_importance() {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    std::vector<float> g, gn;
    booster_->importance(g, gn);
    py::dict d;
    d["gain"] = py::array_t<float>(g.size(), g.data());
    d["gain_normalized"] = py::array_t<float>(gn.size(), gn.data());
    return d;
  }

  void save(const std::string& path) {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    booster_->save(path);
  }

  void load(const std::string& path) {
    booster_.reset(new GpuBooster());
    booster_->load(path);
    n_classes_ = booster_->info.n_classes > 1 ? (uint32_t)booster_->info.n_classes : 2u;
    n_features_ = booster_->info.n_features;
    is_fitted_ = true;
  }

  py::dict get_params() const {
    py::dict d;
    d["n_estimators"] = p_.n_estimators;
    d["learning_rate"] = p_.learning_rate;
    d["max_depth"] = p_.max_depth;
    d["max_bins"] = p_.max_bins;
    d["subsample"] = subsample_;
    d["colsample_bytree"] = colsample_;
    d["lambda_l2"] = p_.lambda_l2;
    d["use_goss"] = use_goss_;
    d["use_gradtree"] = use_gradtree_;
    d["n_classes"] = n_classes_;
    return d;
  }

  py::list get_booster_dump() const {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    return booster_->dump();
  }
  float get_base_prediction() const {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    return booster_->info.base_prediction;
  }
  int get_n_features() const {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    return n_features_;
  }
  size_t n_trees() const { return booster_ ? (size_t)booster_->info.n_trees : 0; }
  uint32_t n_classes() const { return n_classes_; }
  double train_seconds() const { return booster_ ? booster_->stats.seconds : 0.0; }

 private:
  tc_train_params p_{};
  std::string loss_, mode_;
  float subsample_, colsample_;
  bool use_goss_, use_gradtree_, use_ordered_, auto_interactions_;
  int verbosity_;
  int es_rounds_ = 50;
  CatSpec cat_;
  bool onehot_ = false;
  std::unique_ptr<GpuBooster> booster_;
  uint32_t n_classes_ = 2;
  int n_features_ = 0;
  bool is_fitted_ = false;
};

// ------------------------------------------------------------------- regressor

class TurboCatRegressor {
 public:
  TurboCatRegressor(int n_estimators, float learning_rate, int max_depth, const std::string& loss,
                    const std::string& mode, float subsample, float colsample_bytree, bool use_goss,
                    float goss_top_rate, float goss_other_rate, int early_stopping_rounds, float lambda_l2,
                    float min_child_weight, int max_leaves, const std::string& grow_policy, int n_threads, int seed,
                    int verbosity)
      : mode_(mode), subsample_(subsample), use_goss_(use_goss), verbosity_(verbosity) {
    p_ = base_params();
    p_.loss = TC_LOSS_MSE;
    p_.n_estimators = n_estimators;
    p_.learning_rate = learning_rate;
    p_.max_depth = max_depth;
    p_.lambda_l2 = lambda_l2;
    p_.min_child_weight = min_child_weight;
    if (!(loss == "mse" || loss == "l2"))
      throw std::invalid_argument("loss '" + loss + "' is not on the device path (mse)");
    p_.subsample = subsample;
    p_.colsample_bytree = colsample_bytree;
    p_.seed = (uint64_t)(int64_t)seed;
    p_.use_goss = use_goss ? 1 : 0;  // python/bindings.cpp:570-572
    p_.goss_top_rate = goss_top_rate;
    p_.goss_other_rate = goss_other_rate;
    (void)early_stopping_rounds;
    (void)max_leaves; (void)grow_policy; (void)n_threads;
  }

  void fit(FArray X, FArray y) {
    check_2d(X, "X");
    const uint32_t n = (uint32_t)X.shape(0);
    const uint16_t f = (uint16_t)X.shape(1);
    if ((size_t)y.size() != n) throw std::runtime_error("X and y have different numbers of rows");
    if (mode_ == "small") warn("mode='small' (regular trees) is not on the device path; building symmetric trees");
    {
      py::gil_scoped_release nogil;
      booster_.reset(new GpuBooster());
      booster_->fit(X.data(), n, f, y.data(), p_);
    }
    n_features_ = f;
    is_fitted_ = true;
    train_X_ = X;  // a reference, not a copy: debug_predict compares against the training rows
    if (verbosity_ > 0)
      py::print("[TurboCat-B200] trained", booster_->info.n_trees, "trees in", booster_->stats.seconds, "s (device)");
  }

  py::list tree_info() const { return booster_ ? booster_->tree_info() : py::list(); }

  // Diagnostics of python/bindings.cpp:832-964 for the symmetric path: the
  // bins of the first rows of X under the training edges, the first tree's
  // path for the first samples (level by level: the level-order node index,
  // split, the sample's bin and the direction, right = bin != 255 && bin >
  // split bin), the bins of the first training rows and the value ranges of
  // the first features in the training set and in X.  Without the training
  // rows (a loaded model) the training entries are empty.
  py::dict debug_predict(FArray X) const {
    if (!is_fitted_ || !booster_) throw std::runtime_error("Model not fitted");
    check_2d(X, "X");
    const int64_t n = X.shape(0);
    const int f = (int)X.shape(1);
    if (f != booster_->info.n_features)
      throw std::runtime_error("X has " + std::to_string(f) + " features, the model " +
                               std::to_string(booster_->info.n_features));
    std::vector<float> e;
    std::vector<uint16_t> ne;
    booster_->edges(e, ne);
    const float* x = X.data();
    auto bin_of = [&](const float* rows, int64_t i, int j) {
      return GpuBooster::host_bin(rows[i * f + j], e.data() + (size_t)j * 255, ne[j]);
    };
    py::dict result;
    py::list bin_variance;
    for (int j = 0; j < std::min(f, 10); ++j) {
      std::set<int> uniq;
      for (int64_t i = 0; i < std::min<int64_t>(n, 100); ++i) uniq.insert(bin_of(x, i, j));
      py::list sample_bins;
      for (int64_t i = 0; i < std::min<int64_t>(n, 10); ++i) sample_bins.append(bin_of(x, i, j));
      py::dict fi;
      fi["feature"] = j;
      fi["unique_bins"] = uniq.size();
      fi["sample_bins"] = sample_bins;
      bin_variance.append(fi);
    }
    result["bin_variance"] = bin_variance;
    py::list traces;
    const tc_model_info& inf = booster_->info;
    if (inf.n_trees > 0) {
      const int D = inf.max_depth, L = 1 << D;
      std::vector<int32_t> depth(inf.n_trees);
      std::vector<uint16_t> feat((size_t)inf.n_trees * D);
      std::vector<uint8_t> sbin((size_t)inf.n_trees * D);
      std::vector<float> lv((size_t)inf.n_trees * L);
      tc_model_export(booster_->model->m, depth.data(), feat.data(), sbin.data(), nullptr, nullptr, lv.data(),
                      nullptr, nullptr, nullptr);
      for (int64_t row = 0; row < std::min<int64_t>(n, 5); ++row) {
        py::dict tr;
        tr["sample_idx"] = row;
        py::list path;
        uint32_t idx = 0;
        for (int k = 0; k < depth[0]; ++k) {
          const int fj = feat[k], b = bin_of(x, row, fj);
          const bool right = b != 255 && b > (int)sbin[k];
          py::dict step;
          step["node_idx"] = (int)((1u << k) - 1 + idx);
          step["split_feature"] = fj;
          step["split_bin"] = (int)sbin[k];
          step["sample_bin"] = b;
          step["go_right"] = right;
          path.append(step);
          idx = (idx << 1) | (right ? 1u : 0u);
        }
        tr["path"] = path;
        tr["leaf_idx"] = (int)idx;
        tr["leaf_value"] = lv[idx];
        traces.append(tr);
      }
    }
    result["sample_traces"] = traces;
    py::list train_bins, raw_compare;
    const bool have_train = train_X_.size() > 0 && train_X_.ndim() == 2 && train_X_.shape(1) == f;
    const int64_t nt = have_train ? train_X_.shape(0) : 0;
    const float* xt = have_train ? train_X_.data() : nullptr;
    if (have_train) {
      for (int j = 0; j < std::min(f, 10); ++j) {
        std::set<int> uniq;
        for (int64_t i = 0; i < std::min<int64_t>(nt, 100); ++i) uniq.insert(bin_of(xt, i, j));
        py::dict fi;
        fi["feature"] = j;
        fi["unique_bins"] = uniq.size();
        train_bins.append(fi);
      }
    }
    for (int j = 0; j < std::min(f, 5); ++j) {
      auto range = [&](const float* rows, int64_t m, float& lo, float& hi) {
        lo = 1e30f;
        hi = -1e30f;
        for (int64_t i = 0; i < m; ++i) {
          const float v = rows[i * f + j];
          if (!std::isnan(v)) { lo = std::min(lo, v); hi = std::max(hi, v); }
        }
      };
      py::dict cmp;
      cmp["feature"] = j;
      if (have_train) {
        float lo, hi;
        range(xt, nt, lo, hi);
        cmp["train_min"] = lo;
        cmp["train_max"] = hi;
      }
      float lo, hi;
      range(x, n, lo, hi);
      cmp["test_min"] = lo;
      cmp["test_max"] = hi;
      raw_compare.append(cmp);
    }
    result["train_bin_variance"] = train_bins;
    result["raw_value_comparison"] = raw_compare;
    return result;
  }

  std::vector<float> predict(FArray X, bool timing) {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    check_2d(X, "X");
    std::vector<float> out;
    const auto t0 = std::chrono::steady_clock::now();
    {
      py::gil_scoped_release nogil;
      out = booster_->predict(X.data(), (uint32_t)X.shape(0), (uint16_t)X.shape(1), TC_TRANSFORM_RAW);
    }
    if (timing) {
      const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
      std::printf("[TIMING] predict total: %.1fms\n", ms);
      std::fflush(stdout);
    }
    return out;
  }

  size_t n_trees() const { return booster_ ? (size_t)booster_->info.n_trees : 0; }
  float base_prediction() const { return booster_ ? booster_->info.base_prediction : 0.0f; }

  void save(const std::string& path) {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    booster_->save(path);
  }
  void load(const std::string& path) {
    booster_.reset(new GpuBooster());
    booster_->load(path);
    n_features_ = booster_->info.n_features;
    is_fitted_ = true;
    train_X_ = FArray();
  }
  py::list get_booster_dump() const {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    return booster_->dump();
  }
  int get_n_features() const {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    return n_features_;
  }
  py::dict debug_info() const {
    py::dict d;
    d["n_trees"] = n_trees();
    d["base_prediction"] = base_prediction();
    d["is_fitted"] = is_fitted_;
    return d;
  }
  py::dict feature_importance() {
    if (!is_fitted_) throw std::runtime_error("Model not fitted");
    std::vector<float> g, gn;
    booster_->importance(g, gn);
    py::dict d;
    d["gain"] = py::array_t<float>(g.size(), g.data());
    d["gain_normalized"] = py::array_t<float>(gn.size(), gn.data());
    return d;
  }
  double train_seconds() const { return booster_ ? booster_->stats.seconds : 0.0; }

 private:
  tc_train_params p_{};
  std::string mode_;
  float subsample_;
  bool use_goss_;
  int verbosity_;
  std::unique_ptr<GpuBooster> booster_;
  FArray train_X_;
  int n_features_ = 0;
  bool is_fitted_ = false;
};

void print_info() {
  py::print("TurboCat B200 engine: symmetric-tree training and inference on sm_100a (libtcgpu.so)");
}

}  // namespace

// ------------------------------------------------------------------- metrics
// The `metrics` submodule (python/bindings.cpp:1139-1224) over the formulas
// that include/turbocat/metrics.hpp:363-470 defines: FP32 sums in row order,
// a row is positive when y_true > 0.5 and predicted positive when
// y_pred >= threshold.  roc_auc, pr_auc and find_optimal_threshold have no
// source in the reference tree (src/metrics/metrics.cpp is missing), so they
// raise.
enum class MetricType : uint8_t { LogLoss = 0, Accuracy, Precision, Recall, F1, ROC_AUC, PR_AUC, MSE, MAE, RMSE };

struct Confusion {
  uint32_t tp = 0, tn = 0, fp = 0, fn = 0;
};

Confusion confusion(const FArray& yt, const FArray& yp, float thr) {
  if (yt.size() != yp.size()) throw std::runtime_error("y_true and y_pred have different lengths");
  Confusion c;
  const float* t = yt.data();
  const float* p = yp.data();
  for (py::ssize_t i = 0; i < yt.size(); ++i) {
    const bool actual = t[i] > 0.5f, pred = p[i] >= thr;
    if (actual && pred) ++c.tp;
    else if (!actual && !pred) ++c.tn;
    else if (!actual && pred) ++c.fp;
    else ++c.fn;
  }
  return c;
}
float precision_of(const Confusion& c) { return c.tp + c.fp > 0 ? (float)c.tp / (float)(c.tp + c.fp) : 0.0f; }
float recall_of(const Confusion& c) { return c.tp + c.fn > 0 ? (float)c.tp / (float)(c.tp + c.fn) : 0.0f; }

float metric_mse(const FArray& yt, const FArray& yp) {
  if (yt.size() != yp.size()) throw std::runtime_error("y_true and y_pred have different lengths");
  float sum = 0.0f;
  for (py::ssize_t i = 0; i < yt.size(); ++i) {
    const float d = yt.data()[i] - yp.data()[i];
    sum += d * d;
  }
  return sum / (float)yt.size();
}

[[noreturn]] void metric_unavailable(const char* name) {
  throw std::runtime_error(std::string(name) +
                           " is unavailable: the reference declares it but ships no source for it "
                           "(src/metrics/metrics.cpp is missing)");
}

PYBIND11_MODULE(_turbocat, m) {
  m.doc() = "TurboCat symmetric-tree path on NVIDIA B200 (sm_100a)";
  m.attr("__version__") = "0.4.2+b200";

  py::class_<TurboCatClassifier>(m, "TurboCatClassifier")
      .def(py::init<int, float, int, int, float, float, float, float, const std::string&, bool, float, float, bool,
                    bool, bool, const std::string&, const std::string&, int, const std::string&, const std::string&,
                    bool, int, const std::string&, int, int, int>(),
           py::arg("n_estimators") = 500, py::arg("learning_rate") = 0.2f, py::arg("max_depth") = 6,
           py::arg("max_bins") = 255, py::arg("subsample") = 1.0f, py::arg("colsample_bytree") = 1.0f,
           py::arg("min_child_weight") = 1.0f, py::arg("lambda_l2") = 1.0f, py::arg("loss") = "logloss",
           py::arg("use_goss") = false, py::arg("goss_top_rate") = 0.2f, py::arg("goss_other_rate") = 0.1f,
           py::arg("use_gradtree") = false, py::arg("use_symmetric") = false, py::arg("use_ordered_boosting") = false,
           py::arg("grow_policy") = "depthwise", py::arg("mode") = "auto", py::arg("early_stopping_rounds") = 50,
           py::arg("early_stopping_metric") = "loss", py::arg("cat_encoding") = "ordered",
           py::arg("auto_interactions") = false, py::arg("max_interactions") = 10,
           py::arg("interaction_method") = "split", py::arg("n_threads") = -1, py::arg("seed") = 42,
           py::arg("verbosity") = 1)
      .def("fit", &TurboCatClassifier::fit, py::arg("X"), py::arg("y"), py::arg("X_val") = FArray(),
           py::arg("y_val") = FArray(), py::arg("cat_features") = std::vector<int>())
      .def("predict", &TurboCatClassifier::predict, py::arg("X"))
      .def("predict_proba", &TurboCatClassifier::predict_proba)
      .def("predict_proba_nobinning_fast", &TurboCatClassifier::predict_proba_nobinning_fast)
      .def("feature_importance", &TurboCatClassifier::feature_importance)
      .def("save", &TurboCatClassifier::save)
      .def("load", &TurboCatClassifier::load)
      .def("get_params", &TurboCatClassifier::get_params)
      .def("get_booster_dump", &TurboCatClassifier::get_booster_dump)
      .def("get_base_prediction", &TurboCatClassifier::get_base_prediction)
      .def("get_n_features", &TurboCatClassifier::get_n_features)
      .def_property_readonly("n_trees", &TurboCatClassifier::n_trees)
      .def_property_readonly("n_classes_", &TurboCatClassifier::n_classes)
      .def_property_readonly("train_seconds", &TurboCatClassifier::train_seconds);

  py::class_<TurboCatRegressor>(m, "TurboCatRegressor")
      .def(py::init<int, float, int, const std::string&, const std::string&, float, float, bool, float, float, int,
                    float, float, int, const std::string&, int, int, int>(),
           py::arg("n_estimators") = 500, py::arg("learning_rate") = 0.1f, py::arg("max_depth") = 6,
           py::arg("loss") = "mse", py::arg("mode") = "auto", py::arg("subsample") = 1.0f,
           py::arg("colsample_bytree") = 1.0f, py::arg("use_goss") = false, py::arg("goss_top_rate") = 0.2f,
           py::arg("goss_other_rate") = 0.1f, py::arg("early_stopping_rounds") = 50, py::arg("lambda_l2") = 3.0f,
           py::arg("min_child_weight") = 1.0f, py::arg("max_leaves") = 64, py::arg("grow_policy") = "depthwise",
           py::arg("n_threads") = -1, py::arg("seed") = 42, py::arg("verbosity") = 1)
      .def("fit", &TurboCatRegressor::fit)
      .def("predict", &TurboCatRegressor::predict, py::arg("X"), py::arg("timing") = false)
      .def("predict_fast", &TurboCatRegressor::predict, py::arg("X"), py::arg("timing") = false)
      .def("predict_nobinning", &TurboCatRegressor::predict, py::arg("X"), py::arg("timing") = false)
      .def("predict_nobinning_fast", &TurboCatRegressor::predict, py::arg("X"), py::arg("timing") = false)
      .def("debug_info", &TurboCatRegressor::debug_info)
      .def("tree_info", &TurboCatRegressor::tree_info)
      .def("debug_predict", &TurboCatRegressor::debug_predict)
      .def("feature_importance", &TurboCatRegressor::feature_importance)
      .def("save", &TurboCatRegressor::save)
      .def("load", &TurboCatRegressor::load)
      .def("get_booster_dump", &TurboCatRegressor::get_booster_dump)
      .def("get_n_features", &TurboCatRegressor::get_n_features)
      .def_property_readonly("n_trees", &TurboCatRegressor::n_trees)
      .def_property_readonly("base_prediction", &TurboCatRegressor::base_prediction)
      .def_property_readonly("train_seconds", &TurboCatRegressor::train_seconds);

  m.def("print_info", &print_info, "Print TurboCat library information");

  auto metrics = m.def_submodule("metrics", "Evaluation metrics for TurboCat");
  py::enum_<MetricType>(metrics, "MetricType")
      .value("LogLoss", MetricType::LogLoss)
      .value("Accuracy", MetricType::Accuracy)
      .value("Precision", MetricType::Precision)
      .value("Recall", MetricType::Recall)
      .value("F1", MetricType::F1)
      .value("ROC_AUC", MetricType::ROC_AUC)
      .value("PR_AUC", MetricType::PR_AUC)
      .value("MSE", MetricType::MSE)
      .value("MAE", MetricType::MAE)
      .value("RMSE", MetricType::RMSE)
      .export_values();
  metrics.def("roc_auc", [](FArray, FArray) -> float { metric_unavailable("roc_auc"); }, "Compute ROC-AUC score",
              py::arg("y_true"), py::arg("y_pred"));
  metrics.def("pr_auc", [](FArray, FArray) -> float { metric_unavailable("pr_auc"); }, "Compute PR-AUC score",
              py::arg("y_true"), py::arg("y_pred"));
  metrics.def(
      "log_loss",
      [](FArray yt, FArray yp, float eps) {
        if (yt.size() != yp.size()) throw std::runtime_error("y_true and y_pred have different lengths");
        float loss = 0.0f;
        for (py::ssize_t i = 0; i < yt.size(); ++i) {
          const float p = std::max(eps, std::min(1.0f - eps, yp.data()[i]));
          const float y = yt.data()[i];
          loss -= y * std::log(p) + (1.0f - y) * std::log(1.0f - p);
        }
        return loss / (float)yt.size();
      },
      "Compute log loss", py::arg("y_true"), py::arg("y_pred"), py::arg("eps") = 1e-15f);
  metrics.def(
      "accuracy",
      [](FArray yt, FArray yp, float thr) {
        const Confusion c = confusion(yt, yp, thr);
        const uint32_t total = c.tp + c.tn + c.fp + c.fn;
        return total > 0 ? (float)(c.tp + c.tn) / (float)total : 0.0f;
      },
      "Compute accuracy", py::arg("y_true"), py::arg("y_pred"), py::arg("threshold") = 0.5f);
  metrics.def(
      "precision", [](FArray yt, FArray yp, float thr) { return precision_of(confusion(yt, yp, thr)); },
      "Compute precision", py::arg("y_true"), py::arg("y_pred"), py::arg("threshold") = 0.5f);
  metrics.def(
      "recall", [](FArray yt, FArray yp, float thr) { return recall_of(confusion(yt, yp, thr)); },
      "Compute recall", py::arg("y_true"), py::arg("y_pred"), py::arg("threshold") = 0.5f);
  metrics.def(
      "f1_score",
      [](FArray yt, FArray yp, float thr) {
        const Confusion c = confusion(yt, yp, thr);
        const float p = precision_of(c), r = recall_of(c);
        return p + r > 0 ? 2.0f * p * r / (p + r) : 0.0f;
      },
      "Compute F1 score", py::arg("y_true"), py::arg("y_pred"), py::arg("threshold") = 0.5f);
  metrics.def(
      "find_optimal_threshold",
      [](FArray, FArray, MetricType, int) -> float { metric_unavailable("find_optimal_threshold"); },
      "Find optimal threshold for a metric", py::arg("y_true"), py::arg("y_pred"),
      py::arg("metric") = MetricType::F1, py::arg("n_thresholds") = 100);
  metrics.def("mse", &metric_mse, "Compute mean squared error", py::arg("y_true"), py::arg("y_pred"));
  metrics.def(
      "mae",
      [](FArray yt, FArray yp) {
        if (yt.size() != yp.size()) throw std::runtime_error("y_true and y_pred have different lengths");
        float sum = 0.0f;
        for (py::ssize_t i = 0; i < yt.size(); ++i) sum += std::abs(yt.data()[i] - yp.data()[i]);
        return sum / (float)yt.size();
      },
      "Compute mean absolute error", py::arg("y_true"), py::arg("y_pred"));
  metrics.def(
      "rmse", [](FArray yt, FArray yp) { return std::sqrt(metric_mse(yt, yp)); },
      "Compute root mean squared error", py::arg("y_true"), py::arg("y_pred"));
}
