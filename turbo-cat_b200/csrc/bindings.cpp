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

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <memory>
#include <mutex>
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

// Host-side booster: the counterpart of turbocat::Booster for the symmetric path.
class GpuBooster {
 public:
  std::unique_ptr<ModelPtr> model;
  tc_model_info info{};
  tc_train_stats stats{};

  // With a validation set (Xv, yv, nv > 0) the fit follows Booster::train's
  // valid_data branch: validation loss every iteration, early stopping after
  // `es_rounds` iterations without improvement (src/boosting/booster.cpp:255-371).
  void fit(const float* X, uint32_t n, uint16_t f, const float* y, const tc_train_params& p,
           const float* Xv = nullptr, const float* yv = nullptr, uint32_t nv = 0, int es_rounds = 50) {
    tc_ctx* ctx = device_context();
    tc_dataset* ds = nullptr;
    tc_dataset* vds = nullptr;
    check(tc_dataset_upload(ctx, X, n, f, y, &ds), ctx);
    tc_status s = tc_quantize(ds, (uint16_t)p.max_bins, 1, nullptr, nullptr);
    tc_model* m = nullptr;
    if (s == TC_OK && nv == 0) s = tc_train(ctx, ds, &p, &m, &stats);
    if (s == TC_OK && nv > 0) {
      tc_trainer* tr = nullptr;
      s = tc_dataset_upload(ctx, Xv, nv, f, yv, &vds);
      if (s == TC_OK) s = tc_trainer_create(ctx, ds, &p, &tr);
      if (s == TC_OK) s = tc_trainer_set_validation(tr, vds, es_rounds);
      if (s == TC_OK) s = tc_trainer_step(tr, p.n_estimators, 1);
      if (s == TC_OK) s = tc_trainer_model(tr, &m);
      if (s == TC_OK) s = tc_trainer_stats(tr, &stats);
      if (tr) tc_trainer_destroy(tr);
    }
    if (vds) tc_dataset_destroy(vds);
    tc_dataset_destroy(ds);
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
    (void)cat_encoding; (void)max_interactions;
    (void)interaction_method; (void)n_threads;
  }

  void fit(FArray X, FArray y, FArray X_val, FArray y_val, std::vector<int> cat_features) {
    check_2d(X, "X");
    if (y.ndim() != 1) throw std::runtime_error("y must be 1-dimensional");
    const uint32_t n = (uint32_t)X.shape(0);
    const uint16_t f = (uint16_t)X.shape(1);
    if ((size_t)y.shape(0) != n) throw std::runtime_error("X and y have different numbers of rows");
    if (mode_ == "small") warn("mode='small' (regular trees) is not on the device path; building symmetric trees");
    if (colsample_ < 1.0f && verbosity_ > 1) warn("colsample_bytree has no effect on symmetric trees");
    if (use_gradtree_ || use_ordered_ || auto_interactions_)
      warn("use_gradtree / use_ordered_boosting / auto_interactions are not on the device path and are ignored");
    if (!cat_features.empty()) throw std::invalid_argument("cat_features are not supported on the device path");
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
    {
      py::gil_scoped_release nogil;
      booster_.reset(new GpuBooster());
      if (has_val)
        booster_->fit(X.data(), n, f, yp, p, X_val.data(), y_val.data(), (uint32_t)X_val.shape(0), es_rounds_);
      else
        booster_->fit(X.data(), n, f, yp, p);
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
      out = booster_->predict(X.data(), n, f, K > 1 ? TC_TRANSFORM_SOFTMAX : TC_TRANSFORM_SIGMOID);
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
    if (verbosity_ > 0)
      py::print("[TurboCat-B200] trained", booster_->info.n_trees, "trees in", booster_->stats.seconds, "s (device)");
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
  int n_features_ = 0;
  bool is_fitted_ = false;
};

void print_info() {
  py::print("TurboCat B200 engine: symmetric-tree training and inference on sm_100a (libtcgpu.so)");
}

}  // namespace

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
      .def("feature_importance", &TurboCatRegressor::feature_importance)
      .def("save", &TurboCatRegressor::save)
      .def("load", &TurboCatRegressor::load)
      .def("get_booster_dump", &TurboCatRegressor::get_booster_dump)
      .def("get_n_features", &TurboCatRegressor::get_n_features)
      .def_property_readonly("n_trees", &TurboCatRegressor::n_trees)
      .def_property_readonly("base_prediction", &TurboCatRegressor::base_prediction)
      .def_property_readonly("train_seconds", &TurboCatRegressor::train_seconds);

  m.def("print_info", &print_info, "Print TurboCat library information");
}
