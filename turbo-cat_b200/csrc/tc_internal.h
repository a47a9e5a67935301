// Internal declarations shared by the libtcgpu.so translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tcgpu.h"

namespace tc {

constexpr int kNanBin = 255;      // bin of NaN rows; always routed left
constexpr int kSlots = 256;       // histogram slots per (node, feature): bins 0..254 + NaN
constexpr int kMaxDepth = 12;     // deepest tree the trainer builds
constexpr int kModelMaxDepth = 13;  // deepest tree a model may hold (import, TCAT, prediction)
constexpr int kMaxClasses = 64;

inline size_t round_up(size_t x, size_t m) { return (x + m - 1) / m * m; }

}  // namespace tc

struct tc_ctx {
  int device = 0;
  int sm_count = 148;
  size_t budget = 0;
  size_t in_use = 0;
  size_t peak = 0;
  int fail_next = 0;
  cudaStream_t stream = nullptr;       // training, binning, uploads
  cudaStream_t pred_stream = nullptr;  // tc_predict / tc_predict_device (NULL stream)
  std::string err;
  std::mutex mu;                     // guards allocation accounting and err
  std::map<void*, size_t> allocs;
  // training calls (tc_train, tc_build_tree, tc_trainer_*) on one context
  // run one at a time: they share the context's stream and tuner state
  std::recursive_mutex train_mu;
  // tc_predict's device staging (grow-only, one caller at a time)
  std::mutex pred_mu;
  void* pred_scratch = nullptr;
  size_t pred_scratch_bytes = 0;
  // small predictions: pinned host staging mapped into the device's address
  // space (inputs read and outputs written by the kernel in place), and
  // device partial sums with a completion counter
  float* pin_io = nullptr;           // [pin_floats] inputs, then outputs
  float* pin_io_dev = nullptr;       // its device alias
  size_t pin_floats = 0;
  void* small_scratch = nullptr;     // partials [blocks][rows][K] + counter
  size_t small_scratch_bytes = 0;
  // staging of large uploads: two pinned chunks filled by host threads while
  // the other one is copied to the device (tc_data.cu); guarded by train_mu
  void* up_stage[2] = {nullptr, nullptr};
  cudaEvent_t up_ev[2] = {nullptr, nullptr};
  // latency worker: a persistent kernel serving small requests of one model
  // through a pinned mailbox (tc_predict.cu); guarded by pred_mu
  void* lw_box = nullptr;            // mailbox, host pointer (pinned, mapped)
  void* lw_box_dev = nullptr;        // its device alias
  void* lw_dev = nullptr;            // announcement words, counter, partials
  cudaStream_t lw_stream = nullptr;
  const tc_model* lw_model = nullptr;
  bool lw_running = false;
  int lw_blocks = 0;
  uint32_t lw_seq = 0;
  bool lw_enabled = true;

  tc_status fail(tc_status code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    std::lock_guard<std::mutex> g(mu);
    err = buf;
    return code;
  }
  tc_status cuda_fail(cudaError_t e, const char* what) {
    return fail(TC_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
  }
  // Device allocation with budget accounting and test fault injection.
  tc_status alloc(void** p, size_t bytes, const char* what);
  void release(void* p);
};

#define TC_CUDA(ctx, call)                                         \
  do {                                                             \
    cudaError_t e_ = (call);                                       \
    if (e_ != cudaSuccess) return (ctx)->cuda_fail(e_, #call);     \
  } while (0)

#define TC_TRY(expr)                    \
  do {                                  \
    tc_status s_ = (expr);              \
    if (s_ != TC_OK) return s_;         \
  } while (0)

// A device buffer owned by a context.
template <class T>
struct DevBuf {
  tc_ctx* ctx = nullptr;
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { reset(); }
  tc_status alloc(tc_ctx* c, size_t count, const char* what) {
    reset();
    ctx = c;
    void* q = nullptr;
    tc_status s = c->alloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16, what);
    if (s != TC_OK) return s;
    p = static_cast<T*>(q);
    n = count;
    return TC_OK;
  }
  void reset() {
    if (p && ctx) ctx->release(p);
    p = nullptr;
    n = 0;
  }
  size_t bytes() const { return n * sizeof(T); }
};

struct tc_dataset {
  tc_ctx* ctx = nullptr;
  uint32_t n = 0;
  uint32_t f = 0;
  uint32_t groups = 0;       // 32-feature groups of the tiled bin matrix
  uint32_t nt = 0;           // rows of a tile block (n rounded up to 32)
  uint32_t wlast = 0;        // bytes per row of the last group's block: 4, 8, 16 or 32
  uint64_t gstride = 0;      // bytes of one full group block (32 x nt)
  uint32_t np = 0;           // column stride of the column-major bin matrix (n rounded up to 16)
  bool quantized = false;
  int max_bins = 255;
  DevBuf<float> X;           // [n][f] row-major input
  DevBuf<float> y;           // [n] labels (may be empty)
  DevBuf<uint8_t> bins_t;    // feature-group tiles: group g is a [nt][32] block (the last [nt][wlast])
  DevBuf<uint8_t> bins_cm;   // [f][np]
  DevBuf<float> edges;       // [f][256]
  DevBuf<uint16_t> n_edges;  // [f]
  DevBuf<uint32_t> nan_any;  // [f] nonzero: the feature has NaN rows
  std::vector<float> h_edges;       // [f][255]
  std::vector<uint16_t> h_n_edges;  // [f]
  // Categorical columns encoded by target statistics (tc_encode_categorical):
  // X holds each row's encoding in those columns, and binning uses the
  // reference's TS edge rule and lower_bound for them (ts[j] = 1).  Encoded
  // column c (0 .. nc-1) is feature cat_feats[c]; its global table (sorted
  // categories -> smoothed mean, for tc_apply_bins) is entries
  // [cat_off[c], cat_off[c] + cat_len[c]) of cat_keys / cat_vals.
  std::vector<uint8_t> h_ts;         // [f]
  DevBuf<uint8_t> ts;                // [f]
  std::vector<uint16_t> h_cat_feats; // [nc]
  std::vector<uint32_t> h_cat_off;   // [nc]
  std::vector<uint32_t> h_cat_len;   // [nc]
  DevBuf<uint16_t> cat_feats;        // [nc]
  DevBuf<uint32_t> cat_off;          // [nc]
  DevBuf<uint32_t> cat_len;          // [nc]
  DevBuf<uint32_t> cat_keys;         // [sum of the segment counts]
  DevBuf<float> cat_vals;            // [sum of the segment counts]
  float cat_prior = 0.0f;
  uint64_t id = 0;                   // unique per dataset of the process
  uint64_t encoded_by = 0;           // id of the dataset whose tables encoded X (tc_apply_bins)
};

// Flat device-resident symmetric ensemble (the FastFloatEnsemble layout,
// include/turbocat/fast_float_ensemble.hpp:90-100).
struct tc_model {
  tc_ctx* ctx = nullptr;
  tc_model_info info{};
  std::vector<int32_t> depth;       // [T]
  std::vector<uint16_t> feature;    // [T][D]
  std::vector<uint8_t> bin;         // [T][D]
  std::vector<float> threshold;     // [T][D]
  std::vector<float> gain;          // [T][D]
  std::vector<float> leaves;        // [T][2^D]
  std::vector<float> weights;       // [T]
  std::vector<float> edges;         // [f][255]
  std::vector<uint16_t> n_edges;    // [f]
  // device copies used by the predict kernels
  DevBuf<uint2> d_splits;           // [T][D] (feature, threshold bits), padded to depth D
  DevBuf<float> d_leaves;           // [T][2^D] (weights folded in, padded trees' leaves spread)
  DevBuf<uint2> d_bsplits;          // binned form: [T][D] (virtual feature's column, byte-wise 128 - k)
  DevBuf<float> d_bord;             // binned form: borders of every virtual feature, Eytzinger order
  DevBuf<uint2> d_vdesc;            // binned form: (feature, border offset | search steps << 24)
  int n_virtual = 0, n_bord = 0;
  // regular (depth-wise) trees of a model the reference trained with
  // mode="small" (served for prediction only; tc_predict.cu)
  bool regular = false;
  std::vector<uint8_t> tcat;        // the stream as loaded (saved back byte for byte)
  DevBuf<uint4> d_rnodes;           // (feature | bin << 16 | leaf << 24, left, right, value bits), global indices
  DevBuf<uint32_t> d_rroots;        // [T] first node of each tree
  DevBuf<float> d_rweights;         // [T]
  DevBuf<float> d_redges;           // [f][255] bin edges
  DevBuf<int32_t> d_rnedges;        // [f]
  tc_status upload();
};

namespace tc {

// Stops the latency worker (if one runs) and waits for it; with m, only if
// it serves m.  Caller holds ctx->pred_mu (tc_predict.cu).
void stop_latency_worker(tc_ctx* ctx, const tc_model* m);

// Quantization entry (tc_data.cu).
tc_status quantize(tc_dataset* ds, int max_bins, int compat_u8);
tc_status encode_categorical(tc_dataset* ds, const uint16_t* feats, uint16_t nc, const tc_cat_params* p,
                             const uint32_t* order);
// Regular (depth-wise) trees (tc_regular.cu).
tc_status train_regular(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_model** out,
                        tc_train_stats* stats);

// Prediction (tc_predict.cu): raw scores [n][K] (+ transform) on device buffers.
tc_status predict_device(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint32_t f,
                         int transform, float* out, cudaStream_t stream);

// Serving request table entry for the coalesced predict kernel.
struct ReqDesc {
  const float* X;     // device pointer to the request's rows [n][f]
  float* out;         // device pointer to its outputs [n][K]
  uint32_t n;
  uint32_t row_begin; // first global row of this request in the batch
  int32_t model;      // index into the model table
  int32_t transform;
};
struct ModelDesc {
  const uint2* splits;   // float form
  const float* leaves;
  const uint2* bsplits;  // binned form (nullptr: the model has none)
  const float* bord;
  const uint2* vdesc;
  int32_t n_trees;
  int32_t max_depth;
  int32_t n_classes;
  int32_t n_features;
  float base;
  int32_t n_virtual;
  int32_t n_bord;
  int32_t pad;
};
// Coalesced prediction over a request table: job j covers tiles
// [tile_begin[j], tile_begin[j+1]) of PRED_ROWS rows each.
// Launch shape of a batch: dynamic shared memory and stage sizes that fit
// every model of the batch.
struct PredictPlan {
  size_t smem;
  int leaf_stage;   // floats of one leaf stage
  int split_stage;  // splits of one split stage
};
PredictPlan predict_plan(const tc_model* const* models, int n);
tc_status predict_batched(tc_ctx* ctx, const ModelDesc* d_models, const ReqDesc* d_reqs, int n_reqs,
                          const uint32_t* d_tile_begin, uint32_t n_tiles, const PredictPlan& plan,
                          cudaStream_t stream);
uint32_t predict_tiles(uint32_t n);
ModelDesc model_desc(const tc_model* m);

}  // namespace tc
