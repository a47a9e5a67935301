/*
 * tcgpu.h -- C ABI of the B200-native TurboCat symmetric-tree engine
 * (libtcgpu.so).
 *
 * Plain pointers and sizes only.  Every entry point returns a tc_status;
 * on failure a message is kept per context (tc_last_error).  No call aborts
 * the process or traps the device.
 *
 * Each entry point names the reference interface it replaces
 * (ispromadhka/Turbo-Cat, paths relative to that project).
 *
 * Data conventions
 *   X          row-major float32 [n][f], C-contiguous (the layout the
 *              reference's facade forces, python/turbocat/__init__.py:441-446)
 *   bins       column-major uint8 [f][n] (BinnedData, include/turbocat/dataset.hpp:27-82);
 *              NaN rows hold bin 255 and always route left
 *   edges      float32 [f][255], first n_edges[j] entries used
 *   trees      T trees, iteration-major and class-minor for multiclass;
 *              per tree: depth, (feature, bin, float threshold, gain) per
 *              level padded to max_depth, 2^max_depth leaf values (padded)
 *
 * Threads: dataset and training calls (tc_dataset_*, tc_quantize,
 * tc_apply_bins, tc_encode_categorical, tc_train, tc_train_regular,
 * tc_build_tree, tc_trainer_*) on one context run one at a time; tc_predict
 * calls on one context run one at a time, on a stream of their own, so they
 * may run while another thread trains; tc_server_submit/poll may be called
 * from any thread.  The reference
 * is not thread-safe at all (thread_local pools and mutable caches,
 * src/tree/symmetric_tree.cpp:57-89).
 */
#ifndef TCGPU_H
#define TCGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  TC_OK = 0,
  TC_ERR_INVALID_ARG = 1,  /* std::invalid_argument in the reference (include/turbocat/config.hpp:399-418) */
  TC_ERR_OOM = 2,          /* device allocation failed or the context's memory budget is exhausted */
  TC_ERR_TIMEOUT = 3,      /* a bounded host-side wait on the device ran out */
  TC_ERR_CUDA = 4,         /* a CUDA runtime error; the message names it */
  TC_ERR_NOT_FITTED = 5,   /* "Model not fitted" (python/bindings.cpp:289-291) */
  TC_ERR_FORMAT = 6,       /* malformed TCAT stream (src/boosting/booster.cpp:1120-1130) */
  TC_ERR_BUSY = 7          /* serving queue full / request not finished */
} tc_status;

enum { TC_LOSS_LOGLOSS = 0, TC_LOSS_MSE = 1, TC_LOSS_FOCAL = 2, TC_LOSS_SOFTMAX = 3 };
enum { TC_TRANSFORM_RAW = 0, TC_TRANSFORM_SIGMOID = 1, TC_TRANSFORM_SOFTMAX = 2 };
enum { TC_TASK_BINARY = 0, TC_TASK_MULTICLASS = 1, TC_TASK_REGRESSION = 2 }; /* TaskType, include/turbocat/types.hpp:242-247 */

typedef struct tc_ctx tc_ctx;
typedef struct tc_dataset tc_dataset;
typedef struct tc_trainer tc_trainer;
typedef struct tc_model tc_model;
typedef struct tc_server tc_server;

/* ---------------------------------------------------------------- context */

/* Creates a context on CUDA device `device` with a device-memory budget in
 * bytes (0 = no limit beyond the device).  Replaces the reference's
 * HistogramBuilder::create(DeviceConfig) seam (src/tree/histogram.cpp:558-561,
 * DeviceType::CUDA at include/turbocat/config.hpp:196-201), which only ever
 * returned the CPU builder. */
tc_status tc_ctx_create(int device, size_t mem_budget, tc_ctx** out);
void tc_ctx_destroy(tc_ctx* ctx);
/* Message of the last failed call on this context (never NULL). */
const char* tc_last_error(const tc_ctx* ctx);
/* Bytes currently allocated by the context and its objects, and the peak. */
tc_status tc_ctx_memory(const tc_ctx* ctx, size_t* in_use, size_t* peak);
/* Fault-injection hook for host-side tests: the next `count` device
 * allocations made through this context fail with TC_ERR_OOM. */
tc_status tc_ctx_fail_next_allocs(tc_ctx* ctx, int count);
/* Bounded wait (milliseconds) for all work queued by this context. */
tc_status tc_ctx_synchronize(tc_ctx* ctx, int timeout_ms);
/* Small predict requests (tc_predict, at most 64 rows) through the context's
 * persistent latency worker (enabled = 1, the default) or by one kernel
 * launch each (0); disabling stops a running worker. */
tc_status tc_ctx_set_latency_worker(tc_ctx* ctx, int enabled);

/* ---------------------------------------------------------------- dataset */

/* Copies X (row-major [n][f]) and optional labels y [n] to the device.
 * Replaces Dataset::from_dense (src/core/dataset.cpp:50-94). */
tc_status tc_dataset_upload(tc_ctx* ctx, const float* X, uint32_t n, uint16_t f, const float* y,
                            tc_dataset** out);
void tc_dataset_destroy(tc_dataset* ds);

/* Quantile binning on the device.  Replaces Dataset::compute_bins /
 * compute_quantile_bins / find_bin (src/core/dataset.cpp:176-344).
 * compat_uint8_count = 1 reproduces the reference's uint8 truncation of the
 * unique-value count (actual_bins = min(max_bins, (uint8)U),
 * src/core/dataset.cpp:308).  edges_out [f][255] and n_edges_out [f] are
 * optional host outputs. */
tc_status tc_quantize(tc_dataset* ds, uint16_t max_bins, int compat_uint8_count, float* edges_out,
                      uint16_t* n_edges_out);
/* Bins ds with the edges of ref (a quantized dataset of the same context and
 * feature count): bin = number of ref's edges <= x, NaN -> 255, the same
 * assignment tc_quantize makes for numeric features; ds can then be trained
 * on, predicted from (tc_predict_dataset) or exported like a quantized
 * dataset.  ref's categorical columns (tc_encode_categorical) are first
 * replaced in ds's X by ref's global encoding of each row's category, 0.5
 * for a category ref never saw, then binned the same way.  Replaces
 * Dataset::apply_bins (src/core/dataset.cpp:346-379). */
tc_status tc_apply_bins(tc_dataset* ds, const tc_dataset* ref);
/* Host copy of the binned matrix, column-major [f][n]
 * (BinnedData::column, include/turbocat/dataset.hpp:27-82). */
tc_status tc_dataset_bins(const tc_dataset* ds, uint8_t* bins_out);
/* Host copy of the dataset's feature matrix X [n][f] as the device holds it
 * (categorical columns hold their encodings once encoded). */
tc_status tc_dataset_features(const tc_dataset* ds, float* X_out);

/* Categorical target statistics (Dataset::compute_target_statistics,
 * src/core/dataset.cpp:679-865). */
#define TC_CAT_ORDERED 0 /* ordered TS: each row sees the rows before it in a random order */
#define TC_CAT_CV 1      /* cross-validated TS: each row sees the rows of the other folds */
typedef struct {
  int32_t method;     /* TC_CAT_ORDERED or TC_CAT_CV */
  float prior_weight; /* smoothing weight a of (sum + a * prior) / (count + a); the reference's is 1 */
  int32_t cv_folds;   /* folds of TC_CAT_CV (2 .. 255); the reference's is 5 */
  uint64_t seed;      /* draws the order / folds when `order` is NULL */
} tc_cat_params;
/* Replaces the categorical columns `features` of a labelled, not yet
 * quantized dataset by their per-row target statistics and records each
 * feature's global table (category -> (sum + a * prior) / (count + a) over all
 * rows) for tc_apply_bins.  Category = (uint32)(int64) of the value; NaN rows
 * get the prior (the mean label) and count in no statistic.  `order` (host,
 * optional): TC_CAT_ORDERED, the processing order, a permutation of 0..n-1;
 * TC_CAT_CV, each row's fold (< cv_folds).  NULL draws it from `seed` (the
 * reference draws it from std::random_device, so its runs differ from one
 * another; a given order reproduces them bit for bit).  tc_quantize then bins
 * these columns by the reference's target-statistics rule: A = min(max_bins,
 * U) edges, edge b = the distinct encoding of rank (b+1)*U/(A+1), bin =
 * number of edges < x (src/core/dataset.cpp:183-240). */
tc_status tc_encode_categorical(tc_dataset* ds, const uint16_t* features, uint16_t n_cat,
                                const tc_cat_params* p, const uint32_t* order);
/* One categorical feature's global table, sorted by category: with keys or
 * vals NULL only *len is written (Dataset::target_stats,
 * include/turbocat/dataset.hpp:207-226). */
tc_status tc_category_table(const tc_dataset* ds, uint16_t feature, uint32_t* keys, float* vals,
                            uint32_t* len);

/* --------------------------------------------------------------- training */

typedef struct {
  int32_t loss;             /* TC_LOSS_* */
  int32_t n_classes;        /* K for TC_LOSS_SOFTMAX, else 1 */
  int32_t n_estimators;     /* boosting iterations (K trees each for softmax) */
  int32_t max_depth;        /* 1 .. 12 */
  int32_t max_bins;         /* split scan covers bins 0 .. max_bins-2 */
  int32_t min_samples_leaf;
  float learning_rate;
  float lambda_l2;
  float lambda_l1;
  float min_child_weight;
  float min_split_gain;
  float max_delta_step;
  float focal_gamma;        /* LossConfig::focal_gamma (include/turbocat/config.hpp:108) */
  float focal_alpha;        /* LossConfig::focal_alpha (include/turbocat/config.hpp:109) */
  int32_t batched;          /* 1: all classes and nodes of a level per launch, one CUDA graph per
                               iteration; 0: the plain path, one tree and one level at a time with a
                               host synchronisation per level */
  int32_t hist_features_per_block; /* feature-group width of the histogram kernel: 32 (any value) */
  int32_t hist_rows_per_chunk;     /* 0 = autotune */
  /* Row sampling, Booster::train's sample selection (src/boosting/booster.cpp:198-228):
   * with 0 < subsample < 1 every iteration's trees are built on the first
   * (uint32)(n * subsample) rows of a std::shuffle (std::mt19937_64 seeded by
   * an xorshift64* draw from `seed`, src/core/dataset.cpp:552-562) and
   * applied to all rows; with 0 < colsample_bytree < 1 one more draw per
   * iteration (the reference's feature subset, which its symmetric trees do
   * not use).  0 or >= 1: no sampling / no draw. */
  float subsample;
  float colsample_bytree;
  uint64_t seed;                    /* Config::seed (default 42 in the reference) */
  /* Gradient-based one-side sampling, Dataset::goss_subsample
   * (src/core/dataset.cpp:494-549), selected over subsample as in
   * Booster::train (src/boosting/booster.cpp:200-219): with use_goss != 0
   * every iteration's trees are built on the (uint32)(n * goss_top_rate) rows
   * of largest |gradient| (softmax: the largest |gradient| over the classes,
   * src/boosting/booster.cpp:1327-1348) plus (uint32)(n * goss_other_rate)
   * rows drawn from the rest by a partial Fisher-Yates shuffle
   * (std::mt19937_64 seeded by one xorshift64* draw).  The selection runs
   * on the host from the iteration's gradients (std::nth_element's
   * arrangement decides which rows the draws reach), so every such
   * iteration synchronises with the host.  Rates in [0, 1]. */
  int32_t use_goss;
  float goss_top_rate;              /* reference default 0.2 */
  float goss_other_rate;            /* reference default 0.1 */
} tc_train_params;

typedef struct {
  int32_t n_trees;
  int32_t iterations_done;
  float base_prediction;
  double seconds;           /* device time of the boosting iterations run so far */
  int32_t hist_features_per_block;
  int32_t hist_rows_per_chunk;
  int64_t kernel_launches;  /* kernels launched by the iterations run so far */
  int32_t best_iteration;   /* validation set: iteration of the best validation loss (else -1) */
  int32_t stopped_early;    /* validation set: 1 once the early-stopping rule has fired */
} tc_train_stats;

/* Per-kernel timing of profiled iterations with the algorithmic bytes each
 * kernel class moved: for the histogram kernel R*(F + 8 + 1) +
 * built_nodes*F*255*8, R = rows histogrammed (bin bytes, (grad, hess), node
 * id per row; FP32 (grad, hess) sums per built node, feature and bin).  On
 * the batched path (in_graph = 1) the iteration is captured as a CUDA graph
 * with an event-record node around every launch and replayed, so the times
 * are those of launches inside a graph; iteration_ms sums the replayed
 * iterations from the first launch's start to the last one's end.  GOSS and
 * the plain path are timed launch by launch (in_graph = 0). */
typedef struct {
  char name[16];
  int64_t launches;
  double ms;
  double alg_bytes;
} tc_kernel_time;
typedef struct {
  int32_t n_kernels;
  tc_kernel_time k[12];
  double hist_level_ms[16];     /* histogram kernel time per tree level */
  double hist_level_rows[16];   /* rows histogrammed per tree level */
  double part_level_ms[16];     /* partition kernel time per tree level */
  int32_t in_graph;             /* 1: timed inside a replayed CUDA graph */
  double iteration_ms;          /* profiled iterations, first launch start to last launch end */
} tc_profile;

/* Stateful boosting loop over a quantized dataset.  Replaces
 * Booster::train's iteration loop (src/boosting/booster.cpp:47-418) for
 * symmetric trees, and the composed symmetric multiclass loop built from
 * Booster::train_multiclass (src/boosting/booster.cpp:1263-1395). */
tc_status tc_trainer_create(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_trainer** out);
/* Runs `iterations` more boosting iterations (stream-ordered; returns after
 * queueing unless `sync` != 0). */
tc_status tc_trainer_step(tc_trainer* tr, int32_t iterations, int sync);
/* Forgets all trees and restarts from the base prediction (same data). */
tc_status tc_trainer_reset(tc_trainer* tr);
tc_status tc_trainer_stats(tc_trainer* tr, tc_train_stats* st);
/* Runs `iterations` more boosting iterations launch by launch (no graph),
 * timing every kernel; the trees are the same as tc_trainer_step's. */
tc_status tc_trainer_profile(tc_trainer* tr, int32_t iterations, tc_profile* out);
/* Raw training-set scores [n][K] (base included) after the trees so far. */
tc_status tc_trainer_train_scores(tc_trainer* tr, float* out);
/* Rows the last iteration's trees were built on, one bit per row
 * (row i: bit i % 32 of word i / 32; ceil(n / 32) words, bits past n are 0).
 * Every row when neither subsample nor GOSS is on.  No counterpart in the
 * reference, whose sample indices stay inside Booster::train
 * (src/boosting/booster.cpp:198-232). */
tc_status tc_trainer_sample_mask(tc_trainer* tr, uint32_t* out);
/* Snapshot of the ensemble trained so far as an immutable model. */
tc_status tc_trainer_model(tc_trainer* tr, tc_model** out);
/* Validation set and early stopping, Booster::train's valid_data branch
 * (src/boosting/booster.cpp:255-371; multiclass 1405-1435).  After every
 * iteration its trees are added to the validation predictions (FP32
 * lr * leaf), the validation loss is the loss's compute_loss (mean logloss
 * with p clipped to [1e-7, 1 - 1e-7], mean squared error, robust focal,
 * multiclass cross entropy; summed in FP64 here), an improvement is
 * loss < best - 1e-10, and training stops once the iteration is
 * >= max(50, n_estimators / 10) and `early_stopping_rounds` iterations in a
 * row did not improve (< 0: never stop).  The model keeps every tree up to
 * and including the stopping iteration, as the reference's loop breaks
 * there.  `valid` needs labels and the training set's feature count (raw
 * features; it need not be quantized); call before the first iteration. */
tc_status tc_trainer_set_validation(tc_trainer* tr, const tc_dataset* valid, int32_t early_stopping_rounds);
/* Validation loss of every iteration run so far (iterations_done values). */
tc_status tc_trainer_valid_loss(tc_trainer* tr, double* out);
void tc_trainer_destroy(tc_trainer* tr);

/* One-shot fit: create + step(n_estimators) + model.  Replaces
 * Booster::train (src/boosting/booster.cpp:47). */
tc_status tc_train(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_model** out,
                   tc_train_stats* st);
/* One-shot fit of regular (depth-wise) trees, the reference's mode="small"
 * (Booster::train with use_symmetric = false, src/boosting/booster.cpp:447-520;
 * Tree::build, src/tree/tree.cpp:162-407): per node the best (feature, bin)
 * of SplitFinder (src/tree/histogram.cpp:569-690), the reference's stop rules
 * including its 64-leaf cap in its recursion order (smaller child first), leaf
 * -G/(H + lambda_l2).  Binary logloss, every row in every tree (subsample 1,
 * no GOSS).  The model is a TCAT v3 regular-tree model in the reference's node
 * numbering (tc_model_save_tcat writes it; tc_predict serves it as the
 * reference predicts such models). */
tc_status tc_train_regular(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_model** out,
                           tc_train_stats* st);

/* One symmetric tree on caller-given gradients/hessians [n] over all rows of
 * a quantized dataset.  Replaces SymmetricTree::build
 * (src/tree/symmetric_tree.cpp:34-368) for parity checks.  Outputs per level
 * split feature, bin, float threshold and FP64 gain, the runner-up gain,
 * 2^max_depth leaf values, optionally the per-row leaf index [n] and the
 * FP64 root histogram [f][256][2] (slot 255 = NaN rows).  Returns the depth
 * through *depth_out. */
tc_status tc_build_tree(tc_ctx* ctx, tc_dataset* ds, const float* grad, const float* hess,
                        const tc_train_params* p, int32_t* depth_out, uint16_t* split_feature,
                        uint8_t* split_bin, float* split_threshold, double* split_gain,
                        double* runner_up_gain, float* leaf_values, uint32_t* leaf_index,
                        double* root_hist);

/* Root-level gradient/hessian histogram that allocates no device memory.
 * No counterpart in the reference: it exists for callers that cannot call
 * cudaMalloc -- e.g. a process whose device memory is entirely reserved by
 * another framework's allocator, or a latency-critical request path where a
 * driver allocation (which can synchronise the device, and can fail) is not
 * allowed.  All buffers are the caller's device memory: bins_rm row-major
 * uint8 [n][row_stride] (NaN rows in bin 255), grad/hess float [n],
 * hist_out FP64 [f][256][2] (grad, hess).  Scratch is a fixed 16 MiB
 * device array inside the library (every GPU that loads the library holds it
 * until the process exits); at most 8192 features, larger f is rejected with
 * TC_ERR_INVALID_ARG.  The first call on a device resolves that array's
 * device address in the device's primary context (the one the CUDA runtime
 * uses; a caller that drives its own driver-API context is not supported,
 * and the address is not valid after cudaDeviceReset), so make the first
 * call before any stream capture.  Calls share the array: calls that overlap
 * on the GPU race (serialise them on one stream).  A block sums at most
 * 16384 rows in FP32; larger inputs run as several passes merged into
 * hist_out in FP64.  Queued on `stream` (NULL = the context's stream, in
 * which case the call waits for any training call on the context to finish,
 * so that it never joins the trainer's graph capture); returns without
 * synchronising.  The calling thread's current device is left unchanged. */
tc_status tc_histogram_root_noalloc(tc_ctx* ctx, const uint8_t* bins_rm, uint32_t n, uint16_t f,
                                    uint32_t row_stride, const float* grad, const float* hess,
                                    double* hist_out, void* stream);

/* ------------------------------------------------------------------ model */

typedef struct {
  int32_t n_trees;
  int32_t n_classes;        /* 1 for binary / regression */
  int32_t max_depth;        /* padding width of the per-tree arrays */
  int32_t n_features;
  int32_t task;             /* TC_TASK_* */
  float base_prediction;
  float learning_rate;
  float lambda_l2;
} tc_model_info;

tc_status tc_model_info_get(const tc_model* m, tc_model_info* info);
/* Copies the ensemble to host arrays (any may be NULL):
 * depth [T], feature/bin/threshold/gain [T][max_depth], leaves [T][2^max_depth],
 * weights [T], edges [f][255] + n_edges [f]. */
tc_status tc_model_export(const tc_model* m, int32_t* depth, uint16_t* feature, uint8_t* bin,
                          float* threshold, float* gain, float* leaves, float* weights,
                          float* edges, uint16_t* n_edges);
/* Builds a device-resident model from host arrays (layouts as in export). */
tc_status tc_model_import(tc_ctx* ctx, const tc_model_info* info, const int32_t* depth,
                          const uint16_t* feature, const uint8_t* bin, const float* threshold,
                          const float* gain, const float* leaves, const float* weights,
                          const float* edges, const uint16_t* n_edges, tc_model** out);
/* TCAT v3 stream (Booster::save_binary / load_binary,
 * src/boosting/booster.cpp:1049-1203 and src/tree/symmetric_tree.cpp:1199-1239).
 * tc_model_save_tcat: pass buf = NULL to query the size.
 * tc_model_load_tcat also reads single-output models of regular (depth-wise)
 * trees (the reference's mode="small"; src/tree/tree.cpp:1748-1840): they
 * predict through tc_predict / tc_predict_device as the reference predicts
 * them (its binning against the model's edges, then the node walk) and save
 * back byte for byte; tc_model_export and tc_server_add_model refuse them. */
tc_status tc_model_save_tcat(const tc_model* m, uint8_t* buf, size_t* len);
tc_status tc_model_load_tcat(tc_ctx* ctx, const uint8_t* buf, size_t len, tc_model** out);
void tc_model_destroy(tc_model* m);

/* ------------------------------------------------------------- prediction */

/* Raw-float ensemble prediction from host buffers: X [n][f] row-major,
 * out [n][K] (K = 1 for binary/regression).  transform: TC_TRANSFORM_RAW,
 * _SIGMOID (binary probability of class 1) or _SOFTMAX (multiclass).
 * Replaces Booster::predict_raw_nobinning_fast / predict_proba_nobinning_fast
 * (src/boosting/booster.cpp:899-945) and SymmetricEnsemble::predict_batch_raw_fast
 * (src/tree/symmetric_tree.cpp:1133-1149).
 * Requests of at most 64 rows (at most 512 features, 16 classes) are served
 * by a persistent kernel of the context (a few SMs) that polls a pinned
 * mailbox, so they cost no kernel launch; it serves one model at a time
 * (restarted when another model is asked for or its model is destroyed) and
 * ends by itself after 20 ms without a request (the next one relaunches it).
 * A device-wide synchronisation therefore waits up to 20 ms after the last
 * small request.  Values are identical for identical inputs; they may differ
 * in the last bits from the same rows predicted in a larger request. */
tc_status tc_predict(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint16_t f,
                     int32_t transform, float* out);
/* Same on device buffers, queued on `stream` (a cudaStream_t, NULL = the
 * context's prediction stream, not the one training runs on); returns
 * without synchronising. */
tc_status tc_predict_device(tc_ctx* ctx, const tc_model* m, const float* X_dev, uint32_t n,
                            uint16_t f, int32_t transform, float* out_dev, void* stream);
/* Predicts a dataset's rows as the device holds them (after tc_apply_bins,
 * categorical columns hold their encodings), into host `out`
 * (Booster::predict_raw / predict_proba on a binned Dataset,
 * src/boosting/booster.cpp:587-640; a split goes right iff x >= its
 * threshold, which is bin > split bin for the training edges). */
tc_status tc_predict_dataset(tc_ctx* ctx, const tc_model* m, const tc_dataset* ds, int32_t transform,
                             float* out);

/* ---------------------------------------------------------------- serving */

typedef struct {
  size_t staging_bytes;     /* device bytes for in-flight request inputs/outputs (admission limit) */
  int32_t max_batch_rows;   /* rows per coalesced launch */
  int32_t coalesce;         /* 1: continuous batching; 0: one launch per request */
  int32_t max_inflight;     /* request slots */
} tc_server_params;

/* A request loop that keeps models resident, admits requests by staging
 * memory, and coalesces requests of uneven row counts into shared launches
 * while earlier batches are still running.  The reference has no serving
 * layer; it answers each predict_proba call synchronously
 * (python/bindings.cpp:288-382). */
tc_status tc_server_create(tc_ctx* ctx, const tc_server_params* p, tc_server** out);
tc_status tc_server_add_model(tc_server* s, const tc_model* m, int32_t* model_id);
/* Queues a request.  X and out stay owned by the caller and must stay valid
 * until tc_server_poll reports completion. */
tc_status tc_server_submit(tc_server* s, int32_t model_id, const float* X, uint32_t n, uint16_t f,
                           int32_t transform, float* out, uint64_t* ticket);
/* Waits up to timeout_us (0 = just test) for a request; *done = 1 when its
 * output is in place, and *latency_s (nullable) receives the time from
 * submission to completion measured inside the server.  A finished ticket is
 * released by the poll that reports it.  Returns TC_ERR_TIMEOUT if the
 * request is still running when the wait ends. */
tc_status tc_server_poll(tc_server* s, uint64_t ticket, int64_t timeout_us, int* done, double* latency_s);
/* Open-loop load replay: submits request i when arrival_s[i] seconds have
 * passed since the call started (spin-timed), collects every completion and
 * writes its latency (submission to completion, seconds) to latency_s[i].
 * Used by the serving benchmark so that arrival timing does not depend on
 * the caller's interpreter. */
typedef struct {
  double arrival_s;
  int32_t model_id;
  int32_t transform;
  const float* X;
  float* out;
  uint32_t n;
  uint16_t f;
  uint16_t pad;
} tc_replay_request;
tc_status tc_server_replay(tc_server* s, const tc_replay_request* reqs, int32_t n_requests, double* latency_s,
                           double* wall_s);
/* Serving statistics: requests completed, launches issued, rows served. */
tc_status tc_server_stats(tc_server* s, uint64_t* completed, uint64_t* launches, uint64_t* rows);
void tc_server_destroy(tc_server* s);

#ifdef __cplusplus
}
#endif
#endif /* TCGPU_H */
