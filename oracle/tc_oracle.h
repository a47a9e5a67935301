/*
 * CPU oracle for the TurboCat symmetric-tree training and inference path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference's
 * algorithm (ispromadhka/Turbo-Cat), used by tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg as the checker.  The product path never
 * links, loads or calls it.
 *
 * Two arithmetic modes:
 *   TCO_REF32  -- the reference's own FP32 arithmetic and summation order
 *                 (sequential row-order sums, FP32 histogram subtraction,
 *                 FP32 gains), so that splits, gains and leaf values come out
 *                 bit-identical to the reference's CPU build.  Pinned against
 *                 the reference itself (oracle/_ref, built by oracle/ref.mk)
 *                 in tests/test_oracle_pin.py.
 *   TCO_FP64   -- the same algorithm with FP64 histograms, node totals,
 *                 gains and leaf solves: the error yardstick that device
 *                 results are reported against.
 */
#ifndef TC_ORACLE_H
#define TC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCO_REF32 0
#define TCO_FP64 1

#define TCO_NAN_BIN 255
#define TCO_MAX_DEPTH 16

enum { TCO_LOSS_LOGLOSS = 0, TCO_LOSS_MSE = 1, TCO_LOSS_FOCAL = 2, TCO_LOSS_SOFTMAX = 3 };

typedef struct {
  int32_t max_depth;
  int32_t max_bins;          /* split scan covers bins 0 .. max_bins-2 */
  int32_t min_samples_leaf;
  float lambda_l2;
  float lambda_l1;
  float min_child_weight;
  float min_split_gain;
  float max_delta_step;
} tco_tree_params;

typedef struct {
  int32_t depth;
  uint16_t feature[TCO_MAX_DEPTH];
  uint8_t bin[TCO_MAX_DEPTH];
  float threshold[TCO_MAX_DEPTH];
  float gain[TCO_MAX_DEPTH];       /* FP32 (REF32) or FP64-rounded gain of the chosen split */
  double gain_top[TCO_MAX_DEPTH];  /* best total gain of the level, in the mode's arithmetic */
  double gain_second[TCO_MAX_DEPTH]; /* runner-up (next best distinct candidate) */
  uint32_t n_candidates[TCO_MAX_DEPTH];
} tco_tree;

/* Quantile binning (src/core/dataset.cpp:278-344).  X is row-major [n][f].
 * bins: column-major [f][n]; edges: [f][255]; n_edges: [f].
 * compat_u8: 1 reproduces the reference's uint8 truncation of the unique
 * count (actual_bins = min(max_bins, (uint8)U), src/core/dataset.cpp:308). */
int tco_quantize(const float* X, uint32_t n, uint32_t f, int32_t max_bins, int32_t compat_u8,
                 uint8_t* bins, float* edges, uint16_t* n_edges);

/* Losses (src/boosting/loss.cpp). */
void tco_grad_logloss(const float* y, const float* pred, float* g, float* h, uint32_t n);
void tco_grad_mse(const float* y, const float* pred, float* g, float* h, uint32_t n);
void tco_grad_focal(const float* y, const float* pred, float* g, float* h, uint32_t n, float gamma,
                    float alpha);
/* pred, g, h row-major [n][K] (src/boosting/loss.cpp:287-318). */
void tco_grad_softmax(const float* y, const float* pred, float* g, float* h, uint32_t n, uint32_t K);
float tco_init_prediction(int32_t loss, const float* y, uint32_t n);

/* One symmetric tree (src/tree/symmetric_tree.cpp:34-368) over all rows.
 * leaf_values: [2^max_depth]; leaf_index (nullable): [n], the per-row leaf
 * after the final accepted level.  root_hist (nullable): [f][256][2] FP64
 * (grad, hess) of the root level, slot 255 holding NaN rows. */
int tco_build_tree(const uint8_t* bins, uint32_t n, uint32_t f, const float* edges,
                   const uint16_t* n_edges, const float* g, const float* h,
                   const tco_tree_params* p, int32_t mode, tco_tree* out, float* leaf_values,
                   uint32_t* leaf_index, double* root_hist);
/* The same over the rows of `rows0` (n0 of them, in that order: FP32 sums
 * follow the list order); rows0 = NULL: all rows. */
int tco_build_tree_rows(const uint8_t* bins, uint32_t n, uint32_t f, const float* edges,
                        const uint16_t* n_edges, const float* g, const float* h,
                        const tco_tree_params* p, int32_t mode, const uint32_t* rows0, uint32_t n0,
                        tco_tree* out, float* leaf_values, uint32_t* leaf_index, double* root_hist);

/* FP64 level histograms for an arbitrary node assignment: out[node][f][256][2]. */
void tco_histogram(const uint8_t* bins, uint32_t n, uint32_t f, const float* g, const float* h,
                   const uint32_t* node_of_row, uint32_t n_nodes, double* out);

/* Full fit (Booster::train, src/boosting/booster.cpp:47-252, and the
 * composed symmetric multiclass loop).  bins/edges from tco_quantize.
 * Trees are written iteration-major, class-minor: T = n_estimators * K.
 * depth: [T]; feature/bin/threshold: [T][max_depth]; leaves [T][2^max_depth].
 * train_pred (nullable): raw scores [n][K] after the last tree.
 * gain (nullable): [T][max_depth] split gains; grad_trace / hess_trace
 * (nullable): [n_estimators][n][K] gradients of every iteration. */
typedef struct {
  int32_t loss;
  int32_t n_classes;  /* K for softmax, else 1 */
  int32_t n_estimators;
  float learning_rate;
  float focal_gamma;
  float focal_alpha;
  tco_tree_params tree;
  /* row sampling (src/boosting/booster.cpp:198-228): subsample < 1 builds
   * each iteration's trees on the rows random_subsample picks (in its
   * order); colsample_bytree < 1 only advances the random state (the
   * symmetric build ignores the feature subset); seed = Config::seed. */
  float subsample;
  float colsample_bytree;
  uint64_t seed;
  /* GOSS (Dataset::goss_subsample, src/core/dataset.cpp:494-549), chosen
   * over subsample (booster.cpp:200-219): each iteration's rows from its
   * gradients (softmax: the largest |g| over the classes,
   * booster.cpp:1327-1348) and one next_random() draw. */
  int32_t use_goss;
  float goss_top_rate;
  float goss_other_rate;
} tco_fit_params;

/* xorshift64* step (src/boosting/booster.cpp:1219-1225). */
uint64_t tco_next_random(uint64_t* state);
/* src/core/dataset.cpp:552-562: writes the first (uint32)(n * ratio)
 * shuffled row ids to out, returns their count. */
uint32_t tco_random_subsample(uint32_t n, float ratio, uint64_t seed, uint32_t* out);
/* src/core/dataset.cpp:494-549 over per-row |g| values: writes the sampled
 * row ids in the reference's order, returns their count. */
uint32_t tco_goss_subsample(uint32_t n, const float* absg, float top_rate, float other_rate, uint64_t seed,
                            uint32_t* out);

int tco_fit(const uint8_t* bins, uint32_t n, uint32_t f, const float* edges,
            const uint16_t* n_edges, const float* y, const tco_fit_params* p, int32_t mode,
            float* base_out, int32_t* depth, uint16_t* feature, uint8_t* bin, float* threshold,
            float* leaves, float* train_pred, double* min_margin_out, float* gain,
            float* grad_trace, float* hess_trace);

/* Raw-float ensemble prediction in FP64 (the FastFloatEnsemble rule,
 * include/turbocat/fast_float_ensemble.hpp:122-137: go right iff x is not NaN
 * and x >= threshold).  Trees of class t % K add into column t % K.
 * out: [n][K] raw scores (base added). */
void tco_predict(const float* X, uint32_t n, uint32_t f, int32_t n_trees, int32_t K,
                 int32_t max_depth, const int32_t* depth, const uint16_t* feature,
                 const float* threshold, const float* leaves, const float* weights, float base,
                 double* out);

#ifdef __cplusplus
}
#endif
#endif
