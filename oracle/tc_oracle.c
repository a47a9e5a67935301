/*
 * CPU oracle for the TurboCat symmetric-tree path -- TEST INFRASTRUCTURE ONLY
 * (see tc_oracle.h).  Each function cites the reference file:line it
 * restates.  Built with -ffp-contract=off: every fused multiply-add that the
 * reference's compiled code performs is written out here with fmaf(), so the
 * REF32 mode reproduces the reference bit for bit (pinned by
 * tests/test_oracle_pin.py against the reference build in oracle/_ref).
 */
#include "tc_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Binning: src/core/dataset.cpp:278-344                                      */
/* ------------------------------------------------------------------------ */

static int cmp_float(const void* a, const void* b) {
  const float x = *(const float*)a, y = *(const float*)b;
  return (x < y) ? -1 : (x > y) ? 1 : 0;
}

/* std::upper_bound(edges, edges+m, v) - edges  (src/core/dataset.cpp:336-344) */
static uint8_t upper_bound_bin(const float* e, uint32_t m, float v) {
  uint32_t lo = 0, hi = m;
  while (lo < hi) {
    const uint32_t mid = (lo + hi) >> 1;
    if (v < e[mid]) hi = mid; else lo = mid + 1;
  }
  return (uint8_t)lo;
}

int tco_quantize(const float* X, uint32_t n, uint32_t f, int32_t max_bins, int32_t compat_u8,
                 uint8_t* bins, float* edges, uint16_t* n_edges) {
  if (max_bins < 2 || max_bins > 255) return -1;
  int err = 0;
#pragma omp parallel for schedule(dynamic)
  for (int64_t jj = 0; jj < (int64_t)f; ++jj) {
    const uint32_t j = (uint32_t)jj;
    float* v = (float*)malloc((size_t)(n ? n : 1) * sizeof(float));
    if (!v) { err = -2; continue; }
    uint32_t m = 0;
    for (uint32_t i = 0; i < n; ++i) {
      const float x = X[(size_t)i * f + j];
      if (!isnan(x)) v[m++] = x;
    }
    float* ej = edges + (size_t)j * 255;
    uint8_t* bj = bins + (size_t)j * n;
    if (m == 0) {
      /* all NaN: one edge {0.0f}, every row in the NaN bin (dataset.cpp:296-303) */
      ej[0] = 0.0f;
      n_edges[j] = 1;
      for (uint32_t i = 0; i < n; ++i) bj[i] = (uint8_t)max_bins;
      free(v);
      continue;
    }
    qsort(v, m, sizeof(float), cmp_float);
    /* std::unique with operator== (so -0.0 and +0.0 merge) */
    uint32_t u = 1;
    for (uint32_t i = 1; i < m; ++i) {
      if (!(v[i] == v[u - 1])) v[u++] = v[i];
    }
    /* actual_bins = min(n_bins, (BinIndex)values.size())  (dataset.cpp:308) */
    uint32_t a = compat_u8 ? (uint32_t)(uint8_t)u : u;
    if (a > (uint32_t)max_bins) a = (uint32_t)max_bins;
    uint32_t ne = 0;
    for (uint32_t b = 1; b < a; ++b) {
      const size_t idx = (size_t)b * u / a;
      if (ne == 0 || v[idx] > ej[ne - 1]) ej[ne++] = v[idx];
    }
    n_edges[j] = (uint16_t)ne;
    for (uint32_t i = 0; i < n; ++i) {
      const float x = X[(size_t)i * f + j];
      /* NaN rows take the NaN bin; the reference writes n_bins there
       * (dataset.cpp:328), which equals 255 for the default max_bins. */
      bj[i] = isnan(x) ? (uint8_t)TCO_NAN_BIN : upper_bound_bin(ej, ne, x);
    }
    free(v);
  }
  return err;
}

/* ------------------------------------------------------------------------ */
/* Losses: src/boosting/loss.cpp                                              */
/* ------------------------------------------------------------------------ */

static inline float maxps(float a, float b) { return a > b ? a : b; }
static inline float minps(float a, float b) { return a < b ? a : b; }

/* fast_exp_avx2 lane arithmetic (loss.cpp:34-69): degree-5 polynomial for
 * 2^frac after a round-to-nearest split of x*log2(e). */
static float ref_fast_exp(float x) {
  x = maxps(x, -88.0f);
  x = minps(x, 88.0f);
  const float t = x * 1.4426950408889634f;
  const float ti = nearbyintf(t);
  const float tf = t - ti;
  float poly = fmaf(0.0013333558146428443f, tf, 0.009618129107628477f);
  poly = fmaf(poly, tf, 0.05550410866482046f);
  poly = fmaf(poly, tf, 0.2402265069591007f);
  poly = fmaf(poly, tf, 0.6931471805599453f);
  poly = fmaf(poly, tf, 1.0f);
  const int32_t e = ((int32_t)ti + 127) << 23;
  float pow2;
  memcpy(&pow2, &e, sizeof(pow2));
  return poly * pow2;
}

/* fast_sigmoid_avx2 (loss.cpp:71-82) */
static float ref_fast_sigmoid(float x) {
  x = maxps(x, -15.0f);
  x = minps(x, 15.0f);
  const float ex = ref_fast_exp(0.0f - x);
  return 1.0f / (1.0f + ex);
}

/* LogLoss::compute_gradients (loss.cpp:123-211): the AVX2 body covers the
 * first floor(n/8)*8 rows, the scalar std::exp tail the rest. */
void tco_grad_logloss(const float* y, const float* pred, float* g, float* h, uint32_t n) {
  const uint32_t nv = (n / 8) * 8;
  for (uint32_t i = 0; i < nv; ++i) {
    const float p = ref_fast_sigmoid(pred[i]);
    g[i] = p - y[i];
    const float hh = p * (1.0f - p);
    h[i] = maxps(hh, 1e-6f);
  }
  for (uint32_t i = nv; i < n; ++i) {
    const float pr = fmaxf(-15.0f, fminf(15.0f, pred[i]));
    const float p = 1.0f / (1.0f + expf(-pr));
    g[i] = p - y[i];
    h[i] = fmaxf(p * (1.0f - p), 1e-6f);
  }
}

/* MSELoss::compute_gradients (loss.cpp:348-362) */
void tco_grad_mse(const float* y, const float* pred, float* g, float* h, uint32_t n) {
  for (uint32_t i = 0; i < n; ++i) {
    g[i] = 2.0f * (pred[i] - y[i]);
    h[i] = 2.0f;
  }
}

/* RobustFocalLoss::compute_gradients (loss.cpp:505-539), class weights 1. */
void tco_grad_focal(const float* y, const float* pred, float* g, float* h, uint32_t n, float gamma,
                    float alpha) {
  for (uint32_t i = 0; i < n; ++i) {
    const float p = 1.0f / (1.0f + expf(-pred[i]));
    const float yy = y[i];
    /* y*p + (1-y)*(1-p): exact for y in {0,1} whichever product is fused */
    float pt = fmaf(yy, p, (1.0f - yy) * (1.0f - p));
    pt = fmaxf(pt, 1e-7f);
    const float at = fmaf(yy, alpha, (1.0f - yy) * (1.0f - alpha));
    const float cw = fmaf(yy, 1.0f, (1.0f - yy) * 1.0f);
    const float fw = powf(1.0f - pt, gamma);
    const float coef = at * cw * fw;
    g[i] = coef * (p - yy);
    const float hh = coef * p * (1.0f - p);
    h[i] = fmaxf(hh, 1e-6f);
  }
}

/* CrossEntropyLoss::compute_multiclass_gradients + softmax (loss.cpp:273-318) */
void tco_grad_softmax(const float* y, const float* pred, float* g, float* h, uint32_t n, uint32_t K) {
  float pr[256];
  for (uint32_t i = 0; i < n; ++i) {
    const float* in = pred + (size_t)i * K;
    float mx = in[0];
    for (uint32_t c = 1; c < K; ++c) if (mx < in[c]) mx = in[c];
    float sum = 0.0f;
    for (uint32_t c = 0; c < K; ++c) {
      pr[c] = expf(in[c] - mx);
      sum += pr[c];
    }
    for (uint32_t c = 0; c < K; ++c) pr[c] /= sum;
    const uint32_t label = (uint32_t)y[i];
    for (uint32_t c = 0; c < K; ++c) {
      const float p = pr[c];
      const float t = (c == label) ? 1.0f : 0.0f;
      g[(size_t)i * K + c] = p - t;
      h[(size_t)i * K + c] = fmaxf(p * (1.0f - p), 1e-6f);
    }
  }
}

/* Loss::init_prediction: LogLoss loss.cpp:217-226, MSE loss.cpp:364-370,
 * RobustFocal loss.cpp:545-553, CrossEntropy loss.cpp:269-271. */
float tco_init_prediction(int32_t loss, const float* y, uint32_t n) {
  if (loss == TCO_LOSS_SOFTMAX) return 0.0f;
  float sum = 0.0f;
  for (uint32_t i = 0; i < n; ++i) sum += y[i];
  float p = sum / (float)n;
  if (loss == TCO_LOSS_MSE) return p;
  p = fmaxf(1e-7f, fminf(1.0f - 1e-7f, p));
  return logf(p / (1.0f - p));
}

/* ------------------------------------------------------------------------ */
/* Histograms and the symmetric level build: src/tree/symmetric_tree.cpp      */
/* ------------------------------------------------------------------------ */

typedef struct { float g, h; uint32_t c; } hb32;
typedef struct { double g, h; uint32_t c; } hb64;

/* CPUHistogramBuilder::build / build_feature_scalar (histogram.cpp:62-205,
 * 307-378): per feature, rows in list order, FP32 running sums per bin.
 * NaN rows go to slot 255 of the feature's own 256-slot row. */
static void hist32(const uint8_t* bins, uint32_t n, uint32_t f, const float* g, const float* h,
                   const uint32_t* rows, uint32_t nr, hb32* out) {
  memset(out, 0, (size_t)f * 256 * sizeof(hb32));
#pragma omp parallel for schedule(static)
  for (int64_t jj = 0; jj < (int64_t)f; ++jj) {
    const uint8_t* col = bins + (size_t)jj * n;
    hb32* o = out + (size_t)jj * 256;
    for (uint32_t k = 0; k < nr; ++k) {
      const uint32_t r = rows[k];
      const uint8_t b = col[r];
      o[b].g += g[r];
      o[b].h += h[r];
      o[b].c += 1;
    }
  }
}

static void hist64(const uint8_t* bins, uint32_t n, uint32_t f, const float* g, const float* h,
                   const uint32_t* rows, uint32_t nr, hb64* out) {
  memset(out, 0, (size_t)f * 256 * sizeof(hb64));
#pragma omp parallel for schedule(static)
  for (int64_t jj = 0; jj < (int64_t)f; ++jj) {
    const uint8_t* col = bins + (size_t)jj * n;
    hb64* o = out + (size_t)jj * 256;
    for (uint32_t k = 0; k < nr; ++k) {
      const uint32_t r = rows[k];
      const uint8_t b = col[r];
      o[b].g += (double)g[r];
      o[b].h += (double)h[r];
      o[b].c += 1;
    }
  }
}

void tco_histogram(const uint8_t* bins, uint32_t n, uint32_t f, const float* g, const float* h,
                   const uint32_t* node_of_row, uint32_t n_nodes, double* out) {
  memset(out, 0, (size_t)n_nodes * f * 256 * 2 * sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t jj = 0; jj < (int64_t)f; ++jj) {
    const uint8_t* col = bins + (size_t)jj * n;
    for (uint32_t r = 0; r < n; ++r) {
      const uint32_t nd = node_of_row[r];
      if (nd >= n_nodes) continue;
      double* o = out + (((size_t)nd * f + (size_t)jj) * 256 + col[r]) * 2;
      o[0] += (double)g[r];
      o[1] += (double)h[r];
    }
  }
}

/* SymmetricTree::compute_leaf_value (symmetric_tree.cpp:753-775) */
static float leaf32(float G, float H, const tco_tree_params* p) {
  if (H < 1e-10f) return 0.0f;
  float v = -G / (H + p->lambda_l2);
  if (p->lambda_l1 > 0) {
    if (v > p->lambda_l1) v -= p->lambda_l1;
    else if (v < -p->lambda_l1) v += p->lambda_l1;
    else v = 0.0f;
  }
  if (p->max_delta_step > 0) v = fmaxf(-p->max_delta_step, fminf(p->max_delta_step, v));
  return v;
}

static float leaf64(double G, double H, const tco_tree_params* p) {
  if (H < 1e-10) return 0.0f;
  double v = -G / (H + (double)p->lambda_l2);
  const double l1 = (double)p->lambda_l1;
  if (l1 > 0) {
    if (v > l1) v -= l1;
    else if (v < -l1) v += l1;
    else v = 0.0;
  }
  const double md = (double)p->max_delta_step;
  if (md > 0) v = fmax(-md, fmin(md, v));
  return (float)v;
}

/* Track the best and the runner-up candidate of a level.  The reference
 * keeps the first (lowest feature, then lowest bin) of equal gains: a
 * candidate replaces the best only when strictly greater
 * (symmetric_tree.cpp:163-193, 240-262). */
typedef struct {
  double top, second;
  int32_t f, b;
  float top32;
  uint32_t n;
} best_t;

static void best_push(best_t* s, double gain, float gain32, int32_t f, int32_t b) {
  s->n++;
  if (gain > s->top) {
    s->second = s->top;
    s->top = gain;
    s->top32 = gain32;
    s->f = f;
    s->b = b;
  } else if (gain > s->second) {
    s->second = gain;
  }
}

int tco_build_tree(const uint8_t* bins, uint32_t n, uint32_t f, const float* edges,
                   const uint16_t* n_edges, const float* g, const float* h,
                   const tco_tree_params* p, int32_t mode, tco_tree* out, float* leaf_values,
                   uint32_t* leaf_index, double* root_hist) {
  return tco_build_tree_rows(bins, n, f, edges, n_edges, g, h, p, mode, NULL, n, out, leaf_values,
                             leaf_index, root_hist);
}

int tco_build_tree_rows(const uint8_t* bins, uint32_t n, uint32_t f, const float* edges,
                        const uint16_t* n_edges, const float* g, const float* h,
                        const tco_tree_params* p, int32_t mode, const uint32_t* rows0, uint32_t n0,
                        tco_tree* out, float* leaf_values, uint32_t* leaf_index, double* root_hist) {
  const int32_t D = p->max_depth;
  if (D < 0 || D > TCO_MAX_DEPTH) return -1;
  const uint32_t max_nodes = 1u << D;
  const int32_t nb_scan = (int32_t)(uint8_t)p->max_bins - 1; /* b < max_bins-1 */
  const float lam = p->lambda_l2;
  const double lam64 = (double)p->lambda_l2;
  memset(out, 0, sizeof(*out));

  /* node row lists: stable (row-ascending) per node */
  uint32_t* rows_cur = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
  uint32_t* rows_nxt = (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t));
  uint32_t* start = (uint32_t*)calloc((size_t)max_nodes * 2 + 1, sizeof(uint32_t));
  uint32_t* cnt = (uint32_t*)calloc((size_t)max_nodes * 2, sizeof(uint32_t));
  uint32_t* nstart = (uint32_t*)calloc((size_t)max_nodes * 2 + 1, sizeof(uint32_t));
  uint32_t* ncnt = (uint32_t*)calloc((size_t)max_nodes * 2, sizeof(uint32_t));
  float* sg32 = (float*)calloc((size_t)max_nodes * 2, sizeof(float));
  float* sh32 = (float*)calloc((size_t)max_nodes * 2, sizeof(float));
  double* sg64 = (double*)calloc((size_t)max_nodes * 2, sizeof(double));
  double* sh64 = (double*)calloc((size_t)max_nodes * 2, sizeof(double));
  float* ng32 = (float*)calloc((size_t)max_nodes * 2, sizeof(float));
  float* nh32 = (float*)calloc((size_t)max_nodes * 2, sizeof(float));
  double* ng64 = (double*)calloc((size_t)max_nodes * 2, sizeof(double));
  double* nh64 = (double*)calloc((size_t)max_nodes * 2, sizeof(double));
  const size_t hsz = (size_t)f * 256;
  hb32* H32 = NULL; hb32* N32 = NULL;
  hb64* H64 = NULL; hb64* N64 = NULL;
  if (mode == TCO_REF32) {
    H32 = (hb32*)calloc(hsz * max_nodes, sizeof(hb32));
    N32 = (hb32*)calloc(hsz * max_nodes, sizeof(hb32));
  } else {
    H64 = (hb64*)calloc(hsz * max_nodes, sizeof(hb64));
    N64 = (hb64*)calloc(hsz * max_nodes, sizeof(hb64));
  }
  int rc = 0;
  if (!rows_cur || !rows_nxt || !start || !cnt || (!H32 && !H64) || (!N32 && !N64)) { rc = -2; goto done; }

  if (!rows0) n0 = n;
  for (uint32_t i = 0; i < n0; ++i) rows_cur[i] = rows0 ? rows0[i] : i;
  start[0] = 0;
  cnt[0] = n0;
  {
    float G = 0.0f, H = 0.0f;
    double G64 = 0.0, H64s = 0.0;
    for (uint32_t q = 0; q < n0; ++q) {
      const uint32_t i = rows_cur[q];
      G += g[i]; H += h[i];
      G64 += (double)g[i]; H64s += (double)h[i];
    }
    sg32[0] = G; sh32[0] = H; sg64[0] = G64; sh64[0] = H64s;
  }

  int32_t depth = 0;
  for (int32_t d = 0; d < D; ++d) {
    const uint32_t nn = 1u << d;
    /* stop rule (symmetric_tree.cpp:116-124) */
    int stop = 1;
    for (uint32_t k = 0; k < nn; ++k) {
      const double hs = (mode == TCO_REF32) ? (double)sh32[k] : sh64[k];
      const int hess_ok = (mode == TCO_REF32) ? (sh32[k] >= p->min_child_weight * 2)
                                              : (hs >= (double)(p->min_child_weight * 2));
      if (cnt[k] >= (uint32_t)p->min_samples_leaf * 2u && hess_ok) { stop = 0; break; }
    }
    if (stop) break;

    if (d == 0) {
      if (mode == TCO_REF32) hist32(bins, n, f, g, h, rows_cur, n0, H32);
      else hist64(bins, n, f, g, h, rows_cur, n0, H64);
      if (root_hist) {
        for (size_t q = 0; q < hsz; ++q) {
          root_hist[2 * q] = mode == TCO_REF32 ? (double)H32[q].g : H64[q].g;
          root_hist[2 * q + 1] = mode == TCO_REF32 ? (double)H32[q].h : H64[q].h;
        }
      }
    }

    /* level scan (symmetric_tree.cpp:135-262) */
    best_t best = {-1e30, -1e30, -1, -1, -1e30f, 0};
    if (mode == TCO_REF32) {
      float pg[1u << TCO_MAX_DEPTH];
      for (uint32_t k = 0; k < nn; ++k) {
        pg[k] = 0.0f;
        if (sh32[k] > 1e-10f) pg[k] = (sg32[k] * sg32[k]) / (sh32[k] + lam);
      }
      float lg[1u << TCO_MAX_DEPTH], lh[1u << TCO_MAX_DEPTH];
      for (uint32_t j = 0; j < f; ++j) {
        for (uint32_t k = 0; k < nn; ++k) {
          const hb32* o = H32 + ((size_t)k * f + j) * 256;
          lg[k] = o[TCO_NAN_BIN].g;  /* NaN rows route left */
          lh[k] = o[TCO_NAN_BIN].h;
        }
        for (int32_t b = 0; b < nb_scan; ++b) {
          if (d == 0) {
            const hb32* o = H32 + (size_t)j * 256;
            lg[0] += o[b].g;
            lh[0] += o[b].h;
            const float rg = sg32[0] - lg[0];
            const float rh = sh32[0] - lh[0];
            if (lh[0] < 1e-10f || rh < 1e-10f) continue;
            const float lgain = (lg[0] * lg[0]) / (lh[0] + lam);
            const float rgain = (rg * rg) / (rh + lam);
            const float gain = 0.5f * (lgain + rgain - pg[0]);
            best_push(&best, (double)gain, gain, (int32_t)j, b);
          } else {
            float total = 0.0f;
            for (uint32_t k = 0; k < nn; ++k) {
              const hb32* o = H32 + ((size_t)k * f + j) * 256;
              lg[k] += o[b].g;
              lh[k] += o[b].h;
              if (cnt[k] == 0) continue;
              const float rg = sg32[k] - lg[k];
              const float rh = sh32[k] - lh[k];
              if (lh[k] < 1e-10f || rh < 1e-10f) continue;
              const float lgain = (lg[k] * lg[k]) / (lh[k] + lam);
              const float rgain = (rg * rg) / (rh + lam);
              /* total_gain += 0.5f * (...): contracted to an FMA by the
               * reference's -O3 -mfma build */
              total = fmaf(0.5f, lgain + rgain - pg[k], total);
            }
            best_push(&best, (double)total, total, (int32_t)j, b);
          }
        }
      }
    } else {
      double pg[1u << TCO_MAX_DEPTH];
      for (uint32_t k = 0; k < nn; ++k) {
        pg[k] = 0.0;
        if (sh64[k] > 1e-10) pg[k] = (sg64[k] * sg64[k]) / (sh64[k] + lam64);
      }
      double* sufg = (double*)malloc((size_t)nn * 257 * sizeof(double));
      double* sufh = (double*)malloc((size_t)nn * 257 * sizeof(double));
      double lg[1u << TCO_MAX_DEPTH], lh[1u << TCO_MAX_DEPTH];
      for (uint32_t j = 0; j < f; ++j) {
        /* suffix sums over regular bins so an empty side is exactly zero */
        for (uint32_t k = 0; k < nn; ++k) {
          const hb64* o = H64 + ((size_t)k * f + j) * 256;
          double* sgk = sufg + (size_t)k * 257;
          double* shk = sufh + (size_t)k * 257;
          sgk[255] = 0.0; shk[255] = 0.0;
          for (int32_t b = 254; b >= 0; --b) { sgk[b] = sgk[b + 1] + o[b].g; shk[b] = shk[b + 1] + o[b].h; }
          lg[k] = o[TCO_NAN_BIN].g;
          lh[k] = o[TCO_NAN_BIN].h;
        }
        for (int32_t b = 0; b < nb_scan; ++b) {
          double total = 0.0;
          int any = 0;
          for (uint32_t k = 0; k < nn; ++k) {
            const hb64* o = H64 + ((size_t)k * f + j) * 256;
            lg[k] += o[b].g;
            lh[k] += o[b].h;
            if (cnt[k] == 0) continue;
            const double rg = sufg[(size_t)k * 257 + b + 1];
            const double rh = sufh[(size_t)k * 257 + b + 1];
            if (lh[k] < 1e-10 || rh < 1e-10) continue;
            total += 0.5 * ((lg[k] * lg[k]) / (lh[k] + lam64) + (rg * rg) / (rh + lam64) - pg[k]);
            any = 1;
          }
          if (d == 0 && !any) continue;
          best_push(&best, total, (float)total, (int32_t)j, b);
        }
      }
      free(sufg);
      free(sufh);
    }

    out->n_candidates[d] = best.n;
    out->gain_top[d] = best.top;
    out->gain_second[d] = best.second;
    if (best.f < 0) break;                                   /* no candidate: gain -1e30 */
    if (best.top32 < p->min_split_gain) break;               /* symmetric_tree.cpp:276-278 */
    float thr = 0.0f;
    if ((uint32_t)best.f < f) {
      const uint16_t ne = n_edges[best.f];
      if ((uint32_t)best.b < ne) thr = edges[(size_t)best.f * 255 + best.b];
      else if (ne > 0) thr = edges[(size_t)best.f * 255 + ne - 1];
    }
    out->feature[d] = (uint16_t)best.f;
    out->bin[d] = (uint8_t)best.b;
    out->threshold[d] = thr;
    out->gain[d] = best.top32;
    depth = d + 1;

    /* partition (symmetric_tree.cpp:287-327): left iff NaN or bin <= t */
    const uint8_t* col = bins + (size_t)best.f * n;
    const uint8_t t = (uint8_t)best.b;
    uint32_t pos = 0;
    for (uint32_t k = 0; k < nn; ++k) {
      float lg32 = 0.0f, lh32 = 0.0f, rg32 = 0.0f, rh32 = 0.0f;
      double lg64 = 0.0, lh64 = 0.0, rg64 = 0.0, rh64 = 0.0;
      const uint32_t l = 2 * k, r = 2 * k + 1;
      nstart[l] = pos;
      for (uint32_t q = 0; q < cnt[k]; ++q) {
        const uint32_t row = rows_cur[start[k] + q];
        const uint8_t b = col[row];
        if (b == TCO_NAN_BIN || b <= t) {
          rows_nxt[pos++] = row;
          lg32 += g[row]; lh32 += h[row]; lg64 += g[row]; lh64 += h[row];
        }
      }
      ncnt[l] = pos - nstart[l];
      nstart[r] = pos;
      for (uint32_t q = 0; q < cnt[k]; ++q) {
        const uint32_t row = rows_cur[start[k] + q];
        const uint8_t b = col[row];
        if (!(b == TCO_NAN_BIN || b <= t)) {
          rows_nxt[pos++] = row;
          rg32 += g[row]; rh32 += h[row]; rg64 += g[row]; rh64 += h[row];
        }
      }
      ncnt[r] = pos - nstart[r];
      ng32[l] = lg32; nh32[l] = lh32; ng32[r] = rg32; nh32[r] = rh32;
      ng64[l] = lg64; nh64[l] = lh64; ng64[r] = rg64; nh64[r] = rh64;
    }

    /* histogram of the smaller child, larger = parent - smaller
     * (symmetric_tree.cpp:329-349); left is "smaller" on a tie */
    if (depth < D) {
      for (uint32_t k = 0; k < nn; ++k) {
        const uint32_t l = 2 * k, r = 2 * k + 1;
        const int left_small = ncnt[l] <= ncnt[r];
        const uint32_t sm = left_small ? l : r, lg_ = left_small ? r : l;
        if (mode == TCO_REF32) {
          hb32* hs = N32 + (size_t)sm * hsz;
          hb32* hl = N32 + (size_t)lg_ * hsz;
          const hb32* hp = H32 + (size_t)k * hsz;
          if (ncnt[sm] > 0) hist32(bins, n, f, g, h, rows_nxt + nstart[sm], ncnt[sm], hs);
          else memset(hs, 0, hsz * sizeof(hb32));
          for (size_t q = 0; q < hsz; ++q) {
            hl[q].g = hp[q].g - hs[q].g;
            hl[q].h = hp[q].h - hs[q].h;
            hl[q].c = hp[q].c - hs[q].c;
          }
        } else {
          hb64* hs = N64 + (size_t)sm * hsz;
          hb64* hl = N64 + (size_t)lg_ * hsz;
          const hb64* hp = H64 + (size_t)k * hsz;
          if (ncnt[sm] > 0) hist64(bins, n, f, g, h, rows_nxt + nstart[sm], ncnt[sm], hs);
          else memset(hs, 0, hsz * sizeof(hb64));
          for (size_t q = 0; q < hsz; ++q) {
            hl[q].g = hp[q].g - hs[q].g;
            hl[q].h = hp[q].h - hs[q].h;
            hl[q].c = hp[q].c - hs[q].c;
          }
        }
      }
    }
    /* swap level state */
    { uint32_t* t2 = rows_cur; rows_cur = rows_nxt; rows_nxt = t2; }
    { uint32_t* t2 = start; start = nstart; nstart = t2; }
    { uint32_t* t2 = cnt; cnt = ncnt; ncnt = t2; }
    { float* t2 = sg32; sg32 = ng32; ng32 = t2; }
    { float* t2 = sh32; sh32 = nh32; nh32 = t2; }
    { double* t2 = sg64; sg64 = ng64; ng64 = t2; }
    { double* t2 = sh64; sh64 = nh64; nh64 = t2; }
    if (mode == TCO_REF32) { hb32* t2 = H32; H32 = N32; N32 = t2; }
    else { hb64* t2 = H64; H64 = N64; N64 = t2; }
  }
  out->depth = depth;

  /* leaf values (symmetric_tree.cpp:357-367) */
  {
    const uint32_t nl = 1u << depth;
    for (uint32_t k = 0; k < nl; ++k) {
      leaf_values[k] = (mode == TCO_REF32) ? leaf32(sg32[k], sh32[k], p) : leaf64(sg64[k], sh64[k], p);
    }
    if (leaf_index) {
      for (uint32_t k = 0; k < nl; ++k)
        for (uint32_t q = 0; q < cnt[k]; ++q) leaf_index[rows_cur[start[k] + q]] = k;
    }
  }

done:
  free(rows_cur); free(rows_nxt); free(start); free(cnt); free(nstart); free(ncnt);
  free(sg32); free(sh32); free(sg64); free(sh64); free(ng32); free(nh32); free(ng64); free(nh64);
  free(H32); free(N32); free(H64); free(N64);
  return rc;
}

/* ------------------------------------------------------------------------ */
/* Boosting loop: src/boosting/booster.cpp:47-252, 438-463                   */
/* ------------------------------------------------------------------------ */

int tco_fit(const uint8_t* bins, uint32_t n, uint32_t f, const float* edges,
            const uint16_t* n_edges, const float* y, const tco_fit_params* p, int32_t mode,
            float* base_out, int32_t* depth, uint16_t* feature, uint8_t* bin, float* threshold,
            float* leaves, float* train_pred, double* min_margin_out, float* gain,
            float* grad_trace, float* hess_trace) {
  const uint32_t K = (p->loss == TCO_LOSS_SOFTMAX) ? (uint32_t)p->n_classes : 1u;
  const int32_t D = p->tree.max_depth;
  const uint32_t L = 1u << D;
  const float base = tco_init_prediction(p->loss, y, n);
  *base_out = base;
  float* pred = (float*)malloc((size_t)n * K * sizeof(float));
  float* gg = (float*)malloc((size_t)n * K * sizeof(float));
  float* hh = (float*)malloc((size_t)n * K * sizeof(float));
  float* gk = (float*)malloc((size_t)n * sizeof(float));
  float* hk = (float*)malloc((size_t)n * sizeof(float));
  uint32_t* li = (uint32_t*)malloc((size_t)n * sizeof(uint32_t));
  float* lv = (float*)malloc((size_t)L * sizeof(float));
  if (!pred || !gg || !hh || !gk || !hk || !li || !lv) return -2;
  for (size_t i = 0; i < (size_t)n * K; ++i) pred[i] = base;
  double min_margin = 1e300;
  int rc = 0;
  size_t t = 0;
  uint64_t rng = p->seed;
  const int goss = p->use_goss != 0;
  const int sampling = goss || p->subsample < 1.0f;
  uint32_t* sample = sampling ? (uint32_t*)malloc((size_t)(n ? n : 1) * sizeof(uint32_t)) : NULL;
  float* absg = goss ? (float*)malloc((size_t)(n ? n : 1) * sizeof(float)) : NULL;
  for (int32_t it = 0; it < p->n_estimators; ++it) {
    if (p->loss == TCO_LOSS_LOGLOSS) tco_grad_logloss(y, pred, gg, hh, n);
    else if (p->loss == TCO_LOSS_MSE) tco_grad_mse(y, pred, gg, hh, n);
    else if (p->loss == TCO_LOSS_FOCAL) tco_grad_focal(y, pred, gg, hh, n, p->focal_gamma, p->focal_alpha);
    else tco_grad_softmax(y, pred, gg, hh, n, K);
    /* sample selection after the gradients (booster.cpp:198-228): GOSS or
     * the random subsample, then one draw for the feature subset, which the
     * symmetric build does not use */
    uint32_t n_sample = n;
    if (goss) {
      for (uint32_t i = 0; i < n; ++i) {
        float m = 0.0f; /* max |g| over the classes, from 0 (booster.cpp:1333-1339) */
        for (uint32_t k = 0; k < K; ++k) {
          const float a = fabsf(gg[(size_t)i * K + k]);
          m = a > m ? a : m;
        }
        absg[i] = m;
      }
      n_sample = tco_goss_subsample(n, absg, p->goss_top_rate, p->goss_other_rate, tco_next_random(&rng), sample);
    } else if (sampling) {
      n_sample = tco_random_subsample(n, p->subsample, tco_next_random(&rng), sample);
    }
    if (p->colsample_bytree < 1.0f) (void)tco_next_random(&rng);
    if (grad_trace) memcpy(grad_trace + (size_t)it * n * K, gg, (size_t)n * K * sizeof(float));
    if (hess_trace) memcpy(hess_trace + (size_t)it * n * K, hh, (size_t)n * K * sizeof(float));
    for (uint32_t k = 0; k < K; ++k, ++t) {
      const float* gsrc = gg;
      const float* hsrc = hh;
      if (K > 1) {
        for (uint32_t i = 0; i < n; ++i) { gk[i] = gg[(size_t)i * K + k]; hk[i] = hh[(size_t)i * K + k]; }
        gsrc = gk; hsrc = hk;
      }
      tco_tree tr;
      memset(lv, 0, (size_t)L * sizeof(float));
      rc = tco_build_tree_rows(bins, n, f, edges, n_edges, gsrc, hsrc, &p->tree, mode, sample, n_sample, &tr, lv,
                               li, NULL);
      if (rc) goto done;
      if (sampling) {
        /* every row's leaf (SymmetricTree::predict_batch on the bins,
         * src/tree/symmetric_tree.cpp:813-840): bin != 255 && bin > t goes right */
        for (uint32_t i = 0; i < n; ++i) {
          uint32_t idx = 0;
          for (int32_t d = 0; d < tr.depth; ++d) {
            const uint8_t b = bins[(size_t)tr.feature[d] * n + i];
            idx = (idx << 1) | (uint32_t)(b != TCO_NAN_BIN && b > tr.bin[d]);
          }
          li[i] = idx;
        }
      }
      depth[t] = tr.depth;
      for (int32_t d = 0; d < D; ++d) {
        feature[t * D + d] = d < tr.depth ? tr.feature[d] : 0;
        bin[t * D + d] = d < tr.depth ? tr.bin[d] : 0;
        threshold[t * D + d] = d < tr.depth ? tr.threshold[d] : 0.0f;
        if (gain) gain[t * D + d] = d < tr.depth ? tr.gain[d] : 0.0f;
      }
      for (int32_t d = 0; d < tr.depth; ++d) {
        const double top = tr.gain_top[d];
        const double m = (tr.n_candidates[d] > 1) ? (top - tr.gain_second[d]) / fabs(top) : 1e300;
        if (m < min_margin) min_margin = m;
      }
      memcpy(leaves + t * L, lv, (size_t)L * sizeof(float));
      /* preds += lr * leaf (booster.cpp:458-463, fused multiply-add) */
      for (uint32_t i = 0; i < n; ++i) {
        const size_t q = (size_t)i * K + k;
        pred[q] = fmaf(p->learning_rate, lv[li[i]], pred[q]);
      }
    }
  }
  if (train_pred) memcpy(train_pred, pred, (size_t)n * K * sizeof(float));
  if (min_margin_out) *min_margin_out = min_margin;
done:
  free(pred); free(gg); free(hh); free(gk); free(hk); free(li); free(lv); free(sample); free(absg);
  return rc;
}

void tco_predict(const float* X, uint32_t n, uint32_t f, int32_t n_trees, int32_t K,
                 int32_t max_depth, const int32_t* depth, const uint16_t* feature,
                 const float* threshold, const float* leaves, const float* weights, float base,
                 double* out) {
  const uint32_t L = 1u << max_depth;
#pragma omp parallel for schedule(static)
  for (int64_t ii = 0; ii < (int64_t)n; ++ii) {
    const float* row = X + (size_t)ii * f;
    double* o = out + (size_t)ii * K;
    for (int32_t c = 0; c < K; ++c) o[c] = (double)base;
    for (int32_t t = 0; t < n_trees; ++t) {
      uint32_t idx = 0;
      for (int32_t d = 0; d < depth[t]; ++d) {
        const float v = row[feature[(size_t)t * max_depth + d]];
        const int right = !isnan(v) && v >= threshold[(size_t)t * max_depth + d];
        idx = (idx << 1) | (uint32_t)right;
      }
      o[t % K] += (double)weights[t] * (double)leaves[(size_t)t * L + idx];
    }
  }
}
