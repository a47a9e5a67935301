// Symmetric (oblivious) tree boosting on the device.
//
// Restates Booster::train (src/boosting/booster.cpp:47-252, 438-463) and
// SymmetricTree::build (src/tree/symmetric_tree.cpp:34-368) level by level:
//
//   grad       pred += lr * leaf(prev tree) (fused), loss gradients/hessians,
//              leaf ids reset, per-block root sums            [one pass over rows]
//   per level d = 0 .. D-1, for all classes k at once:
//     hist     FP32 shared-memory histograms of the level's build set -- the
//              root at d = 0, the smaller child of every sibling pair after --
//              over row-major uint8 bins gathered through the node-grouped row
//              list; one FP32 partial per (segment chunk, feature group)
//     merge    FP64 sum of the partials (the cross-block merge) and the FP64
//              sibling subtraction larger = parent - smaller
//     scan     per (feature, node group): FP64 prefix (left, NaN slot
//              included: NaN routes left) and suffix (right) sums and the
//              Newton gain of every bin for every node, summed over nodes
//     pick     per class: argmax over (feature, bin), lowest feature then
//              lowest bin on ties (the reference keeps the first strictly
//              greater gain), stop rules, the split goes into the model
//     part     leaf = 2*leaf + go_right, go_right = bin != 255 && bin > t;
//              per-block child counts and FP64 child sums
//     reduce   child totals, smaller child per pair, scatter offsets
//     plan     (one block) segment starts, rows per chunk and the chunk counts
//              the histogram kernel decodes into work items,
//              the stop pre-check, leaf values when the tree is complete
//     scatter  node-grouped row list of the smaller children
//
// Every kernel reads the per-class "done" flag and returns early once a
// tree has stopped, so an iteration is a fixed launch sequence that is
// captured once as a CUDA graph and replayed (the batched path).  The plain
// path launches one class and one level at a time with a host
// synchronisation after every level.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <numeric>
#include <random>
#include <string>
#include <thread>
#include <vector>

#include "tc_internal.h"
#include "tc_loss.cuh"

namespace tc {
namespace {

constexpr int HIST_THREADS = 1024;  // one histogram block per SM (its accumulators take 128 KB)
constexpr int HIST_BATCH = 32;    // rows per warp batch (one per lane)
constexpr int PART_THREADS = 512;
constexpr int GRAD_UNROLL = 4;    // rows per thread with their loads in flight together (one class)
constexpr int kSoftmaxMaxK = 16;  // softmax classes at most (checked when a trainer is created)
constexpr int SCAN_WARPS = 8;     // warps per scan block
constexpr int SCAN_NODES = 16;    // nodes per scan block (2 per warp; measured: 32 per block 4% slower on 1M x 100 depth 8)
static_assert(SCAN_WARPS * 32 == 256, "a scan block also runs the 256-thread pick");
constexpr int PLAN_THREADS = 1024;
constexpr int kHistRowsMax = 65535;  // rows of a histogram item: its 16-bit low fields sum without overflow
constexpr int VALID_BLOCKS = 296;  // blocks of the validation kernel (fixed: its partial sums have a fixed order)

struct NodeStat {
  double G, H;
  uint32_t cnt;
  uint32_t pad;
};

// Per-class, per-tree control block on the device.
struct ClassState {
  int32_t done;        // 0 growing, 1 stopped (leaves pending), 2 finalized
  int32_t depth;       // accepted splits
  int32_t f, b;        // split of the current level
  int32_t skew;        // one node of the current level holds more than 1/8 of the rows
  int32_t hot;         // with skew: that node (the largest; the lowest index on a tie)
};

// Early-stopping state of a validation set (device).
struct EsState {
  float best;          // best validation loss so far (the reference keeps it in FP32)
  int32_t best_iter;
  int32_t no_improve;  // iterations in a row without improvement
  int32_t stopped;     // set once the stopping rule fires
  int32_t stop_iter;
  uint32_t ctr;        // completion counter of the loss blocks
};

// Per-(class, feature) best candidate of a level.
struct FeatBest {
  double gain, second;
  int32_t b, valid;
};

struct DevCfg {
  uint32_t n, f, np;
  uint32_t groups, wlast;        // 32-feature groups of the bin tiles; bytes per row of the last one
  uint64_t gstride;              // bytes of one full group block
  int32_t K, D, nb_scan, loss;
  int32_t KT, k0;                // classes in the model; first class of this launch view
  int32_t msl;
  float lr, lam, l1, mcw, msg, mds, gamma, alpha;
  int32_t G, W;                  // feature groups, group width (32*J)
  int32_t PB;                    // partition blocks
  int32_t item_cap;              // capacity of the partial buffer (items)
  int32_t n_scan_groups_max;
  int32_t hist_grid;             // persistent histogram blocks
  int32_t target_items;          // work items aimed for per histogram launch
  int32_t rows_min;              // smallest rows per histogram chunk
  int32_t rows_fixed;            // > 0: fixed rows per chunk (tuning override)
  float hconst;                  // > 0: every row's hessian equals this (histogram counts rows)
  uint32_t nv;                   // validation rows (0: no validation set)
  int32_t es_rounds;             // early_stopping_rounds (< 0: never stop)
  int32_t es_min_iter;           // first iteration the stopping rule may fire at
  int32_t sampled;               // 1: only the rows of smask grow this iteration's trees
};

struct DevPtrs {
  const uint8_t* bins_t;         // feature-group tiles (tc_dataset::bins_t)
  const uint8_t* bins_cm;
  const float* edges;            // [f][256]
  const uint16_t* n_edges;
  const uint32_t* nan_any;       // [f] nonzero: the feature has NaN rows
  const float* y;
  float* pred;                   // [K][n]
  float2* gh;                    // [K][n]
  float2* cgh;                   // [K][n] (grad, hess) of the rows list, in its order
  uint16_t* leaf;                // [K][n]
  uint32_t* rows;                // [K][n]
  double2* hist[2];              // [K][2^(D-1)][F][256]
  double2* acc;                  // [K][2^(D-1)][F][256] FP64 sums of the level's smaller children (the
                                 // root at level 0), added by the histogram items; the scan reads and re-zeroes them
  int32_t* cum;                  // [K*2^(D-1) + 1] cumulative item counts per segment (chunk-major)
  int32_t* rchunk;               // [1] rows per chunk at the current level
  int32_t* seg_start;            // [K][2^(D-1)]
  int32_t* seg_len;              // [K][2^(D-1)]
  int32_t* small;                // [K][2^(D-1)] child index of the smaller sibling
  NodeStat* nstat;               // [K][D+1][2^D]
  uint32_t* pcnt;                // [K][PB][2^D]
  double2* psum;                 // [K][PB][2^D]
  uint32_t* blk_off;             // [K][PB][2^(D-1)]
  double* gpart;                 // [K][F][NG][256]
  uint8_t* gany;                 // [K][F][NG][256]
  FeatBest* fbest;               // [K][F]
  uint32_t* counters;            // [K] completion counters of the pick blocks
  uint32_t* fcnt;                // [K][F] completion counters of a feature's scan blocks
  int32_t* hist_ctr;             // [1] next histogram work item (reset by the plan kernel)
  uint32_t* red_ctr;             // [1] completion counter of the fused reduce + plan kernel
  ClassState* cs;                // [K]
  int32_t* iter;                 // [1] boosting iteration (tree slot = iter*KT + k0 + k)
  // model arrays (capacity T = n_estimators*K)
  int32_t* m_depth;              // [T]
  uint16_t* m_feat;              // [T][D]
  uint8_t* m_bin;                // [T][D]
  float* m_thr;                  // [T][D]
  double* m_gain;                // [T][D]
  double* m_second;              // [T][D]
  float* m_leaves;               // [T][2^D]
  double* root_hist_out;         // optional [F][256][2]
  uint64_t* lvl_rows;            // [16] rows histogrammed at level d (all classes), written by the plan
  uint32_t* lvl_nodes;           // [16] nodes histogrammed at level d (all classes)
  // validation set
  const float* xv;               // [nv][f] raw features
  const float* yv;               // [nv] labels
  float* vpred;                  // [K][nv] raw validation predictions
  double* vpart;                 // [VALID_BLOCKS] partial loss sums
  double* vloss;                 // [n_estimators] validation loss per iteration
  EsState* es;
  const uint32_t* smask;         // [ceil(n/32)] rows sampled this iteration (bit per row)
};

__device__ __forceinline__ bool row_sampled(const DevCfg& c, const DevPtrs& P, uint32_t i) {
  return !c.sampled || ((P.smask[i >> 5] >> (i & 31)) & 1u);
}

__device__ __forceinline__ size_t hist_index(const DevCfg& c, int k, int node, int f, int b) {
  return (((size_t)k * (1u << (c.D > 0 ? c.D - 1 : 0)) + node) * c.f + f) * kSlots + b;
}

__device__ __forceinline__ int pairs_at(int d) { return d == 0 ? 1 : (1 << (d - 1)); }

// ------------------------------------------------------------------ grad --

// One thread per row: applies the previous tree of every class
// (preds += lr * leaf, fused multiply-add as in src/boosting/booster.cpp:458-463),
// computes the gradients and resets the leaf ids; then per-block root sums
// (FP64, fixed order) go to psum[k][block][0] / pcnt.
// One class's root sums: per-thread FP64 partials (rows in increasing
// order), reduced in a fixed order (warp shuffles, then the warps in order)
// into the block's slot of the partition sums, which the level -1 reduce
// reads; cnt = the thread's sampled rows.
__device__ void store_root_partials(const DevCfg& c, const DevPtrs& P, int k, double g, double h, uint32_t cnt) {
  __shared__ double sG[16], sH[16];
  __shared__ uint32_t sCnt[16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int o = 16; o; o >>= 1) {
    g += __shfl_down_sync(0xffffffffu, g, o);
    h += __shfl_down_sync(0xffffffffu, h, o);
    cnt += __shfl_down_sync(0xffffffffu, cnt, o);
  }
  if (lane == 0) { sG[warp] = g; sH[warp] = h; sCnt[warp] = cnt; }
  __syncthreads();
  if (threadIdx.x == 0) {
    double tg = 0.0, th = 0.0;
    uint32_t tc = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { tg += sG[w]; th += sH[w]; tc += sCnt[w]; }
    const size_t o = ((size_t)k * c.PB + blockIdx.x) * (1 << c.D);
    P.psum[o] = make_double2(tg, th);
    P.pcnt[o] = tc;
  }
  __syncthreads();
}

// Root sums of the block's rows [r0, r1) for every class, from P.gh.
__device__ void root_sums(const DevCfg& c, const DevPtrs& P, uint32_t r0, uint32_t r1) {
  uint32_t my_cnt = 0;
  for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) my_cnt += row_sampled(c, P, i) ? 1u : 0u;
  for (int k = 0; k < c.K; ++k) {
    double g = 0.0, h = 0.0;
    for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
      const float2 v = P.gh[(size_t)k * c.n + i];
      g += (double)v.x;
      h += (double)v.y;
    }
    store_root_partials(c, P, k, g, h, my_cnt);
  }
}

// SOFTMAX: the K-class path (the row's classes loaded together); else one class.
template <bool SOFTMAX>
__global__ void __launch_bounds__(512, 2) k_grad(DevCfg c, DevPtrs P, int use_given_gh) {
  const int K = SOFTMAX ? c.K : 1;
  const int it = *P.iter;
  const uint32_t n_vec = (c.n / 8) * 8;
  const uint32_t rows_per_block = (c.n + gridDim.x - 1) / gridDim.x;
  const uint32_t r0 = blockIdx.x * rows_per_block;
  const uint32_t r1 = min(c.n, r0 + rows_per_block);
  const int L = 1 << c.D;
  if (!SOFTMAX) {
    // one class: GRAD_UNROLL rows per thread with their loads issued first,
    // and the root sums taken on the way (same rows, same order as root_sums)
    const bool upd = it > 0 && !use_given_gh;
    const size_t tl = upd ? ((size_t)(it - 1) * c.KT + c.k0) * L : 0;
    double sg = 0.0, sh = 0.0;
    uint32_t cnt = 0;
    for (uint32_t base = r0 + threadIdx.x; base < r1; base += blockDim.x * GRAD_UNROLL) {
      float pr[GRAD_UNROLL], yv[GRAD_UNROLL], lv[GRAD_UNROLL];
      uint16_t lf[GRAD_UNROLL];
      float2 given[GRAD_UNROLL];
#pragma unroll
      for (int u = 0; u < GRAD_UNROLL; ++u) {
        const uint32_t i = base + u * blockDim.x;
        if (i < r1) {
          if (upd) lf[u] = P.leaf[i];
          if (!use_given_gh) {
            pr[u] = P.pred[i];
            yv[u] = P.y[i];
          } else {
            given[u] = P.gh[i];
          }
        }
      }
      if (upd) {
#pragma unroll
        for (int u = 0; u < GRAD_UNROLL; ++u)
          if (base + u * blockDim.x < r1) lv[u] = P.m_leaves[tl + lf[u]];
      }
#pragma unroll
      for (int u = 0; u < GRAD_UNROLL; ++u) {
        const uint32_t i = base + u * blockDim.x;
        if (i >= r1) continue;
        const bool in = row_sampled(c, P, i);
        float2 v;
        if (!use_given_gh) {
          float p = pr[u];
          if (upd) {
            p = __fmaf_rn(c.lr, lv[u], p);
            P.pred[i] = p;
          }
          float g, h;
          loss_grad(c.loss, p, yv[u], i, n_vec, c.gamma, c.alpha, g, h);
          // rows outside this iteration's sample add nothing to any sum
          v = in ? make_float2(g, h) : make_float2(0.0f, 0.0f);
          P.gh[i] = v;
        } else {
          v = given[u];
        }
        P.leaf[i] = 0;
        sg += (double)v.x;
        sh += (double)v.y;
        cnt += in ? 1u : 0u;
      }
    }
    store_root_partials(c, P, 0, sg, sh, cnt);
    return;
  }
  // softmax (K classes, K <= 16): a row's K predictions and leaf ids are
  // loaded together (unrolled over the class bound, guarded by K)
  for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x) {
    float pr[kSoftmaxMaxK];
#pragma unroll
    for (int k = 0; k < kSoftmaxMaxK; ++k)
      if (k < K) pr[k] = P.pred[(size_t)k * c.n + i];
    if (it > 0 && !use_given_gh) {
      uint16_t lf[kSoftmaxMaxK];
#pragma unroll
      for (int k = 0; k < kSoftmaxMaxK; ++k)
        if (k < K) lf[k] = P.leaf[(size_t)k * c.n + i];
      const size_t t0 = (size_t)(it - 1) * c.KT + c.k0;
#pragma unroll
      for (int k = 0; k < kSoftmaxMaxK; ++k) {
        if (k < K) {
          pr[k] = __fmaf_rn(c.lr, P.m_leaves[(t0 + k) * L + lf[k]], pr[k]);
          P.pred[(size_t)k * c.n + i] = pr[k];
        }
      }
    }
    if (!use_given_gh) {
      // CrossEntropyLoss::compute_multiclass_gradients + softmax (src/boosting/loss.cpp:273-318)
      const bool in = row_sampled(c, P, i);
      float mx = pr[0];
#pragma unroll
      for (int k = 1; k < kSoftmaxMaxK; ++k)
        if (k < K) mx = fmaxf(mx, pr[k]);
      float sum = 0.0f;
#pragma unroll
      for (int k = 0; k < kSoftmaxMaxK; ++k)
        if (k < K) sum = __fadd_rn(sum, expf(__fsub_rn(pr[k], mx)));
      const int label = (int)P.y[i];
#pragma unroll
      for (int k = 0; k < kSoftmaxMaxK; ++k) {
        if (k < K) {
          const float p = __fdiv_rn(expf(__fsub_rn(pr[k], mx)), sum);
          const float g = __fsub_rn(p, (k == label) ? 1.0f : 0.0f);
          const float h = fmaxf(__fmul_rn(p, __fsub_rn(1.0f, p)), 1e-6f);
          // rows outside this iteration's sample add nothing to any sum
          P.gh[(size_t)k * c.n + i] = in ? make_float2(g, h) : make_float2(0.0f, 0.0f);
        }
      }
    }
#pragma unroll
    for (int k = 0; k < kSoftmaxMaxK; ++k)
      if (k < K) P.leaf[(size_t)k * c.n + i] = 0;
  }
  root_sums(c, P, r0, r1);
}

// GOSS iterations: the gradients of every row are in place (k_grad ran
// without a sample); the host has since chosen the sample from them.  Rows
// outside it get zero gradients for all classes, and the root sums and
// counts are redone over the sample.
__global__ void __launch_bounds__(512) k_goss_root(DevCfg c, DevPtrs P) {
  const uint32_t rows_per_block = (c.n + gridDim.x - 1) / gridDim.x;
  const uint32_t r0 = blockIdx.x * rows_per_block;
  const uint32_t r1 = min(c.n, r0 + rows_per_block);
  for (uint32_t i = r0 + threadIdx.x; i < r1; i += blockDim.x)
    if (!row_sampled(c, P, i))
      for (int k = 0; k < c.K; ++k) P.gh[(size_t)k * c.n + i] = make_float2(0.0f, 0.0f);
  __syncthreads();
  root_sums(c, P, r0, r1);
}

// Applies the last tree's leaves to the predictions (end of training / before
// reading training scores).
__global__ void k_apply_last(DevCfg c, DevPtrs P) {
  const int it = *P.iter;
  if (it <= 0) return;
  const int L = 1 << c.D;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < c.n; i += gridDim.x * blockDim.x) {
    for (int k = 0; k < c.K; ++k) {
      const size_t t = (size_t)(it - 1) * c.KT + c.k0 + k;
      const float v = P.m_leaves[t * L + P.leaf[(size_t)k * c.n + i]];
      float& pr = P.pred[(size_t)k * c.n + i];
      pr = __fmaf_rn(c.lr, v, pr);
      P.leaf[(size_t)k * c.n + i] = 0;
    }
  }
}


// ------------------------------------------------------------------ hist --

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const uint32_t s = (uint32_t)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

struct HistShape {
  static constexpr int W = 32;                          // histogram columns (features) of an item
  static constexpr int WARPS = HIST_THREADS / 32;
  static constexpr int S = 2;                           // staging depth per warp (batches in flight)
  static constexpr int FIELDS = 4;                      // u32 accumulators per (slot, column)
  static constexpr size_t hist_bytes = (size_t)kSlots * FIELDS * W * 4;    // 128 KB
  static constexpr size_t warp_bytes = (size_t)S * HIST_BATCH * (W + 8);   // bins + (grad, hess)
  static constexpr size_t smem = hist_bytes + WARPS * warp_bytes;
};
static_assert(HistShape::smem <= 227 * 1024 - 1024, "histogram shared memory");

// Work item -> segment (class, pair) through the cumulative item counts.
__device__ __forceinline__ int find_seg(const int32_t* cum, int nseg, int item) {
  int lo = 0, hi = nseg - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (cum[mid] <= item) lo = mid; else hi = mid - 1;
  }
  return lo;
}

// Bin slots of a histogram column: a feature with n_edges edges uses bins
// 0 .. n_edges (span = n_edges + 1) and the NaN slot 255, so the slots past
// its span are free.  A feature without NaN rows keeps private copies of its
// column there for different warps (copy c of bin b in slot c*span + b, at
// most 255/span copies, so bin + offset never reaches 255), which spreads the
// updates of few-bin features over more addresses.  A feature with NaN rows
// keeps one copy.
struct HistCol {
  int span, copies;
};
__device__ __forceinline__ HistCol hist_col(const DevPtrs& P, int f, int nf) {
  if (f >= nf) return {255, 1};
  const int span = (int)P.n_edges[f] + 1;
  return {span, P.nan_any[f] ? 1 : min(HIST_THREADS / 32, max(1, 255 / span))};
}

__device__ __forceinline__ void red_add_u32(uint32_t a, uint32_t v) {
  asm volatile("red.shared.add.u32 [%0], %1;" ::"r"(a), "r"(v) : "memory");
}

// Exact fixed-point accumulation.
//
// Each row's grad (and hess) becomes the integer v = round(x * 2^e), with a
// power of two 2^e chosen per work item from the item's own sum S of |x|
// over its rows (FP64): e is the largest value with 2^e * S + rows / 2
// below 2^46, so every partial sum of any bin has |sum v| < 2^46.  v is kept
// as two unsigned 32-bit shared accumulators, hi = v >> 16 (arithmetic, so
// |sum hi| < 2^31) and lo = v & 0xffff (an item has at most 65535 rows, so
// sum lo < 2^32): integer sums are exact, independent of the order of the
// atomics, and 32-bit shared integer atomics run at about twice the rate of
// FP32 shared atomics on this part (measured, and unlike FP32 they do not
// slow down when many lanes hit few addresses).  A row is represented to
// within 2^-(e+1) <= S * 2^-46 ... 2^-47: relative to the item's total |x|,
// about 1e-14; the sum of a bin is exact on top of that.
// Accumulators per (slot, column): 0 grad hi, 1 grad lo, 2 hess hi (CNT: the
// row count; every row's hessian is the same constant, MSE: h = 2), 3 hess lo.
constexpr double kFixLimit = 70368744177664.0;  // 2^46

__device__ __forceinline__ int fix_exponent(double S, double rows) {
  if (!(S > 0.0)) return 0;
  // a relative margin for the rounding of the FP64 sum S itself
  const double room = kFixLimit * (1.0 - 0x1p-20) - 0.5 * rows;
  int e = ilogb(room / S);      // floor(log2(room / S))
  if (ldexp(S, e) > room) --e;  // against rounding of the division
  return max(-126, min(100, e));
}
__device__ __forceinline__ float exp2i(int e) { return __int_as_float((e + 127) << 23); }

struct FixRow {
  uint32_t ghi, glo, hhi, hlo;
};
__device__ __forceinline__ FixRow fix_row(float g, float h, float sg, float sh) {
  FixRow r;
  const long long vg = __float2ll_rn(g * sg);  // exact product: sg is a power of two
  r.ghi = (uint32_t)(vg >> 16);
  r.glo = (uint32_t)vg & 0xffffu;
  const long long vh = __float2ll_rn(h * sh);
  r.hhi = (uint32_t)(vh >> 16);
  r.hlo = (uint32_t)vh & 0xffffu;
  return r;
}

// Persistent blocks (one per SM) over work items; an item is one chunk of one
// segment's rows (the root at d = 0, a smaller child after) for one group of
// 32 features, and the items of a chunk's groups are adjacent (chunk-major),
// so blocks that run together read the same rows and the L2 serves a row's
// (grad, hess) to every group.
//
// An item starts with a pass over its rows' (grad, hess) (contiguous in list
// order) for the sums that fix its scales.  Then every warp runs its own copy
// pipeline: lane l stages row l of a 32-row batch (its 32-byte group slice
// from the feature-group tiles, and its (grad, hess)) by cp.async into the
// warp's private buffers, one batch ahead of the updates, with the row ids of
// gathered rows fetched a further batch ahead; no block barrier is taken
// until the item is done.  The item ends by adding its exact sums, converted
// to FP64, to the segment's FP64 accumulator in global memory.
//
// Shared histogram layout: column fastest, so a column always hits the same
// bank: uint32 hist[(4 * slot + field) * 32 + column].  A wide group is
// updated four rows at a time: lane (r = l/8, c = l%8) loads the 4 bins of
// columns 4c..4c+3 of row r of the quad as one word and, in step s, updates
// column 4c + (s + r) % 4, so the 32 lanes of every step hit 32 different
// banks.  A group of at most 16 features is packed: with p2 = next power of
// two >= its width, the 32 columns hold 32/p2 private copies and one warp
// instruction updates 32/p2 rows; the copies are summed when the item ends.
// Columns past a group's width (padding bytes, all bin 0: one hot address)
// are not updated.  Each lane keeps the shared address of (its warp's copy of)
// every column it updates, so an update is a byte permute, an add and the
// integer atomics.
template <bool CNT>
__global__ void __launch_bounds__(HIST_THREADS, 1) k_hist(DevCfg c, DevPtrs P, int d) {
  using S_ = HistShape;
  constexpr int W = S_::W, S = S_::S, B = HIST_BATCH;
  constexpr uint32_t SLOT_BYTES = 4 * S_::FIELDS * W;   // 512: the 4 fields of one slot
  constexpr uint32_t FB = 4 * W;                         // bytes between two fields of a slot
  extern __shared__ __align__(16) unsigned char smraw[];
  uint32_t* hist = reinterpret_cast<uint32_t*>(smraw);
  const uint32_t hbase = (uint32_t)__cvta_generic_to_shared(hist);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  uint8_t* w_bins = smraw + S_::hist_bytes + (size_t)warp * S_::warp_bytes;        // [S][B][W]
  float2* w_gh = reinterpret_cast<float2*>(w_bins + (size_t)S * B * W);            // [S][B]
  __shared__ double s_sum[2][HIST_THREADS / 32];
  const int P2 = pairs_at(d);
  const int nseg = c.K * P2;
  const int n_items = P.cum[nseg];
  const int R = *P.rchunk;
  const int Pmax = 1 << (c.D - 1);
  // quad mapping of this lane: row qr of a quad, columns 4*c4 .. 4*c4+3;
  // byte-permute selectors that move byte (s + qr) % 4 of the word to bits 8..15
  const int qr = lane >> 3, c4 = lane & 7;
  uint32_t sel[4];
#pragma unroll
  for (int s = 0; s < 4; ++s) sel[s] = 0x4404u | ((uint32_t)((s + qr) & 3) << 4);
  for (int q = threadIdx.x; q < kSlots * S_::FIELDS * W; q += blockDim.x) hist[q] = 0u;
  __syncthreads();
  // Items are claimed from a counter (blocks that drew cheap items take
  // more), the next one while the current one runs.  Item ci*G + g is chunk
  // ci (over all segments) of group g; a narrow last group costs a fraction
  // of a wide one, so its items are handed out after all the wide ones and
  // fill the gaps at the end.
  const int n_chunks = n_items / c.G;
  const int gw = (c.G > 1 && (int)c.f - (c.G - 1) * W <= 16) ? c.G - 1 : c.G;  // wide groups
  auto claim_to_item = [&](int cl) {
    if (gw == c.G || cl >= n_items) return cl;
    return cl < n_chunks * gw ? (cl / gw) * c.G + cl % gw : (cl - n_chunks * gw) * c.G + gw;
  };
  __shared__ int s_item[2];
  if (threadIdx.x == 0) s_item[0] = claim_to_item(atomicAdd(P.hist_ctr, 1));
  __syncthreads();
  int item = s_item[0];
  for (int it = 1; item < n_items; ++it) {
    if (threadIdx.x == 0) s_item[it & 1] = claim_to_item(atomicAdd(P.hist_ctr, 1));
    const int seg = find_seg(P.cum, nseg, item);
    const int local = item - P.cum[seg];
    const int ch_idx = local / c.G;
    const int g = local - ch_idx * c.G;
    const int k = seg / P2, p = seg - k * P2;
    const int g0 = g * W;
    const int gsize = min(W, (int)c.f - g0);
    const int p2 = gsize <= 1 ? 1 : (gsize <= 2 ? 2 : (gsize <= 4 ? 4 : (gsize <= 8 ? 8 : (gsize <= 16 ? 16 : 32))));
    const bool narrow = p2 <= 16;
    // the segment's ceil(len / R) chunks have equal sizes (within one row)
    const int s0 = d == 0 ? 0 : P.seg_start[k * Pmax + p];
    const int sl = d == 0 ? (int)c.n : P.seg_len[k * Pmax + p];
    const int nch = (sl + R - 1) / R;
    const int start = s0 + (int)((long long)sl * ch_idx / nch);
    const int end = s0 + (int)((long long)sl * (ch_idx + 1) / nch);
    const uint32_t* rows = P.rows + (size_t)k * c.n;
    // (grad, hess) in list order: the root's rows are 0..n-1, a smaller
    // child's were copied next to its row ids by the scatter kernel
    const float2* gh = (d == 0 ? P.gh : P.cgh) + (size_t)k * c.n;
    // the item's scales: FP64 sums of |grad| and |hess| over its rows (every
    // thread a fixed stride, the warps in a fixed order)
    int eg, eh;
    float sg, sh;
    {
      double sa = 0.0, sb = 0.0;
#pragma unroll 4
      for (int r = start + threadIdx.x; r < end; r += blockDim.x) {
        const float2 v = gh[r];
        sa += (double)fabsf(v.x);
        sb += (double)fabsf(v.y);
      }
      for (int o = 16; o; o >>= 1) {
        sa += __shfl_xor_sync(0xffffffffu, sa, o);
        sb += __shfl_xor_sync(0xffffffffu, sb, o);
      }
      if (lane == 0) { s_sum[0][warp] = sa; s_sum[1][warp] = sb; }
      __syncthreads();
      sa = 0.0;
      sb = 0.0;
      for (int w = 0; w < nwarps; ++w) { sa += s_sum[0][w]; sb += s_sum[1][w]; }
      eg = fix_exponent(sa, (double)(end - start));
      eh = CNT ? 0 : fix_exponent(sb, (double)(end - start));
      sg = exp2i(eg);
      sh = exp2i(eh);
    }
    // shared address of this warp's copy of each column the lane updates;
    // columns past the group's width are skipped (their padding bytes are
    // all bin 0, a single hot address)
    uint32_t ab[4];
    uint32_t live = 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
      const int col = 4 * c4 + ((s + qr) & 3);
      const HistCol hc = hist_col(P, g0 + col, (int)c.f);
      ab[s] = hbase + SLOT_BYTES * (uint32_t)((warp % hc.copies) * hc.span) + 4u * col;
      if (col < gsize) live |= 1u << s;
    }
    // the two 16-byte pieces of a row's group slice in the feature-group
    // tiles; the last group's narrower block copies only its width
    const uint32_t gwid = (uint32_t)g + 1 == c.groups ? c.wlast : 32u;
    const uint8_t* tile = P.bins_t + (uint64_t)g * c.gstride;
    const int nb = (end - start + B - 1) / B;   // batches in the item; warp w takes w, w+nwarps, ...
    uint32_t rid_next = 0;
#define TC_FETCH_ID(bi)                                                                      \
    {                                                                                        \
      const int r_ = start + (bi) * B + lane;                                                \
      rid_next = ((bi) < nb && r_ < end) ? (d == 0 ? (uint32_t)r_ : rows[r_]) : 0u;          \
    }
#define TC_ISSUE(bi, st_)                                                                    \
    {                                                                                        \
      if ((bi) < nb && start + (bi) * B + lane < end) {                                      \
        uint8_t* dst_ = w_bins + ((size_t)(st_) * B + lane) * W;                             \
        const uint8_t* src_ = tile + (size_t)rid_next * gwid;                                \
        if (gwid == 32) {                                                                    \
          cp_async16(dst_, src_);                                                            \
          cp_async16(dst_ + 16, src_ + 16);                                                  \
        } else if (gwid == 16) {                                                             \
          cp_async16(dst_, src_);                                                            \
        } else if (gwid == 8) {                                                              \
          cp_async8(dst_, src_);                                                             \
        } else {                                                                             \
          cp_async4(dst_, src_);                                                             \
        }                                                                                    \
        cp_async8(w_gh + (st_) * B + lane, gh + start + (bi) * B + lane);                     \
      }                                                                                      \
      cp_async_commit();                                                                     \
    }
    int bi = warp;
    TC_FETCH_ID(bi);
    TC_ISSUE(bi, 0);
    TC_FETCH_ID(bi + nwarps);
    for (int t = 0; bi < nb; ++t, bi += nwarps) {
      const int st = t & 1;
      TC_ISSUE(bi + nwarps, st ^ 1);       // the next batch streams in while this one is counted
      TC_FETCH_ID(bi + 2 * nwarps);        // row ids for the batch after, behind this batch's updates
      cp_async_wait<1>();
      __syncwarp();
      const int nvalid = min(B, end - (start + bi * B));
      const uint8_t* sb = w_bins + (size_t)st * B * W;
      const float2* sv = w_gh + st * B;
      if (!narrow) {
        // the batch's bins and (grad, hess) go to registers first, so the
        // loads are not ordered behind the updates (they share the memory space)
        const uint32_t* sw = reinterpret_cast<const uint32_t*>(sb);
        uint32_t wd[B / 4];
        float vx[B / 4], vy[B / 4];
#pragma unroll
        for (int qd = 0; qd < B / 4; ++qd) {
          const int row = 4 * qd + qr;
          const float2 v = sv[row];
          vx[qd] = v.x;
          vy[qd] = v.y;
          wd[qd] = sw[row * (W / 4) + c4];
        }
#pragma unroll
        for (int qd = 0; qd < B / 4; ++qd) {
          if (4 * qd + qr < nvalid) {
            const FixRow fr = fix_row(vx[qd], vy[qd], sg, sh);
#pragma unroll
            for (int s = 0; s < 4; ++s) {
              // __byte_perm gives bin * 256; a slot is SLOT_BYTES = 512 bytes
              const uint32_t a = ab[s] + 2u * __byte_perm(wd[qd], 0u, sel[s]);
              if (live & (1u << s)) {
                red_add_u32(a, fr.ghi);
                red_add_u32(a + FB, fr.glo);
                if (CNT) {
                  red_add_u32(a + 2 * FB, 1u);
                } else {
                  red_add_u32(a + 2 * FB, fr.hhi);
                  red_add_u32(a + 3 * FB, fr.hlo);
                }
              }
            }
          }
        }
      } else {
        // packed narrow group: lane (copy, column) of rows i .. i + 32/p2 - 1,
        // four instructions' rows loaded ahead of their updates
        const int rpi = 32 / p2;
        const int my_row = lane / p2, my_col = lane - my_row * p2;
        const HistCol hc = hist_col(P, g0 + my_col, (int)c.f);
        const uint32_t abn = hbase + SLOT_BYTES * (uint32_t)((warp % hc.copies) * hc.span) + 4u * lane;
        for (int i0 = 0; i0 < B; i0 += 4 * rpi) {
          uint32_t bb[4];
          float gx[4], gy[4];
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            const int row = min(i0 + u * rpi + my_row, B - 1);
            const float2 v = sv[row];
            gx[u] = v.x;
            gy[u] = v.y;
            bb[u] = sb[row * W + my_col];
          }
#pragma unroll
          for (int u = 0; u < 4; ++u) {
            if (i0 + u * rpi + my_row < nvalid && my_col < gsize) {
              const FixRow fr = fix_row(gx[u], gy[u], sg, sh);
              const uint32_t a = abn + SLOT_BYTES * bb[u];
              red_add_u32(a, fr.ghi);
              red_add_u32(a + FB, fr.glo);
              if (CNT) {
                red_add_u32(a + 2 * FB, 1u);
              } else {
                red_add_u32(a + 2 * FB, fr.hhi);
                red_add_u32(a + 3 * FB, fr.hlo);
              }
            }
          }
        }
      }
      __syncwarp();
    }
#undef TC_FETCH_ID
#undef TC_ISSUE
    cp_async_wait<0>();
    __syncthreads();
    // add the item's exact sums (copies summed as integers), converted to
    // FP64, to the segment's FP64 accumulator (zero sums are not sent), and
    // clear the histogram for the next item; a thread clears exactly the
    // slots it reads
    double2* dst = P.acc + (((size_t)k * Pmax + p) * c.f + g0) * kSlots;
    const int ncp = narrow ? 32 / p2 : 1;     // packed copies of a narrow group
    // blockDim.x is a multiple of W: a thread's column is the same on every pass
    const int col = threadIdx.x % W;
    const HistCol fc = hist_col(P, g0 + col, (int)c.f);
    for (int q = threadIdx.x; q < kSlots * W; q += blockDim.x) {
      const int b = q / W;
      long long G = 0, H = 0;
      if (!narrow || col < p2) {
        const int kc = b == kNanBin ? 1 : (b < fc.span ? fc.copies : 0);
        for (int cc = 0; cc < kc; ++cc) {
          const int slot = b == kNanBin ? kNanBin : cc * fc.span + b;
          for (int cp = 0; cp < ncp; ++cp) {
            uint32_t* o = hist + 4 * slot * W + cp * p2 * (narrow ? 1 : 0) + col;
            G += (long long)(int32_t)o[0] * 65536 + (long long)o[W];
            if (CNT) H += (long long)o[2 * W];
            else H += (long long)(int32_t)o[2 * W] * 65536 + (long long)o[3 * W];
            if (!narrow) {
              o[0] = 0u;
              o[W] = 0u;
              o[2 * W] = 0u;
              o[3 * W] = 0u;
            }
          }
        }
      }
      if (col < gsize) {
        const double gd = ldexp((double)G, -eg);
        const double hd = CNT ? (double)c.hconst * (double)H : ldexp((double)H, -eh);
        double2* o = dst + (size_t)col * kSlots + b;
        if (gd != 0.0) atomicAdd(&o->x, gd);
        if (hd != 0.0) atomicAdd(&o->y, hd);
      }
    }
    if (narrow) {
      __syncthreads();
      for (int q = threadIdx.x; q < kSlots * S_::FIELDS * 32; q += blockDim.x) hist[q] = 0u;
    }
    __syncthreads();
    item = s_item[it & 1];
  }
}

// ------------------------------------------------------------------ scan --

__device__ void pick_body(const DevCfg& c, const DevPtrs& P, int d, int f, int k, bool direct, double s_in,
                          uint8_t any_in);

// grid (F, node groups, K), SCAN_WARPS warps.  A warp scores one node at a
// time: lane l holds bins 8l .. 8l+7 (bin 255 = NaN rows, added to the left
// side); left sums are NaN + prefix, right sums an independent suffix, so an
// empty side is exactly zero.  Per-bin gains (the reference's formula,
// src/tree/symmetric_tree.cpp:161-178 and 221-236) accumulate in FP64 over
// the warp's nodes; the block then sums its warps in a fixed order.
__global__ void __launch_bounds__(SCAN_WARPS * 32) k_scan(DevCfg c, DevPtrs P, int d) {
  __shared__ double s_acc[SCAN_WARPS][kSlots];
  __shared__ uint8_t s_any[SCAN_WARPS][kSlots];
  const int f = blockIdx.x, ng = blockIdx.y, k = blockIdx.z;
  if (P.cs[k].done) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nn = 1 << d;
  const double lam = (double)c.lam;
  double2* cur = P.hist[d & 1];
  const double2* par = P.hist[(d & 1) ^ 1];
  const int Pmax = 1 << (c.D - 1);
  // the next level reads this level's histograms as parents, the reduce
  // kernel reads the split feature's row for the children's sums (and the
  // root's is the tree builder's root-histogram output)
  const NodeStat* ns = P.nstat + ((size_t)k * (c.D + 1) + d) * (1 << c.D);
  double acc[8];
  uint32_t anyb = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) acc[i] = 0.0;
  const int n0 = ng * SCAN_NODES, n1 = min(nn, n0 + SCAN_NODES);
  for (int node = n0 + warp; node < n1; node += SCAN_WARPS) {
    const NodeStat st = ns[node];
    if (st.cnt == 0) continue;
    // the smaller child of a pair (and the root) is the items' FP64 sum; the
    // larger one is parent - smaller (FP64)
    const int pr = d == 0 ? 0 : node >> 1;
    const double2* ap = P.acc + (((size_t)k * Pmax + pr) * c.f + f) * kSlots + lane * 8;
    double hg[8], hh[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const double2 v = ap[i];
      hg[i] = v.x;
      hh[i] = v.y;
    }
    if (d > 0 && node != P.small[k * Pmax + pr]) {
      const double2* pp = par + hist_index(c, k, pr, f, 0) + lane * 8;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const double2 v = pp[i];
        hg[i] = v.x - hg[i];
        hh[i] = v.y - hh[i];
      }
    }
    {
      double2* hp = cur + hist_index(c, k, node, f, 0) + lane * 8;
#pragma unroll
      for (int i = 0; i < 8; ++i) hp[i] = make_double2(hg[i], hh[i]);
    }
    const double nan_g = __shfl_sync(0xffffffffu, hg[7], 31);
    const double nan_h = __shfl_sync(0xffffffffu, hh[7], 31);
    if (lane == 31) { hg[7] = 0.0; hh[7] = 0.0; }  // NaN slot is not a regular bin
    double tg = 0.0, th = 0.0;
#pragma unroll
    for (int i = 0; i < 8; ++i) { tg += hg[i]; th += hh[i]; }
    // exclusive prefix and suffix of the lane totals
    double pg = tg, ph = th, sg = tg, sh = th;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double ug = __shfl_up_sync(0xffffffffu, pg, o), uh = __shfl_up_sync(0xffffffffu, ph, o);
      const double dg = __shfl_down_sync(0xffffffffu, sg, o), dh = __shfl_down_sync(0xffffffffu, sh, o);
      if (lane >= o) { pg += ug; ph += uh; }
      if (lane + o < 32) { sg += dg; sh += dh; }
    }
    // the node's totals from its own histogram (lane 31's inclusive prefix
    // plus the NaN slot: one value for the whole warp), so that the parent
    // term of every bin's gain is consistent with its left and right sums
    const double Gn = __shfl_sync(0xffffffffu, pg, 31) + nan_g;
    const double Hn = __shfl_sync(0xffffffffu, ph, 31) + nan_h;
    pg -= tg; ph -= th;  // exclusive prefix
    sg -= tg; sh -= th;  // exclusive suffix
    const double pgain = (Hn > 1e-10) ? (Gn * Gn) / (Hn + lam) : 0.0;
    // right side of bin 8l+i: this lane's bins above i plus all lanes above
    double rsg[8], rsh[8];
    {
      double ag = sg, ah = sh;
#pragma unroll
      for (int i = 7; i >= 0; --i) {
        rsg[i] = ag;
        rsh[i] = ah;
        ag += hg[i];
        ah += hh[i];
      }
    }
    double lg = nan_g + pg, lh = nan_h + ph;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      lg += hg[i];
      lh += hh[i];
      const int b = lane * 8 + i;
      if (b < c.nb_scan && lh >= 1e-10 && rsh[i] >= 1e-10) {
        // GL^2/(HL+lam) + GR^2/(HR+lam) over one FP64 division
        const double dl = lh + lam, dr = rsh[i] + lam;
        acc[i] += 0.5 * ((lg * lg * dr + rsg[i] * rsg[i] * dl) / (dl * dr) - pgain);
        anyb |= 1u << i;
      }
    }
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    s_acc[warp][lane * 8 + i] = acc[i];
    s_any[warp][lane * 8 + i] = (anyb >> i) & 1u;
  }
  __syncthreads();
  // blockDim.x == kSlots: thread b sums bin b over the warps
  const int b = threadIdx.x;
  // the accumulators of this block's pairs (this feature) start the next level at zero
  for (int pr = (d == 0 ? 0 : n0 >> 1); pr < (d == 0 ? 1 : (n1 + 1) >> 1); ++pr)
    P.acc[(((size_t)k * Pmax + pr) * c.f + f) * kSlots + b] = make_double2(0.0, 0.0);
  double sb = 0.0;
  uint8_t ab = 0;
  for (int w = 0; w < SCAN_WARPS; ++w) {
    sb += s_acc[w][b];
    ab |= s_any[w][b];
  }
  if (gridDim.y == 1) {  // the only block of its feature: its sums go straight to the pick
    pick_body(c, P, d, f, k, true, sb, ab);
    return;
  }
  const size_t o = (((size_t)k * c.f + f) * c.n_scan_groups_max + ng) * kSlots + b;
  P.gpart[o] = sb;
  P.gany[o] = ab;
  // the last node-group block of feature f (completion counter; nobody
  // waits) picks the feature's best bin, and the class's last feature its split
  __shared__ bool s_fdone;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const uint32_t prev = atomicAdd(&P.fcnt[(size_t)k * c.f + f], 1u);
    s_fdone = prev == gridDim.y - 1;
  }
  __syncthreads();
  if (!s_fdone) return;
  __threadfence();
  if (threadIdx.x == 0) P.fcnt[(size_t)k * c.f + f] = 0;  // re-armed for the next level / graph replay
  pick_body(c, P, d, f, k, false, 0.0, 0);
}

// ------------------------------------------------------------------ pick --

__device__ __forceinline__ bool better(double ga, int fa, int ba, double gb, int fb, int bb) {
  if (ga != gb) return ga > gb;
  if (fa != fb) return fa < fb;
  return ba < bb;
}

// Called by the 256 threads (= bins) of the scan block that completes feature
// f of class k: sums the node-group partials of every bin (or takes the
// block's own sums, `direct`), keeps the best bin (lowest bin on equal gain)
// and the runner-up; the last feature block of the class (completion
// counter, no waiting) reduces the features in ascending order -- the
// reference keeps the first strictly greater gain, i.e. lowest feature then
// lowest bin -- applies the stop rule and records the split.
__device__ void pick_body(const DevCfg& c, const DevPtrs& P, int d, int f, int k, bool direct, double s_in,
                          uint8_t any_in) {
  __shared__ double s_g[256], s_2[256];
  __shared__ int s_b[256];
  __shared__ bool s_last;
  ClassState& cs = P.cs[k];
  const int b = threadIdx.x;
  const int ngroups = ((1 << d) + SCAN_NODES - 1) / SCAN_NODES;
  double s = s_in;
  uint8_t any = any_in;
  if (!direct) {
    const size_t o = ((size_t)k * c.f + f) * c.n_scan_groups_max * kSlots + b;
    for (int g = 0; g < ngroups; ++g) {
      s += P.gpart[o + (size_t)g * kSlots];
      any |= P.gany[o + (size_t)g * kSlots];
    }
  }
  const bool cand = b < c.nb_scan && (d > 0 || any);
  s_g[b] = cand ? s : -1e300;
  s_2[b] = -1e300;
  s_b[b] = cand ? b : 0x7fffffff;
  __syncthreads();
  for (int stride = 128; stride > 0; stride >>= 1) {
    if (b < stride) {
      const int q = b + stride;
      const double rest = fmax(s_2[b], s_2[q]);
      if (better(s_g[q], 0, s_b[q], s_g[b], 0, s_b[b])) {
        s_2[b] = fmax(s_g[b], rest);
        s_g[b] = s_g[q];
        s_b[b] = s_b[q];
      } else {
        s_2[b] = fmax(s_g[q], rest);
      }
    }
    __syncthreads();
  }
  if (b == 0) {
    FeatBest fb;
    fb.gain = s_g[0];
    fb.second = s_2[0];
    fb.b = s_b[0];
    fb.valid = s_b[0] != 0x7fffffff;
    P.fbest[(size_t)k * c.f + f] = fb;
    __threadfence();
    const uint32_t prev = atomicAdd(&P.counters[k], 1u);
    s_last = prev == c.f - 1;
  }
  __syncthreads();
  if (!s_last) return;
  // last block of class k: reduce the features (fixed order per thread, then a tree)
  __threadfence();
  double bg = -1e300, b2 = -1e300;
  int bf = 0x7fffffff, bbin = 0x7fffffff;
  for (int ff = b; ff < (int)c.f; ff += blockDim.x) {
    const FeatBest fb = P.fbest[(size_t)k * c.f + ff];
    if (!fb.valid) continue;
    const double rest = fmax(b2, fb.second);
    if (better(fb.gain, ff, fb.b, bg, bf, bbin)) {
      b2 = fmax(bg, rest);
      bg = fb.gain; bf = ff; bbin = fb.b;
    } else {
      b2 = fmax(fb.gain, rest);
    }
  }
  __syncthreads();
  s_g[b] = bg; s_2[b] = b2; s_b[b] = bbin;
  __shared__ int s_f[256];
  s_f[b] = bf;
  __syncthreads();
  for (int stride = 128; stride > 0; stride >>= 1) {
    if (b < stride) {
      const int q = b + stride;
      const double rest = fmax(s_2[b], s_2[q]);
      if (better(s_g[q], s_f[q], s_b[q], s_g[b], s_f[b], s_b[b])) {
        s_2[b] = fmax(s_g[b], rest);
        s_g[b] = s_g[q]; s_f[b] = s_f[q]; s_b[b] = s_b[q];
      } else {
        s_2[b] = fmax(s_g[q], rest);
      }
    }
    __syncthreads();
  }
  if (b == 0) {
    P.counters[k] = 0;  // re-armed for the next level / graph replay
    const double best = s_g[0];
    const int bf0 = s_f[0], bb0 = s_b[0];
    const int t = *P.iter * c.KT + c.k0 + k;
    // no candidate (the reference's gain stays -1e30) or below
    // min_split_gain (src/tree/symmetric_tree.cpp:276-278; FP32 compare there)
    if (bf0 == 0x7fffffff || (float)best < c.msg) {
      cs.done = 1;
      return;
    }
    float thr = 0.0f;
    const int ne = P.n_edges[bf0];
    if (bb0 < ne) thr = P.edges[(size_t)bf0 * kSlots + bb0];
    else if (ne > 0) thr = P.edges[(size_t)bf0 * kSlots + ne - 1];
    P.m_feat[(size_t)t * c.D + d] = (uint16_t)bf0;
    P.m_bin[(size_t)t * c.D + d] = (uint8_t)bb0;
    P.m_thr[(size_t)t * c.D + d] = thr;
    P.m_gain[(size_t)t * c.D + d] = best;
    P.m_second[(size_t)t * c.D + d] = s_2[0];
    cs.f = bf0;
    cs.b = bb0;
    cs.depth = d + 1;
  }
}

// ------------------------------------------------------------- partition --

// grid (PB, K).  Rows of the split level get their child leaf index
// (2*leaf + right, right = bin != 255 && bin > t) and every block counts its
// sampled rows per child; the children's (grad, hess) sums come from their
// parent's histogram (the reduce kernel), so no row's (grad, hess) is read
// here.  With 2 or 4 children (8 when a thread has many rows) every thread
// counts in registers and each warp reduces once at the end; with 16-256
// children the lanes add into per-warp copies of the counts with shared
// atomics, except that when one node holds more than 1/8 of the rows its two
// children are counted in registers; beyond that a warp's rows are grouped
// per distinct child (a match over the warp) first.  Four rows per thread are
// loaded before any is used.
constexpr int PART_UNROLL = 4;
template <int NCH>  // 2, 4, 8 children: per-thread register counts; 0: per-warp child groups;
                    // -1: per-lane atomics into per-warp copies of the counts, the skewed
                    // level's largest node counted in registers
__global__ void __launch_bounds__(PART_THREADS) k_partition(DevCfg c, DevPtrs P, int d) {
  extern __shared__ unsigned char smraw[];
  const int k = blockIdx.y;
  const ClassState cs = P.cs[k];
  if (cs.done || cs.depth != d + 1) return;
  const int nch = 1 << (d + 1);
  const int ncopy = NCH < 0 ? PART_THREADS / 32 : 1;  // copies of the counts (one per warp)
  uint32_t* sC = reinterpret_cast<uint32_t*>(smraw);
  for (int q = threadIdx.x; q < nch * ncopy; q += blockDim.x) sC[q] = 0;
  __syncthreads();
  const uint32_t rpb = (c.n + gridDim.x - 1) / gridDim.x;
  const uint32_t r0 = blockIdx.x * rpb, r1 = min(c.n, r0 + rpb);
  const uint8_t* col = P.bins_cm + (size_t)cs.f * c.np;
  uint16_t* leaf = P.leaf + (size_t)k * c.n;
  const uint8_t t = (uint8_t)cs.b;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  constexpr int NR = NCH > 0 ? NCH : 1;
  uint32_t ac[NR];
#pragma unroll
  for (int cc = 0; cc < NR; ++cc) ac[cc] = 0;
  uint32_t hc[2] = {0u, 0u};  // NCH < 0, skewed level: the largest node's children
  for (uint32_t base = r0; base < r1; base += blockDim.x * PART_UNROLL) {
    uint8_t bb[PART_UNROLL];
    uint16_t lf[PART_UNROLL];
#pragma unroll
    for (int u = 0; u < PART_UNROLL; ++u) {
      const uint32_t i = base + u * blockDim.x + threadIdx.x;
      if (i < r1) {
        bb[u] = col[i];
        lf[u] = leaf[i];
      }
    }
#pragma unroll
    for (int u = 0; u < PART_UNROLL; ++u) {
      const uint32_t i = base + u * blockDim.x + threadIdx.x;
      int nl = -1;
      if (i < r1) {
        const uint32_t right = (bb[u] != (uint8_t)kNanBin && bb[u] > t) ? 1u : 0u;
        nl = (int)(((uint32_t)lf[u] << 1) | right);
        leaf[i] = (uint16_t)nl;
        if (!row_sampled(c, P, i)) nl = -1;  // its leaf moves on; it is not counted
      }
      if (NCH > 0) {
#pragma unroll
        for (int cc = 0; cc < NR; ++cc) ac[cc] += nl == cc ? 1u : 0u;
      } else if (NCH < 0) {
        if (nl >= 0) {
          if (cs.skew && (nl >> 1) == cs.hot) hc[nl & 1] += 1u;
          else atomicAdd(&sC[warp * nch + nl], 1u);
        }
      } else {
        // the first lane of each child's group adds the group's size
        const unsigned m = __match_any_sync(0xffffffffu, nl);
        if (nl >= 0 && lane == __ffs(m) - 1) atomicAdd(&sC[nl], (uint32_t)__popc(m));
      }
    }
  }
  if (NCH > 0) {
#pragma unroll
    for (int cc = 0; cc < NR; ++cc) {
      const uint32_t cnt = __reduce_add_sync(0xffffffffu, ac[cc]);
      if (lane == 0 && cnt) atomicAdd(&sC[cc], cnt);
    }
  }
  if (NCH < 0 && cs.skew) {
#pragma unroll
    for (int cc = 0; cc < 2; ++cc) {
      const uint32_t cnt = __reduce_add_sync(0xffffffffu, hc[cc]);
      if (lane == 0 && cnt) atomicAdd(&sC[warp * nch + 2 * cs.hot + cc], cnt);
    }
  }
  __syncthreads();
  const int L = 1 << c.D;
  for (int q = threadIdx.x; q < nch; q += blockDim.x) {
    uint32_t cn = 0;
    for (int w = 0; w < ncopy; ++w) cn += sC[w * nch + q];  // the warps' copies
    P.pcnt[((size_t)k * c.PB + blockIdx.x) * L + q] = cn;
  }
}

// grid (pairs, K), 512 threads (>= PB).  Child totals (fixed-order FP64
// sums over blocks), the smaller sibling (left on a tie,
// src/tree/symmetric_tree.cpp:337-339) and each block's scatter offset of
// its rows of the smaller child (exclusive scan over blocks).
__device__ __forceinline__ void node_reduce_body(const DevCfg& c, const DevPtrs& P, int d) {
  const int k = blockIdx.y, p = blockIdx.x;
  const ClassState cs = P.cs[k];
  const bool root = d < 0;  // root reduction after the gradient pass
  if (!root && (cs.done || cs.depth != d + 1)) return;
  const int L = 1 << c.D;
  __shared__ double s_g[2][512], s_h[2][512];
  __shared__ uint32_t s_c[2][512];
  __shared__ uint32_t s_w[16];
  const int nkids = root ? 1 : 2;
  const int blk = threadIdx.x;
  uint32_t my_cnt[2] = {0, 0};
  // row counts per child from the partition blocks; (G, H) of the root from
  // the gradient pass's block sums, of two children from their parent's
  // histogram row of the split feature: left = NaN slot + bins 0 .. b,
  // right = bins b+1 .. 254 (exact sums of the level's histogram)
  const double2* hrow = root ? nullptr : P.hist[d & 1] + hist_index(c, k, p, cs.f, 0);
  for (int kid = 0; kid < nkids; ++kid) {
    const int child = root ? 0 : 2 * p + kid;
    double g = 0.0, h = 0.0;
    uint32_t cn = 0;
    if (blk < c.PB) {
      const size_t o = ((size_t)k * c.PB + blk) * L + child;
      if (root) {
        const double2 v = P.psum[o];
        g = v.x;
        h = v.y;
      }
      cn = P.pcnt[o];
    }
    if (!root && blk < kSlots) {
      const bool left = blk == kNanBin || blk <= cs.b;
      if (left == (kid == 0)) {
        const double2 v = hrow[blk];
        g = v.x;
        h = v.y;
      }
    }
    my_cnt[kid] = cn;
    s_g[kid][blk] = g; s_h[kid][blk] = h; s_c[kid][blk] = cn;
  }
  __syncthreads();
  for (int s = 256; s > 0; s >>= 1) {
    if (blk < s) {
      for (int kid = 0; kid < nkids; ++kid) {
        s_g[kid][blk] += s_g[kid][blk + s];
        s_h[kid][blk] += s_h[kid][blk + s];
        s_c[kid][blk] += s_c[kid][blk + s];
      }
    }
    __syncthreads();
  }
  const int lvl = root ? 0 : d + 1;
  NodeStat* ns = P.nstat + ((size_t)k * (c.D + 1) + lvl) * L;
  if (root) {
    if (blk == 0) ns[0] = NodeStat{s_g[0][0], s_h[0][0], s_c[0][0], 0};
    return;
  }
  const uint32_t cl = s_c[0][0], cr = s_c[1][0];
  const int sm = (cl <= cr) ? 0 : 1;
  const int Pmax = 1 << (c.D - 1);
  if (blk == 0) {
    // an empty child has zero sums (its parent's histogram row is not
    // written when the parent itself is empty)
    ns[2 * p] = cl ? NodeStat{s_g[0][0], s_h[0][0], cl, 0} : NodeStat{0.0, 0.0, 0u, 0};
    ns[2 * p + 1] = cr ? NodeStat{s_g[1][0], s_h[1][0], cr, 0} : NodeStat{0.0, 0.0, 0u, 0};
    if (d + 1 < c.D) {
      P.small[k * Pmax + p] = 2 * p + sm;
      P.seg_len[k * Pmax + p] = (int)(sm ? cr : cl);
    }
  }
  if (d + 1 >= c.D) return;
  // exclusive scan over blocks of the smaller child's counts
  const uint32_t v = my_cnt[sm];
  const int lane = blk & 31, warp = blk >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) s_w[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += s_w[w];
  if (blk < c.PB) P.blk_off[((size_t)k * c.PB + blk) * Pmax + p] = before + x - v;
}

// One block.  For the level d about to be histogrammed: per class the stop
// pre-check (src/tree/symmetric_tree.cpp:116-124) and, for a finished tree,
// its leaf values (src/tree/symmetric_tree.cpp:357-367, 753-775); then the
// rows per chunk for this level and the cumulative chunk counts over
// (class, pair, feature group), which the histogram kernel decodes into work
// items.
constexpr int kPlanSegs = 4096;  // (class, pair) segment lengths the plan keeps in shared memory

__device__ __forceinline__ void plan_body(const DevCfg& c, const DevPtrs& P, int d) {
  __shared__ long long s_rows;
  __shared__ int s_nodes;
  __shared__ int s_warp[32];
  __shared__ int s_carry;
  __shared__ int s_len[kPlanSegs];  // [class][pair] rows of level d (0: the class grows no more)
  const int Pmax = 1 << (c.D - 1);
  const int L = 1 << c.D;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = (int)(blockDim.x >> 5);
  const int np2 = pairs_at(d);
  const int nsg = c.K * np2;
  const bool cached = nsg <= kPlanSegs;
  if (tid == 0) { s_rows = 0; s_nodes = 0; }
  __syncthreads();
  // Per class, one warp each (classes w, w + warps, ...): no block barriers.
  for (int k = warp; k < c.K; k += nwarps) {
    ClassState& cs = P.cs[k];
    int done = cs.done, depth = cs.depth;
    if (d == 0) { done = 0; depth = 0; }
    if (d == 0 && c.nv > 0 && P.es->stopped) done = 2;  // early-stopped: no more trees
    const bool alive = !done && (d == 0 || depth == d) && d < c.D;
    int go = 0;
    if (alive) {
      const NodeStat* ns = P.nstat + ((size_t)k * (c.D + 1) + d) * L;
      uint32_t maxcnt = 0;
      for (int q = lane; q < (1 << d); q += 32) {
        const uint32_t cnt = ns[q].cnt;
        if (cnt >= (uint32_t)c.msl * 2u && (float)ns[q].H >= c.mcw * 2.0f) go = 1;
        maxcnt = max(maxcnt, cnt);
      }
      go = __any_sync(0xffffffffu, go);
      for (int o = 16; o; o >>= 1) maxcnt = max(maxcnt, __shfl_xor_sync(0xffffffffu, maxcnt, o));
      int hot = INT32_MAX;  // the largest node, the lowest index on a tie
      for (int q = lane; q < (1 << d); q += 32)
        if (ns[q].cnt == maxcnt) hot = min(hot, q);
      for (int o = 16; o; o >>= 1) hot = min(hot, __shfl_xor_sync(0xffffffffu, hot, o));
      if (lane == 0) {
        const uint32_t tot = P.nstat[((size_t)k * (c.D + 1)) * L].cnt;  // rows of the level (the root's count)
        cs.skew = (uint64_t)maxcnt * 8u > (uint64_t)tot ? 1 : 0;
        cs.hot = hot == INT32_MAX ? 0 : hot;
      }
    }
    if (!done && !(alive && go)) done = 1;
    if (done == 1) {
      // the tree is complete: its leaves (src/tree/symmetric_tree.cpp:357-367, 753-775)
      const int t = *P.iter * c.KT + c.k0 + k;
      const NodeStat* ns = P.nstat + ((size_t)k * (c.D + 1) + depth) * L;
      for (int q = lane; q < L; q += 32) {
        float v = 0.0f;
        if (q < (1 << depth)) {
          const double H = ns[q].H;
          if (H >= 1e-10) {
            double x = -ns[q].G / (H + (double)c.lam);
            const double l1 = (double)c.l1;
            if (l1 > 0) x = x > l1 ? x - l1 : (x < -l1 ? x + l1 : 0.0);
            const double md = (double)c.mds;
            if (md > 0) x = fmax(-md, fmin(md, x));
            v = (float)x;
          }
        }
        P.m_leaves[(size_t)t * L + q] = v;
      }
      if (lane == 0) P.m_depth[t] = depth;
      done = 2;
    }
    if (!done) {
      // segment starts (exclusive scan over the pairs' lengths), 32 at a time
      int carry = 0;
      for (int base = 0; base < np2; base += 32) {
        const int p = base + lane;
        const int len = p < np2 ? (d == 0 ? (int)c.n : P.seg_len[k * Pmax + p]) : 0;
        int x = len;
        for (int o = 1; o < 32; o <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, x, o);
          if (lane >= o) x += y;
        }
        if (p < np2) {
          P.seg_start[k * Pmax + p] = carry + x - len;
          if (cached) s_len[k * np2 + p] = len;
        }
        carry += __shfl_sync(0xffffffffu, x, 31);
      }
      if (lane == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&s_rows), (unsigned long long)carry);
        atomicAdd(&s_nodes, np2);
      }
    } else if (cached) {
      for (int p = lane; p < np2; p += 32) s_len[k * np2 + p] = 0;
    }
    __syncwarp();
    if (lane == 0) {
      if (d == 0) cs.depth = 0;
      cs.done = done;
    }
  }
  __syncthreads();
  // rows of segment sgi (class, pair) for the chunking below
  auto seg_rows = [&](int sgi) -> int {
    if (cached) return s_len[sgi];
    const int k = sgi / np2, p = sgi % np2;
    if (P.cs[k].done) return 0;
    return d == 0 ? (int)c.n : P.seg_len[k * Pmax + p];
  };
  // Rows per chunk for this level: the smallest R (from the even split up)
  // for which the level has at most target_items items.  Every group counts,
  // the narrow last one too: measured, items that all run in one wave beat
  // a second wave of cheap narrow items after the wide ones.
  __shared__ int s_R;
  __shared__ long long s_cnt;
  const int gw = c.G;
  if (tid == 0) {
    int R = c.rows_fixed;
    if (R <= 0) R = (int)max((long long)c.rows_min, (s_rows * gw + c.target_items - 1) / c.target_items);
    s_R = min(R, kHistRowsMax);
  }
  __syncthreads();
  for (int round = 0; c.rows_fixed <= 0 && round < 16; ++round) {
    const int Rt = s_R;
    if (tid == 0) s_cnt = 0;
    __syncthreads();
    long long mine = 0;
    for (int sgi = tid; sgi < nsg; sgi += blockDim.x) mine += (seg_rows(sgi) + Rt - 1) / Rt;
    for (int o = 16; o; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
    if (lane == 0 && mine) atomicAdd(reinterpret_cast<unsigned long long*>(&s_cnt), (unsigned long long)mine);
    __syncthreads();
    const long long items = s_cnt * gw;
    __syncthreads();
    if (items <= c.target_items) break;
    if (tid == 0) s_R = (int)min((long long)kHistRowsMax, (long long)Rt * items / c.target_items + 1);
    __syncthreads();
  }
  if (tid == 0) {
    *P.rchunk = s_R;
    s_carry = 0;
  }
  __syncthreads();
  const int R = s_R;
  // cumulative item counts over segments (class, pair): chunks x groups
  for (int base = 0; base < nsg; base += blockDim.x) {
    const int sgi = base + tid;
    const int chunks = sgi < nsg ? (seg_rows(sgi) + R - 1) / R * c.G : 0;
    int x = chunks;
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    int before = s_carry;
    for (int w = 0; w < warp; ++w) before += s_warp[w];
    if (sgi < nsg) P.cum[sgi] = min(before + x - chunks, c.item_cap);
    __syncthreads();
    if (tid == blockDim.x - 1) s_carry = before + x;
    __syncthreads();
  }
  if (tid == 0) {
    P.cum[nsg] = min(s_carry, c.item_cap);
    *P.hist_ctr = 0;
    if (d < 16) {
      P.lvl_rows[d] = (uint64_t)s_rows;
      P.lvl_nodes[d] = (uint32_t)s_nodes;
    }
  }
}

__global__ void __launch_bounds__(PLAN_THREADS) k_plan(DevCfg c, DevPtrs P, int d) { plan_body(c, P, d); }

// grid (nodes of level d, K): the reduce above; with FUSE_PLAN the last block
// to finish (completion counter, nobody waits) also plans level d + 1, so a
// level needs one launch less.
template <bool FUSE_PLAN>
__global__ void __launch_bounds__(512) k_node_reduce(DevCfg c, DevPtrs P, int d) {
  node_reduce_body(c, P, d);
  if (FUSE_PLAN) {
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      const uint32_t prev = atomicAdd(P.red_ctr, 1u);
      s_last = prev == gridDim.x * gridDim.y - 1;
    }
    __syncthreads();
    if (s_last) {
      __threadfence();
      if (threadIdx.x == 0) *P.red_ctr = 0;  // re-armed for the next launch / graph replay
      plan_body(c, P, d + 1);
    }
  }
}

// grid (PB, K).  Row ids of the smaller children, grouped by pair, and their
// (grad, hess) in the same order (the next level's histogram reads them
// contiguously).
constexpr int SCAT_UNROLL = 4;
__global__ void __launch_bounds__(PART_THREADS) k_scatter(DevCfg c, DevPtrs P, int d) {
  extern __shared__ uint32_t s_cur[];  // [np2] counters, [np2] list offsets of this block, [np2] smaller child
  const int k = blockIdx.y;
  if (P.cs[k].done) return;
  const int Pmax = 1 << (c.D - 1);
  const int np2 = 1 << d;  // pairs at level d+1
  uint32_t* s_base = s_cur + np2;
  int* s_small = reinterpret_cast<int*>(s_base + np2);
  for (int q = threadIdx.x; q < np2; q += blockDim.x) {
    s_cur[q] = 0;
    s_base[q] = P.seg_start[k * Pmax + q] + P.blk_off[((size_t)k * c.PB + blockIdx.x) * Pmax + q];
    s_small[q] = P.small[k * Pmax + q];
  }
  __syncthreads();
  const uint32_t rpb = (c.n + gridDim.x - 1) / gridDim.x;
  const uint32_t r0 = blockIdx.x * rpb, r1 = min(c.n, r0 + rpb);
  const uint16_t* leaf = P.leaf + (size_t)k * c.n;
  uint32_t* rows = P.rows + (size_t)k * c.n;
  const float2* gh = P.gh + (size_t)k * c.n;
  float2* cgh = P.cgh + (size_t)k * c.n;
  const int lane = threadIdx.x & 31;
  const unsigned lt = (1u << lane) - 1u;
  for (uint32_t base = r0; base < r1; base += blockDim.x * SCAT_UNROLL) {
    // SCAT_UNROLL rows per thread: leaf indices, then the kept rows' (grad, hess)
    int key[SCAT_UNROLL];  // pair of a smaller-child row, else -1
    float2 g[SCAT_UNROLL];
#pragma unroll
    for (int u = 0; u < SCAT_UNROLL; ++u) {
      const uint32_t i = base + u * blockDim.x + threadIdx.x;
      key[u] = -1;
      if (i < r1 && row_sampled(c, P, i)) {
        const int ch = leaf[i];
        if (ch == s_small[ch >> 1]) key[u] = ch >> 1;
      }
    }
#pragma unroll
    for (int u = 0; u < SCAT_UNROLL; ++u)
      if (key[u] >= 0) g[u] = gh[base + u * blockDim.x + threadIdx.x];
#pragma unroll
    for (int u = 0; u < SCAT_UNROLL; ++u) {
      // a group of 32 rows without a smaller-child row needs no slot (most
      // groups on deep, skewed levels)
      if (__ballot_sync(0xffffffffu, key[u] >= 0) == 0u) continue;
      // one shared atomic per distinct pair of the warp; lanes keep their order
      const unsigned m = __match_any_sync(0xffffffffu, key[u]);
      const int leader = __ffs(m) - 1;
      uint32_t slot = 0;
      if (key[u] >= 0 && lane == leader) slot = atomicAdd(&s_cur[key[u]], (uint32_t)__popc(m));
      slot = __shfl_sync(0xffffffffu, slot, leader) + __popc(m & lt);
      if (key[u] >= 0) {
        const uint32_t pos = s_base[key[u]] + slot;
        rows[pos] = base + u * blockDim.x + threadIdx.x;
        cgh[pos] = g[u];
      }
    }
  }
}

__global__ void k_next_iter(DevPtrs P) { *P.iter += 1; }

// Validation set after an iteration (Booster::train's valid_data branch,
// src/boosting/booster.cpp:255-371; multiclass src/boosting/booster.cpp:1405-1435):
// the iteration's trees are added to the validation predictions (lr * leaf,
// FP32 fused multiply-add as the reference's compiled update), the loss is
// each loss's compute_loss term (FP32 per row as the reference,
// src/boosting/loss.cpp:110-121, 232-244, 336-346, 475-503; the sum in FP64
// here, in a fixed order), and the last block applies the stopping rule:
// improvement when loss < best - 1e-10 (FP32 compare); stop once
// iteration >= max(50, n_estimators/10) and early_stopping_rounds
// iterations in a row did not improve.
__device__ __forceinline__ float valid_term(const DevCfg& c, const float* pr, float y) {
  if (c.loss == TC_LOSS_MSE) {
    const float diff = pr[0] - y;
    return diff * diff;
  }
  if (c.loss == TC_LOSS_LOGLOSS) {
    float p = 1.0f / (1.0f + expf(-pr[0]));
    p = fmaxf(1e-7f, fminf(1.0f - 1e-7f, p));
    return -y * logf(p) - (1.0f - y) * logf(1.0f - p);
  }
  if (c.loss == TC_LOSS_FOCAL) {
    // RobustFocalLoss with the reference's defaults: mu = 0.1 (config robust_mu),
    // class weights 1 (set_class_weights is never called)
    const float p = 1.0f / (1.0f + expf(-pr[0]));
    float pt = y * p + (1.0f - y) * (1.0f - p);
    const float robust = 1.0f - 0.1f * powf(fabsf(2.0f * pt - 1.0f), 2.0f);
    pt = fmaxf(pt, 1e-7f);
    const float at = y * c.alpha + (1.0f - y) * (1.0f - c.alpha);
    const float focal = powf(1.0f - pt, c.gamma);
    return -at * focal * robust * 1.0f * logf(pt);
  }
  // softmax cross entropy (src/boosting/loss.cpp:273-285 softmax)
  float mx = pr[0];
  for (int k = 1; k < c.K; ++k) mx = fmaxf(mx, pr[k]);
  float sum = 0.0f, el = 0.0f;
  const int label = (int)y;
  for (int k = 0; k < c.K; ++k) {
    const float e = expf(pr[k] - mx);
    sum += e;
    if (k == label) el = e;
  }
  return -logf(fmaxf(el / sum, 1e-7f));
}

__global__ void __launch_bounds__(256) k_valid(DevCfg c, DevPtrs P) {
  __shared__ double s_part[256];
  __shared__ bool s_last;
  const int it = *P.iter;
  EsState* es = P.es;
  const bool stopped = es->stopped != 0;
  const int L = 1 << c.D;
  double part = 0.0;
  for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < c.nv; r += gridDim.x * blockDim.x) {
    float pr[kSoftmaxMaxK];
    const float* xr = P.xv + (size_t)r * c.f;
    for (int k = 0; k < c.K; ++k) {
      float vp = P.vpred[(size_t)k * c.nv + r];
      if (!stopped) {
        const size_t t = (size_t)it * c.KT + c.k0 + k;
        const int dep = P.m_depth[t];
        uint32_t idx = 0;
        for (int d = 0; d < dep; ++d)
          idx = (idx << 1) | (uint32_t)(xr[P.m_feat[t * c.D + d]] >= P.m_thr[t * c.D + d]);  // false for NaN
        vp = __fmaf_rn(c.lr, P.m_leaves[t * L + idx], vp);
        P.vpred[(size_t)k * c.nv + r] = vp;
      }
      pr[k] = vp;
    }
    part += (double)valid_term(c, pr, P.yv[r]);
  }
  s_part[threadIdx.x] = part;
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h) s_part[threadIdx.x] += s_part[threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    P.vpart[blockIdx.x] = s_part[0];
    __threadfence();
    s_last = atomicAdd(&es->ctr, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!s_last || threadIdx.x != 0) return;
  __threadfence();
  es->ctr = 0;
  double sum = 0.0;
  for (int b = 0; b < (int)gridDim.x; ++b) sum += P.vpart[b];
  const float loss = (float)(sum / (double)c.nv);
  P.vloss[it] = sum / (double)c.nv;
  if (stopped) return;
  if (loss < es->best - 1e-10f) {
    es->best = loss;
    es->best_iter = it;
    es->no_improve = 0;
  } else {
    ++es->no_improve;
  }
  if (c.es_rounds >= 0 && it >= c.es_min_iter && es->no_improve >= c.es_rounds) {
    es->stopped = 1;
    es->stop_iter = it;
  }
}

__global__ void k_fill_f32(float* p, size_t n, float v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) p[i] = v;
}

__global__ void k_root_hist_out(DevCfg c, DevPtrs P) {
  // root histogram of class 0 (level 0, node 0), FP64 [F][256][2]
  const double2* h = P.hist[0];
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < (size_t)c.f * kSlots;
       q += (size_t)gridDim.x * blockDim.x) {
    const double2 v = h[q];
    P.root_hist_out[2 * q] = v.x;
    P.root_hist_out[2 * q + 1] = v.y;
  }
}

}  // namespace
}  // namespace tc

// ---------------------------------------------------------------- trainer --

using namespace tc;

#define TC_CUDA_VOID(call) (void)(call)

struct tc_trainer {
  tc_ctx* ctx = nullptr;
  tc_dataset* ds = nullptr;
  tc_train_params prm{};
  DevCfg cfg{};
  DevPtrs ptr{};
  int J = 2;
  int hist_grid = 0;
  int T_cap = 0;
  int iters_done = 0;
  float base = 0.0f;
  bool base_known = false;       // base computed from the labels (they do not change)
  double seconds = 0.0;
  bool scores_dirty = false;
  cudaGraphExec_t graph = nullptr;       // one iteration (batched path)
  cudaGraphExec_t graph_goss = nullptr;  // a GOSS iteration after its host-side selection
  void drop_graphs() {
    if (graph) cudaGraphExecDestroy(graph);
    if (graph_goss) cudaGraphExecDestroy(graph_goss);
    graph = graph_goss = nullptr;
  }
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  DevBuf<float> pred;
  DevBuf<float2> gh, cgh;
  DevBuf<uint16_t> leaf;
  DevBuf<uint32_t> rows;
  DevBuf<double2> hist0, hist1;
  DevBuf<double2> acc;
  DevBuf<int32_t> cum, rchunk, seg_start, seg_len, small, iter;
  DevBuf<FeatBest> fbest;
  DevBuf<uint32_t> counters;
  DevBuf<int32_t> hist_ctr;
  DevBuf<uint32_t> red_ctr, fcnt;
  DevBuf<NodeStat> nstat;
  DevBuf<uint32_t> pcnt, blk_off;
  DevBuf<double2> psum;
  DevBuf<double> gpart;
  DevBuf<uint8_t> gany;
  DevBuf<ClassState> cs;
  DevBuf<int32_t> m_depth;
  DevBuf<uint16_t> m_feat;
  DevBuf<uint8_t> m_bin;
  DevBuf<float> m_thr, m_leaves;
  DevBuf<double> m_gain, m_second;
  DevBuf<double> root_hist;
  DevBuf<uint64_t> lvl_rows;     // per-level build-set rows / nodes (profiling)
  DevBuf<uint32_t> lvl_nodes;
  // validation set and early stopping (optional)
  const tc_dataset* vds = nullptr;
  DevBuf<float> vpred;
  DevBuf<double> vpart, vloss;
  DevBuf<EsState> es;
  bool es_stopped = false;       // the host has seen the stopping rule fire
  int best_iter = -1;
  // row sampling (optional): per-iteration bit masks made on the host
  bool sampling = false;
  uint64_t rng_state = 0;
  DevBuf<uint32_t> smask;
  uint32_t* h_mask = nullptr;    // pinned: 2 sets x SAMPLE_CHUNK masks
  cudaEvent_t mask_ev[2] = {nullptr, nullptr};
  int mask_set = 0;
  // GOSS (optional): the sample of an iteration is chosen on the host from
  // its gradients
  bool goss = false;
  float2* h_gh = nullptr;        // pinned: the iteration's (grad, hess) of every row and class
  uint32_t* h_gmask = nullptr;   // pinned: its sample mask
  std::vector<std::pair<float, uint32_t>> goss_rank;

  ~tc_trainer() {
    for (cudaEvent_t e : mask_ev)
      if (e) cudaEventDestroy(e);
    if (h_mask) cudaFreeHost(h_mask);
    if (h_gh) cudaFreeHost(h_gh);
    if (h_gmask) cudaFreeHost(h_gmask);
    for (cudaEvent_t e : ev_pool) cudaEventDestroy(e);
    drop_graphs();
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
  }

  bool given_gh = false;
  bool tuned = false;
  int hist_waves = 2;
  int hist_rows_min = 512;  // smallest rows per histogram work item
  int64_t launches = 0;
  int launches_per_iter = 0;
  // profiling: when prof != nullptr every launch is bracketed by events
  struct ProfRec {
    int cls;
    cudaEvent_t a, b;
    double bytes;
    int level;
    double rows;
  };
  std::vector<ProfRec>* prof = nullptr;
  bool prof_capture = false;     // profiling events become external event-record nodes of a graph
  std::vector<cudaEvent_t> ev_pool;
  size_t ev_used = 0;
  int cur_cls = -1;
  void mark_begin(int cls, cudaStream_t st);
  void mark_end(cudaStream_t st, double bytes = 0.0);
  tc_status setup(int given_gh_rows_only);
  tc_status configure(int J, int waves);
  tc_status autotune();
  void launch_level(const DevCfg& c, const DevPtrs& P, int d, cudaStream_t st);
  tc_status enqueue_iteration(cudaStream_t st);
  tc_status enqueue_rest(cudaStream_t st);
  tc_status run_plain_iteration(cudaStream_t st, bool grad = true);
  uint64_t next_random();
  tc_status enable_goss();
  void goss_select(uint64_t seed, uint32_t* words);
  tc_status goss_iteration(cudaStream_t st);
  tc_status init_predictions();
  tc_status init_validation();
  tc_status set_validation(const tc_dataset* v, int rounds);
  tc_status enable_sampling();
  void make_masks(int m, uint32_t* out);
  tc_status launch_iterations(int m, cudaStream_t st);
  tc_status step(int iters, bool sync);
};

tc_status tc_trainer::setup(int) {
  const uint32_t n = ds->n, f = ds->f;
  const int K = prm.loss == TC_LOSS_SOFTMAX ? prm.n_classes : 1;
  const int D = prm.max_depth;
  const int PB = ctx->sm_count * 2;
  if (PB > 512) return ctx->fail(TC_ERR_INVALID_ARG, "too many SMs for the partition reduction");
  const int Pmax = 1 << (D - 1);
  const int L = 1 << D;
  const int ngroups_max = (L / 2 + SCAN_NODES - 1) / SCAN_NODES;
  const int G = 1, W = 32;  // placeholders until configure()

  cfg.n = n; cfg.f = f; cfg.np = ds->np;
  cfg.groups = ds->groups; cfg.wlast = ds->wlast; cfg.gstride = ds->gstride;
  cfg.K = K; cfg.KT = K; cfg.k0 = 0; cfg.D = D; cfg.nb_scan = (int)(uint8_t)prm.max_bins - 1; cfg.loss = prm.loss;
  cfg.msl = prm.min_samples_leaf; cfg.lr = prm.learning_rate; cfg.lam = prm.lambda_l2; cfg.l1 = prm.lambda_l1;
  cfg.mcw = prm.min_child_weight; cfg.msg = prm.min_split_gain; cfg.mds = prm.max_delta_step;
  cfg.gamma = prm.focal_gamma; cfg.alpha = prm.focal_alpha;
  cfg.G = G; cfg.W = W; cfg.PB = PB;
  cfg.n_scan_groups_max = std::max(1, ngroups_max);
  cfg.rows_min = 512;
  cfg.rows_fixed = prm.hist_rows_per_chunk > 0 ? std::min(prm.hist_rows_per_chunk, kHistRowsMax) : 0;
  // MSE's hessian is 2 for every row (src/boosting/loss.cpp:348-362)
  // counted hessians need every listed row to carry h = 2; with row
  // sampling the root lists all rows and the unsampled ones carry 0
  cfg.hconst = (prm.loss == TC_LOSS_MSE && !given_gh && !(prm.subsample > 0.0f && prm.subsample < 1.0f) &&
                !prm.use_goss)
                   ? 2.0f : 0.0f;

  T_cap = prm.n_estimators * K;
  TC_TRY(pred.alloc(ctx, (size_t)K * n, "predictions"));
  TC_TRY(gh.alloc(ctx, (size_t)K * n, "gradients"));
  TC_TRY(cgh.alloc(ctx, (size_t)K * n, "gradients of the row lists"));
  TC_TRY(leaf.alloc(ctx, (size_t)K * n, "leaf ids"));
  TC_TRY(rows.alloc(ctx, (size_t)K * n, "row lists"));
  const size_t hsz = (size_t)K * Pmax * f * kSlots;
  TC_TRY(hist0.alloc(ctx, hsz, "level histograms"));
  TC_TRY(hist1.alloc(ctx, hsz, "level histograms"));
  TC_TRY(acc.alloc(ctx, hsz, "histogram accumulators"));
  TC_CUDA(ctx, cudaMemset(acc.p, 0, acc.bytes()));
  TC_TRY(rchunk.alloc(ctx, 1, "chunk rows"));
  TC_TRY(seg_start.alloc(ctx, (size_t)K * Pmax, "segments"));
  TC_TRY(seg_len.alloc(ctx, (size_t)K * Pmax, "segments"));
  TC_TRY(small.alloc(ctx, (size_t)K * Pmax, "segments"));
  TC_TRY(iter.alloc(ctx, 1, "iteration"));
  TC_TRY(nstat.alloc(ctx, (size_t)K * (D + 1) * L, "node stats"));
  TC_TRY(pcnt.alloc(ctx, (size_t)K * PB * L, "partition counts"));
  TC_TRY(psum.alloc(ctx, (size_t)K * PB * L, "partition sums"));
  TC_TRY(blk_off.alloc(ctx, (size_t)K * PB * Pmax, "scatter offsets"));
  TC_TRY(gpart.alloc(ctx, (size_t)K * f * cfg.n_scan_groups_max * kSlots, "gain partials"));
  TC_TRY(gany.alloc(ctx, (size_t)K * f * cfg.n_scan_groups_max * kSlots, "gain flags"));
  TC_TRY(fbest.alloc(ctx, (size_t)K * f, "feature bests"));
  TC_TRY(counters.alloc(ctx, K, "pick counters"));
  TC_TRY(hist_ctr.alloc(ctx, 1, "histogram item counter"));
  TC_TRY(red_ctr.alloc(ctx, 1, "reduce completion counter"));
  TC_TRY(fcnt.alloc(ctx, (size_t)K * f, "scan completion counters"));
  TC_TRY(cs.alloc(ctx, K, "class state"));
  TC_TRY(m_depth.alloc(ctx, T_cap, "model"));
  TC_TRY(m_feat.alloc(ctx, (size_t)T_cap * D, "model"));
  TC_TRY(m_bin.alloc(ctx, (size_t)T_cap * D, "model"));
  TC_TRY(m_thr.alloc(ctx, (size_t)T_cap * D, "model"));
  TC_TRY(m_gain.alloc(ctx, (size_t)T_cap * D, "model"));
  TC_TRY(m_second.alloc(ctx, (size_t)T_cap * D, "model"));
  TC_TRY(m_leaves.alloc(ctx, (size_t)T_cap * L, "model"));
  TC_TRY(lvl_rows.alloc(ctx, 16, "level rows"));
  TC_TRY(lvl_nodes.alloc(ctx, 16, "level nodes"));
  TC_CUDA(ctx, cudaMemset(lvl_rows.p, 0, lvl_rows.bytes()));
  TC_CUDA(ctx, cudaMemset(lvl_nodes.p, 0, lvl_nodes.bytes()));
  TC_CUDA(ctx, cudaMemset(counters.p, 0, counters.bytes()));
  TC_CUDA(ctx, cudaMemset(red_ctr.p, 0, red_ctr.bytes()));
  TC_CUDA(ctx, cudaMemset(fcnt.p, 0, fcnt.bytes()));

  ptr.bins_t = ds->bins_t.p; ptr.bins_cm = ds->bins_cm.p; ptr.edges = ds->edges.p; ptr.n_edges = ds->n_edges.p;
  ptr.nan_any = ds->nan_any.p;
  ptr.y = ds->y.p; ptr.pred = pred.p; ptr.gh = gh.p; ptr.cgh = cgh.p; ptr.leaf = leaf.p; ptr.rows = rows.p;
  ptr.hist[0] = hist0.p; ptr.hist[1] = hist1.p; ptr.acc = acc.p; ptr.rchunk = rchunk.p;
  ptr.seg_start = seg_start.p; ptr.seg_len = seg_len.p; ptr.small = small.p; ptr.nstat = nstat.p;
  ptr.pcnt = pcnt.p; ptr.psum = psum.p; ptr.blk_off = blk_off.p; ptr.gpart = gpart.p; ptr.gany = gany.p;
  ptr.fbest = fbest.p; ptr.counters = counters.p; ptr.hist_ctr = hist_ctr.p; ptr.red_ctr = red_ctr.p; ptr.fcnt = fcnt.p; ptr.cs = cs.p; ptr.iter = iter.p;
  ptr.m_depth = m_depth.p; ptr.m_feat = m_feat.p; ptr.m_bin = m_bin.p; ptr.m_thr = m_thr.p; ptr.m_gain = m_gain.p;
  ptr.m_second = m_second.p; ptr.m_leaves = m_leaves.p; ptr.root_hist_out = nullptr;
  ptr.lvl_rows = lvl_rows.p; ptr.lvl_nodes = lvl_nodes.p;

  cudaFuncSetAttribute(k_hist<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HistShape::smem);
  cudaFuncSetAttribute(k_hist<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)HistShape::smem);
  cudaFuncSetAttribute(k_partition<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * L);
  cudaFuncSetAttribute(k_partition<-1>, cudaFuncAttributeMaxDynamicSharedMemorySize, 4 * 256 * (PART_THREADS / 32));
  TC_CUDA(ctx, cudaEventCreate(&ev0));
  TC_CUDA(ctx, cudaEventCreate(&ev1));
  return configure(1, 2);  // 32-column feature groups (the only width), 2 waves before tuning
}

// Feature-group width (32*J columns) and work items per histogram launch
// (waves x resident histogram blocks); (re)sizes the partial buffer.
tc_status tc_trainer::configure(int J_, int waves) {
  const uint32_t f = cfg.f;
  const int K = cfg.K, D = cfg.D;
  const int Pmax = 1 << (D - 1);
  J = J_;
  const int W = 32 * J;
  const int G = (int)((f + W - 1) / W);
  hist_grid = ctx->sm_count;  // one 1024-thread block per SM
  hist_waves = waves;
  long long cap = (long long)waves * hist_grid + (long long)K * Pmax * G + 1;
  if (cfg.rows_fixed) cap += (long long)K * G * ((cfg.n + cfg.rows_fixed - 1) / cfg.rows_fixed + 1);
  cap += (long long)K * G * (cfg.n / kHistRowsMax + 1);  // chunks of at most kHistRowsMax rows
  cfg.G = G;
  cfg.W = W;
  cfg.hist_grid = hist_grid;
  cfg.target_items = waves * hist_grid;
  cfg.rows_min = hist_rows_min;
  cfg.item_cap = (int)cap;

  TC_TRY(cum.alloc(ctx, (size_t)K * Pmax * G + 1, "chunk counts"));
  ptr.cum = cum.p;
  drop_graphs();
  return TC_OK;
}

namespace {
std::mutex g_tune_mu;
std::map<std::string, std::array<int, 3>> g_tune_cache;  // shape -> (J, waves, rows_min)
}  // namespace

// Project autotuner: times a few iterations for every items-per-launch
// candidate (1, 2, 4, 8 waves of histogram work items) on this dataset shape,
// keeps the fastest, caches it per (rows, features, depth, classes, SMs) and
// restarts the model from the base prediction.
tc_status tc_trainer::autotune() {
  char key[160];
  snprintf(key, sizeof(key), "%u/%u/%d/%d/%d/%d", cfg.n, cfg.f, cfg.D, cfg.K, ctx->sm_count, prm.loss);
  {
    std::lock_guard<std::mutex> g(g_tune_mu);
    auto it = g_tune_cache.find(key);
    if (it != g_tune_cache.end()) {
      hist_rows_min = it->second[2];
      TC_TRY(configure(it->second[0], it->second[1]));
      tuned = true;
      return TC_OK;
    }
  }
  cudaStream_t st = ctx->stream;
  // 64-column groups (one block per SM) measured slower on every configuration
  // (C2: 1.7 vs 1.2 ms/iteration, C3: 9.3 vs 7.0); they stay available as a
  // parameter but are not tried
  const int jmax = 1;
  double best = 1e30;
  int bj = J, bw = hist_waves, br = hist_rows_min;
  // candidates (waves, rows_min): 1, 2, 4, 8 waves of items of at least 512
  // rows; on small shapes also one wave of larger items (fewer items flush
  // fewer partial histograms into the same accumulators)
  std::vector<std::pair<int, int>> cand = {{1, 512}, {2, 512}, {4, 512}, {8, 512}};
  if ((long long)cfg.n * (long long)((cfg.f + 31) / 32) <= 8LL * ctx->sm_count * 8192) {
    cand.push_back({1, 2048});
    cand.push_back({1, 8192});
  }
  // every candidate restarts from the base prediction and replays the same
  // first iterations; the best of two timed runs of them counts
  const int trial_iters = 2;  // + 1 warm-up: 3 <= n_estimators iterations (checked by the caller)
  for (int rep = 0; rep < 2; ++rep) {
    for (int j = 1; j <= jmax; ++j) {
      for (const auto& wr : cand) {
        const int waves = wr.first;
        hist_rows_min = wr.second;
        TC_TRY(configure(j, waves));
        TC_TRY(init_predictions());
        enqueue_iteration(st);  // warm-up (first touch of the buffers)
        TC_TRY(init_predictions());
        TC_CUDA(ctx, cudaEventRecord(ev0, st));
        for (int i = 0; i < trial_iters; ++i) enqueue_iteration(st);
        TC_CUDA(ctx, cudaEventRecord(ev1, st));
        TC_CUDA(ctx, cudaEventSynchronize(ev1));
        float ms = 0.0f;
        TC_CUDA(ctx, cudaEventElapsedTime(&ms, ev0, ev1));
        if (ms < best) {
          best = ms;
          bj = j;
          bw = waves;
          br = hist_rows_min;
        }
      }
    }
  }
  hist_rows_min = br;
  TC_TRY(configure(bj, bw));
  TC_TRY(init_predictions());
  launches = 0;
  tuned = true;
  std::lock_guard<std::mutex> g(g_tune_mu);
  g_tune_cache[key] = {bj, bw, br};
  return TC_OK;
}

enum { KC_GRAD, KC_HIST, KC_MERGE, KC_SCAN, KC_PART, KC_REDUCE, KC_SCATTER, KC_OTHER, KC_N };
static const char* kKernelNames[KC_N] = {"grad", "hist", "merge", "scan_pick", "partition",
                                         "reduce_plan", "scatter", "other"};

void tc_trainer::mark_begin(int cls, cudaStream_t st) {
  ++launches;
  if (!prof) return;
  if (ev_used + 2 > ev_pool.size()) {
    for (int i = 0; i < 64; ++i) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
  }
  ProfRec r{cls, ev_pool[ev_used], ev_pool[ev_used + 1], 0.0, -1, 0.0};
  ev_used += 2;
  if (prof_capture) cudaEventRecordWithFlags(r.a, st, cudaEventRecordExternal);
  else cudaEventRecord(r.a, st);
  prof->push_back(r);
}

void tc_trainer::mark_end(cudaStream_t st, double bytes) {
  if (!prof) return;
  if (prof_capture) cudaEventRecordWithFlags(prof->back().b, st, cudaEventRecordExternal);
  else cudaEventRecord(prof->back().b, st);
  prof->back().bytes = bytes;
}

// Algorithmic bytes of a histogram launch over `rows` listed rows and `nodes`
// built nodes: rows x (F bin bytes + 8 bytes of (grad, hess) + 1 byte of node
// id) + nodes x F x 255 bins x 8 bytes of (grad, hess) sums.
static double hist_alg_bytes(double rows, double nodes, uint32_t f) {
  return rows * ((double)f + 9.0) + nodes * (double)f * 255.0 * 8.0;
}

// All launches of level d for the classes of view (c, P).
void tc_trainer::launch_level(const DevCfg& c, const DevPtrs& P, int d, cudaStream_t st) {
  const int K = c.K, D = c.D;
  double hist_bytes = 0.0, hist_rows = 0.0;
  if (prof && !prof_capture) {
    // algorithmic bytes: rows histogrammed at this level (device counts)
    TC_CUDA_VOID(cudaStreamSynchronize(st));
    std::vector<ClassState> h(K);
    cudaMemcpy(h.data(), P.cs, K * sizeof(ClassState), cudaMemcpyDeviceToHost);
    const int Pmax = 1 << (D - 1);
    double rows = 0.0, nodes = 0.0;
    for (int k = 0; k < K; ++k) {
      if (h[k].done) continue;
      if (d == 0) {
        rows += c.n;
        nodes += 1;
      } else {
        std::vector<int32_t> sl(1 << (d - 1));
        cudaMemcpy(sl.data(), P.seg_len + (size_t)k * Pmax, sl.size() * sizeof(int32_t), cudaMemcpyDeviceToHost);
        for (int32_t v : sl) rows += v;
        nodes += (double)sl.size();
      }
    }
    hist_bytes = hist_alg_bytes(rows, nodes, c.f);
    hist_rows = rows;
  }
  mark_begin(KC_HIST, st);
  if (c.hconst > 0.0f) k_hist<true><<<hist_grid, HIST_THREADS, HistShape::smem, st>>>(c, P, d);
  else k_hist<false><<<hist_grid, HIST_THREADS, HistShape::smem, st>>>(c, P, d);
  mark_end(st, hist_bytes);
  if (prof) {
    prof->back().level = d;
    prof->back().rows = hist_rows;
  }
  const int ng = ((1 << d) + SCAN_NODES - 1) / SCAN_NODES;
  mark_begin(KC_SCAN, st);
  k_scan<<<dim3(c.f, ng, K), SCAN_WARPS * 32, 0, st>>>(c, P, d);  // + pick
  mark_end(st);
  mark_begin(KC_PART, st);
  {
    const dim3 pg(c.PB, K);
    const size_t psm = 4 * (2 << d);
    // register counts pay a fixed per-warp reduction at the end: for 8
    // children they win only with enough rows per thread
    const bool many_rows = c.n / (uint32_t)c.PB >= 16u * PART_THREADS;
    if (d == 0) k_partition<2><<<pg, PART_THREADS, psm, st>>>(c, P, d);
    else if (d == 1) k_partition<4><<<pg, PART_THREADS, psm, st>>>(c, P, d);
    else if (d == 2 && many_rows) k_partition<8><<<pg, PART_THREADS, psm, st>>>(c, P, d);
    else if (d >= 3 && (2 << d) <= 256)
      k_partition<-1><<<pg, PART_THREADS, psm * (PART_THREADS / 32), st>>>(c, P, d);
    else k_partition<0><<<pg, PART_THREADS, psm, st>>>(c, P, d);
  }
  mark_end(st, (double)c.n * K * (1 + 2 + 2));
  if (prof) prof->back().level = d;
  mark_begin(KC_REDUCE, st);
  k_node_reduce<true><<<dim3(1 << d, K), 512, 0, st>>>(c, P, d);  // + plan of level d + 1
  mark_end(st);
  if (d + 1 < D) {
    mark_begin(KC_SCATTER, st);
    k_scatter<<<dim3(c.PB, K), PART_THREADS, 3 * sizeof(uint32_t) * (1 << d), st>>>(c, P, d);
    mark_end(st);
  }
}

// The whole iteration as a fixed launch sequence (graph-capturable).
static void launch_grad(const DevCfg& c, const DevPtrs& P, int use_given_gh, cudaStream_t st) {
  if (c.K > 1) k_grad<true><<<c.PB, 512, 0, st>>>(c, P, use_given_gh);
  else k_grad<false><<<c.PB, 512, 0, st>>>(c, P, use_given_gh);
}

tc_status tc_trainer::enqueue_iteration(cudaStream_t st) {
  mark_begin(KC_GRAD, st);
  launch_grad(cfg, ptr, 0, st);
  mark_end(st, (double)cfg.n * cfg.K * (4 + 4 + 8 + 2 + 8) + (double)cfg.n * 4);
  return enqueue_rest(st);
}

// An iteration after its gradients: root reduce (+ plan of level 0), the
// levels, the validation step and the iteration counter.
tc_status tc_trainer::enqueue_rest(cudaStream_t st) {
  const int K = cfg.K, D = cfg.D;
  mark_begin(KC_REDUCE, st);
  k_node_reduce<true><<<dim3(1, K), 512, 0, st>>>(cfg, ptr, -1);  // + plan of level 0
  mark_end(st);
  for (int d = 0; d < D; ++d) launch_level(cfg, ptr, d, st);
  if (cfg.nv > 0) {
    mark_begin(KC_OTHER, st);
    k_valid<<<VALID_BLOCKS, 256, 0, st>>>(cfg, ptr);
    mark_end(st, (double)cfg.nv * (cfg.f * 4.0 + 4.0 + cfg.K * 8.0));
  }
  mark_begin(KC_OTHER, st);
  k_next_iter<<<1, 1, 0, st>>>(ptr);
  mark_end(st);
  return TC_OK;
}

// Class-k view of the device state (K = 1 launches of the plain path).
static DevPtrs class_view(const DevCfg& c, const DevPtrs& P, int k, DevCfg* one) {
  DevPtrs pk = P;
  const size_t n = c.n;
  const int Pmax = 1 << (c.D - 1), L = 1 << c.D;
  *one = c;
  one->K = 1;
  one->k0 = k;
  pk.pred += k * n; pk.gh += k * n; pk.cgh += k * n; pk.leaf += k * n; pk.rows += k * n;
  pk.hist[0] += (size_t)k * Pmax * c.f * kSlots;
  pk.hist[1] += (size_t)k * Pmax * c.f * kSlots;
  pk.acc += (size_t)k * Pmax * c.f * kSlots;
  pk.seg_start += k * Pmax; pk.seg_len += k * Pmax;
  pk.small += k * Pmax; pk.nstat += (size_t)k * (c.D + 1) * L;
  pk.fbest += (size_t)k * c.f; pk.counters += k; pk.fcnt += (size_t)k * c.f;
  pk.pcnt += (size_t)k * c.PB * L; pk.psum += (size_t)k * c.PB * L; pk.blk_off += (size_t)k * c.PB * Pmax;
  pk.gpart += (size_t)k * c.f * c.n_scan_groups_max * kSlots;
  pk.gany += (size_t)k * c.f * c.n_scan_groups_max * kSlots;
  pk.cs += k;
  return pk;
}

// The plain path: one class and one level per launch group, a host
// synchronisation after every level (the host reads the stop flag), no graph.
tc_status tc_trainer::run_plain_iteration(cudaStream_t st, bool grad) {
  const int K = cfg.K, D = cfg.D;
  if (grad) launch_grad(cfg, ptr, 0, st);
  k_node_reduce<false><<<dim3(1, K), 512, 0, st>>>(cfg, ptr, -1);
  for (int k = 0; k < K; ++k) {
    DevCfg one;
    DevPtrs pk = class_view(cfg, ptr, k, &one);
    k_plan<<<1, PLAN_THREADS, 0, st>>>(one, pk, 0);
    for (int d = 0; d < D; ++d) {
      TC_CUDA(ctx, cudaStreamSynchronize(st));
      ClassState h;
      TC_CUDA(ctx, cudaMemcpy(&h, pk.cs, sizeof(h), cudaMemcpyDeviceToHost));
      if (h.done) break;
      launch_level(one, pk, d, st);
    }
  }
  if (cfg.nv > 0) k_valid<<<VALID_BLOCKS, 256, 0, st>>>(cfg, ptr);
  k_next_iter<<<1, 1, 0, st>>>(ptr);
  TC_CUDA(ctx, cudaGetLastError());
  return TC_OK;
}

tc_status tc_trainer::init_predictions() {
  cudaStream_t st = ctx->stream;
  // base prediction on the host from the labels (Loss::init_prediction,
  // src/boosting/loss.cpp:217-226, 364-370, 545-553; 0 for softmax)
  if (!base_known) base = 0.0f;
  if (!base_known && prm.loss != TC_LOSS_SOFTMAX && !given_gh) {
    std::vector<float> y(cfg.n);
    TC_CUDA(ctx, cudaMemcpyAsync(y.data(), ds->y.p, cfg.n * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaStreamSynchronize(st));
    float sum = 0.0f;
    for (uint32_t i = 0; i < cfg.n; ++i) sum += y[i];
    float p = sum / (float)cfg.n;
    if (prm.loss == TC_LOSS_MSE) {
      base = p;
    } else {
      p = std::max(1e-7f, std::min(1.0f - 1e-7f, p));
      base = std::log(p / (1.0f - p));
    }
  }
  base_known = true;
  k_fill_f32<<<4 * ctx->sm_count, 256, 0, st>>>(pred.p, (size_t)cfg.K * cfg.n, base);
  TC_CUDA(ctx, cudaGetLastError());
  TC_CUDA(ctx, cudaMemsetAsync(leaf.p, 0, leaf.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(iter.p, 0, sizeof(int32_t), st));
  TC_CUDA(ctx, cudaMemsetAsync(cs.p, 0, cs.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_depth.p, 0, m_depth.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_feat.p, 0, m_feat.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_bin.p, 0, m_bin.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_thr.p, 0, m_thr.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_gain.p, 0, m_gain.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_second.p, 0, m_second.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(m_leaves.p, 0, m_leaves.bytes(), st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  iters_done = 0;
  seconds = 0.0;
  rng_state = prm.seed;  // Booster: rng_state_ = config_.seed (src/boosting/booster.cpp:35-41)
  if (cfg.nv > 0) TC_TRY(init_validation());
  return TC_OK;
}

constexpr int SAMPLE_CHUNK = 8;  // iterations per host batch of sample masks / early-stopping look

// Booster::next_random (src/boosting/booster.cpp:1219-1225): xorshift64*.
uint64_t tc_trainer::next_random() {
  uint64_t x = rng_state;
  x ^= x >> 12;
  x ^= x << 25;
  x ^= x >> 27;
  rng_state = x;
  return x * 0x2545F4914F6CDD1DULL;
}

// Sample masks of the next m iterations, in iteration order: per iteration an
// xorshift64* draw seeds the row shuffle (src/boosting/booster.cpp:213-217,
// src/core/dataset.cpp:552-562: std::shuffle with std::mt19937_64, first
// (uint32)(n * subsample) rows), then one draw for the feature subset when
// colsample_bytree < 1 (booster.cpp:223-227; symmetric trees do not use it).
// The shuffles run on host threads, one per iteration.
void tc_trainer::make_masks(int m, uint32_t* out) {
  const uint32_t n = cfg.n;
  const size_t words = (n + 31) / 32;
  std::vector<uint64_t> seeds(m);
  for (int i = 0; i < m; ++i) {
    seeds[i] = next_random();
    if (prm.colsample_bytree > 0.0f && prm.colsample_bytree < 1.0f) (void)next_random();
  }
  const float ratio = prm.subsample;
  auto one = [n, words, ratio](uint64_t seed, uint32_t* w) {
    const uint32_t keep = static_cast<uint32_t>(n * ratio);  // Index * Float, as the reference
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    std::mt19937_64 rng(seed);
    std::shuffle(idx.begin(), idx.end(), rng);
    std::memset(w, 0, words * sizeof(uint32_t));
    for (uint32_t q = 0; q < keep; ++q) w[idx[q] >> 5] |= 1u << (idx[q] & 31);
  };
  std::vector<std::thread> th;
  for (int i = 1; i < m; ++i) th.emplace_back(one, seeds[i], out + (size_t)i * words);
  if (m > 0) one(seeds[0], out);
  for (auto& t : th) t.join();
}

tc_status tc_trainer::enable_sampling() {
  sampling = true;
  const size_t words = (cfg.n + 31) / 32;
  TC_TRY(smask.alloc(ctx, words, "row sample mask"));
  TC_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&h_mask), 2 * SAMPLE_CHUNK * words * sizeof(uint32_t),
                             cudaHostAllocDefault));
  for (cudaEvent_t& e : mask_ev) TC_CUDA(ctx, cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  TC_CUDA(ctx, cudaMemsetAsync(smask.p, 0xff, words * sizeof(uint32_t), ctx->stream));  // until the first sample
  cfg.sampled = 1;
  ptr.smask = smask.p;
  drop_graphs();
  return TC_OK;
}

tc_status tc_trainer::enable_goss() {
  goss = true;
  const size_t words = (cfg.n + 31) / 32;
  TC_TRY(smask.alloc(ctx, words, "row sample mask"));
  TC_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&h_gh), (size_t)cfg.K * cfg.n * sizeof(float2),
                             cudaHostAllocDefault));
  TC_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&h_gmask), words * sizeof(uint32_t), cudaHostAllocDefault));
  goss_rank.resize(cfg.n);
  TC_CUDA(ctx, cudaMemsetAsync(smask.p, 0xff, words * sizeof(uint32_t), ctx->stream));  // until the first sample
  cfg.sampled = 1;
  ptr.smask = smask.p;
  drop_graphs();
  return TC_OK;
}

// The sample of one GOSS iteration from its gradients in h_gh, as
// Dataset::goss_subsample (src/core/dataset.cpp:494-549): the
// (uint32)(n * top_rate) rows of largest |g| (std::nth_element over
// (|g|, row) pairs, descending), then (uint32)(n * other_rate) rows (at most
// the rest) taken by a partial Fisher-Yates shuffle of the rest as
// nth_element left it, std::uniform_int_distribution<uint32_t> over
// std::mt19937_64 seeded by `seed`.  Softmax ranks rows by the largest |g|
// over the classes (src/boosting/booster.cpp:1327-1348).  The draws reach
// positions of nth_element's arrangement, so the same library calls are
// made (libstdc++, as in the reference build); no other order would select
// the same rows.
void tc_trainer::goss_select(uint64_t seed, uint32_t* words) {
  const uint32_t n = cfg.n;
  const int K = cfg.K;
  std::memset(words, 0, ((n + 31) / 32) * sizeof(uint32_t));
  const uint32_t top_n = static_cast<uint32_t>(n * prm.goss_top_rate);  // Index * Float, as the reference
  uint32_t other_n = static_cast<uint32_t>(n * prm.goss_other_rate);
  if (top_n == 0 && other_n == 0) return;  // an empty sample: the trees are single leaves of 0
  auto& a = goss_rank;
  for (uint32_t i = 0; i < n; ++i) {
    float m = 0.0f;
    if (K == 1) {
      m = std::abs(h_gh[i].x);
    } else {
      for (int k = 0; k < K; ++k) m = std::max(m, std::abs(h_gh[(size_t)k * n + i].x));
    }
    a[i] = {m, i};
  }
  if (top_n > 0 && top_n < n)
    std::nth_element(a.begin(), a.begin() + top_n, a.end(),
                     [](const std::pair<float, uint32_t>& l, const std::pair<float, uint32_t>& r) {
                       return l.first > r.first;
                     });
  auto keep = [words](uint32_t row) { words[row >> 5] |= 1u << (row & 31); };
  for (uint32_t i = 0; i < top_n; ++i) keep(a[i].second);
  if (other_n > 0 && top_n < n) {
    const uint32_t rest = n - top_n;
    other_n = std::min(other_n, rest);
    std::mt19937_64 rng(seed);
    for (uint32_t i = 0; i < other_n; ++i) {
      std::uniform_int_distribution<uint32_t> pick(i, rest - 1);
      const uint32_t j = pick(rng);
      if (i != j) std::swap(a[top_n + i], a[top_n + j]);
      keep(a[top_n + i].second);
    }
  }
}

// One GOSS iteration: the gradients of every row (k_grad without a sample),
// copied to the host, which draws the iteration's random numbers (the GOSS
// seed, then the feature-subset draw when colsample_bytree < 1) and picks the
// sample; then the rest of the iteration (one graph on the batched path).
tc_status tc_trainer::goss_iteration(cudaStream_t st) {
  const uint32_t n = cfg.n;
  const size_t words = (n + 31) / 32;
  DevCfg all = cfg;
  all.sampled = 0;
  mark_begin(KC_GRAD, st);
  launch_grad(all, ptr, 0, st);
  mark_end(st, (double)n * cfg.K * (4 + 4 + 8 + 2 + 8) + (double)n * 4);
  TC_CUDA(ctx, cudaGetLastError());
  TC_CUDA(ctx, cudaMemcpyAsync(h_gh, gh.p, (size_t)cfg.K * n * sizeof(float2), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  const uint64_t seed = next_random();
  if (prm.colsample_bytree > 0.0f && prm.colsample_bytree < 1.0f) (void)next_random();
  goss_select(seed, h_gmask);
  TC_CUDA(ctx, cudaMemcpyAsync(smask.p, h_gmask, words * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  if (prm.batched && !prof) {
    if (!graph_goss) {
      cudaGraph_t g;
      const int64_t l0 = launches;
      TC_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
      k_goss_root<<<cfg.PB, 512, 0, st>>>(cfg, ptr);
      ++launches;
      enqueue_rest(st);
      TC_CUDA(ctx, cudaStreamEndCapture(st, &g));
      launches_per_iter = (int)(launches - l0);
      launches = l0;
      cudaError_t e = cudaGraphInstantiate(&graph_goss, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaGraphInstantiate");
    }
    TC_CUDA(ctx, cudaGraphLaunch(graph_goss, st));
    launches += launches_per_iter;
  } else if (prm.batched) {  // profiled: launch by launch
    mark_begin(KC_OTHER, st);
    k_goss_root<<<cfg.PB, 512, 0, st>>>(cfg, ptr);
    mark_end(st, (double)n * cfg.K * 8.0);
    enqueue_rest(st);
  } else {
    k_goss_root<<<cfg.PB, 512, 0, st>>>(cfg, ptr);
    TC_TRY(run_plain_iteration(st, false));
  }
  TC_CUDA(ctx, cudaGetLastError());
  return TC_OK;
}

// Validation predictions start at the base prediction (booster.cpp:93-96),
// the stopping state at best = 1e30 (booster.cpp:119-121).
tc_status tc_trainer::init_validation() {
  cudaStream_t st = ctx->stream;
  k_fill_f32<<<4 * ctx->sm_count, 256, 0, st>>>(vpred.p, (size_t)cfg.K * cfg.nv, base);
  TC_CUDA(ctx, cudaGetLastError());
  EsState h{};
  h.best = 1e30f;
  h.best_iter = 0;
  h.stop_iter = -1;
  TC_CUDA(ctx, cudaMemcpyAsync(es.p, &h, sizeof(h), cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaMemsetAsync(vloss.p, 0, vloss.bytes(), st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  es_stopped = false;
  best_iter = -1;
  return TC_OK;
}

tc_status tc_trainer::set_validation(const tc_dataset* v, int rounds) {
  if (v->ctx != ctx) return ctx->fail(TC_ERR_INVALID_ARG, "validation set belongs to another context");
  if (v->f != cfg.f) return ctx->fail(TC_ERR_INVALID_ARG, "validation set has %u features, training %u", v->f, cfg.f);
  if (v->n == 0 || v->y.n < v->n) return ctx->fail(TC_ERR_INVALID_ARG, "validation set needs rows and labels");
  if (iters_done > 0) return ctx->fail(TC_ERR_INVALID_ARG, "set the validation set before the first iteration");
  vds = v;
  cfg.nv = v->n;
  cfg.es_rounds = rounds;
  cfg.es_min_iter = std::max(50, prm.n_estimators / 10);
  TC_TRY(vpred.alloc(ctx, (size_t)cfg.K * v->n, "validation predictions"));
  TC_TRY(vpart.alloc(ctx, VALID_BLOCKS, "validation partial losses"));
  TC_TRY(vloss.alloc(ctx, std::max(1, prm.n_estimators), "validation losses"));
  TC_TRY(es.alloc(ctx, 1, "early-stopping state"));
  ptr.xv = v->X.p;
  ptr.yv = v->y.p;
  ptr.vpred = vpred.p;
  ptr.vpart = vpart.p;
  ptr.vloss = vloss.p;
  ptr.es = es.p;
  drop_graphs();
  return init_validation();
}

// One or more iterations on the stream: the captured graph (or the plain
// path); with row sampling each iteration is preceded by the copy of its
// sample mask, the masks of a batch being made on the host while the
// previous batch runs.
tc_status tc_trainer::launch_iterations(int m, cudaStream_t st) {
  if (goss) {
    for (int i = 0; i < m; ++i) TC_TRY(goss_iteration(st));
    return TC_OK;
  }
  if (prm.batched && !graph) {
    cudaGraph_t g;
    const int64_t l0 = launches;
    TC_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    enqueue_iteration(st);
    TC_CUDA(ctx, cudaStreamEndCapture(st, &g));
    launches_per_iter = (int)(launches - l0);
    launches = l0;
    cudaError_t e = cudaGraphInstantiate(&graph, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaGraphInstantiate");
  }
  const size_t words = (cfg.n + 31) / 32;
  uint32_t* set = nullptr;
  if (sampling) {
    TC_CUDA(ctx, cudaEventSynchronize(mask_ev[mask_set]));  // the set's previous copies are done
    set = h_mask + (size_t)mask_set * SAMPLE_CHUNK * words;
    make_masks(m, set);
  }
  for (int i = 0; i < m; ++i) {
    if (sampling)
      TC_CUDA(ctx, cudaMemcpyAsync(smask.p, set + (size_t)i * words, words * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, st));
    if (prm.batched) {
      TC_CUDA(ctx, cudaGraphLaunch(graph, st));
      launches += launches_per_iter;
    } else {
      TC_TRY(run_plain_iteration(st));
    }
  }
  if (sampling) {
    TC_CUDA(ctx, cudaEventRecord(mask_ev[mask_set], st));
    mask_set ^= 1;
  }
  return TC_OK;
}

tc_status tc_trainer::step(int iters, bool sync) {
  cudaStream_t st = ctx->stream;
  if (iters < 0 || iters_done + iters > prm.n_estimators)
    return ctx->fail(TC_ERR_INVALID_ARG, "step(%d) exceeds n_estimators=%d (done %d)", iters,
                     prm.n_estimators, iters_done);
  if (iters == 0 || es_stopped) return TC_OK;
  TC_CUDA(ctx, cudaEventRecord(ev0, st));
  int done = 0;
  if (cfg.nv == 0 && !sampling && !goss) {
    TC_TRY(launch_iterations(iters, st));
    done = iters;
  } else {
    // batches of iterations; with a validation set a look at the stopping
    // state after each (iterations launched past the stop grow no tree)
    while (done < iters && !es_stopped) {
      const int m = std::min(SAMPLE_CHUNK, iters - done);
      TC_TRY(launch_iterations(m, st));
      done += m;
      if (cfg.nv > 0) {
        EsState h{};
        TC_CUDA(ctx, cudaMemcpyAsync(&h, es.p, sizeof(h), cudaMemcpyDeviceToHost, st));
        TC_CUDA(ctx, cudaStreamSynchronize(st));
        best_iter = h.best_iter;
        if (h.stopped) {
          es_stopped = true;
          done = h.stop_iter + 1 - iters_done;  // trees up to and including the stopping iteration
        }
      }
    }
    sync = true;
  }
  TC_CUDA(ctx, cudaEventRecord(ev1, st));
  TC_CUDA(ctx, cudaGetLastError());
  iters_done += done;
  scores_dirty = true;
  if (sync) {
    TC_CUDA(ctx, cudaEventSynchronize(ev1));
    float ms = 0.0f;
    TC_CUDA(ctx, cudaEventElapsedTime(&ms, ev0, ev1));
    seconds += ms * 1e-3;
  }
  return TC_OK;
}

// ------------------------------------------------------------------ C ABI --

static tc_status validate(tc_ctx* ctx, const tc_dataset* ds, const tc_train_params* p) {
  if (!ds->quantized) return ctx->fail(TC_ERR_INVALID_ARG, "dataset is not quantized");
  if (p->max_depth < 1 || p->max_depth > kMaxDepth)
    return ctx->fail(TC_ERR_INVALID_ARG, "max_depth must be in [1, %d]", kMaxDepth);
  if (p->max_bins < 2 || p->max_bins > 255)
    return ctx->fail(TC_ERR_INVALID_ARG, "max_bins cannot exceed 255 (uint8 limit)");
  if (!(p->learning_rate > 0.0f) || p->learning_rate > 1.0f)
    return ctx->fail(TC_ERR_INVALID_ARG, "learning_rate must be in (0, 1]");
  if (p->loss < TC_LOSS_LOGLOSS || p->loss > TC_LOSS_SOFTMAX) return ctx->fail(TC_ERR_INVALID_ARG, "unknown loss");
  if (p->loss == TC_LOSS_SOFTMAX && (p->n_classes < 3 || p->n_classes > 16))
    return ctx->fail(TC_ERR_INVALID_ARG, "softmax needs 3 <= n_classes <= 16");
  if (p->n_estimators < 0) return ctx->fail(TC_ERR_INVALID_ARG, "n_estimators must be >= 0");
  if (ds->n == 0) return ctx->fail(TC_ERR_INVALID_ARG, "empty dataset");
  if (p->use_goss && !(p->goss_top_rate >= 0.0f && p->goss_top_rate <= 1.0f && p->goss_other_rate >= 0.0f &&
                       p->goss_other_rate <= 1.0f))
    return ctx->fail(TC_ERR_INVALID_ARG, "goss_top_rate and goss_other_rate must be in [0, 1]");
  if (p->loss != TC_LOSS_SOFTMAX || true) {
    if (!ds->y.p) return ctx->fail(TC_ERR_INVALID_ARG, "dataset has no labels");
  }
  return TC_OK;
}

extern "C" {

tc_status tc_trainer_create(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_trainer** out) {
  if (!ctx || !ds || !p || !out) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  *out = nullptr;
  cudaSetDevice(ctx->device);
  TC_TRY(validate(ctx, ds, p));
  tc_trainer* tr = new tc_trainer();
  tr->ctx = ctx;
  tr->ds = ds;
  tr->prm = *p;
  tc_status s = tr->setup(0);
  if (s == TC_OK) s = tr->init_predictions();
  // tuning runs up to three throw-away iterations: it needs that many tree slots
  if (s == TC_OK && p->hist_features_per_block == 0 && p->n_estimators >= 3) s = tr->autotune();
  // row sampling starts after tuning (the tuner's trial iterations use every row)
  if (s == TC_OK && p->use_goss) s = tr->enable_goss();  // GOSS is chosen over subsample (booster.cpp:200-219)
  else if (s == TC_OK && p->subsample > 0.0f && p->subsample < 1.0f) s = tr->enable_sampling();
  if (s != TC_OK) {
    delete tr;
    return s;
  }
  *out = tr;
  return TC_OK;
}

tc_status tc_trainer_step(tc_trainer* tr, int32_t iterations, int sync) {
  if (!tr) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(tr->ctx->train_mu);
  cudaSetDevice(tr->ctx->device);
  return tr->step(iterations, sync != 0);
}

tc_status tc_trainer_reset(tc_trainer* tr) {
  if (!tr) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(tr->ctx->train_mu);
  cudaSetDevice(tr->ctx->device);
  return tr->init_predictions();
}

tc_status tc_trainer_stats(tc_trainer* tr, tc_train_stats* st) {
  if (!tr || !st) return TC_ERR_INVALID_ARG;
  st->n_trees = tr->iters_done * tr->cfg.K;
  st->iterations_done = tr->iters_done;
  st->base_prediction = tr->base;
  st->seconds = tr->seconds;
  st->hist_features_per_block = tr->cfg.W;
  st->hist_rows_per_chunk = tr->cfg.rows_fixed ? tr->cfg.rows_fixed : -tr->cfg.target_items;
  st->kernel_launches = tr->launches;
  st->best_iteration = tr->cfg.nv > 0 ? tr->best_iter : -1;
  st->stopped_early = tr->es_stopped ? 1 : 0;
  return TC_OK;
}

tc_status tc_trainer_set_validation(tc_trainer* tr, const tc_dataset* valid, int32_t early_stopping_rounds) {
  if (!tr || !valid) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(tr->ctx->train_mu);
  cudaSetDevice(tr->ctx->device);
  return tr->set_validation(valid, early_stopping_rounds);
}

tc_status tc_trainer_valid_loss(tc_trainer* tr, double* out) {
  if (!tr || !out) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = tr->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  if (tr->cfg.nv == 0) return ctx->fail(TC_ERR_INVALID_ARG, "no validation set");
  cudaSetDevice(ctx->device);
  if (tr->iters_done > 0) {
    TC_CUDA(ctx, cudaMemcpyAsync(out, tr->vloss.p, tr->iters_done * sizeof(double), cudaMemcpyDeviceToHost,
                                 ctx->stream));
    TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  }
  return TC_OK;
}

// Harvests one profiled iteration's events into `out`; histogram launches
// get their algorithmic bytes from the level's build set when `lvl` is given
// (the in-graph path records it on the device).
static void harvest_profile(const std::vector<tc_trainer::ProfRec>& recs, const uint64_t* lvl_rows,
                            const uint32_t* lvl_nodes, uint32_t f, tc_profile* out) {
  for (const auto& r : recs) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, r.a, r.b);
    tc_kernel_time& k = out->k[r.cls];
    double bytes = r.bytes;
    double rows = r.rows;
    if (lvl_rows && r.cls == KC_HIST && r.level >= 0 && r.level < 16) {
      rows = (double)lvl_rows[r.level];
      bytes = hist_alg_bytes(rows, (double)lvl_nodes[r.level], f);
    }
    k.launches += 1;
    k.ms += ms;
    k.alg_bytes += bytes;
    if (r.level >= 0 && r.level < 16 && r.cls == KC_HIST) {
      out->hist_level_ms[r.level] += ms;
      out->hist_level_rows[r.level] += rows;
    }
    if (r.level >= 0 && r.level < 16 && r.cls == KC_PART) out->part_level_ms[r.level] += ms;
  }
  if (!recs.empty()) {
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, recs.front().a, recs.back().b);
    out->iteration_ms += ms;
  }
}

tc_status tc_trainer_profile(tc_trainer* tr, int32_t iterations, tc_profile* out) {
  if (!tr || !out || iterations < 0) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(tr->ctx->train_mu);
  tc_ctx* ctx = tr->ctx;
  cudaSetDevice(ctx->device);
  if (tr->iters_done + iterations > tr->prm.n_estimators)
    return ctx->fail(TC_ERR_INVALID_ARG, "profile(%d) exceeds n_estimators", iterations);
  cudaStream_t st = ctx->stream;
  std::vector<tc_trainer::ProfRec> recs;
  std::vector<uint32_t> mask;
  if (tr->sampling) mask.resize((tr->cfg.n + 31) / 32);
  auto copy_mask = [&]() -> tc_status {
    if (tr->sampling) {  // this iteration's row sample, as step() would use
      tr->make_masks(1, mask.data());
      TC_CUDA(ctx, cudaMemcpyAsync(tr->smask.p, mask.data(), mask.size() * sizeof(uint32_t),
                                   cudaMemcpyHostToDevice, st));
    }
    return TC_OK;
  };
  // The batched path is timed inside the graph it replays: the iteration is
  // captured once more with an event-record node around every launch, and
  // that graph is replayed per profiled iteration (the events of one replay
  // are read before the next).  GOSS iterations and the plain path, which
  // synchronise with the host inside an iteration, are timed launch by launch.
  const bool in_graph = tr->prm.batched && !tr->goss;
  out->in_graph = in_graph ? 1 : 0;
  if (in_graph) {
    tr->prof = &recs;
    tr->prof_capture = true;
    tr->ev_used = 0;
    const int64_t l0 = tr->launches;
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      tr->enqueue_iteration(st);
      e = cudaStreamEndCapture(st, &g);
    }
    tr->prof = nullptr;
    tr->prof_capture = false;
    const int64_t per_iter = tr->launches - l0;
    tr->launches = l0;
    if (e != cudaSuccess) return ctx->cuda_fail(e, "profiled iteration capture");
    cudaGraphExec_t gx = nullptr;
    e = cudaGraphInstantiate(&gx, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "profiled iteration instantiate");
    uint64_t lr[16];
    uint32_t ln[16];
    for (int i = 0; i < iterations; ++i) {
      tc_status ms = copy_mask();
      if (ms == TC_OK) {
        e = cudaGraphLaunch(gx, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = cudaMemcpy(lr, tr->lvl_rows.p, sizeof(lr), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(ln, tr->lvl_nodes.p, sizeof(ln), cudaMemcpyDeviceToHost);
      }
      if (ms != TC_OK || e != cudaSuccess) {
        cudaGraphExecDestroy(gx);
        return ms != TC_OK ? ms : ctx->cuda_fail(e, "profiled iteration");
      }
      harvest_profile(recs, lr, ln, tr->cfg.f, out);
      tr->launches += per_iter;
    }
    cudaGraphExecDestroy(gx);
  } else {
    tr->prof = &recs;
    tr->ev_used = 0;
    for (int i = 0; i < iterations; ++i) {
      tc_status ms = copy_mask();
      if (ms != TC_OK) {
        tr->prof = nullptr;
        return ms;
      }
      if (tr->goss) {
        tc_status gs = tr->goss_iteration(st);
        if (gs != TC_OK) {
          tr->prof = nullptr;
          return gs;
        }
      } else {
        tr->enqueue_iteration(st);
      }
      // harvest every iteration so that the event pool stays small
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        tr->prof = nullptr;
        return ctx->cuda_fail(e, "profiled iteration");
      }
      harvest_profile(recs, nullptr, nullptr, tr->cfg.f, out);
      recs.clear();
      tr->ev_used = 0;
    }
    tr->prof = nullptr;
  }
  tr->iters_done += iterations;
  tr->scores_dirty = true;
  out->n_kernels = KC_N;
  for (int c = 0; c < KC_N; ++c) {
    std::strncpy(out->k[c].name, kKernelNames[c], sizeof(out->k[c].name) - 1);
  }
  return TC_OK;
}

tc_status tc_trainer_sample_mask(tc_trainer* tr, uint32_t* out) {
  if (!tr || !out) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = tr->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  const uint32_t n = tr->cfg.n;
  const size_t words = (n + 31) / 32;
  if (tr->sampling || tr->goss) {
    TC_CUDA(ctx, cudaMemcpyAsync(out, tr->smask.p, words * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
    TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  } else {
    std::fill(out, out + words, 0xffffffffu);
  }
  if (n % 32) out[words - 1] &= (1u << (n % 32)) - 1u;
  return TC_OK;
}

tc_status tc_trainer_train_scores(tc_trainer* tr, float* out) {
  if (!tr || !out) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = tr->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  // apply the last tree to a scratch copy so that training can continue
  DevBuf<float> tmp;
  DevBuf<uint16_t> lf;
  TC_TRY(tmp.alloc(ctx, tr->pred.n, "score copy"));
  TC_TRY(lf.alloc(ctx, tr->leaf.n, "leaf copy"));
  TC_CUDA(ctx, cudaMemcpyAsync(tmp.p, tr->pred.p, tr->pred.bytes(), cudaMemcpyDeviceToDevice, st));
  TC_CUDA(ctx, cudaMemcpyAsync(lf.p, tr->leaf.p, tr->leaf.bytes(), cudaMemcpyDeviceToDevice, st));
  DevPtrs P = tr->ptr;
  P.pred = tmp.p;
  P.leaf = lf.p;
  k_apply_last<<<tr->ctx->sm_count * 4, 256, 0, st>>>(tr->cfg, P);
  const uint32_t n = tr->cfg.n;
  const int K = tr->cfg.K;
  std::vector<float> h((size_t)K * n);
  TC_CUDA(ctx, cudaMemcpyAsync(h.data(), tmp.p, h.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  for (uint32_t i = 0; i < n; ++i)
    for (int k = 0; k < K; ++k) out[(size_t)i * K + k] = h[(size_t)k * n + i];
  return TC_OK;
}

tc_status tc_trainer_model(tc_trainer* tr, tc_model** out) {
  if (!tr || !out) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = tr->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  cudaStream_t st = ctx->stream;
  const int K = tr->cfg.K, D = tr->cfg.D, L = 1 << D;
  const int T = tr->iters_done * K;
  tc_model* m = new tc_model();
  m->ctx = ctx;
  m->info.n_trees = T;
  m->info.n_classes = K;
  m->info.max_depth = D;
  m->info.n_features = (int)tr->cfg.f;
  m->info.task = tr->prm.loss == TC_LOSS_SOFTMAX ? TC_TASK_MULTICLASS
                 : (tr->prm.loss == TC_LOSS_MSE ? TC_TASK_REGRESSION : TC_TASK_BINARY);
  m->info.base_prediction = tr->base;
  m->info.learning_rate = tr->prm.learning_rate;
  m->info.lambda_l2 = tr->prm.lambda_l2;
  m->depth.resize(T);
  m->feature.resize((size_t)T * D);
  m->bin.resize((size_t)T * D);
  m->threshold.resize((size_t)T * D);
  m->gain.resize((size_t)T * D);
  m->leaves.resize((size_t)T * L);
  m->weights.assign(T, tr->prm.learning_rate);
  std::vector<double> g64((size_t)T * D);
  auto cp = [&](void* dst, const void* src, size_t bytes) {
    return cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, st);
  };
  cudaError_t e = cudaSuccess;
  if (T > 0) {
    e = cp(m->depth.data(), tr->m_depth.p, (size_t)T * sizeof(int32_t));
    if (e == cudaSuccess) e = cp(m->feature.data(), tr->m_feat.p, (size_t)T * D * sizeof(uint16_t));
    if (e == cudaSuccess) e = cp(m->bin.data(), tr->m_bin.p, (size_t)T * D);
    if (e == cudaSuccess) e = cp(m->threshold.data(), tr->m_thr.p, (size_t)T * D * sizeof(float));
    if (e == cudaSuccess) e = cp(g64.data(), tr->m_gain.p, (size_t)T * D * sizeof(double));
    if (e == cudaSuccess) e = cp(m->leaves.data(), tr->m_leaves.p, (size_t)T * L * sizeof(float));
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    delete m;
    return ctx->cuda_fail(e, "model download");
  }
  for (size_t q = 0; q < g64.size(); ++q) m->gain[q] = (float)g64[q];
  m->edges = tr->ds->h_edges;
  m->n_edges = tr->ds->h_n_edges;
  tc_status s = m->upload();
  if (s != TC_OK) {
    delete m;
    return s;
  }
  *out = m;
  return TC_OK;
}

void tc_trainer_destroy(tc_trainer* tr) {
  if (!tr) return;
  // serialised with the context's training calls: the stream may be capturing in another thread
  std::lock_guard<std::recursive_mutex> train_lock(tr->ctx->train_mu);
  cudaSetDevice(tr->ctx->device);
  cudaStreamSynchronize(tr->ctx->stream);
  delete tr;
}

tc_status tc_train(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_model** out, tc_train_stats* st) {
  if (!ctx || !ds || !p || !out) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  tc_trainer* tr = nullptr;
  TC_TRY(tc_trainer_create(ctx, ds, p, &tr));
  tc_status s = tr->step(p->n_estimators, true);
  if (s == TC_OK) s = tc_trainer_model(tr, out);
  if (s == TC_OK && st) tc_trainer_stats(tr, st);
  tc_trainer_destroy(tr);
  return s;
}

tc_status tc_build_tree(tc_ctx* ctx, tc_dataset* ds, const float* grad, const float* hess,
                        const tc_train_params* p, int32_t* depth_out, uint16_t* split_feature,
                        uint8_t* split_bin, float* split_threshold, double* split_gain,
                        double* runner_up_gain, float* leaf_values, uint32_t* leaf_index,
                        double* root_hist) {
  if (!ctx || !ds || !grad || !hess || !p || !depth_out) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  tc_train_params q = *p;
  q.loss = TC_LOSS_MSE;  // labels unused: gradients are given
  q.n_classes = 1;
  q.n_estimators = 1;
  if (!ds->quantized) return ctx->fail(TC_ERR_INVALID_ARG, "dataset is not quantized");
  if (q.max_depth < 1 || q.max_depth > kMaxDepth)
    return ctx->fail(TC_ERR_INVALID_ARG, "max_depth must be in [1, %d]", kMaxDepth);
  if (q.max_bins < 2 || q.max_bins > 255) return ctx->fail(TC_ERR_INVALID_ARG, "max_bins must be in [2, 255]");
  tc_trainer* tr = new tc_trainer();
  tr->ctx = ctx;
  tr->ds = ds;
  tr->prm = q;
  tr->given_gh = true;
  tc_status s = tr->setup(1);
  if (s == TC_OK) s = tr->init_predictions();
  if (s != TC_OK) {
    delete tr;
    return s;
  }
  cudaStream_t st = ctx->stream;
  const uint32_t n = ds->n;
  std::vector<float2> h(n);
  for (uint32_t i = 0; i < n; ++i) h[i] = make_float2(grad[i], hess[i]);
  DevBuf<double> rh;
  cudaError_t e = cudaMemcpyAsync(tr->gh.p, h.data(), n * sizeof(float2), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) { delete tr; return ctx->cuda_fail(e, "gradient upload"); }
  if (root_hist) {
    s = rh.alloc(ctx, (size_t)ds->f * kSlots * 2, "root histogram");
    if (s != TC_OK) { delete tr; return s; }
    tr->ptr.root_hist_out = rh.p;
  }
  // one iteration with the given gradients
  const int D = tr->cfg.D;
  launch_grad(tr->cfg, tr->ptr, 1, st);
  k_node_reduce<false><<<dim3(1, 1), 512, 0, st>>>(tr->cfg, tr->ptr, -1);
  k_plan<<<1, PLAN_THREADS, 0, st>>>(tr->cfg, tr->ptr, 0);
  for (int d = 0; d < D; ++d) {
    tr->launch_level(tr->cfg, tr->ptr, d, st);
    if (d == 0 && root_hist) k_root_hist_out<<<64, 256, 0, st>>>(tr->cfg, tr->ptr);
  }
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) { delete tr; return ctx->cuda_fail(e, "tree build"); }
  int32_t dep = 0;
  const int L = 1 << D;
  std::vector<uint16_t> lf;
  e = cudaMemcpy(&dep, tr->m_depth.p, sizeof(int32_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && split_feature) e = cudaMemcpy(split_feature, tr->m_feat.p, D * sizeof(uint16_t), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && split_bin) e = cudaMemcpy(split_bin, tr->m_bin.p, D, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && split_threshold) e = cudaMemcpy(split_threshold, tr->m_thr.p, D * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && split_gain) e = cudaMemcpy(split_gain, tr->m_gain.p, D * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && runner_up_gain) e = cudaMemcpy(runner_up_gain, tr->m_second.p, D * sizeof(double), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && leaf_values) e = cudaMemcpy(leaf_values, tr->m_leaves.p, L * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && leaf_index) {
    lf.resize(n);
    e = cudaMemcpy(lf.data(), tr->leaf.p, n * sizeof(uint16_t), cudaMemcpyDeviceToHost);
    for (uint32_t i = 0; i < n && e == cudaSuccess; ++i) leaf_index[i] = lf[i];
  }
  if (e == cudaSuccess && root_hist) e = cudaMemcpy(root_hist, rh.p, rh.bytes(), cudaMemcpyDeviceToHost);
  delete tr;
  if (e != cudaSuccess) return ctx->cuda_fail(e, "tree download");
  *depth_out = dep;
  return TC_OK;
}

}  // extern "C"
