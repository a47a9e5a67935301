// Regular (depth-wise) trees trained on the device: Booster::train with
// use_symmetric = false (src/boosting/booster.cpp:47-418, 447-520), Tree::build
// and its depth-wise recursion (src/tree/tree.cpp:162-407), SplitFinder
// (src/tree/histogram.cpp:569-690) and Tree::make_leaf (src/tree/tree.cpp:655-683).
//
// A tree grows level by level on the device: per level, one histogram of
// exact fixed-point sums per open node (64-bit integer atomics: order-free and
// exact, so a child's sums equal its parent's prefix sums bit for bit), one
// block per open node scoring every (feature, bin) in FP64 with the
// reference's first-maximum rule, and a partition of the rows by each node's
// own split.  The host reads each level's best splits (a few dozen bytes a
// node) and decides which nodes split.  The reference's recursion visits the
// smaller child's subtree first and stops splitting once 64 leaves exist;
// the host replays that order on the grown tree to apply the cap and to
// number the nodes as the reference does.  The finished tree updates the
// predictions on the device (fused multiply-add, as the reference's build)
// and the model is the reference's TCAT v3 regular-tree stream, served by
// the regular-tree predictor.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "tc_internal.h"
#include "tc_loss.cuh"

namespace tc {
namespace {

constexpr int RG_THREADS = 256;
constexpr int RG_SCAN_WARPS = 8;
constexpr int RG_MAX_LEAVES = 64;  // TreeConfig::max_leaves (include/turbocat/config.hpp:29)
constexpr int RG_SLOTS = 256;      // histogram slots per (node, feature): bins 0..254, NaN 255

struct RgBest {  // one open node: its exact totals and its best split
  double G, H;
  uint32_t C;
  int32_t feature;  // -1: no split meets the constraints
  int32_t bin;
  int32_t pad;
  double gain, GL, HL;
  uint32_t CL;
  uint32_t pad2;
};

// Per-row logloss gradients of the current predictions (the reference's
// arithmetic, tc_loss.cuh) and the largest |g| and h over the rows, as float
// bits (non-negative floats order as integers).
__global__ void k_rg_grad(const float* __restrict__ y, const float* __restrict__ pred, float2* __restrict__ gh,
                          uint32_t n, int loss, uint32_t* __restrict__ amax) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t mg = 0, mh = 0;
  if (i < n) {
    float g, h;
    loss_grad(loss, pred[i], y[i], i, (n / 8) * 8, 2.0f, 0.25f, g, h);
    gh[i] = make_float2(g, h);
    mg = __float_as_uint(fabsf(g));
    mh = __float_as_uint(fabsf(h));
  }
  for (int o = 16; o; o >>= 1) {
    mg = max(mg, __shfl_xor_sync(0xffffffffu, mg, o));
    mh = max(mh, __shfl_xor_sync(0xffffffffu, mh, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&amax[0], mg);
    atomicMax(&amax[1], mh);
  }
}

// Exact histograms of the open nodes: v = round(x * 2^e) added as 64-bit
// integers (two's complement), so sums are exact whatever the order.
__global__ void k_rg_hist(const uint8_t* __restrict__ bins, uint32_t np, uint32_t n, uint32_t f,
                          const int32_t* __restrict__ slot, const float2* __restrict__ gh, double sg, double sh,
                          unsigned long long* __restrict__ HG, unsigned long long* __restrict__ HH,
                          uint32_t* __restrict__ HC) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int32_t s = slot[r];
  if (s < 0) return;
  const float2 v = gh[r];
  const unsigned long long qg = (unsigned long long)llrint((double)v.x * sg);
  const unsigned long long qh = (unsigned long long)llrint((double)v.y * sh);
  const size_t base = (size_t)s * f * RG_SLOTS;
  for (uint32_t j = 0; j < f; ++j) {
    const size_t at = base + (size_t)j * RG_SLOTS + bins[(size_t)j * np + r];
    atomicAdd(&HG[at], qg);
    atomicAdd(&HH[at], qh);
    atomicAdd(&HC[at], 1u);
  }
}

struct Cand {
  double gain;
  int32_t feature, bin;
  double GL, HL;
  uint32_t CL;
};

// a better than b: higher gain, then the lower (feature, bin) -- the
// reference's strict ">" over features and bins in increasing order
__device__ __forceinline__ bool better(const Cand& a, const Cand& b) {
  if (a.gain != b.gain) return a.gain > b.gain;
  if (a.feature != b.feature) return a.feature < b.feature;
  return a.bin < b.bin;
}

__device__ __forceinline__ Cand shfl_cand(const Cand& c, int o) {
  Cand r;
  r.gain = __shfl_xor_sync(0xffffffffu, c.gain, o);
  r.feature = __shfl_xor_sync(0xffffffffu, c.feature, o);
  r.bin = __shfl_xor_sync(0xffffffffu, c.bin, o);
  r.GL = __shfl_xor_sync(0xffffffffu, c.GL, o);
  r.HL = __shfl_xor_sync(0xffffffffu, c.HL, o);
  r.CL = __shfl_xor_sync(0xffffffffu, c.CL, o);
  return r;
}

struct ScanCfg {
  uint32_t f;
  int nb;  // candidates b = 0 .. nb-2 (the reference scans max_bins - 1 thresholds)
  double inv_g, inv_h;
  double lam, mcw, msg;
  uint32_t msl;
};

// One block per open node; a warp per feature, lane l holding bins 8l .. 8l+7.
__global__ void __launch_bounds__(RG_SCAN_WARPS * 32) k_rg_scan(ScanCfg sc, const unsigned long long* __restrict__ HG,
                                                                const unsigned long long* __restrict__ HH,
                                                                const uint32_t* __restrict__ HC,
                                                                RgBest* __restrict__ out) {
  __shared__ Cand s_best[RG_SCAN_WARPS];
  __shared__ long long s_tot[3];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t node_base = (size_t)blockIdx.x * sc.f * RG_SLOTS;
  // node totals from feature 0 (every row sits in one slot of every feature)
  if (warp == 0) {
    long long tg = 0, th = 0, tc = 0;
    for (int q = 0; q < 8; ++q) {
      const size_t at = node_base + lane * 8 + q;
      tg += (long long)HG[at];
      th += (long long)HH[at];
      tc += HC[at];
    }
    for (int o = 16; o; o >>= 1) {
      tg += __shfl_xor_sync(0xffffffffu, tg, o);
      th += __shfl_xor_sync(0xffffffffu, th, o);
      tc += __shfl_xor_sync(0xffffffffu, tc, o);
    }
    if (lane == 0) {
      s_tot[0] = tg;
      s_tot[1] = th;
      s_tot[2] = tc;
    }
  }
  __syncthreads();
  const long long TG = s_tot[0], TH = s_tot[1];
  const uint32_t TC = (uint32_t)s_tot[2];
  const double G = (double)TG * sc.inv_g, H = (double)TH * sc.inv_h;
  const double pg = G * G / (H + sc.lam);
  Cand best{-INFINITY, 0x7fffffff, 0x7fffffff, 0.0, 0.0, 0u};
  for (uint32_t j = warp; j < sc.f; j += RG_SCAN_WARPS) {
    const size_t fb = node_base + (size_t)j * RG_SLOTS + lane * 8;
    long long vg[8], vh[8];
    uint32_t vc[8];
    long long lg = 0, lh = 0;
    uint32_t lc = 0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      vg[q] = (long long)HG[fb + q];
      vh[q] = (long long)HH[fb + q];
      vc[q] = HC[fb + q];
      lg += vg[q];
      lh += vh[q];
      lc += vc[q];
    }
    // exclusive prefix of the lanes' totals
    long long xg = lg, xh = lh;
    uint32_t xc = lc;
    for (int o = 1; o < 32; o <<= 1) {
      const long long a = __shfl_up_sync(0xffffffffu, xg, o);
      const long long b = __shfl_up_sync(0xffffffffu, xh, o);
      const uint32_t c = __shfl_up_sync(0xffffffffu, xc, o);
      if (lane >= o) {
        xg += a;
        xh += b;
        xc += c;
      }
    }
    long long pgi = xg - lg, phi = xh - lh;
    uint32_t pci = xc - lc;
    Cand lb{-INFINITY, 0x7fffffff, 0x7fffffff, 0.0, 0.0, 0u};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      pgi += vg[q];
      phi += vh[q];
      pci += vc[q];
      const int b = lane * 8 + q;
      if (b > sc.nb - 2) continue;
      const uint32_t cl = pci, cr = TC - pci;
      const double GL = (double)pgi * sc.inv_g, HL = (double)phi * sc.inv_h;
      const double GR = (double)(TG - pgi) * sc.inv_g, HR = (double)(TH - phi) * sc.inv_h;
      if (cl < sc.msl || cr < sc.msl || HL < sc.mcw || HR < sc.mcw) continue;
      const double gain = 0.5 * ((GL * GL / (HL + sc.lam) + GR * GR / (HR + sc.lam)) - pg);
      if (!(gain >= sc.msg)) continue;
      if (gain > lb.gain) lb = Cand{gain, (int32_t)j, b, GL, HL, cl};
    }
    for (int o = 16; o; o >>= 1) {
      const Cand other = shfl_cand(lb, o);
      if (better(other, lb)) lb = other;
    }
    if (better(lb, best)) best = lb;
  }
  if (lane == 0) s_best[warp] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    Cand b = s_best[0];
    for (int w = 1; w < RG_SCAN_WARPS; ++w)
      if (better(s_best[w], b)) b = s_best[w];
    RgBest r{};
    r.G = G;
    r.H = H;
    r.C = TC;
    r.feature = b.gain > -INFINITY ? b.feature : -1;
    r.bin = b.bin;
    r.gain = b.gain;
    r.GL = b.GL;
    r.HL = b.HL;
    r.CL = b.CL;
    out[blockIdx.x] = r;
  }
}

// Rows of the open nodes move to their child's slot at the next level (-1:
// the child is a leaf); NaN (bin 255) goes left, as the reference partitions.
__global__ void k_rg_partition(const uint8_t* __restrict__ bins, uint32_t np, uint32_t n, int32_t* __restrict__ slot,
                               const int32_t* __restrict__ feat, const int32_t* __restrict__ thr,
                               const int32_t* __restrict__ lslot, const int32_t* __restrict__ rslot) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  const int32_t s = slot[r];
  if (s < 0) return;
  if (feat[s] < 0) {
    slot[r] = -1;
    return;
  }
  const uint32_t b = bins[(size_t)feat[s] * np + r];
  slot[r] = (b != 255u && (int32_t)b > thr[s]) ? rslot[s] : lslot[s];
}

// The finished tree on every row (Tree::predict on the binned dataset,
// src/tree/tree.cpp:929-950: NaN follows default_left, else right iff
// bin > split bin), then predictions += lr * leaf (fused multiply-add).
// node = (feature | bin << 16 | is_leaf << 24 | default_left << 25, left, right, value bits)
__global__ void k_rg_apply(const uint8_t* __restrict__ bins, uint32_t np, uint32_t n, const uint4* __restrict__ nodes,
                           int n_nodes, float lr, float* __restrict__ pred) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= n) return;
  int i = 0;
  for (int step = 0; step < n_nodes; ++step) {  // a walk visits each node at most once
    const uint4 nd = nodes[i];
    if ((nd.x >> 24) & 1u) break;
    const uint32_t b = bins[(size_t)(nd.x & 0xffffu) * np + r];
    const bool right = b == 255u ? !((nd.x >> 25) & 1u) : b > ((nd.x >> 16) & 0xffu);
    i = (int)(right ? nd.z : nd.y);
  }
  pred[r] = __fmaf_rn(lr, __uint_as_float(nodes[i].w), pred[r]);
}

__global__ void k_rg_fill(float* p, uint32_t n, float v) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = v;
}

// Host side of one grown node.
struct GNode {
  int depth = 0;
  double G = 0, H = 0;
  uint32_t C = 0;
  bool split = false;
  int feature = 0, bin = 0;
  double gain = 0, GL = 0, HL = 0;
  uint32_t CL = 0;
  int left = -1, right = -1;  // grown-node ids
};

struct FNode {  // a node of the finished tree, in the reference's numbering
  uint16_t feature = 0;
  uint8_t bin = 0;
  uint8_t flags = 3;  // is_leaf | default_left << 1 (TreeNode's defaults)
  uint16_t left = 0, right = 0;
  float value = 0.0f, gain = 0.0f;
};

template <class T>
void put(std::vector<uint8_t>& b, const T& v) {
  const uint8_t* p = reinterpret_cast<const uint8_t*>(&v);
  b.insert(b.end(), p, p + sizeof(T));
}

}  // namespace

tc_status train_regular(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_model** out,
                        tc_train_stats* stats) {
  const uint32_t n = ds->n, f = ds->f;
  if (!ds->quantized) return ctx->fail(TC_ERR_NOT_FITTED, "dataset not quantized");
  if (n == 0 || ds->y.n < n) return ctx->fail(TC_ERR_INVALID_ARG, "regular trees need rows and labels");
  if (p->loss != TC_LOSS_LOGLOSS)
    return ctx->fail(TC_ERR_INVALID_ARG, "regular trees on the device: binary logloss only (the reference's "
                                         "regression preset grows leaf-wise trees)");
  if (p->subsample < 1.0f || p->use_goss)
    return ctx->fail(TC_ERR_INVALID_ARG, "regular trees on the device: every row in every tree (no subsample/GOSS)");
  if (p->max_depth < 1 || p->max_depth > kMaxDepth)
    return ctx->fail(TC_ERR_INVALID_ARG, "max_depth must be in [1, %d]", kMaxDepth);
  if (p->max_bins < 2 || p->max_bins > 255) return ctx->fail(TC_ERR_INVALID_ARG, "max_bins must be in [2, 255]");
  if (p->n_estimators < 0) return ctx->fail(TC_ERR_INVALID_ARG, "n_estimators must be >= 0");
  cudaStream_t st = ctx->stream;
  const auto t0 = std::chrono::steady_clock::now();
  // base prediction (Loss::init_prediction, src/boosting/loss.cpp:217-226)
  float base;
  {
    std::vector<float> y(n);
    TC_CUDA(ctx, cudaMemcpyAsync(y.data(), ds->y.p, n * sizeof(float), cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaStreamSynchronize(st));
    float sum = 0.0f;
    for (uint32_t i = 0; i < n; ++i) sum += y[i];
    float q = sum / (float)n;
    q = std::max(1e-7f, std::min(1.0f - 1e-7f, q));
    base = std::log(q / (1.0f - q));
  }
  const int D = p->max_depth, nb = p->max_bins;
  const int max_open = 1 << (D - 1);  // open nodes at the deepest scanned level
  DevBuf<float> pred;
  DevBuf<float2> gh;
  DevBuf<int32_t> slot, lvl;  // lvl: feat, thr, lslot, rslot per open node
  DevBuf<uint32_t> amax, HC;
  DevBuf<unsigned long long> HG, HH;
  DevBuf<RgBest> best;
  DevBuf<uint4> dnodes;
  TC_TRY(pred.alloc(ctx, n, "regular-tree predictions"));
  TC_TRY(gh.alloc(ctx, n, "regular-tree gradients"));
  TC_TRY(slot.alloc(ctx, n, "row node slots"));
  TC_TRY(lvl.alloc(ctx, (size_t)4 * max_open, "level splits"));
  TC_TRY(amax.alloc(ctx, 2, "gradient maxima"));
  TC_TRY(best.alloc(ctx, max_open, "best splits"));
  TC_TRY(dnodes.alloc(ctx, 65535, "finished tree"));
  const uint32_t rb = (n + RG_THREADS - 1) / RG_THREADS;
  k_rg_fill<<<rb, RG_THREADS, 0, st>>>(pred.p, n, base);
  const float lr = p->learning_rate;
  const double lam = p->lambda_l2;
  std::vector<std::vector<FNode>> trees;
  std::vector<uint16_t> tree_depth;
  int64_t launches = 1;
  for (int it = 0; it < p->n_estimators; ++it) {
    TC_CUDA(ctx, cudaMemsetAsync(amax.p, 0, amax.bytes(), st));
    k_rg_grad<<<rb, RG_THREADS, 0, st>>>(ds->y.p, pred.p, gh.p, n, TC_LOSS_LOGLOSS, amax.p);
    uint32_t hm[2];
    TC_CUDA(ctx, cudaMemcpyAsync(hm, amax.p, sizeof(hm), cudaMemcpyDeviceToHost, st));
    TC_CUDA(ctx, cudaStreamSynchronize(st));
    ++launches;
    // fixed-point scales: n * max|x| * 2^e < 2^62, so no sum can overflow
    double mx[2];
    for (int k = 0; k < 2; ++k) {
      float v;
      std::memcpy(&v, &hm[k], 4);
      mx[k] = std::max((double)v, 1e-30);
    }
    const double sg = std::ldexp(1.0, (int)std::floor(62.0 - std::log2((double)n * mx[0])) - 1);
    const double sh = std::ldexp(1.0, (int)std::floor(62.0 - std::log2((double)n * mx[1])) - 1);
    const uint32_t msl = (uint32_t)std::max(0, p->min_samples_leaf);
    ScanCfg sc{f, nb, 1.0 / sg, 1.0 / sh, lam, (double)p->min_child_weight, (double)p->min_split_gain, msl};
    // grow level by level
    std::vector<GNode> g(1);
    std::vector<int> open{0};
    TC_CUDA(ctx, cudaMemsetAsync(slot.p, 0, slot.bytes(), st));
    for (int d = 0; !open.empty(); ++d) {
      const int A = (int)open.size();
      const size_t hs = (size_t)A * f * RG_SLOTS;
      if (HG.n < hs) {  // histograms of the level's open nodes (grow-only)
        TC_TRY(HG.alloc(ctx, hs, "regular-tree gradient histograms"));
        TC_TRY(HH.alloc(ctx, hs, "regular-tree hessian histograms"));
        TC_TRY(HC.alloc(ctx, hs, "regular-tree count histograms"));
      }
      TC_CUDA(ctx, cudaMemsetAsync(HG.p, 0, hs * sizeof(unsigned long long), st));
      TC_CUDA(ctx, cudaMemsetAsync(HH.p, 0, hs * sizeof(unsigned long long), st));
      TC_CUDA(ctx, cudaMemsetAsync(HC.p, 0, hs * sizeof(uint32_t), st));
      k_rg_hist<<<rb, RG_THREADS, 0, st>>>(ds->bins_cm.p, ds->np, n, f, slot.p, gh.p, sg, sh, HG.p, HH.p, HC.p);
      k_rg_scan<<<A, RG_SCAN_WARPS * 32, 0, st>>>(sc, HG.p, HH.p, HC.p, best.p);
      std::vector<RgBest> hb(A);
      TC_CUDA(ctx, cudaMemcpyAsync(hb.data(), best.p, A * sizeof(RgBest), cudaMemcpyDeviceToHost, st));
      TC_CUDA(ctx, cudaStreamSynchronize(st));
      launches += 2;
      std::vector<int32_t> lv((size_t)4 * A, -1);  // feat | thr | lslot | rslot
      std::vector<int> next;
      for (int a = 0; a < A; ++a) {
        const int gi = open[a];
        const RgBest& bb = hb[a];
        if (d == 0) {  // the root's totals and stop rules; children take their parent's split sums
          g[gi].G = bb.G;
          g[gi].H = bb.H;
          g[gi].C = bb.C;
          if (g[gi].C < 2u * msl || g[gi].H < 2.0 * (double)p->min_child_weight) continue;
        }
        if (bb.feature < 0 || bb.gain < p->min_split_gain) continue;
        g[gi].split = true;
        g[gi].feature = bb.feature;
        g[gi].bin = bb.bin;
        g[gi].gain = bb.gain;
        g[gi].GL = bb.GL;
        g[gi].HL = bb.HL;
        g[gi].CL = bb.CL;
        lv[a] = bb.feature;
        lv[A + a] = bb.bin;
        const GNode par = g[gi];
        for (int side = 0; side < 2; ++side) {
          GNode c;
          c.depth = d + 1;
          c.G = side ? par.G - par.GL : par.GL;
          c.H = side ? par.H - par.HL : par.HL;
          c.C = side ? par.C - par.CL : par.CL;
          const int id = (int)g.size();
          if (side) g[gi].right = id; else g[gi].left = id;
          // the reference's stop rules other than the leaf cap: such a child is
          // a leaf whatever happens, so it is not scanned
          const bool stop = c.depth >= D || c.C < 2u * msl || c.H < 2.0 * (double)p->min_child_weight;
          int32_t s = -1;
          if (!stop) {
            s = (int32_t)next.size();
            next.push_back(id);
          }
          lv[(side ? 3 : 2) * A + a] = s;
          g.push_back(c);
        }
      }
      TC_CUDA(ctx, cudaMemcpyAsync(lvl.p, lv.data(), lv.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st));
      k_rg_partition<<<rb, RG_THREADS, 0, st>>>(ds->bins_cm.p, ds->np, n, slot.p, lvl.p, lvl.p + A, lvl.p + 2 * A,
                                                lvl.p + 3 * A);
      TC_CUDA(ctx, cudaStreamSynchronize(st));  // lv is read by the copy
      ++launches;
      open.swap(next);
    }
    // replay of the reference's recursion: numbering and the leaf cap
    std::vector<FNode> fn(1);
    int n_leaves = 0, depth_max = 0;
    std::vector<int> stack_g{0}, stack_f{0};
    // explicit DFS: a split node pushes its children so that the smaller one is visited first
    while (!stack_g.empty()) {
      const int gi = stack_g.back(), fi = stack_f.back();
      stack_g.pop_back();
      stack_f.pop_back();
      const GNode& nd = g[gi];
      depth_max = std::max(depth_max, nd.depth);
      if (!nd.split || n_leaves >= RG_MAX_LEAVES) {
        float v = (float)(-nd.G / (nd.H + lam));
        if (p->max_delta_step > 0.0f) v = std::max(-p->max_delta_step, std::min(p->max_delta_step, v));
        fn[fi].flags = 3;
        fn[fi].value = v;
        ++n_leaves;
        continue;
      }
      const uint16_t li = (uint16_t)fn.size(), ri = (uint16_t)(fn.size() + 1);
      fn.resize(fn.size() + 2);
      FNode& x = fn[fi];
      x.feature = (uint16_t)nd.feature;
      x.bin = (uint8_t)nd.bin;
      const uint32_t cl = g[nd.left].C, cr = g[nd.right].C;
      x.flags = (cl >= cr ? 2 : 0);  // learn_missing_direction (src/tree/tree.cpp:356-359)
      x.left = li;
      x.right = ri;
      x.gain = (float)nd.gain;
      if (cl <= cr) {  // smaller (left) first: pushed last
        stack_g.push_back(nd.right);
        stack_f.push_back(ri);
        stack_g.push_back(nd.left);
        stack_f.push_back(li);
      } else {
        stack_g.push_back(nd.left);
        stack_f.push_back(li);
        stack_g.push_back(nd.right);
        stack_f.push_back(ri);
      }
    }
    if (fn.size() > 65535) return ctx->fail(TC_ERR_INVALID_ARG, "tree %d has too many nodes", it);
    std::vector<uint4> dn(fn.size());
    for (size_t i = 0; i < fn.size(); ++i) {
      const FNode& x = fn[i];
      uint32_t vb;
      std::memcpy(&vb, &x.value, 4);
      dn[i] = make_uint4((uint32_t)x.feature | (uint32_t)x.bin << 16 | (uint32_t)(x.flags & 1) << 24 |
                             (uint32_t)((x.flags >> 1) & 1) << 25,
                         x.left, x.right, vb);
    }
    TC_CUDA(ctx, cudaMemcpyAsync(dnodes.p, dn.data(), dn.size() * sizeof(uint4), cudaMemcpyHostToDevice, st));
    k_rg_apply<<<rb, RG_THREADS, 0, st>>>(ds->bins_cm.p, ds->np, n, dnodes.p, (int)dn.size(), lr, pred.p);
    TC_CUDA(ctx, cudaStreamSynchronize(st));
    ++launches;
    trees.push_back(std::move(fn));
    tree_depth.push_back((uint16_t)depth_max);
  }
  TC_CUDA(ctx, cudaGetLastError());
  // the model: TCAT v3 with regular trees (Booster::save_binary,
  // src/boosting/booster.cpp:1049-1110; Tree::save, src/tree/tree.cpp:1748-1793)
  std::vector<uint8_t> b;
  b.insert(b.end(), {'T', 'C', 'A', 'T'});
  put(b, (uint32_t)3);
  put(b, base);
  put(b, (uint8_t)TC_TASK_BINARY);
  put(b, (uint32_t)2);
  put(b, lr);
  put(b, (uint16_t)D);
  put(b, (float)lam);
  put(b, (uint8_t)0);  // regular trees
  put(b, (uint64_t)f);
  for (uint32_t j = 0; j < f; ++j) {
    const uint16_t k = ds->h_n_edges[j];
    put(b, (uint64_t)k);
    for (uint16_t e = 0; e < k; ++e) put(b, ds->h_edges[(size_t)j * 255 + e]);
  }
  put(b, (uint64_t)trees.size());
  for (size_t t = 0; t < trees.size(); ++t) put(b, lr);
  for (size_t t = 0; t < trees.size(); ++t) {
    const auto& fn = trees[t];
    uint16_t leaves = 0;
    for (const FNode& x : fn) leaves += (x.flags & 1) ? 1 : 0;
    put(b, tree_depth[t]);
    put(b, (uint32_t)1);
    put(b, (uint32_t)fn.size());
    put(b, leaves);
    put(b, (uint16_t)D);
    put(b, (float)lam);
    for (const FNode& x : fn) {
      put(b, x.feature);
      put(b, x.bin);
      put(b, x.flags);
      put(b, x.left);
      put(b, x.right);
      put(b, x.value);
      put(b, x.gain);
    }
  }
  TC_TRY(tc_model_load_tcat(ctx, b.data(), b.size(), out));
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->n_trees = (int32_t)trees.size();
    stats->iterations_done = (int32_t)trees.size();
    stats->base_prediction = base;
    stats->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    stats->kernel_launches = launches;
    stats->best_iteration = (int32_t)trees.size() - 1;
  }
  return TC_OK;
}

}  // namespace tc

extern "C" tc_status tc_train_regular(tc_ctx* ctx, tc_dataset* ds, const tc_train_params* p, tc_model** out,
                                      tc_train_stats* stats) {
  if (!ctx || !ds || !p || !out) return TC_ERR_INVALID_ARG;
  if (ds->ctx != ctx) return ctx->fail(TC_ERR_INVALID_ARG, "the dataset belongs to another context");
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  *out = nullptr;
  return tc::train_regular(ctx, ds, p, out, stats);
}
