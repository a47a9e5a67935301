// Oblivious-ensemble prediction on raw float features, the model object and
// the TCAT v3 stream.
//
// Prediction restates FastFloatEnsemble (include/turbocat/fast_float_ensemble.hpp:122-137,
// 139-664; src/tree/fast_float_ensemble.cpp:23-276): per tree the leaf index is
// built from depth bit-compares, bit = !isnan(x) && x >= threshold, first
// split in the most significant bit, and the weighted leaf values are summed;
// then the base prediction is added (src/boosting/booster.cpp:920-924) and the
// sigmoid (include/turbocat/loss.hpp:99-101) or softmax
// (src/boosting/loss.cpp:320-330) applied.
//
// Kernel layout: a block owns a tile of rows of one job (one request of a
// coalesced serving batch, or the whole input of a single call).  The
// tile's rows are staged in shared memory (row stride f+1 words, so threads
// reading the same feature of different rows hit different banks), trees are
// streamed through shared memory in chunks of packed (feature, threshold)
// pairs and weight-folded leaves, two chunks in flight (cp.async: the next
// chunk lands while the current one is walked), and every thread walks all
// trees for its row.
#include <algorithm>
#include <chrono>
#include <cstring>

#include "tc_internal.h"

namespace tc {
namespace {

constexpr int PRED_ROWS = 128;
constexpr int PRED_THREADS = 512;                 // a row tile: up to 128 rows x 4 tree groups
constexpr int PRED_LEAF_FLOATS = 8192;      // shared floats for two chunks of leaves (2 x 16 KB)
constexpr int PRED_LEAF_STAGE = PRED_LEAF_FLOATS / 2;
constexpr int PRED_CHUNK = 128;             // trees per chunk at most (two chunks in flight)
constexpr int PRED_MAX_K = 16;

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void cp_async4(void* s, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async8(void* s, const void* g) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async16(void* s, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_addr(s)), "l"(g) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

struct JobTable {
  const ReqDesc* reqs;         // nullptr: single job held inline
  const ModelDesc* models;
  const uint32_t* tile_begin;  // [n_jobs + 1] first tile of each job
  int n_jobs;
  int max_depth;               // largest model depth in the batch (shared sizing)
  int max_f;                   // largest feature count in the batch
  ReqDesc one_req;
  ModelDesc one_model;
};

__device__ __forceinline__ float sigmoidf_ref(float x) { return 1.0f / (1.0f + expf(-x)); }

// NT full-depth trees of depth DD walked together: every split is loaded
// first, then every feature value, then the compares, so the shared-memory
// loads of the NT trees are in flight together instead of one dependent
// chain per level.
template <int NT, int DD>
__device__ __forceinline__ void walk_full(const uint2* __restrict__ s_split, const float* __restrict__ xr,
                                          const float* __restrict__ lv, int t, int TG, float4& sum) {
  constexpr int L = 1 << DD;
  uint2 q[NT][DD];
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    if constexpr (DD % 2 == 0) {
      // a tree's splits start on a 16-byte boundary: two per 128-bit load
      const uint4* sp = reinterpret_cast<const uint4*>(s_split + (t + u * TG) * DD);
#pragma unroll
      for (int d = 0; d < DD / 2; ++d) {
        const uint4 v = sp[d];
        q[u][2 * d] = make_uint2(v.x, v.y);
        q[u][2 * d + 1] = make_uint2(v.z, v.w);
      }
    } else {
#pragma unroll
      for (int d = 0; d < DD; ++d) q[u][d] = s_split[(t + u * TG) * DD + d];
    }
  }
  float xv[NT][DD];
#pragma unroll
  for (int u = 0; u < NT; ++u)
#pragma unroll
    for (int d = 0; d < DD; ++d) xv[u][d] = xr[q[u][d].x];
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    uint32_t idx = 0;
#pragma unroll
    for (int d = 0; d < DD; ++d)
      if (xv[u][d] >= __uint_as_float(q[u][d].y)) idx |= 1u << (DD - 1 - d);  // false for NaN
    const float v = lv[(t + u * TG) * L + idx];
    if (u == 0) sum.x += v;
    else if (u == 1) sum.y += v;
    else if (u == 2) sum.z += v;
    else sum.w += v;
  }
}

__global__ void __launch_bounds__(PRED_THREADS) k_predict(JobTable jt) {
  extern __shared__ float smp[];
  ReqDesc rq;
  ModelDesc md;
  uint32_t tile;
  if (jt.reqs == nullptr) {
    rq = jt.one_req;
    md = jt.one_model;
    tile = blockIdx.x;
  } else {
    // job lookup: last job whose first tile <= blockIdx.x
    int lo = 0, hi = jt.n_jobs - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (jt.tile_begin[mid] <= blockIdx.x) lo = mid; else hi = mid - 1;
    }
    rq = jt.reqs[lo];
    md = jt.models[rq.model];
    tile = blockIdx.x - jt.tile_begin[lo];
  }
  const uint32_t r0 = tile * PRED_ROWS;
  if (r0 >= rq.n) return;
  const uint32_t nr = min((uint32_t)PRED_ROWS, rq.n - r0);
  // row slots of this tile (a power of two >= nr); the block's other threads
  // split the trees, so a small request still uses every thread
  int RT = PRED_ROWS;
  while (RT > 1 && (uint32_t)(RT >> 1) >= nr) RT >>= 1;
  const int TG = PRED_THREADS / RT;
  const int f = md.n_features;
  const int fs = f + 1;
  const int D = md.max_depth;
  const int L = 1 << D;
  // leaves of shallow trees are staged in shared memory with the splits;
  // deeper trees (64 leaves or more) gather their leaf from global memory
  // (L2), so a chunk still holds PRED_CHUNK trees' splits (measured on 1M
  // rows: depth 6 is 6% faster from L2, depth 4 2% slower)
  const bool leaves_global = L >= 64;
  const int tchunk = leaves_global ? PRED_CHUNK : max(1, min(PRED_CHUNK, PRED_LEAF_STAGE / L));
  const int Dmax = max(1, jt.max_depth);
  float* s_x = smp;                                  // [PRED_ROWS][f+1]
  float* s_leaf = s_x + PRED_ROWS * (jt.max_f + 1);  // 2 x [tchunk][L]
  uint2* s_split = reinterpret_cast<uint2*>(s_leaf + PRED_LEAF_FLOATS);  // 2 x [tchunk][D]
  int* s_depth = reinterpret_cast<int*>(s_split + 2 * PRED_CHUNK * Dmax);  // 2 x [tchunk]
  // Every copy into shared memory is asynchronous (cp.async): the row tile
  // and the first tree chunk, then chunk c + 1 while chunk c is walked.
  const float* Xt = rq.X + (size_t)r0 * f;
  // a warp copies whole rows (lane = feature), no division by f
  for (uint32_t i = threadIdx.x >> 5; i < nr; i += blockDim.x >> 5)
    for (int j = threadIdx.x & 31; j < f; j += 32) cp_async4(&s_x[i * fs + j], &Xt[(size_t)i * f + j]);
  auto issue_chunk = [&](int t0, int buf) {
    const int tn = min(tchunk, md.n_trees - t0);
    if (!leaves_global) {
      float* dl = s_leaf + buf * PRED_LEAF_STAGE;
      const float* gl = md.leaves + (size_t)t0 * L;
      const int cnt = tn * L;
      if ((((size_t)t0 * L) & 3) == 0 && (cnt & 3) == 0) {
        for (int q = threadIdx.x; q < cnt / 4; q += blockDim.x) cp_async16(dl + 4 * q, gl + 4 * q);
      } else {
        for (int q = threadIdx.x; q < cnt; q += blockDim.x) cp_async4(dl + q, gl + q);
      }
    }
    uint2* ds = s_split + buf * PRED_CHUNK * Dmax;
    for (int q = threadIdx.x; q < tn * D; q += blockDim.x) cp_async8(ds + q, md.splits + (size_t)t0 * D + q);
    int* dd = s_depth + buf * PRED_CHUNK;
    for (int q = threadIdx.x; q < tn; q += blockDim.x) cp_async4(dd + q, md.depth + t0 + q);
  };
  if (md.n_trees > 0) issue_chunk(0, 0);
  cp_async_commit();
  const int K = md.n_classes;
  float acc[PRED_MAX_K];
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k) acc[k] = 0.0f;
  const int row = threadIdx.x % RT;
  const int tg = threadIdx.x / RT;
  const float* xr = s_x + row * fs;
  for (int t0 = 0, buf = 0; t0 < md.n_trees; t0 += tchunk, buf ^= 1) {
    const int tn = min(tchunk, md.n_trees - t0);
    if (t0 + tchunk < md.n_trees) issue_chunk(t0 + tchunk, buf ^ 1);
    cp_async_commit();
    cp_async_wait_prev();  // this thread's copies of the row tile and of chunk t0 have landed
    const float* lv = leaves_global ? md.leaves + (size_t)t0 * L : s_leaf + buf * PRED_LEAF_STAGE;
    const uint2* s_split_c = s_split + buf * PRED_CHUNK * Dmax;
    const int* s_depth_c = s_depth + buf * PRED_CHUNK;
    bool full_here = true;
    for (int q = threadIdx.x; q < tn; q += blockDim.x) full_here = full_here && s_depth_c[q] == D;
    // the barrier also publishes every thread's copies; every tree of the chunk has depth D?
    const bool all_full = __syncthreads_and(full_here) != 0;
    if ((uint32_t)row < nr) {
      if (K == 1) {
        // full-depth trees in groups (depth <= 8: 4 at a time, 9-10: 2),
        // partial sums combined in a fixed order; other trees one by one
        float4 s4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        int t = tg;
        const int NT = D <= 8 ? 4 : 2;
        if (D <= 10) {
          for (; t + (NT - 1) * TG < tn; t += NT * TG) {
            if (!all_full) {
              bool full = true;
              for (int u = 0; u < NT; ++u) full = full && s_depth_c[t + u * TG] == D;
              if (!full) break;
            }
            switch (D) {
              case 1: walk_full<4, 1>(s_split_c, xr, lv, t, TG, s4); break;
              case 2: walk_full<4, 2>(s_split_c, xr, lv, t, TG, s4); break;
              case 3: walk_full<4, 3>(s_split_c, xr, lv, t, TG, s4); break;
              case 4: walk_full<4, 4>(s_split_c, xr, lv, t, TG, s4); break;
              case 5: walk_full<4, 5>(s_split_c, xr, lv, t, TG, s4); break;
              case 6: walk_full<4, 6>(s_split_c, xr, lv, t, TG, s4); break;
              case 7: walk_full<4, 7>(s_split_c, xr, lv, t, TG, s4); break;
              case 8: walk_full<4, 8>(s_split_c, xr, lv, t, TG, s4); break;
              case 9: walk_full<2, 9>(s_split_c, xr, lv, t, TG, s4); break;
              default: walk_full<2, 10>(s_split_c, xr, lv, t, TG, s4); break;
            }
          }
        }
        for (; t < tn; t += TG) {
          const int dep = s_depth_c[t];
          const uint2* sp = s_split_c + t * D;
          uint32_t idx = 0;
          for (int d = 0; d < dep; ++d) {
            const uint2 q = sp[d];
            idx = (idx << 1) | (uint32_t)(xr[q.x] >= __uint_as_float(q.y));  // false for NaN
          }
          s4.x += lv[t * L + idx];
        }
        acc[0] += (s4.x + s4.y) + (s4.z + s4.w);
      } else {
        for (int t = tg; t < tn; t += TG) {
          const int dep = s_depth_c[t];
          const uint2* sp = s_split_c + t * D;
          uint32_t idx = 0;
          for (int d = 0; d < dep; ++d) {
            const uint2 q = sp[d];
            idx = (idx << 1) | (uint32_t)(xr[q.x] >= __uint_as_float(q.y));
          }
          const int cls = (t0 + t) % K;
          const float v = lv[t * L + idx];
#pragma unroll
          for (int k = 0; k < PRED_MAX_K; ++k)
            if (k == cls) acc[k] += v;
        }
      }
    }
    __syncthreads();  // chunk t0's buffers are refilled by the next iteration's copies
  }
  cp_async_wait_all();
  // combine the thread groups' partial sums (pairwise, fixed order)
  __syncthreads();
  float* s_red = s_leaf;  // [TG][RT][K]: TG*RT = PRED_THREADS, 512*16 floats = PRED_LEAF_FLOATS
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k)
    if (k < K) s_red[(tg * RT + row) * K + k] = acc[k];
  __syncthreads();
  for (int h = TG >> 1; h > 0; h >>= 1) {
    if (tg < h) {
      for (int k = 0; k < K; ++k) s_red[(tg * RT + row) * K + k] += s_red[((tg + h) * RT + row) * K + k];
    }
    __syncthreads();
  }
  if (tg != 0 || (uint32_t)row >= nr) return;
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k)
    if (k < K) acc[k] = s_red[row * K + k];
  float* o = rq.out + (size_t)(r0 + row) * K;
  if (rq.transform == TC_TRANSFORM_SOFTMAX && K > 1) {
    float mx = -INFINITY;
    for (int k = 0; k < K; ++k) mx = fmaxf(mx, acc[k] + md.base);
    float sum = 0.0f;
    float e[PRED_MAX_K];
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k) {
      if (k < K) {
        e[k] = expf(acc[k] + md.base - mx);
        sum += e[k];
      }
    }
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k)
      if (k < K) o[k] = e[k] / sum;
  } else {
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k) {
      if (k < K) {
        const float raw = acc[k] + md.base;
        o[k] = (rq.transform == TC_TRANSFORM_SIGMOID) ? sigmoidf_ref(raw) : raw;
      }
    }
  }
}

// Small requests (at most SMALL_ROWS rows): the trees are split over the
// blocks of one launch instead of streamed through one block, as few blocks
// as the (row, tree) walks need (one block for a single row).  Block b walks
// trees [b*T/NB, (b+1)*T/NB) for every row of the request (row slot =
// thread % RT, tree lane = thread / RT, trees in order within a lane) and
// sums its lanes pairwise in a fixed order; with several blocks each stores
// one partial per (row, class) and the last block to finish (completion
// counter; nobody waits) adds them in block order.  The block that finishes
// adds the base, applies the transform and writes the outputs (which may be
// pinned host memory mapped into the device).  The rows come from device
// memory or, for the smallest requests, from the launch parameters.
constexpr int SMALL_ROWS = 64;
constexpr int SMALL_INLINE = 928;  // floats of a request carried in the launch parameters (4 KB in all)
struct SmallRows {
  float v[SMALL_INLINE];
};
constexpr int SMALL_THREADS = 512;
constexpr int SMALL_WALKS_PER_BLOCK = 4096;  // (row, tree) walks per block: one block for a single row
constexpr int SMALL_MAX_F = 512;   // features of a small request (its rows fit in shared memory)

__global__ void __launch_bounds__(SMALL_THREADS) k_predict_small(ModelDesc md, const float* __restrict__ X, uint32_t n,
                                                                  int transform, float* __restrict__ partial,
                                                                  uint32_t* __restrict__ counter,
                                                                  float* __restrict__ out, SmallRows inl) {
  extern __shared__ float sm_small[];
  const int f = md.n_features, fs = f + 1;
  const int K = md.n_classes, D = md.max_depth, L = 1 << D;
  float* s_x = sm_small;                         // [n][f+1]
  float* s_red = s_x + n * fs;                   // [SMALL_THREADS][K]
  for (uint32_t i = threadIdx.x >> 5; i < n; i += blockDim.x >> 5)
    for (int j = threadIdx.x & 31; j < f; j += 32) s_x[i * fs + j] = X ? X[(size_t)i * f + j] : inl.v[i * f + j];
  __syncthreads();
  int RT = SMALL_ROWS;
  while (RT > 1 && (uint32_t)(RT >> 1) >= n) RT >>= 1;
  const int TG = blockDim.x / RT;
  const int row = threadIdx.x % RT, tg = threadIdx.x / RT;
  const int T = md.n_trees, NB = gridDim.x;
  const int t0 = (int)((long long)T * blockIdx.x / NB), t1 = (int)((long long)T * (blockIdx.x + 1) / NB);
  float acc[PRED_MAX_K];
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k) acc[k] = 0.0f;
  if ((uint32_t)row < n) {
    const float* xr = s_x + row * fs;
    for (int t = t0 + tg; t < t1; t += TG) {
      // the tree's depth and every split are loaded before any compare (one
      // round trip to L2 instead of one per level); a shallower tree ignores
      // its padding splits
      const uint2* sp = md.splits + (size_t)t * D;
      uint2 q[kMaxDepth];
#pragma unroll
      for (int d = 0; d < kMaxDepth; ++d)
        if (d < D) q[d] = sp[d];
      const int dep = md.depth[t];
      uint32_t idx = 0;
#pragma unroll
      for (int d = 0; d < kMaxDepth; ++d)
        if (d < dep) idx = (idx << 1) | (uint32_t)(xr[q[d].x] >= __uint_as_float(q[d].y));  // false for NaN
      const float v = md.leaves[(size_t)t * L + idx];
      const int cls = K == 1 ? 0 : t % K;
#pragma unroll
      for (int k = 0; k < PRED_MAX_K; ++k)
        if (k == cls) acc[k] += v;
    }
  }
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k)
    if (k < K) s_red[threadIdx.x * K + k] = acc[k];
  __syncthreads();
  for (int h = TG >> 1; h > 0; h >>= 1) {  // lanes pairwise, fixed order
    if (tg < h)
      for (int k = 0; k < K; ++k) s_red[threadIdx.x * K + k] += s_red[(threadIdx.x + h * RT) * K + k];
    __syncthreads();
  }
  if (NB > 1) {
    if (tg == 0 && (uint32_t)row < n)
      for (int k = 0; k < K; ++k) partial[((size_t)blockIdx.x * n + row) * K + k] = s_red[row * K + k];
    __shared__ bool s_last;
    __syncthreads();
    if (threadIdx.x == 0) {
      __threadfence();
      s_last = atomicAdd(counter, 1u) == (uint32_t)NB - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
  }
  for (uint32_t r = threadIdx.x; r < n; r += blockDim.x) {
    float v[PRED_MAX_K];
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k) v[k] = NB > 1 ? 0.0f : (k < K ? s_red[r * K + k] : 0.0f);
    for (int b = 0; NB > 1 && b < NB; ++b)
#pragma unroll
      for (int k = 0; k < PRED_MAX_K; ++k)
        if (k < K) v[k] += __ldcg(&partial[((size_t)b * n + r) * K + k]);
    float* o = out + (size_t)r * K;
    if (transform == TC_TRANSFORM_SOFTMAX && K > 1) {
      float mx = -INFINITY;
      for (int k = 0; k < K; ++k) mx = fmaxf(mx, v[k] + md.base);
      float sum = 0.0f, e[PRED_MAX_K];
#pragma unroll
      for (int k = 0; k < PRED_MAX_K; ++k)
        if (k < K) { e[k] = expf(v[k] + md.base - mx); sum += e[k]; }
#pragma unroll
      for (int k = 0; k < PRED_MAX_K; ++k)
        if (k < K) o[k] = e[k] / sum;
    } else {
#pragma unroll
      for (int k = 0; k < PRED_MAX_K; ++k) {
        if (k < K) {
          const float raw = v[k] + md.base;
          o[k] = transform == TC_TRANSFORM_SIGMOID ? sigmoidf_ref(raw) : raw;
        }
      }
    }
  }
  if (NB > 1 && threadIdx.x == 0) *counter = 0u;  // re-armed for the next call
}

size_t predict_smem(int max_f, int max_depth) {
  return (size_t)PRED_ROWS * (max_f + 1) * 4 + PRED_LEAF_FLOATS * 4 +
         (size_t)2 * PRED_CHUNK * std::max(1, max_depth) * 8 + 2 * PRED_CHUNK * 4;
}

tc_status launch_predict(tc_ctx* ctx, const JobTable& jt, uint32_t n_tiles, cudaStream_t stream) {
  if (n_tiles == 0) return TC_OK;
  const size_t smem = predict_smem(jt.max_f, jt.max_depth);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_done = true;
  }
  if (smem > 200 * 1024)
    return ctx->fail(TC_ERR_INVALID_ARG, "too many features for the predict kernel (%d)", jt.max_f);
  k_predict<<<n_tiles, PRED_THREADS, smem, stream>>>(jt);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ctx->cuda_fail(e, "k_predict");
  return TC_OK;
}

}  // namespace

tc_status predict_batched(tc_ctx* ctx, const ModelDesc* d_models, const ReqDesc* d_reqs, int n_reqs,
                          const uint32_t* d_tile_begin, uint32_t n_tiles, int max_depth_all, int max_f,
                          cudaStream_t stream) {
  JobTable jt{};
  jt.reqs = d_reqs;
  jt.models = d_models;
  jt.tile_begin = d_tile_begin;
  jt.n_jobs = n_reqs;
  jt.max_depth = max_depth_all;
  jt.max_f = max_f;
  return launch_predict(ctx, jt, n_tiles, stream);
}

uint32_t predict_tiles(uint32_t n) { return (n + PRED_ROWS - 1) / PRED_ROWS; }

}  // namespace tc

using namespace tc;

// Packs splits as (feature, threshold bits) and folds the tree weights into
// the leaves (w * leaf in FP32, the product the reference forms per tree).
tc_status tc_model::upload() {
  const int T = info.n_trees, D = info.max_depth, L = 1 << D;
  std::vector<uint2> sp((size_t)std::max(1, T * D));
  std::vector<float> lv((size_t)std::max(1, T * L));
  for (int t = 0; t < T; ++t) {
    for (int d = 0; d < D; ++d) {
      uint32_t bits;
      std::memcpy(&bits, &threshold[(size_t)t * D + d], 4);
      sp[(size_t)t * D + d] = make_uint2(feature[(size_t)t * D + d], bits);
    }
    for (int l = 0; l < L; ++l) lv[(size_t)t * L + l] = weights[t] * leaves[(size_t)t * L + l];
  }
  TC_TRY(d_splits.alloc(ctx, sp.size(), "model splits"));
  TC_TRY(d_leaves.alloc(ctx, lv.size(), "model leaves"));
  TC_TRY(d_depth.alloc(ctx, std::max(1, T), "model depths"));
  TC_CUDA(ctx, cudaMemcpy(d_splits.p, sp.data(), sp.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  TC_CUDA(ctx, cudaMemcpy(d_leaves.p, lv.data(), lv.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (T > 0) TC_CUDA(ctx, cudaMemcpy(d_depth.p, depth.data(), T * sizeof(int32_t), cudaMemcpyHostToDevice));
  return TC_OK;
}

namespace tc {

ModelDesc model_desc(const tc_model* m) {
  ModelDesc d{};
  d.splits = m->d_splits.p;
  d.leaves = m->d_leaves.p;
  d.depth = m->d_depth.p;
  d.n_trees = m->info.n_trees;
  d.max_depth = m->info.max_depth;
  d.n_classes = m->info.n_classes;
  d.n_features = m->info.n_features;
  d.base = m->info.base_prediction;
  return d;
}

tc_status predict_device(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint32_t f, int transform,
                         float* out, cudaStream_t stream) {
  if (n == 0) return TC_OK;
  JobTable jt{};
  jt.reqs = nullptr;
  jt.n_jobs = 1;
  jt.max_depth = m->info.max_depth;
  jt.max_f = (int)f;
  jt.one_model = model_desc(m);
  jt.one_req = ReqDesc{X, out, n, 0, 0, transform};
  return launch_predict(ctx, jt, predict_tiles(n), stream);
}

}  // namespace tc

// ------------------------------------------------------------------ C ABI --

namespace {

void put(std::vector<uint8_t>& b, const void* p, size_t n) {
  const uint8_t* q = static_cast<const uint8_t*>(p);
  b.insert(b.end(), q, q + n);
}

struct Reader {
  const uint8_t* p;
  size_t n, off = 0;
  bool ok = true;
  template <class T>
  T get() {
    T v{};
    if (off + sizeof(T) > n) { ok = false; return v; }
    std::memcpy(&v, p + off, sizeof(T));
    off += sizeof(T);
    return v;
  }
  bool bytes(void* dst, size_t k) {
    if (off + k > n) { ok = false; return false; }
    std::memcpy(dst, p + off, k);
    off += k;
    return true;
  }
};

}  // namespace

extern "C" {

tc_status tc_model_info_get(const tc_model* m, tc_model_info* info) {
  if (!m || !info) return TC_ERR_INVALID_ARG;
  *info = m->info;
  return TC_OK;
}

tc_status tc_model_export(const tc_model* m, int32_t* depth, uint16_t* feature, uint8_t* bin, float* threshold,
                          float* gain, float* leaves, float* weights, float* edges, uint16_t* n_edges) {
  if (!m) return TC_ERR_INVALID_ARG;
  auto cp = [](void* dst, const auto& v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(v[0]));
  };
  cp(depth, m->depth);
  cp(feature, m->feature);
  cp(bin, m->bin);
  cp(threshold, m->threshold);
  cp(gain, m->gain);
  cp(leaves, m->leaves);
  cp(weights, m->weights);
  cp(edges, m->edges);
  cp(n_edges, m->n_edges);
  return TC_OK;
}

tc_status tc_model_import(tc_ctx* ctx, const tc_model_info* info, const int32_t* depth, const uint16_t* feature,
                          const uint8_t* bin, const float* threshold, const float* gain, const float* leaves,
                          const float* weights, const float* edges, const uint16_t* n_edges, tc_model** out) {
  if (!ctx || !info || !out) return TC_ERR_INVALID_ARG;
  *out = nullptr;
  const int T = info->n_trees, D = info->max_depth, L = 1 << (D > 0 ? D : 0);
  if (T < 0 || D < 0 || D > 13 || info->n_classes < 1 || info->n_classes > 16 || info->n_features < 1)
    return ctx->fail(TC_ERR_INVALID_ARG, "invalid model shape (trees %d, depth %d, classes %d, features %d)", T, D,
                     info->n_classes, info->n_features);
  if (T > 0 && (!depth || !feature || !threshold || !leaves))
    return ctx->fail(TC_ERR_INVALID_ARG, "missing model arrays");
  cudaSetDevice(ctx->device);
  tc_model* m = new tc_model();
  m->ctx = ctx;
  m->info = *info;
  m->depth.assign(depth, depth + T);
  for (int t = 0; t < T; ++t) {
    if (m->depth[t] < 0 || m->depth[t] > D) {
      delete m;
      return ctx->fail(TC_ERR_INVALID_ARG, "tree %d depth %d exceeds max_depth %d", t, depth[t], D);
    }
    for (int d = 0; d < m->depth[t]; ++d) {
      if (feature[(size_t)t * D + d] >= info->n_features) {
        delete m;
        return ctx->fail(TC_ERR_INVALID_ARG, "tree %d level %d splits on feature %d >= %d", t, d,
                         feature[(size_t)t * D + d], info->n_features);
      }
    }
  }
  m->feature.assign(feature, feature + (size_t)T * D);
  m->bin = bin ? std::vector<uint8_t>(bin, bin + (size_t)T * D) : std::vector<uint8_t>((size_t)T * D, 0);
  m->threshold.assign(threshold, threshold + (size_t)T * D);
  m->gain = gain ? std::vector<float>(gain, gain + (size_t)T * D) : std::vector<float>((size_t)T * D, 0.0f);
  m->leaves.assign(leaves, leaves + (size_t)T * L);
  m->weights = weights ? std::vector<float>(weights, weights + T) : std::vector<float>(T, info->learning_rate);
  if (edges && n_edges) {
    m->n_edges.assign(n_edges, n_edges + info->n_features);
    m->edges.assign(edges, edges + (size_t)info->n_features * 255);
  }
  tc_status s = m->upload();
  if (s != TC_OK) {
    delete m;
    return s;
  }
  *out = m;
  return TC_OK;
}

// TCAT v3 writer (src/boosting/booster.cpp:1049-1118, src/tree/symmetric_tree.cpp:1199-1215):
// host-endian, size_t counts.
tc_status tc_model_save_tcat(const tc_model* m, uint8_t* buf, size_t* len) {
  if (!m || !len) return TC_ERR_INVALID_ARG;
  std::vector<uint8_t> b;
  put(b, "TCAT", 4);
  const uint32_t version = 3;
  put(b, &version, 4);
  put(b, &m->info.base_prediction, 4);
  const uint8_t task = (uint8_t)m->info.task;
  put(b, &task, 1);
  const uint32_t ncls = m->info.task == TC_TASK_MULTICLASS ? (uint32_t)m->info.n_classes : 2u;
  put(b, &ncls, 4);
  put(b, &m->info.learning_rate, 4);
  const uint16_t md = (uint16_t)m->info.max_depth;
  put(b, &md, 2);
  put(b, &m->info.lambda_l2, 4);
  const uint8_t sym = 1;
  put(b, &sym, 1);
  const uint64_t nf = m->n_edges.size();
  put(b, &nf, 8);
  for (uint64_t j = 0; j < nf; ++j) {
    const uint64_t ne = m->n_edges[j];
    put(b, &ne, 8);
    if (ne) put(b, &m->edges[j * 255], ne * 4);
  }
  const uint64_t nt = (uint64_t)m->info.n_trees;
  put(b, &nt, 8);
  for (uint64_t t = 0; t < nt; ++t) put(b, &m->weights[t], 4);
  const int D = m->info.max_depth;
  for (uint64_t t = 0; t < nt; ++t) {
    const uint16_t dep = (uint16_t)m->depth[t];
    put(b, &dep, 2);
    for (int d = 0; d < dep; ++d) {
      const size_t q = t * D + d;
      put(b, &m->feature[q], 2);
      put(b, &m->bin[q], 1);
      put(b, &m->threshold[q], 4);
      put(b, &m->gain[q], 4);
    }
    const uint64_t nl = 1ull << dep;
    put(b, &nl, 8);
    put(b, &m->leaves[t << D], nl * 4);
  }
  if (!buf) {
    *len = b.size();
    return TC_OK;
  }
  if (*len < b.size()) {
    *len = b.size();
    return m->ctx->fail(TC_ERR_INVALID_ARG, "TCAT buffer too small (%zu bytes needed)", b.size());
  }
  std::memcpy(buf, b.data(), b.size());
  *len = b.size();
  return TC_OK;
}

// TCAT v3 reader (Booster::load_binary, src/boosting/booster.cpp:1120-1203);
// symmetric models only.
tc_status tc_model_load_tcat(tc_ctx* ctx, const uint8_t* buf, size_t len, tc_model** out) {
  if (!ctx || !buf || !out) return TC_ERR_INVALID_ARG;
  Reader r{buf, len};
  char magic[4];
  if (!r.bytes(magic, 4) || std::memcmp(magic, "TCAT", 4) != 0)
    return ctx->fail(TC_ERR_FORMAT, "Invalid TurboCat model file");
  const uint32_t version = r.get<uint32_t>();
  if (version != 3) return ctx->fail(TC_ERR_FORMAT, "Unsupported TurboCat model version: %u", version);
  tc_model_info info{};
  info.base_prediction = r.get<float>();
  info.task = r.get<uint8_t>();
  const uint32_t ncls = r.get<uint32_t>();
  info.learning_rate = r.get<float>();
  info.max_depth = r.get<uint16_t>();
  info.lambda_l2 = r.get<float>();
  const uint8_t sym = r.get<uint8_t>();
  if (!r.ok) return ctx->fail(TC_ERR_FORMAT, "truncated TCAT header");
  if (!sym) return ctx->fail(TC_ERR_FORMAT, "TCAT model holds regular trees; only symmetric trees are served");
  if (info.max_depth > 16) return ctx->fail(TC_ERR_FORMAT, "TCAT max_depth %d too large", info.max_depth);
  info.n_classes = info.task == TC_TASK_MULTICLASS ? (int)ncls : 1;
  if (info.n_classes < 1 || info.n_classes > 16) return ctx->fail(TC_ERR_FORMAT, "TCAT class count %u", ncls);
  const uint64_t nf = r.get<uint64_t>();
  if (!r.ok || nf == 0 || nf > 65535) return ctx->fail(TC_ERR_FORMAT, "TCAT feature count");
  info.n_features = (int)nf;
  std::vector<float> edges((size_t)nf * 255, 0.0f);
  std::vector<uint16_t> ne(nf);
  for (uint64_t j = 0; j < nf; ++j) {
    const uint64_t k = r.get<uint64_t>();
    if (!r.ok || k > 255) return ctx->fail(TC_ERR_FORMAT, "TCAT edge count");
    ne[j] = (uint16_t)k;
    if (k && !r.bytes(&edges[j * 255], k * 4)) return ctx->fail(TC_ERR_FORMAT, "truncated TCAT edges");
  }
  const uint64_t nt = r.get<uint64_t>();
  if (!r.ok || nt > (1ull << 24)) return ctx->fail(TC_ERR_FORMAT, "TCAT tree count");
  info.n_trees = (int)nt;
  const int D = info.max_depth, L = 1 << D;
  std::vector<float> w(nt);
  for (uint64_t t = 0; t < nt; ++t) w[t] = r.get<float>();
  std::vector<int32_t> depth(nt);
  std::vector<uint16_t> feat(nt * D, 0);
  std::vector<uint8_t> bin(nt * D, 0);
  std::vector<float> thr(nt * D, 0.0f), gain(nt * D, 0.0f), leaves(nt * L, 0.0f);
  for (uint64_t t = 0; t < nt && r.ok; ++t) {
    const uint16_t dep = r.get<uint16_t>();
    if (dep > D) return ctx->fail(TC_ERR_FORMAT, "TCAT tree %llu depth %u > max_depth %d", (unsigned long long)t, dep, D);
    depth[t] = dep;
    for (int d = 0; d < dep; ++d) {
      feat[t * D + d] = r.get<uint16_t>();
      bin[t * D + d] = r.get<uint8_t>();
      thr[t * D + d] = r.get<float>();
      gain[t * D + d] = r.get<float>();
    }
    const uint64_t nl = r.get<uint64_t>();
    if (!r.ok || nl > (uint64_t)L) return ctx->fail(TC_ERR_FORMAT, "TCAT leaf count");
    if (!r.bytes(&leaves[t * L], nl * 4)) return ctx->fail(TC_ERR_FORMAT, "truncated TCAT leaves");
  }
  if (!r.ok) return ctx->fail(TC_ERR_FORMAT, "truncated TCAT stream");
  const tc_status s = tc_model_import(ctx, &info, depth.data(), feat.data(), bin.data(), thr.data(), gain.data(),
                                      leaves.data(), w.data(), edges.data(), ne.data(), out);
  if (s == TC_ERR_INVALID_ARG) return TC_ERR_FORMAT;
  return s;
}

void tc_model_destroy(tc_model* m) { delete m; }

// Small request (n <= SMALL_ROWS): inputs and outputs through the context's
// pinned mapped staging, one launch of k_predict_small, one synchronisation.
// The staging and the device partials are allocated once, at their largest
// (SMALL_ROWS rows of SMALL_MAX_F features; one partial block per SM).
static tc_status predict_small(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint32_t f,
                               int32_t transform, float* out) {
  const int K = m->info.n_classes;
  const int T = m->info.n_trees;
  const long long walks = (long long)n * T;
  const int NB = (int)std::max<long long>(1, std::min<long long>(std::min(ctx->sm_count, T),
                                                                  (walks + SMALL_WALKS_PER_BLOCK - 1) /
                                                                      SMALL_WALKS_PER_BLOCK));
  const size_t in_cap = (size_t)SMALL_ROWS * SMALL_MAX_F;         // floats
  const size_t out_cap = (size_t)SMALL_ROWS * PRED_MAX_K;
  if (!ctx->pin_io) {
    // [inputs][outputs][the sequence word]
    TC_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&ctx->pin_io), (in_cap + out_cap + 16) * sizeof(float),
                               cudaHostAllocMapped));
    std::memset(ctx->pin_io, 0, (in_cap + out_cap + 16) * sizeof(float));
    TC_CUDA(ctx, cudaHostGetDevicePointer(reinterpret_cast<void**>(&ctx->pin_io_dev), ctx->pin_io, 0));
    ctx->pin_floats = in_cap + out_cap + 16;
  }
  if (!ctx->small_scratch) {
    // [256 B counter][partials: SMs x SMALL_ROWS x PRED_MAX_K][inputs: in_cap]
    const size_t bytes = 256 + ((size_t)ctx->sm_count * SMALL_ROWS * PRED_MAX_K + in_cap) * sizeof(float);
    TC_TRY(ctx->alloc(&ctx->small_scratch, bytes, "small predict partials"));
    TC_CUDA(ctx, cudaMemset(ctx->small_scratch, 0, bytes));
    ctx->small_scratch_bytes = bytes;
  }
  cudaStream_t st = ctx->pred_stream;
  uint32_t* counter = static_cast<uint32_t*>(ctx->small_scratch);
  float* partial = reinterpret_cast<float*>(static_cast<char*>(ctx->small_scratch) + 256);
  float* dx = partial + (size_t)ctx->sm_count * SMALL_ROWS * PRED_MAX_K;
  const size_t in_f = (size_t)n * f, out_f = (size_t)n * K;
  // A request of at most SMALL_INLINE floats travels in the launch's own
  // parameters; larger ones go to device memory in one copy from the pinned
  // buffer (measured: a kernel that reads its input over the bus in place
  // takes ~6 us longer than the copy).  Outputs are written by the kernel
  // straight into the mapped buffer.
  thread_local SmallRows inl_buf;
  SmallRows* inl = &inl_buf;
  const float* xk = nullptr;
  if (in_f <= (size_t)SMALL_INLINE) {
    std::memcpy(inl->v, X, in_f * sizeof(float));
  } else {
    std::memcpy(ctx->pin_io, X, in_f * sizeof(float));
    TC_CUDA(ctx, cudaMemcpyAsync(dx, ctx->pin_io, in_f * sizeof(float), cudaMemcpyHostToDevice, st));
    xk = dx;
  }
  const size_t smem = ((size_t)n * (f + 1) + (size_t)SMALL_THREADS * K) * sizeof(float);
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_predict_small, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_done = true;
  }
  k_predict_small<<<NB, SMALL_THREADS, smem, st>>>(model_desc(m), xk, n, transform, partial, counter,
                                                   ctx->pin_io_dev + in_cap, *inl);
  TC_CUDA(ctx, cudaGetLastError());
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  std::memcpy(out, ctx->pin_io + in_cap, out_f * sizeof(float));
  return TC_OK;
}

tc_status tc_predict(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint16_t f, int32_t transform,
                     float* out) {
  if (!ctx || !m || (!X && n) || (!out && n)) return TC_ERR_INVALID_ARG;
  if (f != (uint32_t)m->info.n_features)
    return ctx->fail(TC_ERR_INVALID_ARG, "X has %u features, the model expects %d", f, m->info.n_features);
  if (n == 0) return TC_OK;
  cudaSetDevice(ctx->device);
  const int K = m->info.n_classes;
  if (n <= (uint32_t)SMALL_ROWS && K <= PRED_MAX_K && f <= SMALL_MAX_F && m->info.n_trees > 0) {
    std::lock_guard<std::mutex> g(ctx->pred_mu);
    return predict_small(ctx, m, X, n, f, transform, out);
  }
  // input and output share one grow-only device buffer of the context, so a
  // call allocates nothing once the largest batch has been seen
  const size_t in_bytes = ((size_t)n * f * sizeof(float) + 255) / 256 * 256;
  const size_t need = in_bytes + (size_t)n * K * sizeof(float);
  std::lock_guard<std::mutex> g(ctx->pred_mu);
  if (ctx->pred_scratch_bytes < need) {
    if (ctx->pred_scratch) {
      cudaStreamSynchronize(ctx->pred_stream);
      ctx->release(ctx->pred_scratch);
      ctx->pred_scratch = nullptr;
      ctx->pred_scratch_bytes = 0;
    }
    const size_t cap = std::max(need, (size_t)1 << 20);
    TC_TRY(ctx->alloc(&ctx->pred_scratch, cap, "predict staging"));
    ctx->pred_scratch_bytes = cap;
  }
  float* dx = static_cast<float*>(ctx->pred_scratch);
  float* dout = reinterpret_cast<float*>(static_cast<char*>(ctx->pred_scratch) + in_bytes);
  cudaStream_t st = ctx->pred_stream;  // not the training stream, which another thread may be capturing
  TC_CUDA(ctx, cudaMemcpyAsync(dx, X, (size_t)n * f * sizeof(float), cudaMemcpyHostToDevice, st));
  TC_TRY(tc::predict_device(ctx, m, dx, n, f, transform, dout, st));
  TC_CUDA(ctx, cudaMemcpyAsync(out, dout, (size_t)n * K * sizeof(float), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  return TC_OK;
}

tc_status tc_predict_device(tc_ctx* ctx, const tc_model* m, const float* X_dev, uint32_t n, uint16_t f,
                            int32_t transform, float* out_dev, void* stream) {
  if (!ctx || !m || (!X_dev && n) || (!out_dev && n)) return TC_ERR_INVALID_ARG;
  if (f != (uint32_t)m->info.n_features)
    return ctx->fail(TC_ERR_INVALID_ARG, "X has %u features, the model expects %d", f, m->info.n_features);
  cudaSetDevice(ctx->device);
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->pred_stream;
  return tc::predict_device(ctx, m, X_dev, n, f, transform, out_dev, st);
}

}  // extern "C"
