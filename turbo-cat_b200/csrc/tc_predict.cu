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
// Device model.  Every tree is padded to the model's depth D (a padding
// split's bit is always 0; leaf l of a tree of depth d moves to l << (D - d))
// and the tree weight is folded into the leaves.  Float form: splits are
// (feature, threshold bits), the padding threshold NaN.  Binned form
// (single-output models): per feature, the model's distinct thresholds sorted
// and cut into virtual features of at most 127 borders; a row's bin on a
// virtual feature is the number of its borders <= x (NaN: 0), and
// x >= threshold  <=>  bin >= k, k the threshold's rank in its virtual
// feature + 1 (the same float compare, so the leaf index is exact).  The
// binarisation restates Dataset::apply_bins (src/core/dataset.cpp:346-379)
// with the model's borders in place of the training edges.
//
// Kernel layout: a block owns a tile of 128 rows of one job (one request of a
// coalesced serving batch, or the whole input of a single call); the tile's
// rows are staged row-major in shared memory (odd row stride: threads reading
// the same feature of different rows hit different banks).  Trees stream
// through shared memory in chunks (splits and leaves, two chunks in flight:
// cp.async, the next chunk lands while the current one is walked).
//
// Binned walk (models with a binned form): the tile is binarised once into a
// byte per (virtual feature, row) (Eytzinger-ordered borders: the i-th step of
// every search reads one of 2^i consecutive words), column-major, so the
// 32-bit word l of a column holds rows 4l..4l+3.  Lane l of each warp owns
// those rows; a split costs one 32-bit shared load and a byte-wise add
// (b + 128 - k sets bit 7 exactly when b >= k: bins are at most 127) for all
// four rows, and the level bits are gathered per byte with a shift and a mask.
// The 8 warps walk every 8th tree (warp w: trees w, w + 8, ...) and their
// sums are added in warp order.  Other models (multiclass, or no binned form)
// split the block's threads as row slots x tree groups, one row per thread,
// and add the groups' sums pairwise in a fixed order.  Which walk a tile
// takes depends only on its model, so a request gives the same bits alone or
// in a batch.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>

#include "tc_internal.h"

namespace tc {
namespace {

constexpr int PRED_ROWS = 128;
constexpr int PRED_THREADS = 256;
constexpr int PRED_WARPS = PRED_THREADS / 32;
constexpr int PRED_LEAF_STAGE_MIN = 4096;       // floats of one leaf stage at least (16 KB)
constexpr int PRED_STAGED_MAX_DEPTH = 5;        // deeper trees gather their leaves from global memory (L2)
constexpr int PRED_CHUNK = 128;                 // trees per chunk at most
constexpr int PRED_MAX_K = 16;
constexpr int BIN_MAX_BORDERS = 127;            // borders of one virtual feature (bins 0..127)
constexpr int BIN_MAX_VIRTUAL = 512;            // virtual features of a binned model (column offset < 2^16)
constexpr uint32_t kNaNBits = 0x7fc00000u;      // padding split threshold: x >= NaN is false

__host__ __device__ constexpr int row_stride(int f) { return f | 1; }  // odd: conflict-free column reads
__host__ __device__ constexpr size_t align16(size_t b) { return (b + 15) & ~(size_t)15; }

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
  int leaf_stage;              // floats of one leaf stage
  int split_stage;             // splits of one split stage
  ReqDesc one_req;
  ModelDesc one_model;
};

__device__ __forceinline__ float sigmoidf_ref(float x) { return 1.0f / (1.0f + expf(-x)); }

// Trees per chunk for a model of depth D (L leaves): bounded by both stages,
// at least one tree per warp (the host sizes the stages for that).
__device__ __forceinline__ int chunk_trees(int D, int L, int leaf_stage, int split_stage) {
  int c = min(PRED_CHUNK, split_stage / max(1, D));
  if (D <= PRED_STAGED_MAX_DEPTH) c = min(c, leaf_stage / L);
  return c;
}

// 32-bit shared-memory loads (shared-window addresses: 32-bit address
// arithmetic, no generic-to-shared conversion).
__device__ __forceinline__ uint4 lds128(uint32_t a) {
  uint4 v;
  asm volatile("ld.shared.v4.u32 {%0, %1, %2, %3}, [%4];\n" : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w) : "r"(a));
  return v;
}
__device__ __forceinline__ uint2 lds64(uint32_t a) {
  uint2 v;
  asm volatile("ld.shared.v2.u32 {%0, %1}, [%2];\n" : "=r"(v.x), "=r"(v.y) : "r"(a));
  return v;
}
__device__ __forceinline__ uint32_t lds32(uint32_t a) {
  uint32_t v;
  asm volatile("ld.shared.u32 %0, [%1];\n" : "=r"(v) : "r"(a));
  return v;
}
__device__ __forceinline__ float ldsf(uint32_t a) {
  float v;
  asm volatile("ld.shared.f32 %0, [%1];\n" : "=f"(v) : "r"(a));
  return v;
}

// NT binned trees (t, t + PRED_WARPS, ...) of depth D for the lane's 4 rows.
// Splits are stored in processing order: levels 7..0, then D-1..8, so that
// after the shifts byte i of `a` holds the first min(D, 8) levels of row i
// with level 0 in bit 7, and byte i of `b` the levels from 8 on.  Addresses:
// spc = the chunk's splits, sbl = this lane's word of bin column 0 (both in
// shared memory); leaves in shared memory (lvs) or, for GL, global (lvg).
template <int NT, int D, bool GL>
__device__ __forceinline__ void walk_bins4(uint32_t spc, uint32_t sbl, uint32_t lvs, const float* __restrict__ lvg,
                                           int t, float4& acc) {
  constexpr int L = 1 << D;
  uint2 q[NT][D];
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    const uint32_t sp = spc + (uint32_t)((t + u * PRED_WARPS) * D) * 8u;
    if constexpr (D % 2 == 0) {
#pragma unroll
      for (int d = 0; d < D / 2; ++d) {  // a tree's splits start on a 16-byte boundary
        const uint4 v = lds128(sp + 16u * d);
        q[u][2 * d] = make_uint2(v.x, v.y);
        q[u][2 * d + 1] = make_uint2(v.z, v.w);
      }
    } else {
#pragma unroll
      for (int d = 0; d < D; ++d) q[u][d] = lds64(sp + 8u * d);
    }
  }
  uint32_t w[NT][D];
#pragma unroll
  for (int u = 0; u < NT; ++u)
#pragma unroll
    for (int d = 0; d < D; ++d) w[u][d] = lds32(sbl + q[u][d].x);
#pragma unroll
  for (int u = 0; u < NT; ++u) {
    uint32_t a = 0, b = 0;
#pragma unroll
    for (int d = 0; d < D; ++d) {
      const uint32_t s = w[u][d] + q[u][d].y;  // bit 7 of byte i: bin of row i >= k
      if (d < 8) a = (a >> 1) | (s & 0x80808080u);
      else b = (b >> 1) | (s & 0x80808080u);
    }
    uint32_t idx[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const uint32_t hi = (a >> (8 * i)) & 0xffu;
      if constexpr (D <= 8) idx[i] = hi >> (8 - D);
      else idx[i] = (hi << (D - 8)) | (((b >> (8 * i)) & 0xffu) >> (16 - D));
    }
    const int tt = t + u * PRED_WARPS;
    float v[4];
    if constexpr (GL) {
      const float* lv = lvg + (size_t)tt * L;
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = __ldg(lv + idx[i]);
    } else {
      const uint32_t lv = lvs + (uint32_t)(tt * L) * 4u;
#pragma unroll
      for (int i = 0; i < 4; ++i) v[i] = ldsf(lv + 4u * idx[i]);
    }
    acc.x += v[0];
    acc.y += v[1];
    acc.z += v[2];
    acc.w += v[3];
  }
}

// The chunk's trees of warp w: pairs while two remain (depth <= 10), then one
// at a time; the sums go into acc in tree order either way.
template <int D, bool GL>
__device__ __forceinline__ void walk_chunk_bins4(uint32_t spc, uint32_t sbl, uint32_t lvs, const float* lvg, int w,
                                                 int tn, float4& acc) {
  int t = w;
  if constexpr (D <= 10)
    for (; t + PRED_WARPS < tn; t += 2 * PRED_WARPS) walk_bins4<2, D, GL>(spc, sbl, lvs, lvg, t, acc);
  for (; t < tn; t += PRED_WARPS) walk_bins4<1, D, GL>(spc, sbl, lvs, lvg, t, acc);
}

__global__ void __launch_bounds__(PRED_THREADS, 2) k_predict(JobTable jt) {
  extern __shared__ __align__(16) float smp[];
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
  const int nr = (int)min((uint32_t)PRED_ROWS, rq.n - r0);
  const int f = md.n_features;
  // row stride: for the binned walk, rows of a feature count that is a
  // multiple of 4 (16-byte aligned input) are staged densely by 16-byte
  // copies; others by 4-byte copies at an odd stride (conflict-free column
  // reads, which the float walk does once per split)
  const bool dense = md.bsplits != nullptr && (f & 3) == 0 && (reinterpret_cast<uintptr_t>(rq.X) & 15) == 0;
  const int fs = dense ? f : row_stride(f);
  const int D = md.max_depth;
  const int L = 1 << D;
  const int K = md.n_classes;
  const int LS = jt.leaf_stage, SS = jt.split_stage;
  const bool leaves_global = D > PRED_STAGED_MAX_DEPTH;
  const int tchunk = chunk_trees(D, L, LS, SS);
  const bool binned = md.bsplits != nullptr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // Regions.  Binned: [bins V x 128 B][borders][virtual features][U]; the
  // row tile lives in U until the tile is binarised, then U holds the
  // stages.  Float: [row tile][stages].
  char* base = reinterpret_cast<char*>(smp);
  const int V = md.n_virtual;
  uint8_t* s_bins = reinterpret_cast<uint8_t*>(base);
  float* s_bord = reinterpret_cast<float*>(base + align16((size_t)V * PRED_ROWS));
  uint2* s_vd = reinterpret_cast<uint2*>(reinterpret_cast<char*>(s_bord) + align16((size_t)md.n_bord * 4));
  char* U = binned ? reinterpret_cast<char*>(s_vd) + align16((size_t)V * 8) : base;
  float* s_x = reinterpret_cast<float*>(U);                      // [128][fs]
  char* stages = binned ? U : U + align16((size_t)PRED_ROWS * fs * 4);
  float* s_leaf = reinterpret_cast<float*>(stages);              // 2 x [LS]
  uint2* s_split = reinterpret_cast<uint2*>(s_leaf + 2 * (size_t)LS);  // 2 x [SS]
  // the tile's rows: one contiguous range of nr x f floats
  {
    const float* Xt = rq.X + (size_t)r0 * f;
    if (dense) {
      for (int q = threadIdx.x; q < nr * (f >> 2); q += PRED_THREADS) cp_async16(s_x + 4 * q, Xt + 4 * q);
    } else {
      for (int i = warp; i < nr; i += PRED_WARPS)  // a warp copies whole rows, lane = feature
        for (int j = lane; j < f; j += 32) cp_async4(&s_x[i * fs + j], &Xt[(size_t)i * f + j]);
    }
  }
  const uint2* gsplits = binned ? md.bsplits : md.splits;
  auto issue_chunk = [&](int t0, int buf) {
    const int tn = min(tchunk, md.n_trees - t0);
    if (!leaves_global) {
      float* dl = s_leaf + buf * LS;
      const float* gl = md.leaves + (size_t)t0 * L;
      const int cnt = tn * L;
      if (L >= 4) {
        for (int q = threadIdx.x; q < cnt / 4; q += PRED_THREADS) cp_async16(dl + 4 * q, gl + 4 * q);
      } else {
        for (int q = threadIdx.x; q < cnt; q += PRED_THREADS) cp_async4(dl + q, gl + q);
      }
    }
    uint2* ds = s_split + buf * SS;
    for (int q = threadIdx.x; q < tn * D; q += PRED_THREADS) cp_async8(ds + q, gsplits + (size_t)t0 * D + q);
  };
  if (binned) {
    // borders and virtual features (16-byte copies: both arrays are padded
    // to whole 16-byte units on the device)
    for (int q = threadIdx.x; q < (md.n_bord + 3) / 4; q += PRED_THREADS) cp_async16(s_bord + 4 * q, md.bord + 4 * q);
    for (int q = threadIdx.x; q < (V + 1) / 2; q += PRED_THREADS) cp_async16(s_vd + 2 * q, md.vdesc + 2 * q);
    cp_async_commit();
    cp_async_wait_all();
    __syncthreads();
    // binarise: warp w takes virtual features w, w + 8, ...; lane l rows
    // l, l + 32, l + 64, l + 96 (rows past the tile's last get bin 0)
    for (int v = warp; v < V; v += PRED_WARPS) {
      const uint2 vd = s_vd[v];
      const float* bt = s_bord + (vd.y & 0xffffffu);
      const int h = (int)(vd.y >> 24);
      float x[4];
      uint32_t nd[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = lane + 32 * i;
        x[i] = r < nr ? s_x[r * fs + vd.x] : 0.0f;
        nd[i] = 0;
      }
      for (int s = 0; s < h; ++s)
#pragma unroll
        for (int i = 0; i < 4; ++i) nd[i] = 2 * nd[i] + 1 + (uint32_t)(bt[nd[i]] <= x[i]);  // NaN: false
      const uint32_t first_leaf = (1u << h) - 1;
#pragma unroll
      for (int i = 0; i < 4; ++i) {
        const int r = lane + 32 * i;
        s_bins[v * PRED_ROWS + r] = r < nr ? (uint8_t)(nd[i] - first_leaf) : (uint8_t)0;
      }
    }
    __syncthreads();  // the bins are complete and the row tile's space is free for the stages
  }
  if (md.n_trees > 0) issue_chunk(0, 0);
  cp_async_commit();
  // binned walk state
  float4 acc4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  const uint32_t sbl = smem_addr(s_bins) + 4u * lane;
  // per-row walk state: row slots (a power of two >= nr) x tree groups
  int RT = PRED_ROWS;
  while (RT > 1 && (RT >> 1) >= nr) RT >>= 1;
  const int TG = PRED_THREADS / RT;
  const int row = threadIdx.x % RT, tg = threadIdx.x / RT;
  const float* xr = s_x + row * fs;
  float acc[PRED_MAX_K];
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k) acc[k] = 0.0f;
  for (int t0 = 0, buf = 0; t0 < md.n_trees; t0 += tchunk, buf ^= 1) {
    const int tn = min(tchunk, md.n_trees - t0);
    if (t0 + tchunk < md.n_trees) issue_chunk(t0 + tchunk, buf ^ 1);
    cp_async_commit();
    cp_async_wait_prev();  // this thread's copies of the tile and of chunk t0 have landed
    __syncthreads();       // ... and everybody's
    const float* lvc = leaves_global ? md.leaves + (size_t)t0 * L : s_leaf + buf * LS;
    const uint2* spc = s_split + buf * SS;
    if (binned) {
      const uint32_t spa = smem_addr(spc), lva = smem_addr(leaves_global ? s_leaf : lvc);
      switch (D) {
        case 1: walk_chunk_bins4<1, false>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 2: walk_chunk_bins4<2, false>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 3: walk_chunk_bins4<3, false>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 4: walk_chunk_bins4<4, false>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 5: walk_chunk_bins4<5, false>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 6: walk_chunk_bins4<6, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 7: walk_chunk_bins4<7, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 8: walk_chunk_bins4<8, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 9: walk_chunk_bins4<9, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 10: walk_chunk_bins4<10, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 11: walk_chunk_bins4<11, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        case 12: walk_chunk_bins4<12, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
        default: walk_chunk_bins4<13, true>(spa, sbl, lva, lvc, warp, tn, acc4); break;
      }
    } else if (row < nr) {
      for (int t = tg; t < tn; t += TG) {
        const uint2* sp = spc + t * D;
        uint2 q[kModelMaxDepth];
#pragma unroll
        for (int d = 0; d < kModelMaxDepth; ++d)
          if (d < D) q[d] = sp[d];
        float xv[kModelMaxDepth];
#pragma unroll
        for (int d = 0; d < kModelMaxDepth; ++d)
          if (d < D) xv[d] = xr[q[d].x];
        uint32_t idx = 0;
#pragma unroll
        for (int d = 0; d < kModelMaxDepth; ++d)
          if (d < D) idx = idx + idx + (uint32_t)(xv[d] >= __uint_as_float(q[d].y));  // false for NaN
        const float v = lvc[(size_t)t * L + idx];
        const int cls = K == 1 ? 0 : (t0 + t) % K;
#pragma unroll
        for (int k = 0; k < PRED_MAX_K; ++k)
          if (k == cls) acc[k] += v;
      }
    }
    __syncthreads();  // chunk t0's buffers are refilled by the next iteration's copies
  }
  cp_async_wait_all();
  __syncthreads();
  float* s_red = s_leaf;  // at least 2 x 4096 floats
  float* o = rq.out + (size_t)r0 * K;
  if (binned) {
    // [warp][128 rows]; row sums in warp order
    *reinterpret_cast<float4*>(&s_red[warp * PRED_ROWS + 4 * lane]) = acc4;
    __syncthreads();
    if (threadIdx.x >= nr) return;
    const int r = threadIdx.x;
    float s = s_red[r];
#pragma unroll
    for (int w = 1; w < PRED_WARPS; ++w) s += s_red[w * PRED_ROWS + r];
    const float raw = s + md.base;
    o[r] = (rq.transform == TC_TRANSFORM_SIGMOID) ? sigmoidf_ref(raw) : raw;
    return;
  }
  // [TG][RT][K] (TG*RT = PRED_THREADS, 256 x 16 floats <= one leaf stage)
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
  if (tg != 0 || row >= nr) return;
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k)
    if (k < K) acc[k] = s_red[row * K + k];
  o += (size_t)row * K;
  if (rq.transform == TC_TRANSFORM_SOFTMAX && K > 1) {
    float mx = -INFINITY;
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k)
      if (k < K) mx = fmaxf(mx, acc[k] + md.base);
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

constexpr int SMALL_ROWS = 64;
constexpr int SMALL_INLINE = 928;  // floats of a request carried in the launch parameters (4 KB in all)
struct SmallRows {
  float v[SMALL_INLINE];
};
constexpr int SMALL_THREADS = 512;
constexpr int SMALL_WALKS_PER_BLOCK = 4096;  // (row, tree) walks per block: one block for a single row
constexpr int SMALL_MAX_F = 512;   // features of a small request (its rows fit in shared memory)

// Trees [t0, t1) for the n rows staged in s_x ([n][f+1]): row slot =
// thread % RT, tree lane = thread / RT, trees in order within a lane, the
// lanes summed pairwise in a fixed order.  Tree t's splits and leaves are
// read at splits + (t - tb) * D and leaves + (t - tb) * 2^D (the model's
// arrays with tb = 0, or a block's slice of them in shared memory).  Leaves
// the block's sum of row r, class k in s_red[r * K + k] ([SMALL_THREADS][K]
// scratch).
__device__ __forceinline__ void small_trees(const ModelDesc& md, const float* __restrict__ s_x, uint32_t n, int t0,
                                            int t1, float* __restrict__ s_red, const uint2* __restrict__ splits,
                                            const float* __restrict__ leaves, int tb) {
  const int fs = md.n_features + 1;
  const int K = md.n_classes, D = md.max_depth, L = 1 << D;
  int RT = SMALL_ROWS;
  while (RT > 1 && (uint32_t)(RT >> 1) >= n) RT >>= 1;
  const int TG = blockDim.x / RT;
  const int row = threadIdx.x % RT, tg = threadIdx.x / RT;
  float acc[PRED_MAX_K];
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k) acc[k] = 0.0f;
  if ((uint32_t)row < n) {
    const float* xr = s_x + row * fs;
    // one tree: every split loaded before any compare; padding splits give 0 bits
    auto leaf_of = [&](int t) -> float {
      const uint2* sp = splits + (size_t)(t - tb) * D;
      uint2 q[kModelMaxDepth];
#pragma unroll
      for (int d = 0; d < kModelMaxDepth; ++d)
        if (d < D) q[d] = sp[d];
      uint32_t idx = 0;
#pragma unroll
      for (int d = 0; d < kModelMaxDepth; ++d)
        if (d < D) idx = idx + idx + (uint32_t)(xr[q[d].x] >= __uint_as_float(q[d].y));  // false for NaN
      return leaves[(size_t)(t - tb) * L + idx];
    };
    auto add = [&](int t, float v) {
      const int cls = K == 1 ? 0 : t % K;
#pragma unroll
      for (int k = 0; k < PRED_MAX_K; ++k)
        if (k == cls) acc[k] += v;
    };
    int t = t0 + tg;
    for (; t + TG < t1; t += 2 * TG) {  // two trees in flight, added in order
      const float v0 = leaf_of(t), v1 = leaf_of(t + TG);
      add(t, v0);
      add(t + TG, v1);
    }
    for (; t < t1; t += TG) add(t, leaf_of(t));
  }
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k)
    if (k < K) s_red[threadIdx.x * K + k] = acc[k];
  __syncthreads();
  // lanes pairwise, fixed order: thread t adds thread t + h * RT; once
  // h * RT <= 16 every pair lies in warp 0, which finishes with shuffles
  int h = TG >> 1;
  for (; h > 0 && h * RT >= 32; h >>= 1) {
    if (tg < h)
      for (int k = 0; k < K; ++k) s_red[threadIdx.x * K + k] += s_red[(threadIdx.x + h * RT) * K + k];
    __syncthreads();
  }
  if (h > 0) {
    if (threadIdx.x < 32) {
      for (int k = 0; k < K; ++k) {
        float v = s_red[threadIdx.x * K + k];
        for (int hh = h; hh > 0; hh >>= 1) v += __shfl_down_sync(0xffffffffu, v, hh * RT);
        if (threadIdx.x < RT) s_red[threadIdx.x * K + k] = v;
      }
    }
    __syncthreads();
  }
}

// Raw scores v[0..K) of one row plus the base, transformed, into o[0..K).
__device__ __forceinline__ void small_store(const ModelDesc& md, int transform, const float* v, float* o) {
  const int K = md.n_classes;
  if (transform == TC_TRANSFORM_SOFTMAX && K > 1) {
    float mx = -INFINITY;
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k)
      if (k < K) mx = fmaxf(mx, v[k] + md.base);
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

// With nb > 1 blocks taking part: store this block's sums
// (partial[block][row][K]); the last of the nb blocks to finish (completion
// counter; nobody waits) returns true and the blocks' sums are then
// complete, to be added in block order.
__device__ __forceinline__ bool small_publish(const ModelDesc& md, uint32_t n, const float* s_red, float* partial,
                                              uint32_t* counter, uint32_t nb) {
  const int K = md.n_classes;
  for (uint32_t r = threadIdx.x; r < n; r += blockDim.x)
    for (int k = 0; k < K; ++k) partial[((size_t)blockIdx.x * n + r) * K + k] = s_red[r * K + k];
  __shared__ bool s_last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();  // the block's partials (ordered before it by the barrier) before the count
    s_last = atomicAdd(counter, 1u) == nb - 1;
    if (s_last) __threadfence();
  }
  __syncthreads();
  return s_last;
}

// Row r's raw sums: this block's alone (nb == 1), or the nb blocks' partials
// in block order, read from s_comb when the last block staged them there
// (all loads in flight together), else from L2 one by one.
__device__ __forceinline__ void small_row_sums(const ModelDesc& md, uint32_t n, uint32_t r, const float* s_red,
                                               const float* partial, uint32_t nb, const float* s_comb, float* v) {
  const int K = md.n_classes;
#pragma unroll
  for (int k = 0; k < PRED_MAX_K; ++k) v[k] = nb > 1 ? 0.0f : (k < K ? s_red[r * K + k] : 0.0f);
  for (uint32_t b = 0; nb > 1 && b < nb; ++b)
#pragma unroll
    for (int k = 0; k < PRED_MAX_K; ++k)
      if (k < K) v[k] += s_comb ? s_comb[((size_t)b * n + r) * K + k] : __ldcg(&partial[((size_t)b * n + r) * K + k]);
}

// Small requests (at most SMALL_ROWS rows): the trees are split over the
// blocks of one launch instead of streamed through one block, as few blocks
// as the (row, tree) walks need (one block for a single row).  Block b walks
// trees [b*T/NB, (b+1)*T/NB) for every row of the request; with several
// blocks each stores one partial per (row, class) and the last block to
// finish adds them in block order.  The block that finishes adds the base,
// applies the transform and writes the outputs (which may be pinned host
// memory mapped into the device).  The rows come from device memory or, for
// the smallest requests, from the launch parameters.
__global__ void __launch_bounds__(SMALL_THREADS) k_predict_small(ModelDesc md, const float* __restrict__ X, uint32_t n,
                                                                  int transform, float* __restrict__ partial,
                                                                  uint32_t* __restrict__ counter,
                                                                  float* __restrict__ out, SmallRows inl) {
  extern __shared__ float sm_small[];
  const int f = md.n_features, fs = f + 1;
  const int K = md.n_classes;
  float* s_x = sm_small;                         // [n][f+1]
  float* s_red = s_x + n * fs;                   // [SMALL_THREADS][K]
  for (uint32_t i = threadIdx.x >> 5; i < n; i += blockDim.x >> 5)
    for (int j = threadIdx.x & 31; j < f; j += 32) s_x[i * fs + j] = X ? X[(size_t)i * f + j] : inl.v[i * f + j];
  __syncthreads();
  const int T = md.n_trees, NB = gridDim.x;
  small_trees(md, s_x, n, (int)((long long)T * blockIdx.x / NB), (int)((long long)T * (blockIdx.x + 1) / NB), s_red,
              md.splits, md.leaves, 0);
  if (NB > 1 && !small_publish(md, n, s_red, partial, counter, NB)) return;
  for (uint32_t r = threadIdx.x; r < n; r += blockDim.x) {
    float v[PRED_MAX_K];
    small_row_sums(md, n, r, s_red, partial, NB, nullptr, v);
    small_store(md, transform, v, out + (size_t)r * K);
  }
  if (NB > 1 && threadIdx.x == 0) *counter = 0u;  // re-armed for the next call
}

// ------------------------------------------------------- latency worker --
// A persistent cooperative kernel serving small requests of one model
// without a launch per request.  The host writes a request's rows into a
// pinned mailbox mapped into the device, then its request word (sequence,
// transform, rows); block 0 polls that word (system-scope acquire loads, a
// short sleep between polls), copies the rows into device memory and
// announces the request to the other blocks through a device word
// (generation counter); every block walks its tree range, the last block
// adds the partials in block order, writes the outputs into the mailbox and
// publishes seq_done (system-scope release).  Every wait is bounded: block 0
// stops after LW_IDLE_NS without a request or LW_LIFE_NS in all (or when the
// host sets stop), announces that, and the others follow; their own waits
// give up after LW_LIFE_NS + LW_IDLE_NS.  On exit block 0 sets `exited`; the
// host then launches a new worker for the next request.
struct LwBox {
  uint32_t req;        // host -> device: sequence << 16 | transform << 8 | rows
  uint32_t stop;
  uint32_t pad0[14];
  uint32_t seq_done;   // device -> host: sequence of the last answered request
  uint32_t exited;
  uint32_t pad1[14];
  float x[SMALL_ROWS * SMALL_MAX_F];
  float out[SMALL_ROWS * PRED_MAX_K];
};
constexpr uint64_t LW_IDLE_NS = 20000000ull;    // 20 ms without a request
constexpr uint64_t LW_LIFE_NS = 2000000000ull;  // 2 s per launch
constexpr int LW_MAX_BLOCKS = 32;
constexpr int LW_FLAG_WORDS = 64;               // [0] blocks done with a request, [32] blocks that left

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_acquire_sys(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_sys(uint32_t* p, uint32_t v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ unsigned long long ld_acquire_gpu_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release_gpu_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
constexpr uint32_t kLwEnd = 0xffffffffu;  // announcement: the worker ends (a request never has 255 rows)

// Block b of the nb blocks serving a request of n rows takes rows
// [n b / nb, n (b + 1) / nb) (nb = min(worker blocks, n)), loads them from the
// pinned mailbox itself (16-byte loads of the aligned range, all in flight
// together), walks every tree for them (the model from global memory, L2
// resident; its splits in shared memory when they fit) and writes their
// outputs into the mailbox; the last block to
// finish (completion counter) publishes seq_done.  One thread of block 0
// polls the request word (system-scope acquire loads over the bus) and
// announces each request, or the end, to the other blocks through a device
// word (generation counter).  Shared memory: [rows 64 x (f+1)][sums 512 x K].
__global__ void __launch_bounds__(SMALL_THREADS) k_predict_worker(ModelDesc md, LwBox* box, uint32_t* flag,
                                                                   uint32_t seen, int resident_splits) {
  extern __shared__ __align__(16) float sm_w[];
  __shared__ uint32_t s_cmd, s_req;
  const int f = md.n_features, fs = f + 1, K = md.n_classes, T = md.n_trees, D = md.max_depth;
  float* s_x = sm_w;                                   // [rows][f+1]
  float* s_red = s_x + (size_t)SMALL_ROWS * fs;        // [SMALL_THREADS][K]
  // the model's splits, copied once per launch when they fit (leaves stay in L2)
  uint2* s_sp = reinterpret_cast<uint2*>(s_red + (size_t)SMALL_THREADS * K);
  const uint2* splits = md.splits;
  if (resident_splits) {
    for (int q = threadIdx.x; q < T * D; q += blockDim.x) s_sp[q] = md.splits[q];
    splits = s_sp;
  }
  uint32_t* counter = flag;                            // blocks done with the current request
  uint32_t* exits = flag + 32;                         // blocks that have left
  // block 0's announcement: generation << 32 | request word (kLwEnd: leave),
  // one 64-bit word, so a block that sees a generation sees its request
  unsigned long long* ann = reinterpret_cast<unsigned long long*>(flag + 16);
  const uint64_t t_start = global_ns();
  uint32_t gen = 0;  // thread 0: the last generation announced / seen
  for (;;) {
    if (threadIdx.x == 0) {
      uint32_t req = kLwEnd;
      if (blockIdx.x == 0) {
        const uint64_t t_idle = global_ns();
        for (;;) {
          const uint32_t r = ld_acquire_sys(&box->req);
          if ((r >> 16) != seen) {
            req = r;
            break;
          }
          if (ld_acquire_sys(&box->stop)) break;
          const uint64_t now = global_ns();
          if (now - t_idle > LW_IDLE_NS || now - t_start > LW_LIFE_NS) break;
        }
        ++gen;
        if (gridDim.x > 1) st_release_gpu_u64(ann, (unsigned long long)gen << 32 | req);
      } else {
        const uint64_t t_wait = global_ns();
        for (;;) {
          const unsigned long long a = ld_acquire_gpu_u64(ann);
          if ((uint32_t)(a >> 32) != gen) {  // the latest announcement (earlier ones were not ours)
            gen = (uint32_t)(a >> 32);
            req = (uint32_t)a;
            break;
          }
          if (global_ns() - t_wait > LW_LIFE_NS + LW_IDLE_NS) break;  // leaves
        }
      }
      s_cmd = req == kLwEnd ? 2u : 1u;
      s_req = req;
    }
    __syncthreads();
    if (s_cmd != 1) break;
    const uint32_t n = min(s_req & 0xffu, (uint32_t)SMALL_ROWS);
    const int tr = (int)((s_req >> 8) & 0xffu);
    const uint32_t nb = min(gridDim.x, max(n, 1u));
    if (blockIdx.x < nb) {
      const uint32_t rb0 = n * blockIdx.x / nb, rb1 = n * (blockIdx.x + 1) / nb, nr = rb1 - rb0;
      // elements [rb0 f, rb1 f) of the rows, through the 16-byte units covering them
      const uint32_t e0 = rb0 * (uint32_t)f, e1 = rb1 * (uint32_t)f;
      const float4* src = reinterpret_cast<const float4*>(box->x);
      for (uint32_t q = e0 / 4 + threadIdx.x; q < (e1 + 3) / 4; q += blockDim.x) {
        const float4 v = __ldcv(src + q);
        const float e[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const uint32_t i = 4 * q + c;
          if (i >= e0 && i < e1) s_x[((i - e0) / f) * fs + (i - e0) % f] = e[c];
        }
      }
      __syncthreads();
      small_trees(md, s_x, nr, 0, T, s_red, splits, md.leaves, 0);
      for (uint32_t r = threadIdx.x; r < nr; r += blockDim.x) {
        float v[PRED_MAX_K];
        small_row_sums(md, nr, r, s_red, nullptr, 1, nullptr, v);
        small_store(md, tr, v, box->out + (size_t)(rb0 + r) * K);
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        if (nb == 1) {
          // a release at system scope: the outputs (ordered before it by the
          // barrier) are visible to whoever sees seq_done
          st_release_sys(&box->seq_done, s_req >> 16);
        } else {
          // the block's outputs are visible system-wide before the count; the
          // last block publishes seq_done
          __threadfence_system();
          if (atomicAdd(counter, 1u) == nb - 1) {
            *counter = 0u;
            st_release_sys(&box->seq_done, s_req >> 16);
          }
        }
      }
    }
    seen = s_req >> 16;
    __syncthreads();  // s_cmd / s_req are rewritten by the next poll
  }
  if (threadIdx.x == 0 && atomicAdd(exits, 1u) == gridDim.x - 1) st_release_sys(&box->exited, 1u);
}

// ------------------------------------------------------ regular trees --
// Models of regular (depth-wise) trees the reference trained with
// mode="small" are served as the reference predicts them
// (Booster::predict_raw_fast, src/boosting/booster.cpp:680-870, and
// TreeEnsemble::predict_batch_optimized, src/tree/tree.cpp:1471-1560): each
// row is binned against the model's edges (NaN -> 255; a feature of at most
// 16 edges takes the number of edges <= x, one of more edges std::lower_bound,
// the number of edges < x), then every tree is walked in order (right iff
// bin != 255 and bin > the node's bin) and sum = fma(weight, leaf, sum) in
// FP32, as the reference's build computes it; then + base and the transform.
// A block takes RB rows: their bins in shared memory, one thread per row
// walking the trees (nodes from L2).  Node children always follow their
// parent (checked at load), so every walk ends.
struct RegDesc {
  const uint4* nodes;
  const uint32_t* roots;
  const float* weights;
  const float* edges;   // [f][255]
  const int32_t* nedges;
  int32_t n_trees, n_features, n_nodes;
  float base;
};

__global__ void __launch_bounds__(128) k_predict_regular(RegDesc rd, const float* __restrict__ X, uint32_t n,
                                                         int rows_per_block, int transform, float* __restrict__ out) {
  extern __shared__ uint8_t s_b[];  // [rows_per_block][f]
  const int f = rd.n_features;
  const uint32_t r0 = blockIdx.x * (uint32_t)rows_per_block;
  const int nr = (int)min((uint32_t)rows_per_block, n - r0);
  for (int q = threadIdx.x; q < nr * f; q += blockDim.x) {
    const int r = q / f, j = q - r * f;
    const float x = X[(size_t)(r0 + r) * f + j];
    uint32_t b = 255;
    if (!isnan(x)) {
      const float* e = rd.edges + (size_t)j * 255;
      const int ne = rd.nedges[j];
      int lo = 0, hi = ne;  // first edge with x < e (at most 16 edges) or x <= e (more)
      if (ne <= 16) {
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (e[mid] <= x) lo = mid + 1; else hi = mid;
        }
      } else {
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (e[mid] < x) lo = mid + 1; else hi = mid;
        }
      }
      b = (uint32_t)lo;  // 255 beyond the last of 255 edges: routed left like NaN, as in the reference
    }
    s_b[q] = (uint8_t)b;
  }
  __syncthreads();
  const int r = threadIdx.x;
  if (r >= nr) return;
  const uint8_t* row = s_b + (size_t)r * f;
  float sum = 0.0f;
  for (int t = 0; t < rd.n_trees; ++t) {
    uint32_t node = rd.roots[t];
    uint4 nd = rd.nodes[node];
    for (int guard = 0; !(nd.x >> 24) && guard < rd.n_nodes; ++guard) {
      const uint32_t b = row[nd.x & 0xffffu];
      node = (b != 255u && b > ((nd.x >> 16) & 0xffu)) ? nd.z : nd.y;
      nd = rd.nodes[node];
    }
    sum = fmaf(rd.weights[t], __uint_as_float(nd.w), sum);
  }
  const float raw = sum + rd.base;
  out[r0 + r] = transform == TC_TRANSFORM_SIGMOID ? sigmoidf_ref(raw) : raw;
}

// Stage sizes for a batch whose deepest model has depth max_depth: a leaf
// stage holds at least one tree per warp (16 KB at least); a split stage
// holds the splits of as many trees as the leaf stage takes, for every depth
// up to max_depth.
void stage_sizes(int max_depth, int* leaf_stage, int* split_stage) {
  const int Ls = 1 << std::min(std::max(max_depth, 0), PRED_STAGED_MAX_DEPTH);
  const int LS = std::max(PRED_LEAF_STAGE_MIN, PRED_WARPS * Ls);
  int SS = PRED_WARPS;
  for (int d = 1; d <= max_depth; ++d) {
    const int trees = d <= PRED_STAGED_MAX_DEPTH ? std::min(PRED_CHUNK, LS >> d) : PRED_CHUNK;
    SS = std::max(SS, trees * d);
  }
  *leaf_stage = LS;
  *split_stage = (SS + 1) & ~1;  // whole 16-byte pairs
}

// Shared memory of one model's tiles (the larger of its two layouts).
size_t model_smem(int n_features, int n_virtual, int n_bord, bool binned, int leaf_stage, int split_stage) {
  const size_t S = (size_t)2 * leaf_stage * 4 + (size_t)2 * split_stage * 8;
  const size_t T = align16((size_t)PRED_ROWS * row_stride(n_features) * 4);
  size_t need = T + S;
  if (binned) {
    const size_t X = align16((size_t)n_virtual * PRED_ROWS) + align16((size_t)n_bord * 4) + align16((size_t)n_virtual * 8);
    need = std::max(need, X + std::max(T, S));
  }
  return need;
}

constexpr size_t PRED_SMEM_MAX = 220 * 1024;

tc_status launch_predict(tc_ctx* ctx, JobTable& jt, const PredictPlan& plan, uint32_t n_tiles, cudaStream_t stream) {
  if (n_tiles == 0) return TC_OK;
  jt.leaf_stage = plan.leaf_stage;
  jt.split_stage = plan.split_stage;
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_predict, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PRED_SMEM_MAX);
    attr_done = true;
  }
  if (plan.smem > PRED_SMEM_MAX)
    return ctx->fail(TC_ERR_INVALID_ARG, "the model's features do not fit the predict kernel's row tile (%zu bytes)",
                     plan.smem);
  k_predict<<<n_tiles, PRED_THREADS, plan.smem, stream>>>(jt);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ctx->cuda_fail(e, "k_predict");
  return TC_OK;
}

}  // namespace

PredictPlan predict_plan(const tc_model* const* models, int n) {
  int max_depth = 0;
  for (int i = 0; i < n; ++i) max_depth = std::max(max_depth, models[i]->info.max_depth);
  PredictPlan p{};
  stage_sizes(max_depth, &p.leaf_stage, &p.split_stage);
  for (int i = 0; i < n; ++i) {
    const tc_model* m = models[i];
    p.smem = std::max(p.smem, model_smem(m->info.n_features, m->n_virtual, m->n_bord, m->d_bsplits.p != nullptr,
                                         p.leaf_stage, p.split_stage));
  }
  return p;
}

tc_status predict_batched(tc_ctx* ctx, const ModelDesc* d_models, const ReqDesc* d_reqs, int n_reqs,
                          const uint32_t* d_tile_begin, uint32_t n_tiles, const PredictPlan& plan,
                          cudaStream_t stream) {
  JobTable jt{};
  jt.reqs = d_reqs;
  jt.models = d_models;
  jt.tile_begin = d_tile_begin;
  jt.n_jobs = n_reqs;
  return launch_predict(ctx, jt, plan, n_tiles, stream);
}

uint32_t predict_tiles(uint32_t n) { return (n + PRED_ROWS - 1) / PRED_ROWS; }

}  // namespace tc

using namespace tc;

namespace {

// Fills t[0 .. n) (n = 2^h - 1) with vals in Eytzinger (breadth-first) order:
// an in-order walk of the implicit tree visits vals in sorted order.
void eytzinger_fill(const std::vector<float>& vals, std::vector<float>& t, size_t base, size_t n, size_t i,
                    size_t& next) {
  if (i >= n) return;
  eytzinger_fill(vals, t, base, n, 2 * i + 1, next);
  t[base + i] = next < vals.size() ? vals[next] : std::nanf("");
  ++next;
  eytzinger_fill(vals, t, base, n, 2 * i + 2, next);
}

}  // namespace

// The device model: every tree padded to the model's depth (padding splits:
// feature 0 against a NaN threshold, whose bit is always 0; leaf l of a tree
// of depth d moves to l << (D - d)), the tree weights folded into the leaves
// (w * leaf in FP32, the product the reference forms per tree), the float
// splits (feature, threshold bits) and, for single-output models, the binned
// form (virtual features, Eytzinger-ordered borders, binned splits).
tc_status tc_model::upload() {
  const int T = info.n_trees, D = info.max_depth, L = 1 << D, F = info.n_features;
  std::vector<uint2> sp((size_t)std::max(1, T * D));
  std::vector<float> lv((size_t)std::max(1, T * L), 0.0f);
  for (int t = 0; t < T; ++t) {
    const int dt = depth[t];
    for (int d = 0; d < D; ++d) {
      uint32_t bits = kNaNBits, j = 0;
      if (d < dt) {
        std::memcpy(&bits, &threshold[(size_t)t * D + d], 4);
        j = feature[(size_t)t * D + d];
      }
      sp[(size_t)t * D + d] = make_uint2(j, bits);
    }
    for (int l = 0; l < (1 << dt); ++l) lv[(size_t)t * L + ((size_t)l << (D - dt))] = weights[t] * leaves[(size_t)t * L + l];
  }
  TC_TRY(d_splits.alloc(ctx, sp.size(), "model splits"));
  TC_TRY(d_leaves.alloc(ctx, lv.size(), "model leaves"));
  TC_CUDA(ctx, cudaMemcpy(d_splits.p, sp.data(), sp.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  TC_CUDA(ctx, cudaMemcpy(d_leaves.p, lv.data(), lv.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (info.n_classes != 1 || D < 1) return TC_OK;
  // binned form: distinct thresholds per feature (-0.0 and +0.0 are one)
  std::vector<std::vector<float>> u((size_t)F);
  for (int t = 0; t < T; ++t)
    for (int d = 0; d < depth[t]; ++d) {
      const float th = threshold[(size_t)t * D + d];
      if (!std::isnan(th)) u[feature[(size_t)t * D + d]].push_back(th);
    }
  struct VF { int j, start, cnt; };
  std::vector<VF> vf;
  std::vector<int> first_v((size_t)F, -1);
  for (int j = 0; j < F; ++j) {
    auto& a = u[j];
    std::sort(a.begin(), a.end());
    a.erase(std::unique(a.begin(), a.end(), [](float x, float y) { return x == y; }), a.end());
    for (int s0 = 0; s0 < (int)a.size(); s0 += BIN_MAX_BORDERS) {
      if (first_v[j] < 0) first_v[j] = (int)vf.size();
      vf.push_back({j, s0, std::min(BIN_MAX_BORDERS, (int)a.size() - s0)});
    }
  }
  if (vf.empty()) vf.push_back({0, 0, 0});  // padding splits read virtual feature 0
  if ((int)vf.size() > BIN_MAX_VIRTUAL) return TC_OK;  // served by the float walk
  std::vector<float> bord;
  std::vector<uint2> vd;
  for (const VF& v : vf) {
    int h = 0;
    while ((1 << h) - 1 < v.cnt) ++h;
    const size_t n = ((size_t)1 << h) - 1, off = bord.size();
    if (off + n >= ((size_t)1 << 24)) return TC_OK;
    bord.resize(off + n);
    std::vector<float> vals;
    if (v.cnt) vals.assign(u[v.j].begin() + v.start, u[v.j].begin() + v.start + v.cnt);
    size_t next = 0;
    eytzinger_fill(vals, bord, off, n, 0, next);
    vd.push_back(make_uint2((uint32_t)v.j, (uint32_t)off | ((uint32_t)h << 24)));
  }
  const int V = (int)vd.size(), B = (int)bord.size();
  {
    int LS, SS;
    stage_sizes(D, &LS, &SS);
    if (model_smem(F, V, B, true, LS, SS) > PRED_SMEM_MAX) return TC_OK;  // served by the float walk
  }
  while (bord.size() % 4) bord.push_back(std::nanf(""));  // whole 16-byte copies
  if (vd.size() % 2) vd.push_back(make_uint2(0, 0));
  // binned splits in processing order: levels min(D,8)-1 .. 0, then D-1 .. 8
  std::vector<uint2> bs((size_t)T * D);
  for (int t = 0; t < T; ++t) {
    for (int p = 0; p < D; ++p) {
      const int lev = D <= 8 ? D - 1 - p : (p < 8 ? 7 - p : D - 1 - (p - 8));
      uint2 q = make_uint2(0, 0);  // padding: k = 128, never reached by a bin
      if (lev < depth[t]) {
        const float th = threshold[(size_t)t * D + lev];
        if (!std::isnan(th)) {
          const int j = feature[(size_t)t * D + lev];
          const int r = (int)(std::lower_bound(u[j].begin(), u[j].end(), th) - u[j].begin());
          const int v = first_v[j] + r / BIN_MAX_BORDERS, k = r % BIN_MAX_BORDERS + 1;
          q = make_uint2((uint32_t)v * PRED_ROWS, (uint32_t)(128 - k) * 0x01010101u);
        }
      }
      bs[(size_t)t * D + p] = q;
    }
  }
  TC_TRY(d_bsplits.alloc(ctx, std::max<size_t>(1, bs.size()), "binned model splits"));
  TC_TRY(d_bord.alloc(ctx, bord.size(), "model borders"));
  TC_TRY(d_vdesc.alloc(ctx, vd.size(), "model virtual features"));
  if (!bs.empty())
    TC_CUDA(ctx, cudaMemcpy(d_bsplits.p, bs.data(), bs.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  TC_CUDA(ctx, cudaMemcpy(d_bord.p, bord.data(), bord.size() * sizeof(float), cudaMemcpyHostToDevice));
  TC_CUDA(ctx, cudaMemcpy(d_vdesc.p, vd.data(), vd.size() * sizeof(uint2), cudaMemcpyHostToDevice));
  n_virtual = V;
  n_bord = B;
  return TC_OK;
}

namespace tc {

ModelDesc model_desc(const tc_model* m) {
  ModelDesc d{};
  d.splits = m->d_splits.p;
  d.leaves = m->d_leaves.p;
  d.bsplits = m->d_bsplits.p;
  d.bord = m->d_bord.p;
  d.vdesc = m->d_vdesc.p;
  d.n_virtual = m->n_virtual;
  d.n_bord = m->n_bord;
  d.n_trees = m->info.n_trees;
  d.max_depth = m->info.max_depth;
  d.n_classes = m->info.n_classes;
  d.n_features = m->info.n_features;
  d.base = m->info.base_prediction;
  return d;
}

void stop_latency_worker(tc_ctx* ctx, const tc_model* m) {
  if (!ctx->lw_running || (m && ctx->lw_model != m)) return;
  volatile LwBox* box = static_cast<volatile LwBox*>(ctx->lw_box);
  box->stop = 1u;
  cudaStreamSynchronize(ctx->lw_stream);
  box->stop = 0u;
  ctx->lw_running = false;
  ctx->lw_model = nullptr;
}

tc_status predict_device(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint32_t f, int transform,
                         float* out, cudaStream_t stream) {
  if (n == 0) return TC_OK;
  if (m->regular) {
    RegDesc rd{m->d_rnodes.p, m->d_rroots.p, m->d_rweights.p, m->d_redges.p, m->d_rnedges.p,
               m->info.n_trees, m->info.n_features, (int)m->d_rnodes.n, m->info.base_prediction};
    const int rpb = (int)std::max<size_t>(1, std::min<size_t>(128, (size_t)160 * 1024 / std::max<uint32_t>(1, f)));
    const size_t smem = (size_t)rpb * f;
    static bool attr_done = false;
    if (!attr_done) {
      cudaFuncSetAttribute(k_predict_regular, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
      attr_done = true;
    }
    k_predict_regular<<<(n + rpb - 1) / rpb, 128, smem, stream>>>(rd, X, n, rpb, transform, out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return ctx->cuda_fail(e, "k_predict_regular");
    return TC_OK;
  }
  JobTable jt{};
  jt.reqs = nullptr;
  jt.n_jobs = 1;
  jt.one_model = model_desc(m);
  jt.one_req = ReqDesc{X, out, n, 0, 0, transform};
  return launch_predict(ctx, jt, predict_plan(&m, 1), predict_tiles(n), stream);
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
  if (m->regular)
    return m->ctx->fail(TC_ERR_INVALID_ARG, "a model of regular trees has no symmetric-tree export");
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
  if (T < 0 || D < 0 || D > kModelMaxDepth || info->n_classes < 1 || info->n_classes > 16 || info->n_features < 1)
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
  if (m->regular) {  // the stream as loaded (the reference's own bytes)
    if (buf) {
      if (*len < m->tcat.size()) return TC_ERR_INVALID_ARG;
      std::memcpy(buf, m->tcat.data(), m->tcat.size());
    }
    *len = m->tcat.size();
    return TC_OK;
  }
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

// The regular-tree branch of the TCAT v3 reader (Booster::load_binary,
// src/boosting/booster.cpp:1140-1203; Tree::load, src/tree/tree.cpp:1795-1840):
// single-output models (multiclass regular trees are refused).
static tc_status load_regular(tc_ctx* ctx, Reader& r, tc_model_info info, const uint8_t* buf, size_t len,
                              tc_model** out) {
  if (info.task == TC_TASK_MULTICLASS) return ctx->fail(TC_ERR_FORMAT, "multiclass regular trees are not served");
  info.n_classes = 1;
  const uint64_t nf = r.get<uint64_t>();
  if (!r.ok || nf == 0 || nf > 65535) return ctx->fail(TC_ERR_FORMAT, "TCAT feature count");
  std::vector<float> edges((size_t)nf * 255, 0.0f);
  std::vector<int32_t> ne(nf);
  for (uint64_t j = 0; j < nf; ++j) {
    const uint64_t k = r.get<uint64_t>();
    if (!r.ok || k > 255) return ctx->fail(TC_ERR_FORMAT, "TCAT edge count");
    ne[j] = (int32_t)k;
    if (k && !r.bytes(&edges[j * 255], k * 4)) return ctx->fail(TC_ERR_FORMAT, "truncated TCAT edges");
  }
  const uint64_t nt = r.get<uint64_t>();
  if (!r.ok || nt > (1ull << 24)) return ctx->fail(TC_ERR_FORMAT, "TCAT tree count");
  std::vector<float> w(nt);
  for (uint64_t t = 0; t < nt; ++t) w[t] = r.get<float>();
  std::vector<uint4> nodes;
  std::vector<uint32_t> roots(nt);
  for (uint64_t t = 0; t < nt && r.ok; ++t) {
    r.get<uint16_t>();  // depth
    const uint32_t tcls = r.get<uint32_t>();
    const uint32_t nn = r.get<uint32_t>();
    r.get<uint16_t>();  // leaves
    r.get<uint16_t>();  // max_depth
    r.get<float>();     // lambda_l2
    if (!r.ok) break;
    if (tcls > 1) return ctx->fail(TC_ERR_FORMAT, "multiclass regular trees are not served");
    if (nn == 0 || nn > 65535)
      return ctx->fail(TC_ERR_FORMAT, "TCAT tree %llu has %u nodes", (unsigned long long)t, nn);
    roots[t] = (uint32_t)nodes.size();
    for (uint32_t i = 0; i < nn && r.ok; ++i) {
      const uint16_t feat = r.get<uint16_t>();
      const uint8_t bin = r.get<uint8_t>();
      const uint8_t flags = r.get<uint8_t>();
      const uint16_t lc = r.get<uint16_t>(), rc = r.get<uint16_t>();
      const float value = r.get<float>();
      r.get<float>();  // gain
      const bool leaf = flags & 1u;
      // children follow their parent (the reference adds them after it), so walks end
      if (!leaf && (feat >= nf || lc <= i || rc <= i || lc >= nn || rc >= nn))
        return ctx->fail(TC_ERR_FORMAT, "TCAT tree %llu node %u: bad split", (unsigned long long)t, i);
      uint32_t vb;
      std::memcpy(&vb, &value, 4);
      nodes.push_back(make_uint4((uint32_t)feat | (uint32_t)bin << 16 | (leaf ? 1u : 0u) << 24,
                                 leaf ? 0u : roots[t] + lc, leaf ? 0u : roots[t] + rc, vb));
    }
  }
  if (!r.ok) return ctx->fail(TC_ERR_FORMAT, "truncated TCAT stream");
  info.n_trees = (int)nt;
  info.n_features = (int)nf;
  cudaSetDevice(ctx->device);
  tc_model* m = new tc_model();
  m->ctx = ctx;
  m->info = info;
  m->regular = true;
  m->tcat.assign(buf, buf + len);
  m->weights = w;
  auto up = [&]() -> tc_status {
    TC_TRY(m->d_rnodes.alloc(ctx, std::max<size_t>(1, nodes.size()), "regular tree nodes"));
    TC_TRY(m->d_rroots.alloc(ctx, std::max<size_t>(1, nt), "regular tree roots"));
    TC_TRY(m->d_rweights.alloc(ctx, std::max<size_t>(1, nt), "regular tree weights"));
    TC_TRY(m->d_redges.alloc(ctx, edges.size(), "regular model edges"));
    TC_TRY(m->d_rnedges.alloc(ctx, ne.size(), "regular model edge counts"));
    if (!nodes.empty())
      TC_CUDA(ctx, cudaMemcpy(m->d_rnodes.p, nodes.data(), nodes.size() * sizeof(uint4), cudaMemcpyHostToDevice));
    if (nt) {
      TC_CUDA(ctx, cudaMemcpy(m->d_rroots.p, roots.data(), nt * 4, cudaMemcpyHostToDevice));
      TC_CUDA(ctx, cudaMemcpy(m->d_rweights.p, w.data(), nt * 4, cudaMemcpyHostToDevice));
    }
    TC_CUDA(ctx, cudaMemcpy(m->d_redges.p, edges.data(), edges.size() * 4, cudaMemcpyHostToDevice));
    TC_CUDA(ctx, cudaMemcpy(m->d_rnedges.p, ne.data(), ne.size() * 4, cudaMemcpyHostToDevice));
    return TC_OK;
  };
  const tc_status s = up();
  if (s != TC_OK) {
    delete m;
    return s;
  }
  *out = m;
  return TC_OK;
}

// TCAT v3 reader (Booster::load_binary, src/boosting/booster.cpp:1120-1203):
// symmetric models here, regular ones through load_regular.
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
  if (!sym) return load_regular(ctx, r, info, buf, len, out);
  if (info.max_depth > kModelMaxDepth) return ctx->fail(TC_ERR_FORMAT, "TCAT max_depth %d too large", info.max_depth);
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

void tc_model_destroy(tc_model* m) {
  if (!m) return;
  if (m->ctx) {
    std::lock_guard<std::mutex> g(m->ctx->pred_mu);
    tc::stop_latency_worker(m->ctx, m);
  }
  delete m;
}

// Latency worker launch for model m (caller holds pred_mu; no worker runs).
static tc_status lw_launch(tc_ctx* ctx, const tc_model* m) {
  if (!ctx->lw_box) {
    TC_CUDA(ctx, cudaHostAlloc(&ctx->lw_box, sizeof(LwBox), cudaHostAllocMapped));
    std::memset(ctx->lw_box, 0, sizeof(LwBox));
    TC_CUDA(ctx, cudaHostGetDevicePointer(&ctx->lw_box_dev, ctx->lw_box, 0));
  }
  if (!ctx->lw_dev)
    TC_TRY(ctx->alloc(&ctx->lw_dev, LW_FLAG_WORDS * 4, "latency worker counters"));
  if (!ctx->lw_stream) TC_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->lw_stream, cudaStreamNonBlocking));
  static bool attr_done = false;
  if (!attr_done) {
    cudaFuncSetAttribute(k_predict_worker, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
    attr_done = true;
  }
  const int T = m->info.n_trees, K = m->info.n_classes, f = m->info.n_features, D = m->info.max_depth;
  const size_t base_smem = ((size_t)SMALL_ROWS * (f + 1) + (size_t)SMALL_THREADS * K) * sizeof(float);
  const size_t split_bytes = (size_t)T * D * sizeof(uint2);
  int resident = base_smem % 8 == 0 && base_smem + split_bytes <= 160 * 1024 ? 1 : 0;
  const size_t smem = base_smem + (resident ? split_bytes : 0);
  // blocks: a 64-row request split so that a block walks ~4096 (row, tree) pairs
  const long long want = ((long long)T * SMALL_ROWS + SMALL_WALKS_PER_BLOCK - 1) / SMALL_WALKS_PER_BLOCK;
  int per_sm = 0;
  TC_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_predict_worker, SMALL_THREADS, smem));
  if (per_sm < 1) return ctx->fail(TC_ERR_INVALID_ARG, "latency worker does not fit a multiprocessor");
  const int NB = (int)std::max<long long>(
      1, std::min<long long>({want, (long long)SMALL_ROWS, (long long)LW_MAX_BLOCKS,
                              (long long)std::max(1, ctx->sm_count / 4), (long long)per_sm * ctx->sm_count}));
  volatile LwBox* box = static_cast<volatile LwBox*>(ctx->lw_box);
  box->exited = 0u;
  box->stop = 0u;
  TC_CUDA(ctx, cudaMemsetAsync(ctx->lw_dev, 0, LW_FLAG_WORDS * 4, ctx->lw_stream));
  ModelDesc md = model_desc(m);
  LwBox* bd = static_cast<LwBox*>(ctx->lw_box_dev);
  uint32_t* flag = static_cast<uint32_t*>(ctx->lw_dev);
  uint32_t seen = box->seq_done;
  void* args[] = {&md, &bd, &flag, &seen, &resident};
  TC_CUDA(ctx, cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(k_predict_worker), dim3(NB),
                                           dim3(SMALL_THREADS), args, smem, ctx->lw_stream));
  ctx->lw_running = true;
  ctx->lw_model = m;
  ctx->lw_blocks = NB;
  return TC_OK;
}

// Small request through the latency worker (caller holds pred_mu): rows into
// the mailbox, then the request word, spin on seq_done.  A worker
// that ended (idle, lifetime) is relaunched; it serves the pending request.
static tc_status predict_worker(tc_ctx* ctx, const tc_model* m, const float* X, uint32_t n, uint32_t f,
                                int32_t transform, float* out) {
  if (ctx->lw_running && ctx->lw_model != m) tc::stop_latency_worker(ctx, nullptr);
  if (ctx->lw_running && static_cast<volatile LwBox*>(ctx->lw_box)->exited) {  // ended (idle or lifetime)
    cudaStreamSynchronize(ctx->lw_stream);
    ctx->lw_running = false;
  }
  if (!ctx->lw_running) TC_TRY(lw_launch(ctx, m));
  LwBox* box = static_cast<LwBox*>(ctx->lw_box);
  volatile LwBox* vb = box;
  std::memcpy(box->x, X, (size_t)n * f * sizeof(float));
  const uint32_t seq = ctx->lw_seq = (ctx->lw_seq + 1u) & 0xffffu;  // 16-bit sequence; only inequality matters
  std::atomic_thread_fence(std::memory_order_seq_cst);
  vb->req = seq << 16 | (uint32_t)transform << 8 | n;
  const auto t0 = std::chrono::steady_clock::now();
  for (uint32_t spin = 1;; ++spin) {
    if (vb->seq_done == seq) break;
    if ((spin & 1023u) == 0u) {
      if (vb->exited) {  // the worker ended before it saw the request
        cudaStreamSynchronize(ctx->lw_stream);
        ctx->lw_running = false;
        TC_TRY(lw_launch(ctx, m));
      }
      if (std::chrono::steady_clock::now() - t0 > std::chrono::seconds(5)) {
        tc::stop_latency_worker(ctx, nullptr);
        return ctx->fail(TC_ERR_TIMEOUT, "latency worker did not answer request %u", seq);
      }
    }
  }
  std::atomic_thread_fence(std::memory_order_seq_cst);
  std::memcpy(out, box->out, (size_t)n * m->info.n_classes * sizeof(float));
  return TC_OK;
}

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

// Grows the context's predict staging to `need` bytes (pred_mu held).
static tc_status grow_pred_scratch(tc_ctx* ctx, size_t need) {
  if (ctx->pred_scratch_bytes >= need) return TC_OK;
  if (ctx->pred_scratch) {
    cudaStreamSynchronize(ctx->pred_stream);
    ctx->release(ctx->pred_scratch);
    ctx->pred_scratch = nullptr;
    ctx->pred_scratch_bytes = 0;
  }
  const size_t cap = std::max(need, (size_t)1 << 20);
  TC_TRY(ctx->alloc(&ctx->pred_scratch, cap, "predict staging"));
  ctx->pred_scratch_bytes = cap;
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
  if (!m->regular && n <= (uint32_t)SMALL_ROWS && K <= PRED_MAX_K && f <= SMALL_MAX_F && m->info.n_trees > 0) {
    std::lock_guard<std::mutex> g(ctx->pred_mu);
    if (ctx->lw_enabled) return predict_worker(ctx, m, X, n, f, transform, out);
    return predict_small(ctx, m, X, n, f, transform, out);
  }
  // input and output share one grow-only device buffer of the context, so a
  // call allocates nothing once the largest batch has been seen
  const size_t in_bytes = ((size_t)n * f * sizeof(float) + 255) / 256 * 256;
  const size_t need = in_bytes + (size_t)n * K * sizeof(float);
  std::lock_guard<std::mutex> g(ctx->pred_mu);
  TC_TRY(grow_pred_scratch(ctx, need));
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

tc_status tc_predict_dataset(tc_ctx* ctx, const tc_model* m, const tc_dataset* ds, int32_t transform, float* out) {
  if (!ctx || !m || !ds || (!out && ds->n)) return TC_ERR_INVALID_ARG;
  if (ds->ctx != ctx) return ctx->fail(TC_ERR_INVALID_ARG, "the dataset belongs to another context");
  if (ds->f != (uint32_t)m->info.n_features)
    return ctx->fail(TC_ERR_INVALID_ARG, "the dataset has %u features, the model expects %d", ds->f, m->info.n_features);
  if (ds->n == 0) return TC_OK;
  cudaSetDevice(ctx->device);
  const size_t bytes = (size_t)ds->n * m->info.n_classes * sizeof(float);
  std::lock_guard<std::mutex> g(ctx->pred_mu);
  TC_TRY(grow_pred_scratch(ctx, bytes));
  float* dout = static_cast<float*>(ctx->pred_scratch);
  cudaStream_t st = ctx->pred_stream;
  TC_TRY(tc::predict_device(ctx, m, ds->X.p, ds->n, ds->f, transform, dout, st));
  TC_CUDA(ctx, cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  return TC_OK;
}

}  // extern "C"
