// Dataset upload and device quantile binning.
//
// Restates Dataset::compute_quantile_bins / find_bin
// (src/core/dataset.cpp:278-344) on the device:
//   1. every feature column becomes order-preserving uint32 keys
//      (-0.0 folded onto +0.0, NaN to the all-ones key so it sorts last);
//   2. a segmented LSD radix sort (4 x 8-bit passes, stable, one segment per
//      feature) orders each column;
//   3. a flag/scan pass over the sorted keys counts the U distinct non-NaN
//      values and picks edge b (b = 1 .. A-1) as the distinct value of rank
//      floor(b*U/A), A = min(max_bins, U) -- or min(max_bins, U mod 256)
//      in the reference-compatible mode (the reference truncates U to
//      uint8, src/core/dataset.cpp:308);
//   4. bin = number of edges <= x (std::upper_bound), NaN -> bin 255,
//      written both as feature-group tiles (histogram kernels: group g of 32
//      features is one contiguous [rows][32] block, so a row's slice of a
//      group is one aligned 32-byte sector and a run of rows is one
//      contiguous range; the last group's block is only 4, 8, 16 or 32
//      bytes wide) and column-major [f][np] (partition kernels, export).
#include <algorithm>
#include <atomic>
#include <cmath>

#include <cstring>
#include <thread>

#include "tc_internal.h"

namespace tc {
namespace {

constexpr int RS_THREADS = 256;
constexpr int RS_ITEMS = 16;
constexpr int RS_TILE = RS_THREADS * RS_ITEMS;
constexpr uint32_t NAN_KEY = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t float_key(float x) {
  if (isnan(x)) return NAN_KEY;
  if (x == 0.0f) x = 0.0f;  // fold -0.0 onto +0.0 (std::unique treats them as equal)
  const uint32_t u = __float_as_uint(x);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__device__ __forceinline__ float key_float(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  return __uint_as_float(u);
}

// X [n][f] row-major -> keys [f][n] via 32x32 shared-memory tiles.
__global__ void k_make_keys(const float* __restrict__ X, uint32_t n, uint32_t f,
                            uint32_t* __restrict__ keys) {
  __shared__ uint32_t t[32][33];
  const uint32_t r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t r = r0 + i, c = c0 + threadIdx.x;
    if (r < n && c < f) t[i][threadIdx.x] = float_key(X[(size_t)r * f + c]);
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const uint32_t c = c0 + i, r = r0 + threadIdx.x;
    if (r < n && c < f) keys[(size_t)c * n + r] = t[threadIdx.x][i];
  }
}

__global__ void k_radix_count(const uint32_t* __restrict__ keys, uint32_t n, uint32_t n_tiles,
                              int shift, uint32_t* __restrict__ counts) {
  __shared__ uint32_t h[256];
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  h[threadIdx.x] = 0;
  __syncthreads();
  const uint32_t* kj = keys + (size_t)j * n;
  for (int it = 0; it < RS_ITEMS; ++it) {
    const uint32_t idx = tile * RS_TILE + it * RS_THREADS + threadIdx.x;
    if (idx < n) atomicAdd(&h[(kj[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  counts[((size_t)j * 256 + threadIdx.x) * n_tiles + tile] = h[threadIdx.x];
}

// Exclusive scan, in place, of each segment a[j*m .. j*m+m); totals[j] = sum.
__global__ void k_segment_scan(uint32_t* __restrict__ a, uint32_t m, uint32_t* __restrict__ totals) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t carry_s;
  uint32_t* s = a + (size_t)blockIdx.x * m;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x == 0) carry_s = 0;
  __syncthreads();
  for (uint32_t base = 0; base < m; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const uint32_t v = i < m ? s[i] : 0u;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < nw ? warp_sums[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      if (lane < nw) warp_sums[lane] = w;  // inclusive
    }
    __syncthreads();
    const uint32_t carry = carry_s;
    const uint32_t excl = carry + (warp ? warp_sums[warp - 1] : 0u) + x - v;
    if (i < m) s[i] = excl;
    __syncthreads();
    if (threadIdx.x == 0) carry_s = carry + warp_sums[nw - 1];
    __syncthreads();
  }
  if (threadIdx.x == 0 && totals) totals[blockIdx.x] = carry_s;
}

// Stable scatter of one radix pass.  Keys of a tile are visited in index
// order (round-major, then thread order); a key's slot is its digit's global
// offset for the tile + the count of equal digits before it in the tile.
__global__ void k_radix_scatter(const uint32_t* __restrict__ kin, uint32_t* __restrict__ kout,
                                uint32_t n, uint32_t n_tiles, int shift,
                                const uint32_t* __restrict__ offsets,
                                const uint32_t* __restrict__ vin = nullptr, uint32_t* __restrict__ vout = nullptr) {
  __shared__ uint32_t s_base[256];
  __shared__ uint32_t s_run[256];
  __shared__ uint32_t s_w[RS_THREADS / 32][256];
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  s_base[tid] = offsets[((size_t)j * 256 + tid) * n_tiles + tile];
  s_run[tid] = 0;
  for (int w = 0; w < RS_THREADS / 32; ++w) s_w[w][tid] = 0;
  __syncthreads();
  const uint32_t* ki = kin + (size_t)j * n;
  uint32_t* ko = kout + (size_t)j * n;
  const uint32_t lt = (1u << lane) - 1u;
  for (int it = 0; it < RS_ITEMS; ++it) {
    const uint32_t idx = tile * RS_TILE + it * RS_THREADS + tid;
    const bool valid = idx < n;
    const uint32_t key = valid ? ki[idx] : 0u;
    const uint32_t d = valid ? ((key >> shift) & 255u) : 256u;
    const uint32_t mask = __match_any_sync(0xffffffffu, d);
    const uint32_t rank = __popc(mask & lt);
    if (valid && rank == 0) s_w[warp][d] = __popc(mask);
    __syncthreads();
    {
      uint32_t run = s_run[tid];
      for (int w = 0; w < RS_THREADS / 32; ++w) {
        const uint32_t c = s_w[w][tid];
        s_w[w][tid] = run;
        run += c;
      }
      s_run[tid] = run;
    }
    __syncthreads();
    if (valid) {
      const uint32_t slot = s_base[d] + s_w[warp][d] + rank;
      ko[slot] = key;
      if (vout) vout[(size_t)j * n + slot] = vin[(size_t)j * n + idx];  // payload rides along
    }
    __syncthreads();
    for (int w = 0; w < RS_THREADS / 32; ++w) s_w[w][tid] = 0;
    __syncthreads();
  }
}

__device__ __forceinline__ bool uniq_flag(const uint32_t* kj, uint32_t idx, uint32_t n) {
  if (idx >= n) return false;
  const uint32_t k = kj[idx];
  return k != NAN_KEY && (idx == 0 || kj[idx - 1] != k);
}

__global__ void k_unique_count(const uint32_t* __restrict__ keys, uint32_t n, uint32_t n_tiles,
                               uint32_t* __restrict__ tile_cnt) {
  __shared__ uint32_t s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  const uint32_t* kj = keys + (size_t)j * n;
  uint32_t c = 0;
  for (int it = 0; it < RS_ITEMS; ++it) c += uniq_flag(kj, tile * RS_TILE + it * RS_THREADS + threadIdx.x, n);
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s, c);
  __syncthreads();
  if (threadIdx.x == 0) tile_cnt[(size_t)j * n_tiles + tile] = s;
}

__device__ __forceinline__ uint32_t actual_bins(uint32_t U, int max_bins, int compat_u8) {
  const uint32_t a = compat_u8 ? (U & 255u) : U;
  return a < (uint32_t)max_bins ? a : (uint32_t)max_bins;
}

// Picks edge b-1 = distinct value of rank floor(b*U/A) for b = 1 .. A-1.
__global__ void k_unique_pick(const uint32_t* __restrict__ keys, uint32_t n, uint32_t n_tiles,
                              const uint32_t* __restrict__ tile_off, const uint32_t* __restrict__ U_,
                              int max_bins, int compat_u8, const uint8_t* __restrict__ ts,
                              float* __restrict__ edges) {
  __shared__ uint32_t warp_sums[RS_THREADS / 32];
  __shared__ uint32_t run_s;
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  const uint32_t* kj = keys + (size_t)j * n;
  const uint64_t U = U_[j];
  // numeric: edge b-1 = rank floor(b*U/A), b = 1 .. A-1; target statistics:
  // edge b-1 = rank floor(b*U/(A+1)), b = 1 .. A (src/core/dataset.cpp:221-224)
  const uint64_t A = actual_bins((uint32_t)U, max_bins, compat_u8) + (ts && ts[j] ? 1 : 0);
  if (A < 2) return;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) run_s = tile_off[(size_t)j * n_tiles + tile];
  __syncthreads();
  for (int it = 0; it < RS_ITEMS; ++it) {
    const uint32_t idx = tile * RS_TILE + it * RS_THREADS + threadIdx.x;
    const uint32_t fl = uniq_flag(kj, idx, n);
    uint32_t x = fl;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    uint32_t before = run_s;
    for (int w = 0; w < warp; ++w) before += warp_sums[w];
    if (fl) {
      const uint64_t r = before + x - 1;  // distinct-value rank
      // the smallest b with floor(b*U/A) >= r; b >= 1 (with A > U, as the
      // target-statistics rule has for A = U, rank 0 is edge 0)
      const uint64_t b = max((r * A + U - 1) / U, (uint64_t)1);
      if (b >= 1 && b <= A - 1 && (b * U) / A == r) edges[(size_t)j * kSlots + (b - 1)] = key_float(kj[idx]);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < RS_THREADS / 32; ++w) t += warp_sums[w];
      run_s += t;
    }
    __syncthreads();
  }
}

__global__ void k_edge_meta(const uint32_t* __restrict__ U_, uint32_t f, int max_bins, int compat_u8,
                            const uint8_t* __restrict__ ts, float* __restrict__ edges,
                            uint16_t* __restrict__ n_edges) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= f) return;
  const uint32_t U = U_[j];
  if (U == 0) {  // every value NaN: one edge {0.0f} (src/core/dataset.cpp:296-303)
    edges[(size_t)j * kSlots] = 0.0f;
    n_edges[j] = 1;
    return;
  }
  const uint32_t A = actual_bins(U, max_bins, compat_u8);
  n_edges[j] = (uint16_t)((ts && ts[j]) ? A : (A >= 2 ? A - 1 : 0));
}

constexpr int AB_ROWS = 256;

// bin = #edges <= x (upper_bound), NaN -> 255; target-statistics columns
// (ts[j]) take #edges < x (lower_bound, src/core/dataset.cpp:226-235); writes
// both bin layouts.  Block (row tile, group): 256 rows of the 32 features of
// group blockIdx.y.
__global__ void k_assign_bins(const float* __restrict__ X, uint32_t n, uint32_t f,
                              const float* __restrict__ edges, const uint16_t* __restrict__ n_edges,
                              const uint8_t* __restrict__ ts,
                              uint8_t* __restrict__ bins_t, uint64_t gstride, uint32_t nt, uint32_t wlast,
                              uint8_t* __restrict__ bins_cm, uint32_t np, uint32_t* __restrict__ nan_any) {
  __shared__ float s_e[32][kSlots + 1];
  __shared__ int s_ne[32];
  __shared__ uint8_t s_b[32][AB_ROWS + 4];
  __shared__ int s_nan[32];
  __shared__ int s_ts[32];
  const uint32_t j0 = blockIdx.y * 32, r0 = blockIdx.x * AB_ROWS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int q = tid; q < 32 * kSlots; q += blockDim.x) {
    const int jj = q / kSlots, e = q % kSlots;
    s_e[jj][e] = (j0 + jj < f) ? edges[(size_t)(j0 + jj) * kSlots + e] : 0.0f;
  }
  if (tid < 32) {
    s_ne[tid] = (j0 + tid < f) ? (int)n_edges[j0 + tid] : 0;
    s_ts[tid] = (ts && j0 + tid < f) ? (int)ts[j0 + tid] : 0;
    s_nan[tid] = 0;
  }
  __syncthreads();
  const uint32_t j = j0 + lane;
  for (int i = warp; i < AB_ROWS; i += nw) {
    const uint32_t r = r0 + i;
    uint8_t b = 0;
    if (r < n && j < f) {
      const float x = X[(size_t)r * f + j];
      if (isnan(x)) {
        b = (uint8_t)kNanBin;
        s_nan[lane] = 1;
      } else {
        int lo = 0, hi = s_ne[lane];
        const bool lower = s_ts[lane] != 0;
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          const float e = s_e[lane][mid];
          if (lower ? (x <= e) : (x < e)) hi = mid; else lo = mid + 1;
        }
        b = (uint8_t)lo;
        if (lo == kNanBin) s_nan[lane] = 1;  // a target-statistics column's top bin shares the NaN slot
      }
    }
    s_b[lane][i] = b;
  }
  __syncthreads();
  if (tid < 32 && s_nan[tid] && j0 + tid < f) atomicOr(&nan_any[j0 + tid], 1u);
  // column-major rows of this tile
  for (int q = tid; q < 32 * AB_ROWS; q += blockDim.x) {
    const int jj = q / AB_ROWS, i = q % AB_ROWS;
    const uint32_t r = r0 + i;
    if (j0 + jj < f && r < np) bins_cm[(size_t)(j0 + jj) * np + r] = (r < n) ? s_b[jj][i] : (uint8_t)0;
  }
  // the group's tile block: rows r0.. at a stride of the group's width
  const uint32_t w = (blockIdx.y == gridDim.y - 1) ? wlast : 32u;
  uint8_t* blk = bins_t + (uint64_t)blockIdx.y * gstride;
  for (int q = tid; q < 32 * AB_ROWS; q += blockDim.x) {
    const int i = q / 32, jj = q % 32;
    const uint32_t r = r0 + i;
    if (r < nt && (uint32_t)jj < w) blk[(size_t)r * w + jj] = (r < n && j0 + jj < f) ? s_b[jj][i] : (uint8_t)0;
  }
}

// ------------------------------------------- categorical target statistics
//
// Dataset::compute_ordered_target_statistics / compute_cv_target_statistics
// (src/core/dataset.cpp:722-865) on the device.  Each encoded column's rows
// are keyed by category in processing order and stably sorted (the radix sort
// above, the row index riding along), so every category becomes one
// contiguous segment in processing order.  One thread then walks a segment
// with the reference's float arithmetic: the running sums depend on the order
// of the additions in float, so they are kept sequential in the reference's
// order rather than scanned in parallel.  The walk writes each row's encoding
// into X and the category's global entry into the table; segments come in
// category order, so the table comes out sorted.

constexpr uint32_t CAT_NAN = 0xFFFFFFFFu;  // key of NaN rows; category 0xFFFFFFFF shares it, the walk tells them apart
constexpr int CAT_MAX_FOLDS = 32;
constexpr int CAT_THREADS = 256;

// static_cast<Index>(val) as x86-64 compiles it: truncate to 64 bits, keep the low 32.
__device__ __forceinline__ uint32_t category_of(float x) { return (uint32_t)(unsigned long long)(long long)x; }

// 32-bit integer finaliser ("lowbias32", C. Wellons' hash prospector).
__host__ __device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// Processing order of the ordered method and folds of the cross-validated
// one.  Drawn from the seed: position p -> row by a 4-round Feistel bijection
// on [0, 4^half) with cycle walking into [0, n) (a permutation with no sort
// and no table); fold of a row = hash of the row mod folds.  Or given by the
// caller (`given`: row of each position / fold of each row).
struct CatOrder {
  uint32_t key[4];
  uint32_t half;
  uint32_t folds;
  int cv;
  const uint32_t* given;
};

__device__ __forceinline__ uint32_t feistel(uint32_t x, const CatOrder& o) {
  const uint32_t m = (1u << o.half) - 1u;
  uint32_t l = x >> o.half, r = x & m;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const uint32_t t = l ^ (mix32(r ^ o.key[i]) & m);
    l = r;
    r = t;
  }
  return (l << o.half) | r;
}

__device__ __forceinline__ uint32_t order_row(uint32_t p, uint32_t n, const CatOrder& o) {
  if (o.given) return o.given[p];
  uint32_t x = p;
  do x = feistel(x, o); while (x >= n);  // ends: p's cycle under the bijection returns to p < n
  return x;
}

__device__ __forceinline__ uint32_t fold_of(uint32_t row, const CatOrder& o) {
  return o.given ? o.given[row] : mix32(mix32(row ^ o.key[0]) + o.key[1]) % o.folds;
}

// std::accumulate(labels, 0.0f) / n (src/core/dataset.cpp:685): one thread
// adds in row order, the block stages the labels through shared memory.
__global__ void k_label_prior(const float* __restrict__ y, uint32_t n, float* __restrict__ prior) {
  __shared__ float s[2048];
  float acc = 0.0f;
  for (uint32_t base = 0; base < n; base += 2048) {
    const uint32_t m = min(2048u, n - base);
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) s[i] = y[base + i];
    __syncthreads();
    if (threadIdx.x == 0)
      for (uint32_t i = 0; i < m; ++i) acc = __fadd_rn(acc, s[i]);
  }
  if (threadIdx.x == 0) prior[0] = n ? __fdiv_rn(acc, __uint2float_rn(n)) : 0.0f;
}

// keys[c][p] = category of the row at position p of column feats[c],
// rows[c][p] = that row (positions in processing order; rows in row order for
// the cross-validated method).
__global__ void k_cat_keys(const float* __restrict__ X, uint32_t n, uint32_t f,
                           const uint16_t* __restrict__ feats, CatOrder o, uint32_t* __restrict__ keys,
                           uint32_t* __restrict__ rows) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (p >= n) return;
  const uint32_t row = o.cv ? p : order_row(p, n, o);
  const float v = X[(size_t)row * f + feats[c]];
  keys[(size_t)c * n + p] = isnan(v) ? CAT_NAN : category_of(v);
  rows[(size_t)c * n + p] = row;
}

__device__ __forceinline__ uint32_t seg_flag(const uint32_t* kj, uint32_t idx, uint32_t n) {
  return idx < n && (idx == 0 || kj[idx - 1] != kj[idx]);
}

__global__ void k_seg_count(const uint32_t* __restrict__ keys, uint32_t n, uint32_t n_tiles,
                            uint32_t* __restrict__ tile_cnt) {
  __shared__ uint32_t s;
  if (threadIdx.x == 0) s = 0;
  __syncthreads();
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  const uint32_t* kj = keys + (size_t)j * n;
  uint32_t c = 0;
  for (int it = 0; it < RS_ITEMS; ++it) c += seg_flag(kj, tile * RS_TILE + it * RS_THREADS + threadIdx.x, n);
  for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(&s, c);
  __syncthreads();
  if (threadIdx.x == 0) tile_cnt[(size_t)j * n_tiles + tile] = s;
}

// starts[j][rank] = first sorted position of the rank-th segment of column j.
__global__ void k_seg_starts(const uint32_t* __restrict__ keys, uint32_t n, uint32_t n_tiles,
                             const uint32_t* __restrict__ tile_off, uint32_t* __restrict__ starts,
                             uint32_t* __restrict__ segid) {
  __shared__ uint32_t warp_sums[RS_THREADS / 32];
  __shared__ uint32_t run_s;
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  const uint32_t* kj = keys + (size_t)j * n;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) run_s = tile_off[(size_t)j * n_tiles + tile];
  __syncthreads();
  for (int it = 0; it < RS_ITEMS; ++it) {
    const uint32_t idx = tile * RS_TILE + it * RS_THREADS + threadIdx.x;
    const uint32_t fl = seg_flag(kj, idx, n);
    uint32_t x = fl;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    uint32_t before = run_s;
    for (int w = 0; w < warp; ++w) before += warp_sums[w];
    if (fl) starts[(size_t)j * n + before + x - 1] = idx;
    if (segid && idx < n) segid[(size_t)j * n + idx] = before + x - 1;  // rank of idx's segment
    __syncthreads();
    if (threadIdx.x == 0) {
      uint32_t t = 0;
      for (int w = 0; w < RS_THREADS / 32; ++w) t += warp_sums[w];
      run_s += t;
    }
    __syncthreads();
  }
}

// One thread per category segment: the row encodings and the category's
// global entry.  Ordered (src/core/dataset.cpp:738-780): a row sees the sum
// and count of its category's rows before it, the prior when there are none.
// Cross-validated (src/core/dataset.cpp:799-863): per-fold sums in row order,
// a row sees the other folds' sums added in fold order.  Smoothing
// (sum + a * prior) / (count + a); NaN rows get the prior and count nowhere.
__global__ void k_cat_walk(const float* __restrict__ y, float* __restrict__ X, uint32_t n, uint32_t f,
                           const uint16_t* __restrict__ feats, const uint32_t* __restrict__ keys,
                           const uint32_t* __restrict__ rows, const uint32_t* __restrict__ starts,
                           const uint32_t* __restrict__ nseg, const uint32_t* __restrict__ off,
                           const float* __restrict__ prior_p, float pw, CatOrder o,
                           uint32_t* __restrict__ tab_keys, float* __restrict__ tab_vals,
                           uint32_t* __restrict__ tab_len) {
  const uint32_t c = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t S = nseg[c];
  if (s >= S) return;
  const size_t base = (size_t)c * n;
  const uint32_t begin = starts[base + s], end = s + 1 < S ? starts[base + s + 1] : n;
  const uint32_t feat = feats[c];
  const float prior = *prior_p;
  const float wp = __fmul_rn(pw, prior);
  auto smooth = [&](float sum, uint32_t cnt) {
    return __fdiv_rn(__fadd_rn(sum, wp), __fadd_rn(__uint2float_rn(cnt), pw));
  };
  float total = 0.0f;
  uint32_t count = 0;
  if (!o.cv) {
    for (uint32_t i = begin; i < end; ++i) {
      const uint32_t row = rows[base + i];
      float* xp = X + (size_t)row * f + feat;
      if (isnan(*xp)) {
        *xp = prior;
        continue;
      }
      *xp = count ? smooth(total, count) : prior;
      total = __fadd_rn(total, y[row]);
      ++count;
    }
  } else {
    float fs[CAT_MAX_FOLDS];
    uint32_t fc[CAT_MAX_FOLDS];
    for (uint32_t q = 0; q < o.folds; ++q) {
      fs[q] = 0.0f;
      fc[q] = 0;
    }
    for (uint32_t i = begin; i < end; ++i) {
      const uint32_t row = rows[base + i];
      if (isnan(X[(size_t)row * f + feat])) continue;
      const uint32_t fd = fold_of(row, o);
      fs[fd] = __fadd_rn(fs[fd], y[row]);
      ++fc[fd];
    }
    for (uint32_t i = begin; i < end; ++i) {
      const uint32_t row = rows[base + i];
      float* xp = X + (size_t)row * f + feat;
      if (isnan(*xp)) {
        *xp = prior;
        continue;
      }
      const uint32_t fd = fold_of(row, o);
      float sum = 0.0f;
      uint32_t cnt = 0;
      for (uint32_t q = 0; q < o.folds; ++q) {
        if (q == fd) continue;
        sum = __fadd_rn(sum, fs[q]);
        cnt += fc[q];
      }
      *xp = smooth(sum, cnt);
    }
    for (uint32_t q = 0; q < o.folds; ++q) {
      total = __fadd_rn(total, fs[q]);
      count += fc[q];
    }
  }
  const uint32_t at = off[c] + s;
  tab_keys[at] = keys[base + begin];
  tab_vals[at] = count ? smooth(total, count) : prior;
  if (s == S - 1) tab_len[c] = count ? S : S - 1;  // a last segment of NaN rows only is no category
}

// ---- exact labels: every partial sum is an integer below 2^24 in magnitude,
// so float adds them exactly in any order and the running sums can be
// prefix sums (ordered) or atomic fold totals (cross-validated), one thread
// per row instead of one per category.  Class ids always are; the sequential
// walk above serves every other label.

// flags[0] |= 1 if some label is not an integer of magnitude <= 2^24;
// sum[0] += sum |label|, sum[1] += sum label (two's complement), as integers.
// With exact labels the latter is the reference's float sum of the labels.
__global__ void k_label_exact(const float* __restrict__ y, uint32_t n, unsigned long long* __restrict__ sum,
                              uint32_t* __restrict__ flags) {
  unsigned long long s = 0, t = 0;
  uint32_t bad = 0;
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float w = y[i], v = fabsf(w);
    if (!(v <= 16777216.0f) || v != truncf(v)) {  // NaN fails the first test
      bad = 1;
    } else {
      s += (unsigned long long)v;
      t += (unsigned long long)(long long)w;
    }
  }
  for (int o = 16; o; o >>= 1) {
    s += __shfl_xor_sync(0xffffffffu, s, o);
    t += __shfl_xor_sync(0xffffffffu, t, o);
    bad |= __shfl_xor_sync(0xffffffffu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    if (s) atomicAdd(&sum[0], s);
    if (t) atomicAdd(&sum[1], t);
    if (bad) atomicOr(flags, 1u);
  }
}

// Per tile of sorted positions: sum of the labels and count of the rows that
// are not NaN.
__global__ void k_cat_tile_sums(const float* __restrict__ X, const float* __restrict__ y, uint32_t n, uint32_t f,
                                const uint16_t* __restrict__ feats, const uint32_t* __restrict__ rows,
                                uint32_t n_tiles, long long* __restrict__ tsum, uint32_t* __restrict__ tcnt) {
  __shared__ long long ws[RS_THREADS / 32];
  __shared__ uint32_t wc[RS_THREADS / 32];
  const uint32_t c = blockIdx.y, tile = blockIdx.x, feat = feats[c];
  long long sm = 0;
  uint32_t k = 0;
  for (int it = 0; it < RS_ITEMS; ++it) {
    const uint32_t idx = tile * RS_TILE + it * RS_THREADS + threadIdx.x;
    if (idx >= n) break;
    const uint32_t row = rows[(size_t)c * n + idx];
    if (!isnan(X[(size_t)row * f + feat])) {
      sm += (long long)y[row];
      ++k;
    }
  }
  for (int o = 16; o; o >>= 1) {
    sm += __shfl_xor_sync(0xffffffffu, sm, o);
    k += __shfl_xor_sync(0xffffffffu, k, o);
  }
  if ((threadIdx.x & 31) == 0) {
    ws[threadIdx.x >> 5] = sm;
    wc[threadIdx.x >> 5] = k;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    long long a = 0;
    uint32_t b = 0;
    for (int w = 0; w < RS_THREADS / 32; ++w) {
      a += ws[w];
      b += wc[w];
    }
    tsum[(size_t)c * n_tiles + tile] = a;
    tcnt[(size_t)c * n_tiles + tile] = b;
  }
}

// Exclusive scan of the tile totals of each column, in place (one thread per
// column: a few thousand tiles).
__global__ void k_cat_tile_scan(long long* __restrict__ tsum, uint32_t* __restrict__ tcnt, uint32_t n_tiles) {
  if (threadIdx.x != 0) return;
  long long a = 0;
  uint32_t b = 0;
  long long* ts = tsum + (size_t)blockIdx.x * n_tiles;
  uint32_t* tc = tcnt + (size_t)blockIdx.x * n_tiles;
  for (uint32_t t = 0; t < n_tiles; ++t) {
    const long long x = ts[t];
    const uint32_t y = tc[t];
    ts[t] = a;
    tc[t] = b;
    a += x;
    b += y;
  }
}

// P[c][i] / C[c][i]: label sum / row count of the non-NaN rows at sorted
// positions before i (i = 0 .. n).
__global__ void k_cat_prefix(const float* __restrict__ X, const float* __restrict__ y, uint32_t n, uint32_t f,
                             const uint16_t* __restrict__ feats, const uint32_t* __restrict__ rows, uint32_t n_tiles,
                             const long long* __restrict__ toff, const uint32_t* __restrict__ tcoff,
                             long long* __restrict__ P, uint32_t* __restrict__ C) {
  __shared__ long long ws[RS_THREADS / 32];
  __shared__ uint32_t wc[RS_THREADS / 32];
  __shared__ long long run_s;
  __shared__ uint32_t run_c;
  const uint32_t c = blockIdx.y, tile = blockIdx.x, feat = feats[c];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const size_t base = (size_t)c * (n + 1);
  if (threadIdx.x == 0) {
    run_s = toff[(size_t)c * n_tiles + tile];
    run_c = tcoff[(size_t)c * n_tiles + tile];
  }
  __syncthreads();
  for (int it = 0; it < RS_ITEMS; ++it) {
    const uint32_t idx = tile * RS_TILE + it * RS_THREADS + threadIdx.x;
    long long v = 0;
    uint32_t k = 0;
    if (idx < n) {
      const uint32_t row = rows[(size_t)c * n + idx];
      if (!isnan(X[(size_t)row * f + feat])) {
        v = (long long)y[row];
        k = 1;
      }
    }
    long long xs = v;
    uint32_t xc = k;
    for (int o = 1; o < 32; o <<= 1) {
      const long long a = __shfl_up_sync(0xffffffffu, xs, o);
      const uint32_t b = __shfl_up_sync(0xffffffffu, xc, o);
      if (lane >= o) {
        xs += a;
        xc += b;
      }
    }
    if (lane == 31) {
      ws[warp] = xs;
      wc[warp] = xc;
    }
    __syncthreads();
    long long bs = run_s;
    uint32_t bc = run_c;
    for (int w = 0; w < warp; ++w) {
      bs += ws[w];
      bc += wc[w];
    }
    if (idx < n) {
      P[base + idx] = bs + xs - v;
      C[base + idx] = bc + xc - k;
      if (idx == n - 1) {
        P[base + n] = bs + xs;
        C[base + n] = bc + xc;
      }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      for (int w = 0; w < RS_THREADS / 32; ++w) {
        run_s += ws[w];
        run_c += wc[w];
      }
    }
    __syncthreads();
  }
}

// Ordered method, one thread per sorted position: the rows of its category
// before it are the positions [segment start, i).
__global__ void k_cat_rows_ordered(float* __restrict__ X, uint32_t n, uint32_t f,
                                   const uint16_t* __restrict__ feats, const uint32_t* __restrict__ rows,
                                   const uint32_t* __restrict__ segid, const uint32_t* __restrict__ starts,
                                   const long long* __restrict__ P, const uint32_t* __restrict__ C,
                                   const float* __restrict__ prior_p, float pw) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (i >= n) return;
  const size_t base = (size_t)c * n, pb = (size_t)c * (n + 1);
  const uint32_t row = rows[base + i];
  float* xp = X + (size_t)row * f + feats[c];
  const float prior = *prior_p;
  if (isnan(*xp)) {
    *xp = prior;
    return;
  }
  const uint32_t b = starts[base + segid[base + i]];
  const uint32_t k = C[pb + i] - C[pb + b];
  const float sum = __ll2float_rn(P[pb + i] - P[pb + b]);  // exact: |sum| <= 2^24
  *xp = k ? __fdiv_rn(__fadd_rn(sum, __fmul_rn(pw, prior)), __fadd_rn(__uint2float_rn(k), pw)) : prior;
}

// Table entries of the ordered method from the prefix sums.
__global__ void k_cat_table_prefix(const uint32_t* __restrict__ keys, uint32_t n, const uint32_t* __restrict__ starts,
                                   const uint32_t* __restrict__ nseg, const uint32_t* __restrict__ off,
                                   const long long* __restrict__ P, const uint32_t* __restrict__ C,
                                   const float* __restrict__ prior_p, float pw, uint32_t* __restrict__ tab_keys,
                                   float* __restrict__ tab_vals, uint32_t* __restrict__ tab_len) {
  const uint32_t c = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t S = nseg[c];
  if (s >= S) return;
  const size_t base = (size_t)c * n, pb = (size_t)c * (n + 1);
  const uint32_t b = starts[base + s], e = s + 1 < S ? starts[base + s + 1] : n;
  const uint32_t k = C[pb + e] - C[pb + b];
  const float prior = *prior_p;
  const float sum = __ll2float_rn(P[pb + e] - P[pb + b]);
  const uint32_t at = off[c] + s;
  tab_keys[at] = keys[base + b];
  tab_vals[at] = k ? __fdiv_rn(__fadd_rn(sum, __fmul_rn(pw, prior)), __fadd_rn(__uint2float_rn(k), pw)) : prior;
  if (s == S - 1) tab_len[c] = k ? S : S - 1;
}

// Cross-validated method: per (category, fold) label sums and counts by
// atomics (integers: exact in any order).
__global__ void k_cat_fold_sums(const float* __restrict__ X, const float* __restrict__ y, uint32_t n, uint32_t f,
                                const uint16_t* __restrict__ feats, const uint32_t* __restrict__ rows,
                                const uint32_t* __restrict__ segid, const uint32_t* __restrict__ off, CatOrder o,
                                unsigned long long* __restrict__ fsum, uint32_t* __restrict__ fcnt) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (i >= n) return;
  const size_t base = (size_t)c * n;
  const uint32_t row = rows[base + i];
  if (isnan(X[(size_t)row * f + feats[c]])) return;
  const size_t at = ((size_t)off[c] + segid[base + i]) * o.folds + fold_of(row, o);
  atomicAdd(&fsum[at], (unsigned long long)(long long)y[row]);
  atomicAdd(&fcnt[at], 1u);
}

__global__ void k_cat_rows_cv(float* __restrict__ X, uint32_t n, uint32_t f, const uint16_t* __restrict__ feats,
                              const uint32_t* __restrict__ rows, const uint32_t* __restrict__ segid,
                              const uint32_t* __restrict__ off, CatOrder o,
                              const unsigned long long* __restrict__ fsum, const uint32_t* __restrict__ fcnt,
                              const float* __restrict__ prior_p, float pw) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (i >= n) return;
  const size_t base = (size_t)c * n;
  const uint32_t row = rows[base + i];
  float* xp = X + (size_t)row * f + feats[c];
  const float prior = *prior_p;
  if (isnan(*xp)) {
    *xp = prior;
    return;
  }
  const size_t at = ((size_t)off[c] + segid[base + i]) * o.folds;
  const uint32_t fd = fold_of(row, o);
  long long sm = 0;
  uint32_t k = 0;
  for (uint32_t q = 0; q < o.folds; ++q) {
    if (q == fd) continue;
    sm += (long long)fsum[at + q];
    k += fcnt[at + q];
  }
  *xp = __fdiv_rn(__fadd_rn(__ll2float_rn(sm), __fmul_rn(pw, prior)), __fadd_rn(__uint2float_rn(k), pw));
}

__global__ void k_cat_table_cv(const uint32_t* __restrict__ keys, uint32_t n, const uint32_t* __restrict__ starts,
                               const uint32_t* __restrict__ nseg, const uint32_t* __restrict__ off, CatOrder o,
                               const unsigned long long* __restrict__ fsum, const uint32_t* __restrict__ fcnt,
                               const float* __restrict__ prior_p, float pw, uint32_t* __restrict__ tab_keys,
                               float* __restrict__ tab_vals, uint32_t* __restrict__ tab_len) {
  const uint32_t c = blockIdx.y, s = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t S = nseg[c];
  if (s >= S) return;
  const size_t at = ((size_t)off[c] + s) * o.folds;
  long long sm = 0;
  uint32_t k = 0;
  for (uint32_t q = 0; q < o.folds; ++q) {
    sm += (long long)fsum[at + q];
    k += fcnt[at + q];
  }
  const float prior = *prior_p;
  const uint32_t t = off[c] + s;
  tab_keys[t] = keys[(size_t)c * n + starts[(size_t)c * n + s]];
  tab_vals[t] = k ? __fdiv_rn(__fadd_rn(__ll2float_rn(sm), __fmul_rn(pw, prior)), __fadd_rn(__uint2float_rn(k), pw))
                  : prior;
  if (s == S - 1) tab_len[c] = k ? S : S - 1;
}

// Dataset::apply_bins' categorical branch (src/core/dataset.cpp:362-372):
// a row's category -> the reference's global encoding (binary search of the
// sorted table), 0.5 for a category it never saw (encode_category's default,
// include/turbocat/dataset.hpp:218-226); NaN stays NaN (bin 255).
__global__ void k_cat_lookup(float* __restrict__ X, uint32_t n, uint32_t f, const uint16_t* __restrict__ feats,
                             const uint32_t* __restrict__ off, const uint32_t* __restrict__ len,
                             const uint32_t* __restrict__ tkeys, const float* __restrict__ tvals) {
  const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (r >= n) return;
  float* xp = X + (size_t)r * f + feats[c];
  const float x = *xp;
  if (isnan(x)) return;
  const uint32_t k = category_of(x);
  const uint32_t b = off[c], e = off[c] + len[c];
  uint32_t lo = b, hi = e;
  while (lo < hi) {
    const uint32_t mid = lo + (hi - lo) / 2;
    if (tkeys[mid] < k) lo = mid + 1; else hi = mid;
  }
  *xp = (lo < e && tkeys[lo] == k) ? tvals[lo] : 0.5f;
}

}  // namespace

tc_status quantize(tc_dataset* ds, int max_bins, int compat_u8) {
  tc_ctx* ctx = ds->ctx;
  const uint32_t n = ds->n, f = ds->f;
  cudaStream_t st = ctx->stream;
  const uint32_t n_tiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  const uint8_t* ts = ds->h_cat_feats.empty() ? nullptr : ds->ts.p;
  DevBuf<uint32_t> ka, kb, counts, tcnt, U;
  TC_TRY(ka.alloc(ctx, (size_t)n * f, "sort keys"));
  TC_TRY(kb.alloc(ctx, (size_t)n * f, "sort keys (alt)"));
  TC_TRY(counts.alloc(ctx, (size_t)f * 256 * n_tiles, "radix counts"));
  TC_TRY(tcnt.alloc(ctx, (size_t)f * n_tiles, "unique tile counts"));
  TC_TRY(U.alloc(ctx, f, "unique counts"));
  TC_TRY(ds->edges.alloc(ctx, (size_t)f * kSlots, "bin edges"));
  TC_TRY(ds->n_edges.alloc(ctx, f, "edge counts"));
  TC_TRY(ds->nan_any.alloc(ctx, f, "NaN flags"));
  TC_CUDA(ctx, cudaMemsetAsync(ds->nan_any.p, 0, ds->nan_any.bytes(), st));
  TC_TRY(ds->bins_t.alloc(ctx, (size_t)(ds->groups - 1) * ds->gstride + (size_t)ds->wlast * ds->nt,
                          "feature-group bin tiles"));
  TC_TRY(ds->bins_cm.alloc(ctx, (size_t)f * ds->np, "column-major bins"));
  TC_CUDA(ctx, cudaMemsetAsync(ds->edges.p, 0, ds->edges.bytes(), st));

  if (n > 0) {
    dim3 tg((n + 31) / 32, (f + 31) / 32);
    k_make_keys<<<tg, dim3(32, 8), 0, st>>>(ds->X.p, n, f, ka.p);
    uint32_t* src = ka.p;
    uint32_t* dst = kb.p;
    for (int shift = 0; shift < 32; shift += 8) {
      k_radix_count<<<dim3(n_tiles, f), RS_THREADS, 0, st>>>(src, n, n_tiles, shift, counts.p);
      k_segment_scan<<<f, 1024, 0, st>>>(counts.p, 256 * n_tiles, nullptr);
      k_radix_scatter<<<dim3(n_tiles, f), RS_THREADS, 0, st>>>(src, dst, n, n_tiles, shift, counts.p);
      std::swap(src, dst);
    }
    k_unique_count<<<dim3(n_tiles, f), RS_THREADS, 0, st>>>(src, n, n_tiles, tcnt.p);
    k_segment_scan<<<f, 1024, 0, st>>>(tcnt.p, n_tiles, U.p);
    k_unique_pick<<<dim3(n_tiles, f), RS_THREADS, 0, st>>>(src, n, n_tiles, tcnt.p, U.p, max_bins,
                                                            compat_u8, ts, ds->edges.p);
  } else {
    TC_CUDA(ctx, cudaMemsetAsync(U.p, 0, U.bytes(), st));
  }
  k_edge_meta<<<(f + 127) / 128, 128, 0, st>>>(U.p, f, max_bins, compat_u8, ts, ds->edges.p, ds->n_edges.p);
  TC_CUDA(ctx, cudaMemsetAsync(ds->bins_t.p, 0, ds->bins_t.bytes(), st));
  if (n > 0) {
    dim3 ag((n + AB_ROWS - 1) / AB_ROWS, ds->groups);
    k_assign_bins<<<ag, 256, 0, st>>>(ds->X.p, n, f, ds->edges.p, ds->n_edges.p, ts, ds->bins_t.p,
                                      ds->gstride, ds->nt, ds->wlast, ds->bins_cm.p, ds->np, ds->nan_any.p);
  }
  TC_CUDA(ctx, cudaGetLastError());
  // host copy of the edges for model export / thresholds
  std::vector<float> e((size_t)f * kSlots);
  ds->h_n_edges.resize(f);
  TC_CUDA(ctx, cudaMemcpyAsync(e.data(), ds->edges.p, e.size() * sizeof(float), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaMemcpyAsync(ds->h_n_edges.data(), ds->n_edges.p, f * sizeof(uint16_t),
                               cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  ds->h_edges.assign((size_t)f * 255, 0.0f);
  for (uint32_t j = 0; j < f; ++j)
    for (uint32_t k = 0; k < ds->h_n_edges[j] && k < 255; ++k) ds->h_edges[(size_t)j * 255 + k] = e[(size_t)j * kSlots + k];
  ds->quantized = true;
  ds->max_bins = max_bins;
  return TC_OK;
}

tc_status apply_bins(tc_dataset* ds, const tc_dataset* ref) {
  tc_ctx* ctx = ds->ctx;
  if (ref->ctx != ctx) return ctx->fail(TC_ERR_INVALID_ARG, "the reference dataset belongs to another context");
  if (!ref->quantized) return ctx->fail(TC_ERR_NOT_FITTED, "reference dataset not quantized");
  if (ref->f != ds->f)
    return ctx->fail(TC_ERR_INVALID_ARG, "feature counts differ (%u vs reference %u)", ds->f, ref->f);
  if (ref == ds) return TC_OK;  // already binned with its own edges
  cudaStream_t st = ctx->stream;
  const uint32_t n = ds->n, f = ds->f;
  if (!ref->h_cat_feats.empty() && ds->encoded_by != ref->id) {
    if (!ds->h_cat_feats.empty() || ds->encoded_by)
      return ctx->fail(TC_ERR_INVALID_ARG, "the dataset's categorical columns are already encoded");
    const uint32_t nc = (uint32_t)ref->h_cat_feats.size();
    if (n > 0) {
      k_cat_lookup<<<dim3((n + CAT_THREADS - 1) / CAT_THREADS, nc), CAT_THREADS, 0, st>>>(
          ds->X.p, n, f, ref->cat_feats.p, ref->cat_off.p, ref->cat_len.p, ref->cat_keys.p, ref->cat_vals.p);
      TC_CUDA(ctx, cudaGetLastError());
    }
    ds->encoded_by = ref->id;
  }
  TC_TRY(ds->edges.alloc(ctx, (size_t)f * kSlots, "bin edges"));
  TC_TRY(ds->n_edges.alloc(ctx, f, "edge counts"));
  TC_TRY(ds->nan_any.alloc(ctx, f, "NaN flags"));
  TC_TRY(ds->bins_t.alloc(ctx, (size_t)(ds->groups - 1) * ds->gstride + (size_t)ds->wlast * ds->nt,
                          "feature-group bin tiles"));
  TC_TRY(ds->bins_cm.alloc(ctx, (size_t)f * ds->np, "column-major bins"));
  TC_CUDA(ctx, cudaMemcpyAsync(ds->edges.p, ref->edges.p, ds->edges.bytes(), cudaMemcpyDeviceToDevice, st));
  TC_CUDA(ctx, cudaMemcpyAsync(ds->n_edges.p, ref->n_edges.p, ds->n_edges.bytes(), cudaMemcpyDeviceToDevice, st));
  TC_CUDA(ctx, cudaMemsetAsync(ds->nan_any.p, 0, ds->nan_any.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(ds->bins_t.p, 0, ds->bins_t.bytes(), st));
  if (n > 0) {
    dim3 ag((n + AB_ROWS - 1) / AB_ROWS, ds->groups);
    k_assign_bins<<<ag, 256, 0, st>>>(ds->X.p, n, f, ds->edges.p, ds->n_edges.p, nullptr, ds->bins_t.p,
                                      ds->gstride, ds->nt, ds->wlast, ds->bins_cm.p, ds->np, ds->nan_any.p);
    TC_CUDA(ctx, cudaGetLastError());
  }
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  ds->h_edges = ref->h_edges;
  ds->h_n_edges = ref->h_n_edges;
  ds->quantized = true;
  ds->max_bins = ref->max_bins;
  return TC_OK;
}

namespace {
uint64_t splitmix64(uint64_t& x) {  // S. Vigna's SplitMix64 step
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
}  // namespace

tc_status encode_categorical(tc_dataset* ds, const uint16_t* feats, uint16_t nc, const tc_cat_params* p,
                             const uint32_t* order) {
  tc_ctx* ctx = ds->ctx;
  const uint32_t n = ds->n, f = ds->f;
  if (nc == 0) return TC_OK;
  if (!feats || !p) return ctx->fail(TC_ERR_INVALID_ARG, "features and parameters are required");
  if (ds->quantized) return ctx->fail(TC_ERR_INVALID_ARG, "encode the categorical columns before tc_quantize");
  if (!ds->h_cat_feats.empty() || ds->encoded_by)
    return ctx->fail(TC_ERR_INVALID_ARG, "the dataset's categorical columns are already encoded");
  if (n == 0 || ds->y.n < n) return ctx->fail(TC_ERR_INVALID_ARG, "target statistics need rows and labels");
  if (p->method != TC_CAT_ORDERED && p->method != TC_CAT_CV)
    return ctx->fail(TC_ERR_INVALID_ARG, "unknown target-statistics method %d", p->method);
  const bool cv = p->method == TC_CAT_CV;
  if (cv && (p->cv_folds < 1 || p->cv_folds > CAT_MAX_FOLDS))
    return ctx->fail(TC_ERR_INVALID_ARG, "cv_folds must be in [1, %d]", CAT_MAX_FOLDS);
  if (!std::isfinite(p->prior_weight)) return ctx->fail(TC_ERR_INVALID_ARG, "prior_weight must be finite");
  std::vector<uint8_t> seen(f, 0);
  for (uint16_t c = 0; c < nc; ++c) {
    if (feats[c] >= f) return ctx->fail(TC_ERR_INVALID_ARG, "categorical feature %u out of range", feats[c]);
    if (seen[feats[c]]++) return ctx->fail(TC_ERR_INVALID_ARG, "categorical feature %u listed twice", feats[c]);
  }
  if (order) {  // checked here: the kernels index rows by it
    if (cv) {
      for (uint32_t i = 0; i < n; ++i)
        if (order[i] >= (uint32_t)p->cv_folds) return ctx->fail(TC_ERR_INVALID_ARG, "fold %u of row %u", order[i], i);
    } else {
      std::vector<uint8_t> hit(n, 0);
      for (uint32_t i = 0; i < n; ++i)
        if (order[i] >= n || hit[order[i]]++) return ctx->fail(TC_ERR_INVALID_ARG, "order is not a permutation");
    }
  }
  cudaStream_t st = ctx->stream;
  const uint32_t n_tiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
  DevBuf<uint32_t> ka, kb, ra, rb, counts, tcnt, nseg, starts, segid, given, lab_flag;
  DevBuf<unsigned long long> lab_sum;
  DevBuf<float> prior;
  TC_TRY(ka.alloc(ctx, (size_t)nc * n, "category keys"));
  TC_TRY(kb.alloc(ctx, (size_t)nc * n, "category keys (alt)"));
  TC_TRY(ra.alloc(ctx, (size_t)nc * n, "category rows"));
  TC_TRY(rb.alloc(ctx, (size_t)nc * n, "category rows (alt)"));
  TC_TRY(counts.alloc(ctx, (size_t)nc * 256 * n_tiles, "radix counts"));
  TC_TRY(tcnt.alloc(ctx, (size_t)nc * n_tiles, "segment tile counts"));
  TC_TRY(nseg.alloc(ctx, nc, "segment counts"));
  TC_TRY(starts.alloc(ctx, (size_t)nc * n, "segment starts"));
  TC_TRY(segid.alloc(ctx, (size_t)nc * n, "segment of each position"));
  TC_TRY(prior.alloc(ctx, 1, "label prior"));
  TC_TRY(lab_sum.alloc(ctx, 2, "label sums"));
  TC_TRY(lab_flag.alloc(ctx, 1, "label flags"));
  TC_TRY(ds->cat_feats.alloc(ctx, nc, "categorical features"));
  TC_TRY(ds->cat_off.alloc(ctx, nc, "category table offsets"));
  TC_TRY(ds->cat_len.alloc(ctx, nc, "category table lengths"));
  TC_TRY(ds->ts.alloc(ctx, f, "target-statistics flags"));
  CatOrder o{};
  uint64_t sm = p->seed;
  for (int i = 0; i < 4; ++i) o.key[i] = (uint32_t)splitmix64(sm);
  o.half = 1;
  while ((1ull << (2 * o.half)) < n) ++o.half;
  o.folds = cv ? (uint32_t)p->cv_folds : 1u;
  o.cv = cv ? 1 : 0;
  if (order) {
    TC_TRY(given.alloc(ctx, n, "given order"));
    TC_CUDA(ctx, cudaMemcpyAsync(given.p, order, (size_t)n * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    o.given = given.p;
  }
  TC_CUDA(ctx, cudaMemcpyAsync(ds->cat_feats.p, feats, nc * sizeof(uint16_t), cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaMemsetAsync(lab_sum.p, 0, lab_sum.bytes(), st));
  TC_CUDA(ctx, cudaMemsetAsync(lab_flag.p, 0, sizeof(uint32_t), st));
  k_label_exact<<<std::min<uint32_t>((n + 255) / 256, 4 * (uint32_t)ctx->sm_count), 256, 0, st>>>(ds->y.p, n, lab_sum.p,
                                                                                             lab_flag.p);
  k_cat_keys<<<dim3((n + CAT_THREADS - 1) / CAT_THREADS, nc), CAT_THREADS, 0, st>>>(ds->X.p, n, f,
                                                                                   ds->cat_feats.p, o, ka.p, ra.p);
  uint32_t *ks = ka.p, *kd = kb.p, *rs = ra.p, *rd = rb.p;
  for (int shift = 0; shift < 32; shift += 8) {
    k_radix_count<<<dim3(n_tiles, nc), RS_THREADS, 0, st>>>(ks, n, n_tiles, shift, counts.p);
    k_segment_scan<<<nc, 1024, 0, st>>>(counts.p, 256 * n_tiles, nullptr);
    k_radix_scatter<<<dim3(n_tiles, nc), RS_THREADS, 0, st>>>(ks, kd, n, n_tiles, shift, counts.p, rs, rd);
    std::swap(ks, kd);
    std::swap(rs, rd);
  }
  k_seg_count<<<dim3(n_tiles, nc), RS_THREADS, 0, st>>>(ks, n, n_tiles, tcnt.p);
  k_segment_scan<<<nc, 1024, 0, st>>>(tcnt.p, n_tiles, nseg.p);
  k_seg_starts<<<dim3(n_tiles, nc), RS_THREADS, 0, st>>>(ks, n, n_tiles, tcnt.p, starts.p, segid.p);
  TC_CUDA(ctx, cudaGetLastError());
  std::vector<uint32_t> S(nc);
  unsigned long long h_lab_sum[2] = {0, 0};
  uint32_t h_lab_flag = 1;
  TC_CUDA(ctx, cudaMemcpyAsync(S.data(), nseg.p, nc * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaMemcpyAsync(h_lab_sum, lab_sum.p, sizeof(h_lab_sum), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaMemcpyAsync(&h_lab_flag, lab_flag.p, sizeof(h_lab_flag), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  // integer labels whose magnitudes sum to at most 2^24: every float partial
  // sum is exact, so the sums need not be sequential
  const bool exact = h_lab_flag == 0 && h_lab_sum[0] <= (1ull << 24);
  // the prior, std::accumulate(labels, 0.0f) / n: with exact labels the float
  // sum is the integer sum (converted exactly) and the division is done here
  // in float; otherwise one device thread adds the labels in row order
  const float h_prior = exact ? (float)(long long)h_lab_sum[1] / (float)n : 0.0f;
  if (exact) TC_CUDA(ctx, cudaMemcpyAsync(prior.p, &h_prior, sizeof(float), cudaMemcpyHostToDevice, st));
  else k_label_prior<<<1, 1024, 0, st>>>(ds->y.p, n, prior.p);
  ds->h_cat_off.assign(nc, 0);
  size_t total = 0;
  uint32_t smax = 0;
  for (uint16_t c = 0; c < nc; ++c) {
    ds->h_cat_off[c] = (uint32_t)total;
    total += S[c];
    smax = std::max(smax, S[c]);
  }
  TC_TRY(ds->cat_keys.alloc(ctx, total, "category table keys"));
  TC_TRY(ds->cat_vals.alloc(ctx, total, "category table values"));
  TC_CUDA(ctx, cudaMemcpyAsync(ds->cat_off.p, ds->h_cat_off.data(), nc * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
  const dim3 rg((n + CAT_THREADS - 1) / CAT_THREADS, nc), sg((smax + 127) / 128, nc);
  const float pw = p->prior_weight;
  if (!exact) {
    k_cat_walk<<<sg, 128, 0, st>>>(ds->y.p, ds->X.p, n, f, ds->cat_feats.p, ks, rs, starts.p, nseg.p, ds->cat_off.p,
                                   prior.p, pw, o, ds->cat_keys.p, ds->cat_vals.p, ds->cat_len.p);
  } else if (!cv) {
    DevBuf<long long> tsum, P;
    DevBuf<uint32_t> tcnt2, Cn;
    TC_TRY(tsum.alloc(ctx, (size_t)nc * n_tiles, "tile label sums"));
    TC_TRY(tcnt2.alloc(ctx, (size_t)nc * n_tiles, "tile row counts"));
    TC_TRY(P.alloc(ctx, (size_t)nc * (n + 1), "label prefix sums"));
    TC_TRY(Cn.alloc(ctx, (size_t)nc * (n + 1), "row prefix counts"));
    k_cat_tile_sums<<<dim3(n_tiles, nc), RS_THREADS, 0, st>>>(ds->X.p, ds->y.p, n, f, ds->cat_feats.p, rs, n_tiles,
                                                              tsum.p, tcnt2.p);
    k_cat_tile_scan<<<nc, 32, 0, st>>>(tsum.p, tcnt2.p, n_tiles);
    k_cat_prefix<<<dim3(n_tiles, nc), RS_THREADS, 0, st>>>(ds->X.p, ds->y.p, n, f, ds->cat_feats.p, rs, n_tiles,
                                                           tsum.p, tcnt2.p, P.p, Cn.p);
    k_cat_table_prefix<<<sg, 128, 0, st>>>(ks, n, starts.p, nseg.p, ds->cat_off.p, P.p, Cn.p, prior.p, pw,
                                           ds->cat_keys.p, ds->cat_vals.p, ds->cat_len.p);
    k_cat_rows_ordered<<<rg, CAT_THREADS, 0, st>>>(ds->X.p, n, f, ds->cat_feats.p, rs, segid.p, starts.p, P.p, Cn.p,
                                                   prior.p, pw);
    TC_CUDA(ctx, cudaGetLastError());
    TC_CUDA(ctx, cudaStreamSynchronize(st));  // before the scratch buffers go
  } else {
    DevBuf<unsigned long long> fsum;
    DevBuf<uint32_t> fcnt;
    TC_TRY(fsum.alloc(ctx, total * o.folds, "fold label sums"));
    TC_TRY(fcnt.alloc(ctx, total * o.folds, "fold row counts"));
    TC_CUDA(ctx, cudaMemsetAsync(fsum.p, 0, fsum.bytes(), st));
    TC_CUDA(ctx, cudaMemsetAsync(fcnt.p, 0, fcnt.bytes(), st));
    k_cat_fold_sums<<<rg, CAT_THREADS, 0, st>>>(ds->X.p, ds->y.p, n, f, ds->cat_feats.p, rs, segid.p, ds->cat_off.p, o,
                                                fsum.p, fcnt.p);
    k_cat_table_cv<<<sg, 128, 0, st>>>(ks, n, starts.p, nseg.p, ds->cat_off.p, o, fsum.p, fcnt.p, prior.p, pw,
                                       ds->cat_keys.p, ds->cat_vals.p, ds->cat_len.p);
    k_cat_rows_cv<<<rg, CAT_THREADS, 0, st>>>(ds->X.p, n, f, ds->cat_feats.p, rs, segid.p, ds->cat_off.p, o, fsum.p,
                                              fcnt.p, prior.p, pw);
    TC_CUDA(ctx, cudaGetLastError());
    TC_CUDA(ctx, cudaStreamSynchronize(st));
  }
  TC_CUDA(ctx, cudaGetLastError());
  ds->h_cat_len.assign(nc, 0);
  TC_CUDA(ctx, cudaMemcpyAsync(ds->h_cat_len.data(), ds->cat_len.p, nc * sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
  TC_CUDA(ctx, cudaMemcpyAsync(&ds->cat_prior, prior.p, sizeof(float), cudaMemcpyDeviceToHost, st));
  ds->h_ts.assign(f, 0);
  for (uint16_t c = 0; c < nc; ++c) ds->h_ts[feats[c]] = 1;
  TC_CUDA(ctx, cudaMemcpyAsync(ds->ts.p, ds->h_ts.data(), f, cudaMemcpyHostToDevice, st));
  TC_CUDA(ctx, cudaStreamSynchronize(st));  // the host vectors above are read by the copies
  ds->h_cat_feats.assign(feats, feats + nc);
  return TC_OK;
}

}  // namespace tc

namespace {

constexpr size_t kUpChunk = (size_t)128 << 20;  // bytes of one pinned staging chunk

// Host -> device copy of a large pageable buffer (a page-locked one is copied
// directly): chunks are copied into two
// pinned staging buffers by host threads (each a slice of the chunk) while
// the other buffer's chunk is on its way to the device, so the transfer runs
// at the link's rate instead of the driver's single-threaded pageable copy.
tc_status upload_staged(tc_ctx* ctx, void* dst, const void* src, size_t bytes, cudaStream_t st) {
  cudaPointerAttributes pa;
  bool pinned = false;
  if (cudaPointerGetAttributes(&pa, src) == cudaSuccess) pinned = pa.type == cudaMemoryTypeHost;
  else cudaGetLastError();
  if (pinned || bytes <= 2 * kUpChunk) {  // page-locked already: one DMA at the link's rate
    TC_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    return TC_OK;
  }
  for (int b = 0; b < 2; ++b) {
    if (!ctx->up_stage[b]) TC_CUDA(ctx, cudaHostAlloc(&ctx->up_stage[b], kUpChunk, cudaHostAllocDefault));
    if (!ctx->up_ev[b]) TC_CUDA(ctx, cudaEventCreateWithFlags(&ctx->up_ev[b], cudaEventDisableTiming));
  }
  const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
  const int nt = (int)std::min(16u, std::max(1u, hw / 2));
  const char* s = static_cast<const char*>(src);
  char* d = static_cast<char*>(dst);
  std::vector<std::thread> ts;
  for (size_t off = 0, b = 0; off < bytes; off += kUpChunk, b ^= 1) {
    const size_t len = std::min(kUpChunk, bytes - off);
    TC_CUDA(ctx, cudaEventSynchronize(ctx->up_ev[b]));  // this buffer's previous chunk has left
    char* stage = static_cast<char*>(ctx->up_stage[b]);
    ts.clear();
    size_t done_to = 0;  // bytes of the chunk copied on this thread when no helper thread could start
    try {
      for (int t = 0; t < nt; ++t) {
        const size_t a = len * t / nt, e = len * (t + 1) / nt;
        ts.emplace_back([=] { std::memcpy(stage + a, s + off + a, e - a); });
        done_to = e;
      }
    } catch (const std::exception&) {
      std::memcpy(stage + done_to, s + off + done_to, len - done_to);
    }
    for (auto& th : ts) th.join();
    TC_CUDA(ctx, cudaMemcpyAsync(d + off, stage, len, cudaMemcpyHostToDevice, st));
    TC_CUDA(ctx, cudaEventRecord(ctx->up_ev[b], st));
  }
  return TC_OK;
}

}  // namespace

extern "C" {

tc_status tc_dataset_upload(tc_ctx* ctx, const float* X, uint32_t n, uint16_t f, const float* y,
                            tc_dataset** out) {
  if (!ctx || !out || (!X && n > 0) || f == 0) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  *out = nullptr;
  cudaSetDevice(ctx->device);
  static std::atomic<uint64_t> next_id{1};
  tc_dataset* ds = new tc_dataset();
  ds->ctx = ctx;
  ds->id = next_id.fetch_add(1);
  ds->n = n;
  ds->f = f;
  ds->groups = (f + 31) / 32;
  ds->nt = (uint32_t)tc::round_up(n > 0 ? n : 1, 32);
  {
    const uint32_t last = f - 32 * (ds->groups - 1);  // features in the last group, 1 .. 32
    ds->wlast = last <= 4 ? 4 : (last <= 8 ? 8 : (last <= 16 ? 16 : 32));
  }
  ds->gstride = (uint64_t)32 * ds->nt;
  ds->np = (uint32_t)tc::round_up(n > 0 ? n : 1, 16);
  tc_status s = ds->X.alloc(ctx, (size_t)n * f, "training matrix");
  if (s == TC_OK && y) s = ds->y.alloc(ctx, n, "labels");
  if (s != TC_OK) {
    delete ds;
    return s;
  }
  cudaError_t e = cudaSuccess;
  if (n > 0 && upload_staged(ctx, ds->X.p, X, (size_t)n * f * sizeof(float), ctx->stream) != TC_OK) {
    delete ds;
    return TC_ERR_CUDA;
  }
  if (e == cudaSuccess && y && n > 0)
    e = cudaMemcpyAsync(ds->y.p, y, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, ctx->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
  if (e != cudaSuccess) {
    delete ds;
    return ctx->cuda_fail(e, "dataset upload");
  }
  *out = ds;
  return TC_OK;
}

void tc_dataset_destroy(tc_dataset* ds) {
  if (!ds) return;
  if (!ds->ctx) {
    delete ds;
    return;
  }
  std::lock_guard<std::recursive_mutex> train_lock(ds->ctx->train_mu);
  delete ds;
}

tc_status tc_quantize(tc_dataset* ds, uint16_t max_bins, int compat_uint8_count, float* edges_out,
                      uint16_t* n_edges_out) {
  if (!ds) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = ds->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  if (max_bins < 2 || max_bins > 255)
    return ctx->fail(TC_ERR_INVALID_ARG, "max_bins must be in [2, 255] (uint8 bins; got %u)", max_bins);
  cudaSetDevice(ctx->device);
  TC_TRY(tc::quantize(ds, max_bins, compat_uint8_count ? 1 : 0));
  if (edges_out) std::copy(ds->h_edges.begin(), ds->h_edges.end(), edges_out);
  if (n_edges_out) std::copy(ds->h_n_edges.begin(), ds->h_n_edges.end(), n_edges_out);
  return TC_OK;
}

tc_status tc_apply_bins(tc_dataset* ds, const tc_dataset* ref) {
  if (!ds || !ref) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = ds->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  return tc::apply_bins(ds, ref);
}

tc_status tc_dataset_bins(const tc_dataset* ds, uint8_t* bins_out) {
  if (!ds || !bins_out) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = ds->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  if (!ds->quantized) return ctx->fail(TC_ERR_NOT_FITTED, "dataset not quantized");
  cudaSetDevice(ctx->device);
  TC_CUDA(ctx, cudaMemcpy2DAsync(bins_out, ds->n, ds->bins_cm.p, ds->np, ds->n, ds->f,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

tc_status tc_dataset_features(const tc_dataset* ds, float* X_out) {
  if (!ds || (!X_out && ds->n)) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = ds->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  if (ds->n == 0) return TC_OK;
  TC_CUDA(ctx, cudaMemcpyAsync(X_out, ds->X.p, ds->X.bytes(), cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

tc_status tc_encode_categorical(tc_dataset* ds, const uint16_t* features, uint16_t n_cat,
                                const tc_cat_params* p, const uint32_t* order) {
  if (!ds) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = ds->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  return tc::encode_categorical(ds, features, n_cat, p, order);
}

tc_status tc_category_table(const tc_dataset* ds, uint16_t feature, uint32_t* keys, float* vals, uint32_t* len) {
  if (!ds || !len) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = ds->ctx;
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  size_t c = 0;
  while (c < ds->h_cat_feats.size() && ds->h_cat_feats[c] != feature) ++c;
  if (c == ds->h_cat_feats.size()) return ctx->fail(TC_ERR_INVALID_ARG, "feature %u is not an encoded column", feature);
  *len = ds->h_cat_len[c];
  if (!keys || !vals || *len == 0) return TC_OK;
  cudaSetDevice(ctx->device);
  const size_t at = ds->h_cat_off[c];
  TC_CUDA(ctx, cudaMemcpyAsync(keys, ds->cat_keys.p + at, *len * sizeof(uint32_t), cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaMemcpyAsync(vals, ds->cat_vals.p + at, *len * sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  TC_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TC_OK;
}

}  // extern "C"
