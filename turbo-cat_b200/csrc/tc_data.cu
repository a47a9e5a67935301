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
                                const uint32_t* __restrict__ offsets) {
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
    if (valid) ko[s_base[d] + s_w[warp][d] + rank] = key;
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
                              int max_bins, int compat_u8, float* __restrict__ edges) {
  __shared__ uint32_t warp_sums[RS_THREADS / 32];
  __shared__ uint32_t run_s;
  const uint32_t j = blockIdx.y, tile = blockIdx.x;
  const uint32_t* kj = keys + (size_t)j * n;
  const uint64_t U = U_[j];
  const uint64_t A = actual_bins((uint32_t)U, max_bins, compat_u8);
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
      const uint64_t b = (r * A + U - 1) / U;
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
                            float* __restrict__ edges, uint16_t* __restrict__ n_edges) {
  const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= f) return;
  const uint32_t U = U_[j];
  if (U == 0) {  // every value NaN: one edge {0.0f} (src/core/dataset.cpp:296-303)
    edges[(size_t)j * kSlots] = 0.0f;
    n_edges[j] = 1;
    return;
  }
  const uint32_t A = actual_bins(U, max_bins, compat_u8);
  n_edges[j] = (uint16_t)(A >= 2 ? A - 1 : 0);
}

constexpr int AB_ROWS = 256;

// bin = #edges <= x (upper_bound), NaN -> 255; writes both bin layouts.
// Block (row tile, group): 256 rows of the 32 features of group blockIdx.y.
__global__ void k_assign_bins(const float* __restrict__ X, uint32_t n, uint32_t f,
                              const float* __restrict__ edges, const uint16_t* __restrict__ n_edges,
                              uint8_t* __restrict__ bins_t, uint64_t gstride, uint32_t nt, uint32_t wlast,
                              uint8_t* __restrict__ bins_cm, uint32_t np, uint32_t* __restrict__ nan_any) {
  __shared__ float s_e[32][kSlots + 1];
  __shared__ int s_ne[32];
  __shared__ uint8_t s_b[32][AB_ROWS + 4];
  __shared__ int s_nan[32];
  const uint32_t j0 = blockIdx.y * 32, r0 = blockIdx.x * AB_ROWS;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
  for (int q = tid; q < 32 * kSlots; q += blockDim.x) {
    const int jj = q / kSlots, e = q % kSlots;
    s_e[jj][e] = (j0 + jj < f) ? edges[(size_t)(j0 + jj) * kSlots + e] : 0.0f;
  }
  if (tid < 32) {
    s_ne[tid] = (j0 + tid < f) ? (int)n_edges[j0 + tid] : 0;
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
        while (lo < hi) {
          const int mid = (lo + hi) >> 1;
          if (x < s_e[lane][mid]) hi = mid; else lo = mid + 1;
        }
        b = (uint8_t)lo;
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

}  // namespace

tc_status quantize(tc_dataset* ds, int max_bins, int compat_u8) {
  tc_ctx* ctx = ds->ctx;
  const uint32_t n = ds->n, f = ds->f;
  cudaStream_t st = ctx->stream;
  const uint32_t n_tiles = (uint32_t)((n + RS_TILE - 1) / RS_TILE);
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
                                                            compat_u8, ds->edges.p);
  } else {
    TC_CUDA(ctx, cudaMemsetAsync(U.p, 0, U.bytes(), st));
  }
  k_edge_meta<<<(f + 127) / 128, 128, 0, st>>>(U.p, f, max_bins, compat_u8, ds->edges.p, ds->n_edges.p);
  TC_CUDA(ctx, cudaMemsetAsync(ds->bins_t.p, 0, ds->bins_t.bytes(), st));
  if (n > 0) {
    dim3 ag((n + AB_ROWS - 1) / AB_ROWS, ds->groups);
    k_assign_bins<<<ag, 256, 0, st>>>(ds->X.p, n, f, ds->edges.p, ds->n_edges.p, ds->bins_t.p, ds->gstride,
                                      ds->nt, ds->wlast, ds->bins_cm.p, ds->np, ds->nan_any.p);
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
    k_assign_bins<<<ag, 256, 0, st>>>(ds->X.p, n, f, ds->edges.p, ds->n_edges.p, ds->bins_t.p, ds->gstride,
                                      ds->nt, ds->wlast, ds->bins_cm.p, ds->np, ds->nan_any.p);
    TC_CUDA(ctx, cudaGetLastError());
  }
  TC_CUDA(ctx, cudaStreamSynchronize(st));
  ds->h_edges = ref->h_edges;
  ds->h_n_edges = ref->h_n_edges;
  ds->quantized = true;
  ds->max_bins = ref->max_bins;
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
  tc_dataset* ds = new tc_dataset();
  ds->ctx = ctx;
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

}  // extern "C"
