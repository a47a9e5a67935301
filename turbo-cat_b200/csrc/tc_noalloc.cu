// Root-level histogram that allocates nothing.
//
// Same arithmetic as the trainer's histogram path (FP32 shared-memory
// accumulation per block, FP64 merge across blocks), but the per-block FP32
// partials live in a fixed file-scope device array instead of memory
// obtained from cudaMalloc, so a caller that cannot allocate device memory
// can still build histograms on buffers it already owns.
#include <algorithm>
#include <mutex>

#include "tc_internal.h"

namespace {

constexpr int NA_W = 64;                  // feature columns per block
constexpr int NA_MAX_ITEMS = 128;         // (row chunk, feature group) partials held at once
constexpr int NA_THREADS = 512;
constexpr int NA_MAX_DEVICES = 64;
constexpr uint32_t NA_CHUNK_ROWS = 16384; // rows summed in FP32 by one block, at most

// 128 partials x 256 bins x 64 columns x (grad, hess) FP32 = 16 MiB per device.
// Every GPU that loads this library holds it until the process exits.
static __device__ __align__(256) float2 tc_noalloc_scratch[NA_MAX_ITEMS * tc::kSlots * NA_W];

std::mutex g_na_mu;
float2* g_na_ptr[NA_MAX_DEVICES] = {};

// Restores the calling thread's current device on every return path (the
// entry point is meant to be embedded in another framework's process).
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// grid (items); item = chunk * G + group; the chunks of one pass start at row r_base.
__global__ void __launch_bounds__(NA_THREADS) k_hist_root_na(const uint8_t* __restrict__ bins, uint32_t n,
                                                            uint32_t f, uint32_t fs, const float* __restrict__ g,
                                                            const float* __restrict__ h, uint32_t r_base,
                                                            uint32_t rows_per_chunk, int G,
                                                            float2* __restrict__ scratch) {
  extern __shared__ float sm[];
  const int item = blockIdx.x;
  const int chunk = item / G, grp = item % G;
  const int g0 = grp * NA_W;
  const int gsize = min(NA_W, (int)f - g0);
  for (int q = threadIdx.x; q < 2 * tc::kSlots * NA_W; q += blockDim.x) sm[q] = 0.0f;
  __syncthreads();
  const uint32_t r0 = r_base + (uint32_t)chunk * rows_per_chunk;
  const uint32_t r1 = r0 < n ? min(n, r0 + rows_per_chunk) : r0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (uint32_t r = r0 + warp; r < r1; r += nw) {
    const float gv = g[r], hv = h[r];
    const uint8_t* br = bins + (size_t)r * fs + g0;
#pragma unroll
    for (int j = 0; j < NA_W / 32; ++j) {
      const int col = lane + 32 * j;
      if (col < gsize) {
        const int b = br[col];
        atomicAdd(&sm[(2 * b) * NA_W + col], gv);
        atomicAdd(&sm[(2 * b + 1) * NA_W + col], hv);
      }
    }
  }
  __syncthreads();
  // every slot of this item's partial is rewritten: no stale contents survive
  float2* out = scratch + (size_t)item * tc::kSlots * NA_W;
  for (int q = threadIdx.x; q < tc::kSlots * NA_W; q += blockDim.x) {
    const int b = q / NA_W, col = q % NA_W;
    out[q] = make_float2(sm[(2 * b) * NA_W + col], sm[(2 * b + 1) * NA_W + col]);
  }
}

// grid (f), 256 threads = bins: FP64 sum of one pass's chunk partials in a
// fixed order; the first pass stores, later passes add to hist_out.
__global__ void k_merge_root_na(const float2* __restrict__ scratch, int chunks, int G, uint32_t f, int accumulate,
                                double* __restrict__ out) {
  const int j = blockIdx.x, b = threadIdx.x;
  const int grp = j / NA_W, col = j % NA_W;
  double sg = 0.0, sh = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const float2 v = scratch[((size_t)(c * G + grp) * tc::kSlots + b) * NA_W + col];
    sg += (double)v.x;
    sh += (double)v.y;
  }
  double* o = out + ((size_t)j * tc::kSlots + b) * 2;
  if (accumulate) {
    sg += o[0];
    sh += o[1];
  }
  o[0] = sg;
  o[1] = sh;
}

}  // namespace

extern "C" tc_status tc_histogram_root_noalloc(tc_ctx* ctx, const uint8_t* bins_rm, uint32_t n, uint16_t f,
                                               uint32_t row_stride, const float* grad, const float* hess,
                                               double* hist_out, void* stream) {
  if (!ctx || !bins_rm || !grad || !hess || !hist_out || f == 0) return TC_ERR_INVALID_ARG;
  if (row_stride < f) return ctx->fail(TC_ERR_INVALID_ARG, "row_stride %u < features %u", row_stride, f);
  const int G = (f + NA_W - 1) / NA_W;
  if (G > NA_MAX_ITEMS)
    return ctx->fail(TC_ERR_INVALID_ARG,
                     "tc_histogram_root_noalloc: %u features exceed its fixed scratch (at most %d features)", f,
                     NA_MAX_ITEMS * NA_W);
  if (ctx->device < 0 || ctx->device >= NA_MAX_DEVICES)
    return ctx->fail(TC_ERR_INVALID_ARG, "device %d beyond the no-alloc device table", ctx->device);
  DeviceGuard restore;
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(TC_ERR_CUDA, "cudaSetDevice failed");
  float2* scratch = nullptr;
  {
    // once per device, with that device current: the host-side symbol is a
    // stand-in, the kernel needs the array's device address (in the
    // runtime's primary context of the device, which every call here uses)
    std::lock_guard<std::mutex> g(g_na_mu);
    if (!g_na_ptr[ctx->device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, tc_noalloc_scratch);
      if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaGetSymbolAddress(tc_noalloc_scratch)");
      g_na_ptr[ctx->device] = static_cast<float2*>(p);
    }
    scratch = g_na_ptr[ctx->device];
  }
  // With no stream given the work goes on the context's stream, which the
  // trainer captures into CUDA graphs while it holds the training lock; the
  // enqueue takes the same lock so that it never lands inside a capture.
  std::unique_lock<std::recursive_mutex> train_lock(ctx->train_mu, std::defer_lock);
  if (!stream) train_lock.lock();
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  // A pass holds at most NA_MAX_ITEMS / G chunks of at most NA_CHUNK_ROWS
  // rows (a block never sums more rows than that in FP32); larger inputs
  // take several passes, each merged into hist_out in FP64.
  const int chunks_max = std::max(1, NA_MAX_ITEMS / G);
  const uint32_t want = (uint32_t)std::max<uint64_t>(1, ((uint64_t)n + 1023) / 1024);
  const uint32_t rows_per_chunk =
      (uint32_t)std::min<uint64_t>(NA_CHUNK_ROWS, ((uint64_t)n + std::min<uint32_t>(want, chunks_max) - 1) /
                                                      std::min<uint32_t>(want, chunks_max));
  const size_t smem = (size_t)2 * tc::kSlots * NA_W * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_hist_root_na, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaFuncSetAttribute");
  if (n > 0) {
    const uint64_t rows_per_pass = (uint64_t)chunks_max * rows_per_chunk;
    int pass = 0;
    for (uint64_t r = 0; r < n; r += rows_per_pass, ++pass) {
      const uint64_t left = n - r;
      const int chunks = (int)std::min<uint64_t>(chunks_max, (left + rows_per_chunk - 1) / rows_per_chunk);
      k_hist_root_na<<<chunks * G, NA_THREADS, smem, st>>>(bins_rm, n, f, row_stride, grad, hess, (uint32_t)r,
                                                          rows_per_chunk, G, scratch);
      k_merge_root_na<<<f, tc::kSlots, 0, st>>>(scratch, chunks, G, f, pass > 0 ? 1 : 0, hist_out);
    }
  } else {
    e = cudaMemsetAsync(hist_out, 0, (size_t)f * tc::kSlots * 2 * sizeof(double), st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaMemsetAsync");
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return ctx->cuda_fail(e, "tc_histogram_root_noalloc launch");
  return TC_OK;
}
