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

// 128 partials x 256 bins x 64 columns x (grad, hess) FP32 = 16 MiB per device.
// Every GPU that loads this library holds it until the process exits.
static __device__ __align__(256) float2 tc_noalloc_scratch[NA_MAX_ITEMS * tc::kSlots * NA_W];

std::mutex g_na_mu;
float2* g_na_ptr[NA_MAX_DEVICES] = {};

// grid (items); item = chunk * G + group.
__global__ void __launch_bounds__(NA_THREADS) k_hist_root_na(const uint8_t* __restrict__ bins, uint32_t n,
                                                            uint32_t f, uint32_t fs, const float* __restrict__ g,
                                                            const float* __restrict__ h, uint32_t rows_per_chunk,
                                                            int G, float2* __restrict__ scratch) {
  extern __shared__ float sm[];
  const int item = blockIdx.x;
  const int chunk = item / G, grp = item % G;
  const int g0 = grp * NA_W;
  const int gsize = min(NA_W, (int)f - g0);
  for (int q = threadIdx.x; q < 2 * tc::kSlots * NA_W; q += blockDim.x) sm[q] = 0.0f;
  __syncthreads();
  const uint32_t r0 = (uint32_t)chunk * rows_per_chunk;
  const uint32_t r1 = min(n, r0 + rows_per_chunk);
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

// grid (f), 256 threads = bins: FP64 sum of the chunks' partials, fixed order.
__global__ void k_merge_root_na(const float2* __restrict__ scratch, int chunks, int G, uint32_t f,
                                double* __restrict__ out) {
  const int j = blockIdx.x, b = threadIdx.x;
  const int grp = j / NA_W, col = j % NA_W;
  double sg = 0.0, sh = 0.0;
  for (int c = 0; c < chunks; ++c) {
    const float2 v = scratch[((size_t)(c * G + grp) * tc::kSlots + b) * NA_W + col];
    sg += (double)v.x;
    sh += (double)v.y;
  }
  out[((size_t)j * tc::kSlots + b) * 2] = sg;
  out[((size_t)j * tc::kSlots + b) * 2 + 1] = sh;
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
  if (cudaSetDevice(ctx->device) != cudaSuccess) return ctx->fail(TC_ERR_CUDA, "cudaSetDevice failed");
  float2* scratch = nullptr;
  {
    // once per device, with that device current: the host-side symbol is a
    // stand-in, the kernel needs the array's device address
    std::lock_guard<std::mutex> g(g_na_mu);
    if (!g_na_ptr[ctx->device]) {
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, tc_noalloc_scratch);
      if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaGetSymbolAddress(tc_noalloc_scratch)");
      g_na_ptr[ctx->device] = static_cast<float2*>(p);
    }
    scratch = g_na_ptr[ctx->device];
  }
  cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ctx->stream;
  const int chunks = std::max(1, std::min(NA_MAX_ITEMS / G, (int)((n + 1023) / 1024)));
  const uint32_t rows_per_chunk = (n + chunks - 1) / chunks;
  const size_t smem = (size_t)2 * tc::kSlots * NA_W * sizeof(float);
  cudaError_t e = cudaFuncSetAttribute(k_hist_root_na, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaFuncSetAttribute");
  if (n > 0) {
    k_hist_root_na<<<chunks * G, NA_THREADS, smem, st>>>(bins_rm, n, f, row_stride, grad, hess,
                                                        rows_per_chunk, G, scratch);
    k_merge_root_na<<<f, tc::kSlots, 0, st>>>(scratch, chunks, G, f, hist_out);
  } else {
    e = cudaMemsetAsync(hist_out, 0, (size_t)f * tc::kSlots * 2 * sizeof(double), st);
    if (e != cudaSuccess) return ctx->cuda_fail(e, "cudaMemsetAsync");
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return ctx->cuda_fail(e, "tc_histogram_root_noalloc launch");
  return TC_OK;
}
