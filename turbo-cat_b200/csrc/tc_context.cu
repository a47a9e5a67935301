// Context: device selection, stream, device-memory accounting, errors.
#include <chrono>
#include <thread>

#include "tc_internal.h"

tc_status tc_ctx::alloc(void** p, size_t bytes, const char* what) {
  {
    std::lock_guard<std::mutex> g(mu);
    if (fail_next > 0) {
      --fail_next;
      err = std::string("injected allocation failure: ") + what;
      return TC_ERR_OOM;
    }
    if (budget && in_use + bytes > budget) {
      char buf[256];
      snprintf(buf, sizeof(buf), "memory budget exceeded allocating %zu bytes for %s (%zu of %zu in use)",
               bytes, what, in_use, budget);
      err = buf;
      return TC_ERR_OOM;
    }
  }
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(TC_ERR_OOM, "cudaMalloc(%zu) for %s: %s", bytes, what, cudaGetErrorString(e));
  }
  std::lock_guard<std::mutex> g(mu);
  allocs[*p] = bytes;
  in_use += bytes;
  if (in_use > peak) peak = in_use;
  return TC_OK;
}

void tc_ctx::release(void* p) {
  if (!p) return;
  size_t bytes = 0;
  {
    std::lock_guard<std::mutex> g(mu);
    auto it = allocs.find(p);
    if (it != allocs.end()) {
      bytes = it->second;
      allocs.erase(it);
      in_use -= bytes;
    }
  }
  cudaFree(p);
}

extern "C" {

tc_status tc_ctx_create(int device, size_t mem_budget, tc_ctx** out) {
  if (!out) return TC_ERR_INVALID_ARG;
  *out = nullptr;
  int count = 0;
  if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0) {
    cudaGetLastError();
    return TC_ERR_CUDA;
  }
  if (device < 0 || device >= count) return TC_ERR_INVALID_ARG;
  if (cudaSetDevice(device) != cudaSuccess) return TC_ERR_CUDA;
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return TC_ERR_CUDA;
  if (prop.major < 10) return TC_ERR_CUDA;  // built for sm_100a only
  tc_ctx* c = new tc_ctx();
  c->device = device;
  c->sm_count = prop.multiProcessorCount;
  c->budget = mem_budget;
  if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete c;
    return TC_ERR_CUDA;
  }
  if (cudaStreamCreateWithFlags(&c->pred_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaStreamDestroy(c->stream);
    delete c;
    return TC_ERR_CUDA;
  }
  *out = c;
  return TC_OK;
}

void tc_ctx_destroy(tc_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  {
    std::lock_guard<std::mutex> g(ctx->pred_mu);
    tc::stop_latency_worker(ctx, nullptr);
  }
  cudaStreamSynchronize(ctx->stream);
  cudaStreamSynchronize(ctx->pred_stream);
  for (auto& kv : ctx->allocs) cudaFree(kv.first);
  ctx->allocs.clear();
  if (ctx->pin_io) cudaFreeHost(ctx->pin_io);
  if (ctx->lw_box) cudaFreeHost(ctx->lw_box);
  for (int b = 0; b < 2; ++b) {
    if (ctx->up_stage[b]) cudaFreeHost(ctx->up_stage[b]);
    if (ctx->up_ev[b]) cudaEventDestroy(ctx->up_ev[b]);
  }
  if (ctx->lw_stream) cudaStreamDestroy(ctx->lw_stream);
  cudaStreamDestroy(ctx->stream);
  cudaStreamDestroy(ctx->pred_stream);
  delete ctx;
}

const char* tc_last_error(const tc_ctx* ctx) {
  if (!ctx) return "null context";
  return ctx->err.c_str();
}

tc_status tc_ctx_memory(const tc_ctx* ctx, size_t* in_use, size_t* peak) {
  if (!ctx) return TC_ERR_INVALID_ARG;
  if (in_use) *in_use = ctx->in_use;
  if (peak) *peak = ctx->peak;
  return TC_OK;
}

tc_status tc_ctx_fail_next_allocs(tc_ctx* ctx, int count) {
  if (!ctx || count < 0) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->mu);
  ctx->fail_next = count;
  return TC_OK;
}

// Polls the context stream instead of blocking in the driver so that a
// stuck device turns into TC_ERR_TIMEOUT rather than a hung caller.
tc_status tc_ctx_set_latency_worker(tc_ctx* ctx, int enabled) {
  if (!ctx) return TC_ERR_INVALID_ARG;
  std::lock_guard<std::mutex> g(ctx->pred_mu);
  cudaSetDevice(ctx->device);
  if (!enabled) tc::stop_latency_worker(ctx, nullptr);
  ctx->lw_enabled = enabled != 0;
  return TC_OK;
}

tc_status tc_ctx_synchronize(tc_ctx* ctx, int timeout_ms) {
  if (!ctx) return TC_ERR_INVALID_ARG;
  // not while another thread's training call may be capturing the stream
  std::lock_guard<std::recursive_mutex> train_lock(ctx->train_mu);
  cudaSetDevice(ctx->device);
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    cudaError_t e = cudaStreamQuery(ctx->stream);
    if (e == cudaSuccess) e = cudaStreamQuery(ctx->pred_stream);
    if (e == cudaSuccess) return TC_OK;
    if (e != cudaErrorNotReady) return ctx->cuda_fail(e, "stream");
    const auto dt = std::chrono::duration_cast<std::chrono::milliseconds>(
                        std::chrono::steady_clock::now() - t0).count();
    if (timeout_ms >= 0 && dt >= timeout_ms)
      return ctx->fail(TC_ERR_TIMEOUT, "device work did not finish within %d ms", timeout_ms);
    std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

}  // extern "C"
