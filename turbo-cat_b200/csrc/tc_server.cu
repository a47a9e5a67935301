// Serving loop: resident models, admission by staging memory, continuous
// batching of predict requests with uneven row counts.
//
// One worker thread owns the device side.  Batch slots (each with its own
// stream, device input/output staging and a request table) cycle through
// free -> filling -> in flight -> completing.  While earlier batches run, the
// worker keeps admitting queued requests into the next free slot (as many as
// its staging rows allow, in arrival order), so newly arrived requests
// overlap the device work of the previous ones; each batch is one
// coalesced launch of the table-driven predict kernel.  With coalescing off
// the loop degenerates to the plain path: one request per launch and one
// launch in flight, host-synchronised.
//
// The reference has no serving layer (predict_proba answers one call
// synchronously, python/bindings.cpp:288-382).
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>

#include "tc_internal.h"

using namespace tc;

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id;
  int model;
  const float* X;
  float* out;
  uint32_t n;
  uint32_t f;
  int K;
  int transform;
  bool pinned_in;
  bool pinned_out;
  Clock::time_point t_submit;
  Clock::time_point t_done;
  std::atomic<int> state{0};  // 0 queued, 1 in flight, 2 done, 3 failed
};

struct Slot {
  cudaStream_t stream = nullptr;
  cudaEvent_t done = nullptr;
  DevBuf<float> d_in;        // [rows_cap][max_f]
  DevBuf<float> d_out;       // [rows_cap][16]
  DevBuf<ReqDesc> d_reqs;    // [req_cap]
  DevBuf<uint32_t> d_tiles;  // [req_cap + 1]
  float* h_in = nullptr;     // pinned staging for pageable inputs
  float* h_out = nullptr;    // pinned staging for pageable outputs
  ReqDesc* h_reqs = nullptr;
  uint32_t* h_tiles = nullptr;
  std::vector<Request*> reqs;
  bool busy = false;
};

}  // namespace

struct tc_server {
  tc_ctx* ctx = nullptr;
  tc_server_params prm{};
  int rows_cap = 0;
  int req_cap = 1024;
  int max_f = 0;
  int max_depth = 0;
  PredictPlan plan{};
  std::vector<std::unique_ptr<Slot>> slots;
  std::vector<ModelDesc> models;
  std::vector<const tc_model*> model_ptrs;
  DevBuf<ModelDesc> d_models;
  std::mutex mu;
  std::condition_variable cv_work;   // worker wake-up
  std::condition_variable cv_done;   // completion notifications
  std::deque<Request*> pending;
  std::unordered_map<uint64_t, Request*> live;
  uint64_t next_id = 1;
  std::atomic<bool> stop{false};
  std::thread worker;
  std::atomic<uint64_t> n_completed{0}, n_launches{0}, n_rows{0};
  std::string worker_err;

  void run();
  bool launch(Slot& s, std::vector<Request*>& batch);
  void complete(Slot& s);
};

static bool is_pinned(const void* p) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return a.type == cudaMemoryTypeHost;
}

bool tc_server::launch(Slot& s, std::vector<Request*>& batch) {
  uint32_t row = 0, tile = 0;
  int j = 0;
  for (Request* r : batch) {
    float* din = s.d_in.p + (size_t)row * max_f;
    const size_t bytes = (size_t)r->n * r->f * sizeof(float);
    if (r->pinned_in) {
      cudaMemcpyAsync(din, r->X, bytes, cudaMemcpyHostToDevice, s.stream);
    } else {
      std::memcpy(s.h_in + (size_t)row * max_f, r->X, bytes);
      cudaMemcpyAsync(din, s.h_in + (size_t)row * max_f, bytes, cudaMemcpyHostToDevice, s.stream);
    }
    s.h_reqs[j] = ReqDesc{din, s.d_out.p + (size_t)row * 16, r->n, row, r->model, r->transform};
    s.h_tiles[j] = tile;
    tile += predict_tiles(r->n);
    row += r->n;
    ++j;
  }
  s.h_tiles[j] = tile;
  cudaMemcpyAsync(s.d_reqs.p, s.h_reqs, j * sizeof(ReqDesc), cudaMemcpyHostToDevice, s.stream);
  cudaMemcpyAsync(s.d_tiles.p, s.h_tiles, (j + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice, s.stream);
  if (predict_batched(ctx, d_models.p, s.d_reqs.p, j, s.d_tiles.p, tile, plan, s.stream) != TC_OK)
    return false;
  for (int q = 0; q < j; ++q) {
    Request* r = batch[q];
    const size_t bytes = (size_t)r->n * r->K * sizeof(float);
    const float* src = s.d_out.p + (size_t)s.h_reqs[q].row_begin * 16;
    if (r->pinned_out) {
      cudaMemcpyAsync(r->out, src, bytes, cudaMemcpyDeviceToHost, s.stream);
    } else {
      cudaMemcpyAsync(s.h_out + (size_t)s.h_reqs[q].row_begin * 16, src, bytes, cudaMemcpyDeviceToHost, s.stream);
    }
  }
  cudaEventRecord(s.done, s.stream);
  s.reqs = batch;
  s.busy = true;
  n_launches.fetch_add(1);
  return cudaGetLastError() == cudaSuccess;
}

void tc_server::complete(Slot& s) {
  int q = 0;
  const auto now = Clock::now();
  for (Request* r : s.reqs) {
    if (!r->pinned_out) {
      // rows of request q start at its row_begin in the slot
      std::memcpy(r->out, s.h_out + (size_t)s.h_reqs[q].row_begin * 16, (size_t)r->n * r->K * sizeof(float));
    }
    n_rows.fetch_add(r->n);
    ++q;
  }
  {
    std::lock_guard<std::mutex> g(mu);
    for (Request* r : s.reqs) {
      r->t_done = now;
      r->state.store(2);
    }
  }
  n_completed.fetch_add(s.reqs.size());
  cv_done.notify_all();
  s.reqs.clear();
  s.busy = false;
}

void tc_server::run() {
  cudaSetDevice(ctx->device);
  const bool coalesce = prm.coalesce != 0;
  for (;;) {
    // 1. retire finished batches
    bool any_busy = false;
    for (auto& sp : slots) {
      Slot& s = *sp;
      if (!s.busy) continue;
      const cudaError_t e = cudaEventQuery(s.done);
      if (e == cudaSuccess) {
        complete(s);
      } else if (e != cudaErrorNotReady) {
        std::lock_guard<std::mutex> g(mu);
        worker_err = cudaGetErrorString(e);
        for (Request* r : s.reqs) r->state.store(3);
        s.reqs.clear();
        s.busy = false;
        cv_done.notify_all();
      } else {
        any_busy = true;
      }
    }
    // 2. admit queued requests into a free slot
    Slot* free_slot = nullptr;
    int busy_count = 0;
    for (auto& sp : slots) {
      if (sp->busy) ++busy_count;
      else if (!free_slot) free_slot = sp.get();
    }
    const int max_busy = coalesce ? (int)slots.size() : 1;
    std::vector<Request*> batch;
    {
      std::unique_lock<std::mutex> lk(mu);
      if (stop.load() && pending.empty() && !any_busy) break;
      if (free_slot && busy_count < max_busy && !pending.empty()) {
        uint32_t rows = 0;
        while (!pending.empty() && (int)batch.size() < req_cap) {
          Request* r = pending.front();
          if (!batch.empty() && (!coalesce || rows + r->n > (uint32_t)rows_cap)) break;
          pending.pop_front();
          r->state.store(1);
          batch.push_back(r);
          rows += r->n;
        }
      } else if (!any_busy) {
        cv_work.wait_for(lk, std::chrono::milliseconds(5));
        continue;
      }
    }
    if (!batch.empty()) {
      if (!launch(*free_slot, batch)) {
        std::lock_guard<std::mutex> g(mu);
        worker_err = "batch launch failed";
        for (Request* r : batch) r->state.store(3);
        cv_done.notify_all();
      }
      if (!coalesce) {
        // plain path: synchronous per request
        cudaEventSynchronize(free_slot->done);
      }
      continue;
    }
    if (any_busy) std::this_thread::yield();
  }
}

extern "C" {

tc_status tc_server_create(tc_ctx* ctx, const tc_server_params* p, tc_server** out) {
  if (!ctx || !p || !out) return TC_ERR_INVALID_ARG;
  *out = nullptr;
  if (p->max_batch_rows < 1 || p->max_inflight < 1 || p->max_inflight > 16)
    return ctx->fail(TC_ERR_INVALID_ARG, "server needs max_batch_rows >= 1 and 1 <= max_inflight <= 16");
  cudaSetDevice(ctx->device);
  tc_server* s = new tc_server();
  s->ctx = ctx;
  s->prm = *p;
  s->rows_cap = p->max_batch_rows;
  // staging is sized when the first model is added (its feature count); the
  // admission limit is the staging budget
  for (int i = 0; i < (p->coalesce ? p->max_inflight : 1); ++i) s->slots.emplace_back(new Slot());
  for (auto& slp : s->slots) {
    Slot& sl = *slp;
    if (cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) != cudaSuccess) {
      delete s;
      return ctx->fail(TC_ERR_CUDA, "server stream creation failed");
    }
  }
  tc_status st = s->d_models.alloc(ctx, 64, "server model table");
  if (st != TC_OK) {
    delete s;
    return st;
  }
  *out = s;
  return TC_OK;
}

tc_status tc_server_add_model(tc_server* s, const tc_model* m, int32_t* model_id) {
  if (!s || !m || !model_id) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = s->ctx;
  if (s->worker.joinable()) return ctx->fail(TC_ERR_BUSY, "models must be added before the first request");
  if (s->models.size() >= 64) return ctx->fail(TC_ERR_INVALID_ARG, "at most 64 resident models");
  if (m->regular) return ctx->fail(TC_ERR_INVALID_ARG, "models of regular trees are served by tc_predict only");
  cudaSetDevice(ctx->device);
  s->models.push_back(model_desc(m));
  s->model_ptrs.push_back(m);
  s->max_f = std::max(s->max_f, m->info.n_features);
  s->max_depth = std::max(s->max_depth, m->info.max_depth);
  s->plan = predict_plan(s->model_ptrs.data(), (int)s->model_ptrs.size());
  TC_CUDA(ctx, cudaMemcpy(s->d_models.p, s->models.data(), s->models.size() * sizeof(ModelDesc),
                          cudaMemcpyHostToDevice));
  *model_id = (int32_t)s->models.size() - 1;
  return TC_OK;
}

static void release_slot(Slot& sl) {
  sl.d_in.reset();
  sl.d_out.reset();
  sl.d_reqs.reset();
  sl.d_tiles.reset();
  if (sl.h_in) cudaFreeHost(sl.h_in);
  if (sl.h_out) cudaFreeHost(sl.h_out);
  if (sl.h_reqs) cudaFreeHost(sl.h_reqs);
  if (sl.h_tiles) cudaFreeHost(sl.h_tiles);
  sl.h_in = sl.h_out = nullptr;
  sl.h_reqs = nullptr;
  sl.h_tiles = nullptr;
}

static tc_status alloc_slot(tc_server* s, Slot& sl) {
  tc_ctx* ctx = s->ctx;
  TC_TRY(sl.d_in.alloc(ctx, (size_t)s->rows_cap * s->max_f, "server input staging"));
  TC_TRY(sl.d_out.alloc(ctx, (size_t)s->rows_cap * 16, "server output staging"));
  TC_TRY(sl.d_reqs.alloc(ctx, s->req_cap, "server request table"));
  TC_TRY(sl.d_tiles.alloc(ctx, s->req_cap + 1, "server tile table"));
  TC_CUDA(ctx, cudaMallocHost(&sl.h_in, (size_t)s->rows_cap * s->max_f * sizeof(float)));
  TC_CUDA(ctx, cudaMallocHost(&sl.h_out, (size_t)s->rows_cap * 16 * sizeof(float)));
  TC_CUDA(ctx, cudaMallocHost(&sl.h_reqs, s->req_cap * sizeof(ReqDesc)));
  TC_CUDA(ctx, cudaMallocHost(&sl.h_tiles, (s->req_cap + 1) * sizeof(uint32_t)));
  return TC_OK;
}

static tc_status ensure_started(tc_server* s) {
  if (s->worker.joinable()) return TC_OK;
  tc_ctx* ctx = s->ctx;
  if (s->models.empty()) return ctx->fail(TC_ERR_NOT_FITTED, "no model added to the server");
  // admission by memory: each slot stages rows_cap rows of max_f inputs and
  // 16 outputs; shrink rows_cap to the staging budget
  const size_t per_row = (size_t)(s->max_f + 16) * sizeof(float);
  if (s->prm.staging_bytes > 0) {
    const size_t rows_budget = s->prm.staging_bytes / (per_row * s->slots.size());
    if (rows_budget < 1) return ctx->fail(TC_ERR_OOM, "staging budget smaller than one row per slot");
    s->rows_cap = (int)std::min<size_t>(s->rows_cap, rows_budget);
  }
  // a set-up that fails partway (budget, pinned memory) releases every
  // slot's buffers, so that the retry of the next submit starts clean
  tc_status st = TC_OK;
  for (auto& slp : s->slots) {
    st = alloc_slot(s, *slp);
    if (st != TC_OK) break;
  }
  if (st != TC_OK) {
    for (auto& slp : s->slots) release_slot(*slp);
    return st;
  }
  s->worker = std::thread([s] { s->run(); });
  return TC_OK;
}

tc_status tc_server_submit(tc_server* s, int32_t model_id, const float* X, uint32_t n, uint16_t f, int32_t transform,
                           float* out, uint64_t* ticket) {
  if (!s || !ticket || (!X && n) || (!out && n)) return TC_ERR_INVALID_ARG;
  tc_ctx* ctx = s->ctx;
  if (model_id < 0 || model_id >= (int)s->models.size()) return ctx->fail(TC_ERR_INVALID_ARG, "unknown model id %d", model_id);
  const ModelDesc& md = s->models[model_id];
  if (f != (uint32_t)md.n_features)
    return ctx->fail(TC_ERR_INVALID_ARG, "request has %u features, model %d expects %d", f, model_id, md.n_features);
  if (n == 0) return ctx->fail(TC_ERR_INVALID_ARG, "empty request");
  {
    std::lock_guard<std::mutex> g(s->mu);
    TC_TRY(ensure_started(s));
  }
  if (n > (uint32_t)s->rows_cap)
    return ctx->fail(TC_ERR_INVALID_ARG, "request of %u rows exceeds the batch capacity %d", n, s->rows_cap);
  Request* r = new Request();
  r->model = model_id;
  r->X = X;
  r->out = out;
  r->n = n;
  r->f = f;
  r->K = md.n_classes;
  r->transform = transform;
  r->pinned_in = is_pinned(X);
  r->pinned_out = is_pinned(out);
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> g(s->mu);
    r->id = s->next_id++;
    s->pending.push_back(r);
    s->live[r->id] = r;
  }
  s->cv_work.notify_one();
  *ticket = r->id;
  return TC_OK;
}

tc_status tc_server_poll(tc_server* s, uint64_t ticket, int64_t timeout_us, int* done, double* latency_s) {
  if (!s || !done) return TC_ERR_INVALID_ARG;
  *done = 0;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->live.find(ticket);
  if (it == s->live.end()) return s->ctx->fail(TC_ERR_INVALID_ARG, "unknown ticket %llu", (unsigned long long)ticket);
  Request* r = it->second;
  const auto deadline = Clock::now() + std::chrono::microseconds(timeout_us > 0 ? timeout_us : 0);
  while (r->state.load() < 2) {
    if (timeout_us <= 0 || Clock::now() >= deadline) return TC_ERR_TIMEOUT;
    s->cv_done.wait_until(lk, deadline);
  }
  const int st = r->state.load();
  if (latency_s) *latency_s = std::chrono::duration<double>(r->t_done - r->t_submit).count();
  s->live.erase(it);
  delete r;
  if (st == 3) return s->ctx->fail(TC_ERR_CUDA, "request failed: %s", s->worker_err.c_str());
  *done = 1;
  return TC_OK;
}

tc_status tc_server_replay(tc_server* s, const tc_replay_request* reqs, int32_t n_requests, double* latency_s,
                           double* wall_s) {
  if (!s || (!reqs && n_requests) || n_requests < 0) return TC_ERR_INVALID_ARG;
  std::vector<uint64_t> tickets(n_requests, 0);
  std::vector<tc_status> sub(n_requests, TC_OK);
  std::atomic<int> submitted{0};
  const auto t0 = Clock::now();
  std::thread gen([&] {
    for (int i = 0; i < n_requests; ++i) {
      const auto at = t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(reqs[i].arrival_s));
      while (Clock::now() < at) {
      }
      sub[i] = tc_server_submit(s, reqs[i].model_id, reqs[i].X, reqs[i].n, reqs[i].f, reqs[i].transform, reqs[i].out,
                                &tickets[i]);
      submitted.store(i + 1, std::memory_order_release);
    }
  });
  tc_status rc = TC_OK;
  for (int i = 0; i < n_requests; ++i) {
    while (submitted.load(std::memory_order_acquire) <= i) std::this_thread::yield();
    if (sub[i] != TC_OK) {
      rc = sub[i];
      continue;
    }
    int done = 0;
    double lat = 0.0;
    tc_status p;
    do {
      p = tc_server_poll(s, tickets[i], 100000, &done, &lat);
    } while (p == TC_ERR_TIMEOUT);
    if (p != TC_OK) rc = p;
    if (latency_s) latency_s[i] = lat;
  }
  gen.join();
  if (wall_s) *wall_s = std::chrono::duration<double>(Clock::now() - t0).count();
  return rc;
}

tc_status tc_server_stats(tc_server* s, uint64_t* completed, uint64_t* launches, uint64_t* rows) {
  if (!s) return TC_ERR_INVALID_ARG;
  if (completed) *completed = s->n_completed.load();
  if (launches) *launches = s->n_launches.load();
  if (rows) *rows = s->n_rows.load();
  return TC_OK;
}

void tc_server_destroy(tc_server* s) {
  if (!s) return;
  cudaSetDevice(s->ctx->device);
  s->stop.store(true);
  s->cv_work.notify_all();
  if (s->worker.joinable()) s->worker.join();
  for (auto& kv : s->live) delete kv.second;
  for (auto& slp : s->slots) {
    Slot& sl = *slp;
    if (sl.stream) cudaStreamSynchronize(sl.stream);
    if (sl.stream) cudaStreamDestroy(sl.stream);
    if (sl.done) cudaEventDestroy(sl.done);
    if (sl.h_in) cudaFreeHost(sl.h_in);
    if (sl.h_out) cudaFreeHost(sl.h_out);
    if (sl.h_reqs) cudaFreeHost(sl.h_reqs);
    if (sl.h_tiles) cudaFreeHost(sl.h_tiles);
  }
  delete s;
}

}  // extern "C"
