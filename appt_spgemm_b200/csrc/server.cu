// Request server: continuous batching of A·A / A·Aᵀ requests with admission by
// a device-memory budget taken from the symbolic pass.
//
// Structure (all host C++ around the engine's own C ABI):
//  - a FIFO of submitted requests guarded by one mutex;
//  - `workers` threads, each with its own non-blocking stream and engine
//    context, so several requests (or merged batches) run on the device at the
//    same time;
//  - a worker takes the oldest request; if it is small (n < batch_rows) it also
//    takes the other queued small requests of the same task (up to batch_max)
//    and runs them as one batched plan (block-diagonal layout), then copies
//    each request's slice of the result into its own buffers;
//  - after planning, a request's exact output size plus the plan workspace is
//    reserved against the budget; the worker waits (condition variable) until
//    enough is free, and rejects requests that could never fit.
// The reference has no serving layer; this follows the serving contract of
// the benchmark configuration (Poisson arrivals, p50/p99 latency).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "kernels.h"

namespace {

using Clock = std::chrono::steady_clock;

struct Request {
  uint64_t id = 0;
  spg_task task = SPG_TASK_AA;
  spg_csr_dev A{};
  int32_t status = SPG_ERR_NOT_READY;
  bool batched = false;
  int64_t nnz_c = 0, products = 0, reserved = 0;
  double submit_ms = 0, start_ms = 0, done_ms = 0;
  int64_t* rowptr = nullptr;
  int32_t* col = nullptr;
  double* val = nullptr;
  std::string error;
};

__global__ void k_rebase(const int64_t* __restrict__ src, int64_t off, int64_t sub, int32_t n,
                         int64_t* __restrict__ dst) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[off + i] - sub;
}

int64_t output_bytes(int32_t n, int64_t nnz) { return 8 * ((int64_t)n + 1) + 12 * nnz; }

}  // namespace

struct spg_server {
  spg_server_config cfg{};
  int device = 0;
  Clock::time_point t0;
  std::mutex mu;
  std::condition_variable cv_queue, cv_done, cv_budget;
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  int64_t reserved = 0, peak = 0, batches = 0;
  bool stopping = false;
  std::vector<std::thread> workers;

  double now_ms() const {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
  }
};

namespace {

void finish(spg_server* s, Request* r, int32_t status, const char* err = nullptr) {
  r->status = status;
  if (err) r->error = err;
  r->done_ms = s->now_ms();
}

// Reserve `need` bytes of the budget, waiting for releases; false when the
// request can never fit (rejected) or the server stops.
bool reserve(spg_server* s, std::unique_lock<std::mutex>& lk, int64_t need) {
  if (need > s->cfg.memory_budget_bytes) return false;
  s->cv_budget.wait(lk, [&] { return s->stopping || s->reserved + need <= s->cfg.memory_budget_bytes; });
  if (s->stopping) return false;
  s->reserved += need;
  s->peak = std::max(s->peak, s->reserved);
  return true;
}

void unreserve(spg_server* s, int64_t bytes) {
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->reserved -= bytes;
  }
  s->cv_budget.notify_all();
}

spg_status alloc_result(Request* r, int32_t n, int64_t nnz, cudaStream_t st) {
  const size_t nz = (size_t)(nnz > 0 ? nnz : 1);
  cudaError_t e = cudaMallocAsync((void**)&r->rowptr, 8 * ((size_t)n + 1), st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&r->col, 4 * nz, st);
  if (e == cudaSuccess) e = cudaMallocAsync((void**)&r->val, 8 * nz, st);
  return e == cudaSuccess ? SPG_OK : SPG_ERR_OOM;
}

void free_result(Request* r, cudaStream_t st) {
  if (r->rowptr) cudaFreeAsync(r->rowptr, st);
  if (r->col) cudaFreeAsync(r->col, st);
  if (r->val) cudaFreeAsync(r->val, st);
  r->rowptr = nullptr;
  r->col = nullptr;
  r->val = nullptr;
}

void run_single(spg_server* s, spg_ctx* ctx, cudaStream_t st, Request* r) {
  spg_plan* p = nullptr;
  spg_status rc = spg_plan_create(ctx, r->task, &r->A, st, &p);
  if (rc != SPG_OK) {
    std::lock_guard<std::mutex> lk(s->mu);
    finish(s, r, rc, spg_last_error_string());
    return;
  }
  spg_plan_info info{};
  spg_plan_get_info(p, &info);
  const int64_t out = output_bytes(r->A.n, info.nnz_c);
  const int64_t need = out + info.workspace_bytes;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    r->products = info.products;
    r->nnz_c = info.nnz_c;
    if (!reserve(s, lk, need)) {
      if (s->stopping) finish(s, r, SPG_ERR_CUDA, "server stopped before the request ran");
      else finish(s, r, SPG_ERR_BUDGET, "request exceeds the memory budget");
      lk.unlock();
      spg_plan_destroy(p);
      return;
    }
    r->reserved = out;
  }
  rc = alloc_result(r, r->A.n, info.nnz_c, st);
  spg_csr_out C{r->A.n, 0, r->rowptr, r->col, r->val};
  if (rc == SPG_OK) rc = spg_execute(p, &C, st);
  if (rc == SPG_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = SPG_ERR_CUDA;
  const std::string err = rc == SPG_OK ? "" : spg_last_error_string();
  spg_plan_destroy(p);
  if (rc != SPG_OK) free_result(r, st);
  unreserve(s, info.workspace_bytes + (rc == SPG_OK ? 0 : out));
  std::lock_guard<std::mutex> lk(s->mu);
  if (rc != SPG_OK) r->reserved = 0;
  finish(s, r, rc, rc == SPG_OK ? nullptr : err.c_str());
}

void run_batch(spg_server* s, spg_ctx* ctx, cudaStream_t st, std::vector<Request*>& rs) {
  std::vector<spg_csr_dev> As;
  for (Request* r : rs) As.push_back(r->A);
  spg_plan* p = nullptr;
  spg_status rc = spg_plan_create_batched(ctx, rs[0]->task, (int32_t)rs.size(), As.data(), st, &p);
  if (rc != SPG_OK) {  // e.g. one bad instance: run each alone to isolate it
    for (Request* r : rs) run_single(s, ctx, st, r);
    return;
  }
  spg_plan_info info{};
  spg_plan_get_info(p, &info);
  std::vector<int64_t> row_off(rs.size() + 1), nnz_off(rs.size() + 1);
  spg_plan_batch_offsets(p, row_off.data(), nnz_off.data());
  int64_t outs = 0;
  std::vector<int64_t> out_r(rs.size());
  for (size_t b = 0; b < rs.size(); ++b) {
    out_r[b] = output_bytes(rs[b]->A.n, nnz_off[b + 1] - nnz_off[b]);
    outs += out_r[b];
  }
  // the concatenated output and the workspace are temporary
  const int64_t temp = output_bytes(info.n, info.nnz_c) + info.workspace_bytes;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    if (!reserve(s, lk, outs + temp)) {
      lk.unlock();
      spg_plan_destroy(p);
      for (Request* r : rs) run_single(s, ctx, st, r);
      return;
    }
    ++s->batches;
    for (size_t b = 0; b < rs.size(); ++b) {
      rs[b]->batched = true;
      rs[b]->reserved = out_r[b];
      rs[b]->nnz_c = nnz_off[b + 1] - nnz_off[b];
    }
  }
  Request cat;
  rc = alloc_result(&cat, info.n, info.nnz_c, st);
  spg_csr_out C{info.n, 0, cat.rowptr, cat.col, cat.val};
  if (rc == SPG_OK) rc = spg_execute(p, &C, st);
  for (size_t b = 0; b < rs.size() && rc == SPG_OK; ++b) {
    Request* r = rs[b];
    const int64_t nz = nnz_off[b + 1] - nnz_off[b];
    rc = alloc_result(r, r->A.n, nz, st);
    if (rc != SPG_OK) break;
    k_rebase<<<(r->A.n + 256) / 256, 256, 0, st>>>(cat.rowptr, row_off[b], nnz_off[b], r->A.n,
                                                    r->rowptr);
    SPG_COUNT_LAUNCH();
    if (nz > 0) {
      cudaMemcpyAsync(r->col, cat.col + nnz_off[b], 4 * (size_t)nz, cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(r->val, cat.val + nnz_off[b], 8 * (size_t)nz, cudaMemcpyDeviceToDevice, st);
    }
  }
  free_result(&cat, st);
  if (rc == SPG_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = SPG_ERR_CUDA;
  const std::string err = rc == SPG_OK ? "" : spg_last_error_string();
  spg_plan_destroy(p);
  if (rc != SPG_OK)
    for (Request* r : rs) free_result(r, st);
  unreserve(s, temp + (rc == SPG_OK ? 0 : outs));
  std::lock_guard<std::mutex> lk(s->mu);
  for (size_t b = 0; b < rs.size(); ++b) {
    // the product count of an instance: the batch total split by its output share
    rs[b]->products = info.nnz_c > 0 ? (int64_t)((double)info.products * (double)rs[b]->nnz_c /
                                                 (double)info.nnz_c) : 0;
    if (rc != SPG_OK) rs[b]->reserved = 0;
    finish(s, rs[b], rc, rc == SPG_OK ? nullptr : err.c_str());
  }
}

void worker_main(spg_server* s, int index) {
  (void)index;
  cudaSetDevice(s->device);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  spg_config cfg{};
  cfg.struct_size = sizeof(spg_config);
  cfg.device = s->device;
  cfg.pool_release_bytes = 64ll << 20;  // give freed memory back: the budget is global
  spg_ctx* ctx = nullptr;
  const bool ok = spg_create(&ctx, &cfg) == SPG_OK;
  for (;;) {
    std::vector<Request*> rs;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_queue.wait(lk, [&] { return s->stopping || !s->queue.empty(); });
      if (s->queue.empty()) break;  // stopping with nothing left
      Request* r = s->reqs[s->queue.front()].get();
      s->queue.pop_front();
      rs.push_back(r);
      if (r->A.n < s->cfg.batch_rows) {
        for (auto it = s->queue.begin(); it != s->queue.end() && (int)rs.size() < s->cfg.batch_max;) {
          Request* q = s->reqs[*it].get();
          if (q->task == r->task && q->A.n < s->cfg.batch_rows) {
            rs.push_back(q);
            it = s->queue.erase(it);
          } else {
            ++it;
          }
        }
      }
      const double t = s->now_ms();
      for (Request* q : rs) q->start_ms = t;
    }
    if (!ok) {
      std::lock_guard<std::mutex> lk(s->mu);
      for (Request* q : rs) finish(s, q, SPG_ERR_CUDA, "worker context could not be created");
    } else if (rs.size() == 1) {
      run_single(s, ctx, st, rs[0]);
    } else {
      run_batch(s, ctx, st, rs);
    }
    s->cv_done.notify_all();
  }
  if (ctx) spg_destroy(ctx);
  cudaStreamDestroy(st);
}

}  // namespace

extern "C" {

spg_status spg_server_create(const spg_server_config* cfg, spg_server** out) {
  spg::clear_error();
  if (!out) return spg::set_error(SPG_ERR_INVALID_ARG, "null server pointer");
  *out = nullptr;
  spg_server* s = new spg_server();
  if (cfg && cfg->struct_size > 0) {
    const size_t sz = std::min((size_t)cfg->struct_size, sizeof(spg_server_config));
    std::memcpy(&s->cfg, cfg, sz);
  }
  s->cfg.struct_size = sizeof(spg_server_config);
  if (s->cfg.workers <= 0) s->cfg.workers = 4;
  if (s->cfg.workers > 64) s->cfg.workers = 64;
  if (s->cfg.memory_budget_bytes <= 0) s->cfg.memory_budget_bytes = 150ll * 1000 * 1000 * 1000;
  if (s->cfg.batch_rows <= 0) s->cfg.batch_rows = 65536;
  if (s->cfg.batch_max <= 0) s->cfg.batch_max = 64;
  if (cudaGetDevice(&s->device) != cudaSuccess) {
    delete s;
    return spg::set_error(SPG_ERR_CUDA, "no CUDA device");
  }
  s->t0 = Clock::now();
  for (int i = 0; i < s->cfg.workers; ++i) s->workers.emplace_back(worker_main, s, i);
  *out = s;
  return SPG_OK;
}

spg_status spg_server_submit(spg_server* s, spg_task task, const spg_csr_dev* A, uint64_t* id) {
  spg::clear_error();
  if (!s || !A || !id) return spg::set_error(SPG_ERR_INVALID_ARG, "null argument");
  if (task != SPG_TASK_AA && task != SPG_TASK_AAT && task != SPG_TASK_AATS)
    return spg::set_error(SPG_ERR_INVALID_ARG, "unknown task %d", (int)task);
  if (A->n < 0 || A->nnz < 0 || !A->rowptr || (A->nnz > 0 && (!A->col || !A->val)))
    return spg::set_error(SPG_ERR_INVALID_ARG, "bad matrix descriptor");
  auto r = std::make_unique<Request>();
  r->task = task;
  r->A = *A;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stopping) return spg::set_error(SPG_ERR_INVALID_ARG, "server is stopping");
    r->id = s->next_id++;
    r->submit_ms = s->now_ms();
    *id = r->id;
    s->queue.push_back(r->id);
    s->reqs[r->id] = std::move(r);
  }
  s->cv_queue.notify_one();
  return SPG_OK;
}

static void fill_info(const Request* r, spg_request_info* info) {
  info->id = r->id;
  info->status = r->status;
  info->task = r->task;
  info->n = r->A.n;
  info->batched = r->batched ? 1 : 0;
  info->nnz_c = r->nnz_c;
  info->products = r->products;
  info->reserved_bytes = r->reserved;
  info->submit_ms = r->submit_ms;
  info->start_ms = r->start_ms;
  info->done_ms = r->done_ms;
}

spg_status spg_server_poll(spg_server* s, uint64_t id, spg_request_info* info) {
  spg::clear_error();
  if (!s || !info) return spg::set_error(SPG_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end()) return spg::set_error(SPG_ERR_INVALID_ARG, "unknown request %llu",
                                                 (unsigned long long)id);
  fill_info(it->second.get(), info);
  return SPG_OK;
}

spg_status spg_server_wait(spg_server* s, uint64_t id, int32_t timeout_ms, spg_request_info* info) {
  spg::clear_error();
  if (!s) return spg::set_error(SPG_ERR_INVALID_ARG, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(id);
  if (it == s->reqs.end())
    return spg::set_error(SPG_ERR_INVALID_ARG, "unknown request %llu", (unsigned long long)id);
  Request* r = it->second.get();
  auto done = [&] { return r->status != SPG_ERR_NOT_READY; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, done);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), done)) {
    if (info) fill_info(r, info);
    return spg::set_error(SPG_ERR_TIMEOUT, "request %llu not done after %d ms",
                          (unsigned long long)id, timeout_ms);
  }
  if (info) fill_info(r, info);
  return SPG_OK;
}

spg_status spg_server_copy_result(spg_server* s, uint64_t id, int64_t* rowptr, int32_t* col,
                                  double* val) {
  spg::clear_error();
  if (!s || !rowptr) return spg::set_error(SPG_ERR_INVALID_ARG, "null argument");
  Request* r = nullptr;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
      return spg::set_error(SPG_ERR_INVALID_ARG, "unknown request %llu", (unsigned long long)id);
    r = it->second.get();
    if (r->status != SPG_OK || !r->rowptr)
      return spg::set_error(SPG_ERR_NOT_READY, "request %llu has no result (status %d)",
                            (unsigned long long)id, r->status);
  }
  cudaError_t e = cudaMemcpy(rowptr, r->rowptr, 8 * ((size_t)r->A.n + 1), cudaMemcpyDefault);
  if (e == cudaSuccess && r->nnz_c > 0) {
    if (!col || !val) return spg::set_error(SPG_ERR_INVALID_ARG, "null col/val");
    e = cudaMemcpy(col, r->col, 4 * (size_t)r->nnz_c, cudaMemcpyDefault);
    if (e == cudaSuccess) e = cudaMemcpy(val, r->val, 8 * (size_t)r->nnz_c, cudaMemcpyDefault);
  }
  if (e != cudaSuccess) return spg::set_error(SPG_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
  return SPG_OK;
}

spg_status spg_server_release(spg_server* s, uint64_t id) {
  spg::clear_error();
  if (!s) return spg::set_error(SPG_ERR_INVALID_ARG, "null server");
  int64_t bytes = 0;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
      return spg::set_error(SPG_ERR_INVALID_ARG, "unknown request %llu", (unsigned long long)id);
    Request* r = it->second.get();
    if (r->status == SPG_ERR_NOT_READY)
      return spg::set_error(SPG_ERR_NOT_READY, "request %llu still running", (unsigned long long)id);
    free_result(r, nullptr);
    bytes = r->reserved;
    r->reserved = 0;
    s->reserved -= bytes;
  }
  s->cv_budget.notify_all();
  return SPG_OK;
}

spg_status spg_server_stats_get(spg_server* s, spg_server_stats* st) {
  spg::clear_error();
  if (!s || !st) return spg::set_error(SPG_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(st, 0, sizeof(*st));
  std::vector<double> lat;
  st->first_submit_ms = -1;
  for (const auto& kv : s->reqs) {
    const Request* r = kv.second.get();
    ++st->submitted;
    if (st->first_submit_ms < 0 || r->submit_ms < st->first_submit_ms) st->first_submit_ms = r->submit_ms;
    if (r->status == SPG_OK) {
      ++st->completed;
      st->products_completed += r->products;
      lat.push_back(r->done_ms - r->submit_ms);
      st->last_done_ms = std::max(st->last_done_ms, r->done_ms);
    } else if (r->status == SPG_ERR_BUDGET) {
      ++st->rejected;
    } else if (r->status != SPG_ERR_NOT_READY) {
      ++st->failed;
    }
  }
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double q) {
    if (lat.empty()) return 0.0;
    size_t i = (size_t)std::min<double>((double)lat.size() - 1, q * (double)(lat.size() - 1) + 0.5);
    return lat[i];
  };
  st->p50_ms = pct(0.50);
  st->p99_ms = pct(0.99);
  st->max_ms = lat.empty() ? 0.0 : lat.back();
  st->batches = s->batches;
  st->budget_bytes = s->cfg.memory_budget_bytes;
  st->reserved_bytes = s->reserved;
  st->peak_reserved_bytes = s->peak;
  return SPG_OK;
}

spg_status spg_server_destroy(spg_server* s) {
  spg::clear_error();
  if (!s) return SPG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_queue.notify_all();
  s->cv_budget.notify_all();
  for (std::thread& t : s->workers) t.join();
  cudaSetDevice(s->device);
  for (auto& kv : s->reqs) free_result(kv.second.get(), nullptr);
  cudaDeviceSynchronize();
  delete s;
  return SPG_OK;
}

}  // extern "C"
