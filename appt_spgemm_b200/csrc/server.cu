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
//  - with two or more workers, worker 0 takes small requests only, so small
//    requests always have a lane and never queue behind large ones; its stream
//    has the highest priority and the other workers' launches use one CTA per
//    work item (no persistent grids), so small requests' CTAs interleave with
//    a large product's instead of waiting for it to finish;
//  - admission is by a device-memory budget that covers every byte the
//    server holds: before planning, a job reserves an upper bound of its plan
//    workspace (spg_plan_workspace_bound, from the input sizes); after the
//    symbolic pass it needs its exact outputs plus the workspace of the plan and
//    of its execute.  A job that can never fit is rejected (a batch is split
//    into its requests first).  A job that does not fit yet holds nothing: its
//    plan is destroyed and it waits, with its exact need, in the worker's
//    waiting list while the worker takes other work; it is planned again and
//    runs as soon as releases make room, oldest first.  The server also counts
//    the bytes it actually holds (plans, execute workspace, results) and keeps
//    their peak, which never exceeds the budget.
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
  double submit_ms = 0, start_ms = 0, planned_ms = 0, run_ms = 0, done_ms = 0;
  int64_t* rowptr = nullptr;
  int32_t* col = nullptr;
  double* val = nullptr;
  int copying = 0;  // spg_server_copy_result calls reading the result right now
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
  std::condition_variable cv_work, cv_done;  // work: queue, budget or stop changed
  std::deque<uint64_t> queue;
  std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
  uint64_t next_id = 1;
  int64_t reserved = 0, peak = 0, batches = 0;
  int64_t held = 0, held_peak = 0;  // bytes of plans, execute workspace and results alive
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

// One unit of work: a single request or a merged batch, planned (symbolic
// done, sizes known) and waiting for its share of the budget.
struct Job {
  std::vector<Request*> rs;
  spg_plan* p = nullptr;
  spg_plan_info info{};
  std::vector<int64_t> row_off, nnz_off, out_r;  // merged batches
  int64_t outs = 0;  // result bytes, reserved until the client releases them
  int64_t temp = 0;  // plan + execute workspace (and, for a batch, the concatenated C)
  int64_t pre = 0;   // reserved before planning: the workspace bound, or the exact need
  bool known = false;  // planned before: pre is the exact need
  int64_t need() const { return outs + temp; }
};

constexpr size_t kMaxWaiting = 4;  // jobs (holding no memory) a worker keeps waiting

void hold(spg_server* s, int64_t bytes) {  // caller holds the lock
  s->held += bytes;
  s->held_peak = std::max(s->held_peak, s->held);
}

// Queue the requests of batch `j` as single-request jobs.  The worker takes
// jobs from the back of `split`, so they go in newest first and run in
// submission order.
void split_into_requests(const Job& j, std::vector<Job>& split) {
  for (auto it = j.rs.rbegin(); it != j.rs.rend(); ++it) {
    Job one;
    one.rs.push_back(*it);
    split.push_back(std::move(one));
  }
}

// Plan `j` (one request or a batch).  Returns false when the job is gone: a
// single request that failed to plan is finished with the error; a batch
// that failed to plan is split into single-request jobs appended to `split`.
bool plan_job(spg_server* s, spg_ctx* ctx, cudaStream_t st, Job& j, std::vector<Job>& split) {
  if (j.rs.size() == 1) {
    Request* r = j.rs[0];
    spg_status rc = spg_plan_create(ctx, r->task, &r->A, st, &j.p);
    if (rc != SPG_OK) {
      std::lock_guard<std::mutex> lk(s->mu);
      finish(s, r, rc, spg_last_error_string());
      return false;
    }
    spg_plan_get_info(j.p, &j.info);
    j.outs = output_bytes(r->A.n, j.info.nnz_c);
    j.temp = j.info.workspace_bytes + j.info.exec_workspace_bytes;
    std::lock_guard<std::mutex> lk(s->mu);
    hold(s, j.info.workspace_bytes);
    r->products = j.info.products;
    r->nnz_c = j.info.nnz_c;
    r->planned_ms = s->now_ms();
    return true;
  }
  std::vector<spg_csr_dev> As;
  for (Request* r : j.rs) As.push_back(r->A);
  spg_status rc = spg_plan_create_batched(ctx, j.rs[0]->task, (int32_t)j.rs.size(), As.data(), st,
                                          &j.p);
  if (rc != SPG_OK) {  // e.g. one bad instance: plan each alone to isolate it
    split_into_requests(j, split);
    return false;
  }
  spg_plan_get_info(j.p, &j.info);
  const size_t b = j.rs.size();
  j.row_off.assign(b + 1, 0);
  j.nnz_off.assign(b + 1, 0);
  j.out_r.assign(b, 0);
  j.outs = 0;  // a batch planned again after waiting counts its outputs afresh
  spg_plan_batch_offsets(j.p, j.row_off.data(), j.nnz_off.data());
  for (size_t i = 0; i < b; ++i) {
    j.out_r[i] = output_bytes(j.rs[i]->A.n, j.nnz_off[i + 1] - j.nnz_off[i]);
    j.outs += j.out_r[i];
  }
  j.temp = output_bytes(j.info.n, j.info.nnz_c) + j.info.workspace_bytes +
           j.info.exec_workspace_bytes;
  std::lock_guard<std::mutex> lk(s->mu);
  hold(s, j.info.workspace_bytes);
  const double t = s->now_ms();
  for (Request* r : j.rs) r->planned_ms = t;
  return true;
}

// Destroy a job's plan and stop counting its workspace.
void drop_plan(spg_server* s, Job& j) {
  if (!j.p) return;
  spg_plan_destroy(j.p);
  j.p = nullptr;
  std::lock_guard<std::mutex> lk(s->mu);
  s->held -= j.info.workspace_bytes;
}

// Execute an admitted job (its need is reserved) and finish its requests.
void run_job(spg_server* s, cudaStream_t st, Job& j) {
  spg_status rc = SPG_OK;
  const bool batch = j.rs.size() > 1;
  const int64_t run_extra = j.temp - j.info.workspace_bytes;  // execute workspace (+ batch C)
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (batch) ++s->batches;
    hold(s, run_extra + j.outs);
    const double t = s->now_ms();
    for (Request* r : j.rs) r->run_ms = t;
    for (size_t b = 0; b < j.rs.size(); ++b) {
      Request* r = j.rs[b];
      r->batched = batch;
      r->reserved = batch ? j.out_r[b] : j.outs;
      if (batch) r->nnz_c = j.nnz_off[b + 1] - j.nnz_off[b];
    }
  }
  if (!batch) {
    Request* r = j.rs[0];
    rc = alloc_result(r, r->A.n, j.info.nnz_c, st);
    spg_csr_out C{r->A.n, 0, r->rowptr, r->col, r->val};
    if (rc == SPG_OK) rc = spg_execute(j.p, &C, st);
  } else {
    Request cat;
    rc = alloc_result(&cat, j.info.n, j.info.nnz_c, st);
    spg_csr_out C{j.info.n, 0, cat.rowptr, cat.col, cat.val};
    if (rc == SPG_OK) rc = spg_execute(j.p, &C, st);
    for (size_t b = 0; b < j.rs.size() && rc == SPG_OK; ++b) {
      Request* r = j.rs[b];
      const int64_t nz = j.nnz_off[b + 1] - j.nnz_off[b];
      rc = alloc_result(r, r->A.n, nz, st);
      if (rc != SPG_OK) break;
      k_rebase<<<(r->A.n + 256) / 256, 256, 0, st>>>(cat.rowptr, j.row_off[b], j.nnz_off[b],
                                                      r->A.n, r->rowptr);
      SPG_COUNT_LAUNCH();
      if (nz > 0) {
        cudaMemcpyAsync(r->col, cat.col + j.nnz_off[b], 4 * (size_t)nz,
                        cudaMemcpyDeviceToDevice, st);
        cudaMemcpyAsync(r->val, cat.val + j.nnz_off[b], 8 * (size_t)nz,
                        cudaMemcpyDeviceToDevice, st);
      }
    }
    free_result(&cat, st);
  }
  if (rc == SPG_OK && cudaStreamSynchronize(st) != cudaSuccess) rc = SPG_ERR_CUDA;
  const std::string err = rc == SPG_OK ? "" : spg_last_error_string();
  drop_plan(s, j);
  if (rc != SPG_OK)
    for (Request* r : j.rs) free_result(r, st);
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->held -= run_extra + (rc == SPG_OK ? 0 : j.outs);
    s->reserved -= j.temp + (rc == SPG_OK ? 0 : j.outs);
    for (size_t b = 0; b < j.rs.size(); ++b) {
      Request* r = j.rs[b];
      if (batch)  // the product count of an instance: the batch total split by output share
        r->products = j.info.nnz_c > 0 ? (int64_t)((double)j.info.products * (double)r->nnz_c /
                                                   (double)j.info.nnz_c) : 0;
      if (rc != SPG_OK) r->reserved = 0;
      finish(s, r, rc, rc == SPG_OK ? nullptr : err.c_str());
    }
  }
  s->cv_work.notify_all();  // budget returned
  s->cv_done.notify_all();
}

// Take the oldest queued request this worker may serve (the small-request
// lane serves only n < batch_rows) and, if it is small, the other queued
// small requests of the same task, up to batch_max.  Caller holds the lock.
bool take_requests(spg_server* s, bool small_only, std::vector<Request*>& rs) {
  auto it = s->queue.begin();
  for (; it != s->queue.end(); ++it)
    if (!small_only || s->reqs[*it]->A.n < s->cfg.batch_rows) break;
  if (it == s->queue.end()) return false;
  Request* r = s->reqs[*it].get();
  s->queue.erase(it);
  rs.push_back(r);
  if (r->A.n < s->cfg.batch_rows) {
    for (auto q = s->queue.begin(); q != s->queue.end() && (int)rs.size() < s->cfg.batch_max;) {
      Request* x = s->reqs[*q].get();
      if (x->task == r->task && x->A.n < s->cfg.batch_rows) {
        rs.push_back(x);
        q = s->queue.erase(q);
      } else {
        ++q;
      }
    }
  }
  const double t = s->now_ms();
  for (Request* x : rs) x->start_ms = t;
  return true;
}

// Admission before planning: reserve `pre` (the workspace bound of a new job,
// or the exact need of one planned before).  A job whose `pre` exceeds the
// whole budget can never run: a batch is split into its requests, a single
// request is rejected.
enum class Admit { kRun, kWait, kRejected };
Admit admit_pre(spg_server* s, Job& j, std::vector<Job>& split) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (j.pre > s->cfg.memory_budget_bytes) {
    if (j.rs.size() > 1) {
      split_into_requests(j, split);
    } else {
      finish(s, j.rs[0], SPG_ERR_BUDGET, "request exceeds the memory budget");
    }
    return Admit::kRejected;
  }
  if (s->reserved + j.pre <= s->cfg.memory_budget_bytes) {
    s->reserved += j.pre;
    s->peak = std::max(s->peak, s->reserved);
    return Admit::kRun;
  }
  return Admit::kWait;
}

// Admission after planning (its `pre` is reserved): trade it for the exact
// need.  kRun: the need is reserved.  kWait: the need does not fit now; `pre`
// is returned and becomes the need (the caller drops the plan and keeps the
// job waiting).  kRejected: the need exceeds the whole budget.
Admit admit_planned(spg_server* s, Job& j, std::vector<Job>& split) {
  std::lock_guard<std::mutex> lk(s->mu);
  s->reserved -= j.pre;
  if (j.need() > s->cfg.memory_budget_bytes) {
    if (j.rs.size() > 1) {
      split_into_requests(j, split);
    } else {
      finish(s, j.rs[0], SPG_ERR_BUDGET, "request exceeds the memory budget");
    }
    return Admit::kRejected;
  }
  if (s->reserved + j.need() <= s->cfg.memory_budget_bytes) {
    s->reserved += j.need();
    s->peak = std::max(s->peak, s->reserved);
    return Admit::kRun;
  }
  j.pre = j.need();
  j.known = true;
  return Admit::kWait;
}

void worker_main(spg_server* s, int index) {
  cudaSetDevice(s->device);
  // with two or more workers, worker 0 serves small requests only, so they
  // are never queued behind large ones; its stream has the highest priority
  // and the other workers launch one CTA per work item, so the small
  // requests' CTAs start as soon as any of the large ones retire
  const bool small_only = s->cfg.workers >= 2 && index == 0;
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  cudaStream_t st = nullptr;
  cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, small_only ? greatest : least);
  spg_config cfg{};
  cfg.struct_size = sizeof(spg_config);
  cfg.device = s->device;
  cfg.pool_release_bytes = 64ll << 20;  // give freed memory back: the budget is global
  if (s->cfg.workers >= 2 && !small_only) cfg.grid_sms = 1 << 16;
  if (small_only) cfg.bin_streams = 1;  // every launch on the lane's high-priority stream
  spg_ctx* ctx = nullptr;
  const bool ok = spg_create(&ctx, &cfg) == SPG_OK;
  std::deque<Job> waiting;  // admitted to nothing, holding no memory, oldest first
  std::vector<Job> todo;    // taken or split off, to be admitted and planned
  for (;;) {
    Job job;
    bool reserved = false;  // job.pre is reserved
    if (todo.empty()) {
      std::unique_lock<std::mutex> lk(s->mu);
      bool have = false;
      for (;;) {
        if (!waiting.empty() &&
            s->reserved + waiting.front().pre <= s->cfg.memory_budget_bytes) {
          job = std::move(waiting.front());
          waiting.pop_front();
          s->reserved += job.pre;
          s->peak = std::max(s->peak, s->reserved);
          reserved = have = true;
          break;
        }
        std::vector<Request*> rs;
        if (waiting.size() < kMaxWaiting && take_requests(s, small_only, rs)) {
          job.rs = std::move(rs);
          have = true;
          break;
        }
        if (s->stopping) break;
        s->cv_work.wait(lk);
      }
      if (!have) {  // stopping: what still waits does not run
        for (Job& j : waiting)
          for (Request* r : j.rs) finish(s, r, SPG_ERR_CUDA, "server stopped before the request ran");
        waiting.clear();
        lk.unlock();
        s->cv_done.notify_all();
        break;
      }
    } else {
      job = std::move(todo.back());
      todo.pop_back();
    }
    if (!ok) {
      std::lock_guard<std::mutex> lk(s->mu);
      if (reserved) s->reserved -= job.pre;
      for (Request* r : job.rs) finish(s, r, SPG_ERR_CUDA, "worker context could not be created");
      s->cv_done.notify_all();
      continue;
    }
    if (!reserved) {
      std::vector<spg_csr_dev> As;
      for (Request* r : job.rs) As.push_back(r->A);
      if (spg_plan_workspace_bound(ctx, job.rs[0]->task, (int32_t)As.size(), As.data(),
                                   As.size() > 1 ? 1 : 0, &job.pre) != SPG_OK)
        job.pre = 0;
      const Admit a = admit_pre(s, job, todo);
      if (a == Admit::kRejected) {
        s->cv_done.notify_all();
        continue;
      }
      if (a == Admit::kWait) {
        waiting.push_back(std::move(job));
        continue;
      }
    }
    const int64_t pre = job.pre;
    if (!plan_job(s, ctx, st, job, todo)) {  // failed: finished or split
      {
        std::lock_guard<std::mutex> lk(s->mu);
        s->reserved -= pre;
      }
      s->cv_work.notify_all();
      s->cv_done.notify_all();
      continue;
    }
    switch (admit_planned(s, job, todo)) {
      case Admit::kRun:
        run_job(s, st, job);
        break;
      case Admit::kWait:
        drop_plan(s, job);
        waiting.push_back(std::move(job));
        s->cv_work.notify_all();  // its workspace reservation was returned
        break;
      case Admit::kRejected:
        drop_plan(s, job);
        s->cv_work.notify_all();
        s->cv_done.notify_all();
        break;
    }
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
  s->cv_work.notify_all();  // any worker may be the one allowed to take it
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
  info->planned_ms = r->planned_ms;
  info->run_ms = r->run_ms;
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
    if (r->nnz_c > 0 && (!col || !val)) return spg::set_error(SPG_ERR_INVALID_ARG, "null col/val");
    // pin the result: spg_server_release waits until no copy reads it
    ++r->copying;
  }
  cudaError_t e = cudaMemcpy(rowptr, r->rowptr, 8 * ((size_t)r->A.n + 1), cudaMemcpyDefault);
  if (e == cudaSuccess && r->nnz_c > 0) {
    e = cudaMemcpy(col, r->col, 4 * (size_t)r->nnz_c, cudaMemcpyDefault);
    if (e == cudaSuccess) e = cudaMemcpy(val, r->val, 8 * (size_t)r->nnz_c, cudaMemcpyDefault);
  }
  {
    std::lock_guard<std::mutex> lk(s->mu);
    --r->copying;
  }
  s->cv_done.notify_all();
  if (e != cudaSuccess) return spg::set_error(SPG_ERR_CUDA, "copy: %s", cudaGetErrorString(e));
  return SPG_OK;
}

spg_status spg_server_release(spg_server* s, uint64_t id) {
  spg::clear_error();
  if (!s) return spg::set_error(SPG_ERR_INVALID_ARG, "null server");
  int64_t bytes = 0;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end())
      return spg::set_error(SPG_ERR_INVALID_ARG, "unknown request %llu", (unsigned long long)id);
    Request* r = it->second.get();
    if (r->status == SPG_ERR_NOT_READY)
      return spg::set_error(SPG_ERR_NOT_READY, "request %llu still running", (unsigned long long)id);
    // copies of this result started by other threads finish first
    s->cv_done.wait(lk, [&] { return r->copying == 0; });
    free_result(r, nullptr);
    bytes = r->reserved;
    r->reserved = 0;
    s->reserved -= bytes;
    s->held -= bytes;
  }
  s->cv_work.notify_all();
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
  st->held_bytes = s->held;
  st->peak_held_bytes = s->held_peak;
  return SPG_OK;
}

spg_status spg_server_destroy(spg_server* s) {
  spg::clear_error();
  if (!s) return SPG_OK;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stopping = true;
  }
  s->cv_work.notify_all();
  for (std::thread& t : s->workers) t.join();
  cudaSetDevice(s->device);
  for (auto& kv : s->reqs) free_result(kv.second.get(), nullptr);
  cudaDeviceSynchronize();
  delete s;
  return SPG_OK;
}

}  // extern "C"
