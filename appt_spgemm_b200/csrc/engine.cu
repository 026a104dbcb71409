// Host orchestration of the engine: context, plan (pre-pass + binning +
// symbolic), execute (numeric + mirror), multiply, transpose, descriptors and
// the run_ours-compatible call.
//
// The reference's run_ours (src/spgemm_engine.cuh:132-210) allocates and frees
// every buffer per call, issues at least two blocking 8-byte device→host copies
// per phase and hands C to nobody.  Here workspace comes from a per-context
// stream-ordered memory pool, the plan makes two host synchronisations (the
// validation verdict with the bin sizes, then nnz(C); one for small matrices),
// and execute is fully asynchronous and writes C into caller-visible CSR
// arrays.
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <algorithm>
#include <vector>

#include "kernels.h"

namespace spg {
thread_local long long g_kernel_launches = 0;
}

using namespace spg;

struct ProfEntry {
  std::string label;
  cudaEvent_t a, b;
};

struct spg_ctx {
  int device = 0;
  int num_sms = 148;               // SMs the launches size grids for (grid_sms or the device's)
  int device_sms = 148;
  cudaMemPool_t pool = nullptr;
  spg_config cfg{};
  uint32_t* d_status = nullptr;   // device status word (+ scratch, 256 B)
  int64_t* h_pin = nullptr;       // pinned readback area (512 B)
  // profiling: per-kernel events on the launching stream, resolved on read
  bool prof = false;
  std::vector<ProfEntry> pending;
  std::map<std::string, std::pair<double, long long>> prof_acc;
  int32_t tune_timed = 0, tune_pruned = 0;  // the last spg_autotune's candidates
  // concurrent bin launches: side streams forked from the caller's stream
  static constexpr int kMaxSides = 8;
  cudaStream_t side[kMaxSides] = {};
  cudaEvent_t side_done[kMaxSides] = {};
  cudaEvent_t fork_ev = nullptr;
  int nsides = 0;
  std::vector<cudaEvent_t> event_pool;
  long long launch_base = 0;
};

namespace {

cudaEvent_t prof_event(spg_ctx* c) {
  if (!c->event_pool.empty()) {
    cudaEvent_t e = c->event_pool.back();
    c->event_pool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Brackets the kernels launched in its scope with CUDA events when profiling
// is on; the label names the phase and kernel ("num/bin5", "sym/heavy", ...).
struct ProfScope {
  spg_ctx* c;
  cudaStream_t s;
  std::string label;
  cudaEvent_t a = nullptr;
  ProfScope(spg_ctx* ctx, const char* l, cudaStream_t st, int bin = -1) : c(ctx), s(st) {
    if (!c->prof) return;
    label = l;
    if (bin >= 0) label += std::to_string(bin);
    a = prof_event(c);
    cudaEventRecord(a, s);
  }
  ~ProfScope() {
    if (!a) return;
    cudaEvent_t b = prof_event(c);
    cudaEventRecord(b, s);
    c->pending.push_back(ProfEntry{label, a, b});
  }
};

// Launches of different row bins of one phase touch disjoint rows, so they may
// overlap: each bin gets the next side stream (forked from the caller's stream
// by an event, so it starts after everything queued there), and join() makes
// the caller's stream wait for all of them.  With one bin, or bin_streams 1,
// everything stays on the caller's stream.  Fork and join are events, which a
// stream capture records as graph edges.
struct BinFork {
  spg_ctx* c;
  cudaStream_t main;
  int ns;  // side streams in use
  bool on;
  int used = 0;
  BinFork(spg_ctx* ctx, cudaStream_t st, int launches)
      : c(ctx), main(st), ns(std::min(ctx->nsides, (int)ctx->cfg.bin_streams)),
        on(launches > 1 && ns > 1) {
    if (on && cudaEventRecord(c->fork_ev, main) != cudaSuccess) on = false;
  }
  cudaStream_t next() {
    if (!on) return main;
    const int i = used % ns;
    if (used < ns) cudaStreamWaitEvent(c->side[i], c->fork_ev, 0);
    ++used;
    return c->side[i];
  }
  cudaError_t join() {
    if (!on) return cudaSuccess;
    const int k = used < ns ? used : ns;
    for (int i = 0; i < k; ++i) {
      cudaError_t e = cudaEventRecord(c->side_done[i], c->side[i]);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(main, c->side_done[i], 0);
      if (e != cudaSuccess) return e;
    }
    on = false;
    return cudaSuccess;
  }
  ~BinFork() { join(); }
};

void prof_resolve(spg_ctx* c) {
  for (ProfEntry& e : c->pending) {
    float ms = 0.f;
    cudaEventSynchronize(e.b);
    cudaEventElapsedTime(&ms, e.a, e.b);
    auto& slot = c->prof_acc[e.label];
    slot.first += ms;
    slot.second += 1;
    c->event_pool.push_back(e.a);
    c->event_pool.push_back(e.b);
  }
  c->pending.clear();
}

}  // namespace

struct spg_plan {
  spg_ctx* ctx = nullptr;
  spg_task task = SPG_TASK_AA;
  cudaStream_t stream = nullptr;
  MatView A{}, B{};
  int32_t n = 0;
  int G = 8;
  int64_t* f = nullptr;
  int32_t* lo = nullptr;
  int32_t* hi = nullptr;
  int32_t* rownnz = nullptr;
  int32_t* rowlow = nullptr;
  int64_t* rowptr = nullptr;
  int64_t* lowptr = nullptr;
  int32_t* rows_num = nullptr;
  int64_t num_count[kNumBins] = {};
  int64_t num_start[kNumBins] = {};
  int64_t nnz_c = 0;
  int64_t nnz_low = 0;
  spg_plan_info info{};
  std::vector<void*> ptrs;
  int64_t ws_bytes = 0;
  cudaEvent_t exec_done = nullptr;
  // batched plans: instance offsets in the block-diagonal layout
  int32_t count = 0;
  const int32_t* colbase = nullptr;
  std::vector<int64_t> row_off, nnz_off;
  const BatchDesc* d_desc = nullptr;       // instance table on the device
  const int64_t* d_nnz_off = nullptr;
  double* batch_val = nullptr;             // values of the block-diagonal copy
  // A·Aᵀ: how B's values were derived, to redo it when A's values change
  bool symmetric = false;
  TransposeWork tw{};
  int32_t *bt_rowptr = nullptr, *bt_col = nullptr;
  double* bt_val = nullptr;
  // derived values (block-diagonal copy, Aᵀ) still match A: true right after
  // planning; every later execute recomputes them from A's current values
  bool values_fresh = true;
  // heavy rows: per-block distinct-column counts from the symbolic phase
  // (nullptr when their number exceeds heavy_block_budget: the numeric phase
  // then takes the CTA dense-window kernel) and the windowed kernel's cursors
  int64_t* blk_off = nullptr;
  uint16_t* blk_cnt = nullptr;
  int blk_log2 = 12;
  bool heavy_windows = false;  // the windowed heavy kernel runs: execute takes its cursors
  // one-readback plan: every row in one warp-per-row launch per phase, the
  // numeric one with tables of 2^small_log2 slots
  bool small = false;
  int small_log2 = 6;
  int32_t* hqueue = nullptr;  // next row of the CTA-per-row kernels, one counter per bin
                              // (zeroed before each launch; bins may run at once)
  int window_bits = 1 << 20;  // heavy-path shape (heavy_shape)
  int heavy_threads = 1024;
};

struct spg_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
};

namespace {

// Entry of every device-facing call: clear the thread's last error text and a
// pending non-sticky CUDA error left by earlier, unrelated runtime calls, so
// that launch checks below report only this call's failures.
void begin_call() {
  clear_error();
  cudaGetLastError();
}

spg_status cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return SPG_OK;
  cudaGetLastError();  // clear a sticky launch error where possible
  if (e == cudaErrorMemoryAllocation)
    return set_error(SPG_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return set_error(SPG_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define TRY_CUDA(expr, what)                               \
  do {                                                     \
    cudaError_t e_ = (expr);                               \
    if (e_ != cudaSuccess) return cuda_status(e_, (what)); \
  } while (0)

#define TRY(expr)                   \
  do {                              \
    spg_status s_ = (expr);         \
    if (s_ != SPG_OK) return s_;    \
  } while (0)

spg_status status_from_bits(uint32_t bits) {
  if (bits == 0) return SPG_OK;
  if (bits & DEV_ERR_INVALID_CSR)
    return set_error(SPG_ERR_INVALID_CSR,
                     "input CSR invalid: rowptr must start at 0, be monotone and end at nnz; "
                     "columns must lie in [0,n) and strictly increase within each row");
  if (bits & DEV_ERR_HASH_FULL) return set_error(SPG_ERR_HASH_FULL, "a hash table probe ran out");
  if (bits & DEV_ERR_OVERFLOW)
    return set_error(SPG_ERR_CUDA, "a row produced more entries than its symbolic count");
  return set_error(SPG_ERR_CUDA, "device status word 0x%x", bits);
}

// The one-readback plan takes A·A and A·Aᵀ of matrices up to these sizes.
constexpr int64_t kSmallMaxNnzDefault = (int64_t)1 << 20;
constexpr int32_t kSmallMaxN = 65536;
// Its symbolic table (2^11 slots per warp) holds rows of up to this many
// products at 75% load; a larger row sends the plan to the regular path.
constexpr int kSmallSymLog2 = 11;
constexpr int64_t kSmallCap = 1536;

spg_config merged_config(const spg_config* user) {
  spg_config c{};
  if (user && user->struct_size >= (int32_t)sizeof(int32_t)) {
    size_t sz = (size_t)user->struct_size < sizeof(spg_config) ? (size_t)user->struct_size
                                                               : sizeof(spg_config);
    std::memcpy(&c, user, sz);
  }
  c.struct_size = sizeof(spg_config);
  if (c.max_smem_slots <= 0) c.max_smem_slots = 8192;
  // 0 = chosen per plan from n (heavy_shape)
  if (c.heavy_threads < 0) c.heavy_threads = 0;
  if (c.heavy_threads > 1024) c.heavy_threads = 1024;
  c.heavy_threads = (c.heavy_threads + 31) / 32 * 32;
  // windows are whole 4-word groups and fit the shared bitmap (≤ 2^20 bits)
  if (c.window_bits < 0) c.window_bits = 0;
  if (c.window_bits > (1 << 20)) c.window_bits = 1 << 20;
  c.window_bits = (c.window_bits + 1023) / 1024 * 1024;
  auto clamp_pct = [](int32_t v, int32_t dflt) { return v <= 0 ? dflt : (v < 20 ? 20 : (v > 90 ? 90 : v)); };
  c.sym_load_pct = clamp_pct(c.sym_load_pct, 75);
  c.num_load_pct = clamp_pct(c.num_load_pct, 66);
  if (c.lanes_per_row != 0 && c.lanes_per_row != 4 && c.lanes_per_row != 8 &&
      c.lanes_per_row != 16 && c.lanes_per_row != 32)
    c.lanes_per_row = 0;
  if (c.heavy_block_budget <= 0) c.heavy_block_budget = (int64_t)1 << 27;  // 256 MB of counts
  if (c.grid_sms < 0) c.grid_sms = 0;
  if (c.grid_sms > (1 << 16)) c.grid_sms = 1 << 16;
  if (c.small_max_nnz == 0) c.small_max_nnz = kSmallMaxNnzDefault;
  if (c.dense_max_words == 0) c.dense_max_words = -1;  // off unless asked for
  if (c.bin_streams <= 0) c.bin_streams = 1;  // one stream unless asked for
  if (c.bin_streams > 4) c.bin_streams = 4;
  if (c.dense_max_words > ((int64_t)1 << kDenseMaxLog2W))
    c.dense_max_words = (int64_t)1 << kDenseMaxLog2W;
  if (c.heavy_vcap == 0) c.heavy_vcap = -1;  // in place in C unless asked for
  if (c.heavy_vcap > 0) {  // a power of two in [1024, 16384]
    int64_t v = 1024;
    while (v * 2 <= c.heavy_vcap && v < 16384) v *= 2;
    c.heavy_vcap = v;
  }
  return c;
}

// Heavy-path shape of a plan: the bitmap window covers the whole column range
// when it can (next power of two >= n, at most 2^20), and windows of up to
// 2^19 columns run 512-thread CTAs, two per SM, so one CTA's barrier waits
// overlap the other's work (R-MAT 2^18: heavy numeric 80.6 -> 70.4 ms); a
// 2^20 window keeps one 1024-thread CTA per SM.  Explicit config values win.
void heavy_shape(const spg_config& c, int32_t n, int* window_bits, int* threads) {
  int wb = c.window_bits;
  if (wb <= 0) {
    wb = 1024;
    while (wb < n && wb < (1 << 20)) wb <<= 1;
  }
  *window_bits = wb;
  *threads = c.heavy_threads > 0 ? c.heavy_threads : (wb <= (1 << 19) ? 512 : 1024);
}

int grid_sms_of(const spg_config& c, int device_sms) {
  return c.grid_sms > 0 ? (int)c.grid_sms : device_sms;
}

constexpr int64_t kHeavySplitDefault = 128;  // mean B-row length

// Smallest exact row count that the numeric binning sends to the heavy path
// (table of more than 2^num_lg slots at num_load percent).
int64_t numeric_heavy_min(int num_lg, int num_load) {
  int64_t l = 1, h = (int64_t)1 << 40;
  while (l < h) {
    const int64_t mid = (l + h) / 2;
    int lg = ceil_log2_64(mid * 100 / num_load + 1);
    if (lg < kMinTableLog2) lg = kMinTableLog2;
    if (lg > num_lg) h = mid; else l = mid + 1;
  }
  return l;
}

// Windows of the heavy numeric kernel: at most this many distinct columns,
// within its table's load limit and the radix sort's room (3m <= 2T,
// m + 256 <= T); blocks above it are cut into windows of 2^sub_log2 columns.
int heavy_cap(int num_load) {
  const int T = 1 << kHeavyTableLog2;
  int cap = (int)((int64_t)T * num_load / 100);
  cap = std::min(cap, 2 * T / 3);
  cap = std::min(cap, T - 256);
  return std::max(cap, 32);
}

int table_log2_cap(int slots) {
  int lg = ceil_log2_64(slots < 16 ? 16 : slots);
  if (lg > kMaxTableLog2) lg = kMaxTableLog2;
  if ((1 << lg) > slots && lg > kMinTableLog2) --lg;  // largest power of two <= slots
  return lg;
}

template <class T>
spg_status palloc(spg_plan* p, T** out, int64_t count) {
  size_t bytes = sizeof(T) * (size_t)(count > 0 ? count : 1);
  void* ptr = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&ptr, bytes, p->ctx->pool, p->stream);
  if (e != cudaSuccess) return cuda_status(e, "workspace allocation");
  p->ptrs.push_back(ptr);
  p->ws_bytes += (int64_t)bytes;
  *out = (T*)ptr;
  return SPG_OK;
}

spg_status check_matrix(const spg_csr_dev* A) {
  if (!A) return set_error(SPG_ERR_INVALID_ARG, "null matrix");
  if (A->n < 0 || A->nnz < 0) return set_error(SPG_ERR_INVALID_ARG, "negative n or nnz");
  if (A->nnz > INT32_MAX)
    return set_error(SPG_ERR_UNSUPPORTED, "nnz(A) = %lld exceeds int32 row pointers",
                     (long long)A->nnz);
  if (!A->rowptr) return set_error(SPG_ERR_INVALID_ARG, "null rowptr");
  if (A->nnz > 0 && (!A->col || !A->val)) return set_error(SPG_ERR_INVALID_ARG, "null col/val");
  return SPG_OK;
}

// Validate A on the device and wait for the verdict (spg_describe).
// When sym_tval is given, the values of Aᵀ for a structurally symmetric A are
// gathered in the same round trip and *symmetric tells whether that held.
spg_status validate_device(spg_ctx* ctx, const MatView& A, cudaStream_t st,
                           double* sym_tval = nullptr, bool* symmetric = nullptr) {
  TRY_CUDA(cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(uint32_t), st), "status reset");
  {
    ProfScope ps(ctx, "plan/validate", st);
    TRY_CUDA(launch_validate(A, ctx->d_status, st), "validate");
  }
  if (sym_tval) {
    ProfScope ps(ctx, "plan/transpose_sym", st);
    TRY_CUDA(launch_sym_transpose_vals(A, sym_tval, (int*)(ctx->d_status + 1), st),
             "symmetric transpose");
  }
  TRY_CUDA(cudaMemcpyAsync(ctx->h_pin, ctx->d_status, 2 * sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, st), "status readback");
  TRY_CUDA(cudaStreamSynchronize(st), "validate sync");
  const uint32_t* h = (const uint32_t*)ctx->h_pin;
  if (symmetric) *symmetric = h[1] == 0;
  return status_from_bits(h[0]);
}

// Bytes execute_impl takes from the pool for the duration of an execute for
// the Gram mirror: its cursors, lower parts and segment-sort list (0 for the
// other tasks; the heavy rows' cursors are added by the caller).
int64_t exec_workspace(int64_t n, bool gram, int64_t nnz_low) {
  if (!gram) return 0;
  const int64_t nn = n > 0 ? n : 1;
  return 4 * nn + 12 * (nnz_low > 0 ? nnz_low : 1) + 4 * nn + 4;
}

// Upper bound of the workspace plan_build allocates (a plan's workspace_bytes)
// for a matrix of n rows and nnz entries, from the sizes alone: every palloc of
// plan_build at its largest (the transpose counted whenever the task needs
// Aᵀ, the heavy-row counts and cursors always).  The serving loop reserves it
// against its budget before planning.
int64_t plan_workspace_bound(const spg_config& cfg, spg_task task, int64_t n, int64_t nnz) {
  const int64_t nn = n > 0 ? n : 1, nz = nnz > 0 ? nnz : 1;
  const int64_t scan = (int64_t)scan_tmp_bytes(n);
  const int64_t nblocks = (n + kBinRowsPerBlock - 1) / kBinRowsPerBlock;
  int64_t b = 0;
  if (task != SPG_TASK_AA) {
    b += 8 * nz;                                  // values of Aᵀ
    b += 4 * (nn + 1) + 4 * nz + 4 * nn + 4 * nn  // Aᵀ rowptr/col, counts, cursors
         + scan + 4 * nz + 8 * nz + 4 * nn + 4;   // scan, staging copy, long list
  }
  b += 8 * nn + 4 * nn + 4 * nn + 4;                              // f, lo, hi, queue
  b += 4 * kNumBins * (nblocks > 0 ? nblocks : 1) + 8 * 4 * kNumBins + 4 * nn;  // binning
  b += 4 * nn + 8 * (nn + 1) + scan;                              // heavy block offsets
  const int64_t per_row_blocks = (nn + 1023) / 1024 + 1;
  const int64_t blocks = nn > cfg.heavy_block_budget / per_row_blocks ? cfg.heavy_block_budget
                                                                      : nn * per_row_blocks;
  b += 2 * blocks;                                                // heavy block counts
  b += 4 * nn;                                                    // row counts
  if (task == SPG_TASK_AATS) b += 4 * nn + scan + 8 * (nn + 1);   // lower counts, offsets
  b += scan + 8 * (nn + 1);                                       // C row pointers
  b += 4 * nn + 32;                                               // numeric rows, stats
  return b + 64 * 1024;  // pool rounding of the ~40 allocations
}

void plan_free(spg_plan* p) {
  if (!p) return;
  if (p->exec_done) {
    cudaStreamWaitEvent(p->stream, p->exec_done, 0);
    cudaEventDestroy(p->exec_done);
  }
  for (void* ptr : p->ptrs) cudaFreeAsync(ptr, p->stream);
  delete p;
}

// The plan of a small A·A or A·Aᵀ with one host synchronisation.  The regular
// plan waits three times (validation verdict, bin sizes, nnz(C)); on a
// matrix of a few thousand rows those round trips and the per-bin launches
// are most of the call.  Here every kernel runs before the verdict is known
// (the pre-pass and the transpose check every index they use; a row with an
// invalid index gets f = −1 and is skipped), every row takes one
// warp-per-row symbolic launch with a 2048-slot table, and one readback
// brings the verdict, nnz(C) and the row statistics together.  A·Aᵀ always
// uses the counting-sort transpose (no symmetric-pattern shortcut, which would
// need the verdict first).  A row of more than kSmallCap products reports
// DEV_ERR_SMALL_CAP, and the caller plans again on the regular path
// (*fallback).  Execute then runs one numeric launch over all rows.
spg_status plan_build_small(spg_plan* p, const spg_csr_dev* Ad, bool* fallback) {
  *fallback = false;
  spg_ctx* ctx = p->ctx;
  cudaStream_t st = p->stream;
  const int32_t n = Ad->n;
  const int64_t nnz = Ad->nnz;
  const bool aat = p->task == SPG_TASK_AAT;
  p->small = true;
  p->n = n;
  p->A = MatView{n, nnz, Ad->rowptr, Ad->col, Ad->val};
  p->info.n = n;
  p->info.task = p->task;
  p->info.nnz_a = nnz;
  // one allocation, carved into 256-byte aligned pieces
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off += (bytes + 255) & ~(size_t)255;
    return o;
  };
  const size_t nn = (size_t)(n > 0 ? n : 1), nz = (size_t)(nnz > 0 ? nnz : 1);
  const size_t o_f = take(8 * nn), o_lo = take(4 * nn), o_hi = take(4 * nn),
               o_cnt = take(4 * nn), o_rp = take(8 * (nn + 1)), o_scan = take(scan_tmp_bytes(n)),
               o_stats = take(32), o_q = take(4 * kNumBins);
  size_t o_bp = 0, o_bi = 0, o_bx = 0, o_tc = 0, o_tu = 0, o_ts = 0, o_tk = 0, o_tv = 0,
         o_ll = 0, o_lc = 0;
  if (aat) {
    o_bp = take(4 * (nn + 1));
    o_bi = take(4 * nz);
    o_bx = take(8 * nz);
    o_tc = take(4 * nn);
    o_tu = take(4 * nn);
    o_ts = take(scan_tmp_bytes(n));
    o_tk = take(4 * nz);
    o_tv = take(8 * nz);
    o_ll = take(4 * nn);
    o_lc = take(4);
  }
  char* w = nullptr;
  TRY(palloc(p, &w, (int64_t)off));
  p->f = (int64_t*)(w + o_f);
  p->lo = (int32_t*)(w + o_lo);
  p->hi = (int32_t*)(w + o_hi);
  p->rownnz = (int32_t*)(w + o_cnt);
  p->rowptr = (int64_t*)(w + o_rp);
  p->hqueue = (int32_t*)(w + o_q);
  unsigned long long* stats = (unsigned long long*)(w + o_stats);
  TRY_CUDA(cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(uint32_t), st), "status reset");
  if (aat) {
    TransposeWork tw{};
    tw.cnt = (int32_t*)(w + o_tc);
    tw.cursor = (int32_t*)(w + o_tu);
    tw.scan_tmp = (void*)(w + o_ts);
    tw.tmp_col = (int32_t*)(w + o_tk);
    tw.tmp_val = (double*)(w + o_tv);
    tw.long_list = (int32_t*)(w + o_ll);
    tw.long_count = (int32_t*)(w + o_lc);
    tw.status = ctx->d_status;
    p->bt_rowptr = (int32_t*)(w + o_bp);
    p->bt_col = (int32_t*)(w + o_bi);
    p->bt_val = (double*)(w + o_bx);
    // slots an invalid input leaves unwritten hold column 0, so the row sort
    // stays in range; the plan then fails on the verdict
    TRY_CUDA(cudaMemsetAsync(tw.tmp_col, 0, 4 * nz, st), "memset");
    ProfScope ps(ctx, "plan/transpose", st);
    TRY_CUDA(launch_transpose(p->A, p->bt_rowptr, p->bt_col, p->bt_val, tw, ctx->num_sms, st),
             "transpose");
    p->tw = tw;
    p->B = MatView{n, nnz, p->bt_rowptr, p->bt_col, p->bt_val};
  } else {
    p->B = p->A;
  }
  {  // the pre-pass also validates A
    ProfScope ps(ctx, "plan/prepass", st);
    TRY_CUDA(launch_prepass(p->A, p->B, p->f, p->lo, p->hi, st, ctx->d_status), "prepass");
  }
  RowArgs ra{};
  ra.A = p->A;
  ra.B = p->B;
  ra.rows = nullptr;
  ra.nrows = n;
  ra.G = 32;
  ra.rownnz = p->rownnz;
  ra.status = ctx->d_status;
  ra.lo = p->lo;
  ra.hi = p->hi;
  ra.fsmall = p->f;
  ra.fcap = kSmallCap;
  if (n > 0) {
    ProfScope ps(ctx, "sym/small", st);
    TRY_CUDA(launch_hash_w32(kSmallSymLog2, false, false, ra, ctx->num_sms, st), "symbolic");
  }
  {
    ProfScope ps(ctx, "plan/scan", st);
    TRY_CUDA(launch_scan_stats_small(p->rownnz, p->f, n, p->rowptr, stats, w + o_scan, st),
             "row pointer scan");
  }
  int64_t* hp = ctx->h_pin;
  TRY_CUDA(cudaMemcpyAsync(hp, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st),
           "readback");
  TRY_CUDA(cudaMemcpyAsync(hp + 1, p->rowptr + n, sizeof(int64_t), cudaMemcpyDeviceToHost, st),
           "readback");
  TRY_CUDA(cudaMemcpyAsync(hp + 2, stats, sizeof(unsigned long long) * 3, cudaMemcpyDeviceToHost,
                           st), "readback");
  TRY_CUDA(cudaStreamSynchronize(st), "plan sync");
  const uint32_t bits = *(const uint32_t*)hp;
  if (bits & DEV_ERR_INVALID_CSR) return status_from_bits(DEV_ERR_INVALID_CSR);
  if (bits & DEV_ERR_SMALL_CAP) {
    *fallback = true;
    return SPG_OK;
  }
  TRY(status_from_bits(bits));
  const unsigned long long* sv = (const unsigned long long*)(hp + 2);
  p->nnz_c = n > 0 ? hp[1] : 0;
  p->info.nnz_c = p->nnz_c;
  p->info.products = (int64_t)sv[0];
  p->info.products_computed = (int64_t)sv[0];
  p->info.max_row_products = (int64_t)sv[1];
  p->info.max_row_nnz = (int64_t)sv[2];
  p->info.heavy_rows = 0;
  p->info.bins_used = 1;
  p->info.symmetric_pattern = 0;
  // numeric table: the exact largest row at the numeric load, 16 to 2048
  // slots; tables below 2048 slots run rows on lane groups sized to B's mean
  // row length (several rows per warp), 2048 a warp per row
  int lg = ceil_log2_64((int64_t)sv[2] * 100 / ctx->cfg.num_load_pct + 1);
  p->small_log2 = lg < kMinTableLog2 ? kMinTableLog2 : (lg > 11 ? 11 : lg);
  if (ctx->cfg.lanes_per_row > 0) {
    p->G = ctx->cfg.lanes_per_row;
  } else {
    const double mean = n > 0 ? (double)nnz / n : 1.0;
    int g = 4;
    while (g < 32 && g < mean) g <<= 1;
    p->G = g;
  }
  p->info.output_bytes = 8 * ((int64_t)n + 1) + 12 * p->nnz_c;
  p->info.workspace_bytes = p->ws_bytes;
  p->info.exec_workspace_bytes = 0;
  return SPG_OK;
}

bool small_plan_eligible(const spg_ctx* ctx, spg_task task, const spg_csr_dev* A) {
  const spg_config& c = ctx->cfg;
  return (task == SPG_TASK_AA || task == SPG_TASK_AAT) && c.small_max_nnz > 0 &&
         A->nnz <= c.small_max_nnz && A->n <= kSmallMaxN && !c.force_heavy;
}

spg_status plan_build(spg_plan* p, const spg_csr_dev* Ad) {
  spg_ctx* ctx = p->ctx;
  cudaStream_t st = p->stream;
  const int32_t n = Ad->n;
  const bool gram = p->task == SPG_TASK_AATS;
  p->n = n;
  p->A = MatView{n, Ad->nnz, Ad->rowptr, Ad->col, Ad->val};
  p->info.n = n;
  p->info.task = p->task;
  p->info.nnz_a = Ad->nnz;
  // B = A; or Aᵀ: for a structurally symmetric A only its values move, gathered
  // here; otherwise the counting-sort transpose builds it.  Nothing waits for
  // the validation verdict or the symmetry check: the pre-pass and the binning
  // check every index they use, and the verdict and the check come back with
  // the bin sizes (sync #1 of the plan); an A·Aᵀ whose pattern turns out not
  // to be symmetric is then transposed and binned again (one more sync).
  double* bx = nullptr;
  if (p->task != SPG_TASK_AA) TRY(palloc(p, &bx, Ad->nnz));
  TRY_CUDA(cudaMemsetAsync(ctx->d_status, 0, 2 * sizeof(uint32_t), st), "status reset");
  if (bx) {
    ProfScope ps(ctx, "plan/transpose_sym", st);
    TRY_CUDA(launch_sym_transpose_vals(p->A, bx, (int*)(ctx->d_status + 1), st),
             "symmetric transpose");
  }
  p->bt_val = bx;
  p->symmetric = p->task != SPG_TASK_AA;  // until the check says otherwise
  p->B = p->task == SPG_TASK_AA ? p->A : MatView{n, Ad->nnz, Ad->rowptr, Ad->col, bx};
  auto build_transpose = [&]() -> spg_status {
    int32_t *bp, *bi;
    TRY(palloc(p, &bp, (int64_t)n + 1));
    TRY(palloc(p, &bi, Ad->nnz));
    TransposeWork w{};
    void* scan_tmp;
    TRY(palloc(p, &w.cnt, n));
    TRY(palloc(p, &w.cursor, n));
    TRY(palloc(p, (char**)&scan_tmp, (int64_t)scan_tmp_bytes(n)));
    w.scan_tmp = scan_tmp;
    TRY(palloc(p, &w.tmp_col, Ad->nnz));
    TRY(palloc(p, &w.tmp_val, Ad->nnz));
    TRY(palloc(p, &w.long_list, n));
    TRY(palloc(p, &w.long_count, 1));
    w.status = ctx->d_status;
    ProfScope ps(ctx, "plan/transpose", st);
    TRY_CUDA(launch_transpose(p->A, bp, bi, bx, w, ctx->num_sms, st), "transpose");
    p->B = MatView{n, Ad->nnz, bp, bi, bx};
    p->tw = w;
    p->bt_rowptr = bp;
    p->bt_col = bi;
    p->symmetric = false;
    return SPG_OK;
  };

  // lanes per row in the sub-warp bins: next power of two of B's mean row length
  if (ctx->cfg.lanes_per_row > 0) {
    p->G = ctx->cfg.lanes_per_row;
  } else {
    double mean = n > 0 ? (double)Ad->nnz / n : 1.0;
    int g = 4;
    while (g < 32 && g < mean) g <<= 1;
    p->G = g;
  }

  // pre-pass and symbolic binning (host sync #1: verdict, symmetry, bin sizes)
  TRY(palloc(p, &p->f, n));
  TRY(palloc(p, &p->lo, n));
  TRY(palloc(p, &p->hi, n));
  TRY(palloc(p, &p->hqueue, kNumBins));
  const int nblocks = (n + kBinRowsPerBlock - 1) / kBinRowsPerBlock;
  int32_t* hist;
  int64_t* counts;
  int32_t* rows_sym;
  TRY(palloc(p, &hist, (int64_t)kNumBins * (nblocks > 0 ? nblocks : 1)));
  TRY(palloc(p, &counts, 4 * kNumBins));
  TRY(palloc(p, &rows_sym, n));
  const int force = ctx->cfg.force_heavy ? 1 : 0;
  const int num_lg = table_log2_cap(ctx->cfg.max_smem_slots);
  // short-B-row rows beyond the warp kernel's largest table go heavy too
  // (windowed warp kernel), with the same mean-length rule as the heavy split
  const int64_t split = ctx->cfg.heavy_split > 0 ? (int64_t)ctx->cfg.heavy_split
                                                 : kHeavySplitDefault;
  const int short_lg = std::min(num_lg, 11);
  // bitmap bins (not for the Gram path): the largest bitmap the config allows
  int dense_lw = -1;
  if (!gram && ctx->cfg.dense_max_words >= (1 << kDenseMinLog2W)) {
    dense_lw = kDenseMinLog2W;
    while (dense_lw < kDenseMaxLog2W && ((int64_t)2 << dense_lw) <= ctx->cfg.dense_max_words)
      ++dense_lw;
  }
  BinSource bsym{0, n, p->f, p->lo, p->hi, nullptr, nullptr, kMaxTableLog2, force,
                 ctx->cfg.sym_load_pct,
                 numeric_heavy_min(num_lg, ctx->cfg.num_load_pct),
                 p->A.rowptr, split, short_lg,
                 numeric_heavy_min(short_lg, ctx->cfg.num_load_pct), dense_lw};
  // column blocks of the heavy rows: 1024 columns (windows are packed from
  // the counts; a block above the window cap, 675 columns at the default
  // load, is cut into fixed 512-column windows); wider when that many counts
  // would exceed heavy_block_budget (chosen after the readback below)
  p->blk_log2 = 10;
  heavy_shape(ctx->cfg, n, &p->window_bits, &p->heavy_threads);
  int32_t* nblk;
  void* btmp;
  TRY(palloc(p, &nblk, n));
  TRY(palloc(p, &p->blk_off, (int64_t)n + 1));
  TRY(palloc(p, (char**)&btmp, (int64_t)scan_tmp_bytes(n)));
  int64_t* hp = p->ctx->h_pin;
  // pre-pass, binning and block offsets over the current B, then one readback
  // of the bin sizes, the heavy blocks' total and the two status words
  auto bin_pass = [&]() -> spg_status {
    {  // the pre-pass also validates A (the verdict comes back below)
      ProfScope ps(ctx, "plan/prepass", st);
      TRY_CUDA(launch_prepass(p->A, p->B, p->f, p->lo, p->hi, st, ctx->d_status), "prepass");
    }
    {
      ProfScope ps(ctx, "plan/bin_sym", st);
      TRY_CUDA(launch_bin_rows(bsym, hist, counts, rows_sym, st), "symbolic binning");
    }
    {
      ProfScope ps(ctx, "plan/heavy_blocks", st);
      TRY_CUDA(launch_heavy_blocks(bsym, p->blk_log2, nblk, p->blk_off, btmp, st),
               "heavy blocks");
    }
    TRY_CUDA(cudaMemcpyAsync(hp, counts, sizeof(int64_t) * 2 * kNumBins, cudaMemcpyDeviceToHost,
                             st), "bin readback");
    TRY_CUDA(cudaMemcpyAsync(hp + 2 * kNumBins, p->blk_off + n, sizeof(int64_t),
                             cudaMemcpyDeviceToHost, st), "bin readback");
    TRY_CUDA(cudaMemcpyAsync(hp + 2 * kNumBins + 1, ctx->d_status, 2 * sizeof(uint32_t),
                             cudaMemcpyDeviceToHost, st), "status readback");
    TRY_CUDA(cudaStreamSynchronize(st), "bin sync");
    const uint32_t* words = (const uint32_t*)(hp + 2 * kNumBins + 1);
    if (words[0] & DEV_ERR_INVALID_CSR) return status_from_bits(DEV_ERR_INVALID_CSR);
    return SPG_OK;
  };
  TRY(bin_pass());
  if (p->symmetric && ((const uint32_t*)(hp + 2 * kNumBins + 1))[1] != 0) {
    // A·Aᵀ of a pattern that is not symmetric: transpose and bin again
    TRY(build_transpose());
    TRY(bin_pass());
  }
  p->info.symmetric_pattern = p->symmetric ? 1 : 0;
  int64_t sym_count[kNumBins], sym_start[kNumBins];
  for (int b = 0; b < kNumBins; ++b) {
    sym_count[b] = hp[b];
    sym_start[b] = hp[kNumBins + b];
  }
  // Σ over heavy rows of ((hi − lo) >> b) + 1 is at most
  // total_1024 / 2^(b−10) + rows, so the wider blocks need no second readback
  int64_t total_blocks = hp[2 * kNumBins];
  const int64_t heavy_sym = sym_count[kHeavyBin];
  const int64_t budget = ctx->cfg.heavy_block_budget;
  while (total_blocks > budget && p->blk_log2 < 20 &&
         p->window_bits % (2 << p->blk_log2) == 0) {
    ++p->blk_log2;
    total_blocks = (hp[2 * kNumBins] >> (p->blk_log2 - 10)) + heavy_sym;
  }
  if (p->blk_log2 > 10) {
    ProfScope ps(ctx, "plan/heavy_blocks", st);
    TRY_CUDA(launch_heavy_blocks(bsym, p->blk_log2, nblk, p->blk_off, btmp, st), "heavy blocks");
  }
  if (total_blocks > 0 && total_blocks <= budget) TRY(palloc(p, &p->blk_cnt, total_blocks));

  // symbolic phase
  TRY(palloc(p, &p->rownnz, n));
  TRY_CUDA(cudaMemsetAsync(p->rownnz, 0, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), st), "memset");
  if (gram) {
    TRY(palloc(p, &p->rowlow, n));
    TRY_CUDA(cudaMemsetAsync(p->rowlow, 0, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), st),
             "memset");
  }
  RowArgs ra{};
  ra.A = p->A;
  ra.B = p->B;
  ra.rownnz = p->rownnz;
  ra.rowlow = p->rowlow;
  ra.status = ctx->d_status;
  ra.queue = p->hqueue;
  ra.lo = p->lo;
  ra.hi = p->hi;
  int bins_used = 0;
  for (int b = 1; b < kNumBins; ++b)
    if (sym_count[b] > 0) ++bins_used;
  BinFork fork(ctx, st, bins_used);
  for (int b = 1; b <= kNumTableBins; ++b) {
    if (sym_count[b] == 0) continue;
    RowArgs r = ra;
    r.rows = rows_sym + sym_start[b];
    r.nrows = (int32_t)sym_count[b];
    r.G = hash_bin_lanes(b, p->G);
    r.queue = p->hqueue + b;
    const cudaStream_t bs = fork.next();
    ProfScope ps(ctx, "sym/bin", bs, b);
    TRY_CUDA(launch_hash_bin(b, false, gram, r, ctx->num_sms, bs), "symbolic");
  }
  for (int b = kDenseBin0; b < kNumBins; ++b) {
    if (sym_count[b] == 0) continue;
    RowArgs r = ra;
    r.rows = rows_sym + sym_start[b];
    r.nrows = (int32_t)sym_count[b];
    const cudaStream_t bs = fork.next();
    ProfScope ps(ctx, "sym/dense", bs, b - kDenseBin0 + kDenseMinLog2W);
    TRY_CUDA(launch_dense_bin(b, false, r, ctx->num_sms, bs), "symbolic");
  }
  if (sym_count[kHeavyBin] > 0) {
    HeavyArgs h{};
    h.r = ra;
    h.r.rows = rows_sym + sym_start[kHeavyBin];
    h.r.nrows = (int32_t)sym_count[kHeavyBin];
    h.lo = p->lo;
    h.hi = p->hi;
    h.window_bits = p->window_bits;
    h.blk_off = p->blk_off;
    h.blk_cnt = p->blk_cnt;
    h.blk_log2 = p->blk_log2;
    h.queue = p->hqueue + kHeavyBin;
    const cudaStream_t bs = fork.next();
    ProfScope ps(ctx, "sym/heavy", bs);
    TRY_CUDA(launch_heavy(false, gram, h, p->heavy_threads, ctx->num_sms, bs),
             "symbolic heavy");
  }
  TRY_CUDA(fork.join(), "join");

  // C row pointers (and lower-part offsets of the Gram mirror)
  void* scan_tmp;
  TRY(palloc(p, (char**)&scan_tmp, (int64_t)scan_tmp_bytes(n)));
  TRY(palloc(p, &p->rowptr, (int64_t)n + 1));
  {
    ProfScope ps(ctx, "plan/scan", st);
    TRY_CUDA(launch_scan_i32_i64(p->rownnz, p->rowptr, n, scan_tmp, st), "row pointer scan");
  }
  if (gram) {
    void* scan_tmp2;
    TRY(palloc(p, (char**)&scan_tmp2, (int64_t)scan_tmp_bytes(n)));
    TRY(palloc(p, &p->lowptr, (int64_t)n + 1));
    TRY_CUDA(launch_scan_i32_i64(p->rowlow, p->lowptr, n, scan_tmp2, st), "lower scan");
  }

  // numeric binning by exact counts, stats; host sync #2 (nnz(C))
  TRY(palloc(p, &p->rows_num, n));
  BinSource bnum{1, n, p->f, p->lo, p->hi, p->rownnz, gram ? p->rowlow : nullptr, num_lg, force,
                 ctx->cfg.num_load_pct, 0, p->A.rowptr, split, short_lg, 0, dense_lw};
  {
    ProfScope ps(ctx, "plan/bin_num", st);
    TRY_CUDA(launch_bin_rows(bnum, hist, counts + 2 * kNumBins, p->rows_num, st),
             "numeric binning");
  }
  unsigned long long* stats = nullptr;
  TRY(palloc(p, &stats, 4));
  TRY_CUDA(launch_row_stats(p->f, p->rownnz, n, stats, st), "row stats");
  TRY_CUDA(cudaMemcpyAsync(hp, counts + 2 * kNumBins, sizeof(int64_t) * 2 * kNumBins,
                           cudaMemcpyDeviceToHost, st), "readback");
  TRY_CUDA(cudaMemcpyAsync(hp + 2 * kNumBins, p->rowptr + n, sizeof(int64_t),
                           cudaMemcpyDeviceToHost, st), "readback");
  if (gram)
    TRY_CUDA(cudaMemcpyAsync(hp + 2 * kNumBins + 1, p->lowptr + n, sizeof(int64_t),
                             cudaMemcpyDeviceToHost, st), "readback");
  TRY_CUDA(cudaMemcpyAsync(hp + 2 * kNumBins + 2, stats, sizeof(unsigned long long) * 3,
                           cudaMemcpyDeviceToHost, st), "readback");
  TRY_CUDA(cudaMemcpyAsync(hp + 2 * kNumBins + 5, ctx->d_status, sizeof(uint32_t),
                           cudaMemcpyDeviceToHost, st), "readback");
  TRY_CUDA(cudaStreamSynchronize(st), "plan sync");
  TRY(status_from_bits(*(uint32_t*)(hp + 2 * kNumBins + 5)));
  for (int b = 0; b < kNumBins; ++b) {
    p->num_count[b] = hp[b];
    p->num_start[b] = hp[kNumBins + b];
  }
  p->nnz_c = n > 0 ? hp[2 * kNumBins] : 0;
  p->nnz_low = (gram && n > 0) ? hp[2 * kNumBins + 1] : 0;
  const unsigned long long* sv = (const unsigned long long*)(hp + 2 * kNumBins + 2);
  p->info.nnz_c = p->nnz_c;
  p->info.products = (int64_t)sv[0];
  p->info.products_computed = (int64_t)sv[0];
  p->info.max_row_products = (int64_t)sv[1];
  p->info.max_row_nnz = (int64_t)sv[2];
  p->info.heavy_rows = p->num_count[kHeavyBin];
  p->heavy_windows = p->num_count[kHeavyBin] > 0 && p->blk_cnt;
  for (int b = 1; b < kNumBins; ++b)
    if (p->num_count[b] > 0) ++bins_used;
  p->info.bins_used = bins_used;
  p->info.output_bytes = 8 * ((int64_t)n + 1) + 12 * p->nnz_c;
  p->info.workspace_bytes = p->ws_bytes;
  p->info.exec_workspace_bytes = exec_workspace(n, gram, p->nnz_low) +
                                 (p->heavy_windows ? 16 * Ad->nnz : 0);
  return SPG_OK;
}

spg_status execute_impl(spg_plan* p, spg_csr_out* C, cudaStream_t st) {
  spg_ctx* ctx = p->ctx;
  const int32_t n = p->n;
  const bool gram = p->task == SPG_TASK_AATS;
  if (!C) return set_error(SPG_ERR_INVALID_ARG, "null output");
  if (C->n != n) return set_error(SPG_ERR_INVALID_ARG, "output n %d != %d", C->n, n);
  if (!C->rowptr || (p->nnz_c > 0 && (!C->col || !C->val)))
    return set_error(SPG_ERR_INVALID_ARG, "null output arrays");
  C->nnz = p->nnz_c;
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  TRY_CUDA(cudaMemcpyAsync(C->rowptr, p->rowptr, sizeof(int64_t) * ((size_t)n + 1),
                           cudaMemcpyDeviceToDevice, st), "rowptr copy");
  // The plan fixed the structure; A's values may have changed since.  Unless
  // this is the first execute after planning, recompute the values derived
  // from A (the block-diagonal copy of a batch, the values of Aᵀ).
  if (!p->values_fresh) {
    if (p->count > 0) {
      ProfScope ps(ctx, "exec/batch_vals", st);
      TRY_CUDA(launch_batch_vals(p->d_desc, p->d_nnz_off, p->count, p->A.nnz, p->batch_val,
                                 ctx->num_sms, st), "batch values");
    }
    if (p->task != SPG_TASK_AA) {
      ProfScope ps(ctx, "exec/transpose_vals", st);
      if (p->symmetric) {
        TRY_CUDA(cudaMemsetAsync(ctx->d_status + 1, 0, sizeof(uint32_t), st), "memset");
        TRY_CUDA(launch_sym_transpose_vals(p->A, p->bt_val, (int*)(ctx->d_status + 1), st),
                 "transpose values");
      } else {
        TRY_CUDA(launch_transpose(p->A, p->bt_rowptr, p->bt_col, p->bt_val, p->tw, ctx->num_sms,
                                  st), "transpose");
      }
    }
  }
  p->values_fresh = false;
  std::vector<void*> tmp;
  auto talloc = [&](void** ptr, size_t bytes) -> spg_status {
    cudaError_t e = cudaMallocFromPoolAsync(ptr, bytes ? bytes : 1, ctx->pool, st);
    if (e != cudaSuccess) return cuda_status(e, "execute workspace");
    tmp.push_back(*ptr);
    return SPG_OK;
  };
  spg_status result = SPG_OK;
  do {
    if (p->nnz_c == 0) break;
    RowArgs ra{};
    ra.A = p->A;
    ra.B = p->B;
    ra.rowptr = p->rowptr;
    ra.cnt_in = p->rownnz;
    ra.low_in = p->rowlow;
    ra.ccol = C->col;
    ra.cval = C->val;
    ra.status = ctx->d_status;
    ra.queue = p->hqueue;
    ra.lo = p->lo;
    ra.hi = p->hi;
    ra.colbase = p->colbase;
    if (gram) {
      void *cur, *lc, *lv;
      if ((result = talloc(&cur, sizeof(int32_t) * (size_t)n)) != SPG_OK) break;
      if ((result = talloc(&lc, sizeof(int32_t) * (size_t)p->nnz_low)) != SPG_OK) break;
      if ((result = talloc(&lv, sizeof(double) * (size_t)p->nnz_low)) != SPG_OK) break;
      cudaError_t e = cudaMemsetAsync(cur, 0, sizeof(int32_t) * (size_t)n, st);
      if (e != cudaSuccess) { result = cuda_status(e, "memset"); break; }
      ra.lowptr = p->lowptr;
      ra.cursor = (int32_t*)cur;
      ra.lcol = (int32_t*)lc;
      ra.lval = (double*)lv;
    }
    // the heavy rows' cursors are taken from the pool before the bins fork, so
    // their allocation is ordered before every stream that uses them
    int4* hcur = nullptr;
    if (p->num_count[kHeavyBin] > 0 && p->heavy_windows) {  // one int4 per entry of A
      void* hc;
      if ((result = talloc(&hc, sizeof(int4) * (size_t)p->A.nnz)) != SPG_OK) break;
      hcur = (int4*)hc;
    }
    int launches = p->small && n > 0 ? 1 : 0;
    for (int b = 1; b < kNumBins; ++b)
      if (p->num_count[b] > 0) launches += b == kHeavyBin && p->heavy_windows ? 2 : 1;
    BinFork fork(ctx, st, launches);
    if (p->small && n > 0) {
      RowArgs r = ra;
      r.rows = nullptr;
      r.nrows = n;
      const int bin = p->small_log2 - kMinTableLog2 + 1;
      r.G = hash_bin_lanes(bin, p->G);
      ProfScope ps(ctx, "num/small", st);
      cudaError_t e = launch_hash_bin(bin, true, false, r, ctx->num_sms, st);
      if (e != cudaSuccess) result = cuda_status(e, "numeric");
    }
    for (int b = 1; b <= kNumTableBins && result == SPG_OK; ++b) {
      if (p->num_count[b] == 0) continue;
      RowArgs r = ra;
      r.rows = p->rows_num + p->num_start[b];
      r.nrows = (int32_t)p->num_count[b];
      r.G = hash_bin_lanes(b, p->G);
      r.queue = p->hqueue + b;
      const cudaStream_t bs = fork.next();
      ProfScope ps(ctx, "num/bin", bs, b);
      cudaError_t e = launch_hash_bin(b, true, gram, r, ctx->num_sms, bs);
      if (e != cudaSuccess) result = cuda_status(e, "numeric");
    }
    for (int b = kDenseBin0; b < kNumBins && result == SPG_OK; ++b) {
      if (p->num_count[b] == 0) continue;
      RowArgs r = ra;
      r.rows = p->rows_num + p->num_start[b];
      r.nrows = (int32_t)p->num_count[b];
      const cudaStream_t bs = fork.next();
      ProfScope ps(ctx, "num/dense", bs, b - kDenseBin0 + kDenseMinLog2W);
      cudaError_t e = launch_dense_bin(b, true, r, ctx->num_sms, bs);
      if (e != cudaSuccess) result = cuda_status(e, "numeric");
    }
    if (result != SPG_OK) break;
    if (p->num_count[kHeavyBin] > 0) {
      HeavyArgs h{};
      h.r = ra;
      h.r.rows = p->rows_num + p->num_start[kHeavyBin];
      h.r.nrows = (int32_t)p->num_count[kHeavyBin];
      h.lo = p->lo;
      h.hi = p->hi;
      h.window_bits = p->window_bits;
      h.blk_off = p->blk_off;
      h.blk_cnt = p->blk_cnt;
      h.blk_log2 = p->blk_log2;
      h.cap = heavy_cap(ctx->cfg.num_load_pct);
      h.sub_log2 = 31 - __builtin_clz((unsigned)h.cap);  // largest power of two <= cap
      if (h.sub_log2 > p->blk_log2) h.sub_log2 = p->blk_log2;
      h.hcur = hcur;
      h.queue = p->hqueue + kHeavyBin;
      // rows fed by many short B rows stream through the warp kernel's
      // windows; rows dominated by long B rows, rows of more than 2^17
      // products, or all rows without block counts take the CTA kernel (the
      // two take disjoint rows, so they run on streams of their own)
      const bool windows = p->heavy_windows;
      h.f = p->f;
      h.split = !windows ? 0
                : ctx->cfg.heavy_split > 0 ? (int64_t)ctx->cfg.heavy_split : kHeavySplitDefault;
      // CTA rows: values in shared memory window by window when the block
      // counts and cursors exist and the configuration allows it
      const bool shared_values = windows && ctx->cfg.heavy_vcap >= 0;
      const int win_threads = ctx->cfg.heavy_threads > 512 ? 1024 : 512;
      h.vcap = ctx->cfg.heavy_vcap > 0 ? (int32_t)ctx->cfg.heavy_vcap : 8192;
      h.wcap_bits = win_threads > 512 ? (1 << 18) : (1 << 17);
      cudaError_t e = cudaSuccess;
      if (windows) {
        const cudaStream_t bs = fork.next();
        ProfScope ps(ctx, "num/heavy_w32", bs);
        e = launch_heavy_w32(gram, h, ctx->num_sms, bs);
      }
      if (e == cudaSuccess) {
        const cudaStream_t bs = fork.next();
        ProfScope ps(ctx, "num/heavy", bs);
        e = shared_values ? launch_heavy_win(gram, h, win_threads, ctx->num_sms, bs)
                          : launch_heavy(true, gram, h, p->heavy_threads, ctx->num_sms, bs);
      }
      if (e != cudaSuccess) { result = cuda_status(e, "numeric heavy"); break; }
    }
    {
      const cudaError_t e = fork.join();
      if (e != cudaSuccess) { result = cuda_status(e, "join"); break; }
    }
    if (gram && p->nnz_low > 0) {
      void *ll, *lcnt;
      if ((result = talloc(&ll, sizeof(int32_t) * (size_t)n)) != SPG_OK) break;
      if ((result = talloc(&lcnt, sizeof(int32_t))) != SPG_OK) break;
      SegSortArgs sa{};
      sa.nseg = n;
      sa.src_off64 = p->lowptr;
      sa.dst_off64 = p->rowptr;
      sa.lens = p->rowlow;
      sa.src_key = ra.lcol;
      sa.src_val = ra.lval;
      sa.dst_key = C->col;
      sa.dst_val = C->val;
      sa.key_bound = n;
      sa.long_list = (int32_t*)ll;
      sa.long_count = (int32_t*)lcnt;
      sa.status = ctx->d_status;
      ProfScope ps(ctx, "num/mirror_sort", st);
      cudaError_t e = launch_segsort(sa, ctx->num_sms, st);
      if (e != cudaSuccess) { result = cuda_status(e, "mirror sort"); break; }
    }
  } while (0);
  for (void* ptr : tmp) cudaFreeAsync(ptr, st);
  if (result != SPG_OK) return result;
  // the plan's workspace must outlive this execution: plan_free waits for this
  // event (not recorded while capturing a graph, whose launches the caller orders)
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  TRY_CUDA(cudaStreamIsCapturing(st, &cap), "capture status");
  if (cap == cudaStreamCaptureStatusNone) {
    if (!p->exec_done)
      TRY_CUDA(cudaEventCreateWithFlags(&p->exec_done, cudaEventDisableTiming), "event");
    TRY_CUDA(cudaEventRecord(p->exec_done, st), "event record");
  }
  return SPG_OK;
}

spg_task parse_task(const char* t, bool* ok) {
  *ok = true;
  if (t && std::strcmp(t, "AA") == 0) return SPG_TASK_AA;
  if (t && std::strcmp(t, "AAt") == 0) return SPG_TASK_AAT;
  if (t && std::strcmp(t, "AAtS") == 0) return SPG_TASK_AATS;
  *ok = false;
  return SPG_TASK_AA;
}

}  // namespace

extern "C" {

spg_status spg_create(spg_ctx** out, const spg_config* cfg) {
  begin_call();
  if (!out) return set_error(SPG_ERR_INVALID_ARG, "null context pointer");
  *out = nullptr;
  spg_ctx* ctx = new spg_ctx();
  ctx->cfg = merged_config(cfg);
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) {
    delete ctx;
    return cuda_status(e, "cudaGetDevice (is a CUDA GPU present?)");
  }
  if (cfg && cfg->struct_size > 0 && cfg->device > 0) dev = cfg->device;
  ctx->device = dev;
  spg_status st = SPG_OK;
  do {
    if ((e = cudaSetDevice(dev)) != cudaSuccess) { st = cuda_status(e, "cudaSetDevice"); break; }
    if ((e = cudaDeviceGetAttribute(&ctx->device_sms, cudaDevAttrMultiProcessorCount, dev)) !=
        cudaSuccess) { st = cuda_status(e, "device attribute"); break; }
    ctx->num_sms = grid_sms_of(ctx->cfg, ctx->device_sms);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    if ((e = cudaMemPoolCreate(&ctx->pool, &props)) != cudaSuccess) {
      st = cuda_status(e, "memory pool");
      break;
    }
    uint64_t thr = ctx->cfg.pool_release_bytes > 0 ? (uint64_t)ctx->cfg.pool_release_bytes
                                                   : UINT64_MAX;
    cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    if ((e = cudaMalloc(&ctx->d_status, 256)) != cudaSuccess) { st = cuda_status(e, "status"); break; }
    if ((e = cudaMemset(ctx->d_status, 0, 256)) != cudaSuccess) { st = cuda_status(e, "status"); break; }
    if ((e = cudaMallocHost(&ctx->h_pin, 512)) != cudaSuccess) { st = cuda_status(e, "pinned"); break; }
    if ((e = cudaEventCreateWithFlags(&ctx->fork_ev, cudaEventDisableTiming)) != cudaSuccess) {
      st = cuda_status(e, "event");
      break;
    }
    // side streams for concurrent bins (bin_streams > 1 at creation or later)
    for (int i = 0; i < 4; ++i) {
      if ((e = cudaStreamCreateWithFlags(&ctx->side[i], cudaStreamNonBlocking)) != cudaSuccess ||
          (e = cudaEventCreateWithFlags(&ctx->side_done[i], cudaEventDisableTiming)) != cudaSuccess) {
        st = cuda_status(e, "side stream");
        break;
      }
      ctx->nsides = i + 1;
    }
    if (st != SPG_OK) break;
  } while (0);
  if (st != SPG_OK) {
    spg_destroy(ctx);
    return st;
  }
  *out = ctx;
  return SPG_OK;
}

spg_status spg_destroy(spg_ctx* ctx) {
  begin_call();
  if (!ctx) return SPG_OK;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  prof_resolve(ctx);
  for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
  if (ctx->d_status) cudaFree(ctx->d_status);
  if (ctx->h_pin) cudaFreeHost(ctx->h_pin);
  for (int i = 0; i < spg_ctx::kMaxSides; ++i) {
    if (ctx->side[i]) cudaStreamDestroy(ctx->side[i]);
    if (ctx->side_done[i]) cudaEventDestroy(ctx->side_done[i]);
  }
  if (ctx->fork_ev) cudaEventDestroy(ctx->fork_ev);
  if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
  delete ctx;
  return SPG_OK;
}

spg_status spg_check_device_status(spg_ctx* ctx, void* stream) {
  begin_call();
  if (!ctx) return set_error(SPG_ERR_INVALID_ARG, "null context");
  cudaStream_t st = (cudaStream_t)stream;
  TRY_CUDA(cudaMemcpyAsync(ctx->h_pin, ctx->d_status, sizeof(uint32_t), cudaMemcpyDeviceToHost, st),
           "status readback");
  TRY_CUDA(cudaStreamSynchronize(st), "status sync");
  uint32_t bits = *(uint32_t*)ctx->h_pin;
  TRY_CUDA(cudaMemsetAsync(ctx->d_status, 0, sizeof(uint32_t), st), "status reset");
  return status_from_bits(bits);
}

spg_status spg_plan_create(spg_ctx* ctx, spg_task task, const spg_csr_dev* A, void* stream,
                           spg_plan** out) {
  begin_call();
  if (!ctx || !out) return set_error(SPG_ERR_INVALID_ARG, "null context or plan pointer");
  *out = nullptr;
  if (task != SPG_TASK_AA && task != SPG_TASK_AAT && task != SPG_TASK_AATS)
    return set_error(SPG_ERR_INVALID_ARG, "unknown task %d", (int)task);
  TRY(check_matrix(A));
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  spg_plan* p = new spg_plan();
  p->ctx = ctx;
  p->task = task;
  p->stream = (cudaStream_t)stream;
  spg_status st = SPG_OK;
  bool regular = true;
  if (small_plan_eligible(ctx, task, A)) {
    bool fallback = false;
    st = plan_build_small(p, A, &fallback);
    if (st == SPG_OK && fallback) {  // a row beyond the small table: plan again
      plan_free(p);
      p = new spg_plan();
      p->ctx = ctx;
      p->task = task;
      p->stream = (cudaStream_t)stream;
    } else {
      regular = false;
    }
  }
  if (regular) st = plan_build(p, A);
  if (st != SPG_OK) {
    // keep the message of the failure, then release what was allocated
    cudaStreamSynchronize(p->stream);
    plan_free(p);
    return st;
  }
  *out = p;
  return SPG_OK;
}

spg_status spg_plan_get_info(const spg_plan* plan, spg_plan_info* info) {
  begin_call();
  if (!plan || !info) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  *info = plan->info;
  return SPG_OK;
}

spg_status spg_execute(spg_plan* plan, spg_csr_out* C, void* stream) {
  begin_call();
  if (!plan) return set_error(SPG_ERR_INVALID_ARG, "null plan");
  return execute_impl(plan, C, (cudaStream_t)stream);
}

spg_status spg_plan_destroy(spg_plan* plan) {
  begin_call();
  if (!plan) return SPG_OK;
  cudaSetDevice(plan->ctx->device);
  plan_free(plan);
  return SPG_OK;
}

spg_status spg_plan_create_batched(spg_ctx* ctx, spg_task task, int32_t count,
                                   const spg_csr_dev* As, void* stream, spg_plan** out) {
  begin_call();
  if (!ctx || !out || !As || count < 1)
    return set_error(SPG_ERR_INVALID_ARG, "null argument or count < 1");
  *out = nullptr;
  if (task != SPG_TASK_AA && task != SPG_TASK_AAT && task != SPG_TASK_AATS)
    return set_error(SPG_ERR_INVALID_ARG, "unknown task %d", (int)task);
  std::vector<BatchDesc> desc((size_t)count);
  std::vector<int64_t> row_off((size_t)count + 1, 0), nnz_off((size_t)count + 1, 0);
  for (int32_t b = 0; b < count; ++b) {
    spg_status s = check_matrix(&As[b]);
    if (s != SPG_OK) return set_error(s, "instance %d: %s", b, spg_last_error_string());
    desc[b] = BatchDesc{As[b].rowptr, As[b].col, As[b].val, As[b].n, 0, As[b].nnz, row_off[b],
                        nnz_off[b]};
    row_off[b + 1] = row_off[b] + As[b].n;
    nnz_off[b + 1] = nnz_off[b] + As[b].nnz;
  }
  const int64_t N = row_off[count], NNZ = nnz_off[count];
  if (N > INT32_MAX || NNZ > INT32_MAX)
    return set_error(SPG_ERR_UNSUPPORTED,
                     "batch of %lld rows / %lld entries exceeds the int32 block-diagonal layout",
                     (long long)N, (long long)NNZ);
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  spg_plan* p = new spg_plan();
  p->ctx = ctx;
  p->task = task;
  p->stream = (cudaStream_t)stream;
  p->count = count;
  p->row_off = row_off;
  cudaStream_t st = p->stream;
  spg_status s = SPG_OK;
  int32_t *rp = nullptr, *col = nullptr, *cb = nullptr;
  double* val = nullptr;
  BatchDesc* d_desc = nullptr;
  int64_t *d_row_off = nullptr, *d_nnz_off = nullptr, *d_cnnz_off = nullptr;
  do {
    if ((s = palloc(p, &rp, N + 1)) != SPG_OK) break;
    if ((s = palloc(p, &col, NNZ)) != SPG_OK) break;
    if ((s = palloc(p, &val, NNZ)) != SPG_OK) break;
    if ((s = palloc(p, &cb, N)) != SPG_OK) break;
    if ((s = palloc(p, &d_desc, count)) != SPG_OK) break;
    if ((s = palloc(p, &d_row_off, (int64_t)count + 1)) != SPG_OK) break;
    if ((s = palloc(p, &d_nnz_off, (int64_t)count + 1)) != SPG_OK) break;
    if ((s = palloc(p, &d_cnnz_off, (int64_t)count + 1)) != SPG_OK) break;
    cudaError_t e = cudaMemcpyAsync(d_desc, desc.data(), sizeof(BatchDesc) * desc.size(),
                                    cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_row_off, row_off.data(), sizeof(int64_t) * row_off.size(),
                          cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_nnz_off, nnz_off.data(), sizeof(int64_t) * nnz_off.size(),
                          cudaMemcpyHostToDevice, st);
    // instance checks report into status word 2 (word 0 is reset by validation)
    if (e == cudaSuccess) e = cudaMemsetAsync(ctx->d_status + 2, 0, sizeof(uint32_t), st);
    if (e == cudaSuccess) {
      ProfScope ps(ctx, "plan/batch_concat", st);
      e = launch_batch_concat(d_desc, d_row_off, d_nnz_off, count, N, NNZ, rp, col, val, cb,
                              ctx->d_status + 2, ctx->num_sms, st);
    }
    if (e != cudaSuccess) { s = cuda_status(e, "batch concatenation"); break; }
    p->colbase = cb;
    p->d_desc = d_desc;
    p->d_nnz_off = d_nnz_off;
    p->batch_val = val;
    spg_csr_dev big{(int32_t)N, NNZ, rp, col, val};
    if ((s = plan_build(p, &big)) != SPG_OK) break;
    // instance checks and the per-instance C offsets, one more round trip
    e = launch_gather_offsets(p->rowptr, d_row_off, count, d_cnnz_off, st);
    std::vector<int64_t> cnnz((size_t)count + 1);
    uint32_t bad = 0;
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(cnnz.data(), d_cnnz_off, sizeof(int64_t) * cnnz.size(),
                          cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(&bad, ctx->d_status + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { s = cuda_status(e, "batch offsets"); break; }
    if (bad) {
      s = set_error(SPG_ERR_INVALID_CSR,
                    "an instance's rowptr does not run from 0 to its nnz, or a column lies "
                    "outside [0, n) of its instance");
      break;
    }
    p->nnz_off = cnnz;
  } while (0);
  if (s != SPG_OK) {
    cudaStreamSynchronize(st);
    plan_free(p);
    return s;
  }
  *out = p;
  return SPG_OK;
}

spg_status spg_plan_workspace_bound(const spg_ctx* ctx, spg_task task, int32_t count,
                                    const spg_csr_dev* As, int32_t batched, int64_t* bytes) {
  begin_call();
  if (!ctx || !As || !bytes || count < 1 || (!batched && count != 1))
    return set_error(SPG_ERR_INVALID_ARG, "null argument, count < 1, or count != 1 unbatched");
  if (task != SPG_TASK_AA && task != SPG_TASK_AAT && task != SPG_TASK_AATS)
    return set_error(SPG_ERR_INVALID_ARG, "unknown task %d", (int)task);
  int64_t N = 0, NNZ = 0;
  for (int32_t b = 0; b < count; ++b) {
    if (As[b].n < 0 || As[b].nnz < 0) return set_error(SPG_ERR_INVALID_ARG, "negative n or nnz");
    N += As[b].n;
    NNZ += As[b].nnz;
  }
  int64_t w = plan_workspace_bound(ctx->cfg, task, N, NNZ);
  if (batched)  // the block-diagonal copy, column bases, instance table and offsets
    w += 4 * (N + 1) + 12 * (NNZ > 0 ? NNZ : 1) + 4 * (N > 0 ? N : 1) +
         (int64_t)sizeof(BatchDesc) * count + 3 * 8 * ((int64_t)count + 1);
  *bytes = w;
  return SPG_OK;
}

spg_status spg_plan_batch_offsets(const spg_plan* plan, int64_t* row_off, int64_t* nnz_off) {
  begin_call();
  if (!plan) return set_error(SPG_ERR_INVALID_ARG, "null plan");
  if (plan->count == 0) return set_error(SPG_ERR_INVALID_ARG, "not a batched plan");
  if (row_off) std::memcpy(row_off, plan->row_off.data(), sizeof(int64_t) * plan->row_off.size());
  if (nnz_off) std::memcpy(nnz_off, plan->nnz_off.data(), sizeof(int64_t) * plan->nnz_off.size());
  return SPG_OK;
}

spg_status spg_graph_capture(spg_plan* plan, spg_csr_out* C, void* stream, spg_graph** out) {
  begin_call();
  if (!plan || !C || !out) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  *out = nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  if (!st || st == cudaStreamLegacy || st == cudaStreamPerThread)
    return set_error(SPG_ERR_INVALID_ARG, "graph capture needs a created (non-default) stream");
  TRY_CUDA(cudaSetDevice(plan->ctx->device), "set device");
  TRY_CUDA(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "begin capture");
  plan->values_fresh = false;  // every launch recomputes values derived from A
  spg_status s = execute_impl(plan, C, st);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(st, &g);
  if (s != SPG_OK) {
    if (g) cudaGraphDestroy(g);
    return s;
  }
  if (e != cudaSuccess) return cuda_status(e, "end capture");
  cudaGraphExec_t ex = nullptr;
  e = cudaGraphInstantiate(&ex, g, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(g);
    return cuda_status(e, "graph instantiate");
  }
  spg_graph* gr = new spg_graph();
  gr->graph = g;
  gr->exec = ex;
  *out = gr;
  return SPG_OK;
}

spg_status spg_graph_launch(spg_graph* graph, void* stream) {
  begin_call();
  if (!graph) return set_error(SPG_ERR_INVALID_ARG, "null graph");
  TRY_CUDA(cudaGraphLaunch(graph->exec, (cudaStream_t)stream), "graph launch");
  return SPG_OK;
}

spg_status spg_graph_destroy(spg_graph* graph) {
  begin_call();
  if (!graph) return SPG_OK;
  if (graph->exec) cudaGraphExecDestroy(graph->exec);
  if (graph->graph) cudaGraphDestroy(graph->graph);
  delete graph;
  return SPG_OK;
}

spg_status spg_set_config(spg_ctx* ctx, const spg_config* cfg) {
  begin_call();
  if (!ctx || !cfg) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  const int dev = ctx->device;
  ctx->cfg = merged_config(cfg);
  ctx->cfg.device = dev;
  ctx->num_sms = grid_sms_of(ctx->cfg, ctx->device_sms);
  return SPG_OK;
}

spg_status spg_get_config(const spg_ctx* ctx, spg_config* cfg) {
  begin_call();
  if (!ctx || !cfg) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  *cfg = ctx->cfg;
  return SPG_OK;
}

namespace {

// One full product (plan, output allocation, execute, release) with the
// context's current tuning, timed with events on `st`.
spg_status tune_run(spg_ctx* ctx, spg_task task, int32_t count, const spg_csr_dev* As,
                    cudaStream_t st, float* ms, int64_t* heavy_rows) {
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  TRY_CUDA(cudaEventCreate(&e0), "event");
  TRY_CUDA(cudaEventCreate(&e1), "event");
  cudaEventRecord(e0, st);
  spg_plan* p = nullptr;
  spg_status s = count == 1 ? spg_plan_create(ctx, task, As, st, &p)
                            : spg_plan_create_batched(ctx, task, count, As, st, &p);
  spg_csr_out C{};
  if (s == SPG_OK) {
    if (heavy_rows) *heavy_rows = p->info.heavy_rows;
    C.n = p->n;
    const size_t nz = (size_t)(p->nnz_c > 0 ? p->nnz_c : 1);
    cudaError_t e = cudaMallocFromPoolAsync((void**)&C.rowptr, 8 * ((size_t)p->n + 1), ctx->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void**)&C.col, 4 * nz, ctx->pool, st);
    if (e == cudaSuccess) e = cudaMallocFromPoolAsync((void**)&C.val, 8 * nz, ctx->pool, st);
    s = e == cudaSuccess ? execute_impl(p, &C, st) : cuda_status(e, "autotune output");
    if (C.rowptr) cudaFreeAsync(C.rowptr, st);
    if (C.col) cudaFreeAsync(C.col, st);
    if (C.val) cudaFreeAsync(C.val, st);
    plan_free(p);
  }
  cudaEventRecord(e1, st);
  cudaEventSynchronize(e1);
  float t = 0.f;
  cudaEventElapsedTime(&t, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t;
  return s;
}

}  // namespace

spg_status spg_autotune(spg_ctx* ctx, spg_task task, int32_t count, const spg_csr_dev* As,
                        int32_t reps, spg_config* best, void* stream) {
  begin_call();
  if (!ctx || !As || count < 1) return set_error(SPG_ERR_INVALID_ARG, "bad arguments");
  if (reps < 1) reps = 3;
  cudaStream_t st = (cudaStream_t)stream;
  const spg_config start = ctx->cfg;
  int64_t heavy = 0;
  auto measure = [&](const spg_config& c, float* out) -> spg_status {
    ctx->cfg = merged_config(&c);
    ctx->cfg.device = start.device;
    float t;
    spg_status s = tune_run(ctx, task, count, As, st, &t, &heavy);  // warm-up
    std::vector<float> v;
    for (int r = 0; r < reps && s == SPG_OK; ++r) {
      s = tune_run(ctx, task, count, As, st, &t, nullptr);
      v.push_back(t);
    }
    if (s != SPG_OK) return s;
    std::sort(v.begin(), v.end());
    *out = v[v.size() / 2];
    return SPG_OK;
  };
  // Structural features of the input, as the reference's dispatcher reads
  // them (bench/dispatch.cu:26-38), computed on the device: for a batch, the
  // mean degree over all instances and the largest row / column degree.
  int64_t tot_n = 0, tot_nnz = 0;
  int32_t max_deg = 0, max_col = 0;
  for (int32_t b = 0; b < count; ++b) {
    spg_descriptors d{};
    spg_status ds = spg_describe(ctx, &As[b], &d, stream);
    if (ds != SPG_OK) {
      ctx->cfg = start;
      return ds;
    }
    tot_n += d.n;
    tot_nnz += d.nnz;
    max_deg = std::max(max_deg, d.max_deg);
    max_col = std::max(max_col, d.max_col_deg);
  }
  const double mean_deg = tot_n > 0 ? (double)tot_nnz / (double)tot_n : 1.0;
  // B rows are A's rows (A·A) or its columns (A·Aᵀ)
  const int64_t max_b = task == SPG_TASK_AA ? max_deg : max_col;
  // a row has at most max_deg · max_b products, so at most that many entries
  const int64_t max_row = (int64_t)max_deg * max_b;
  ctx->tune_timed = 0;
  ctx->tune_pruned = 0;
  spg_config cur = start;
  float cur_ms = 0.f;
  spg_status s = measure(cur, &cur_ms);
  ++ctx->tune_timed;
  if (s != SPG_OK) {
    ctx->cfg = start;
    return s;
  }
  const bool has_heavy = heavy > 0;
  using Field = int32_t spg_config::*;
  struct Knob {
    Field field;
    std::vector<int32_t> values;
    bool heavy_only;
  };
  const std::vector<Knob> knobs = {
      {&spg_config::lanes_per_row, {4, 8, 16, 32}, false},
      {&spg_config::num_load_pct, {40, 50, 66, 80}, false},
      {&spg_config::sym_load_pct, {50, 75, 90}, false},
      {&spg_config::max_smem_slots, {2048, 4096, 8192, 16384}, false},
      {&spg_config::heavy_threads, {256, 512, 1024}, true},
      {&spg_config::window_bits, {1 << 18, 1 << 19, 1 << 20}, true},
      {&spg_config::heavy_split, {1, 32, 128, 512, 1 << 30}, true},
  };
  // Candidates the features rule out are not timed:
  //  - lanes per row of the sub-warp bins: only the powers of two next to the
  //    mean B-row length (a group much wider idles, much narrower serialises);
  //  - the shared-table cap: only when some row can need a table above 2048
  //    slots (max_row entries at the numeric load);
  //  - the heavy-path knobs: only when the plan has heavy rows;
  //  - a single matrix that the one-readback plan takes whole (no row above
  //    its table) runs no binned kernel: only the numeric load matters.
  const bool one_readback = count == 1 && small_plan_eligible(ctx, task, &As[0]) &&
                            max_row <= kSmallCap;
  int near_lanes = 4;
  while (near_lanes < 32 && near_lanes < mean_deg) near_lanes <<= 1;
  const bool big_tables = max_row * 100 / std::max(20, (int)cur.num_load_pct) + 1 > 2048;
  auto pruned = [&](const Knob& k, int32_t v) {
    if (k.heavy_only && !has_heavy) return true;
    if (one_readback && k.field != &spg_config::num_load_pct) return true;
    if (k.field == &spg_config::lanes_per_row)
      return v != near_lanes && v != near_lanes / 2 && v != near_lanes * 2;
    if (k.field == &spg_config::max_smem_slots) return !big_tables;
    return false;
  };
  for (const Knob& k : knobs) {
    for (int32_t v : k.values) {
      if (cur.*(k.field) == v) continue;
      if (pruned(k, v)) {
        ++ctx->tune_pruned;
        continue;
      }
      spg_config c = cur;
      c.*(k.field) = v;
      float t = 0.f;
      ++ctx->tune_timed;
      if (measure(c, &t) != SPG_OK) continue;  // a candidate that fails is skipped
      if (t < cur_ms * 0.98f) {
        cur = merged_config(&c);
        cur_ms = t;
      }
    }
  }
  ctx->cfg = merged_config(&cur);
  ctx->cfg.device = start.device;
  if (best) *best = ctx->cfg;
  begin_call();
  return SPG_OK;
}

spg_status spg_autotune_trials(const spg_ctx* ctx, int32_t* timed, int32_t* pruned) {
  begin_call();
  if (!ctx || !timed || !pruned) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  *timed = ctx->tune_timed;
  *pruned = ctx->tune_pruned;
  return SPG_OK;
}

spg_status spg_multiply(spg_ctx* ctx, spg_task task, const spg_csr_dev* A, spg_csr_out* C,
                        void* stream) {
  begin_call();
  if (!C) return set_error(SPG_ERR_INVALID_ARG, "null output");
  spg_plan* p = nullptr;
  TRY(spg_plan_create(ctx, task, A, stream, &p));
  cudaStream_t st = (cudaStream_t)stream;
  const int32_t n = A->n;
  C->n = n;
  C->nnz = p->nnz_c;
  C->rowptr = nullptr;
  C->col = nullptr;
  C->val = nullptr;
  spg_status s = SPG_OK;
  cudaError_t e = cudaMallocFromPoolAsync((void**)&C->rowptr, sizeof(int64_t) * ((size_t)n + 1),
                                          ctx->pool, st);
  if (e == cudaSuccess)
    e = cudaMallocFromPoolAsync((void**)&C->col, sizeof(int32_t) * (size_t)(p->nnz_c ? p->nnz_c : 1),
                                ctx->pool, st);
  if (e == cudaSuccess)
    e = cudaMallocFromPoolAsync((void**)&C->val, sizeof(double) * (size_t)(p->nnz_c ? p->nnz_c : 1),
                                ctx->pool, st);
  if (e != cudaSuccess) s = cuda_status(e, "output allocation");
  if (s == SPG_OK) s = execute_impl(p, C, st);
  if (s != SPG_OK) {
    if (C->rowptr) cudaFreeAsync(C->rowptr, st);
    if (C->col) cudaFreeAsync(C->col, st);
    if (C->val) cudaFreeAsync(C->val, st);
    C->rowptr = nullptr;
    C->col = nullptr;
    C->val = nullptr;
  }
  plan_free(p);
  return s;
}

spg_status spg_free(spg_ctx* ctx, void* dev_ptr, void* stream) {
  begin_call();
  if (!ctx) return set_error(SPG_ERR_INVALID_ARG, "null context");
  if (!dev_ptr) return SPG_OK;
  TRY_CUDA(cudaFreeAsync(dev_ptr, (cudaStream_t)stream), "free");
  return SPG_OK;
}

spg_status spg_drop_zeros(spg_ctx* ctx, spg_csr_out* C, void* stream) {
  begin_call();
  if (!ctx || !C || !C->rowptr) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  if (C->n < 0 || C->nnz < 0) return set_error(SPG_ERR_INVALID_ARG, "bad output shape");
  if (C->nnz == 0) return SPG_OK;
  if (!C->col || !C->val) return set_error(SPG_ERR_INVALID_ARG, "null output arrays");
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  const int32_t n = C->n;
  spg_plan tmp;  // borrow the plan allocator for the workspace
  tmp.ctx = ctx;
  tmp.stream = (cudaStream_t)stream;
  cudaStream_t st = tmp.stream;
  spg_status rc = SPG_OK;
  int32_t* kept = nullptr;
  int64_t* newptr = nullptr;
  void* scan_tmp = nullptr;
  int32_t* tcol = nullptr;
  double* tval = nullptr;
  std::vector<int64_t> oldp((size_t)n + 1), newp((size_t)n + 1);
  do {
    if ((rc = palloc(&tmp, &kept, n)) != SPG_OK) break;
    if ((rc = palloc(&tmp, &newptr, (int64_t)n + 1)) != SPG_OK) break;
    if ((rc = palloc(&tmp, (char**)&scan_tmp, (int64_t)scan_tmp_bytes(n))) != SPG_OK) break;
    cudaError_t e = launch_count_kept(C->rowptr, C->val, n, kept, st);
    if (e == cudaSuccess) e = launch_scan_i32_i64(kept, newptr, n, scan_tmp, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(oldp.data(), C->rowptr, sizeof(int64_t) * ((size_t)n + 1),
                          cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(newp.data(), newptr, sizeof(int64_t) * ((size_t)n + 1),
                          cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) { rc = cuda_status(e, "drop zeros count"); break; }
    if (oldp[0] != 0 || oldp[n] != C->nnz) {
      rc = set_error(SPG_ERR_INVALID_ARG, "row pointers do not match nnz %lld",
                     (long long)C->nnz);
      break;
    }
    if (newp[n] == C->nnz) break;  // no zero values
    // row chunks of at most `room` old entries (and at least one row)
    int64_t room = (int64_t)1 << 25, longest = 0;
    for (int32_t i = 0; i < n; ++i) longest = std::max(longest, oldp[i + 1] - oldp[i]);
    room = std::min(std::max(room, longest), C->nnz);
    if ((rc = palloc(&tmp, &tcol, room)) != SPG_OK) break;
    if ((rc = palloc(&tmp, &tval, room)) != SPG_OK) break;
    for (int32_t r0 = 0; r0 < n && rc == SPG_OK;) {
      int32_t r1 = r0 + 1;
      while (r1 < n && oldp[r1 + 1] - oldp[r0] <= room) ++r1;
      e = launch_gather_kept(C->rowptr, C->col, C->val, newptr, r0, r1, tcol, tval, st);
      const int64_t m = newp[r1] - newp[r0];
      if (e == cudaSuccess && m > 0)
        e = cudaMemcpyAsync(C->col + newp[r0], tcol, sizeof(int32_t) * (size_t)m,
                            cudaMemcpyDeviceToDevice, st);
      if (e == cudaSuccess && m > 0)
        e = cudaMemcpyAsync(C->val + newp[r0], tval, sizeof(double) * (size_t)m,
                            cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) rc = cuda_status(e, "drop zeros compaction");
      r0 = r1;
    }
    if (rc != SPG_OK) break;
    e = cudaMemcpyAsync(C->rowptr, newptr, sizeof(int64_t) * ((size_t)n + 1),
                        cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) { rc = cuda_status(e, "drop zeros row pointers"); break; }
    C->nnz = newp[n];
  } while (0);
  for (void* ptr : tmp.ptrs) cudaFreeAsync(ptr, st);
  tmp.ptrs.clear();
  return rc;
}

spg_status spg_transpose(spg_ctx* ctx, const spg_csr_dev* A, int32_t* t_rowptr, int32_t* t_col,
                         double* t_val, void* stream) {
  begin_call();
  if (!ctx) return set_error(SPG_ERR_INVALID_ARG, "null context");
  TRY(check_matrix(A));
  if (!t_rowptr || (A->nnz > 0 && (!t_col || !t_val)))
    return set_error(SPG_ERR_INVALID_ARG, "null output arrays");
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  spg_plan tmp;  // borrow the plan allocator for the workspace
  tmp.ctx = ctx;
  tmp.stream = (cudaStream_t)stream;
  const int32_t n = A->n;
  MatView Av{n, A->nnz, A->rowptr, A->col, A->val};
  spg_status st = validate_device(ctx, Av, tmp.stream);
  TransposeWork w{};
  void* scan_tmp = nullptr;
  if (st == SPG_OK) st = palloc(&tmp, &w.cnt, n);
  if (st == SPG_OK) st = palloc(&tmp, &w.cursor, n);
  if (st == SPG_OK) st = palloc(&tmp, (char**)&scan_tmp, (int64_t)scan_tmp_bytes(n));
  if (st == SPG_OK) st = palloc(&tmp, &w.tmp_col, A->nnz);
  if (st == SPG_OK) st = palloc(&tmp, &w.tmp_val, A->nnz);
  if (st == SPG_OK) st = palloc(&tmp, &w.long_list, n);
  if (st == SPG_OK) st = palloc(&tmp, &w.long_count, 1);
  w.scan_tmp = scan_tmp;
  w.status = ctx->d_status;
  if (st == SPG_OK) {
    cudaError_t e = launch_transpose(Av, t_rowptr, t_col, t_val, w, ctx->num_sms, tmp.stream);
    if (e != cudaSuccess) st = cuda_status(e, "transpose");
  }
  for (void* ptr : tmp.ptrs) cudaFreeAsync(ptr, tmp.stream);
  tmp.ptrs.clear();
  return st;
}

spg_status spg_describe(spg_ctx* ctx, const spg_csr_dev* A, spg_descriptors* d, void* stream) {
  begin_call();
  if (!ctx || !d) return set_error(SPG_ERR_INVALID_ARG, "null argument");
  TRY(check_matrix(A));
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  cudaStream_t st = (cudaStream_t)stream;
  const int32_t n = A->n;
  MatView Av{n, A->nnz, A->rowptr, A->col, A->val};
  TRY(validate_device(ctx, Av, st));
  spg_plan tmp;
  tmp.ctx = ctx;
  tmp.stream = st;
  int32_t* cc = nullptr;
  DescAccum* acc = nullptr;
  spg_status s = palloc(&tmp, &cc, n);
  if (s == SPG_OK) s = palloc(&tmp, &acc, 1);
  if (s == SPG_OK) {
    cudaError_t e = cudaMemsetAsync(cc, 0, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), st);
    if (e == cudaSuccess) e = cudaMemsetAsync(acc, 0, sizeof(DescAccum), st);
    if (e == cudaSuccess) e = launch_col_count(Av, cc, st);
    if (e == cudaSuccess) e = launch_describe(Av, cc, acc, st);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(ctx->h_pin, acc, sizeof(DescAccum), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = cuda_status(e, "describe");
  }
  for (void* ptr : tmp.ptrs) cudaFreeAsync(ptr, st);
  tmp.ptrs.clear();
  if (s != SPG_OK) return s;
  DescAccum h;
  std::memcpy(&h, ctx->h_pin, sizeof(h));
  std::memset(d, 0, sizeof(*d));
  d->n = n;
  d->nnz = A->nnz;
  const double nn = n > 0 ? (double)n : 1.0;
  const double nz = A->nnz > 0 ? (double)A->nnz : 1.0;
  d->mean_deg = (double)A->nnz / nn;
  const double var = (double)h.sum_deg2 / nn - d->mean_deg * d->mean_deg;
  d->deg_cv = std::sqrt(var > 0 ? var : 0.0) / (d->mean_deg > 1e-9 ? d->mean_deg : 1e-9);
  d->products_aa = (int64_t)h.prod_aa;
  d->products_aat = (int64_t)h.prod_aat;
  d->fill_aa = (double)h.prod_aa / nz;
  d->fill_aat = (double)h.prod_aat / nz;
  d->max_deg = h.max_deg;
  d->max_col_deg = h.max_col_deg;
  d->bandwidth = h.bandwidth;
  d->pattern_symmetry = A->nnz > 0 ? (double)h.sym_hits / nz : 1.0;
  return SPG_OK;
}

spg_status spg_profile_enable(spg_ctx* ctx, int32_t enable) {
  begin_call();
  if (!ctx) return set_error(SPG_ERR_INVALID_ARG, "null context");
  ctx->prof = enable != 0;
  return SPG_OK;
}

spg_status spg_profile_reset(spg_ctx* ctx) {
  begin_call();
  if (!ctx) return set_error(SPG_ERR_INVALID_ARG, "null context");
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  prof_resolve(ctx);
  ctx->prof_acc.clear();
  ctx->launch_base = g_kernel_launches;
  return SPG_OK;
}

spg_status spg_profile_read(spg_ctx* ctx, char* json, size_t capacity) {
  begin_call();
  if (!ctx || !json || capacity == 0) return set_error(SPG_ERR_INVALID_ARG, "bad arguments");
  TRY_CUDA(cudaSetDevice(ctx->device), "set device");
  prof_resolve(ctx);  // waits for each recorded kernel's end event, nothing else
  std::string out = "{\"launches\": " + std::to_string(g_kernel_launches - ctx->launch_base) +
                    ", \"kernels\": {";
  bool first = true;
  char buf[160];
  for (const auto& kv : ctx->prof_acc) {
    std::snprintf(buf, sizeof(buf), "%s\"%s\": {\"count\": %lld, \"ms\": %.6f}", first ? "" : ", ",
                  kv.first.c_str(), kv.second.second, kv.second.first);
    out += buf;
    first = false;
  }
  out += "}}";
  if (out.size() + 1 > capacity)
    return set_error(SPG_ERR_INVALID_ARG, "profile text needs %zu bytes", out.size() + 1);
  std::memcpy(json, out.c_str(), out.size() + 1);
  return SPG_OK;
}

spg_status spg_checksum(const double* dev_val, int64_t count, double* s, double* as, double* sq) {
  begin_call();
  if (!s || !as || !sq || count < 0 || (count > 0 && !dev_val))
    return set_error(SPG_ERR_INVALID_ARG, "bad checksum arguments");
  std::vector<double> h((size_t)count);
  if (count > 0)
    TRY_CUDA(cudaMemcpy(h.data(), dev_val, sizeof(double) * (size_t)count, cudaMemcpyDeviceToHost),
             "checksum copy");
  double a = 0, b = 0, c = 0;
  for (double x : h) {
    a += x;
    b += x < 0 ? -x : x;
    c += x * x;
  }
  *s = a;
  *as = b;
  *sq = c;
  return SPG_OK;
}

spg_status spg_run_ours(const char* task, const int32_t* dOff, const int32_t* dCol,
                        const double* dVal, int32_t n, int64_t nnz, int32_t reps,
                        spg_eng_result* out) {
  begin_call();
  bool ok;
  spg_task t = parse_task(task, &ok);
  if (!ok) return set_error(SPG_ERR_INVALID_ARG, "task must be AA, AAt or AAtS");
  if (!out || reps < 0) return set_error(SPG_ERR_INVALID_ARG, "bad arguments");
  static thread_local spg_ctx* ctx = nullptr;
  static thread_local int ctx_dev = -1;
  int dev = 0;
  TRY_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
  if (!ctx || ctx_dev != dev) {
    if (ctx) spg_destroy(ctx);
    ctx = nullptr;
    TRY(spg_create(&ctx, nullptr));
    ctx_dev = dev;
  }
  spg_csr_dev A{n, nnz, dOff, dCol, dVal};
  spg_csr_out C{};
  // one checked call
  TRY(spg_multiply(ctx, t, &A, &C, nullptr));
  double s = 0, as = 0, sq = 0;
  spg_status st = spg_checksum(C.val, C.nnz, &s, &as, &sq);
  const int64_t nnz_c = C.nnz;
  spg_free(ctx, C.rowptr, nullptr);
  spg_free(ctx, C.col, nullptr);
  spg_free(ctx, C.val, nullptr);
  if (st != SPG_OK) return st;
  TRY_CUDA(cudaStreamSynchronize(nullptr), "sync");  // the calls' own stream, as run_ours
  float ms = 0.f;
  if (reps > 0) {
    cudaEvent_t e0, e1;
    TRY_CUDA(cudaEventCreate(&e0), "event");
    TRY_CUDA(cudaEventCreate(&e1), "event");
    cudaEventRecord(e0, nullptr);
    for (int r = 0; r < reps && st == SPG_OK; ++r) {
      spg_csr_out Cr{};
      st = spg_multiply(ctx, t, &A, &Cr, nullptr);
      if (st == SPG_OK) {
        spg_free(ctx, Cr.rowptr, nullptr);
        spg_free(ctx, Cr.col, nullptr);
        spg_free(ctx, Cr.val, nullptr);
      }
    }
    cudaEventRecord(e1, nullptr);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    ms /= (float)reps;
  }
  if (st != SPG_OK) return st;
  out->ms = ms;
  out->nnz = nnz_c;
  out->s = s;
  out->as = as;
  out->sq = sq;
  return SPG_OK;
}

}  // extern "C"
