/*
 * spgemm_b200.h — C ABI of the B200 (sm_100a) FP64 SpGEMM engine.
 *
 * Computes C = A·A, C = A·Aᵀ (plain) and C = A·Aᵀ through the symmetric Gram
 * path (upper triangle computed, lower triangle mirrored) for a square n×n CSR
 * matrix A with int32 row pointers / column indices and FP64 values, on one GPU.
 *
 * The reference surface this replaces is the header-only engine
 *   static EngResult run_ours(const char* task, const int* dOff, const int* dCol,
 *                             const double* dVal, int n, int64_t nnz, int reps);
 * (src/spgemm_engine.cuh:132-133), its result record EngResult
 * (src/spgemm_engine.cuh:129) and the CSR1 loader load_bin
 * (src/spgemm_engine.cuh:21-32).  spg_run_ours() reproduces run_ours; the
 * spg_plan_* / spg_execute / spg_multiply calls expose what run_ours keeps
 * internal (the product C itself, with int64 row pointers).
 *
 * Conventions
 *  - Every call returns an spg_status; nothing prints or exits.  The text of the
 *    last error on the calling thread is spg_last_error_string().
 *  - Device pointers are borrowed; streams are cudaStream_t passed as void*.
 *  - Output semantics are structural (pattern product): entries whose products
 *    cancel to 0.0 are kept as explicit zeros, as cuSPARSE and the reference do.
 *  - Column indices of every output row are sorted ascending.  Each output value
 *    is the sum of its products a_ik·b_kj taken in increasing position of k in
 *    row i of A, each product rounded before the add (no fused multiply-add), so
 *    results are bit-reproducible run to run.
 *  - One context per host thread; calls on one context are stream-ordered.
 */
#ifndef SPGEMM_B200_H
#define SPGEMM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPG_ABI_VERSION 1

typedef enum spg_status {
  SPG_OK = 0,
  SPG_ERR_INVALID_ARG = 1,   /* null pointer, bad task, n < 0, ...                */
  SPG_ERR_INVALID_CSR = 2,   /* rowptr not monotone, column out of range,
                                unsorted or duplicate columns in a row          */
  SPG_ERR_OOM = 3,           /* device (or pinned host) allocation failed         */
  SPG_ERR_CUDA = 4,          /* any other CUDA runtime error                      */
  SPG_ERR_HASH_FULL = 5,     /* a bounded hash probe ran out (device status word) */
  SPG_ERR_TIMEOUT = 6,       /* a bounded wait gave up                            */
  SPG_ERR_UNSUPPORTED = 7,   /* size beyond a documented limit                    */
  SPG_ERR_BUDGET = 8,        /* request exceeds the memory budget (admission)     */
  SPG_ERR_NOT_READY = 9,     /* asynchronous result not complete yet              */
  SPG_ERR_IO = 10            /* CSR1 file could not be read / written             */
} spg_status;

typedef enum spg_task {
  SPG_TASK_AA = 0,    /* C = A·A                                        ("AA")   */
  SPG_TASK_AAT = 1,   /* C = A·Aᵀ, Aᵀ built by the engine's transpose   ("AAt")  */
  SPG_TASK_AATS = 2   /* C = A·Aᵀ via upper triangle + mirror           ("AAtS") */
} spg_task;

/* Square CSR matrix on the device, borrowed (int32 row pointers: nnz < 2^31). */
typedef struct spg_csr_dev {
  int32_t n;
  int64_t nnz;
  const int32_t* rowptr; /* n+1 */
  const int32_t* col;    /* nnz, sorted and unique within each row */
  const double* val;     /* nnz */
} spg_csr_dev;

/* Output CSR with int64 row pointers.  For spg_execute the caller owns the
 * buffers (rowptr: n+1, col/val: nnz from the plan); for spg_multiply the
 * engine allocates them from the context pool (release with spg_free). */
typedef struct spg_csr_out {
  int32_t n;
  int64_t nnz;
  int64_t* rowptr;
  int32_t* col;
  double* val;
} spg_csr_out;

/* Engine tuning.  Zero-initialise and set struct_size = sizeof(spg_config);
 * every field left 0 takes its default.  The autotuner fills one of these. */
typedef struct spg_config {
  int32_t struct_size;
  int32_t device;             /* CUDA ordinal; 0 → current device (default)     */
  int32_t lanes_per_row;      /* lanes per row in the sub-warp bins: 4/8/16/32;
                                 0 → chosen from the mean row length of B        */
  int32_t max_smem_slots;     /* largest shared-memory numeric table (slots);
                                 rows beyond go to the heavy path; 0 → 8192      */
  int32_t heavy_threads;      /* threads per CTA on the heavy path; 0 → 512 when
                                 the window is ≤ 2^19 columns (two CTAs per SM),
                                 else 1024                                       */
  int32_t window_bits;        /* column-window width of the dense heavy path
                                 (bits of the shared bitmap, multiple of 1024,
                                 at most 2^20); 0 → the next power of two ≥ n,
                                 at most 2^20                                    */
  int32_t force_heavy;        /* 1 → send every non-empty row to the heavy path
                                 (debug oracle of the binning, as the reference
                                 did by forcing its global path)                 */
  int32_t sym_load_pct;       /* symbolic tables sized for at most this load of
                                 min(products, span), percent 20..90; 0 → 75     */
  int32_t num_load_pct;       /* numeric tables sized for at most this load of
                                 the exact row count, percent 20..90; 0 → 66     */
  int32_t heavy_split;        /* heavy rows of at most 2^17 products whose B
                                 rows average fewer entries than this take the
                                 warp-per-row windowed kernel, the others the
                                 CTA-per-row kernel (1: all CTA); 0 → 128      */
  int64_t pool_release_bytes; /* memory-pool release threshold; 0 → keep all    */
  int64_t heavy_block_budget; /* most per-block column counts kept for heavy
                                 rows (2 bytes each; blocks widen from 1024
                                 columns to stay within it, and without them
                                 every heavy row takes the CTA kernel);
                                 0 → 2^27                                       */
  int64_t grid_sms;           /* SMs the launches size their persistent grids
                                 for; 0 → the device's.  A larger value (up to
                                 2^16) gives one CTA per work item, so CTAs
                                 retire often and work on a higher-priority
                                 stream can start in between (the server's
                                 large-request workers use this)               */
  int64_t small_max_nnz;      /* A·A and A·Aᵀ of matrices with at most this many
                                 entries (and n <= 65,536) are planned with one
                                 host synchronisation (every row in one launch
                                 per phase); a row of more than 1536 products
                                 sends the plan to the regular path; 0 → 2^20,
                                 negative → never                               */
  int64_t heavy_vcap;         /* heavy CTA rows: > 0 → values held in shared
                                 memory per column window of at most this many
                                 columns (1024..16384, a power of two), each
                                 window's values written to C once; 0 or
                                 negative → accumulated in place in C (the
                                 dense-window kernel; the default: measured
                                 faster on R-MAT, the windows multiply the
                                 per-entry barriers)                            */
  int64_t dense_max_words;    /* > 0 → rows whose output column span fits this
                                 many 32-bit bitmap words (256..2048) and is at
                                 most 8 columns per product take the bitmap
                                 kernels (A·A, A·Aᵀ); 0 or negative → never (the
                                 default: the hash tables measured faster on
                                 the stencil)                                   */
  int32_t bin_streams;        /* > 1 → the kernels of different row bins of one
                                 phase run concurrently on up to this many
                                 streams (at most 4, forked from and joined back
                                 into the caller's stream); 0 or 1 → all on the
                                 caller's stream (the default: running the bins
                                 at once measured slower, their persistent
                                 grids contend for the SMs)                     */
  int32_t pad0;
} spg_config;

/* Result record of spg_run_ours: the reference's EngResult {ms, nnz, s, as, sq}
 * (src/spgemm_engine.cuh:129) — mean ms per call over `reps`, nnz(C), and the
 * order-independent checksums Σv, Σ|v|, Σv² of C's values. */
typedef struct spg_eng_result {
  float ms;
  int64_t nnz;
  double s, as, sq;
} spg_eng_result;

/* Structural facts gathered by the pre-pass and the symbolic phase. */
typedef struct spg_plan_info {
  int32_t n;
  int32_t task;
  int64_t nnz_a;
  int64_t nnz_c;              /* exact, structural                              */
  int64_t products;           /* Σ_{(i,k)} nnz(B_k): A·A  Σ_k nnz(A_k)… (metric) */
  int64_t products_computed;  /* products actually multiplied (AAtS: ~half)     */
  int64_t max_row_products;
  int64_t max_row_nnz;
  int64_t heavy_rows;         /* rows on the heavy (CTA-per-row) path           */
  int64_t workspace_bytes;    /* device workspace held by the plan              */
  int64_t output_bytes;       /* 8(n+1) + 12·nnz_c                              */
  int32_t bins_used;
  int32_t symmetric_pattern;  /* A·Aᵀ tasks: 1 when Aᵀ reused A's pattern      */
  int64_t exec_workspace_bytes; /* taken from the pool during each execute      */
} spg_plan_info;

/* Structural descriptors of A (the reference's dispatcher features,
 * bench/dispatch.cu:26-38, computed on the device). */
typedef struct spg_descriptors {
  int32_t n;
  int64_t nnz;
  double mean_deg;
  double deg_cv;              /* std(row nnz) / mean(row nnz)                    */
  double fill_aa;             /* Σ_{(i,k)} deg(k) / nnz                          */
  double fill_aat;            /* Σ_k colcount(k)² / nnz                          */
  int64_t products_aa;
  int64_t products_aat;
  int32_t max_deg;
  int32_t max_col_deg;
  int32_t bandwidth;          /* max |i − j| over entries                        */
  int32_t reserved;
  double pattern_symmetry;    /* fraction of entries (i,j) with (j,i) present    */
} spg_descriptors;

typedef struct spg_ctx spg_ctx;
typedef struct spg_plan spg_plan;

/* ---- version / errors ---------------------------------------------------- */
int32_t spg_abi_version(void);
const char* spg_last_error_string(void);
const char* spg_status_string(spg_status s);

/* ---- context -------------------------------------------------------------- */
spg_status spg_create(spg_ctx** ctx, const spg_config* cfg);
spg_status spg_destroy(spg_ctx* ctx);
/* Device status word written by kernels (bounded probes, …); reading it
 * synchronises the given stream.  Cleared on read. */
spg_status spg_check_device_status(spg_ctx* ctx, void* stream);

/* ---- plan / execute (replaces the sizing half of run_ours) ---------------- */
/* Pre-pass + binning + symbolic phase.  Two host synchronisations, each a
 * small pinned readback: the validity verdict on A with the bin sizes (and,
 * for A·Aᵀ, whether A's pattern is symmetric), then nnz(C); a third when an
 * A·Aᵀ pattern turns out not to be symmetric (it is transposed and binned
 * again); one (verdict, nnz(C) and row statistics together) for the small
 * matrices of spg_config.small_max_nnz.
 * When it returns, no kernel of the plan's symbolic phase is still running.
 * A must stay valid until the plan is destroyed. */
spg_status spg_plan_create(spg_ctx* ctx, spg_task task, const spg_csr_dev* A,
                           void* stream, spg_plan** plan);
spg_status spg_plan_get_info(const spg_plan* plan, spg_plan_info* info);
/* Upper bound of the plan workspace (spg_plan_info.workspace_bytes) that
 * spg_plan_create (batched = 0, count = 1) or spg_plan_create_batched
 * (batched = 1) would allocate for these inputs under ctx's configuration,
 * from their sizes alone (no device work): what a caller with a memory budget
 * reserves before planning.  The reference has no counterpart (its run_ours
 * allocates per call, src/spgemm_engine.cuh:137-181). */
spg_status spg_plan_workspace_bound(const spg_ctx* ctx, spg_task task, int32_t count,
                                    const spg_csr_dev* As, int32_t batched, int64_t* bytes);
/* Numeric phase + in-row sort (+ mirror for AAtS) into caller-owned buffers:
 * C->rowptr (n+1), C->col / C->val (info.nnz_c).  Asynchronous on `stream`.
 * A plan fixes the structure only: a plan may be executed again after A's
 * values (not its pattern) changed, and uses the current values.  Executes of
 * one plan must not overlap (they share the plan's workspace): order them on
 * one stream, or synchronise between streams; separate plans run concurrently. */
spg_status spg_execute(spg_plan* plan, spg_csr_out* C, void* stream);
spg_status spg_plan_destroy(spg_plan* plan);

/* Batched plan: `count` independent square matrices, C_b = A_b·A_b (or A_b·A_bᵀ)
 * for every b.  The instances are laid out on the device as one block-diagonal
 * matrix, so each phase of the plan and of spg_execute runs as one launch over
 * a binned row queue shared by all instances (no per-instance launches or host
 * syncs).  spg_execute then writes the concatenation: instance b owns rows
 * [row_off[b], row_off[b+1]) of C and entries [nnz_off[b], nnz_off[b+1]), with
 * its own column indices.  A_b arrays must stay valid until execution ends. */
spg_status spg_plan_create_batched(spg_ctx* ctx, spg_task task, int32_t count,
                                   const spg_csr_dev* As, void* stream, spg_plan** plan);
/* Instance offsets of a batched plan: row_off and nnz_off hold count+1 entries. */
spg_status spg_plan_batch_offsets(const spg_plan* plan, int64_t* row_off, int64_t* nnz_off);

/* CUDA graph of spg_execute for a plan and fixed output buffers: capture once,
 * launch many times (same structure, same buffers; values of A may change). */
typedef struct spg_graph spg_graph;
spg_status spg_graph_capture(spg_plan* plan, spg_csr_out* C, void* stream, spg_graph** graph);
spg_status spg_graph_launch(spg_graph* graph, void* stream);
spg_status spg_graph_destroy(spg_graph* graph);

/* Replace the tuning of a context (applies to plans created afterwards). */
spg_status spg_set_config(spg_ctx* ctx, const spg_config* cfg);
spg_status spg_get_config(const spg_ctx* ctx, spg_config* cfg);
/* Autotuner: times spg_plan_create + spg_execute of `task` on A (a single
 * matrix, or a batched set when count > 1) over candidate bin thresholds,
 * table loads, lanes per row and heavy-path shapes (coordinate descent,
 * median of `reps` timings each), leaves the best tuning in the context and
 * copies it to *best.  Costs a few dozen products of A. */
spg_status spg_autotune(spg_ctx* ctx, spg_task task, int32_t count, const spg_csr_dev* As,
                        int32_t reps, spg_config* best, void* stream);
/* Candidates of the last spg_autotune on ctx: `timed` configurations run
 * (the start included), `pruned` left out because A's structural features
 * (spg_describe: mean degree, largest row and column degree; the features the
 * reference's dispatcher reads, bench/dispatch.cu:26-38) rule them out. */
spg_status spg_autotune_trials(const spg_ctx* ctx, int32_t* timed, int32_t* pruned);

/* ---- serving ---------------------------------------------------------------
 * A request loop for A·A / A·Aᵀ requests of different sizes.  Worker threads,
 * each with its own stream and engine context, take queued requests as they
 * arrive; several requests are in flight on the device at once.  Requests on
 * small matrices (n < batch_rows) that are queued together with the same task
 * are merged into one batched plan (continuous batching).  Admission: after the
 * symbolic pass gives a request's exact output size, its output plus plan
 * workspace is reserved against the memory budget; a request waits until
 * enough is free (results released), and a request larger than the whole budget
 * is rejected with SPG_ERR_BUDGET.  Inputs and results stay on the device. */
typedef struct spg_server spg_server;
typedef struct spg_server_config {
  int32_t struct_size;
  int32_t workers;             /* requests (or merged batches) in flight; 0 → 4   */
  int64_t memory_budget_bytes; /* device memory reserved at once; 0 → 150 GB     */
  int32_t batch_rows;          /* n below which requests may be merged; 0 → 65536 */
  int32_t batch_max;           /* requests per merged batch; 0 → 64              */
  int64_t reserved[4];
} spg_server_config;

typedef struct spg_request_info {
  uint64_t id;
  int32_t status;              /* SPG_OK done, SPG_ERR_NOT_READY queued/running,
                                  SPG_ERR_BUDGET rejected, other: failed        */
  int32_t task;
  int32_t n;
  int32_t batched;             /* 1 when it ran inside a merged batch           */
  int64_t nnz_c;
  int64_t products;            /* intermediate products; for a request run in a
                                  merged batch, the batch's products split by
                                  the request's share of the output            */
  int64_t reserved_bytes;
  double submit_ms;            /* host clock, ms since the server started       */
  double start_ms;             /* a worker took it from the queue               */
  double done_ms;              /* the GPU finished this request's product        */
  double planned_ms;           /* its (last) symbolic pass ended                */
  double run_ms;               /* admitted with its exact need; execute began   */
} spg_request_info;

typedef struct spg_server_stats {
  int64_t submitted, completed, rejected, failed, batches;
  int64_t products_completed;
  int64_t budget_bytes, reserved_bytes, peak_reserved_bytes;
  double p50_ms, p99_ms, max_ms;   /* latency submit → done of completed requests */
  double first_submit_ms, last_done_ms;
  int64_t held_bytes;          /* device bytes the server holds now: plans,
                                  execute workspace, results not yet released */
  int64_t peak_held_bytes;     /* their peak; never above budget_bytes          */
} spg_server_stats;

spg_status spg_server_create(const spg_server_config* cfg, spg_server** out);
/* Queue a request on a device CSR that stays valid until the request is done. */
spg_status spg_server_submit(spg_server* s, spg_task task, const spg_csr_dev* A, uint64_t* id);
spg_status spg_server_poll(spg_server* s, uint64_t id, spg_request_info* info);
/* Wait until the request is done, rejected or failed; SPG_ERR_TIMEOUT after
 * timeout_ms (negative: no limit). */
spg_status spg_server_wait(spg_server* s, uint64_t id, int32_t timeout_ms, spg_request_info* info);
/* Copy a finished result into caller buffers (device or host): rowptr n+1
 * int64, col/val nnz_c (col and val are checked before anything is copied).
 * The server keeps the result until released; a release issued by another
 * thread during the copy waits for the copy to end. */
spg_status spg_server_copy_result(spg_server* s, uint64_t id, int64_t* rowptr, int32_t* col,
                                  double* val);
/* Drop a finished result: frees its device memory and returns its budget,
 * after any copy of it still running in another thread has ended. */
spg_status spg_server_release(spg_server* s, uint64_t id);
spg_status spg_server_stats_get(spg_server* s, spg_server_stats* st);
/* Stops the workers: requests running on the device finish; a request that
 * would still have to wait for budget ends with an error status instead of
 * running.  Then frees all results.  The server's functions may be called
 * from several host threads; destroy is the last call. */
spg_status spg_server_destroy(spg_server* s);

/* plan + execute with C allocated from the context pool; C->nnz is set. */
spg_status spg_multiply(spg_ctx* ctx, spg_task task, const spg_csr_dev* A,
                        spg_csr_out* C, void* stream);
/* Release a buffer returned by spg_multiply (stream-ordered). */
spg_status spg_free(spg_ctx* ctx, void* dev_ptr, void* stream);

/* ---- profiling ------------------------------------------------------------ */
/* Per-kernel CUDA events recorded on the launching stream (off by default) and
 * a count of the engine's kernel launches on the calling thread.
 * spg_profile_read waits for the recorded kernels (their end events, not the
 * whole device) and writes JSON text
 *   {"launches": L, "kernels": {"<phase>/<kernel>": {"count": c, "ms": t}, ...}}
 * covering the calls since the last spg_profile_reset. */
spg_status spg_profile_enable(spg_ctx* ctx, int32_t enable);
spg_status spg_profile_reset(spg_ctx* ctx);
spg_status spg_profile_read(spg_ctx* ctx, char* json, size_t capacity);

/* ---- numeric-zero switch ----------------------------------------------------
 * Drop, in place, the entries of a finished product C whose value is exactly
 * zero (+0.0 or −0.0), keeping the others in order and updating C->rowptr and
 * C->nnz: the pattern scipy's eliminate_zeros() leaves.  The products
 * themselves keep cancelled entries, as the reference and cuSPARSE do
 * (report/CORRECTNESS_NOTES.md:3-16, :16 names this switch).  Works through
 * a bounded workspace in row chunks, so any size of C compacts in place; it
 * synchronizes `stream` once to learn the new size.  On an error C may be
 * partly compacted. */
spg_status spg_drop_zeros(spg_ctx* ctx, spg_csr_out* C, void* stream);

/* ---- transpose (CSR → CSR of Aᵀ, counting sort; rows sorted) ------------- */
/* Replaces k_colcount/k_scatter/build_At (src/spgemm_engine.cuh:37-44,140-146)
 * with a deterministic result.  Caller-owned outputs: rowptr n+1, col/val nnz. */
spg_status spg_transpose(spg_ctx* ctx, const spg_csr_dev* A, int32_t* t_rowptr,
                         int32_t* t_col, double* t_val, void* stream);

/* Transpose that allocates nothing.  No counterpart in the reference.
 * For callers that may not allocate device memory — applications that carve
 * all GPU memory up front and forbid libraries from calling cudaMalloc /
 * cudaFree, or latency-critical paths where an allocation may synchronise the
 * device.  Same result as spg_transpose; the caller passes A and the outputs
 * (rowptr n+1, col/val nnz), no context.  Its scratch is a static device array
 * of about 6.8 MB that every GPU loading the library holds until exit, which
 * limits A to n <= 65,536 and nnz <= 524,288 (larger inputs: SPG_ERR_UNSUPPORTED).
 * It runs on the current device, and A and the outputs must live there (a
 * buffer on another GPU: SPG_ERR_INVALID_ARG).  The first call on each device
 * resolves that array's address (set-up) and keeps it; make that first call
 * before any stream capture, and do not use the library across a
 * cudaDeviceReset of the device.  All calls share the array: calls that
 * overlap on the GPU (different streams, or threads) race.  Every call first
 * validates A on `stream` and waits there for the verdict (a device-to-host
 * copy and a stream synchronisation), then runs the transpose asynchronously
 * on `stream`. */
spg_status spg_transpose_noalloc(const spg_csr_dev* A, int32_t* t_rowptr, int32_t* t_col,
                                 double* t_val, void* stream);

/* ---- descriptors ----------------------------------------------------------- */
spg_status spg_describe(spg_ctx* ctx, const spg_csr_dev* A, spg_descriptors* d,
                        void* stream);

/* ---- reference-compatible call -------------------------------------------- */
/* Same semantics as run_ours (src/spgemm_engine.cuh:132-210): task "AA", "AAt"
 * or "AAtS"; one checked call, then `reps` timed full calls (plan + execute +
 * transpose), mean ms; nnz(C) and checksums of C's values.  Uses an internal
 * context on the current device and the legacy default stream. */
spg_status spg_run_ours(const char* task, const int32_t* dOff, const int32_t* dCol,
                        const double* dVal, int32_t n, int64_t nnz, int32_t reps,
                        spg_eng_result* out);

/* Order-independent checksums of a device FP64 array (Σv, Σ|v|, Σv²), summed
 * on the host in index order like checksum() (src/spgemm_engine.cuh:116-118). */
spg_status spg_checksum(const double* dev_val, int64_t count, double* s,
                        double* as, double* sq);

/* ---- CSR1 files (src/export_bin.py:6-8 format, load_bin :21-32) ----------- */
/* Host CSR in malloc'd buffers; release with spg_host_csr_free. */
typedef struct spg_host_csr {
  int32_t n;
  int64_t nnz;
  int32_t* rowptr;
  int32_t* col;
  double* val;
} spg_host_csr;
spg_status spg_csr1_read(const char* path, spg_host_csr* out);
spg_status spg_csr1_write(const char* path, const spg_host_csr* A);
void spg_host_csr_free(spg_host_csr* A);
/* Validate a host CSR (monotone rowptr, columns in range, sorted, unique). */
spg_status spg_host_csr_validate(const spg_host_csr* A);

/* ---- synthetic generators (host, deterministic, seeded) ------------------- */
/* 2-D 5-point Laplacian on a side×side grid: 4.0 diagonal, −1.0 neighbours. */
spg_status spg_gen_laplace2d(int32_t side, spg_host_csr* out);
/* 3-D 27-point stencil on side³, values uniform(−1,1) from mt19937_64(seed)
 * drawn per entry in CSR order. */
spg_status spg_gen_stencil27(int32_t side, uint64_t seed, spg_host_csr* out);
/* R-MAT: 2^scale rows, edge_factor·2^scale edge draws with quadrant
 * probabilities (a,b,c,1−a−b−c), duplicates merged into one entry, self-loops
 * kept, values uniform(0,1) drawn per merged entry in CSR order. */
spg_status spg_gen_rmat(int32_t scale, int32_t edge_factor, double a, double b,
                        double c, uint64_t seed, spg_host_csr* out);
/* Random banded: half-bandwidth bw, each off-diagonal in-band entry kept with
 * probability fill, diagonal always present, values uniform(−1,1). */
spg_status spg_gen_banded(int32_t n, int32_t bw, double fill, uint64_t seed,
                          spg_host_csr* out);
/* Erdős–Rényi: row nnz ~ Poisson(lambda) (capped at n), columns uniform
 * without replacement, values uniform(−1,1). */
spg_status spg_gen_er(int32_t n, double lambda, uint64_t seed, spg_host_csr* out);
/* Uniform random sparse matrix with exactly `per_row` sorted random columns in
 * each row (capped at n), values uniform(−1,1); a test workhorse. */
spg_status spg_gen_uniform(int32_t n, int32_t per_row, uint64_t seed,
                           spg_host_csr* out);

#ifdef __cplusplus
}
#endif
#endif /* SPGEMM_B200_H */
