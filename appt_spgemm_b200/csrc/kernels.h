// Host-side launchers of the engine's kernels (defined in the k_*.cu files).
// Every launcher is asynchronous on `stream` and returns the launch error.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "device_common.cuh"
#include "internal.h"

namespace spg {

// Kernels launched by the engine on this thread (every <<<>>> site counts).
extern thread_local long long g_kernel_launches;
#define SPG_COUNT_LAUNCH() (++::spg::g_kernel_launches)

// ---- validation / pre-pass / binning (k_prepass.cu) --------------------------

// Flags DEV_ERR_BAD_INDEX / sets *bad (device int) when A is not a square CSR
// with rowptr[0]=0, monotone rowptr, rowptr[n]=nnz, columns in [0,n) strictly
// increasing within each row.
cudaError_t launch_validate(const MatView& A, uint32_t* status, cudaStream_t s);

// Per row i of C = A·B: products f_i = Σ_{k∈A_i} nnz(B_k) and the column span
// [lo_i, hi_i] of the output row (B rows sorted).  Rows with f_i = 0 get
// lo = INT_MAX, hi = -1; rows that meet an index out of range f_i = −1.  With
// `status`, A is validated in the same pass (launch_validate's checks).
cudaError_t launch_prepass(const MatView& A, const MatView& B, int64_t* f, int32_t* lo,
                           int32_t* hi, cudaStream_t s, uint32_t* status = nullptr);

// What a row's bin is computed from.
struct BinSource {
  int mode;                 // 0: symbolic (from products and span), 1: numeric (from counts)
  int32_t n;
  const int64_t* f;
  const int32_t* lo;
  const int32_t* hi;
  const int32_t* rownnz;    // numeric: entries of the row (plain) or the row total (gram)
  const int32_t* rowlow;    // numeric gram: lower-part count (bin uses rownnz − rowlow)
  int max_log2;             // largest shared table (log2 slots) before the heavy path
  int force_heavy;
  int load_pct;             // table sized for at most this load (percent)
  // symbolic: rows with min(products, span) >= heavy_min also go heavy, so
  // every row the numeric binning sends to the heavy path has block counts
  // from the heavy symbolic kernel (0: no such rule)
  int64_t heavy_min;
  // rows fed by short B rows (products < short_split × nnz(A row); 0: no such
  // rule) go heavy already above 2^short_max_log2 slots (numeric) or from
  // min(products, span) >= short_min (symbolic): the windowed warp kernel
  // serves them better than the CTA-per-row tables, whose per-k barrier idles
  // most of the CTA on short B rows
  const int32_t* arowptr;
  int64_t short_split;
  int short_max_log2;
  int64_t short_min;
  // rows whose output span fits 2^dense_max_log2w bitmap words and is at most
  // 8 columns per product, with at least 64 products (and, numeric, at most
  // kDenseVals entries) take the bitmap bins; dense_max_log2w < kDenseMinLog2W:
  // never (the Gram path, or switched off)
  int dense_max_log2w;
};

__host__ __device__ __forceinline__ int ceil_log2_64(int64_t x) {
  int l = 0;
  while (((int64_t)1 << l) < x) ++l;
  return l;
}

// Table size rule: symbolic tables hold keys only and are sized for the load
// limit (default 75%) of min(products, span); numeric tables hold key+value
// and are sized for the load limit (default 66%) of the exact row count.
// Bin b in 1..kNumTableBins means 2^(b+kMinTableLog2−1) slots.
__host__ __device__ __forceinline__ int row_bin(const BinSource& s, int i) {
  int64_t size;
  if (s.mode == 0) {
    int64_t f = s.f[i];
    if (f <= 0) return kEmptyBin;
    int64_t span = (int64_t)s.hi[i] - (int64_t)s.lo[i] + 1;
    size = f < span ? f : span;
  } else {
    int64_t m = s.rownnz[i] - (s.rowlow ? s.rowlow[i] : 0);
    if (m <= 0) return kEmptyBin;
    size = m;
  }
  const int64_t want = size * 100 / s.load_pct + 1;
  if (s.force_heavy) return kHeavyBin;
  if (s.mode == 0 && s.heavy_min > 0 && size >= s.heavy_min) return kHeavyBin;
  if (s.dense_max_log2w >= kDenseMinLog2W) {
    const int64_t words = ((int64_t)s.hi[i] - s.lo[i] + 32) >> 5;
    const int64_t f = s.f[i];
    // (symbolic: only rows the numeric binning can never send heavy, which
    // need the heavy symbolic kernel's block counts)
    // the bitmap's bookkeeping (clearing, counting, prefixes) grows with the
    // span: worth it only where the span is at most 8 columns per product
    if (f >= 64 && words * 4 <= f && words <= ((int64_t)1 << s.dense_max_log2w) &&
        (s.mode == 0 ? (s.short_split <= 0 || size < s.short_min) : size <= kDenseVals)) {
      int lw = ceil_log2_64(words);
      if (lw < kDenseMinLog2W) lw = kDenseMinLog2W;
      return kDenseBin0 + lw - kDenseMinLog2W;
    }
  }
  int lg = ceil_log2_64(want);
  if (lg < kMinTableLog2) lg = kMinTableLog2;
  if (lg > s.max_log2) return kHeavyBin;
  if (s.short_split > 0 &&
      s.f[i] < s.short_split * ((int64_t)s.arowptr[i + 1] - s.arowptr[i]) &&
      (s.mode == 0 ? size >= s.short_min : lg > s.short_max_log2))
    return kHeavyBin;
  return lg - kMinTableLog2 + 1;
}

constexpr int kBinRowsPerBlock = 1024;  // rows per block of the binning kernels

// Stable binning: rows of each bin listed in increasing row order.
//   hist:  int32[kNumBins * nblocks] (bin-major), nblocks = ceil(n / 1024)
//   counts_out: int64[2*kNumBins] on the device → {count[b]} then {start[b]}
cudaError_t launch_bin_rows(const BinSource& src, int32_t* hist, int64_t* counts_out,
                            int32_t* rows_out, cudaStream_t s);

// Exclusive scan of int32 counts into int64 offsets out[0..n], out[n] = total.
// `tmp` needs scan_tmp_bytes(n) bytes.
size_t scan_tmp_bytes(int64_t n);
cudaError_t launch_scan_i32_i64(const int32_t* in, int64_t* out, int64_t n, void* tmp,
                                cudaStream_t s);
// Same with int32 output (caller guarantees the total fits in int32).
cudaError_t launch_scan_i32_i32(const int32_t* in, int32_t* out, int64_t n, void* tmp,
                                cudaStream_t s);

// ---- shared-memory hash rows (k_rows.cu) ------------------------------------

struct RowArgs {
  MatView A, B;
  const int32_t* rows;      // this bin's rows (nullptr: rows 0..nrows-1)
  int32_t nrows;
  int32_t G;                // lanes per row (warp bins); CTA bins use blockDim
  // symbolic outputs
  int32_t* rownnz;
  int32_t* rowlow;          // gram: columns < row
  // numeric inputs / outputs
  const int64_t* rowptr;    // C row pointers
  const int32_t* cnt_in;    // symbolic counts (expected entries)
  const int32_t* low_in;    // gram: lower counts
  int32_t* ccol;
  double* cval;
  // gram mirror: strict-upper entries appended to a temporary lower store
  const int64_t* lowptr;
  int32_t* cursor;
  int32_t* lcol;
  double* lval;
  uint32_t* status;
  // output column span per row (pre-pass): keys of row i lie in [lo[i], hi[i]]
  const int32_t* lo;
  const int32_t* hi;
  // batched plans: first column of the row's instance, subtracted from every
  // column index written (nullptr for a single matrix)
  const int32_t* colbase;
  // CTA-per-row bins: in a persistent launch rows are drawn from this counter
  // (zeroed by the launcher) as CTAs free up; nullptr: dealt out in turn
  int32_t* queue;
  // the one-readback plan's symbolic launch (warp kernels): rows whose
  // pre-pass product count is negative (an invalid index met) or above fcap
  // (beyond the table) are skipped with a zero count, the latter reported as
  // DEV_ERR_SMALL_CAP; nullptr: every row is processed
  const int64_t* fsmall;
  int64_t fcap;
};

// Writes m sorted packed words ((col − lo) << LOG2T | slot) as a row's columns
// and the values of their table slots, lanes first, first + stride, … (so the
// stores are coalesced); the Gram path also mirrors each entry above the
// diagonal into the lower store through the column's atomic cursor.
template <int LOG2T, bool GRAM>
__device__ __forceinline__ void emit_packed(const RowArgs& a, int row, int lo, int m,
                                            const uint32_t* sorted, const double* vals,
                                            int64_t base, int first, int stride) {
  const int cb = a.colbase ? a.colbase[row] : 0;
  for (int e = first; e < m; e += stride) {
    const uint32_t pk = sorted[e];
    const int j = lo + (int)(pk >> LOG2T);
    const double v = vals[pk & ((1u << LOG2T) - 1u)];
    a.ccol[base + e] = j - cb;
    a.cval[base + e] = v;
    if (GRAM && j > row) {
      const int pos = atomicAdd(&a.cursor[j], 1);
      if (pos < a.low_in[j]) {
        const int64_t d = a.lowptr[j] + pos;
        a.lcol[d] = row - cb;
        a.lval[d] = v;
      } else {
        report(a.status, DEV_ERR_OVERFLOW);
      }
    }
  }
}

// Number of bits needed for the column field of a row spanning [lo, hi].
__device__ __forceinline__ int span_bits(int lo, int hi) {
  const uint32_t span = (uint32_t)(hi - lo);
  return span ? 32 - __clz((int)span) : 0;
}

// Numeric-zero compaction (k_compact.cu): kept (non-zero) entries per row of
// C, and the kept entries of rows [r0, r1) gathered in order into tcol/tval
// at newptr[row] − newptr[r0].
cudaError_t launch_count_kept(const int64_t* rowptr, const double* val, int32_t n, int32_t* kept,
                              cudaStream_t s);
cudaError_t launch_gather_kept(const int64_t* rowptr, const int32_t* col, const double* val,
                               const int64_t* newptr, int32_t r0, int32_t r1, int32_t* tcol,
                               double* tval, cudaStream_t s);

// Warp-per-row kernels (k_rows_w32.cu) for table bins of up to 2048 slots
// with 32 lanes per row; returns cudaErrorNotSupported for other bins.
cudaError_t launch_hash_w32(int log2t, bool numeric, bool gram, const RowArgs& a, int num_sms,
                            cudaStream_t s);

// Launch the kernel of one table bin (1..kNumTableBins).  `gram` selects the
// A·Aᵀ upper-triangle variant (symbolic: split lower/upper counts; numeric:
// upper part only plus the mirror append).
cudaError_t launch_hash_bin(int bin, bool numeric, bool gram, const RowArgs& a, int num_sms,
                            cudaStream_t s);
// Warp-per-row bitmap kernels of the dense bins (k_dense_w32.cu; not Gram).
cudaError_t launch_dense_bin(int bin, bool numeric, const RowArgs& a, int num_sms,
                             cudaStream_t s);
int hash_bin_lanes(int bin, int lanes_cfg);

// ---- heavy rows: dense column windows (k_heavy.cu) --------------------------
struct HeavyArgs {
  RowArgs r;                // rows = heavy list, outputs as in RowArgs
  const int32_t* lo;        // output column span per row
  const int32_t* hi;
  int32_t window_bits;      // W (multiple of 32 * threads)
  // column blocks: heavy row i's span [lo, hi] is cut into blocks of
  // 2^blk_log2 columns from lo; blk_cnt[blk_off[i] + b] is the number of
  // distinct output columns in block b (saturated at 65535), written by the
  // symbolic kernel when blk_cnt is set and read by the windowed numeric one
  const int64_t* blk_off;   // per row (n + 1), 0 blocks for rows not heavy
  uint16_t* blk_cnt;
  int32_t blk_log2;
  int32_t cap;              // numeric: most distinct columns per window
  int32_t sub_log2;         // numeric: window width inside a block above cap
  int4* hcur;               // numeric: per entry of A {B cursor, B row end, next column, 0}
  int32_t vcap;             // shared-value CTA kernel: most values per window
  int32_t wcap_bits;        // shared-value CTA kernel: widest window (bitmap bits)
  // numeric: rows fed by many short B rows (mean length below `split`) take
  // the windowed warp kernel, rows dominated by long B rows the CTA kernel,
  // whose 1024 threads stream each long B row (each kernel skips the other's
  // rows); split 0: all to the CTA kernel
  int64_t split;
  const int64_t* f;         // products per row (pre-pass)
  // CTA kernels: in a persistent launch (fewer CTAs than rows) a CTA takes its
  // next row from this counter (launch_heavy zeroes it on the stream first),
  // so a CTA that drew hub rows does not hold the others back; required
  int32_t* queue;
};

// The heavy row goes to the windowed warp kernel: mean B-row length
// f / nnz(A row) below split, and at most kWarpRowMaxProducts products (one
// warp walks its row alone: a larger row would set the kernel's tail).
constexpr int64_t kWarpRowMaxProducts = (int64_t)1 << 17;
__device__ __forceinline__ bool heavy_row_windowed(const HeavyArgs& h, int row) {
  if (h.split <= 0 || h.f[row] > kWarpRowMaxProducts) return false;
  const int64_t len = (int64_t)h.r.A.rowptr[row + 1] - h.r.A.rowptr[row];
  return h.f[row] < h.split * len;
}
cudaError_t launch_heavy(bool numeric, bool gram, const HeavyArgs& a, int threads, int num_sms,
                         cudaStream_t s);
size_t heavy_smem_bytes(bool numeric, int threads, int window_bits);

// Blocks per row for the heavy rows of `bsym` (0 for the others), scanned into
// blk_off[0..n] (launch_scan_i32_i64 with tmp of scan_tmp_bytes(n)).
cudaError_t launch_heavy_blocks(const BinSource& bsym, int blk_log2, int32_t* nblk,
                                int64_t* blk_off, void* scan_tmp, cudaStream_t s);

// Numeric phase of the CTA rows with their values in shared memory, window by
// window (k_heavy_win.cu); needs blk_cnt, hcur and queue.
cudaError_t launch_heavy_win(bool gram, const HeavyArgs& a, int threads, int num_sms,
                             cudaStream_t s);
size_t heavy_win_smem_bytes(int threads, int vcap, int wcap_bits);

// Windowed numeric phase of heavy rows (k_heavy_w32.cu): a warp per row walks
// the row's column blocks in windows of at most `cap` distinct columns.
cudaError_t launch_heavy_w32(bool gram, const HeavyArgs& a, int num_sms, cudaStream_t s);
constexpr int kHeavyTableLog2 = 10;  // its shared table: 1024 slots per warp

// ---- transpose and segment sort (k_transpose.cu) ----------------------------

// Counting-sort transpose: t_rowptr (n+1) gets the column histogram scan,
// entries are appended per column with atomic cursors into (tmp_col, tmp_val),
// then each column is sorted by row into (t_col, t_val).
// Workspace: cnt/cursor int32[n], scan tmp, tmp_col/tmp_val [nnz], long list.
struct TransposeWork {
  int32_t* cnt;
  int32_t* cursor;
  void* scan_tmp;
  int32_t* tmp_col;
  double* tmp_val;
  int32_t* long_list;   // int32[n]
  int32_t* long_count;  // int32[1]
  uint32_t* status;
};
cudaError_t launch_transpose(const MatView& A, int32_t* t_rowptr, int32_t* t_col, double* t_val,
                             const TransposeWork& w, int num_sms, cudaStream_t s);
// Values of Aᵀ for a structurally symmetric A (Aᵀ keeps A's rowptr and col);
// sets *asym (device int, pre-zeroed) when some entry has no mirror.
cudaError_t launch_sym_transpose_vals(const MatView& A, double* t_val, int* asym, cudaStream_t s);

// Sort segments of unique int keys (with double payloads) from a source store
// into a destination store.  Segment s: source [src_off[s], +len), destination
// [dst_off[s], +len), len = lens ? lens[s] : src_off[s+1] − src_off[s].
struct SegSortArgs {
  int32_t nseg;
  const int64_t* src_off64;
  const int32_t* src_off32;
  const int64_t* dst_off64;
  const int32_t* dst_off32;
  const int32_t* lens;
  const int32_t* src_key;
  const double* src_val;
  int32_t* dst_key;
  double* dst_val;
  int32_t key_bound;     // keys lie in [0, key_bound)
  int32_t* long_list;
  int32_t* long_count;
  uint32_t* status;
};
cudaError_t launch_segsort(const SegSortArgs& a, int num_sms, cudaStream_t s);

// ---- batched plans (k_batch.cu) ---------------------------------------------
struct BatchDesc {          // one instance, as uploaded to the device
  const int32_t* rowptr;
  const int32_t* col;
  const double* val;
  int32_t n;
  int32_t pad;
  int64_t nnz;
  int64_t row_off;          // first row (and column) of the instance in the block diagonal
  int64_t nnz_off;          // first entry of the instance
};
// Block-diagonal concatenation: rowptr (N+1), col/val (NNZ) with columns offset
// by the instance's row_off, colbase[r] = row_off of row r's instance.  Sets
// *bad when an instance's rowptr does not run 0..nnz or a column leaves its block.
cudaError_t launch_batch_concat(const BatchDesc* d, const int64_t* row_off, const int64_t* nnz_off,
                                int count, int64_t N, int64_t NNZ, int32_t* rowptr, int32_t* col,
                                double* val, int32_t* colbase, uint32_t* bad, int num_sms,
                                cudaStream_t s);
// Refresh only the values of the block-diagonal copy from the instances.
cudaError_t launch_batch_vals(const BatchDesc* d, const int64_t* nnz_off, int count, int64_t NNZ,
                              double* val, int num_sms, cudaStream_t s);
// out[b] = rowptr_c[row_off[b]] for b = 0..count.
cudaError_t launch_gather_offsets(const int64_t* rowptr_c, const int64_t* row_off, int count,
                                  int64_t* out, cudaStream_t s);

// ---- descriptors ------------------------------------------------------------
struct DescAccum {        // device accumulators of spg_describe
  unsigned long long sum_deg2;   // Σ deg²
  unsigned long long prod_aa;    // Σ_{(i,k)} deg(k)
  unsigned long long prod_aat;   // Σ_k colcount²
  unsigned long long sym_hits;   // entries (i,j) with (j,i) present
  int max_deg;
  int max_col_deg;
  int bandwidth;
  int pad;
};
cudaError_t launch_describe(const MatView& A, const int32_t* colcount, DescAccum* acc,
                            cudaStream_t s);
// out[0] = Σ f, out[1] = max f, out[2] = max rownnz (out zeroed by the launcher).
cudaError_t launch_row_stats(const int64_t* f, const int32_t* rownnz, int32_t n,
                             unsigned long long* out, cudaStream_t s);
// Row pointers of a small plan and its row statistics: one launch when n fits
// one scan tile, else the scan and launch_row_stats.
cudaError_t launch_scan_stats_small(const int32_t* cnt, const int64_t* f, int64_t n,
                                    int64_t* rowptr, unsigned long long* stats, void* tmp,
                                    cudaStream_t s);
cudaError_t launch_col_count(const MatView& A, int32_t* cnt, cudaStream_t s);

}  // namespace spg
