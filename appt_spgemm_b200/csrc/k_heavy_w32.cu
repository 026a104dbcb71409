// Heavy rows, numeric phase: a warp per row, streamed through column windows.
//
// A heavy row's output does not fit one shared table, so its column span
// [lo, hi] is walked in windows [c0, c1) that each hold at most `cap`
// distinct columns.  The window bounds come from the symbolic phase, which
// recorded the distinct-column count of every block of 2^blk_log2 columns:
// consecutive blocks are grouped while their counts sum to at most `cap`, and
// a block above `cap` on its own is cut into windows of 2^sub_log2 <= cap
// columns (which can never hold more than cap columns).
//
// Per row, every entry p of A's row keeps a cursor into the sorted B row
// k = A.col[p] (global int4 {cursor, row end, next column, 0}).  A window
// visits the entries in order of p, skips those whose next column is >= c1
// (one ballot over 32 entries), and for the others inserts the B entries below
// c1 32 at a time, advancing the cursor; every product is therefore read once
// over all windows.  Insertion is the warp kernels' CAS-first probe with lazy
// value init and one __syncwarp per 32-entry segment, so every value is
// Σ_k a_ik·b_kj added in increasing position of k with each product rounded
// first — bit-identical to the shared-table rows and to the CPU oracle.  The
// first segments of up to D active entries are loaded before any of them is
// inserted.
//
// A finished window is compacted, radix-sorted on (column − c0) in the
// table's own free space and written to the next slots of the row: windows
// are disjoint and increasing, so the row comes out sorted.  No CTA barrier,
// no global read-modify-write: the row's values are written once.
#include <climits>

#include "kernels.h"

namespace spg {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kHeavyD = 4;  // segments loaded ahead

// First block after the window that starts at block b: the longest run of
// blocks (at most max_blocks) whose counts sum to at most cap.  Counts are
// non-negative, so the lanes whose running sum stays within cap form a prefix.
__device__ __forceinline__ int window_end(const uint16_t* cnt, int b, int nb, int cap,
                                          int max_blocks) {
  const int lane = threadIdx.x & 31;
  const int lim = min(nb, b + max_blocks);
  int e = b, tot = 0;
  for (;;) {
    const int idx = e + lane;
    int c = idx < lim ? (int)cnt[idx] : cap + 1;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, c, o);
      if (lane >= o) c += t;
    }
    c += tot;
    const int n_ok = __popc(__ballot_sync(kFull, c <= cap));
    if (n_ok > 0) tot = __shfl_sync(kFull, c, n_ok - 1);
    e += n_ok;
    if (n_ok < 32) break;
  }
  return e;
}

// One window [c0, c1) of row `row`: accumulate, sort and write its entries at
// base + written; returns the number of entries written.
template <int LOG2T, bool GRAM>
__device__ __forceinline__ int heavy_window(const HeavyArgs& h, int row, int ps, int pe, int c0, int c1,
                           int* keys, double* vals, int64_t base, int64_t room) {
  constexpr int T = 1 << LOG2T;
  const RowArgs& a = h.r;
  const int lane = threadIdx.x & 31;
  for (int s = lane * 4; s < T; s += 128) *(int4*)(keys + s) = make_int4(-1, -1, -1, -1);
  __syncwarp();
  for (int g0 = ps; g0 < pe; g0 += 32) {
    const int p = g0 + lane;
    int4 st = make_int4(0, 0, INT_MAX, 0);
    if (p < pe) st = h.hcur[p];
    const bool act = st.z < c1;
    unsigned mask = __ballot_sync(kFull, act);
    if (!mask) continue;
    const double av = act ? a.A.val[p] : 0.0;
    bool moved = false;
    while (mask) {
      int td[kHeavyD], jr[kHeavyD];
      double br[kHeavyD];
#pragma unroll
      for (int d = 0; d < kHeavyD; ++d) {
        td[d] = mask ? __ffs(mask) - 1 : -1;
        if (mask) mask &= mask - 1u;
        jr[d] = INT_MAX;
        br[d] = 0.0;
        if (td[d] >= 0) {
          const int cur = __shfl_sync(kFull, st.x, td[d]);
          const int end = __shfl_sync(kFull, st.y, td[d]);
          if (cur + lane < end) {
            jr[d] = a.B.col[cur + lane];
            br[d] = a.B.val[cur + lane];
          }
        }
      }
#pragma unroll
      for (int d = 0; d < kHeavyD; ++d) {
        const int t = td[d];
        if (t < 0) break;
        const int end = __shfl_sync(kFull, st.y, t);
        const double at = __shfl_sync(kFull, av, t);
        int q = __shfl_sync(kFull, st.x, t);
        int j = jr[d];
        double bv = br[d];
        int next;
        for (;;) {
          const bool valid = j < c1;
          const int nv = __popc(__ballot_sync(kFull, valid));
          if (valid) insert_acc<LOG2T, true>(keys, vals, j, __dmul_rn(at, bv), a.status);
          __syncwarp();  // k-order of the accumulation
          q += nv;
          if (nv < 32) {
            next = __shfl_sync(kFull, j, nv);  // first column >= c1, or INT_MAX past the end
            break;
          }
          if (q >= end) {
            next = INT_MAX;
            break;
          }
          j = q + lane < end ? a.B.col[q + lane] : INT_MAX;
          bv = q + lane < end ? a.B.val[q + lane] : 0.0;
        }
        if (lane == t) {
          st.x = q;
          st.z = next;
          moved = true;
        }
      }
    }
    if (moved) h.hcur[p] = st;
  }
  __syncwarp();

  // compact (packed word, value) pairs to the front, the word holding the
  // column offset from c0 above the compacted position
  int m = 0;
  for (int c = 0; c < T; c += 32) {
    const int s = c + lane;
    const int key = keys[s];
    const double v = vals[s];
    const bool occ = key != kEmptyKey;
    const unsigned bal = __ballot_sync(kFull, occ);
    const int pos = m + __popc(bal & lanemask_lt());
    __syncwarp();
    if (occ) {
      keys[pos] = (int)(((uint32_t)(key - c0) << LOG2T) | (uint32_t)pos);
      vals[pos] = v;
    }
    m += __popc(bal);
    __syncwarp();
  }
  // the radix buffers need 3m <= 2T and m + 256 <= T; windows hold at most
  // cap columns, which the host keeps inside both
  if (m > h.cap || m > room) {
    if (lane == 0) report(a.status, DEV_ERR_OVERFLOW);
    m = max(0, (int)min((int64_t)min(m, h.cap), room));
  }
  const uint32_t* sorted = radix_sort_words<1, 8>((uint32_t*)keys, (uint32_t*)(vals + m), m,
                                                  LOG2T, span_bits(c0, c1 - 1), keys + m, nullptr);
  emit_packed<LOG2T, GRAM>(a, row, c0, m, sorted, vals, base, lane, 32);
  __syncwarp();
  return m;
}

template <int LOG2T, bool GRAM>
__global__ void __launch_bounds__(64, 4) k_heavy_w32(HeavyArgs h) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int T = 1 << LOG2T;
  const RowArgs& a = h.r;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double* vals = (double*)(smem + (size_t)w * T * 12);
  int* keys = (int*)(vals + T);
  const int bw = 1 << h.blk_log2, sw = 1 << h.sub_log2;
  const int max_blocks = max(1, (1 << 20) >> h.blk_log2);  // windows span < 2^21 columns

  for (int r = blockIdx.x * nw + w; r < a.nrows; r += gridDim.x * nw) {
    const int row = a.rows[r];
    const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];
    const int lo = h.lo[row], hi = h.hi[row];
    const int lo_r = GRAM ? max(lo, row) : lo;
    const int32_t low = GRAM ? a.low_in[row] : 0;
    const int64_t expect = (int64_t)a.cnt_in[row] - low;
    if (!heavy_row_windowed(h, row)) continue;  // the CTA kernel's row
    const int64_t base = a.rowptr[row] + low;
    int64_t written = 0;
    if (lo_r <= hi) {
      // cursors at the first B entry >= lo_r of every B row of the row
      for (int p = ps + lane; p < pe; p += 32) {
        const int32_t k = a.A.col[p];
        int s = a.B.rowptr[k];
        const int e = a.B.rowptr[k + 1];
        if (GRAM) {
          int l = s, u = e;  // lower bound of lo_r in the sorted B row
          while (l < u) {
            const int mid = (l + u) >> 1;
            if (a.B.col[mid] < lo_r) l = mid + 1; else u = mid;
          }
          s = l;
        }
        h.hcur[p] = make_int4(s, e, s < e ? a.B.col[s] : INT_MAX, 0);
      }
      __syncwarp();
      const int64_t b0 = h.blk_off[row];
      const int nb = (int)(h.blk_off[row + 1] - b0);
      const uint16_t* cnt = h.blk_cnt + b0;
      int b = (lo_r - lo) >> h.blk_log2;
      while (b < nb) {
        const int bstart = lo + (b << h.blk_log2);
        if ((int)cnt[b] > h.cap) {
          // a dense block: fixed windows of sw columns
          const int bend = (int)min((int64_t)bstart + bw, (int64_t)hi + 1);
          for (int c0 = max(bstart, lo_r); c0 < bend;) {
            const int c1 = min(bend, bstart + ((c0 - bstart) / sw + 1) * sw);
            written += heavy_window<LOG2T, GRAM>(h, row, ps, pe, c0, c1, keys, vals,
                                                 base + written, expect - written);
            c0 = c1;
          }
          ++b;
        } else {
          const int e = window_end(cnt, b, nb, h.cap, max_blocks);
          const int c0 = max(bstart, lo_r);
          const int c1 = (int)min((int64_t)lo + ((int64_t)e << h.blk_log2), (int64_t)hi + 1);
          written += heavy_window<LOG2T, GRAM>(h, row, ps, pe, c0, c1, keys, vals, base + written,
                                               expect - written);
          b = e;
        }
      }
    }
    if (written != expect && lane == 0) report(a.status, DEV_ERR_OVERFLOW);
  }
}

}  // namespace

cudaError_t launch_heavy_w32(bool gram, const HeavyArgs& h, int num_sms, cudaStream_t s) {
  if (h.r.nrows <= 0) return cudaSuccess;
  constexpr int LOG2T = kHeavyTableLog2;
  auto kernel = gram ? k_heavy_w32<LOG2T, true> : k_heavy_w32<LOG2T, false>;
  const int warps = 2;
  const size_t smem = (size_t)warps * ((size_t)12 << LOG2T);
  cudaError_t e;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, warps * 32, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  const int64_t need = (h.r.nrows + warps - 1) / warps;
  if (grid > need) grid = need;
  kernel<<<(unsigned)grid, warps * 32, smem, s>>>(h);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace spg
