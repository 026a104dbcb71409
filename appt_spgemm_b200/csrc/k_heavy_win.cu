// Heavy rows, numeric phase: one CTA per row, values accumulated in shared
// memory window by window and written to C once.
//
// The row's output columns [lo, hi] are walked in windows [c0, c1) chosen from
// the symbolic phase's per-block distinct counts: consecutive blocks while
// their counts sum to at most `vcap` and they span at most `wcap_bits`
// columns; a block above either limit is cut into fixed sub-windows of
// min(vcap, wcap_bits) columns (a power of two), which can never hold more
// than vcap columns.  Every entry p of A's row keeps a cursor into its sorted
// B row (global int4 {cursor, row end, next column, 0}), so each window reads
// only the B entries inside it and each B entry is read once per pass over
// all windows.  Per window:
//  1. mark: the window's columns are set in a shared bitmap (an OR, so in any
//     order: B rows of 256 entries or more are swept by the whole CTA, shorter
//     ones by a warp each);
//  2. ranks: prefix counts per group of 4 bitmap words give each column its
//     position in the window; the columns are written to their CSR slots;
//  3. accumulate: the entries of A's row whose next column lies inside the
//     window are taken in increasing position; for each, the CTA adds
//     round(a_ik·b_kj) to the shared value of every column j of its window
//     part, and one CTA barrier (which also tells whether the B row runs on)
//     separates consecutive entries, so every value is 0.0 + Σ_k in the order
//     of k, each product rounded first — the oracle's sum, bit for bit;
//  4. the window's values are written to C with consecutive stores.
// The dense-window CTA kernel (k_heavy.cu) instead read-modify-writes every
// product in C in global memory behind each barrier, which leaves the SMs
// waiting on L2 round trips and evicts partly accumulated rows to HBM.
#include <climits>

#include "kernels.h"

namespace spg {

namespace {

constexpr int kLongRun = 256;  // B rows at least this long are marked by the whole CTA

// Rank of window bit d: prefix of its 4-word group plus the bits below it.
__device__ __forceinline__ int win_rank(const uint32_t* bm, const int* pre4, int d) {
  const int i = d >> 5, b = d & 31;
  int r = pre4[i >> 2];
  for (int w = i & ~3; w < i; ++w) r += __popc(bm[w]);
  return r + __popc(bm[i] & ((1u << b) - 1u));
}

}  // namespace

// Dynamic shared memory, in the order the kernel lays it out: values (vcap
// doubles), bitmap (wcap/32 words), group prefixes (wcap/128 ints), then per
// thread a staged a_ik (double) and four ints (cursor, end, flag, list), then
// 64 ints of scratch.
size_t heavy_win_smem_bytes(int threads, int vcap, int wcap_bits) {
  return (size_t)vcap * sizeof(double) + (size_t)wcap_bits / 32 * sizeof(uint32_t) +
         (size_t)wcap_bits / 128 * sizeof(int) + (size_t)threads * sizeof(double) +
         (size_t)threads * 4 * sizeof(int) + 64 * sizeof(int);
}

template <bool GRAM, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_heavy_num_win(HeavyArgs h) {
  extern __shared__ __align__(16) unsigned char smem[];
  const RowArgs& a = h.r;
  const int HT = blockDim.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nwarps = HT >> 5;
  const int vcap = h.vcap, wcap = h.wcap_bits;
  double* vals = (double*)smem;
  uint32_t* bm = (uint32_t*)(vals + vcap);
  int* pre4 = (int*)(bm + wcap / 32);
  double* st_a = (double*)(pre4 + wcap / 128);
  int* st_cur = (int*)(st_a + HT);
  int* st_end = st_cur + HT;
  int* st_nxt = st_end + HT;
  int* st_list = st_nxt + HT;
  int* scratch = st_list + HT;  // 64 ints: scans (33), window bounds, counters
  __shared__ int s_next;
  // fixed sub-window width for blocks above the limits: a power of two <= both
  int sub = 1024;
  while (sub * 2 <= vcap && sub * 2 <= wcap) sub *= 2;
  const int bw_log2 = h.blk_log2;
  const long long bwidth = 1LL << bw_log2;

  for (int it = 0;; ++it) {
    const int r = cta_item(h.queue, a.nrows, it, &s_next);
    if (r >= a.nrows) break;
    const int row = a.rows[r];
    if (heavy_row_windowed(h, row)) continue;  // the windowed warp kernel's row
    const int lo = h.lo[row], hi = h.hi[row];
    const int lo_r = GRAM ? max(lo, row) : lo;
    const int32_t low = GRAM ? a.low_in[row] : 0;
    const long long expect = (long long)a.cnt_in[row] - low;
    const int64_t base = a.rowptr[row] + low;
    const int cb = a.colbase ? a.colbase[row] : 0;
    const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];
    long long written = 0;
    if (lo_r <= hi) {
      // cursors at the first B entry >= lo_r of every B row of the row
      for (int32_t p = ps + tid; p < pe; p += HT) {
        const int32_t k = a.A.col[p];
        int s = a.B.rowptr[k];
        const int e = a.B.rowptr[k + 1];
        if (GRAM) {
          int l = s, u = e;
          while (l < u) {
            const int mid = (l + u) >> 1;
            if (a.B.col[mid] < lo_r) l = mid + 1; else u = mid;
          }
          s = l;
        }
        h.hcur[p] = make_int4(s, e, s < e ? a.B.col[s] : INT_MAX, 0);
      }
      const int64_t b0 = h.blk_off[row];
      const int nb = (int)(h.blk_off[row + 1] - b0);
      const uint16_t* cnt = h.blk_cnt + b0;
      // window walk state (thread 0): next block, next column inside a cut block
      int wb = (int)(((long long)lo_r - lo) >> bw_log2);
      long long wsub = -1;
      for (;;) {
        __syncthreads();  // cursors written; the previous window is finished
        if (tid == 0) {
          int c0 = 0, c1 = 0;
          bool done = wb >= nb;
          if (!done) {
            const long long bstart = (long long)lo + ((long long)wb << bw_log2);
            const long long bend = min(bstart + bwidth, (long long)hi + 1);
            if ((int)cnt[wb] > vcap || bwidth > wcap) {
              const long long s0 = wsub >= 0 ? wsub : max(bstart, (long long)lo_r);
              const long long s1 = min(bend, bstart + ((s0 - bstart) / sub + 1) * sub);
              c0 = (int)s0;
              c1 = (int)s1;
              if (s1 >= bend) {
                ++wb;
                wsub = -1;
              } else {
                wsub = s1;
              }
            } else {
              int e = wb, tot = 0;
              while (e < nb && tot + (int)cnt[e] <= vcap && (long long)(e + 1 - wb) * bwidth <= wcap) {
                tot += cnt[e];
                ++e;
              }
              c0 = (int)max(bstart, (long long)lo_r);
              c1 = (int)min((long long)lo + ((long long)e << bw_log2), (long long)hi + 1);
              wb = e;
            }
          }
          scratch[40] = done ? 1 : 0;
          scratch[41] = c0;
          scratch[42] = c1;
        }
        __syncthreads();
        if (scratch[40]) break;
        const int c0 = scratch[41], c1 = scratch[42];
        const int nwords = (c1 - c0 + 31) >> 5;
        const int ngroups = (nwords + 3) >> 2;
        for (int i = tid; i < ngroups * 4; i += HT) bm[i] = 0u;
        __syncthreads();

        // 1. mark the window's columns
        for (int32_t pb = ps; pb < pe; pb += HT) {
          const int n_here = min(HT, pe - pb);
          int cur = 0, end = 0, nxt = INT_MAX;
          if (tid < n_here) {
            const int4 st = h.hcur[pb + tid];
            cur = st.x;
            end = st.y;
            nxt = st.z;
          }
          const bool act = nxt < c1;
          const bool lng = act && end - cur >= kLongRun;
          st_cur[tid] = cur;
          st_end[tid] = end;
          st_nxt[tid] = (act && !lng) ? 1 : 0;
          if (tid == 0) scratch[43] = 0;
          __syncthreads();
          if (lng) st_list[atomicAdd(&scratch[43], 1)] = tid;
          __syncthreads();
          const int nlong = scratch[43];
          for (int i = 0; i < nlong; ++i) {
            const int t = st_list[i];
            const int e = st_end[t];
            for (int q0 = st_cur[t];; q0 += HT) {
              const int q = q0 + tid;
              const int j = q < e ? a.B.col[q] : INT_MAX;
              if (j < c1) {
                const int d = j - c0;
                atomicOr(&bm[d >> 5], 1u << (d & 31));
              }
              if (__syncthreads_or(j >= c1)) break;
            }
          }
          // short runs: a warp each, 32 entries at a time until the window ends
          for (int t = wid; t < n_here; t += nwarps) {
            if (!st_nxt[t]) continue;
            const int e = st_end[t];
            for (int q0 = st_cur[t];; q0 += 32) {
              const int q = q0 + lane;
              const int j = q < e ? a.B.col[q] : INT_MAX;
              if (j < c1) {
                const int d = j - c0;
                atomicOr(&bm[d >> 5], 1u << (d & 31));
              }
              if (__any_sync(0xffffffffu, j >= c1)) break;
            }
          }
          __syncthreads();  // staging reused by the next chunk
        }

        // 2. ranks: prefix of the bit counts per group of 4 words; columns out
        const int per = (ngroups + HT - 1) / HT;
        const int gb = min(ngroups, tid * per), ge = min(ngroups, gb + per);
        int local = 0;
        for (int g = gb; g < ge; ++g)
          local += __popc(bm[4 * g]) + __popc(bm[4 * g + 1]) + __popc(bm[4 * g + 2]) +
                   __popc(bm[4 * g + 3]);
        int tot;
        int run = block_exclusive_scan(local, scratch, &tot);
        const bool fits = tot <= vcap && written + tot <= expect;
        for (int g = gb; g < ge; ++g) {
          pre4[g] = run;
          for (int w = 4 * g; w < 4 * g + 4; ++w) {
            uint32_t wd = bm[w];
            while (wd) {
              const int b = __ffs(wd) - 1;
              wd &= wd - 1u;
              if (fits) a.ccol[base + written + run] = c0 + 32 * w + b - cb;
              ++run;
            }
          }
        }
        if (!fits) {  // the symbolic counts were exceeded: report, keep C untouched
          if (tid == 0) report(a.status, DEV_ERR_OVERFLOW);
          written = expect;
          break;
        }
        for (int i = tid; i < tot; i += HT) vals[i] = 0.0;
        __syncthreads();

        // 3. accumulate in the order of A's row
        for (int32_t pb = ps; pb < pe; pb += HT) {
          const int n_here = min(HT, pe - pb);
          int cur = 0, end = 0, nxt = INT_MAX;
          double av = 0.0;
          if (tid < n_here) {
            const int4 st = h.hcur[pb + tid];
            cur = st.x;
            end = st.y;
            nxt = st.z;
            av = a.A.val[pb + tid];
          }
          const bool act = nxt < c1;
          st_cur[tid] = cur;
          st_end[tid] = end;
          st_a[tid] = av;
          int nact;
          const int pos = block_exclusive_scan(act ? 1 : 0, scratch, &nact);
          if (act) st_list[pos] = tid;
          __syncthreads();
          for (int i = 0; i < nact; ++i) {
            const int t = st_list[i];
            const int s = st_cur[t], e = st_end[t];
            const double at = st_a[t];
            int moved = 0;
            for (int q0 = s;; q0 += HT) {
              const int q = q0 + tid;
              const int j = q < e ? a.B.col[q] : INT_MAX;
              const bool in = j < c1;
              if (in) {
                const int rk = win_rank(bm, pre4, j - c0);
                vals[rk] = __dadd_rn(vals[rk], __dmul_rn(at, a.B.val[q]));
              }
              // the barrier orders this entry's additions before the next
              // entry's, and counts how far the B row ran inside the window
              const int c = __syncthreads_count(in);
              moved += c;
              if (c < HT) break;
            }
            if (tid == 0) {
              const int nc = s + moved;
              h.hcur[pb + t] = make_int4(nc, e, nc < e ? a.B.col[nc] : INT_MAX, 0);
            }
          }
          __syncthreads();  // staging reused by the next chunk
        }

        // 4. the window's values, written once
        for (int i = tid; i < tot; i += HT) a.cval[base + written + i] = vals[i];
        written += tot;
      }
    }
    if (written != expect && tid == 0) report(a.status, DEV_ERR_OVERFLOW);
    if (GRAM) {
      __syncthreads();  // the row's C entries are written
      const long long m = written < expect ? written : expect;
      for (long long t = tid; t < m; t += HT) {
        const int j = a.ccol[base + t] + cb;
        if (j > row) {
          const int pos = atomicAdd(&a.cursor[j], 1);
          if (pos < a.low_in[j]) {
            const int64_t d = a.lowptr[j] + pos;
            a.lcol[d] = row - cb;
            a.lval[d] = a.cval[base + t];
          } else {
            report(a.status, DEV_ERR_OVERFLOW);
          }
        }
      }
    }
    __syncthreads();
  }
}

template <typename K>
static cudaError_t launch_win(K kernel, int threads, size_t smem, const HeavyArgs& h,
                              int num_sms, cudaStream_t s) {
  cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)smem);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > h.r.nrows) grid = h.r.nrows;
  kernel<<<(unsigned)grid, threads, smem, s>>>(h);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_heavy_win(bool gram, const HeavyArgs& h, int threads, int num_sms,
                             cudaStream_t s) {
  if (h.r.nrows <= 0) return cudaSuccess;
  if (!h.queue || !h.hcur || !h.blk_cnt || h.vcap < 1024 || h.wcap_bits < 1024 ||
      (h.wcap_bits & 127) || threads < 64 || threads > 1024 || (threads & 31))
    return cudaErrorInvalidValue;
  const size_t smem = heavy_win_smem_bytes(threads, h.vcap, h.wcap_bits);
  cudaError_t e = cudaMemsetAsync(h.queue, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  if (threads <= 512)
    return gram ? launch_win(k_heavy_num_win<true, 512, 2>, threads, smem, h, num_sms, s)
                : launch_win(k_heavy_num_win<false, 512, 2>, threads, smem, h, num_sms, s);
  return gram ? launch_win(k_heavy_num_win<true, 1024, 1>, threads, smem, h, num_sms, s)
              : launch_win(k_heavy_num_win<false, 1024, 1>, threads, smem, h, num_sms, s);
}

}  // namespace spg
