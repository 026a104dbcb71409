// Heavy rows: one CTA per row over dense column windows.
//
// A row whose table would not fit in shared memory is processed window by
// window over its output column span [lo, hi]: a shared bitmap of W bits marks
// the columns hit in [w0, w0+W).  The symbolic phase counts the bits.  The
// numeric phase turns the bitmap into per-word prefix counts, so a column's
// rank inside the row is prefix[word] + popc(bits below it): the row's column
// indices are written in sorted order straight into their CSR slots, values
// are zeroed there and then accumulated in place, walking row i of A in order
// with a CTA barrier per k (the same k-ordered, product-rounded sum as the
// shared-table rows and the CPU oracle).  No global hash table and no sort
// are needed: the bitmap rank is a counting sort with one bit per key.
//
// In the reference every row above 767 products went to a per-row global hash
// arena of next_pow2(4f/3+1) slots (src/spgemm_engine.cuh:51-57, :79, :101)
// followed by the global radix sort.
#include <algorithm>

#include "kernels.h"

namespace spg {

constexpr size_t kHeavyScratch = 256;

size_t heavy_smem_bytes(bool numeric, int threads, int window_bits) {
  const size_t words = (size_t)window_bits / 32;
  size_t b = words * 4 + (size_t)threads * 12 + kHeavyScratch;  // + staging of B rows
  if (numeric) b += words + (size_t)threads * 8;  // 4-word group prefixes, staged a_ik
  return b;
}

// In a persistent launch rows are drawn from the launch's counter as CTAs free
// up (cta_item).  Rows differ in cost by orders of magnitude (R-MAT hubs), and
// dealing them out in turn left SMs idle (products per CTA, max over mean: 1.20 at R-MAT
// 2^20, 1.50 at 2^18).  Numeric / symbolic heavy time, dealt -> drawn: R-MAT
// 2^20 585 / 69.7 -> 493 / 57.1 ms, 2^18 57.8 / 7.88 -> 46.3 / 5.49 ms, 2^16
// 11.4 / 1.21 -> 6.9 / 0.84 ms.

// B rows at least this long are marked by the whole CTA, shorter ones by one
// warp each.
constexpr int kLongBRow = 256;

// Mark the columns of row `row` that fall in [w0, w0 + 32·nwords) (and, for
// the Gram upper part, are >= row) in the shared bitmap.  Marking is an OR, so
// the B rows need no order: per chunk of blockDim entries of A's row, the
// long B rows (listed in st_long) are swept by the whole CTA one after another
// and the short ones are dealt out to the warps, a B row per warp — no search
// for the B row of a product.
__device__ __forceinline__ void mark_window(const RowArgs& a, int row, long long w0, int nwords,
                                            uint32_t* bm, int* st_bs, int* st_len, int* st_long,
                                            void* scratch) {
  const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];
  const long long wbits = (long long)nwords * 32;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
  int* nlong_p = (int*)scratch;
  for (int32_t pb = ps; pb < pe; pb += blockDim.x) {
    const int cnt = min((int)blockDim.x, pe - pb);
    int bs = 0, len = 0;
    if (tid < cnt) {
      const int32_t k = a.A.col[pb + tid];
      bs = a.B.rowptr[k];
      len = a.B.rowptr[k + 1] - bs;
    }
    st_bs[tid] = bs;
    st_len[tid] = len;
    if (tid == 0) *nlong_p = 0;
    __syncthreads();
    if (len >= kLongBRow) st_long[atomicAdd(nlong_p, 1)] = tid;
    __syncthreads();
    const int nlong = *nlong_p;
    for (int i = 0; i < nlong; ++i) {
      const int t = st_long[i];
      const int32_t b = st_bs[t], l = st_len[t];
      for (int q = tid; q < l; q += blockDim.x) {
        const long long d = (long long)a.B.col[b + q] - w0;
        if (d >= 0 && d < wbits) atomicOr(&bm[d >> 5], 1u << (d & 31));
      }
    }
    for (int t = wid; t < cnt; t += nwarps) {
      const int32_t b = st_bs[t], l = st_len[t];
      if (l >= kLongBRow) continue;
      for (int q = lane; q < l; q += 32) {
        const long long d = (long long)a.B.col[b + q] - w0;
        if (d >= 0 && d < wbits) atomicOr(&bm[d >> 5], 1u << (d & 31));
      }
    }
    __syncthreads();  // staging and the long-row count are reused by the next chunk
  }
}

// At most 32 registers (no spills): 512-thread CTAs over windows of up to 2^18
// columns then run four per SM instead of two (R-MAT 2^18: 9.59 -> 7.90 ms;
// 2^19, three per SM: 24.2 -> 20.0 ms).
template <bool GRAM>
__global__ void __launch_bounds__(1024, 2) k_heavy_sym(HeavyArgs h) {
  extern __shared__ __align__(16) unsigned char smem[];
  const RowArgs& a = h.r;
  const int nw_max = h.window_bits / 32;
  uint32_t* bm = (uint32_t*)smem;
  int* st_bs = (int*)(bm + nw_max);
  int* st_ex = st_bs + blockDim.x;
  int* st_long = st_ex + blockDim.x;
  void* scratch = (void*)(st_long + blockDim.x);
  __shared__ int s_next;
  for (int it = 0;; ++it) {
    const int r = cta_item(h.queue, a.nrows, it, &s_next);
    if (r >= a.nrows) break;
    const int row = a.rows[r];
    const int lo = h.lo[row], hi = h.hi[row];
    long long c = 0, cl = 0;
    for (long long w0 = lo; w0 <= hi; w0 += h.window_bits) {
      const int nwords = (int)min((long long)nw_max, (hi - w0) / 32 + 1);
      for (int i = threadIdx.x; i < nwords; i += blockDim.x) bm[i] = 0u;
      __syncthreads();
      mark_window(a, row, w0, nwords, bm, st_bs, st_ex, st_long, scratch);
      // a warp per column block of the window (32 or more words): the bit
      // counts are the row totals and, when asked for, the block counts
      int lc = 0, lcl = 0;
      const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
      const int wpb = 1 << (h.blk_log2 - 5);
      const long long blk0 = (w0 - lo) >> h.blk_log2;
      for (int blk = wid; blk * wpb < nwords; blk += nwarps) {
        int bc = 0;
        for (int i = blk * wpb + lane; i < min((blk + 1) * wpb, nwords); i += 32) {
          const uint32_t wd = bm[i];
          bc += __popc(wd);
          if (GRAM) {
            const long long c0 = w0 + 32LL * i;
            if (c0 + 32 <= row) lcl += __popc(wd);
            else if (c0 < row) lcl += __popc(wd & ((1u << (unsigned)(row - c0)) - 1u));
          }
        }
        lc += bc;
        if (h.blk_cnt) {
          for (int o = 16; o > 0; o >>= 1) bc += __shfl_xor_sync(0xffffffffu, bc, o);
          if (lane == 0) h.blk_cnt[h.blk_off[row] + blk0 + blk] = (uint16_t)min(bc, 65535);
        }
      }
      c += block_sum64(lc, (long long*)scratch);
      if (GRAM) cl += block_sum64(lcl, (long long*)scratch);
    }
    if (threadIdx.x == 0) {
      a.rownnz[row] = (int)c;
      if (GRAM) a.rowlow[row] = (int)cl;
    }
    __syncthreads();
  }
}

// Rank of bit d inside the window: prefix of its 4-word group plus the bits
// set below it in that group.
__device__ __forceinline__ int window_rank(const uint32_t* bm, const int* pre4, long long d) {
  const int i = (int)(d >> 5), b = (int)(d & 31);
  int r = pre4[i >> 2];
  for (int w = i & ~3; w < i; ++w) r += __popc(bm[w]);
  return r + __popc(bm[i] & ((1u << b) - 1u));
}

// Launched with up to 512 threads the kernel is built for three CTAs per SM
// (40 registers, no spills), so windows of up to 2^18 columns (about 51 KB of
// shared memory) are not held to two CTAs per SM by registers.  R-MAT 2^17,
// A·A / A·Aᵀ: 27.1 / 29.1 -> 24.0 / 24.3 ms; 2^18: 64.9 / 65.7 -> 60.6 / 63.0
// ms.  Four CTAs per SM (32 registers, small spills) were slower: 29.1 and
// 90.4 ms for A·A.
constexpr int kNumMinBlocks512 = 3;

template <bool GRAM, int MAXT, int MINB>
__global__ void __launch_bounds__(MAXT, MINB) k_heavy_num(HeavyArgs h) {
  extern __shared__ __align__(16) unsigned char smem[];
  const RowArgs& a = h.r;
  const int nw_max = h.window_bits / 32;
  const int HT = blockDim.x;
  uint32_t* bm = (uint32_t*)smem;
  int* pre4 = (int*)(bm + nw_max);
  double* st_a = (double*)(pre4 + nw_max / 4);
  int* st_bs = (int*)(st_a + HT);
  int* st_ex = st_bs + HT;
  int* st_long = st_ex + HT;
  void* scratch = (void*)(st_long + HT);
  const int tid = threadIdx.x;
  __shared__ int s_next;
  for (int it = 0;; ++it) {
    const int r = cta_item(h.queue, a.nrows, it, &s_next);
    if (r >= a.nrows) break;
    const int row = a.rows[r];
    const int hi = h.hi[row];
    const int lo = GRAM ? max(h.lo[row], row) : h.lo[row];
    const int32_t low = GRAM ? a.low_in[row] : 0;
    const long long expect = (long long)a.cnt_in[row] - low;
    if (heavy_row_windowed(h, row)) continue;  // the windowed warp kernel's row
    const int64_t base = a.rowptr[row] + low;
    const int cb = a.colbase ? a.colbase[row] : 0;
    long long written = 0;
    for (long long w0 = lo; w0 <= hi; w0 += h.window_bits) {
      const int nwords = (int)min((long long)nw_max, (hi - w0) / 32 + 1);
      const int ngroups = (nwords + 3) >> 2;
      for (int i = tid; i < ngroups * 4; i += HT) bm[i] = 0u;
      __syncthreads();
      mark_window(a, row, w0, nwords, bm, st_bs, st_ex, st_long, scratch);
      // exclusive prefix of the bit counts per group of 4 words
      const int per = (ngroups + HT - 1) / HT;
      const int gb = min(ngroups, tid * per), ge = min(ngroups, gb + per);
      int local = 0;
      for (int g = gb; g < ge; ++g)
        local += __popc(bm[4 * g]) + __popc(bm[4 * g + 1]) + __popc(bm[4 * g + 2]) +
                 __popc(bm[4 * g + 3]);
      int tot;
      int run = block_exclusive_scan(local, (int*)scratch, &tot);
      // zeroed values into the row's CSR slots, consecutive stores (zeroing
      // each value beside its column index, scattered: R-MAT 2^18 60.8 ms,
      // 2^20 603 ms; this way 57.5 and 588 ms)
      const long long nkeep = min((long long)tot, expect - written);
      for (long long i = tid; i < nkeep; i += HT) a.cval[base + written + i] = 0.0;
      // group prefixes and the sorted column indices, each thread the bits of
      // its own groups.  (A warp-wide writer with consecutive stores — entry
      // l + 32i of 32 words found by a search of their bit counts and a select
      // in the word — was no faster at R-MAT 2^18, 57.1 against 57.5 ms, and
      // slower at 2^20, 593-599 against 588 ms.)
      for (int g = gb; g < ge; ++g) {
        pre4[g] = run;
        for (int w = 4 * g; w < 4 * g + 4; ++w) {
          uint32_t wd = bm[w];
          while (wd) {
            const int b = __ffs(wd) - 1;
            wd &= wd - 1u;
            const long long pos = written + run;
            if (pos < expect) a.ccol[base + pos] = (int32_t)(w0 + 32LL * w + b) - cb;
            ++run;
          }
        }
      }
      __syncthreads();
      // k-ordered accumulation in place; the first HT entries of B row t+1 are
      // loaded while row t is accumulated
      const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];
      const long long wbits = (long long)nwords * 32;
      for (int32_t pb = ps; pb < pe; pb += HT) {
        const int cnt = min(HT, pe - pb);
        if (tid < cnt) {
          const int32_t k = a.A.col[pb + tid];
          const int32_t bs = a.B.rowptr[k];
          st_bs[tid] = bs;
          st_ex[tid] = a.B.rowptr[k + 1] - bs;
          st_a[tid] = a.A.val[pb + tid];
        }
        __syncthreads();
        int jn = -1;
        double bn = 0.0;
        if (tid < st_ex[0]) {
          jn = a.B.col[st_bs[0] + tid];
          bn = a.B.val[st_bs[0] + tid];
        }
        for (int t = 0; t < cnt; ++t) {
          const int j = jn;
          const double bv = bn;
          const int32_t bs = st_bs[t], len = st_ex[t];
          const double av = st_a[t];
          if (t + 1 < cnt) {
            jn = -1;
            if (tid < st_ex[t + 1]) {
              jn = a.B.col[st_bs[t + 1] + tid];
              bn = a.B.val[st_bs[t + 1] + tid];
            }
          }
          if (tid < len) {
            const long long d = (long long)j - w0;
            if (d >= 0 && d < wbits) {
              const long long pos = written + window_rank(bm, pre4, d);
              if (pos < expect)
                a.cval[base + pos] = __dadd_rn(a.cval[base + pos], __dmul_rn(av, bv));
            }
          }
          // the rest of a long B row, four entries per thread at a time: their
          // loads, then their read-modify-writes of C, are issued together
          // (the entries of one B row are distinct columns)
          for (int q0 = tid + HT; q0 < len; q0 += 4 * HT) {
            long long pos[4];
            double bv4[4], cur[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
              const int q = q0 + u * HT;
              pos[u] = -1;
              bv4[u] = 0.0;
              if (q < len) {
                const long long d = (long long)a.B.col[bs + q] - w0;
                bv4[u] = a.B.val[bs + q];
                if (d >= 0 && d < wbits) pos[u] = written + window_rank(bm, pre4, d);
              }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
              cur[u] = (pos[u] >= 0 && pos[u] < expect) ? a.cval[base + pos[u]] : 0.0;
#pragma unroll
            for (int u = 0; u < 4; ++u)
              if (pos[u] >= 0 && pos[u] < expect)
                a.cval[base + pos[u]] = __dadd_rn(cur[u], __dmul_rn(av, bv4[u]));
          }
          __syncthreads();
        }
      }
      written += tot;
    }
    if (written != expect && tid == 0) report(a.status, DEV_ERR_OVERFLOW);
    if (GRAM) {
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
static cudaError_t launch_h(K kernel, int threads, size_t smem, const HeavyArgs& h, int num_sms,
                            cudaStream_t s) {
  cudaError_t e;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
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

__global__ void k_heavy_blocks(BinSource bsym, int blk_log2, int32_t* __restrict__ nblk) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < bsym.n;
       i += (int64_t)gridDim.x * blockDim.x)
    nblk[i] = row_bin(bsym, (int)i) == kHeavyBin
                  ? (int32_t)((((int64_t)bsym.hi[i] - bsym.lo[i]) >> blk_log2) + 1)
                  : 0;
}

cudaError_t launch_heavy_blocks(const BinSource& bsym, int blk_log2, int32_t* nblk,
                                int64_t* blk_off, void* scan_tmp, cudaStream_t s) {
  if (bsym.n > 0) {
    const int64_t blocks = std::min<int64_t>(((int64_t)bsym.n + 255) / 256, 4096);
    k_heavy_blocks<<<(unsigned)blocks, 256, 0, s>>>(bsym, blk_log2, nblk);
    SPG_COUNT_LAUNCH();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return launch_scan_i32_i64(nblk, blk_off, bsym.n, scan_tmp, s);
}

cudaError_t launch_heavy(bool numeric, bool gram, const HeavyArgs& h, int threads, int num_sms,
                         cudaStream_t s) {
  if (h.r.nrows <= 0) return cudaSuccess;
  const size_t smem = heavy_smem_bytes(numeric, threads, h.window_bits);
  if (!h.queue) return cudaErrorInvalidValue;  // the kernels draw their rows from it
  cudaError_t e = cudaMemsetAsync(h.queue, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  if (numeric && threads <= 512)
    return gram ? launch_h(k_heavy_num<true, 512, kNumMinBlocks512>, threads, smem, h, num_sms, s)
                : launch_h(k_heavy_num<false, 512, kNumMinBlocks512>, threads, smem, h, num_sms, s);
  if (numeric)
    return gram ? launch_h(k_heavy_num<true, 1024, 1>, threads, smem, h, num_sms, s)
                : launch_h(k_heavy_num<false, 1024, 1>, threads, smem, h, num_sms, s);
  return gram ? launch_h(k_heavy_sym<true>, threads, smem, h, num_sms, s)
              : launch_h(k_heavy_sym<false>, threads, smem, h, num_sms, s);
}

}  // namespace spg
