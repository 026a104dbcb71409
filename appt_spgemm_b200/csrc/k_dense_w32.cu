// Warp-per-row kernels over a bitmap of the row's output column span: the
// path of rows whose span is narrow next to their product count (banded,
// stencil and FEM-like matrices).
//
// A hash row claims a table slot with a shared atomic for every product and
// keeps its values in slot order until a final sort.  Here the warp marks the
// row's columns in a bitmap of the span [lo, hi] (one bit per column): the
// lanes of a 32-wide segment of a sorted B row that fall in the same bitmap
// word are merged with shuffles first, so a segment costs one atomicOr per
// distinct word (a 27-point stencil B row: 9 to 12 instead of 27).  The
// symbolic phase counts the bits.  The numeric phase turns the bitmap into a
// prefix count per word, so column j has rank prefix[w] + popc(bits below it),
// writes the row's columns in order straight from the bitmap, and accumulates
// every product into a dense value array at its rank — walking row i of A in
// order with a __syncwarp per segment, so each value is 0.0 + Σ_k round(a_ik ·
// b_kj) in increasing position of k, bit-identical to the hash rows and the
// oracle.  Ranks of one segment are increasing, so its value accesses are
// almost free of bank conflicts.  No sort.
//
// Shared memory per warp: the bitmap (2^LOG2W words), a 16-bit prefix per word
// and kDenseVals values (numeric).  Rows take this path when their span fits
// 2^LOG2W words, spans at most 8 columns per product, and (numeric) the row
// has at most kDenseVals entries (row_bin).  Opt-in (spg_config.dense_max_words):
// on the 27-point stencil, whose span is ~300 columns per output entry, the
// bitmap's bookkeeping made it slower than the hash tables.
#include <climits>

#include "kernels.h"

namespace spg {

namespace {

constexpr unsigned kFull = 0xffffffffu;

template <int LOG2W, bool NUMERIC>
__host__ __device__ constexpr size_t dense_warp_bytes() {
  return NUMERIC ? ((size_t)kDenseVals * 8 + ((size_t)4 << LOG2W) + ((size_t)2 << LOG2W))
                 : ((size_t)4 << LOG2W);
}

// Marks the columns j (lanes with j >= lo; others pass j < 0) of one segment:
// lanes of one bitmap word are consecutive (B rows are sorted), so each run of
// lanes ORs its bits into its first lane, which sets them.
__device__ __forceinline__ void mark_segment(uint32_t* bm, int j, int lo) {
  const int lane = threadIdx.x & 31;
  const bool on = j >= 0;
  const int d = on ? j - lo : 0;
  const int w = on ? (d >> 5) : -1 - lane;  // lanes without a column never merge
  uint32_t bits = on ? (1u << (d & 31)) : 0u;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t x = __shfl_down_sync(kFull, bits, o);
    const int wx = __shfl_down_sync(kFull, w, o);
    if (lane + o < 32 && wx == w) bits |= x;
  }
  const int wp = __shfl_up_sync(kFull, w, 1);
  if (on && (lane == 0 || wp != w)) atomicOr(&bm[w], bits);
}

}  // namespace

template <int LOG2W, bool NUMERIC>
__global__ void __launch_bounds__(256) k_dense_w32(RowArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int W = 1 << LOG2W;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  unsigned char* base_p = smem + (size_t)wid * dense_warp_bytes<LOG2W, NUMERIC>();
  double* vals = (double*)base_p;
  uint32_t* bm = (uint32_t*)(base_p + (NUMERIC ? (size_t)kDenseVals * 8 : 0));
  uint16_t* pre = (uint16_t*)(bm + W);

  for (int r = blockIdx.x * nw + wid; r < a.nrows; r += gridDim.x * nw) {
    const int row = a.rows[r];
    const int lo = a.lo[row], hi = a.hi[row];
    const int nwords = (int)(((int64_t)hi - lo + 32) >> 5);  // row_bin keeps it <= W
    for (int i = lane * 4; i < nwords; i += 128) *(uint4*)(bm + i) = make_uint4(0, 0, 0, 0);
    __syncwarp();
    const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];

    // mark: segments in any order (an OR); when every B row of a chunk fits
    // one segment, the columns of kMarkAhead segments are loaded before any
    // of them is marked (their loads overlap)
    constexpr int kMarkAhead = 8;
    for (int32_t pb = ps; pb < pe; pb += 32) {
      const int cnt = min(32, pe - pb);
      int bs = 0, len = 0;
      if (lane < cnt) {
        const int32_t k = a.A.col[pb + lane];
        bs = a.B.rowptr[k];
        len = a.B.rowptr[k + 1] - bs;
      }
      if (__all_sync(kFull, len <= 32)) {
        for (int t0 = 0; t0 < cnt; t0 += kMarkAhead) {
          int jr[kMarkAhead];
#pragma unroll
          for (int d = 0; d < kMarkAhead; ++d) {
            const int t = t0 + d;
            const int tb = __shfl_sync(kFull, bs, t & 31), tl = __shfl_sync(kFull, len, t & 31);
            jr[d] = (t < cnt && lane < tl) ? a.B.col[tb + lane] : -1;
          }
#pragma unroll
          for (int d = 0; d < kMarkAhead; ++d) mark_segment(bm, jr[d], lo);
        }
        continue;
      }
      for (int t = 0; t < cnt; ++t) {
        const int tb = __shfl_sync(kFull, bs, t), tl = __shfl_sync(kFull, len, t);
        for (int q = 0; q < tl; q += 32)
          mark_segment(bm, q + lane < tl ? a.B.col[tb + q + lane] : -1, lo);
      }
    }
    __syncwarp();

    if (!NUMERIC) {
      int c = 0;
      for (int i = lane * 4; i < nwords; i += 128) {
        const uint4 v = *(const uint4*)(bm + i);
        c += __popc(v.x) + __popc(v.y) + __popc(v.z) + __popc(v.w);
      }
      for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
      if (lane == 0) a.rownnz[row] = c;
      __syncwarp();
      continue;
    }

    // ranks: lane l owns words [l·per, (l+1)·per); exclusive prefix per word
    const int per = (nwords + 31) >> 5;
    const int w0 = min(nwords, lane * per), w1 = min(nwords, w0 + per);
    int mine = 0;
    for (int i = w0; i < w1; ++i) mine += __popc(bm[i]);
    int incl = mine;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(kFull, incl, o);
      if (lane >= o) incl += t;
    }
    const int m = __shfl_sync(kFull, incl, 31);
    const int expect = a.cnt_in[row];
    const int64_t base = a.rowptr[row];
    if (m != expect || m > kDenseVals) {  // never for valid counts: report, write nothing
      if (lane == 0) report(a.status, DEV_ERR_OVERFLOW);
      __syncwarp();
      continue;
    }
    const int cb = a.colbase ? a.colbase[row] : 0;
    int run = incl - mine;
    for (int i = w0; i < w1; ++i) {
      pre[i] = (uint16_t)run;
      uint32_t wd = bm[i];
      while (wd) {
        const int b = __ffs(wd) - 1;
        wd &= wd - 1u;
        a.ccol[base + run] = lo + 32 * i + b - cb;
        ++run;
      }
    }
    for (int i = lane; i < m; i += 32) vals[i] = 0.0;
    __syncwarp();

    // accumulate in the order of A's row: D segments loaded, then added in turn
    constexpr int D = 4;
    for (int32_t pb = ps; pb < pe; pb += 32) {
      const int cnt = min(32, pe - pb);
      int bs = 0, len = 0;
      double av = 0.0;
      if (lane < cnt) {
        const int32_t k = a.A.col[pb + lane];
        bs = a.B.rowptr[k];
        len = a.B.rowptr[k + 1] - bs;
        av = a.A.val[pb + lane];
      }
      int t = 0, q0 = 0;
      while (t < cnt) {
        int rk[D];
        double pr[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          rk[d] = -1;
          pr[d] = 0.0;
          if (t < cnt) {
            const int tb = __shfl_sync(kFull, bs, t), tl = __shfl_sync(kFull, len, t);
            const double at = __shfl_sync(kFull, av, t);
            if (q0 + lane < tl) {
              const int j = a.B.col[tb + q0 + lane];
              const int dd = j - lo;
              const int w = dd >> 5;
              rk[d] = (int)pre[w] + __popc(bm[w] & ((1u << (dd & 31)) - 1u));
              pr[d] = __dmul_rn(at, a.B.val[tb + q0 + lane]);
            }
            q0 += 32;
            if (q0 >= tl) {
              ++t;
              q0 = 0;
            }
          }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) {
          if (rk[d] >= 0) vals[rk[d]] = __dadd_rn(vals[rk[d]], pr[d]);
          __syncwarp();  // k order: this segment's sums before the next one's
        }
      }
    }
    for (int i = lane; i < m; i += 32) a.cval[base + i] = vals[i];
    __syncwarp();
  }
}

template <int LOG2W, bool NUMERIC>
static cudaError_t launch_dense(const RowArgs& a, int num_sms, cudaStream_t s) {
  auto kernel = k_dense_w32<LOG2W, NUMERIC>;
  const size_t per = dense_warp_bytes<LOG2W, NUMERIC>();
  int rows = 8;  // warps per CTA
  while (rows > 1 && per * rows > 96 * 1024) rows >>= 1;
  const size_t smem = per * rows;
  cudaError_t e;
  if (smem > 48 * 1024) {
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
  }
  e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                           cudaSharedmemCarveoutMaxShared);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, rows * 32, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  const int64_t need = (a.nrows + rows - 1) / rows;
  if (grid > need) grid = need;
  kernel<<<(unsigned)grid, rows * 32, smem, s>>>(a);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_dense_bin(int bin, bool numeric, const RowArgs& a, int num_sms,
                             cudaStream_t s) {
  if (a.nrows <= 0) return cudaSuccess;
  switch (bin - kDenseBin0 + kDenseMinLog2W) {
    case 8: return numeric ? launch_dense<8, true>(a, num_sms, s) : launch_dense<8, false>(a, num_sms, s);
    case 9: return numeric ? launch_dense<9, true>(a, num_sms, s) : launch_dense<9, false>(a, num_sms, s);
    case 10: return numeric ? launch_dense<10, true>(a, num_sms, s) : launch_dense<10, false>(a, num_sms, s);
    case 11: return numeric ? launch_dense<11, true>(a, num_sms, s) : launch_dense<11, false>(a, num_sms, s);
  }
  return cudaErrorNotSupported;
}

}  // namespace spg
