// Structural pre-pass, input validation, stable row binning and prefix scans.
//
// The pre-pass replaces k_flops (src/spgemm_engine.cuh:47-50) — one thread per
// row with a serial loop — by one warp per row reading the row's entries and
// the referenced B row bounds in parallel; it also records the output row's
// column span, which selects between hash tables and dense column windows.
// The binning replaces k_caps (src/spgemm_engine.cuh:51-57), which only chose
// between one 1024-slot shared table and a global arena.
#include <climits>

#include "kernels.h"

namespace spg {

// ---------------------------------------------------------------------------
// validation
// ---------------------------------------------------------------------------
__global__ void k_validate(MatView A, uint32_t* status) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  if (warp == 0 && lane == 0) {
    if (A.rowptr[0] != 0 || (int64_t)A.rowptr[A.n] != A.nnz) report(status, DEV_ERR_INVALID_CSR);
  }
  for (int64_t i = warp; i < A.n; i += nwarps) {
    const int32_t s = A.rowptr[i], e = A.rowptr[i + 1];
    if (s < 0 || e < s || (int64_t)e > A.nnz) {
      if (lane == 0) report(status, DEV_ERR_INVALID_CSR);
      continue;
    }
    bool bad = false;
    for (int32_t p = s + lane; p < e; p += 32) {
      const int32_t j = A.col[p];
      if (j < 0 || j >= A.n) bad = true;
      if (p > s && A.col[p - 1] >= j) bad = true;
    }
    if (__any_sync(0xffffffffu, bad) && lane == 0) report(status, DEV_ERR_INVALID_CSR);
  }
}

cudaError_t launch_validate(const MatView& A, uint32_t* status, cudaStream_t s) {
  const int threads = 256;
  int64_t warps = A.n > 0 ? A.n : 1;
  int64_t blocks = (warps * 32 + threads - 1) / threads;
  if (blocks > 65535 * 8) blocks = 65535 * 8;
  k_validate<<<(unsigned)blocks, threads, 0, s>>>(A, status);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// pre-pass: products and output column span per row (one warp per row)
// ---------------------------------------------------------------------------
// Every index is checked before it is used, so the kernel may run before the
// host has seen the validation verdict: a row that meets a row pointer or
// column outside its range gets f = −1, and the later kernels of the
// one-readback plan skip it.  With `status` set it is also the validation of
// A (k_validate's checks, in the same read of A's rows): a violation sets
// DEV_ERR_INVALID_CSR there.
__global__ void k_prepass(MatView A, MatView B, int64_t* __restrict__ f, int32_t* __restrict__ lo,
                          int32_t* __restrict__ hi, uint32_t* status) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  if (status && warp == 0 && lane == 0 &&
      (A.rowptr[0] != 0 || (int64_t)A.rowptr[A.n] != A.nnz))
    report(status, DEV_ERR_INVALID_CSR);
  for (int64_t i = warp; i < A.n; i += nwarps) {
    int32_t s = A.rowptr[i], e = A.rowptr[i + 1];
    bool bad = s < 0 || e < s || (int64_t)e > A.nnz;
    if (bad) s = e = 0;
    long long prod = 0;
    int mn = INT_MAX, mx = -1;
    bool unsorted = false;
    for (int32_t p = s + lane; p < e; p += 32) {
      const int32_t k = A.col[p];
      if (status && p > s && A.col[p - 1] >= k) unsorted = true;
      if (k < 0 || k >= B.n) {
        bad = true;
        continue;
      }
      const int32_t bs = B.rowptr[k], be = B.rowptr[k + 1];
      if (bs < 0 || be < bs || (int64_t)be > B.nnz) {
        bad = true;
        continue;
      }
      if (be > bs) {
        prod += be - bs;
        mn = min(mn, B.col[bs]);
        mx = max(mx, B.col[be - 1]);
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      prod += __shfl_xor_sync(0xffffffffu, prod, o);
      mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
      mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    bad = __any_sync(0xffffffffu, bad);
    unsorted = __any_sync(0xffffffffu, unsorted);
    if (status && lane == 0 && (bad || unsorted)) report(status, DEV_ERR_INVALID_CSR);
    if (lane == 0) {
      f[i] = bad ? -1 : prod;
      lo[i] = bad ? INT_MAX : mn;
      hi[i] = bad ? -1 : mx;
    }
  }
}

cudaError_t launch_prepass(const MatView& A, const MatView& B, int64_t* f, int32_t* lo,
                           int32_t* hi, cudaStream_t s, uint32_t* status) {
  if (A.n == 0) {
    if (!status) return cudaSuccess;
    // no rows: the validation is rowptr[0] == 0 and nnz == 0 alone
    return launch_validate(A, status, s);
  }
  const int threads = 256;
  int64_t blocks = ((int64_t)A.n * 32 + threads - 1) / threads;
  if (blocks > 148 * 64) blocks = 148 * 64;
  k_prepass<<<(unsigned)blocks, threads, 0, s>>>(A, B, f, lo, hi, status);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// stable binning
// ---------------------------------------------------------------------------
__global__ void k_bin_hist(BinSource src, int32_t* __restrict__ hist, int nblocks) {
  __shared__ int cnt[kNumBins];
  if (threadIdx.x < kNumBins) cnt[threadIdx.x] = 0;
  __syncthreads();
  const int64_t base = (int64_t)blockIdx.x * kBinRowsPerBlock;
  for (int t = threadIdx.x; t < kBinRowsPerBlock; t += blockDim.x) {
    const int64_t i = base + t;
    if (i < src.n) atomicAdd(&cnt[row_bin(src, (int)i)], 1);
  }
  __syncthreads();
  if (threadIdx.x < kNumBins) hist[(int64_t)threadIdx.x * nblocks + blockIdx.x] = cnt[threadIdx.x];
}

// Single block: exclusive scan of the bin-major histogram in place; writes
// per-bin counts and starts.
__global__ void k_bin_offsets(int32_t* hist, int nblocks, int64_t* counts_out) {
  __shared__ int scratch[33];
  __shared__ long long carry;
  __shared__ long long bin_start[kNumBins];
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  const int64_t total = (int64_t)kNumBins * nblocks;
  for (int64_t base = 0; base < total; base += blockDim.x) {
    const int64_t idx = base + threadIdx.x;
    const int v = idx < total ? hist[idx] : 0;
    int tot;
    const int ex = block_exclusive_scan(v, scratch, &tot);
    if (idx < total) hist[idx] = (int32_t)(carry + ex);
    // the start of every bin whose first block lies in this chunk
    if (idx < total && idx % nblocks == 0) bin_start[idx / nblocks] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x < kNumBins) {
    const int b = threadIdx.x;
    const long long start = bin_start[b];
    const long long end = (b + 1 < kNumBins) ? bin_start[b + 1] : carry;
    counts_out[b] = end - start;
    counts_out[kNumBins + b] = start;
  }
}

__global__ void k_bin_scatter(BinSource src, const int32_t* __restrict__ offs, int nblocks,
                              int32_t* __restrict__ rows_out) {
  __shared__ int running[kNumBins];
  __shared__ int warp_cnt[32][kNumBins];
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if (threadIdx.x < kNumBins) running[threadIdx.x] = offs[(int64_t)threadIdx.x * nblocks + blockIdx.x];
  const int64_t base = (int64_t)blockIdx.x * kBinRowsPerBlock;
  for (int round = 0; round < kBinRowsPerBlock; round += blockDim.x) {
    for (int t = threadIdx.x; t < 32 * kNumBins; t += blockDim.x) (&warp_cnt[0][0])[t] = 0;
    __syncthreads();
    const int64_t i = base + round + threadIdx.x;
    const int b = (i < src.n) ? row_bin(src, (int)i) : -1;
    const unsigned same = __match_any_sync(0xffffffffu, b);
    const int rank = __popc(same & lanemask_lt());
    if (b >= 0 && rank == 0) warp_cnt[w][b] = __popc(same);
    __syncthreads();
    int pos = 0;
    if (b >= 0) {
      pos = running[b] + rank;
      for (int ww = 0; ww < w; ++ww) pos += warp_cnt[ww][b];
    }
    __syncthreads();
    if (threadIdx.x < kNumBins) {
      int add = 0;
      for (int ww = 0; ww < nw; ++ww) add += warp_cnt[ww][threadIdx.x];
      running[threadIdx.x] += add;
    }
    if (b >= 0) rows_out[pos] = (int32_t)i;
    __syncthreads();
  }
}

cudaError_t launch_bin_rows(const BinSource& src, int32_t* hist, int64_t* counts_out,
                            int32_t* rows_out, cudaStream_t s) {
  const int nblocks = (int)((src.n + kBinRowsPerBlock - 1) / kBinRowsPerBlock);
  if (nblocks == 0) {
    cudaError_t e = cudaMemsetAsync(counts_out, 0, sizeof(int64_t) * 2 * kNumBins, s);
    return e;
  }
  k_bin_hist<<<nblocks, 256, 0, s>>>(src, hist, nblocks);
  SPG_COUNT_LAUNCH();
  k_bin_offsets<<<1, 1024, 0, s>>>(hist, nblocks, counts_out);
  SPG_COUNT_LAUNCH();
  k_bin_scatter<<<nblocks, 256, 0, s>>>(src, hist, nblocks, rows_out);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// exclusive scans (three phases: tile sums, scan of tile sums, apply)
// ---------------------------------------------------------------------------
constexpr int kScanThreads = 512;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ long long block_exclusive_scan64(long long v, long long* scratch,
                                                           long long* total) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  long long incl = v;
  for (int o = 1; o < 32; o <<= 1) {
    long long t = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += t;
  }
  __syncthreads();
  if (lane == 31) scratch[w] = incl;
  __syncthreads();
  long long before = 0, all = 0;
  for (int i = 0; i < nw; ++i) {
    long long s = scratch[i];
    if (i < w) before += s;
    all += s;
  }
  *total = all;
  return before + incl - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const int32_t* __restrict__ in,
                                                             int64_t n, long long* tile_sums) {
  __shared__ long long scratch[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) s += in[base + k];
  s = block_sum64(s, scratch);
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = s;
}

__global__ void __launch_bounds__(1024) k_scan_tile_sums(long long* tile_sums, int64_t ntiles) {
  __shared__ long long scratch[32];
  __shared__ long long carry;
  if (threadIdx.x == 0) carry = 0;
  __syncthreads();
  for (int64_t b = 0; b < ntiles; b += blockDim.x) {
    const int64_t idx = b + threadIdx.x;
    long long v = idx < ntiles ? tile_sums[idx] : 0;
    long long tot;
    long long ex = block_exclusive_scan64(v, scratch, &tot);
    if (idx < ntiles) tile_sums[idx] = carry + ex;
    __syncthreads();
    if (threadIdx.x == 0) carry += tot;
    __syncthreads();
  }
  if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

template <typename OutT>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int32_t* __restrict__ in,
                                                             OutT* __restrict__ out, int64_t n,
                                                             const long long* tile_sums,
                                                             int64_t ntiles) {
  __shared__ long long scratch[32];
  const int64_t base = (int64_t)blockIdx.x * kScanTile + (int64_t)threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  long long tot;
  long long run = tile_sums[blockIdx.x] + block_exclusive_scan64(s, scratch, &tot);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = (OutT)run;
    run += v[k];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = (OutT)tile_sums[ntiles];
}

// One tile (n <= kScanTile): the whole scan in one launch.
template <typename OutT>
__global__ void __launch_bounds__(kScanThreads) k_scan_single(const int32_t* __restrict__ in,
                                                              OutT* __restrict__ out, int64_t n) {
  __shared__ long long scratch[32];
  const int64_t base = (int64_t)threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  long long s = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = (base + k < n) ? in[base + k] : 0;
    s += v[k];
  }
  long long tot;
  long long run = block_exclusive_scan64(s, scratch, &tot);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = (OutT)run;
    run += v[k];
  }
  if (threadIdx.x == 0) out[n] = (OutT)tot;
}

// One tile: the row-pointer scan and the row statistics (Σ products, max
// products, max row count) of a small plan in a single launch.
__global__ void __launch_bounds__(kScanThreads) k_scan_stats_single(
    const int32_t* __restrict__ cnt, const int64_t* __restrict__ f, int64_t n,
    int64_t* __restrict__ rowptr, unsigned long long* __restrict__ stats) {
  __shared__ long long scratch[32];
  __shared__ unsigned long long red[3][32];
  const int64_t base = (int64_t)threadIdx.x * kScanItems;
  int32_t v[kScanItems];
  long long s = 0;
  unsigned long long sf = 0, mf = 0, mc = 0;
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    const bool in = base + k < n;
    v[k] = in ? cnt[base + k] : 0;
    s += v[k];
    if (in) {
      const unsigned long long fk = (unsigned long long)f[base + k];
      sf += fk;
      mf = fk > mf ? fk : mf;
      const unsigned long long ck = (unsigned long long)v[k];
      mc = ck > mc ? ck : mc;
    }
  }
  long long tot;
  long long run = block_exclusive_scan64(s, scratch, &tot);
#pragma unroll
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) rowptr[base + k] = run;
    run += v[k];
  }
  for (int o = 16; o > 0; o >>= 1) {
    sf += __shfl_xor_sync(0xffffffffu, sf, o);
    const unsigned long long a = __shfl_xor_sync(0xffffffffu, mf, o);
    const unsigned long long b = __shfl_xor_sync(0xffffffffu, mc, o);
    mf = a > mf ? a : mf;
    mc = b > mc ? b : mc;
  }
  const int w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    red[0][w] = sf;
    red[1][w] = mf;
    red[2][w] = mc;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long a = 0, b = 0, c = 0;
    for (int i = 0; i < nw; ++i) {
      a += red[0][i];
      b = red[1][i] > b ? red[1][i] : b;
      c = red[2][i] > c ? red[2][i] : c;
    }
    stats[0] = a;
    stats[1] = b;
    stats[2] = c;
    rowptr[n] = tot;
  }
}

cudaError_t launch_scan_stats_small(const int32_t* cnt, const int64_t* f, int64_t n,
                                    int64_t* rowptr, unsigned long long* stats, void* tmp,
                                    cudaStream_t s) {
  if (n <= 0 || n > kScanTile) {
    cudaError_t e = launch_scan_i32_i64(cnt, rowptr, n, tmp, s);
    if (e != cudaSuccess) return e;
    return launch_row_stats(f, cnt, (int32_t)n, stats, s);
  }
  k_scan_stats_single<<<1, kScanThreads, 0, s>>>(cnt, f, n, rowptr, stats);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

size_t scan_tmp_bytes(int64_t n) {
  int64_t ntiles = (n + kScanTile - 1) / kScanTile;
  return sizeof(long long) * (size_t)(ntiles + 1);
}

template <typename OutT>
static cudaError_t scan_impl(const int32_t* in, OutT* out, int64_t n, void* tmp, cudaStream_t s) {
  long long* tile = (long long*)tmp;
  const int64_t ntiles = (n + kScanTile - 1) / kScanTile;
  if (ntiles == 0) return cudaMemsetAsync(out, 0, sizeof(OutT), s);
  if (ntiles == 1) {
    k_scan_single<OutT><<<1, kScanThreads, 0, s>>>(in, out, n);
    SPG_COUNT_LAUNCH();
    return cudaGetLastError();
  }
  k_scan_tiles<<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, n, tile);
  SPG_COUNT_LAUNCH();
  k_scan_tile_sums<<<1, 1024, 0, s>>>(tile, ntiles);
  SPG_COUNT_LAUNCH();
  k_scan_apply<OutT><<<(unsigned)ntiles, kScanThreads, 0, s>>>(in, out, n, tile, ntiles);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_scan_i32_i64(const int32_t* in, int64_t* out, int64_t n, void* tmp,
                                cudaStream_t s) {
  return scan_impl<int64_t>(in, out, n, tmp, s);
}
cudaError_t launch_scan_i32_i32(const int32_t* in, int32_t* out, int64_t n, void* tmp,
                                cudaStream_t s) {
  return scan_impl<int32_t>(in, out, n, tmp, s);
}

// ---------------------------------------------------------------------------
// column histogram and structural descriptors
// ---------------------------------------------------------------------------
__global__ void k_col_count(MatView A, int32_t* __restrict__ cnt) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < A.nnz; p += stride) {
    const int32_t k = A.col[p];
    if (k >= 0 && k < A.n) atomicAdd(&cnt[k], 1);  // others: invalid input, never counted
  }
}

cudaError_t launch_col_count(const MatView& A, int32_t* cnt, cudaStream_t s) {
  if (A.nnz == 0) return cudaSuccess;
  int64_t blocks = (A.nnz + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  k_col_count<<<(unsigned)blocks, 256, 0, s>>>(A, cnt);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

__global__ void k_describe(MatView A, const int32_t* __restrict__ colcount, DescAccum* acc) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  unsigned long long deg2 = 0, paa = 0, paat = 0, sym = 0;
  int maxdeg = 0, maxcol = 0, band = 0;
  for (int64_t i = warp; i < A.n; i += nwarps) {
    const int32_t s = A.rowptr[i], e = A.rowptr[i + 1];
    if (lane == 0) {
      deg2 += (unsigned long long)(e - s) * (unsigned long long)(e - s);
      maxdeg = max(maxdeg, e - s);
      const unsigned long long c = colcount[i];
      paat += c * c;
      maxcol = max(maxcol, (int)c);
    }
    for (int32_t p = s + lane; p < e; p += 32) {
      const int32_t j = A.col[p];
      paa += (unsigned long long)(A.rowptr[j + 1] - A.rowptr[j]);
      band = max(band, (int)(j > i ? j - i : i - j));
      // is (j, i) present?  binary search for i in row j
      int32_t lo = A.rowptr[j], hi = A.rowptr[j + 1];
      while (lo < hi) {
        int32_t mid = (lo + hi) >> 1;
        if (A.col[mid] < i) lo = mid + 1; else hi = mid;
      }
      if (lo < A.rowptr[j + 1] && A.col[lo] == i) ++sym;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    deg2 += __shfl_xor_sync(0xffffffffu, deg2, o);
    paa += __shfl_xor_sync(0xffffffffu, paa, o);
    paat += __shfl_xor_sync(0xffffffffu, paat, o);
    sym += __shfl_xor_sync(0xffffffffu, sym, o);
    maxdeg = max(maxdeg, __shfl_xor_sync(0xffffffffu, maxdeg, o));
    maxcol = max(maxcol, __shfl_xor_sync(0xffffffffu, maxcol, o));
    band = max(band, __shfl_xor_sync(0xffffffffu, band, o));
  }
  if (lane == 0) {
    atomicAdd(&acc->sum_deg2, deg2);
    atomicAdd(&acc->prod_aa, paa);
    atomicAdd(&acc->prod_aat, paat);
    atomicAdd(&acc->sym_hits, sym);
    atomicMax(&acc->max_deg, maxdeg);
    atomicMax(&acc->max_col_deg, maxcol);
    atomicMax(&acc->bandwidth, band);
  }
}

__global__ void k_row_stats(const int64_t* __restrict__ f, const int32_t* __restrict__ rownnz,
                            int32_t n, unsigned long long* out) {
  unsigned long long sum = 0, mf = 0, mn = 0;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
    const unsigned long long v = (unsigned long long)f[i];
    sum += v;
    mf = v > mf ? v : mf;
    const unsigned long long c = (unsigned long long)rownnz[i];
    mn = c > mn ? c : mn;
  }
  for (int o = 16; o > 0; o >>= 1) {
    sum += __shfl_xor_sync(0xffffffffu, sum, o);
    const unsigned long long a = __shfl_xor_sync(0xffffffffu, mf, o);
    const unsigned long long b = __shfl_xor_sync(0xffffffffu, mn, o);
    mf = a > mf ? a : mf;
    mn = b > mn ? b : mn;
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(&out[0], sum);
    atomicMax(&out[1], mf);
    atomicMax(&out[2], mn);
  }
}

cudaError_t launch_row_stats(const int64_t* f, const int32_t* rownnz, int32_t n,
                             unsigned long long* out, cudaStream_t s) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(unsigned long long) * 3, s);
  if (e != cudaSuccess || n == 0) return e;
  int64_t blocks = ((int64_t)n + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  k_row_stats<<<(unsigned)blocks, 256, 0, s>>>(f, rownnz, n, out);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_describe(const MatView& A, const int32_t* colcount, DescAccum* acc,
                            cudaStream_t s) {
  if (A.n == 0) return cudaSuccess;
  int64_t blocks = ((int64_t)A.n * 32 + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_describe<<<(unsigned)blocks, 256, 0, s>>>(A, colcount, acc);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace spg
