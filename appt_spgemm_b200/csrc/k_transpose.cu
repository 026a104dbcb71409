// CSR → CSR-of-Aᵀ by counting sort, and the segment sort it (and the Gram
// mirror) finishes with.
//
// The reference builds Aᵀ with a global atomicAdd histogram, a Thrust scan and
// a one-thread-per-row atomic-cursor scatter (k_colcount / k_scatter /
// build_At, src/spgemm_engine.cuh:37-44, :140-146), which leaves the entries of
// each Aᵀ row in a run-dependent order.  Here the scatter is one warp per row
// (coalesced reads of A) into a staging copy, and a segment sort then orders
// every Aᵀ row by its row index into the final arrays, so the transpose is
// deterministic and its rows are sorted like cusparseCsr2cscEx2's.
#include <climits>

#include "kernels.h"

namespace spg {

__global__ void k_transpose_scatter(MatView A, const int32_t* __restrict__ t_rowptr,
                                    int32_t* __restrict__ cursor, int32_t* __restrict__ tmp_col,
                                    double* __restrict__ tmp_val) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t i = warp; i < A.n; i += nwarps) {
    int32_t s = A.rowptr[i], e = A.rowptr[i + 1];
    // indices are checked (the one-readback plan runs this before the host has
    // the validation verdict): an invalid input only leaves slots unwritten
    if (s < 0 || e < s || (int64_t)e > A.nnz) s = e = 0;
    for (int32_t p = s + lane; p < e; p += 32) {
      const int32_t k = A.col[p];
      if (k < 0 || k >= A.n) continue;
      const int32_t d = t_rowptr[k] + atomicAdd(&cursor[k], 1);
      if (d >= t_rowptr[k + 1]) continue;
      tmp_col[d] = (int32_t)i;
      tmp_val[d] = A.val[p];
    }
  }
}

// Transpose values of a structurally symmetric A: row k of Aᵀ has A's row-k
// pattern, and Aᵀ[k,i] = A[i,k] is found by binary search for k in row i.
// Any entry without its mirror sets *asym; the caller then falls back to the
// counting sort.  Bounds are checked here because the kernel runs before the
// host has seen the validation verdict.
__global__ void k_sym_transpose_vals(MatView A, double* __restrict__ t_val, int* asym) {
  const int lane = threadIdx.x & 31;
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t k = warp; k < A.n; k += nwarps) {
    // once any warp has found an entry without a mirror the result is discarded
    if (*(volatile int*)asym) break;
    bool miss = false;
    const int32_t s = A.rowptr[k], e = A.rowptr[k + 1];
    if (s < 0 || e < s || (int64_t)e > A.nnz) {
      miss = true;
    } else {
      for (int32_t p = s + lane; p < e; p += 32) {
        const int32_t i = A.col[p];
        if (i < 0 || i >= A.n) {
          miss = true;
          break;
        }
        int32_t lo = A.rowptr[i], hi = A.rowptr[i + 1];
        if (lo < 0 || hi < lo || (int64_t)hi > A.nnz) {
          miss = true;
          break;
        }
        const int32_t end = hi;
        while (lo < hi) {
          const int32_t mid = (lo + hi) >> 1;
          if (A.col[mid] < k) lo = mid + 1; else hi = mid;
        }
        if (lo < end && A.col[lo] == k) {
          t_val[p] = A.val[lo];
        } else {
          miss = true;
          break;
        }
      }
    }
    if (__any_sync(0xffffffffu, miss)) {
      if (lane == 0) atomicOr(asym, 1);
      break;
    }
  }
}

cudaError_t launch_sym_transpose_vals(const MatView& A, double* t_val, int* asym,
                                      cudaStream_t s) {
  if (A.n == 0 || A.nnz == 0) return cudaSuccess;
  int64_t blocks = ((int64_t)A.n * 32 + 255) / 256;
  if (blocks > 148 * 16) blocks = 148 * 16;
  k_sym_transpose_vals<<<(unsigned)blocks, 256, 0, s>>>(A, t_val, asym);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

// ---- segment sort --------------------------------------------------------------
constexpr int kShortSeg = 256;      // warp + shared bitonic
constexpr int kMidSeg = 8192;       // CTA + shared bitonic
constexpr int kLongThreads = 512;
constexpr int kLongWindow = 1 << 18;  // bitmap bits of the long-segment counting sort

__device__ __forceinline__ int64_t seg_src(const SegSortArgs& a, int64_t s) {
  return a.src_off64 ? a.src_off64[s] : (int64_t)a.src_off32[s];
}
__device__ __forceinline__ int64_t seg_dst(const SegSortArgs& a, int64_t s) {
  return a.dst_off64 ? a.dst_off64[s] : (int64_t)a.dst_off32[s];
}
__device__ __forceinline__ int64_t seg_len(const SegSortArgs& a, int64_t s) {
  return a.lens ? (int64_t)a.lens[s] : seg_src(a, s + 1) - seg_src(a, s);
}

// One segment of at most 32·E entries by one warp: (key << 8 | index) words
// sorted in registers, then keys written and payloads gathered by index.
template <int E>
__device__ __forceinline__ void seg_reg_sort(const SegSortArgs& a, int64_t so, int64_t dof,
                                             int len) {
  const int lane = threadIdx.x & 31;
  uint32_t r[E];
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int e = lane * E + i;
    r[i] = e < len ? (((uint32_t)a.src_key[so + e] << 8) | (uint32_t)e) : 0xffffffffu;
  }
  warp_bitonic_sort<E>(r);
#pragma unroll
  for (int i = 0; i < E; ++i) {
    const int e = lane * E + i;
    if (e < len) {
      a.dst_key[dof + e] = (int32_t)(r[i] >> 8);
      a.dst_val[dof + e] = a.src_val[so + (r[i] & 255u)];
    }
  }
}

__global__ void __launch_bounds__(256, 4) k_segsort_short(SegSortArgs a) {
  __shared__ int skeys[8][kShortSeg];
  __shared__ double svals[8][kShortSeg];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const WarpGroup g(32);
  int* keys = skeys[w];
  double* vals = svals[w];
  const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t s = warp; s < a.nseg; s += nwarps) {
    const int64_t len = seg_len(a, s);
    if (len <= 0) continue;
    const int64_t so = seg_src(a, s), dof = seg_dst(a, s);
    if (len > kShortSeg) {
      if (lane == 0) a.long_list[atomicAdd(a.long_count, 1)] = (int32_t)s;
      continue;
    }
    if (a.key_bound <= (1 << 24)) {  // keys fit the (key << 8 | index) packing
      if (len <= 32) seg_reg_sort<1>(a, so, dof, (int)len);
      else if (len <= 64) seg_reg_sort<2>(a, so, dof, (int)len);
      else if (len <= 128) seg_reg_sort<4>(a, so, dof, (int)len);
      else seg_reg_sort<8>(a, so, dof, (int)len);
      continue;
    }
    const int P = next_pow2_int((int)len);
    for (int i = lane; i < P; i += 32) {
      if (i < len) {
        keys[i] = a.src_key[so + i];
        vals[i] = a.src_val[so + i];
      } else {
        keys[i] = INT_MAX;
      }
    }
    __syncwarp();
    bitonic_sort_pairs(g, keys, vals, P);
    for (int i = lane; i < len; i += 32) {
      a.dst_key[dof + i] = keys[i];
      a.dst_val[dof + i] = vals[i];
    }
    __syncwarp();
  }
}

// Long segments (count read on the device): bitonic in shared memory up to
// kMidSeg entries, else a counting sort over bitmap windows of the key range
// (keys are unique, so a key's rank is the number of set bits below it).
__global__ void __launch_bounds__(kLongThreads) k_segsort_long(SegSortArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  __shared__ long long scratch[33];
  __shared__ int s_minmax[2];
  const CtaGroup g;
  const int nlong = *a.long_count;
  for (int li = blockIdx.x; li < nlong; li += gridDim.x) {
    const int64_t s = a.long_list[li];
    const int64_t len = seg_len(a, s);
    const int64_t so = seg_src(a, s), dof = seg_dst(a, s);
    if (len <= kMidSeg) {
      double* vals = (double*)smem;
      int* keys = (int*)(vals + kMidSeg);
      const int P = next_pow2_int((int)len);
      for (int i = threadIdx.x; i < P; i += blockDim.x) {
        if (i < len) {
          keys[i] = a.src_key[so + i];
          vals[i] = a.src_val[so + i];
        } else {
          keys[i] = INT_MAX;
        }
      }
      __syncthreads();
      bitonic_sort_pairs(g, keys, vals, P);
      for (int i = threadIdx.x; i < len; i += blockDim.x) {
        a.dst_key[dof + i] = keys[i];
        a.dst_val[dof + i] = vals[i];
      }
      __syncthreads();
      continue;
    }
    // key range of the segment
    if (threadIdx.x == 0) {
      s_minmax[0] = INT_MAX;
      s_minmax[1] = -1;
    }
    __syncthreads();
    int mn = INT_MAX, mx = -1;
    for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
      const int k = a.src_key[so + i];
      mn = min(mn, k);
      mx = max(mx, k);
    }
    atomicMin(&s_minmax[0], mn);
    atomicMax(&s_minmax[1], mx);
    __syncthreads();
    const int kmin = s_minmax[0], kmax = s_minmax[1];
    uint32_t* bm = (uint32_t*)smem;
    int* pre = (int*)(bm + kLongWindow / 32);
    int64_t written = 0;
    for (long long w0 = kmin; w0 <= kmax; w0 += kLongWindow) {
      const int nwords = (int)min((long long)kLongWindow / 32, (kmax - w0) / 32 + 1);
      for (int i = threadIdx.x; i < nwords; i += blockDim.x) bm[i] = 0u;
      __syncthreads();
      for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
        const long long d = (long long)a.src_key[so + i] - w0;
        if (d >= 0 && d < (long long)nwords * 32) atomicOr(&bm[d >> 5], 1u << (d & 31));
      }
      __syncthreads();
      const int per = (nwords + blockDim.x - 1) / blockDim.x;
      const int wb = min(nwords, (int)threadIdx.x * per), we = min(nwords, wb + per);
      int local = 0;
      for (int i = wb; i < we; ++i) local += __popc(bm[i]);
      int tot;
      int run = block_exclusive_scan(local, (int*)scratch, &tot);
      for (int i = wb; i < we; ++i) {
        pre[i] = run;
        run += __popc(bm[i]);
      }
      __syncthreads();
      for (int64_t i = threadIdx.x; i < len; i += blockDim.x) {
        const int key = a.src_key[so + i];
        const long long d = (long long)key - w0;
        if (d >= 0 && d < (long long)nwords * 32) {
          const int wi = (int)(d >> 5), b = (int)(d & 31);
          const int64_t pos = written + pre[wi] + __popc(bm[wi] & ((1u << b) - 1u));
          if (pos < len) {
            a.dst_key[dof + pos] = key;
            a.dst_val[dof + pos] = a.src_val[so + i];
          }
        }
      }
      written += tot;
      __syncthreads();
    }
    if (written != len && threadIdx.x == 0) report(a.status, DEV_ERR_OVERFLOW);
    __syncthreads();
  }
}

static size_t long_smem_bytes() {
  const size_t bitonic = (size_t)kMidSeg * 12;
  const size_t bitmap = (size_t)kLongWindow / 32 * 8;
  return bitonic > bitmap ? bitonic : bitmap;
}

cudaError_t launch_segsort(const SegSortArgs& a, int num_sms, cudaStream_t s) {
  if (a.nseg <= 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(a.long_count, 0, sizeof(int32_t), s);
  if (e != cudaSuccess) return e;
  int64_t blocks = ((int64_t)a.nseg * 32 + 255) / 256;
  const int64_t cap = (int64_t)num_sms * 8;
  if (blocks > cap) blocks = cap;
  k_segsort_short<<<(unsigned)blocks, 256, 0, s>>>(a);
  SPG_COUNT_LAUNCH();
  const size_t smem = long_smem_bytes();
  e = cudaFuncSetAttribute(k_segsort_long, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k_segsort_long<<<(unsigned)(num_sms * 2), kLongThreads, smem, s>>>(a);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_transpose(const MatView& A, int32_t* t_rowptr, int32_t* t_col, double* t_val,
                             const TransposeWork& w, int num_sms, cudaStream_t s) {
  const int32_t n = A.n;
  cudaError_t e = cudaMemsetAsync(w.cnt, 0, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), s);
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(w.cursor, 0, sizeof(int32_t) * (size_t)(n > 0 ? n : 1), s);
  if (e != cudaSuccess) return e;
  if ((e = launch_col_count(A, w.cnt, s)) != cudaSuccess) return e;
  if ((e = launch_scan_i32_i32(w.cnt, t_rowptr, n, w.scan_tmp, s)) != cudaSuccess) return e;
  if (A.nnz == 0 || n == 0) return cudaSuccess;
  int64_t blocks = ((int64_t)n * 32 + 255) / 256;
  const int64_t cap = (int64_t)num_sms * 16;
  if (blocks > cap) blocks = cap;
  k_transpose_scatter<<<(unsigned)blocks, 256, 0, s>>>(A, t_rowptr, w.cursor, w.tmp_col,
                                                       w.tmp_val);
  SPG_COUNT_LAUNCH();
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  SegSortArgs sa{};
  sa.nseg = n;
  sa.src_off32 = t_rowptr;
  sa.dst_off32 = t_rowptr;
  sa.src_key = w.tmp_col;
  sa.src_val = w.tmp_val;
  sa.dst_key = t_col;
  sa.dst_val = t_val;
  sa.key_bound = n;
  sa.long_list = w.long_list;
  sa.long_count = w.long_count;
  sa.status = w.status;
  return launch_segsort(sa, num_sms, s);
}

}  // namespace spg
