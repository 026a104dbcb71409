// Shared-memory hash rows: the symbolic and numeric phases for every row whose
// table fits in shared memory, one kernel per table-size bin.
//
// Replaces k_symbolic / k_numeric (src/spgemm_engine.cuh:71-115), which ran one
// warp per row over one fixed 1024-slot slice, inserted with atomicCAS on every
// probe, accumulated with atomicAdd(double) in arbitrary order and emitted
// (row·n+col, value) pairs in hash order for a global radix sort.  Here:
//  - the table is sized per bin and the group of lanes per row is sized with it
//    (sub-warp groups for small tables, a whole CTA for the largest);
//  - each probe claims its slot with one CAS (claim-first), and a freshly
//    claimed slot's value is set to 0.0 + a·b, so no value array is cleared;
//  - the numeric phase walks row i of A in order and synchronises the group
//    after each k, so every output value is Σ_k a_ik·b_kj added in increasing
//    position of k with the product rounded first — the same sum the CPU
//    oracle forms, bit for bit;
//  - the row is compacted and bitonic-sorted in shared memory and written to
//    its final CSR slots, so no global sort exists.
#include <climits>
#include <type_traits>

#include "kernels.h"

namespace spg {

__host__ __device__ constexpr size_t row_group_bytes(int T, int G, bool numeric) {
  return numeric ? (size_t)T * 12 + (size_t)G * 16 : (size_t)T * 4 + (size_t)G * 8;
}
constexpr size_t kCtaScratchBytes = 256;  // 32 long longs for block reductions

// Numeric CTA rows of 4096- and 8192-slot tables sort packed words with the
// CTA-wide radix sort; its second buffer (T words) and digit counters (256
// per warp, T/512 warps) follow the scratch.  16384-slot tables keep the
// bitonic pair sort (the extra buffers would not fit beside the table).
template <int LOG2T, bool NUMERIC>
__host__ __device__ constexpr bool cta_radix() {
  return NUMERIC && LOG2T >= 12 && LOG2T <= 13;
}
template <int LOG2T, bool NUMERIC>
__host__ __device__ constexpr size_t cta_radix_bytes() {
  return cta_radix<LOG2T, NUMERIC>() ? ((size_t)4 << LOG2T) + ((size_t)4 << LOG2T) / 2 : 0;
}

// Packs the occupied slots of keys[0..T) as ((key − lo) << LOG2T) | slot and
// moves them to the front in slot order (in place; the values stay in their
// slots).  Returns their count.
template <int LOG2T>
__device__ __forceinline__ int cta_compact_packed(int* keys, int lo, void* scratch) {
  constexpr int T = 1 << LOG2T;
  int m = 0;
  for (int base = 0; base < T; base += blockDim.x) {
    const int s = base + threadIdx.x;
    const int key = s < T ? keys[s] : kEmptyKey;
    const bool occ = key != kEmptyKey;
    int tot;
    const int ex = block_exclusive_scan(occ ? 1 : 0, (int*)scratch, &tot);
    // writes land below base + blockDim.x; the next chunk reads only above
    if (occ) keys[m + ex] = (int)(((uint32_t)(key - lo) << LOG2T) | (uint32_t)s);
    m += tot;
  }
  __syncthreads();
  return m;
}

__device__ __forceinline__ int grp_sum(const WarpGroup& g, int v, void*) { return g.sum(v); }
__device__ __forceinline__ int grp_sum(const CtaGroup&, int v, void* scratch) {
  return (int)block_sum64(v, (long long*)scratch);
}

// Move the occupied slots of keys/vals[0..T) to the front in slot order.
template <int T>
__device__ __forceinline__ int grp_compact(const WarpGroup& g, int* keys, double* vals, void*) {
  int m = 0;
  for (int base = 0; base < T; base += g.G) {
    const int s = base + g.lane;
    const int key = keys[s];
    const double v = vals[s];
    const bool occ = key != kEmptyKey;
    const unsigned bal = g.ballot(occ);
    const int pos = m + __popc(bal & ((1u << g.lane) - 1u));
    g.sync();
    if (occ) {
      keys[pos] = key;
      vals[pos] = v;
    }
    m += __popc(bal);
    g.sync();
  }
  return m;
}

template <int T>
__device__ __forceinline__ int grp_compact(const CtaGroup& g, int* keys, double* vals,
                                           void* scratch) {
  int m = 0;
  for (int base = 0; base < T; base += g.G) {
    const int s = base + g.lane;
    int key = kEmptyKey;
    double v = 0.0;
    if (s < T) {
      key = keys[s];
      v = vals[s];
    }
    const bool occ = key != kEmptyKey;
    int tot;
    const int ex = block_exclusive_scan(occ ? 1 : 0, (int*)scratch, &tot);
    // writes land below base + G; the next chunk reads only slots >= base + G
    if (occ) {
      keys[m + ex] = key;
      vals[m + ex] = v;
    }
    m += tot;
  }
  __syncthreads();
  return m;
}

template <int LOG2T, bool NUMERIC, bool GRAM, class Grp>
__device__ __forceinline__ void hash_row(const Grp& g, const RowArgs& a, const int row,
                                         int* __restrict__ keys, double* __restrict__ vals,
                                         int* st_bs, int* st_len, double* st_a, void* scratch,
                                         uint32_t* rtmp, int* rcnt) {
  constexpr int T = 1 << LOG2T;
  for (int s = g.lane; s < T; s += g.G) keys[s] = kEmptyKey;
  const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];
  for (int32_t pb = ps; pb < pe; pb += g.G) {
    const int cnt = min(g.G, pe - pb);
    g.sync();  // table cleared / previous chunk's staging consumed
    if (g.lane < cnt) {
      const int32_t k = a.A.col[pb + g.lane];
      const int32_t bs = a.B.rowptr[k];
      st_bs[g.lane] = bs;
      st_len[g.lane] = a.B.rowptr[k + 1] - bs;
      if (NUMERIC) st_a[g.lane] = a.A.val[pb + g.lane];
    }
    g.sync();
    for (int t = 0; t < cnt; ++t) {
      const int32_t bs = st_bs[t], len = st_len[t];
      const double av = NUMERIC ? st_a[t] : 0.0;
      for (int q = g.lane; q < len; q += g.G) {
        const int32_t j = a.B.col[bs + q];
        if (NUMERIC && GRAM && j < row) continue;
        // claim-first probe, as in the warp kernels (reading the slot before
        // claiming measured slower: R-MAT 2^18 A·A 62.3 against 60.2 ms)
        insert_acc<LOG2T, NUMERIC>(keys, vals, j,
                                   NUMERIC ? __dmul_rn(av, a.B.val[bs + q]) : 0.0, a.status);
      }
      if (NUMERIC) g.sync();  // k-order of the accumulation
    }
  }
  g.sync();

  if (!NUMERIC) {
    int c = 0, cl = 0;
    for (int s = g.lane; s < T; s += g.G) {
      const int k = keys[s];
      if (k != kEmptyKey) {
        ++c;
        if (GRAM && k < row) ++cl;
      }
    }
    c = grp_sum(g, c, scratch);
    if (GRAM) cl = grp_sum(g, cl, scratch);
    if (g.lane == 0) {
      a.rownnz[row] = c;
      if (GRAM) a.rowlow[row] = cl;
    }
    g.sync();
    return;
  }

  if constexpr (cta_radix<LOG2T, NUMERIC>() && std::is_same<Grp, CtaGroup>::value) {
    const int lo = a.lo[row];
    if ((int64_t)a.hi[row] - lo < ((int64_t)1 << (32 - LOG2T))) {
      int m = cta_compact_packed<LOG2T>(keys, lo, scratch);
      const int32_t low = GRAM ? a.low_in[row] : 0;
      const int expect = a.cnt_in[row] - low;
      if (m != expect) {
        if (g.lane == 0) report(a.status, DEV_ERR_OVERFLOW);
        if (m > expect) m = expect;
      }
      const uint32_t* sorted = radix_sort_words<(T >> 9), 8>(
          (uint32_t*)keys, rtmp, m, LOG2T, span_bits(lo, a.hi[row]), rcnt, (int*)scratch);
      emit_packed<LOG2T, GRAM>(a, row, lo, m, sorted, vals, a.rowptr[row] + low, g.lane, g.G);
      g.sync();  // the table is reused by the next row
      return;
    }
  }

  int m = grp_compact<T>(g, keys, vals, scratch);
  const int P = next_pow2_int(m);
  for (int s = m + g.lane; s < P; s += g.G) keys[s] = INT_MAX;
  g.sync();
  bitonic_sort_pairs(g, keys, vals, P);

  const int32_t low = GRAM ? a.low_in[row] : 0;
  const int expect = a.cnt_in[row] - low;
  if (m != expect) {
    if (g.lane == 0) report(a.status, DEV_ERR_OVERFLOW);
    if (m > expect) m = expect;
  }
  const int64_t base = a.rowptr[row] + low;
  const int cb = a.colbase ? a.colbase[row] : 0;
  for (int t = g.lane; t < m; t += g.G) {
    const int j = keys[t];
    const double v = vals[t];
    a.ccol[base + t] = j - cb;
    a.cval[base + t] = v;
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
  g.sync();  // the table is reused by the group's next row
}

template <int LOG2T, bool NUMERIC, bool GRAM>
__global__ void __launch_bounds__(256) k_hash_warp(RowArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int T = 1 << LOG2T;
  const WarpGroup g(a.G);
  const int rows_per_cta = blockDim.x / a.G;
  const int gi = threadIdx.x / a.G;
  unsigned char* base = smem + (size_t)gi * row_group_bytes(T, a.G, NUMERIC);
  double* vals = (double*)base;
  int *keys, *st_bs, *st_len;
  double* st_a = nullptr;
  if (NUMERIC) {
    keys = (int*)(base + (size_t)T * 8);
    st_a = (double*)(base + (size_t)T * 12);
    st_bs = (int*)(base + (size_t)T * 12 + (size_t)a.G * 8);
  } else {
    keys = (int*)base;
    st_bs = keys + T;
  }
  st_len = st_bs + a.G;
  for (int r = blockIdx.x * rows_per_cta + gi; r < a.nrows; r += gridDim.x * rows_per_cta)
    hash_row<LOG2T, NUMERIC, GRAM>(g, a, a.rows ? a.rows[r] : r, keys, vals, st_bs, st_len,
                                   st_a, nullptr, nullptr, nullptr);
}

template <int LOG2T, bool NUMERIC, bool GRAM>
__global__ void __launch_bounds__(1024) k_hash_cta(RowArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int T = 1 << LOG2T;
  const CtaGroup g;
  const int G = blockDim.x;
  unsigned char* p = smem;
  double* vals = (double*)p;
  if (NUMERIC) p += (size_t)T * 8;
  int* keys = (int*)p;
  p += (size_t)T * 4;
  double* st_a = (double*)p;
  if (NUMERIC) p += (size_t)G * 8;
  int* st_bs = (int*)p;
  int* st_len = st_bs + G;
  void* scratch = (void*)(p + (size_t)G * 8);
  uint32_t* rtmp = (uint32_t*)(p + (size_t)G * 8 + kCtaScratchBytes);
  int* rcnt = (int*)(rtmp + T);
  // in a persistent launch rows are drawn as CTAs free up (R-MAT 2^20 numeric
  // 8192-slot bin 26.5 -> 25.2 ms, 4096-slot 8.5 -> 8.1 ms against dealing
  // them out in turn)
  __shared__ int s_next;
  for (int it = 0;; ++it) {
    const int r = cta_item(a.queue, a.nrows, it, &s_next);
    if (r >= a.nrows) break;
    hash_row<LOG2T, NUMERIC, GRAM>(g, a, a.rows[r], keys, vals, st_bs, st_len, st_a, scratch,
                                   rtmp, rcnt);
  }
}

int hash_bin_lanes(int bin, int lanes_cfg) {
  const int lg = bin + kMinTableLog2 - 1;
  const int T = 1 << lg;
  if (lg == 11) return 32;      // warp per row (k_rows_w32.cu)
  if (lg >= 12) return T / 16;  // one row per CTA: 256 … 1024 threads
  int G = lanes_cfg > T / 8 ? lanes_cfg : T / 8;
  if (G > 32) G = 32;
  if (G > T) G = T;
  if (G < 1) G = 1;
  return G;
}

template <typename K>
static cudaError_t launch_kernel(K kernel, int threads, size_t smem, int nwork_ctas, int num_sms,
                                 const RowArgs& a, cudaStream_t s) {
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
  if (grid > nwork_ctas) grid = nwork_ctas;
  if (grid < 1) grid = 1;
  kernel<<<(unsigned)grid, threads, smem, s>>>(a);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

template <int LOG2T, bool NUMERIC, bool GRAM>
static cudaError_t launch_lg(const RowArgs& a, int num_sms, cudaStream_t s) {
  constexpr int T = 1 << LOG2T;
  if (LOG2T >= 11) {
    const int threads = T / 16;
    const size_t smem = row_group_bytes(T, threads, NUMERIC) + kCtaScratchBytes +
                        cta_radix_bytes<LOG2T, NUMERIC>();
    if (a.queue) {
      const cudaError_t e = cudaMemsetAsync(a.queue, 0, sizeof(int32_t), s);
      if (e != cudaSuccess) return e;
    }
    return launch_kernel(k_hash_cta<LOG2T, NUMERIC, GRAM>, threads, smem, a.nrows, num_sms, a, s);
  }
  const int G = a.G;
  const size_t per = row_group_bytes(T, G, NUMERIC);
  const int unit = 32 / G;  // rows per warp
  int rows = 256 / G;
  const size_t budget = 48 * 1024;
  int by_smem = (int)(budget / per);
  by_smem = (by_smem / unit) * unit;
  if (by_smem < unit) by_smem = unit;
  if (rows > by_smem) rows = by_smem;
  const int threads = rows * G;
  const size_t smem = per * rows;
  const int nwork = (a.nrows + rows - 1) / rows;
  return launch_kernel(k_hash_warp<LOG2T, NUMERIC, GRAM>, threads, smem, nwork, num_sms, a, s);
}

template <bool NUMERIC, bool GRAM>
static cudaError_t launch_mode(int bin, const RowArgs& a, int num_sms, cudaStream_t s) {
  switch (bin + kMinTableLog2 - 1) {
    case 4: return launch_lg<4, NUMERIC, GRAM>(a, num_sms, s);
    case 5: return launch_lg<5, NUMERIC, GRAM>(a, num_sms, s);
    case 6: return launch_lg<6, NUMERIC, GRAM>(a, num_sms, s);
    case 7: return launch_lg<7, NUMERIC, GRAM>(a, num_sms, s);
    case 8: return launch_lg<8, NUMERIC, GRAM>(a, num_sms, s);
    case 9: return launch_lg<9, NUMERIC, GRAM>(a, num_sms, s);
    case 10: return launch_lg<10, NUMERIC, GRAM>(a, num_sms, s);
    case 11: return launch_lg<11, NUMERIC, GRAM>(a, num_sms, s);
    case 12: return launch_lg<12, NUMERIC, GRAM>(a, num_sms, s);
    case 13: return launch_lg<13, NUMERIC, GRAM>(a, num_sms, s);
    case 14: return launch_lg<14, NUMERIC, GRAM>(a, num_sms, s);
  }
  return cudaErrorInvalidValue;
}

cudaError_t launch_hash_bin(int bin, bool numeric, bool gram, const RowArgs& a, int num_sms,
                            cudaStream_t s) {
  if (a.nrows <= 0) return cudaSuccess;
  const int lg = bin + kMinTableLog2 - 1;
  if (a.G == 32 && lg >= 6 && lg <= 11) return launch_hash_w32(lg, numeric, gram, a, num_sms, s);
  if (numeric) return gram ? launch_mode<true, true>(bin, a, num_sms, s)
                           : launch_mode<true, false>(bin, a, num_sms, s);
  return gram ? launch_mode<false, true>(bin, a, num_sms, s)
              : launch_mode<false, false>(bin, a, num_sms, s);
}

}  // namespace spg
