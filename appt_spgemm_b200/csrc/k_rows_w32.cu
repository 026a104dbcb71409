// Warp-per-row shared-memory hash kernels (32 lanes per row, tables of 64 to
// 2048 slots): the path almost every row of banded / FEM-like matrices and of
// sparse random graphs takes.
//
// Per row the warp
//  - holds up to 32 entries of A's row in registers (k, a_ik, B-row bounds)
//    and walks them in order as 32-wide segments of B rows, loading a group of
//    D segments before hashing any of them (a branch-light fast path when
//    every B row of the chunk fits one segment);
//  - inserts keys with a CAS-first linear probe; in the numeric phase the
//    lane that claims a slot stores 0.0 + a·b there and later segments add
//    to it, one __syncwarp per segment keeping the k order of every sum (so
//    no value array is cleared per row);
//  - packs each occupied slot as ((col − lo) << log2T) | slot, sorts the
//    packed words with a register bitonic network (E words per lane), and
//    writes columns and the gathered values to the row's CSR slots; rows of
//    more than 256 entries in tables of 512 slots and up sort the packed words
//    with a stable LSD radix sort over the column bits instead, O(m) per
//    digit rather than the bitonic network's O(m log² m), in the table's own
//    free space.
// Rows whose column span does not fit the packing take the shared-memory
// pair sort.
#include <climits>

#include "kernels.h"

namespace spg {

namespace {

constexpr unsigned kFull = 0xffffffffu;
// Rows of more entries than this sort with the radix sort rather than the
// register bitonic network (8 words per lane up to 256 entries): measured on
// the 512-matrix batch, a threshold of 256 against 128 gave 94.5–94.9 against
// 95.5–96.7 ms, R-MAT 2^18 unchanged.
constexpr int kRadixMin = 256;

// Shared memory of one warp's row: the table's values (numeric) and keys.
template <int LOG2T, bool NUMERIC>
__host__ __device__ constexpr size_t w32_warp_bytes() {
  return NUMERIC ? ((size_t)12 << LOG2T) : ((size_t)4 << LOG2T);
}

// Sorted write-out through packed keys held E per lane in registers.
template <int E, int LOG2T, bool GRAM>
__device__ __forceinline__ void sort_write(const RowArgs& a, int row, int lo, int m, int* keys,
                                          const double* vals, int64_t base) {
  const int lane = threadIdx.x & 31;
  uint32_t r[E];
  // blocked layout, loaded and stored with vector accesses (conflict-free)
  uint32_t* kw = (uint32_t*)keys + lane * E;
  if (E >= 4) {
#pragma unroll
    for (int c = 0; c < E / 4; ++c) {
      const uint4 v = ((const uint4*)kw)[c];
      r[4 * c] = v.x;
      r[4 * c + 1] = v.y;
      r[4 * c + 2] = v.z;
      r[4 * c + 3] = v.w;
    }
  } else if (E == 2) {
    const uint2 v = *(const uint2*)kw;
    r[0] = v.x;
    r[E - 1] = v.y;
  } else {
    r[0] = kw[0];
  }
#pragma unroll
  for (int i = 0; i < E; ++i)
    if (lane * E + i >= m) r[i] = 0xffffffffu;
  warp_bitonic_sort<E>(r);
  __syncwarp();
  if (E >= 4) {
#pragma unroll
    for (int c = 0; c < E / 4; ++c)
      ((uint4*)kw)[c] = make_uint4(r[4 * c], r[4 * c + 1], r[4 * c + 2], r[4 * c + 3]);
  } else if (E == 2) {
    *(uint2*)kw = make_uint2(r[0], r[E - 1]);
  } else {
    kw[0] = r[0];
  }
  __syncwarp();
  emit_packed<LOG2T, GRAM>(a, row, lo, m, (const uint32_t*)keys, vals, base, lane, 32);
}

// Fallback: compact (key, value) pairs in slot order and bitonic-sort them in
// shared memory (for rows whose column span exceeds the 32-bit packing).
template <int LOG2T, bool GRAM>
__device__ __noinline__ void pair_sort_write(const RowArgs& a, int row, int* keys, double* vals,
                                             int64_t base, int expect) {
  constexpr int T = 1 << LOG2T;
  const int lane = threadIdx.x & 31;
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
      keys[pos] = key;
      vals[pos] = v;
    }
    m += __popc(bal);
    __syncwarp();
  }
  const int P = next_pow2_int(m);
  for (int s = m + lane; s < P; s += 32) keys[s] = INT_MAX;
  __syncwarp();
  bitonic_sort_pairs(WarpGroup(32), keys, vals, P);
  if (m > expect) m = expect;
  const int cb = a.colbase ? a.colbase[row] : 0;
  for (int t = lane; t < m; t += 32) {
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
}

}  // namespace

// Five CTAs of 256 threads per SM (48 registers, no spills).  Measured on the
// 96³ stencil step: six for the symbolic kernel (40 registers) 2.28 against
// 2.29 ms; six for both, or six with a prefetch depth of two numeric B rows,
// numeric 5.77 / 5.81 against 5.66 ms; eight (32 registers, spills) 6.09 ms.
template <int LOG2T, bool NUMERIC, bool GRAM>
__global__ void __launch_bounds__(256, 5) k_hash_w32(RowArgs a) {
  extern __shared__ __align__(16) unsigned char smem[];
  constexpr int T = 1 << LOG2T;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
  // rows of more than kRadixMin entries in tables of 512 slots and up take the
  // radix sort, with DBITS-bit digits whose counters fit the table's free tail
  // (in the 256-slot kernel, the stencil's, the radix code alone cost 3.7%)
  constexpr bool RADIX = NUMERIC && LOG2T >= 9;
  constexpr int DBITS = LOG2T == 9 ? 7 : 8;
  unsigned char* base_p = smem + (size_t)w * w32_warp_bytes<LOG2T, NUMERIC>();
  double* vals = (double*)base_p;
  int* keys = (int*)(base_p + (NUMERIC ? (size_t)T * 8 : 0));

  for (int r = blockIdx.x * nw + w; r < a.nrows; r += gridDim.x * nw) {
    const int row = a.rows ? a.rows[r] : r;
    if (!NUMERIC && a.fsmall) {
      const int64_t fr = a.fsmall[row];
      if (fr < 0 || fr > a.fcap) {
        if (lane == 0) {
          if (fr > a.fcap) report(a.status, DEV_ERR_SMALL_CAP);
          a.rownnz[row] = 0;
          if (GRAM) a.rowlow[row] = 0;
        }
        continue;
      }
    }
    // (a table sized per row to its products here, at 75% or 50% load, measured
    // slower on random-graph rows, whose products are nearly all distinct: 512
    // plain calls of the batch mix 224 / 204 ms against 191 ms)
    for (int s = lane * 4; s < T; s += 128) *(int4*)(keys + s) = make_int4(-1, -1, -1, -1);
    __syncwarp();
    const int32_t ps = a.A.rowptr[row], pe = a.A.rowptr[row + 1];
    for (int32_t pb = ps; pb < pe; pb += 32) {
      const int cnt = min(32, pe - pb);
      int bs = 0, len = 0;
      double av = 0.0;
      if (lane < cnt) {
        const int32_t k = a.A.col[pb + lane];
        bs = a.B.rowptr[k];
        len = a.B.rowptr[k + 1] - bs;
        if (NUMERIC) av = a.A.val[pb + lane];
      }
      // B rows loaded ahead of the hashing: 3 (numeric) and 4 (symbolic) measured
      // best on the 96³ stencil step and the 512-batch (numeric 2 / 4 / 6: 5.82 /
      // 5.71 / 6.67 ms per step against 5.64; symbolic 2 / 3 / 8 / 16: 2.28 /
      // 2.08 / 2.14 / 2.23 against 2.05): deeper staging costs registers and
      // instructions in kernels that are issue-bound, not load-latency-bound
      constexpr int D = NUMERIC ? 3 : 4;
      if (__all_sync(kFull, len <= 32)) {
        // Fast path: every B row of the chunk is one 32-wide segment.  Rows
        // t0..t0+D−1 are loaded together, then hashed in order.
        for (int t0 = 0; t0 < cnt; t0 += D) {
          int jr[D];
          double br[D], ar[D];
#pragma unroll
          for (int d = 0; d < D; ++d) {
            const int t = t0 + d;
            const int tb = __shfl_sync(kFull, bs, t & 31);
            const int tl = __shfl_sync(kFull, len, t & 31);
            ar[d] = NUMERIC ? __shfl_sync(kFull, av, t & 31) : 0.0;
            const bool on = t < cnt && lane < tl;
            jr[d] = on ? a.B.col[tb + lane] : -1;
            br[d] = (NUMERIC && on) ? a.B.val[tb + lane] : 0.0;
          }
#pragma unroll
          for (int d = 0; d < D; ++d) {
            const int j = jr[d];
            if (j >= 0 && !(NUMERIC && GRAM && j < row)) {
              insert_acc<LOG2T, NUMERIC>(keys, vals, j, NUMERIC ? __dmul_rn(ar[d], br[d]) : 0.0,
                                         a.status);
            }
            if (NUMERIC) __syncwarp();  // k-order of the accumulation
          }
        }
        continue;
      }
      // General path: walk 32-wide segments (t, q0) of B row t in order, D at
      // a time; the loads of a group are issued before any of it is hashed.
      int t = 0, q0 = 0;
      int sbs = __shfl_sync(kFull, bs, 0), slen = __shfl_sync(kFull, len, 0);
      double sa = NUMERIC ? __shfl_sync(kFull, av, 0) : 0.0;
      while (t < cnt && q0 >= slen) {
        ++t;
        if (t < cnt) {
          sbs = __shfl_sync(kFull, bs, t);
          slen = __shfl_sync(kFull, len, t);
          if (NUMERIC) sa = __shfl_sync(kFull, av, t);
        }
      }
      while (t < cnt) {
        int jr[D];
        double br[D], ar[D];
#pragma unroll
        for (int d = 0; d < D; ++d) {
          jr[d] = -1;
          br[d] = 0.0;
          ar[d] = sa;
          if (t < cnt) {
            if (q0 + lane < slen) {
              jr[d] = a.B.col[sbs + q0 + lane];
              if (NUMERIC) br[d] = a.B.val[sbs + q0 + lane];
            }
            q0 += 32;
            while (t < cnt && q0 >= slen) {
              ++t;
              q0 = 0;
              if (t < cnt) {
                sbs = __shfl_sync(kFull, bs, t);
                slen = __shfl_sync(kFull, len, t);
                if (NUMERIC) sa = __shfl_sync(kFull, av, t);
              }
            }
          }
        }
#pragma unroll
        for (int d = 0; d < D; ++d) {
          const int j = jr[d];
          if (j >= 0 && !(NUMERIC && GRAM && j < row)) {
            insert_acc<LOG2T, NUMERIC>(keys, vals, j, NUMERIC ? __dmul_rn(ar[d], br[d]) : 0.0,
                                       a.status);
          }
          if (NUMERIC) __syncwarp();  // k-order of the accumulation
        }
      }
    }
    __syncwarp();

    if (!NUMERIC) {
      int c = 0, cl = 0;
      for (int s = lane * 4; s < T; s += 128) {
        const int4 k4 = *(const int4*)(keys + s);
        c += (k4.x != kEmptyKey) + (k4.y != kEmptyKey) + (k4.z != kEmptyKey) + (k4.w != kEmptyKey);
        if (GRAM)
          cl += (k4.x != kEmptyKey && k4.x < row) + (k4.y != kEmptyKey && k4.y < row) +
                (k4.z != kEmptyKey && k4.z < row) + (k4.w != kEmptyKey && k4.w < row);
      }
      for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(kFull, c, o);
        if (GRAM) cl += __shfl_xor_sync(kFull, cl, o);
      }
      if (lane == 0) {
        a.rownnz[row] = c;
        if (GRAM) a.rowlow[row] = cl;
      }
      __syncwarp();
      continue;
    }

    const int32_t low = GRAM ? a.low_in[row] : 0;
    const int expect = a.cnt_in[row] - low;
    const int64_t base = a.rowptr[row] + low;
    const int lo = a.lo[row];
    const bool packs = (int64_t)a.hi[row] - lo < ((int64_t)1 << (32 - LOG2T));
    // Radix rows compact (packed word, value) pairs to the front of keys /
    // vals; the sort's second buffer (m words) then lives in vals[m..T) and
    // its 2^DBITS counters in keys[m..T), which needs 3m <= 2T and
    // m + 2^DBITS <= T (true up to a 66% table load).
    const bool radix = RADIX && packs && expect > kRadixMin && 3 * expect <= 2 * T &&
                       expect + (1 << DBITS) <= T;
    if (!packs || (expect > 256 && !radix)) {
      pair_sort_write<LOG2T, GRAM>(a, row, keys, vals, base, expect);
      __syncwarp();
      continue;
    }
    // compact occupied slots as packed words ((col − lo) << LOG2T | index of
    // the value: its slot, or for radix rows its compacted position), in place
    int m = 0;
    for (int c = 0; c < T; c += 32) {
      const int s = c + lane;
      const int key = keys[s];
      const double v = radix ? vals[s] : 0.0;
      const bool occ = key != kEmptyKey;
      const unsigned bal = __ballot_sync(kFull, occ);
      const int pos = m + __popc(bal & lanemask_lt());
      __syncwarp();
      if (occ) {
        keys[pos] = (int)(((uint32_t)(key - lo) << LOG2T) | (uint32_t)(radix ? pos : s));
        if (radix) vals[pos] = v;
      }
      m += __popc(bal);
      __syncwarp();
    }
    if (m != expect && lane == 0) report(a.status, DEV_ERR_OVERFLOW);
    if (m > expect) m = expect;
    if (radix) {
      const uint32_t* sorted = radix_sort_words<1, DBITS>(
          (uint32_t*)keys, (uint32_t*)(vals + m), m, LOG2T, span_bits(lo, a.hi[row]), keys + m,
          nullptr);
      emit_packed<LOG2T, GRAM>(a, row, lo, m, sorted, vals, base, lane, 32);
      __syncwarp();
      continue;
    }
    const int P = next_pow2_int(m);
    if (P <= 32) sort_write<1, LOG2T, GRAM>(a, row, lo, m, keys, vals, base);
    else if (P <= 64) sort_write<2, LOG2T, GRAM>(a, row, lo, m, keys, vals, base);
    else if (P <= 128) sort_write<4, LOG2T, GRAM>(a, row, lo, m, keys, vals, base);
    else sort_write<8, LOG2T, GRAM>(a, row, lo, m, keys, vals, base);
    __syncwarp();
  }
}

template <int LOG2T, bool NUMERIC, bool GRAM>
static cudaError_t launch_w32(const RowArgs& a, int num_sms, cudaStream_t s) {
  auto kernel = k_hash_w32<LOG2T, NUMERIC, GRAM>;
  const size_t per = w32_warp_bytes<LOG2T, NUMERIC>();
  int rows = 8;  // warps (rows) per CTA
  while (rows > 1 && per * rows > 64 * 1024) rows >>= 1;
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

template <bool NUMERIC, bool GRAM>
static cudaError_t w32_mode(int log2t, const RowArgs& a, int num_sms, cudaStream_t s) {
  switch (log2t) {
    case 6: return launch_w32<6, NUMERIC, GRAM>(a, num_sms, s);
    case 7: return launch_w32<7, NUMERIC, GRAM>(a, num_sms, s);
    case 8: return launch_w32<8, NUMERIC, GRAM>(a, num_sms, s);
    case 9: return launch_w32<9, NUMERIC, GRAM>(a, num_sms, s);
    case 10: return launch_w32<10, NUMERIC, GRAM>(a, num_sms, s);
    case 11: return launch_w32<11, NUMERIC, GRAM>(a, num_sms, s);
  }
  return cudaErrorNotSupported;
}

cudaError_t launch_hash_w32(int log2t, bool numeric, bool gram, const RowArgs& a, int num_sms,
                            cudaStream_t s) {
  if (a.nrows <= 0) return cudaSuccess;
  if (numeric) return gram ? w32_mode<true, true>(log2t, a, num_sms, s)
                           : w32_mode<true, false>(log2t, a, num_sms, s);
  return gram ? w32_mode<false, true>(log2t, a, num_sms, s)
              : w32_mode<false, false>(log2t, a, num_sms, s);
}

}  // namespace spg
