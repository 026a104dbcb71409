// Numeric-zero compaction of a finished product: drop the entries whose value
// is exactly zero (+0.0 or −0.0) and keep the others in order, so the result
// has the pattern scipy's eliminate_zeros() leaves (the engine itself keeps
// cancelled entries, as the reference and cuSPARSE do:
// report/CORRECTNESS_NOTES.md:3-16).
//
// The host drives it in row chunks (spg_drop_zeros in engine.cu): per chunk
// the kept entries are gathered into a bounded temporary buffer and copied to
// their final place; every entry only moves towards the front, and a chunk's
// reads finish before its writes, so C is compacted in place whatever its size.
#include "kernels.h"

namespace spg {

namespace {

constexpr unsigned kFull = 0xffffffffu;

// Warp per row: kept entries of the row.
__global__ void k_count_kept(const int64_t* __restrict__ rowptr, const double* __restrict__ val,
                             int32_t n, int32_t* __restrict__ kept) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t i = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < n; i += warps) {
    const int64_t b = rowptr[i], e = rowptr[i + 1];
    int c = 0;
    for (int64_t p = b + lane; p < e; p += 32) c += val[p] != 0.0;
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(kFull, c, o);
    if (lane == 0) kept[i] = c;
  }
}

// Warp per row of [r0, r1): the row's kept entries, in order, to
// tmp[newptr[row] − newptr[r0] …].
__global__ void k_gather_kept(const int64_t* __restrict__ rowptr, const int32_t* __restrict__ col,
                              const double* __restrict__ val, const int64_t* __restrict__ newptr,
                              int32_t r0, int32_t r1, int32_t* __restrict__ tcol,
                              double* __restrict__ tval) {
  const int lane = threadIdx.x & 31;
  const int64_t warps = (int64_t)gridDim.x * (blockDim.x >> 5);
  const int64_t base = newptr[r0];
  for (int64_t i = r0 + (((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5); i < r1;
       i += warps) {
    const int64_t b = rowptr[i], e = rowptr[i + 1];
    int64_t out = newptr[i] - base;
    for (int64_t p0 = b; p0 < e; p0 += 32) {
      const int64_t p = p0 + lane;
      const double v = p < e ? val[p] : 0.0;
      const bool keep = p < e && v != 0.0;
      const unsigned bal = __ballot_sync(kFull, keep);
      if (keep) {
        const int64_t d = out + __popc(bal & lanemask_lt());
        tcol[d] = col[p];
        tval[d] = v;
      }
      out += __popc(bal);
    }
  }
}

unsigned row_grid(int64_t rows) {
  const int64_t g = (rows + 7) / 8;  // 8 warps per CTA
  return (unsigned)(g < 1 ? 1 : (g > 65535 ? 65535 : g));
}

}  // namespace

cudaError_t launch_count_kept(const int64_t* rowptr, const double* val, int32_t n, int32_t* kept,
                              cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  k_count_kept<<<row_grid(n), 256, 0, s>>>(rowptr, val, n, kept);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

cudaError_t launch_gather_kept(const int64_t* rowptr, const int32_t* col, const double* val,
                               const int64_t* newptr, int32_t r0, int32_t r1, int32_t* tcol,
                               double* tval, cudaStream_t s) {
  if (r1 <= r0) return cudaSuccess;
  k_gather_kept<<<row_grid(r1 - r0), 256, 0, s>>>(rowptr, col, val, newptr, r0, r1, tcol, tval);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace spg
