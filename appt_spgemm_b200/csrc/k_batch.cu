// Batched products: many independent square CSR matrices laid out as one
// block-diagonal matrix, so that every phase of the engine (validation,
// pre-pass, binning, symbolic, numeric) runs once over a row queue shared by
// all instances instead of once per instance.  Instance b occupies rows and
// columns [row_off[b], row_off[b+1]) and entries [nnz_off[b], nnz_off[b+1]).
#include "kernels.h"

namespace spg {

constexpr int kBatchSmemTable = 2048;  // instances whose offsets are staged in shared memory

// index b with off[b] <= x < off[b+1] (off ascending, off[0] = 0)
__device__ __forceinline__ int find_instance(const int64_t* off, int count, int64_t x) {
  int lo = 0, hi = count - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= x) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__global__ void k_batch_rows(const BatchDesc* __restrict__ d, const int64_t* __restrict__ row_off,
                             int count, int32_t* __restrict__ rowptr, int32_t* __restrict__ colbase,
                             int64_t N, int64_t NNZ, uint32_t* bad) {
  __shared__ int64_t s_off[kBatchSmemTable + 1];
  const bool staged = count <= kBatchSmemTable;
  if (staged)
    for (int i = threadIdx.x; i <= count; i += blockDim.x) s_off[i] = row_off[i];
  __syncthreads();
  const int64_t* off = staged ? s_off : row_off;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r <= N; r += stride) {
    if (r == N) {
      rowptr[N] = (int32_t)NNZ;
      continue;
    }
    const int b = find_instance(off, count, r);
    const BatchDesc& D = d[b];
    const int64_t i = r - off[b];
    rowptr[r] = (int32_t)(D.rowptr[i] + D.nnz_off);
    colbase[r] = (int32_t)off[b];
    // each instance's own row pointers must start at 0 and end at its nnz
    if (i == 0 && D.rowptr[0] != 0) atomicOr(bad, 1u);
    if (i == D.n - 1 && (int64_t)D.rowptr[D.n] != D.nnz) atomicOr(bad, 1u);
  }
}

__global__ void k_batch_entries(const BatchDesc* __restrict__ d, const int64_t* __restrict__ nnz_off,
                                int count, int32_t* __restrict__ col, double* __restrict__ val,
                                int64_t NNZ, uint32_t* bad) {
  __shared__ int64_t s_off[kBatchSmemTable + 1];
  const bool staged = count <= kBatchSmemTable;
  if (staged)
    for (int i = threadIdx.x; i <= count; i += blockDim.x) s_off[i] = nnz_off[i];
  __syncthreads();
  const int64_t* off = staged ? s_off : nnz_off;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < NNZ; p += stride) {
    const int b = find_instance(off, count, p);
    const BatchDesc& D = d[b];
    const int64_t q = p - off[b];
    const int32_t c = D.col[q];
    // a column outside its own block would silently leak into another instance
    if (c < 0 || c >= D.n) atomicOr(bad, 1u);
    col[p] = c + (int32_t)D.row_off;
    val[p] = D.val[q];
  }
}

cudaError_t launch_batch_concat(const BatchDesc* d, const int64_t* row_off, const int64_t* nnz_off,
                                int count, int64_t N, int64_t NNZ, int32_t* rowptr, int32_t* col,
                                double* val, int32_t* colbase, uint32_t* bad, int num_sms,
                                cudaStream_t s) {
  int64_t blocks = (N + 1 + 255) / 256;
  if (blocks > (int64_t)num_sms * 16) blocks = (int64_t)num_sms * 16;
  k_batch_rows<<<(unsigned)blocks, 256, 0, s>>>(d, row_off, count, rowptr, colbase, N, NNZ, bad);
  SPG_COUNT_LAUNCH();
  if (NNZ > 0) {
    blocks = (NNZ + 255) / 256;
    if (blocks > (int64_t)num_sms * 32) blocks = (int64_t)num_sms * 32;
    k_batch_entries<<<(unsigned)blocks, 256, 0, s>>>(d, nnz_off, count, col, val, NNZ, bad);
    SPG_COUNT_LAUNCH();
  }
  return cudaGetLastError();
}

// Values only (the structure is fixed by the plan): big val[p] = instance val.
__global__ void k_batch_vals(const BatchDesc* __restrict__ d, const int64_t* __restrict__ nnz_off,
                             int count, double* __restrict__ val, int64_t NNZ) {
  __shared__ int64_t s_off[kBatchSmemTable + 1];
  const bool staged = count <= kBatchSmemTable;
  if (staged)
    for (int i = threadIdx.x; i <= count; i += blockDim.x) s_off[i] = nnz_off[i];
  __syncthreads();
  const int64_t* off = staged ? s_off : nnz_off;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; p < NNZ; p += stride) {
    const int b = find_instance(off, count, p);
    val[p] = d[b].val[p - off[b]];
  }
}

cudaError_t launch_batch_vals(const BatchDesc* d, const int64_t* nnz_off, int count, int64_t NNZ,
                              double* val, int num_sms, cudaStream_t s) {
  if (NNZ == 0) return cudaSuccess;
  int64_t blocks = (NNZ + 255) / 256;
  if (blocks > (int64_t)num_sms * 32) blocks = (int64_t)num_sms * 32;
  k_batch_vals<<<(unsigned)blocks, 256, 0, s>>>(d, nnz_off, count, val, NNZ);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

__global__ void k_gather_offsets(const int64_t* __restrict__ rowptr_c,
                                 const int64_t* __restrict__ row_off, int count,
                                 int64_t* __restrict__ out) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b <= count; b += gridDim.x * blockDim.x)
    out[b] = rowptr_c[row_off[b]];
}

cudaError_t launch_gather_offsets(const int64_t* rowptr_c, const int64_t* row_off, int count,
                                  int64_t* out, cudaStream_t s) {
  k_gather_offsets<<<(count + 256) / 256, 256, 0, s>>>(rowptr_c, row_off, count, out);
  SPG_COUNT_LAUNCH();
  return cudaGetLastError();
}

}  // namespace spg
