// spg_transpose_noalloc: the counting-sort transpose with all of its scratch in
// one static device array, for callers that cannot allocate device memory.
//
// Who needs it: applications that carve all GPU memory up front and forbid
// libraries from calling cudaMalloc/cudaFree (a serving process under a fixed
// memory budget, a host framework with its own arena whose accounting a
// hidden allocation would break), and callers on latency-critical paths where
// an allocation may synchronise the device.  They pass inputs and outputs; the
// call itself allocates nothing.
//
// The scratch (status word, column counts, cursors, scan partials, staging
// copy of the entries, long-segment list) is g_noalloc_scratch below: about
// 6.8 MB held by every GPU that loads the library until the process exits.
// It bounds the input to n <= kNoAllocMaxN rows and nnz <= kNoAllocMaxNnz.
// The call runs on the current device; A and the outputs must live there.
// The array's device address is resolved once per device and kept, so the
// library must not be used across a cudaDeviceReset of that device.
#include <cstdio>
#include <mutex>

#include "kernels.h"

namespace {

constexpr int32_t kNoAllocMaxN = 65536;
constexpr int64_t kNoAllocMaxNnz = 524288;

constexpr size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kScanBytes = 8 * ((kNoAllocMaxN + 4095) / 4096 + 1);
constexpr size_t kOffStatus = 0;
constexpr size_t kOffCnt = 256;
constexpr size_t kOffCursor = kOffCnt + align256(4 * (size_t)kNoAllocMaxN);
constexpr size_t kOffScan = kOffCursor + align256(4 * (size_t)kNoAllocMaxN);
constexpr size_t kOffTmpCol = kOffScan + align256(kScanBytes);
constexpr size_t kOffTmpVal = kOffTmpCol + align256(4 * (size_t)kNoAllocMaxNnz);
constexpr size_t kOffLongList = kOffTmpVal + align256(8 * (size_t)kNoAllocMaxNnz);
constexpr size_t kOffLongCount = kOffLongList + align256(4 * (size_t)kNoAllocMaxN);
constexpr size_t kScratchBytes = kOffLongCount + 256;

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_scratch_addr[kMaxDevices] = {};

}  // namespace

// The scratch array.  Host code must not use this name as a device address:
// the address comes from cudaGetSymbolAddress (scratch_for_current_device).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

namespace {

// Set-up, once per device, with that device current: resolve the device
// address of g_noalloc_scratch and keep it for later calls.
spg_status scratch_for_current_device(unsigned char** out, int* num_sms) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return spg::set_error(SPG_ERR_CUDA, "cudaGetDevice: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return spg::set_error(SPG_ERR_UNSUPPORTED, "device ordinal %d beyond %d", dev, kMaxDevices);
  e = cudaDeviceGetAttribute(num_sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess)
    return spg::set_error(SPG_ERR_CUDA, "device attribute: %s", cudaGetErrorString(e));
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return spg::set_error(SPG_ERR_CUDA, "cudaGetSymbolAddress(scratch): %s",
                            cudaGetErrorString(e));
    g_scratch_addr[dev] = (unsigned char*)p;
  }
  *out = g_scratch_addr[dev];
  return SPG_OK;
}

// A device pointer that belongs to another GPU than the current one: the call
// would run its kernels (and its scratch) on the current device and reach the
// buffer through peer access.  Host, managed and unregistered pointers pass.
bool on_other_device(const void* p, int dev) {
  if (!p) return false;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice && at.device != dev;
}

}  // namespace

extern "C" spg_status spg_transpose_noalloc(const spg_csr_dev* A, int32_t* t_rowptr,
                                            int32_t* t_col, double* t_val, void* stream) {
  using spg::set_error;
  spg::clear_error();
  if (!A || A->n < 0 || A->nnz < 0 || !A->rowptr || (A->nnz > 0 && (!A->col || !A->val)))
    return set_error(SPG_ERR_INVALID_ARG, "null or negative input matrix");
  if (!t_rowptr || (A->nnz > 0 && (!t_col || !t_val)))
    return set_error(SPG_ERR_INVALID_ARG, "null output arrays");
  if (A->n > kNoAllocMaxN || A->nnz > kNoAllocMaxNnz)
    return set_error(SPG_ERR_UNSUPPORTED,
                     "spg_transpose_noalloc takes n <= %d and nnz <= %lld (its static scratch is "
                     "%zu bytes); got n = %d, nnz = %lld — use spg_transpose",
                     kNoAllocMaxN, (long long)kNoAllocMaxNnz, kScratchBytes, A->n,
                     (long long)A->nnz);
  if (spg::scan_tmp_bytes(A->n) > kScanBytes)
    return set_error(SPG_ERR_UNSUPPORTED, "scan partials exceed the static scratch");
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) return set_error(SPG_ERR_CUDA, "no current device");
  if (on_other_device(A->rowptr, cur) || on_other_device(A->col, cur) ||
      on_other_device(A->val, cur) || on_other_device(t_rowptr, cur) ||
      on_other_device(t_col, cur) || on_other_device(t_val, cur))
    return set_error(SPG_ERR_INVALID_ARG,
                     "spg_transpose_noalloc runs on the current device (%d); an input or output "
                     "buffer lives on another GPU", cur);
  unsigned char* s = nullptr;
  int num_sms = 0;
  spg_status st = scratch_for_current_device(&s, &num_sms);
  if (st != SPG_OK) return st;

  cudaStream_t cs = (cudaStream_t)stream;
  uint32_t* status = (uint32_t*)(s + kOffStatus);
  const spg::MatView Av{A->n, A->nnz, A->rowptr, A->col, A->val};
  // validate first (the transpose indexes by column), verdict into a host word
  uint32_t bits = 0;
  cudaError_t e = cudaMemsetAsync(status, 0, sizeof(uint32_t), cs);
  if (e == cudaSuccess) e = spg::launch_validate(Av, status, cs);
  if (e == cudaSuccess) e = cudaMemcpyAsync(&bits, status, sizeof(uint32_t), cudaMemcpyDeviceToHost, cs);
  if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
  if (e != cudaSuccess) return set_error(SPG_ERR_CUDA, "validate: %s", cudaGetErrorString(e));
  if (bits & spg::DEV_ERR_INVALID_CSR)
    return set_error(SPG_ERR_INVALID_CSR,
                     "input CSR invalid: rowptr must start at 0, be monotone and end at nnz; "
                     "columns must lie in [0,n) and strictly increase within each row");

  spg::TransposeWork w{};
  w.cnt = (int32_t*)(s + kOffCnt);          // zeroed by launch_transpose
  w.cursor = (int32_t*)(s + kOffCursor);    // zeroed by launch_transpose
  w.scan_tmp = (void*)(s + kOffScan);
  w.tmp_col = (int32_t*)(s + kOffTmpCol);
  w.tmp_val = (double*)(s + kOffTmpVal);
  w.long_list = (int32_t*)(s + kOffLongList);
  w.long_count = (int32_t*)(s + kOffLongCount);  // zeroed by launch_segsort
  w.status = status;
  e = spg::launch_transpose(Av, t_rowptr, t_col, t_val, w, num_sms, cs);
  if (e != cudaSuccess) return set_error(SPG_ERR_CUDA, "transpose: %s", cudaGetErrorString(e));
  return SPG_OK;
}
