// spgemm_b200 <tag> <bin.csr> <AA|AAt|AAtS> [reps]
//
// Command-line twin of the engine, built on the C ABI.  Same arguments and
// stdout protocol as the reference CLI (src/spgemm.cu:128-131, :223-224):
//   "  __chk s=%.6e as=%.6e sq=%.6e"
//   "RESULT,<tag>,<task>,<n>,<nnz>,<C_nnz>,<ms>"
// so the reference's sweep drivers (parse() in bench/run_compare.py:30-40)
// read its output unchanged.  Errors print one line to stderr and exit 1.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>

#include "../../include/spgemm_b200.h"

static int fail(const char* what) {
  std::fprintf(stderr, "spgemm_b200: %s: %s\n", what, spg_last_error_string());
  return 1;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <tag> <bin.csr> <AA|AAt|AAtS> [reps]\n", argv[0]);
    return 1;
  }
  const char* tag = argv[1];
  const char* task = argv[3];
  const int reps = argc > 4 ? std::atoi(argv[4]) : 20;
  spg_host_csr h{};
  if (spg_csr1_read(argv[2], &h) != SPG_OK) return fail("read");
  int32_t *dOff = nullptr, *dCol = nullptr;
  double* dVal = nullptr;
  const size_t nz = (size_t)(h.nnz > 0 ? h.nnz : 1);
  if (cudaMalloc(&dOff, sizeof(int32_t) * ((size_t)h.n + 1)) != cudaSuccess ||
      cudaMalloc(&dCol, sizeof(int32_t) * nz) != cudaSuccess ||
      cudaMalloc(&dVal, sizeof(double) * nz) != cudaSuccess) {
    std::fprintf(stderr, "spgemm_b200: device allocation failed\n");
    return 1;
  }
  cudaMemcpy(dOff, h.rowptr, sizeof(int32_t) * ((size_t)h.n + 1), cudaMemcpyHostToDevice);
  if (h.nnz > 0) {
    cudaMemcpy(dCol, h.col, sizeof(int32_t) * (size_t)h.nnz, cudaMemcpyHostToDevice);
    cudaMemcpy(dVal, h.val, sizeof(double) * (size_t)h.nnz, cudaMemcpyHostToDevice);
  }
  spg_eng_result r{};
  if (spg_run_ours(task, dOff, dCol, dVal, h.n, h.nnz, reps, &r) != SPG_OK) return fail("run");
  std::printf("  __chk s=%.6e as=%.6e sq=%.6e\n", r.s, r.as, r.sq);
  std::printf("RESULT,%s,%s,%d,%lld,%lld,%.4f\n", tag, task, h.n, (long long)h.nnz,
              (long long)r.nnz, r.ms);
  cudaFree(dOff);
  cudaFree(dCol);
  cudaFree(dVal);
  spg_host_csr_free(&h);
  return 0;
}
