// spgemm_b200 <tag> <bin.csr> <AA|AAt|AAtS> [reps]
//
// Command-line twin of the engine, built on the C ABI.  Same arguments and
// stdout protocol as the reference CLI (src/spgemm.cu:128-131, :223-224):
//   "  __chk s=%.6e as=%.6e sq=%.6e"
//   "RESULT,<tag>,<task>,<n>,<nnz>,<C_nnz>,<ms>"
// so the reference's sweep drivers (parse() in bench/run_compare.py:30-40)
// read its output unchanged.  Errors print one line to stderr and exit 1; an
// unknown task is one of them, found before the device is touched (the
// reference computes A·A for any task other than AAt and AAtS,
// src/spgemm.cu:131-132).
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "../../include/spgemm_b200.h"

static int fail(const char* what) {
  std::fprintf(stderr, "spgemm_b200: %s: %s\n", what, spg_last_error_string());
  return 1;
}

static int run(const char* tag, const char* task, int reps, const spg_host_csr& h) {
  int32_t *dOff = nullptr, *dCol = nullptr;
  double* dVal = nullptr;
  const size_t nz = (size_t)(h.nnz > 0 ? h.nnz : 1);
  int rc = 1;
  if (cudaMalloc(&dOff, sizeof(int32_t) * ((size_t)h.n + 1)) != cudaSuccess ||
      cudaMalloc(&dCol, sizeof(int32_t) * nz) != cudaSuccess ||
      cudaMalloc(&dVal, sizeof(double) * nz) != cudaSuccess) {
    std::fprintf(stderr, "spgemm_b200: device allocation failed\n");
  } else if (cudaMemcpy(dOff, h.rowptr, sizeof(int32_t) * ((size_t)h.n + 1),
                        cudaMemcpyHostToDevice) != cudaSuccess ||
             (h.nnz > 0 &&
              (cudaMemcpy(dCol, h.col, sizeof(int32_t) * (size_t)h.nnz,
                          cudaMemcpyHostToDevice) != cudaSuccess ||
               cudaMemcpy(dVal, h.val, sizeof(double) * (size_t)h.nnz,
                          cudaMemcpyHostToDevice) != cudaSuccess))) {
    std::fprintf(stderr, "spgemm_b200: copy to the device failed\n");
  } else {
    spg_eng_result r{};
    if (spg_run_ours(task, dOff, dCol, dVal, h.n, h.nnz, reps, &r) != SPG_OK) {
      fail("run");
    } else {
      std::printf("  __chk s=%.6e as=%.6e sq=%.6e\n", r.s, r.as, r.sq);
      std::printf("RESULT,%s,%s,%d,%lld,%lld,%.4f\n", tag, task, h.n, (long long)h.nnz,
                  (long long)r.nnz, r.ms);
      rc = 0;
    }
  }
  cudaFree(dOff);
  cudaFree(dCol);
  cudaFree(dVal);
  return rc;
}

int main(int argc, char** argv) {
  if (argc < 4) {
    std::fprintf(stderr, "usage: %s <tag> <bin.csr> <AA|AAt|AAtS> [reps]\n", argv[0]);
    return 1;
  }
  const char* tag = argv[1];
  const char* task = argv[3];
  const int reps = argc > 4 ? std::atoi(argv[4]) : 20;
  if (std::strcmp(task, "AA") != 0 && std::strcmp(task, "AAt") != 0 &&
      std::strcmp(task, "AAtS") != 0) {
    std::fprintf(stderr, "spgemm_b200: task must be AA, AAt or AAtS, not '%s'\n", task);
    return 1;
  }
  spg_host_csr h{};
  if (spg_csr1_read(argv[2], &h) != SPG_OK) return fail("read");
  const int rc = run(tag, task, reps, h);
  spg_host_csr_free(&h);
  return rc;
}
