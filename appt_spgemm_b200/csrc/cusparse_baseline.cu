// Vendor baseline harness: times cuSPARSE's generic SpGEMM on the same device
// CSR the engine receives.  Used only by the bench and the tests as the
// comparison point; the engine never calls it (no multi-backend dispatch).
//
// Timing follows the reference's cuSPARSE path (src/cusparse_engine.cuh:45-68):
// for A·Aᵀ the transpose (cusparseCsr2cscEx2) is part of every timed call, and
// every call allocates its buffers and C (workEstimation → compute → copy).
#include <cuda_runtime.h>
#include <cusparse.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

namespace {

struct Fail {
  char* buf;
  int len;
  int operator()(const char* what, int code) const {
    if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s failed (%d)", what, code);
    return -1;
  }
};

#define CU(x, what)                                      \
  do {                                                   \
    cudaError_t e_ = (x);                                \
    if (e_ != cudaSuccess) { rc = fail(what, (int)e_); goto done; } \
  } while (0)
#define SPX(x, what)                                     \
  do {                                                   \
    cusparseStatus_t s_ = (x);                           \
    if (s_ != CUSPARSE_STATUS_SUCCESS) { rc = fail(what, (int)s_); goto done; } \
  } while (0)

// One full product C = A·B (B given), optionally returning C's values' checksums.
int spgemm_once(cusparseHandle_t h, int n, long long nnzA, const int* Ap, const int* Ai,
                const double* Ax, long long nnzB, const int* Bp, const int* Bi, const double* Bx,
                long long* nnz_out, double* chk, const Fail& fail) {
  int rc = 0;
  cusparseSpMatDescr_t mA = nullptr, mB = nullptr, mC = nullptr;
  cusparseSpGEMMDescr_t d = nullptr;
  void *b1 = nullptr, *b2 = nullptr;
  int* Cp = nullptr;
  int* Ci = nullptr;
  double* Cx = nullptr;
  size_t s1 = 0, s2 = 0;
  int64_t r, c, nnzC = 0;
  const double one = 1.0, zero = 0.0;
  const cusparseOperation_t op = CUSPARSE_OPERATION_NON_TRANSPOSE;
  CU(cudaMalloc(&Cp, sizeof(int) * ((size_t)n + 1)), "cudaMalloc C rowptr");
  SPX(cusparseCreateCsr(&mA, n, n, nnzA, (void*)Ap, (void*)Ai, (void*)Ax, CUSPARSE_INDEX_32I,
                        CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F), "createCsr A");
  SPX(cusparseCreateCsr(&mB, n, n, nnzB, (void*)Bp, (void*)Bi, (void*)Bx, CUSPARSE_INDEX_32I,
                        CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F), "createCsr B");
  SPX(cusparseCreateCsr(&mC, n, n, 0, Cp, nullptr, nullptr, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I,
                        CUSPARSE_INDEX_BASE_ZERO, CUDA_R_64F), "createCsr C");
  SPX(cusparseSpGEMM_createDescr(&d), "SpGEMM_createDescr");
  SPX(cusparseSpGEMM_workEstimation(h, op, op, &one, mA, mB, &zero, mC, CUDA_R_64F,
                                    CUSPARSE_SPGEMM_DEFAULT, d, &s1, nullptr), "workEstimation");
  CU(cudaMalloc(&b1, s1 ? s1 : 1), "cudaMalloc buffer1");
  SPX(cusparseSpGEMM_workEstimation(h, op, op, &one, mA, mB, &zero, mC, CUDA_R_64F,
                                    CUSPARSE_SPGEMM_DEFAULT, d, &s1, b1), "workEstimation");
  SPX(cusparseSpGEMM_compute(h, op, op, &one, mA, mB, &zero, mC, CUDA_R_64F,
                             CUSPARSE_SPGEMM_DEFAULT, d, &s2, nullptr), "compute");
  CU(cudaMalloc(&b2, s2 ? s2 : 1), "cudaMalloc buffer2");
  SPX(cusparseSpGEMM_compute(h, op, op, &one, mA, mB, &zero, mC, CUDA_R_64F,
                             CUSPARSE_SPGEMM_DEFAULT, d, &s2, b2), "compute");
  SPX(cusparseSpMatGetSize(mC, &r, &c, &nnzC), "SpMatGetSize");
  CU(cudaMalloc(&Ci, sizeof(int) * (size_t)(nnzC ? nnzC : 1)), "cudaMalloc C col");
  CU(cudaMalloc(&Cx, sizeof(double) * (size_t)(nnzC ? nnzC : 1)), "cudaMalloc C val");
  SPX(cusparseCsrSetPointers(mC, Cp, Ci, Cx), "CsrSetPointers");
  SPX(cusparseSpGEMM_copy(h, op, op, &one, mA, mB, &zero, mC, CUDA_R_64F,
                          CUSPARSE_SPGEMM_DEFAULT, d), "copy");
  if (nnz_out) *nnz_out = nnzC;
  if (chk) {
    std::vector<double> hv((size_t)nnzC);
    if (nnzC) CU(cudaMemcpy(hv.data(), Cx, sizeof(double) * (size_t)nnzC, cudaMemcpyDeviceToHost),
                 "copy C");
    double s = 0, as = 0, sq = 0;
    for (double x : hv) {
      s += x;
      as += x < 0 ? -x : x;
      sq += x * x;
    }
    chk[0] = s;
    chk[1] = as;
    chk[2] = sq;
  }
done:
  if (d) cusparseSpGEMM_destroyDescr(d);
  if (mA) cusparseDestroySpMat(mA);
  if (mB) cusparseDestroySpMat(mB);
  if (mC) cusparseDestroySpMat(mC);
  cudaFree(b1);
  cudaFree(b2);
  cudaFree(Cp);
  cudaFree(Ci);
  cudaFree(Cx);
  return rc;
}

int call_once(cusparseHandle_t h, int task, int n, long long nnz, const int* Ap, const int* Ai,
              const double* Ax, long long* nnz_out, double* chk, const Fail& fail) {
  if (task == 0) return spgemm_once(h, n, nnz, Ap, Ai, Ax, nnz, Ap, Ai, Ax, nnz_out, chk, fail);
  int rc = 0;
  int* Tp = nullptr;
  int* Ti = nullptr;
  double* Tx = nullptr;
  void* buf = nullptr;
  size_t bs = 0;
  CU(cudaMalloc(&Tp, sizeof(int) * ((size_t)n + 1)), "cudaMalloc T rowptr");
  CU(cudaMalloc(&Ti, sizeof(int) * (size_t)(nnz ? nnz : 1)), "cudaMalloc T col");
  CU(cudaMalloc(&Tx, sizeof(double) * (size_t)(nnz ? nnz : 1)), "cudaMalloc T val");
  SPX(cusparseCsr2cscEx2_bufferSize(h, n, n, nnz, Ax, Ap, Ai, Tx, Tp, Ti, CUDA_R_64F,
                                    CUSPARSE_ACTION_NUMERIC, CUSPARSE_INDEX_BASE_ZERO,
                                    CUSPARSE_CSR2CSC_ALG1, &bs), "Csr2cscEx2_bufferSize");
  CU(cudaMalloc(&buf, bs ? bs : 1), "cudaMalloc csr2csc buffer");
  SPX(cusparseCsr2cscEx2(h, n, n, nnz, Ax, Ap, Ai, Tx, Tp, Ti, CUDA_R_64F, CUSPARSE_ACTION_NUMERIC,
                         CUSPARSE_INDEX_BASE_ZERO, CUSPARSE_CSR2CSC_ALG1, buf), "Csr2cscEx2");
  rc = spgemm_once(h, n, nnz, Ap, Ai, Ax, nnz, Tp, Ti, Tx, nnz_out, chk, fail);
done:
  cudaFree(buf);
  cudaFree(Tp);
  cudaFree(Ti);
  cudaFree(Tx);
  return rc;
}

}  // namespace

extern "C" {

// task 0: C = A·A, 1: C = A·Aᵀ.  One checked call (nnz(C), checksums), `warmup`
// untimed calls, then `reps` timed calls; writes the mean, minimum and median
// ms per call (the reference reports the mean, src/cusparse_engine.cuh:45-68;
// its spread from run to run makes the median and minimum worth having).
// Returns 0, or −1 with a message in err (e.g. cuSPARSE cannot hold the product).
int spgb_cusparse_time(int task, const int* dOff, const int* dCol, const double* dVal, int n,
                       long long nnz, int reps, int warmup, float* ms_mean, float* ms_min,
                       float* ms_median, long long* nnz_out, double* chk3, char* err,
                       int errlen) {
  Fail fail{err, errlen};
  if (err && errlen > 0) err[0] = '\0';
  cusparseHandle_t h = nullptr;
  if (cusparseCreate(&h) != CUSPARSE_STATUS_SUCCESS) return fail("cusparseCreate", 0);
  int rc = call_once(h, task, n, nnz, dOff, dCol, dVal, nnz_out, chk3, fail);
  for (int i = 0; i < warmup && rc == 0; ++i)
    rc = call_once(h, task, n, nnz, dOff, dCol, dVal, nullptr, nullptr, fail);
  float total = 0.f, best = 1e30f;
  std::vector<float> all;
  if (rc == 0 && reps > 0) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int i = 0; i < reps && rc == 0; ++i) {
      cudaEventRecord(e0, nullptr);
      rc = call_once(h, task, n, nnz, dOff, dCol, dVal, nullptr, nullptr, fail);
      cudaEventRecord(e1, nullptr);
      cudaEventSynchronize(e1);
      float ms = 0.f;
      cudaEventElapsedTime(&ms, e0, e1);
      total += ms;
      if (ms < best) best = ms;
      all.push_back(ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  cusparseDestroy(h);
  if (rc == 0) {
    if (ms_mean) *ms_mean = reps > 0 ? total / (float)reps : 0.f;
    if (ms_min) *ms_min = reps > 0 ? best : 0.f;
    if (ms_median) {
      std::sort(all.begin(), all.end());
      *ms_median = all.empty() ? 0.f : all[all.size() / 2];
    }
  }
  return rc;
}

}  // extern "C"
