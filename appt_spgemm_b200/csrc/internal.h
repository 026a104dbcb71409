// Internal declarations shared by the engine's host (.cpp) and CUDA (.cu) sources.
#pragma once

#include <stdint.h>

#include "../../include/spgemm_b200.h"

namespace spg {

// ---- error reporting (thread-local last error; never prints, never exits) ----
spg_status set_error(spg_status st, const char* fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;
void clear_error();

// ---- device status word bits (kernels atomicOr these; host maps to status) ----
enum DeviceErrorBits : uint32_t {
  DEV_ERR_HASH_FULL = 1u << 0,  // bounded probe exhausted
  DEV_ERR_OVERFLOW = 1u << 1,   // a row wrote more entries than the symbolic phase counted
  DEV_ERR_BAD_INDEX = 1u << 2,  // a column index outside [0, n) was met
  DEV_ERR_INVALID_CSR = 1u << 3,  // input CSR failed validation
  DEV_ERR_SMALL_CAP = 1u << 4,    // a row exceeds the one-readback plan's table (replan)
};

// ---- engine constants ------------------------------------------------------
constexpr int kEmptyKey = -1;          // empty hash slot
constexpr int kMinTableLog2 = 4;       // smallest shared table: 16 slots
constexpr int kMaxTableLog2 = 14;      // largest shared table: 16384 slots
constexpr int kNumTableBins = kMaxTableLog2 - kMinTableLog2 + 1;  // 11
// Row bins: 0 = empty row, 1..kNumTableBins = shared table of 2^(bin+3) slots,
// kHeavyBin = heavy row (CTA per row, dense column window), kDenseBin0 + b =
// warp row over a bitmap of 2^(kDenseMinLog2W + b) words of its column span.
constexpr int kEmptyBin = 0;
constexpr int kHeavyBin = kNumTableBins + 1;  // 12
constexpr int kDenseMinLog2W = 8;
constexpr int kDenseMaxLog2W = 11;
constexpr int kDenseBin0 = kHeavyBin + 1;     // 13
constexpr int kNumBins = kDenseBin0 + kDenseMaxLog2W - kDenseMinLog2W + 1;  // 17
constexpr int kDenseVals = 256;  // entries of a bitmap-path row (numeric)

}  // namespace spg
