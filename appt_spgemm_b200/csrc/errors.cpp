// Thread-local last-error text and status names of the C ABI.
#include <cstdarg>
#include <cstdio>

#include "internal.h"

namespace spg {

static thread_local char g_last_error[512] = "";

spg_status set_error(spg_status st, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
  va_end(ap);
  return st;
}

void clear_error() { g_last_error[0] = '\0'; }

}  // namespace spg

extern "C" {

int32_t spg_abi_version(void) { return SPG_ABI_VERSION; }

const char* spg_last_error_string(void) { return spg::g_last_error; }

const char* spg_status_string(spg_status s) {
  switch (s) {
    case SPG_OK: return "ok";
    case SPG_ERR_INVALID_ARG: return "invalid argument";
    case SPG_ERR_INVALID_CSR: return "invalid CSR";
    case SPG_ERR_OOM: return "out of memory";
    case SPG_ERR_CUDA: return "CUDA error";
    case SPG_ERR_HASH_FULL: return "hash table full";
    case SPG_ERR_TIMEOUT: return "timeout";
    case SPG_ERR_UNSUPPORTED: return "unsupported";
    case SPG_ERR_BUDGET: return "over memory budget";
    case SPG_ERR_NOT_READY: return "not ready";
    case SPG_ERR_IO: return "I/O error";
  }
  return "unknown status";
}

}  // extern "C"
