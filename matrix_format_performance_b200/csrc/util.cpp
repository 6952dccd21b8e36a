// Library identity, status strings and the thread-local error message.
#include "host_common.h"

#include <cstdarg>
#include <cstdio>
#include <string>

namespace {
thread_local std::string g_last_error;
}

namespace mfp {

int fail(int status, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return status;
}

int ok() {
  g_last_error.clear();
  return MFP_SUCCESS;
}

int check_row_ptr(uint32_t rows, uint32_t nnz, const uint32_t *row_ptr) {
  if (!row_ptr) return fail(MFP_ERROR_INVALID_VALUE, "row_ptr is NULL");
  if (row_ptr[0] != 0) return fail(MFP_ERROR_INVALID_VALUE, "row_ptr[0] = %u, expected 0", row_ptr[0]);
  for (uint32_t r = 0; r < rows; ++r)
    if (row_ptr[r + 1] < row_ptr[r])
      return fail(MFP_ERROR_INVALID_VALUE, "row_ptr decreases at row %u", r);
  if (row_ptr[rows] != nnz)
    return fail(MFP_ERROR_INVALID_VALUE, "row_ptr[rows] = %u, expected nnz = %u", row_ptr[rows], nnz);
  return MFP_SUCCESS;
}

}  // namespace mfp

extern "C" {

int mfp_version(void) { return MFP_VERSION; }

const char *mfp_status_string(int status) {
  switch (status) {
    case MFP_SUCCESS: return "success";
    case MFP_ERROR_INVALID_VALUE: return "invalid value";
    case MFP_ERROR_CUDA: return "CUDA error";
    case MFP_ERROR_OUT_OF_MEMORY: return "out of memory";
    case MFP_ERROR_TOO_LARGE: return "too large";
    case MFP_ERROR_NOT_SUPPORTED: return "not supported";
    case MFP_ERROR_DEVICE_WAIT: return "device wait gave up";
    default: return "unknown status";
  }
}

const char *mfp_last_error(void) { return g_last_error.c_str(); }

}  // extern "C"
