// Host-side helpers shared by the C ABI translation units.
#pragma once

#include <cstdint>
#include <cstddef>

#include "../../include/mfp_spmv.h"

namespace mfp {

// Records a formatted message as the thread's last error and returns status.
int fail(int status, const char *fmt, ...)
#if defined(__GNUC__)
    __attribute__((format(printf, 2, 3)))
#endif
    ;

// Clears the thread's last error and returns MFP_SUCCESS.
int ok();

// Validates a CSR row pointer: rows+1 entries, starts at 0, non-decreasing,
// ends at nnz.
int check_row_ptr(uint32_t rows, uint32_t nnz, const uint32_t *row_ptr);

inline size_t value_size(int value_type) { return value_type == MFP_F64 ? 8 : 4; }

}  // namespace mfp
