// Declaration-only stand-in for Intel MKL (not installed here).  The
// reference's cpu/cpu_matrix_multiplier.cpp includes MKL unconditionally; the
// oracle never calls the MKL path, and the stub definitions in ref_shim.cpp
// abort if it is reached.  Test infrastructure only.
#ifndef MFP_ORACLE_MKL_H
#define MFP_ORACLE_MKL_H
#include "mkl_spblas.h"
#define MKL_ENABLE_AVX2 3
#ifdef __cplusplus
extern "C"
#endif
int mkl_enable_instructions(int);
#endif
