// cuSPARSE yardstick (library code beside the engine; see include/mfp_yardstick.h).
#include "mfp_yardstick.h"

#include <cuda_runtime.h>
#include <cusparse.h>

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

namespace {
thread_local std::string g_err;

int fail(const std::string &m) {
  g_err = m;
  return 2;
}
}  // namespace

extern "C" {

const char *mfp_cusparse_last_error(void) { return g_err.c_str(); }

int mfp_cusparse_spmv(int format, int alg, int vt, uint32_t rows, uint32_t cols, uint32_t nnz, const uint32_t *index,
                      const uint32_t *col_ids, const void *values, const void *x, void *y, uint32_t reps,
                      int flush_l2, void *stream, double *median_s) {
  g_err.clear();
  if ((format != 0 && format != 1) || alg < 0 || alg > 2 || (vt != 0 && vt != 1))
    return fail("bad format, algorithm or value type");
  if (rows >= (1u << 31) || cols >= (1u << 31) || nnz >= (1u << 31)) return fail("sizes exceed 32-bit signed indices");
  if (!index || !y || (nnz && (!col_ids || !values || !x))) return fail("null device array");
  const cudaDataType dt = vt ? CUDA_R_64F : CUDA_R_32F;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cusparseHandle_t h = nullptr;
  cusparseSpMatDescr_t A = nullptr;
  cusparseDnVecDescr_t X = nullptr, Y = nullptr;
  void *buf = nullptr, *flush = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int st = 0;
  const double one = 1.0, zero = 0.0;
  const float onef = 1.f, zerof = 0.f;
  const void *alpha = vt ? (const void *)&one : (const void *)&onef;
  const void *beta = vt ? (const void *)&zero : (const void *)&zerof;
  cusparseSpMVAlg_t a = CUSPARSE_SPMV_ALG_DEFAULT;
  if (alg == 1) a = format == 0 ? CUSPARSE_SPMV_CSR_ALG1 : CUSPARSE_SPMV_COO_ALG1;
  if (alg == 2) a = format == 0 ? CUSPARSE_SPMV_CSR_ALG2 : CUSPARSE_SPMV_COO_ALG2;
  size_t bytes = 0;
  std::vector<double> t;
  auto cs = [&](cusparseStatus_t r, const char *what) {
    if (r != CUSPARSE_STATUS_SUCCESS && !st) st = fail(std::string(what) + ": " + cusparseGetErrorString(r));
    return st == 0;
  };
  auto cu = [&](cudaError_t r, const char *what) {
    if (r != cudaSuccess && !st) st = fail(std::string(what) + ": " + cudaGetErrorString(r));
    return st == 0;
  };
  if (!cs(cusparseCreate(&h), "cusparseCreate") || !cs(cusparseSetStream(h, s), "cusparseSetStream")) goto done;
  if (format == 0) {
    if (!cs(cusparseCreateCsr(&A, rows, cols, nnz, (void *)index, (void *)col_ids, (void *)values,
                              CUSPARSE_INDEX_32I, CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, dt),
            "cusparseCreateCsr"))
      goto done;
  } else {
    if (!cs(cusparseCreateCoo(&A, rows, cols, nnz, (void *)index, (void *)col_ids, (void *)values,
                              CUSPARSE_INDEX_32I, CUSPARSE_INDEX_BASE_ZERO, dt),
            "cusparseCreateCoo"))
      goto done;
  }
  if (!cs(cusparseCreateDnVec(&X, cols, (void *)x, dt), "cusparseCreateDnVec") ||
      !cs(cusparseCreateDnVec(&Y, rows, y, dt), "cusparseCreateDnVec") ||
      !cs(cusparseSpMV_bufferSize(h, CUSPARSE_OPERATION_NON_TRANSPOSE, alpha, A, X, beta, Y, dt, a, &bytes),
          "cusparseSpMV_bufferSize"))
    goto done;
  if (bytes && !cu(cudaMalloc(&buf, bytes), "cudaMalloc")) goto done;
  if (!cs(cusparseSpMV_preprocess(h, CUSPARSE_OPERATION_NON_TRANSPOSE, alpha, A, X, beta, Y, dt, a, buf),
          "cusparseSpMV_preprocess") ||
      !cs(cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, alpha, A, X, beta, Y, dt, a, buf), "cusparseSpMV"))
    goto done;
  if (reps) {
    int dev = 0, l2 = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev);
    const size_t fb = (size_t)std::max(l2, 1 << 20) * 2;
    if (flush_l2 && !cu(cudaMalloc(&flush, fb), "cudaMalloc")) goto done;
    if (!cu(cudaEventCreate(&e0), "cudaEventCreate") || !cu(cudaEventCreate(&e1), "cudaEventCreate")) goto done;
    for (uint32_t i = 0; i < reps && !st; ++i) {
      if (flush) cudaMemsetAsync(flush, (int)(i & 0xff), fb, s);
      cudaEventRecord(e0, s);
      cs(cusparseSpMV(h, CUSPARSE_OPERATION_NON_TRANSPOSE, alpha, A, X, beta, Y, dt, a, buf), "cusparseSpMV");
      cudaEventRecord(e1, s);
      if (cu(cudaEventSynchronize(e1), "cudaEventSynchronize")) {
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        t.push_back(ms * 1e-3);
      }
    }
    if (!st && median_s) {
      std::sort(t.begin(), t.end());
      *median_s = t[t.size() / 2];
    }
  } else {
    cu(cudaStreamSynchronize(s), "cudaStreamSynchronize");
  }
done:
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (flush) cudaFree(flush);
  if (buf) cudaFree(buf);
  if (X) cusparseDestroyDnVec(X);
  if (Y) cusparseDestroyDnVec(Y);
  if (A) cusparseDestroySpMat(A);
  if (h) cusparseDestroy(h);
  return st;
}

}  // extern "C"
