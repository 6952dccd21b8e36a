// Declaration-only stand-in for MKL's sparse BLAS interface (see mkl.h).
#ifndef MFP_ORACLE_MKL_SPBLAS_H
#define MFP_ORACLE_MKL_SPBLAS_H
#ifdef __cplusplus
extern "C" {
#endif
typedef enum { SPARSE_STATUS_SUCCESS = 0 } sparse_status_t;
typedef enum { SPARSE_INDEX_BASE_ZERO = 0, SPARSE_INDEX_BASE_ONE = 1 } sparse_index_base_t;
typedef enum { SPARSE_OPERATION_NON_TRANSPOSE = 10 } sparse_operation_t;
typedef enum { SPARSE_MATRIX_TYPE_GENERAL = 20 } sparse_matrix_type_t;
typedef enum { SPARSE_FILL_MODE_LOWER = 40 } sparse_fill_mode_t;
typedef enum { SPARSE_DIAG_NON_UNIT = 50 } sparse_diag_type_t;
struct matrix_descr {
  sparse_matrix_type_t type;
  sparse_fill_mode_t mode;
  sparse_diag_type_t diag;
};
typedef struct mfp_oracle_sparse_matrix *sparse_matrix_t;
sparse_status_t mkl_sparse_s_create_csr(sparse_matrix_t *, sparse_index_base_t, int, int, int *, int *, int *, float *);
sparse_status_t mkl_sparse_d_create_csr(sparse_matrix_t *, sparse_index_base_t, int, int, int *, int *, int *, double *);
sparse_status_t mkl_sparse_optimize(sparse_matrix_t);
sparse_status_t mkl_sparse_s_mv(sparse_operation_t, float, sparse_matrix_t, struct matrix_descr, const float *, float, float *);
sparse_status_t mkl_sparse_d_mv(sparse_operation_t, double, sparse_matrix_t, struct matrix_descr, const double *, double, double *);
#ifdef __cplusplus
}
#endif
#endif
