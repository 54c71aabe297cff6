/*
 * cblas.h shim for building the reference's CPU path in this container
 * (test infrastructure only: the oracle, never the product).
 *
 * The reference includes <cblas.h> from wrap_lapack.h (source/wrap_lapack.h:18)
 * and calls cblas_dgemm / cblas_zgemm / cblas_dgemmt / cblas_dgemv / cblas_zgemv
 * (source/w_dgemm.h:33, source/lobpcg_d_multi_mpi.h, source/lobpcg_z_multi_mpi.h).
 * There is no system BLAS here; the only BLAS in the image is the OpenBLAS
 * 0.3.30 bundled with scipy, whose exported symbols carry a "scipy_" prefix
 * and use 32-bit integers. This header maps the standard CBLAS names onto it.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

typedef enum CBLAS_ORDER { CblasRowMajor = 101, CblasColMajor = 102 } CBLAS_ORDER;
typedef enum CBLAS_TRANSPOSE { CblasNoTrans = 111, CblasTrans = 112, CblasConjTrans = 113, CblasConjNoTrans = 114 } CBLAS_TRANSPOSE;
typedef enum CBLAS_UPLO { CblasUpper = 121, CblasLower = 122 } CBLAS_UPLO;
typedef CBLAS_ORDER CBLAS_LAYOUT;

void scipy_cblas_dgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int,
                       double, const double*, int, const double*, int, double, double*, int);
void scipy_cblas_zgemm(CBLAS_ORDER, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int, int,
                       const void*, const void*, int, const void*, int, const void*, void*, int);
void scipy_cblas_dgemmt(CBLAS_ORDER, CBLAS_UPLO, CBLAS_TRANSPOSE, CBLAS_TRANSPOSE, int, int,
                        double, const double*, int, const double*, int, double, double*, int);
void scipy_cblas_dgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int, int, double, const double*, int,
                       const double*, int, double, double*, int);
void scipy_cblas_zgemv(CBLAS_ORDER, CBLAS_TRANSPOSE, int, int, const void*, const void*, int,
                       const void*, int, const void*, void*, int);
void scipy_openblas_set_num_threads(int);

#define cblas_dgemm scipy_cblas_dgemm
#define cblas_zgemm scipy_cblas_zgemm
#define cblas_dgemmt scipy_cblas_dgemmt
#define cblas_dgemv scipy_cblas_dgemv
#define cblas_zgemv scipy_cblas_zgemv

#ifdef __cplusplus
}
#endif
