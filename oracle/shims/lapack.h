/*
 * lapack.h shim for building the reference's CPU path in this container
 * (test infrastructure only).
 *
 * The reference calls DSYGVX (source/w_dsygvx.h:78) and ZHEGVX
 * (source/w_zhegvx.h:82) through <lapack.h>. These map onto the scipy-bundled
 * OpenBLAS 0.3.30 Fortran entry points (scipy_dsygvx_, scipy_zhegvx_), passing
 * the gfortran hidden CHARACTER lengths explicitly.
 */
#pragma once
#include <complex>
#include <cstddef>

extern "C" {
void scipy_dsygvx_(const int* itype, const char* jobz, const char* range, const char* uplo,
                   const int* n, double* a, const int* lda, double* b, const int* ldb,
                   const double* vl, const double* vu, const int* il, const int* iu,
                   const double* abstol, int* m, double* w, double* z, const int* ldz,
                   double* work, const int* lwork, int* iwork, int* ifail, int* info,
                   size_t, size_t, size_t);
void scipy_zhegvx_(const int* itype, const char* jobz, const char* range, const char* uplo,
                   const int* n, void* a, const int* lda, void* b, const int* ldb,
                   const double* vl, const double* vu, const int* il, const int* iu,
                   const double* abstol, int* m, double* w, void* z, const int* ldz,
                   void* work, const int* lwork, double* rwork, int* iwork, int* ifail,
                   int* info, size_t, size_t, size_t);
}

#ifndef lapack_complex_double
#define lapack_complex_double std::complex<double>
#endif

inline void DSYGVX(const int* itype, const char* jobz, const char* range, const char* uplo,
                   const int* n, double* a, const int* lda, double* b, const int* ldb,
                   const double* vl, const double* vu, const int* il, const int* iu,
                   const double* abstol, int* m, double* w, double* z, const int* ldz,
                   double* work, const int* lwork, int* iwork, int* ifail, int* info) {
    scipy_dsygvx_(itype, jobz, range, uplo, n, a, lda, b, ldb, vl, vu, il, iu, abstol, m, w, z,
                  ldz, work, lwork, iwork, ifail, info, 1, 1, 1);
}

inline void ZHEGVX(const int* itype, const char* jobz, const char* range, const char* uplo,
                   const int* n, lapack_complex_double* a, const int* lda,
                   lapack_complex_double* b, const int* ldb, const double* vl, const double* vu,
                   const int* il, const int* iu, const double* abstol, int* m, double* w,
                   lapack_complex_double* z, const int* ldz, lapack_complex_double* work,
                   const int* lwork, double* rwork, int* iwork, int* ifail, int* info) {
    scipy_zhegvx_(itype, jobz, range, uplo, n, a, lda, b, ldb, vl, vu, il, iu, abstol, m, w, z,
                  ldz, work, lwork, rwork, iwork, ifail, info, 1, 1, 1);
}
