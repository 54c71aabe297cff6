// Small generalised symmetric eigensolver (small_eig.cu).
#pragma once
#include <cuda_runtime.h>

namespace qg {

constexpr int kSmallEigMax = 80;  // largest pencil one thread block solves in shared memory

// batch problems A_b z = lambda B_b z (k x k, lower triangles, column-major, lda),
// A_b = A + b*stride_ab; eigenvectors to Z + b*stride_z (column-major, ldz), ascending
// eigenvalues to w + b*stride_w, status to info[b]. n_restart > 0: on a Cholesky failure
// solve the leading n_restart pencil and zero the remaining rows of Z (LOBPCG restart).
int small_eig_launch(const double* A, const double* B, int lda, long long stride_ab, int k, int n_restart, double* Z,
                     int ldz, long long stride_z, double* w, long long stride_w, int* info, int batch,
                     cudaStream_t st);

constexpr int kSmallHegMax = 56;  // largest complex pencil (4 k x k complex matrices in shared memory)

// Complex Hermitian counterpart (replaces lapack_ZHEGVX, w_zhegvx.h:24-107, for the
// k-point LOBPCG pencils): batch problems A_b z = lambda B_b z, k x k complex
// (double2 {re, im}), column-major with leading dimension lda, lower triangles read,
// A_b = A + b*stride_ab; eigenvectors to Z + b*stride_z (column-major, ldz; Z may
// alias A: each problem is read completely before its vectors are written), ascending
// eigenvalues to w + b*stride_w, status to info[b] (0 ok, 1 B not positive definite,
// 2 sweep limit reached, vectors kept). skip (may be null): problems with skip[b] != 0
// are left untouched (info 0).
// pivot_floor: a Cholesky pivot of the equilibrated B (unit diagonal) whose square
// falls below it counts as a failure (info 1), so that the caller can take its
// rank-revealing solve instead of a nearly singular factor.
int small_heg_launch(const double2* A, const double2* B, int lda, long long stride_ab, int k, const int* skip,
                     double2* Z, int ldz, long long stride_z, double* w, long long stride_w, int* info, int batch,
                     cudaStream_t st, double pivot_floor = 0.0);

}  // namespace qg
