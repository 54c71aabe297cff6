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

}  // namespace qg
