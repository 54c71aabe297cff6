// Split-BF16x3 Gram products for the mixed-precision LOBPCG (gram_mixed.cu).
#pragma once
#include <cublas_v2.h>

#include "qg_internal.h"

namespace qg {

struct MixedGram {
    static constexpr int kChunk = 13824;  // K rows per FP32-accumulated chunk
    long long N = 0;
    int mmax = 0, nfull = 0, rem = 0;
    DevBuf split_a, split_b, part;

    int setup(long long N, int mmax);
    // bf16 hi/lo copies of the N x m block A (ld N) into slot `which` (0: A side, 1: B side)
    int split(const double* A, int m, int which, cudaStream_t st);
    // C (m x m, ld m) = alpha * A^T B from the split slots (B = A when b_is_a)
    int gram(cublasHandle_t blas, cudaStream_t st, int m, bool b_is_a, double alpha, double* C, int ldc);
    void release();
    ~MixedGram() { release(); }
};

}  // namespace qg
