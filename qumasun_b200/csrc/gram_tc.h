// Split-BF16 Gram products on the tcgen05 tensor cores (gram_tc.cu).
#pragma once
#include "qg_internal.h"

namespace qg {

struct TcGram {
    long long N = 0;
    int mmax = 0, pieces = 3;
    DevBuf split_a, split_b, part;

    // N >= 64 and the driver's tensor-map encoder available
    static bool supported(long long N);
    // N rounded up to the 64-row K block (rows of the pieces, zero past N)
    long long kpad() const;
    int setup(long long N, int mmax, int pieces);
    // bf16 pieces of the N x m block A (ld N, m <= mmax) into slot `which` (0: A side,
    // 1: B side), stored K-block-major; gram() must be given the same m
    int split(const double* A, int m, int which, cudaStream_t st);
    // C (m x m, column-major, ld ldc) = alpha * A^T B from the split slots (B = A when
    // b_is_a); lower: only the tiles on and below the diagonal are computed and
    // written. err: device status word for the kernel's bounded waits.
    int gram(cudaStream_t st, int m, bool b_is_a, bool lower, double alpha, double* C, int ldc, int* err);
    void release();
    ~TcGram() { release(); }
};

}  // namespace qg
