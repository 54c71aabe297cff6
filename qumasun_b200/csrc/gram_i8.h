// FP64-accurate Gram products on the int8 tensor cores (gram_i8.cu).
#pragma once
#include "qg_internal.h"

namespace qg {

// C = alpha * A^T B for tall FP64 blocks A (N x ma) and B (N x nc), ld N. Every column is
// scaled by a power of two, 2^-E_j, so that its largest value is below 127/128, and cut
// into kI8Slices signed 7-bit slices, a = 2^E sum_t d_t 2^-7(t+1), |d_0| <= 127,
// |d_t| <= 64 -- exact, the remainder below 2^-49 of the column's largest value. The
// slice products with t + u <= kI8Slices - 1 (28) run on tcgen05.mma kind::i8 with
// exact int32 accumulation; the 7 sums of equal t + u are scaled and added in FP64. The
// result is as accurate as an FP64 DGEMM (1.6e-15 on unit-norm columns against
// 6e-13 with 5 slices), at the tensor cores' int8 rate.
constexpr int kI8Slices = 7;

struct I8Gram {
    long long N = 0;
    int mmax = 0;
    int m_slot[2] = {0, 0};       // split width of each slot
    DevBuf slices[2], expo[2], part;

    static bool supported(long long N);
    // N rounded up to the 64-row K block (rows of the slices, zero past N)
    long long kpad() const;
    int setup(long long N, int mmax);
    // slices and column exponents of the N x m block A (ld N, m <= mmax) into slot `which`
    int split(const double* A, int m, int which, cudaStream_t st);
    // C (m x m, ld ldc) = alpha * A^T B from slot 0 and slot 1 (slot 0 again when b_is_a);
    // lower: only the tiles that reach the lower triangle
    int gram(cudaStream_t st, int m, bool b_is_a, bool lower, double alpha, double* C, int ldc, int* err);
    // C (ma x nc, ld ldc) = alpha * A^T B over slot 0's first ma columns and columns
    // b_off .. b_off + nc - 1 of slot b_slot
    int gram_rect(cudaStream_t st, int ma, int nc, int b_slot, int b_off, double alpha, double* C, int ldc,
                  int* err);
    void release();
    ~I8Gram() { release(); }
};

}  // namespace qg
