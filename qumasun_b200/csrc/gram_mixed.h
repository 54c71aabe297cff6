// Split-BF16x3 Gram products for the mixed-precision LOBPCG (gram_mixed.cu).
#pragma once
#include <cublas_v2.h>

#include "gram_i8.h"
#include "gram_tc.h"
#include "qg_internal.h"

namespace qg {

struct MixedGram {
    // K rows per FP32-accumulated chunk. The tensor cores' FP32 accumulation of
    // same-sign terms drifts by about kChunk * 4e-9 of the sum (a Gram diagonal over
    // 1.7M rows lost 5e-5 with 13824-row chunks), so chunks stay short and their
    // partials are summed in FP64, kBatch chunks per batched GEMM call.
    static constexpr int kChunk = 1024;
    static constexpr int kBatch = 96;
    long long N = 0;
    int mmax = 0, nfull = 0, rem = 0;
    DevBuf split_a, split_b, part;
    // pieces > 0: the tcgen05 kernel with that many bf16 pieces (gram_tc.cu);
    // 0 (or a row count that is not a multiple of 8): cuBLAS BF16 GEMMs on hi/lo pieces;
    // -1: FP32 copies and FP32 GEMMs (no tensor cores, no TF32)
    int pieces = 3;
    bool use_tc = false;
    TcGram tc;
    // pieces = kI8Slices (7): FP64-accurate products on the int8 tensor cores (gram_i8.cu)
    bool use_i8 = false;
    I8Gram i8;

    int setup(long long N, int mmax, int pieces = 3);
    // bf16 pieces of the N x m block A (ld N) into slot `which` (0: A side, 1: B side)
    int split(const double* A, int m, int which, cudaStream_t st);
    // C (m x m, ld m) = alpha * A^T B from the split slots (B = A when b_is_a); lower:
    // only the lower triangle is needed (the tcgen05 kernel then skips the upper tiles)
    int gram(cublasHandle_t blas, cudaStream_t st, int m, bool b_is_a, bool lower, double alpha, double* C,
             int ldc, int* err);
    int gram_fp32(cublasHandle_t blas, cudaStream_t st, int m, bool b_is_a, double alpha, double* C, int ldc);
    // C (ma x nc, ld ldc) = alpha * A^T B with A = slot 0's first ma columns and B = columns
    // b_off .. of slot b_slot: the int8 path only (QG_ERR_UNSUPPORTED otherwise)
    int gram_rect(cudaStream_t st, int ma, int nc, int b_slot, int b_off, double alpha, double* C, int ldc,
                  int* err) {
        if (!use_i8) return QG_ERR_UNSUPPORTED;
        return i8.gram_rect(st, ma, nc, b_slot, b_off, alpha, C, ldc, err);
    }
    void release();
    ~MixedGram() { release(); }
};

}  // namespace qg
