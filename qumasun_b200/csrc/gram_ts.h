// Tall-skinny Gram products for small LOBPCG blocks (gram_ts.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>

namespace qg {

// Largest column count gram_ts takes.
constexpr int kGramTsMax = 64;

// Blocks the K dimension of each of nprob problems is split over for N rows.
int gram_ts_blocks(long long N, int nprob);
// Doubles of scratch gram_ts needs for nprob problems (two right-hand blocks if two).
size_t gram_ts_scratch_doubles(long long N, int nprob, bool two);

// For p < nprob: C1_p = alpha A_p^T B1_p and (B2 != null) C2_p = alpha A_p^T B2_p,
// A_p = A + p*sA (N x ma, column-major, lda), B*_p = B* + p*sB (N x mb, ldb),
// C*_p = C* + p*sC (ma x mb, column-major, ldc, full matrices); ma, mb <= kGramTsMax.
int gram_ts(const double* A, long long lda, long long sA, const double* B1, const double* B2, long long ldb,
            long long sB, long long N, int ma, int mb, double alpha, double* C1, double* C2, int ldc, long long sC,
            int nprob, double* scratch, cudaStream_t st);

// gram_ts for any ma, mb, in 64 x 64 output tiles launched one after another.
int gram_ts_tiled(const double* A, long long lda, long long sA, const double* B1, const double* B2, long long ldb,
                  long long sB, long long N, int ma, int mb, double alpha, double* C1, double* C2, int ldc,
                  long long sC, int nprob, double* scratch, cudaStream_t st);

// Pencils up to this many columns take gram_ts (cuBLAS's DSYRK / DGEMM above it).
constexpr int kGramTsUpTo = 128;

}  // namespace qg
