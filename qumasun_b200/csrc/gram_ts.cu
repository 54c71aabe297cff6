// Tall-skinny Gram products C = alpha A^T B for the LOBPCG pencils of small blocks
// (the reference's MakeMatrix_d_blas, lobpcg_d_multi_mpi.h:191-250, with K = the
// grid and M, N = the block's columns): A is N x ma, B is N x mb, both column-major
// with leading dimension lda / ldb (state-major blocks), ma, mb <= 64.
//
// cuBLAS spends milliseconds on these shapes (an m x m output has too few tiles to
// spread K = 64k-1.7M rows over the GPU). Here K is split: block b sums rows
// [b*rows, (b+1)*rows) in shared-memory chunks of 24 rows, each thread holding a
// 4 x 4 (or, up to 32 columns, 2 x 2) tile of the output, for one or two right-hand blocks at once
// (A^T B1 and A^T B2 share the reads of A); a second kernel adds the per-block
// partial sums in block order (deterministic) and scales by alpha. Several
// problems (blockIdx.y) run in one launch.
#include "gram_ts.h"
#include "qg_internal.h"

#include <algorithm>

namespace qg {
namespace {

constexpr int kRows = 24;   // rows per shared-memory chunk (3 x 24 x 65 doubles fit the static limit)
constexpr int kT = 16;      // 16 x 16 threads, 4 x 4 outputs each
constexpr int kMax = 64;

template <int TILE>
__global__ void __launch_bounds__(kT * kT) k_gram_ts_partial(const double* __restrict__ A, long long lda,
                                                             long long sA, const double* __restrict__ B1,
                                                             const double* __restrict__ B2, long long ldb,
                                                             long long sB, long long N, int ma, int mb,
                                                             long long rows_per_block, double* __restrict__ part) {
    __shared__ double As[kRows][kMax + 1];
    __shared__ double Bs[2][kRows][kMax + 1];
    const int prob = blockIdx.y;
    A += prob * sA;
    B1 += prob * sB;
    if (B2) B2 += prob * sB;
    const int nb = B2 ? 2 : 1;
    const int t = threadIdx.x;
    const int ti = t / kT, tj = t % kT;
    const long long r0 = (long long)blockIdx.x * rows_per_block;
    const long long r1 = min(N, r0 + rows_per_block);
    double acc[2][TILE][TILE];
#pragma unroll
    for (int q = 0; q < 2; ++q)
#pragma unroll
        for (int i = 0; i < TILE; ++i)
#pragma unroll
            for (int j = 0; j < TILE; ++j) acc[q][i][j] = 0.0;
    for (long long rc = r0; rc < r1; rc += kRows) {
        const int nr = (int)min((long long)kRows, r1 - rc);
        // column-wise coalesced loads: consecutive rows of one column per warp
        for (int e = t; e < kRows * ma; e += kT * kT) {
            const int rr = e % kRows, c = e / kRows;
            As[rr][c] = rr < nr ? A[(long long)c * lda + rc + rr] : 0.0;
        }
        for (int e = t; e < kRows * mb; e += kT * kT) {
            const int rr = e % kRows, c = e / kRows;
            Bs[0][rr][c] = rr < nr ? B1[(long long)c * ldb + rc + rr] : 0.0;
            if (B2) Bs[1][rr][c] = rr < nr ? B2[(long long)c * ldb + rc + rr] : 0.0;
        }
        __syncthreads();
#pragma unroll 4
        for (int rr = 0; rr < kRows; ++rr) {
            double a[TILE], b[TILE];
#pragma unroll
            for (int i = 0; i < TILE; ++i) a[i] = As[rr][ti * TILE + i];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (q >= nb) break;
#pragma unroll
                for (int j = 0; j < TILE; ++j) b[j] = Bs[q][rr][tj * TILE + j];
#pragma unroll
                for (int i = 0; i < TILE; ++i)
#pragma unroll
                    for (int j = 0; j < TILE; ++j) acc[q][i][j] += a[i] * b[j];
            }
        }
        __syncthreads();
    }
    // partial sums, compact: part[((prob * nblocks + block) * nb + q) * ma * mb + i * mb + j]
    const long long msz = (long long)ma * mb;
    double* pb = part + ((long long)prob * gridDim.x + blockIdx.x) * nb * msz;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        if (q >= nb) break;
#pragma unroll
        for (int i = 0; i < TILE; ++i)
#pragma unroll
            for (int j = 0; j < TILE; ++j) {
                const int ii = ti * TILE + i, jj = tj * TILE + j;
                if (ii < ma && jj < mb) pb[(long long)q * msz + ii * mb + jj] = acc[q][i][j];
            }
    }
}

// One warp per output element: lanes take the blocks' partial sums in strides of 32,
// then a fixed shuffle tree (the same order every call).
__global__ void k_gram_ts_reduce(const double* __restrict__ part, int nblocks, int nb, int ma, int mb, double alpha,
                                 double* __restrict__ C1, double* __restrict__ C2, int ldc, long long sC) {
    const int prob = blockIdx.y;
    const int lane = threadIdx.x & 31;
    const int e = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const long long msz = (long long)ma * mb;
    if (e >= nb * msz) return;
    const int q = (int)(e / msz);
    const long long ij = e % msz;
    const int i = (int)(ij / mb), j = (int)(ij % mb);
    const double* p = part + (long long)prob * nblocks * nb * msz + (long long)q * msz + ij;
    double s = 0.0;
    for (int b = lane; b < nblocks; b += 32) s += p[(long long)b * nb * msz];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        double* C = (q == 0 ? C1 : C2) + prob * sC;
        C[i + (long long)j * ldc] = alpha * s;
    }
}

}  // namespace

size_t gram_ts_scratch_doubles(long long N, int nprob, bool two) {
    const int nblocks = gram_ts_blocks(N, nprob);
    return (size_t)nprob * nblocks * (two ? 2 : 1) * kMax * kMax;
}

int gram_ts_blocks(long long N, int nprob) {
    // about 2 blocks per SM over all problems, at least 256 rows each
    const long long per = (2 * 148 + nprob - 1) / nprob;
    const long long b = std::min<long long>(per, (N + 255) / 256);
    return (int)std::max<long long>(1, b);
}

int gram_ts(const double* A, long long lda, long long sA, const double* B1, const double* B2, long long ldb,
            long long sB, long long N, int ma, int mb, double alpha, double* C1, double* C2, int ldc, long long sC,
            int nprob, double* scratch, cudaStream_t st) {
    if (ma <= 0 || mb <= 0 || ma > kMax || mb > kMax || N <= 0 || nprob <= 0) return QG_ERR_UNSUPPORTED;
    const int nblocks = gram_ts_blocks(N, nprob);
    const long long rows = (N + nblocks - 1) / nblocks;
    // 2 x 2 outputs per thread when both sides fit 32 columns (every thread busy)
    if (ma <= 2 * kT && mb <= 2 * kT)
        k_gram_ts_partial<2><<<dim3(nblocks, nprob), kT * kT, 0, st>>>(A, lda, sA, B1, B2, ldb, sB, N, ma, mb, rows,
                                                                        scratch);
    else
        k_gram_ts_partial<4><<<dim3(nblocks, nprob), kT * kT, 0, st>>>(A, lda, sA, B1, B2, ldb, sB, N, ma, mb, rows,
                                                                        scratch);
    const int nb = B2 ? 2 : 1;
    const int tot = nb * ma * mb;  // one warp each, 8 warps per block
    k_gram_ts_reduce<<<dim3((tot + 7) / 8, nprob), 256, 0, st>>>(scratch, nblocks, nb, ma, mb, alpha, C1, C2, ldc,
                                                                 sC);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int gram_ts_tiled(const double* A, long long lda, long long sA, const double* B1, const double* B2, long long ldb,
                  long long sB, long long N, int ma, int mb, double alpha, double* C1, double* C2, int ldc,
                  long long sC, int nprob, double* scratch, cudaStream_t st) {
    for (int i0 = 0; i0 < ma; i0 += kMax)
        for (int j0 = 0; j0 < mb; j0 += kMax) {
            const int ta = std::min(kMax, ma - i0), tb = std::min(kMax, mb - j0);
            const int rc = gram_ts(A + (long long)i0 * lda, lda, sA, B1 + (long long)j0 * ldb,
                                   B2 ? B2 + (long long)j0 * ldb : nullptr, ldb, sB, N, ta, tb, alpha,
                                   C1 + i0 + (long long)j0 * ldc, C2 ? C2 + i0 + (long long)j0 * ldc : nullptr, ldc,
                                   sC, nprob, scratch, st);
            if (rc != QG_OK) return rc;
        }
    return QG_OK;
}

}  // namespace qg

extern "C" int qg_gram_small_d(qg_context ctx, long long N, int ma, int mb, const double* A, const double* B,
                               double alpha, double* C) {
    if (!ctx || N <= 0 || ma <= 0 || mb <= 0 || !A || !B || !C) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    double* scratch = nullptr;
    const size_t bytes = qg::gram_ts_scratch_doubles(N, 1, false) * sizeof(double);
    QG_CUDA_TRY(cudaMallocAsync(reinterpret_cast<void**>(&scratch), bytes, ctx->stream));
    const int rc = qg::gram_ts_tiled(A, N, 0, B, nullptr, N, 0, N, ma, mb, alpha, C, nullptr, ma, 0, 1, scratch,
                                     ctx->stream);
    cudaFreeAsync(scratch, ctx->stream);
    if (rc != QG_OK) return rc;
    QG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return QG_OK;
}
