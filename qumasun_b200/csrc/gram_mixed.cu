// Mixed-precision Gram products for LOBPCG: S = alpha A^T B with A, B tall
// N x m FP64 blocks (ld N), computed as split-BF16x3 with FP32 accumulation:
//   a = a_hi + a_lo,  a_hi = bf16(a),  a_lo = bf16(a - a_hi)   (same for b)
//   a.b ~ a_hi.b_hi + a_hi.b_lo + a_lo.b_hi                      (a_lo.b_lo dropped, ~2^-17 relative)
// The K (grid) dimension is cut into chunks of kChunk rows; every chunk is an
// FP32-accumulated tensor-core product, the chunk partials are summed in FP64 in a
// fixed order (deterministic), so the FP32 error grows with the chunk length only.
// pieces = -1 is the FP32 variant: one FP32 copy of each block and FP32 (non-tensor,
// no TF32) products over the same chunks.
#include <cublas_v2.h>
#include <cuda_bf16.h>

#include <algorithm>

#include "gram_mixed.h"

namespace qg {
namespace {

__global__ void k_split_bf16(const double* __restrict__ src, long long n, __nv_bfloat16* __restrict__ hi,
                             __nv_bfloat16* __restrict__ lo) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const double v = src[i];
        const __nv_bfloat16 h = __double2bfloat16(v);
        hi[i] = h;
        lo[i] = __double2bfloat16(v - (double)__bfloat162float(h));
    }
}

__global__ void k_to_float(const double* __restrict__ src, long long n, float* __restrict__ dst) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) dst[i] = (float)src[i];
}

// C[e] (+)= alpha * sum_c P[c][e] for e < m*m, chunks in order (accumulate: add to C).
__global__ void k_reduce_chunks(const float* __restrict__ P, int nchunk, long long mm, double alpha, int accumulate,
                                double* __restrict__ C) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < mm; e += stride) {
        double s = 0.0;
        for (int c = 0; c < nchunk; ++c) s += (double)P[(long long)c * mm + e];
        C[e] = accumulate ? C[e] + alpha * s : alpha * s;
    }
}

#define QG_MG_BLAS_TRY(expr)                                           \
    do {                                                               \
        cublasStatus_t qg_b_ = (expr);                                 \
        if (qg_b_ != CUBLAS_STATUS_SUCCESS) {                          \
            qg_set_last_error(#expr, "cublas error", __FILE__, __LINE__); \
            return QG_ERR_LIBRARY;                                     \
        }                                                              \
    } while (0)

}  // namespace

int MixedGram::setup(long long N_, int mmax_, int pieces_) {
    N = N_;
    mmax = mmax_;
    pieces = pieces_;
    use_i8 = pieces == kI8Slices && I8Gram::supported(N);
    if (pieces == kI8Slices) return use_i8 ? i8.setup(N, mmax) : QG_ERR_UNSUPPORTED;
    use_tc = pieces > 0 && TcGram::supported(N);
    if (use_tc) return tc.setup(N, mmax, pieces);
    const size_t elems = (size_t)N * mmax;
    const size_t bytes = pieces < 0 ? elems * sizeof(float) : 2 * elems * sizeof(__nv_bfloat16);
    QG_TRY(split_a.reserve(bytes));
    QG_TRY(split_b.reserve(bytes));
    nfull = (int)(N / kChunk);
    rem = (int)(N - (long long)nfull * kChunk);
    const int nparts = std::min(nfull, kBatch) + (rem ? 1 : 0);
    QG_TRY(part.reserve((size_t)std::max(nparts, 1) * mmax * mmax * sizeof(float)));
    return QG_OK;
}

int MixedGram::split(const double* A, int m, int which, cudaStream_t st) {
    if (use_i8) return i8.split(A, m, which, st);
    if (use_tc) return tc.split(A, m, which, st);
    const long long n = N * m;
    DevBuf& b = which == 0 ? split_a : split_b;
    if (pieces < 0) {
        k_to_float<<<148 * 8, 256, 0, st>>>(A, n, b.as<float>());
        QG_CUDA_TRY(cudaGetLastError());
        return QG_OK;
    }
    __nv_bfloat16* hi = b.as<__nv_bfloat16>();
    __nv_bfloat16* lo = hi + (size_t)N * mmax;
    k_split_bf16<<<148 * 8, 256, 0, st>>>(A, n, hi, lo);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int MixedGram::gram(cublasHandle_t blas, cudaStream_t st, int m, bool b_is_a, bool lower, double alpha, double* C,
                    int ldc, int* err) {
    if (use_i8) return i8.gram(st, m, b_is_a, lower, alpha, C, ldc, err);
    if (use_tc) return tc.gram(st, m, b_is_a, lower, alpha, C, ldc, err);
    if (pieces < 0) return gram_fp32(blas, st, m, b_is_a, alpha, C, ldc);
    const __nv_bfloat16* ahi = split_a.as<__nv_bfloat16>();
    const __nv_bfloat16* alo = ahi + (size_t)N * mmax;
    const __nv_bfloat16* bhi = b_is_a ? ahi : split_b.as<__nv_bfloat16>();
    const __nv_bfloat16* blo = bhi + (size_t)N * mmax;
    float* P = part.as<float>();
    const long long mm = (long long)m * m;
    const float one = 1.0f, zero = 0.0f;
    const __nv_bfloat16* As[3] = {ahi, ahi, alo};
    const __nv_bfloat16* Bs[3] = {bhi, blo, bhi};
    QG_MG_BLAS_TRY(cublasSetStream(blas, st));
    if (ldc != m) return QG_ERR_INVALID;
    // batches of up to kBatch chunks: three FP32-accumulated products per chunk, then
    // the batch's chunk partials are added into C in FP64
    bool first = true;
    for (int c0 = 0; c0 < nfull || (first && rem); c0 += kBatch) {
        const int nb = std::max(0, std::min(kBatch, nfull - c0));
        const bool last = c0 + kBatch >= nfull;
        const int tail = (last && rem) ? 1 : 0;
        for (int t = 0; t < 3; ++t) {
            const float* beta = t == 0 ? &zero : &one;
            const long long k0 = (long long)c0 * kChunk;
            if (nb > 0)
                QG_MG_BLAS_TRY(cublasGemmStridedBatchedEx(blas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, kChunk, &one,
                                                          As[t] + k0, CUDA_R_16BF, (int)N, kChunk, Bs[t] + k0,
                                                          CUDA_R_16BF, (int)N, kChunk, beta, P, CUDA_R_32F, m, mm, nb,
                                                          CUBLAS_COMPUTE_32F, CUBLAS_GEMM_DEFAULT));
            if (tail)
                QG_MG_BLAS_TRY(cublasGemmEx(blas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, rem, &one,
                                            As[t] + (long long)nfull * kChunk, CUDA_R_16BF, (int)N,
                                            Bs[t] + (long long)nfull * kChunk, CUDA_R_16BF, (int)N, beta,
                                            P + (long long)nb * mm, CUDA_R_32F, m, CUBLAS_COMPUTE_32F,
                                            CUBLAS_GEMM_DEFAULT));
        }
        k_reduce_chunks<<<148 * 4, 256, 0, st>>>(P, nb + tail, mm, alpha, first ? 0 : 1, C);
        first = false;
        if (last) break;
    }
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int MixedGram::gram_fp32(cublasHandle_t blas, cudaStream_t st, int m, bool b_is_a, double alpha, double* C,
                         int ldc) {
    const float* a = split_a.as<float>();
    const float* b = b_is_a ? a : split_b.as<float>();
    float* P = part.as<float>();
    const long long mm = (long long)m * m;
    const float one = 1.0f, zero = 0.0f;
    QG_MG_BLAS_TRY(cublasSetStream(blas, st));
    if (ldc != m) return QG_ERR_INVALID;
    bool first = true;
    for (int c0 = 0; c0 < nfull || (first && rem); c0 += kBatch) {
        const int nb = std::max(0, std::min(kBatch, nfull - c0));
        const bool last = c0 + kBatch >= nfull;
        const int tail = (last && rem) ? 1 : 0;
        const long long k0 = (long long)c0 * kChunk;
        if (nb > 0)
            QG_MG_BLAS_TRY(cublasGemmStridedBatchedEx(blas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, kChunk, &one, a + k0,
                                                      CUDA_R_32F, (int)N, kChunk, b + k0, CUDA_R_32F, (int)N, kChunk,
                                                      &zero, P, CUDA_R_32F, m, mm, nb, CUBLAS_COMPUTE_32F_PEDANTIC,
                                                      CUBLAS_GEMM_DEFAULT));
        if (tail)
            QG_MG_BLAS_TRY(cublasGemmEx(blas, CUBLAS_OP_T, CUBLAS_OP_N, m, m, rem, &one,
                                        a + (long long)nfull * kChunk, CUDA_R_32F, (int)N,
                                        b + (long long)nfull * kChunk, CUDA_R_32F, (int)N, &zero,
                                        P + (long long)nb * mm, CUDA_R_32F, m, CUBLAS_COMPUTE_32F_PEDANTIC,
                                        CUBLAS_GEMM_DEFAULT));
        k_reduce_chunks<<<148 * 4, 256, 0, st>>>(P, nb + tail, mm, alpha, first ? 0 : 1, C);
        first = false;
        if (last) break;
    }
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

void MixedGram::release() {
    tc.release();
    i8.release();
    split_a.release();
    split_b.release();
    part.release();
}

}  // namespace qg

void qg_release_gram_cache(qg_context c) {
    delete static_cast<qg::MixedGram*>(c->gram_cache);
    c->gram_cache = nullptr;
}

int qg_blas_handle(qg_context c, cublasHandle_t* out);

extern "C" {

int qg_gram_mixed_d(qg_context ctx, long long N, int m, const double* A, const double* B, double alpha, double* C,
                    int pieces) {
    if (!ctx || N <= 0 || m <= 0 || !A || !C || pieces < -1 || (pieces > 3 && pieces != qg::kI8Slices) ||
        pieces == 1)
        return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    cublasHandle_t blas;
    QG_TRY(qg_blas_handle(ctx, &blas));
    // the split buffers are kept on the context and rebuilt when the shape or split changes
    auto* g = static_cast<qg::MixedGram*>(ctx->gram_cache);
    if (!g || g->N != N || g->mmax < m || g->pieces != pieces) {
        qg_release_gram_cache(ctx);
        g = new qg::MixedGram();
        ctx->gram_cache = g;
        QG_TRY(g->setup(N, m, pieces));
    }
    if (pieces > 0 && !g->use_tc && !g->use_i8) return QG_ERR_UNSUPPORTED;
    QG_TRY(g->split(A, m, 0, ctx->stream));
    const bool same = (B == nullptr || B == A);
    if (!same) QG_TRY(g->split(B, m, 1, ctx->stream));
    QG_TRY(g->gram(blas, ctx->stream, m, same, false, alpha, C, m, ctx->dev_status));
    QG_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return qg_context_take_device_status(ctx);
}

}  // extern "C"
