// FP64 Gram blocks with the K dimension split over batched DGEMMs.
//
// The LOBPCG Gram products are tall-skinny: K = N grid points (1.7 M at 120^3) against
// 528-1584 columns. One DGEMM of a 1584 x 528 block has 65 output tiles for 148 SMs and
// runs at ~25 TFLOP/s; DSYRK(X) of the 1584^2 lower triangle costs as much as the full
// square. Here every block is split into K chunks, all chunks of all blocks go to one
// batched DGEMM (several waves of tiles), and one kernel adds each block's partials in
// chunk order -- fixed order, so the result does not depend on the run.
#include "gram_split.h"

#include <algorithm>
#include <cstdio>

namespace qg {

namespace {

__global__ void k_sum_chunks(const double* __restrict__ part, int parts, int nb, long long bmbn, int bm,
                             double alpha, double* const* __restrict__ dst, int ldc) {
    const int b = blockIdx.y;
    double* C = dst[b];
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < bmbn;
         e += (long long)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int c = 0; c < parts; ++c) s += part[((long long)c * nb + b) * bmbn + e];
        const long long i = e % bm, j = e / bm;
        C[i + j * ldc] = alpha * s;
    }
}

}  // namespace

int split_chunks(long long K, int bm, int bn, int nb) {
    const long long tiles = (long long)nb * ((bm + 127) / 128) * ((bn + 127) / 128);
    long long ks = (768 + tiles / 2) / std::max(tiles, 1LL);
    ks = std::min(ks, K / 16384);
    return (int)std::max(1LL, std::min(ks, 16LL));
}

int SplitTn::run(cublasHandle_t blas, cudaStream_t st, long long K, long long lda, int bm, int bn,
                 const std::vector<TnBlock>& blocks, int ldc, double alpha) {
    const int nb = (int)blocks.size();
    if (nb == 0 || bm <= 0 || bn <= 0 || K <= 0) return QG_ERR_INVALID;
    if (K > 0x7fffffffLL || lda > 0x7fffffffLL) return QG_ERR_UNSUPPORTED;
    const int ks = split_chunks(K, bm, bn, nb);
    long long Kc = K / ks;
    if (ks > 1) Kc &= ~31LL;  // chunk starts on 256-byte boundaries of each column
    const long long rem = K - ks * Kc;
    const int parts = ks + (rem > 0 ? 1 : 0);
    const long long bmbn = (long long)bm * bn;
    QG_TRY(part.reserve((size_t)parts * nb * bmbn * sizeof(double)));
    double* P = part.as<double>();
    // pointer arrays: main A/B/C (nb * ks each), remainder A/B/C (nb each), destinations (nb)
    const size_t nmain = (size_t)nb * ks, np = 3 * nmain + 3 * (size_t)nb + nb;
    std::vector<const void*> h(np);
    for (int c = 0; c < ks; ++c)
        for (int b = 0; b < nb; ++b) {
            const size_t e = (size_t)c * nb + b;
            h[e] = blocks[b].A + c * Kc;
            h[nmain + e] = blocks[b].B + c * Kc;
            h[2 * nmain + e] = P + ((long long)c * nb + b) * bmbn;
        }
    for (int b = 0; b < nb; ++b) {
        h[3 * nmain + b] = blocks[b].A + ks * Kc;
        h[3 * nmain + nb + b] = blocks[b].B + ks * Kc;
        h[3 * nmain + 2 * nb + b] = P + ((long long)ks * nb + b) * bmbn;
        h[3 * nmain + 3 * nb + b] = blocks[b].C;
    }
    QG_TRY(ptrs.reserve(np * sizeof(void*)));
    if (h != last || K != last_K) {
        // pageable source: the copy is staged before the call returns, so h may go
        QG_CUDA_TRY(cudaMemcpyAsync(ptrs.ptr, h.data(), np * sizeof(void*), cudaMemcpyHostToDevice, st));
        last = h;
        last_K = K;
    }
    const double* const* d = ptrs.as<const double* const>();
    const double one = 1.0, zero = 0.0;
    if (cublasSetStream(blas, st) != CUBLAS_STATUS_SUCCESS) return QG_ERR_LIBRARY;
    cublasStatus_t s = cublasDgemmBatched(blas, CUBLAS_OP_T, CUBLAS_OP_N, bm, bn, (int)Kc, &one, d, (int)lda,
                                          d + nmain, (int)lda, &zero, const_cast<double* const*>(d + 2 * nmain),
                                          bm, (int)nmain);
    if (s == CUBLAS_STATUS_SUCCESS && rem > 0)
        s = cublasDgemmBatched(blas, CUBLAS_OP_T, CUBLAS_OP_N, bm, bn, (int)rem, &one, d + 3 * nmain, (int)lda,
                               d + 3 * nmain + nb, (int)lda, &zero,
                               const_cast<double* const*>(d + 3 * nmain + 2 * nb), bm, nb);
    if (s != CUBLAS_STATUS_SUCCESS) {
        char m[32];
        snprintf(m, sizeof(m), "cublas status %d", (int)s);
        qg_set_last_error("cublasDgemmBatched", m, __FILE__, __LINE__);
        return QG_ERR_LIBRARY;
    }
    const unsigned gx = (unsigned)std::min<long long>((bmbn + 255) / 256, 1024);
    k_sum_chunks<<<dim3(gx, nb), 256, 0, st>>>(P, parts, nb, bmbn, bm, alpha,
                                                const_cast<double* const*>(d + 3 * nmain + 3 * nb), ldc);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

}  // namespace qg
