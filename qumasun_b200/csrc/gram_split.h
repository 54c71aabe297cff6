// FP64 Gram blocks of tall blocks with the row (K) dimension split over
// batched DGEMMs and the chunk partials added in chunk order (gram_split.cu).
#pragma once
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <vector>

#include "qg_internal.h"

namespace qg {

// One output block: C (bm x bn, column-major, ldc of the call) = alpha A^T B,
// A: K x bm and B: K x bn, column-major with the call's lda.
struct TnBlock {
    const double* A;
    const double* B;
    double* C;
};

// Chunk count for nb blocks of bm x bn over K rows: enough 128 x 128 output tiles
// times chunks to fill the GPU several times over (cuBLAS alone leaves most SMs idle
// at the LOBPCG shapes, e.g. 65 tiles for a 1584 x 528 block), chunks of at least 16k rows.
int split_chunks(long long K, int bm, int bn, int nb);

// Runs the blocks of one shape: the K rows cut into `split_chunks` chunks (the last
// rows into one more chunk when K does not divide), one cublasDgemmBatched per chunk
// length into partial blocks, then one kernel that adds each block's partials in
// chunk order and scales by alpha. The pointer arrays are uploaded only when they
// change, so a solver calling with the same blocks every iteration uploads once.
struct SplitTn {
    DevBuf part, ptrs;
    std::vector<const void*> last;  // pointer arrays of the last upload
    long long last_K = -1;
    int run(cublasHandle_t blas, cudaStream_t st, long long K, long long lda, int bm, int bn,
            const std::vector<TnBlock>& blocks, int ldc, double alpha);
    void release() {
        part.release();
        ptrs.release();
        last.clear();
        last_K = -1;
    }
};

}  // namespace qg
