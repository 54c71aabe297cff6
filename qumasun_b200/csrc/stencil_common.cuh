// Definitions shared by the stencil kernels (hamiltonian.cu, stencil_tma.cu).
#pragma once
#include <cuda_runtime.h>

namespace qg {

template <typename T>
struct HamArgs {
    const T* X;
    long long ldx;
    T* HX;
    long long ldhx;
    int ns;
    const T* V;
    int nx, ny, nz;
    int ty;
    int zslab;
    T c0;
    T cx[4], cy[4], cz[4];
    // nonlocal scatter side (row == nullptr: no nonlocal term)
    const int* row;
    const int* ent_atom;
    const T* ent_val;
    int nch;
    int ncoef;       // na * nch
    const T* coef;   // [ns][ncoef]
    int* err;        // device status word: nonzero after a bounded wait gave up
};

__device__ __forceinline__ int wrap_idx(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}


template <typename T>
int launch_stencil_tma(const HamArgs<T>& a, int order, cudaStream_t st);
// True when launch_stencil_tma accepts this shape and alignment.
template <typename T>
bool stencil_tma_ok(const HamArgs<T>& a, int order);

}  // namespace qg
