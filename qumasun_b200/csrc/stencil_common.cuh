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
    // complex (k-point) states: the imaginary part of a state starts xim (hxim)
    // elements after its real part; dx/dy/dz are the 8th-order first-derivative
    // coefficients 2*coef*g/(840h)*(672, -168, 32, -3) per axis (zero for an
    // axis whose |g| < 1e-8), c0 then carries the -coef*|g|^2 term
    long long xim, hxim;
    T dx[4], dy[4], dz[4];
};

__device__ __forceinline__ int wrap_idx(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}


// nc = 1: real states; nc = 2: complex k-point states (order 8 only).
template <typename T>
int launch_stencil_tma(const HamArgs<T>& a, int order, cudaStream_t st, int nc = 1);
// True when launch_stencil_tma accepts this shape and alignment.
template <typename T>
bool stencil_tma_ok(const HamArgs<T>& a, int order, int nc = 1);

}  // namespace qg
