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
    long long ldc;   // coefficient row length (states, padded to 16)
    const T* coef;   // [na * nch][ldc]
    int* err;        // device status word: nonzero after a bounded wait gave up
    int stall;       // test hook: the ring kernels' producer issues nothing, so the
                     // consumers' bounded waits run out (QG_ERR_TIMEOUT)
    // complex (k-point) states: the imaginary part of a state starts xim (hxim)
    // elements after its real part; dx/dy/dz are the 8th-order first-derivative
    // coefficients 2*coef*g/(840h)*(672, -168, 32, -3) per axis (zero for an
    // axis whose |g| < 1e-8), c0 then carries the -coef*|g|^2 term
    long long xim, hxim;
    T dx[4], dy[4], dz[4];
    // several k-points in one launch (NC = 2): states are grouped by k, nsk per k;
    // state s of k-point k starts at X + k*ldkx + s*ldx (HX + k*ldkhx + s*ldhx), and
    // kco[k*13 + {0, 1..4, 5..8, 9..12}] replaces c0, dx, dy, dz (nsk = 0: one k-point)
    int nsk;
    long long ldkx, ldkhx;
    const T* kco;
};

// first element of global state index s (k-point major when several k-points share a launch)
template <typename T>
__device__ __forceinline__ long long state_offset(const HamArgs<T>& a, int s, bool out) {
    if (a.nsk <= 0) return (long long)s * (out ? a.ldhx : a.ldx);
    const int k = s / a.nsk, sl = s - k * a.nsk;
    return out ? (long long)k * a.ldkhx + (long long)sl * a.ldhx : (long long)k * a.ldkx + (long long)sl * a.ldx;
}

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
// Real states, two output planes per consumer step (stencil_pair.cu).
template <typename T>
int launch_stencil_pair(const HamArgs<T>& a, int order, cudaStream_t st);
template <typename T>
bool stencil_pair_ok(const HamArgs<T>& a, int order);
// Real states, two grid rows per consumer thread, V streamed through the ring (vring) or
// read one plane ahead from global memory (stencil_rows.cu).
template <typename T>
int launch_stencil_rows(const HamArgs<T>& a, int order, cudaStream_t st, bool vring = true);
template <typename T>
bool stencil_rows_ok(const HamArgs<T>& a, int order, bool vring = true);

}  // namespace qg
