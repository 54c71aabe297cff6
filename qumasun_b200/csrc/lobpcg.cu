// Block LOBPCG on the GPU, FP64 (EigenLOBPCG_d_multi, lobpcg_d_multi.h:23-545;
// complex states: Eigen_z_multi_mpi, lobpcg_z_multi_mpi.h:988-1800).
//
// Blocks live on the device as column-major N x n arrays (= the reference's
// state-major layout, one state per column; a split-complex state is two
// consecutive columns {re, im}):
//   W  = [x | r | p]      (3n columns, contiguous)
//   AW = [Ax | Ar | Ap]
//   T  = [x_new | p_new]  (rotation outputs)
// One iteration:
//   Ar = H r                                       (qg::apply_hamiltonian / _z)
//   Sa = W^T AW dV, Sb = W^T W dV                  (lower-triangle blocks of a K-split batched DGEMM;
//                                                   DGEMM for complex; w_dgemm path, lobpcg_d_multi_mpi.h:191-250)
//   Sa z = lambda Sb z, k = 3n (2n on the first step of a first call), Jacobi-equilibrated,
//   cusolverDnDsygvd / Zhegvd (replaces DSYGVX / ZHEGVX, w_dsygvx.h:24-104, UPLO as the
//   reference); if B is not positive definite the step is solved on B's nonsingular subspace
//   p_new = [r p] [Cr; Cp], x_new = x Cx + p_new   (DGEMM; lobpcg_d_multi.h:247-300)
//   renormalise x and p (:491-505); Ax = H x_new, Ap = H p_new (re-applied, not rotated);
//   ei = x.Ax dV; r = Ax - ei x (:506-512)
//   stop when max_j sum r_j^2 dV < tol dV over the lowest n_converge states (:525).
// Column reductions (norms, dots, residuals) are project kernels with one
// block per column and a fixed reduction order (deterministic).
#include <cublas_v2.h>
#include <cusolverDn.h>
#include <cuComplex.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <thread>
#include <vector>

#include "gram_mixed.h"
#include "gram_split.h"
#include "gram_ts.h"
#include "precond.h"
#include "qg_internal.h"
#include "small_eig.h"

#define QG_BLAS_TRY(expr)                                                                   \
    do {                                                                                    \
        cublasStatus_t qg_b_ = (expr);                                                      \
        if (qg_b_ != CUBLAS_STATUS_SUCCESS) {                                               \
            char m_[32];                                                                    \
            snprintf(m_, sizeof(m_), "cublas status %d", (int)qg_b_);                       \
            qg_set_last_error(#expr, m_, __FILE__, __LINE__);                               \
            return QG_ERR_LIBRARY;                                                          \
        }                                                                                   \
    } while (0)

#define QG_SOLVER_TRY(expr)                                                                 \
    do {                                                                                    \
        cusolverStatus_t qg_v_ = (expr);                                                    \
        if (qg_v_ != CUSOLVER_STATUS_SUCCESS) {                                             \
            char m_[32];                                                                    \
            snprintf(m_, sizeof(m_), "cusolver status %d", (int)qg_v_);                     \
            qg_set_last_error(#expr, m_, __FILE__, __LINE__);                               \
            return QG_ERR_LIBRARY;                                                          \
        }                                                                                   \
    } while (0)

int qg_blas_handle(qg_context c, cublasHandle_t* out) {
    if (!c->blas) {
        cublasHandle_t h;
        QG_BLAS_TRY(cublasCreate(&h));
        c->blas = h;
    }
    cublasHandle_t h = static_cast<cublasHandle_t>(c->blas);
    QG_BLAS_TRY(cublasSetStream(h, c->stream));
    QG_BLAS_TRY(cublasSetMathMode(h, CUBLAS_DEFAULT_MATH));
    *out = h;
    return QG_OK;
}

int qg_solver_handle(qg_context c, cusolverDnHandle_t* out) {
    if (!c->solver) {
        cusolverDnHandle_t h;
        QG_SOLVER_TRY(cusolverDnCreate(&h));
        c->solver = h;
    }
    cusolverDnHandle_t h = static_cast<cusolverDnHandle_t>(c->solver);
    QG_SOLVER_TRY(cusolverDnSetStream(h, c->stream));
    *out = h;
    return QG_OK;
}

namespace {

constexpr int kRedThreads = 512;

__device__ __forceinline__ double block_sum(double v) {
    __shared__ double red[kRedThreads / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w];
    }
    return s;  // valid in thread 0
}

// out[j] = scale * sum_i A[j][i] * B[j][i]
__global__ void __launch_bounds__(kRedThreads) k_coldot(const double* __restrict__ A, const double* __restrict__ B,
                                                        long long ld, long long N, double scale,
                                                        double* __restrict__ out) {
    const double* a = A + (long long)blockIdx.x * ld;
    const double* b = B + (long long)blockIdx.x * ld;
    double s = 0.0;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) s += a[i] * b[i];
    s = block_sum(s);
    if (threadIdx.x == 0) out[blockIdx.x] = s * scale;
}

// A[j][:] *= f[j] for the columns of up to two blocks sharing the factors
__global__ void k_scale_cols(double* __restrict__ A, double* __restrict__ B, long long ld, long long N,
                             const double* __restrict__ f) {
    const int j = blockIdx.y;
    const double c = f[j];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        A[(long long)j * ld + i] *= c;
        if (B) B[(long long)j * ld + i] *= c;
    }
}

// dst_j = f_j src_j: the copy of a rotated block and its normalisation in one pass (the
// same product as scaling the copy in place)
__global__ void k_scale_copy(double* __restrict__ dst, const double* __restrict__ src, long long ld, long long N,
                             const double* __restrict__ f) {
    const int j = blockIdx.y;
    const double c = f[j];
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        dst[(long long)j * ld + i] = src[(long long)j * ld + i] * c;
}

// f[j] = 1 / sqrt(norm2[j] * dV)   (Normalize, vecmath.h:128-133)
__global__ void k_inv_norm(const double* __restrict__ norm2, double dV, int n, double* __restrict__ f) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) f[j] = norm2[j] > 0.0 ? 1.0 / sqrt(norm2[j] * dV) : 0.0;  // a zero column stays zero
}

// r_j = Ax_j - ei_j x_j and nr[j] = dV * sum_i r_j(i)^2   (lobpcg_d_multi.h:506-516)
__global__ void __launch_bounds__(kRedThreads) k_residual(const double* __restrict__ Ax, const double* __restrict__ x,
                                                          const double* __restrict__ ei, double* __restrict__ r,
                                                          long long ld, long long N, double dV,
                                                          double* __restrict__ nr) {
    const long long off = (long long)blockIdx.x * ld;
    const double e = ei[blockIdx.x];
    double s = 0.0;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) {
        const double v = Ax[off + i] - e * x[off + i];
        r[off + i] = v;
        s += v * v;
    }
    s = block_sum(s);
    if (threadIdx.x == 0) nr[blockIdx.x] = s * dV;
}

// A2 = D A D, B2 = D B D on the leading k x k block (column-major, ld), D = diag(B)^-1/2;
// one block per column
__global__ void k_equilibrate(const double* __restrict__ A, const double* __restrict__ B, int ld, int k,
                              double* __restrict__ A2, double* __restrict__ B2) {
    const int j = blockIdx.x;
    const double bj = B[j + (long long)j * ld];
    const double dj = bj > 0.0 ? 1.0 / sqrt(bj) : 1.0;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double bi = B[i + (long long)i * ld];
        const double s = (bi > 0.0 ? 1.0 / sqrt(bi) : 1.0) * dj;
        A2[i + (long long)j * ld] = A[i + (long long)j * ld] * s;
        B2[i + (long long)j * ld] = B[i + (long long)j * ld] * s;
    }
}

// Z(i, j) *= diag(B)(i)^-1/2 for rows i < k of the first gridDim.x columns
__global__ void k_rowscale(double* __restrict__ Z, int ld, int k, const double* __restrict__ B, int ldb) {
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double bi = B[i + (long long)i * ldb];
        Z[i + (long long)j * ld] *= bi > 0.0 ? 1.0 / sqrt(bi) : 1.0;
    }
}

// Complex Gram: S(i, j) = <w_i|A w_j> from the real Gram G = W^T AW of the split
// layout (lobpcg_z_multi_mpi.h:214-300: S = (RR + II) + i (RI - IR)), Jacobi-
// equilibrated by d = diag(B)^-1/2 like k_equilibrate; leading k x k block,
// one block per column j.
__global__ void k_gram_to_complex(const double* __restrict__ Ga, const double* __restrict__ Gb, int ldg, int k,
                                  cuDoubleComplex* __restrict__ Ca, cuDoubleComplex* __restrict__ Cb, int ldc) {
    const int j = blockIdx.x;
    auto G = [ldg](const double* M, int r, int c) { return M[r + (long long)c * ldg]; };
    auto dinv = [&](int i) {
        const double b = G(Gb, 2 * i, 2 * i) + G(Gb, 2 * i + 1, 2 * i + 1);
        return b > 0.0 ? 1.0 / sqrt(b) : 1.0;
    };
    const double dj = dinv(j);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double s = dinv(i) * dj;
        const double ar = G(Ga, 2 * i, 2 * j) + G(Ga, 2 * i + 1, 2 * j + 1);
        const double ai = G(Ga, 2 * i, 2 * j + 1) - G(Ga, 2 * i + 1, 2 * j);
        const double br = G(Gb, 2 * i, 2 * j) + G(Gb, 2 * i + 1, 2 * j + 1);
        const double bi = G(Gb, 2 * i, 2 * j + 1) - G(Gb, 2 * i + 1, 2 * j);
        Ca[i + (long long)j * ldc] = make_cuDoubleComplex(ar * s, ai * s);
        Cb[i + (long long)j * ldc] = make_cuDoubleComplex(br * s, bi * s);
    }
}

// Real rotation matrix of the split layout from the complex eigenvectors:
// z = D z' (D as in k_gram_to_complex, rows >= krows zero), then
// M(2i, 2j) = M(2i+1, 2j+1) = Re z(i, j), M(2i, 2j+1) = Im z(i, j), M(2i+1, 2j) = -Im z(i, j),
// so that [re | im] columns times M give the complex product X z. One block per column j < n.
__global__ void k_expand_rotation(const cuDoubleComplex* __restrict__ Z, int ldz, int k, int krows,
                                  const double* __restrict__ Gb, int ldg, double* __restrict__ M, int ldm) {
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        double zr = 0.0, zi = 0.0;
        if (i < krows) {
            const double b = Gb[2 * i + (long long)(2 * i) * ldg] + Gb[2 * i + 1 + (long long)(2 * i + 1) * ldg];
            const double d = b > 0.0 ? 1.0 / sqrt(b) : 1.0;
            const cuDoubleComplex z = Z[i + (long long)j * ldz];
            zr = cuCreal(z) * d;
            zi = cuCimag(z) * d;
        }
        M[2 * i + (long long)(2 * j) * ldm] = zr;
        M[2 * i + 1 + (long long)(2 * j + 1) * ldm] = zr;
        M[2 * i + (long long)(2 * j + 1) * ldm] = zi;
        M[2 * i + 1 + (long long)(2 * j) * ldm] = -zi;
    }
}

// Batched over k-points (blockIdx.y): the pencils of k-point kb at Ga/Gb + kb*gstride
// into Ca/Cb + kb*cstride; k-points with skip[kb] set are left alone.
__global__ void k_gram_to_complex_b(const double* __restrict__ Ga, const double* __restrict__ Gb, int ldg,
                                    long long gstride, int k, cuDoubleComplex* __restrict__ Ca,
                                    cuDoubleComplex* __restrict__ Cb, int ldc, long long cstride,
                                    const int* __restrict__ skip) {
    const int kb = blockIdx.y;
    if (skip[kb]) return;
    const int j = blockIdx.x;
    Ga += kb * gstride;
    Gb += kb * gstride;
    Ca += kb * cstride;
    Cb += kb * cstride;
    auto G = [ldg](const double* M, int r, int c) { return M[r + (long long)c * ldg]; };
    auto dinv = [&](int i) {
        const double b = G(Gb, 2 * i, 2 * i) + G(Gb, 2 * i + 1, 2 * i + 1);
        return b > 0.0 ? 1.0 / sqrt(b) : 1.0;
    };
    const double dj = dinv(j);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double sc = dinv(i) * dj;
        const double ar = G(Ga, 2 * i, 2 * j) + G(Ga, 2 * i + 1, 2 * j + 1);
        const double ai = G(Ga, 2 * i, 2 * j + 1) - G(Ga, 2 * i + 1, 2 * j);
        const double br = G(Gb, 2 * i, 2 * j) + G(Gb, 2 * i + 1, 2 * j + 1);
        const double bi = G(Gb, 2 * i, 2 * j + 1) - G(Gb, 2 * i + 1, 2 * j);
        Ca[i + (long long)j * ldc] = make_cuDoubleComplex(ar * sc, ai * sc);
        Cb[i + (long long)j * ldc] = make_cuDoubleComplex(br * sc, bi * sc);
    }
}

// k_expand_rotation batched over k-points (blockIdx.y); a k-point with skip[kb] set
// gets the identity rotation (its states stay as they are).
__global__ void k_expand_rotation_b(const cuDoubleComplex* __restrict__ Z, int ldz, long long zstride, int k,
                                    const double* __restrict__ Gb, int ldg, long long gstride, double* __restrict__ M,
                                    int ldm, long long mstride, const int* __restrict__ skip) {
    const int kb = blockIdx.y;
    const int j = blockIdx.x;
    M += kb * mstride;
    if (skip[kb]) {
        for (int i = threadIdx.x; i < 2 * k; i += blockDim.x) {
            M[i + (long long)(2 * j) * ldm] = (i == 2 * j) ? 1.0 : 0.0;
            M[i + (long long)(2 * j + 1) * ldm] = (i == 2 * j + 1) ? 1.0 : 0.0;
        }
        return;
    }
    Z += kb * zstride;
    Gb += kb * gstride;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double b = Gb[2 * i + (long long)(2 * i) * ldg] + Gb[2 * i + 1 + (long long)(2 * i + 1) * ldg];
        const double d = b > 0.0 ? 1.0 / sqrt(b) : 1.0;
        const cuDoubleComplex z = Z[i + (long long)j * ldz];
        const double zr = cuCreal(z) * d, zi = cuCimag(z) * d;
        M[2 * i + (long long)(2 * j) * ldm] = zr;
        M[2 * i + 1 + (long long)(2 * j + 1) * ldm] = zr;
        M[2 * i + (long long)(2 * j + 1) * ldm] = zi;
        M[2 * i + 1 + (long long)(2 * j) * ldm] = -zi;
    }
}

// Fills the upper triangle of the leading k x k block from the lower one
// (conjugated for complex entries); one block per column j.
template <typename T>
__global__ void k_mirror_lower(T* __restrict__ A, int ld, int k) {
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < j; i += blockDim.x) {
        const T v = A[j + (long long)i * ld];
        if constexpr (sizeof(T) == 16) A[i + (long long)j * ld] = cuConj(v);
        else A[i + (long long)j * ld] = v;
    }
}

// Steady-state Gram pencil of [x r p] (column-major, pitch k3 = 3n, lower triangle read
// by the eigensolvers): the x/p blocks come from the previous iteration's rotation,
// U = [Bxx | Bxp | Bpp] (n x n each, ld n, before normalisation) scaled by the
// normalisation factors fx (of x) and fp (of p):
//   S(x,x) = fx Bxx fx,  S(p,x) = fp Bxp^T fx,  S(p,p) = fp Bpp fp;
// the r column block was just formed from tall products; its x rows are copied into
// the (r,x) block of the lower triangle. One block per column j < n.
__global__ void k_place_blocks(double* __restrict__ S, int k3, int n, const double* __restrict__ U,
                               const double* __restrict__ fx, const double* __restrict__ fp) {
    const int j = blockIdx.x;
    const double* Bxx = U;
    const double* Bxp = U + (size_t)n * n;
    const double* Bpp = U + 2 * (size_t)n * n;
    const double fxj = fx[j], fpj = fp[j];
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const double xx = fx[i] * Bxx[i + (size_t)j * n] * fxj;
        S[i + (size_t)j * k3] = xx;
        S[(2 * n + i) + (size_t)j * k3] = fp[i] * Bxp[j + (size_t)i * n] * fxj;                 // p_i . x_j
        S[(2 * n + i) + (size_t)(2 * n + j) * k3] = fp[i] * Bpp[i + (size_t)j * n] * fpj;
        S[(n + i) + (size_t)j * k3] = S[j + (size_t)(n + i) * k3];                               // r_i . x_j
    }
}

// T(:, j) = V(:, f + j) / sqrt(s[f + j]) for the kp eigenvectors of B kept.
template <typename T>
__global__ void k_scaled_basis(const T* __restrict__ V, int ld, int k, const double* __restrict__ s, int f,
                               T* __restrict__ Tm) {
    const int j = blockIdx.x;
    const double sc = 1.0 / sqrt(s[f + j]);
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const T v = V[i + (long long)(f + j) * ld];
        if constexpr (sizeof(T) == 16) Tm[i + (long long)j * ld] = make_cuDoubleComplex(cuCreal(v) * sc, cuCimag(v) * sc);
        else Tm[i + (long long)j * ld] = v * sc;
    }
}

// Rotation of a k-point whose states have converged: x_new = x, p_new = 0
// (M = [I; 0; 0], 2k3 x 2nb, ld g); one block per column.
__global__ void k_freeze_rotation(double* __restrict__ M, int g, int rows) {
    const int j = blockIdx.x;
    for (int i = threadIdx.x; i < rows; i += blockDim.x) M[i + (long long)j * g] = (i == j) ? 1.0 : 0.0;
}

struct Timer {
    cudaEvent_t ev[16];
    int n = 0;
    double acc[6] = {0, 0, 0, 0, 0, 0};
    int tag[16];
    bool ok = true;
    Timer() {
        for (auto& e : ev)
            if (cudaEventCreate(&e) != cudaSuccess) ok = false;
    }
    ~Timer() {
        for (auto e : ev) cudaEventDestroy(e);
    }
    void mark(int t, cudaStream_t st) {
        if (n < 16) {
            cudaEventRecord(ev[n], st);
            tag[n++] = t;
        }
    }
    void flush() {  // call after the stream has reached the last mark
        for (int i = 0; i + 1 < n; ++i) {
            float d = 0.f;
            cudaEventElapsedTime(&d, ev[i], ev[i + 1]);
            if (tag[i] >= 0 && tag[i] < 6) acc[tag[i]] += d;
        }
        n = 0;
    }
};

// One LOBPCG instance. c = 1: real states (columns of N); c = 2: split-complex
// states, each {re[N], im[N]} = two consecutive real columns, so every block is
// also a real N x (c n) matrix for the Gram and rotation DGEMMs, and a state is
// one contiguous "column" of L = c N values for norms, dots and residuals.
struct Solver {
    qg_hamiltonian h;
    int n, c;
    long long N, L;
    double dV;
    cudaStream_t st;
    cublasHandle_t blas;
    cusolverDnHandle_t sol;
    DevBuf W, AW, T, S, E, small, work, heg;  // heg: batched complex pencils (k-point solve)
    DevBuf gts;                                // partial sums of the tall-skinny Gram kernel
    DevBuf upd;                                // steady-state Gram reuse: blocks, products, factors
    qg::SplitTn sp_full, sp_upd;               // K-split batched Gram products (full pencil, r blocks)
    double *UA = nullptr, *UB = nullptr, *Tu = nullptr, *fx_d = nullptr, *fp_d = nullptr;
    bool have_update = false;                  // UA/UB hold the rotated x/p blocks of the last step
    int nblk = 3;                              // blocks of W: [x r p], or [x r q p] with the learned block q
    double *q = nullptr, *Aq = nullptr;        // the learned block (nblk = 4)
    int lwork = 0;
    double *x, *r, *p, *Ax, *Ar, *Ap, *Tx, *Tp, *Sa, *Sb, *Sa2, *Sb2, *M;
    double* E0;  // rank-revealing solve scratch: basis, product, reduced pencil, vectors (k3 x k3 each)
    std::vector<double> s_h;
    bool mixed = false;      // reduced-precision Gram products (qg::MixedGram) until the hand-over
    bool i8 = false;         // FP64-accurate Gram products on the int8 tensor cores (QG_FP64_INT8)
    int mixed_pieces = 3;    // qg::MixedGram split: 3 = split-BF16x3 on tcgen05, -1 = FP32
    double trunc_eps = 1e-12;  // relative eigenvalue floor of B in the rank-revealing solve
    qg::MixedGram mg;
    cuDoubleComplex *Ca, *Cb;
    double *ev_d, *nr_d, *f_d, *f2_d, *w_d;
    int* info_d;

    ~Solver() {
        W.release(); AW.release(); T.release(); S.release(); E.release(); small.release();
        work.release(); heg.release(); gts.release(); upd.release();
        sp_full.release(); sp_upd.release();
    }

    int setup() {
        const size_t blk = (size_t)L * n;
        QG_TRY(W.reserve(nblk * blk * sizeof(double)));
        QG_TRY(AW.reserve(nblk * blk * sizeof(double)));
        QG_TRY(T.reserve(2 * blk * sizeof(double)));
        const size_t k3 = (size_t)nblk * n, g3 = c * k3;  // the largest pencil
        // real Gram pair (c k3)^2 each; the equilibrated pencil (k3^2 real or complex each);
        // for c = 2 the real rotation matrix (2 k3 x 2 n)
        QG_TRY(S.reserve((2 * g3 * g3 + 2 * c * k3 * k3 + (c == 2 ? g3 * 2 * n : 0)) * sizeof(double)));
        QG_TRY(small.reserve((5 * k3 + 16) * sizeof(double)));
        QG_TRY(E.reserve(4 * (size_t)c * k3 * k3 * sizeof(double)));
        E0 = E.as<double>();
        s_h.resize(k3);
        x = W.as<double>(); r = x + blk; p = r + (nblk - 2) * blk;
        Ax = AW.as<double>(); Ar = Ax + blk; Ap = Ar + (nblk - 2) * blk;
        if (nblk == 4) {
            q = r + blk;
            Aq = Ar + blk;
        }
        Tx = T.as<double>(); Tp = Tx + blk;
        Sa = S.as<double>(); Sb = Sa + g3 * g3; Sa2 = Sb + g3 * g3; Sb2 = Sa2 + c * k3 * k3;
        M = Sb2 + c * k3 * k3;
        // the triangle DSYRK(X) leaves unwritten stays finite (zero)
        QG_CUDA_TRY(cudaMemsetAsync(S.ptr, 0, S.bytes, st));
        Ca = reinterpret_cast<cuDoubleComplex*>(Sa2);
        Cb = reinterpret_cast<cuDoubleComplex*>(Sb2);
        ev_d = small.as<double>(); nr_d = ev_d + k3; f_d = nr_d + k3; f2_d = f_d + k3; w_d = f2_d + k3;
        info_d = reinterpret_cast<int*>(w_d + k3);
        if (c == 1) {
            QG_SOLVER_TRY(cusolverDnDsygvd_bufferSize(sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                      CUBLAS_FILL_MODE_LOWER, (int)k3, Sa2, (int)k3, Sb2, (int)k3,
                                                      w_d, &lwork));
            int lw2 = 0;
            QG_SOLVER_TRY(cusolverDnDsyevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)k3,
                                                      Sb2, (int)k3, w_d, &lw2));
            lwork = std::max(lwork, lw2);
            QG_TRY(work.reserve((size_t)std::max(lwork, 1) * sizeof(double)));
        } else {
            QG_SOLVER_TRY(cusolverDnZhegvd_bufferSize(sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                      CUBLAS_FILL_MODE_LOWER, (int)k3, Ca, (int)k3, Cb, (int)k3,
                                                      w_d, &lwork));
            int lw2 = 0;
            QG_SOLVER_TRY(cusolverDnZheevd_bufferSize(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, (int)k3,
                                                      Cb, (int)k3, w_d, &lw2));
            lwork = std::max(lwork, lw2);
            QG_TRY(work.reserve((size_t)std::max(lwork, 1) * sizeof(cuDoubleComplex)));
        }
        QG_TRY(h->coef.reserve((c == 1 ? qg::coef_scratch_elems(h, n) : qg::coef_scratch_elems_z(h, 1, n)) *
                               sizeof(double)));
        if (mixed) QG_TRY(mg.setup(N, (int)g3, mixed_pieces));
        if (i8 && c == 1) QG_TRY(mg.setup(N, (int)g3, qg::kI8Slices));
        if (c == 1) {
            const size_t nn = (size_t)n * n;
            QG_TRY(upd.reserve((6 * nn + 2 * k3 * (size_t)n + 2 * (size_t)n) * sizeof(double)));
            UA = upd.as<double>();
            UB = UA + 3 * nn;
            Tu = UB + 3 * nn;
            fx_d = Tu + 2 * k3 * (size_t)n;
            fp_d = fx_d + n;
        }
        return QG_OK;
    }

    // Gram pencil of the steady-state step from the previous rotation (the "direct
    // update" of NextMatrix_d, lobpcg_d_multi_mpi.h:264-460): only the r column block is
    // a tall product, W^T Ar dV and W^T r dV over W = [x r p] (2 * 2 N 3n n flops against
    // 2 N (3n)^2 for the full lower triangles); the x/p blocks come from prepare_update.
    int gram_update(int k3) {
        if (i8) {
            // [x r p]^T Ar and [x r p]^T r (the A side's own columns n .. 2n-1) on the int8 path
            QG_TRY(mg.split(x, k3, 0, st));
            QG_TRY(mg.split(Ar, n, 1, st));
            QG_TRY(mg.gram_rect(st, k3, n, 1, 0, dV, Sa + (size_t)n * k3, k3, h->ctx->dev_status));
            QG_TRY(mg.gram_rect(st, k3, n, 0, n, dV, Sb + (size_t)n * k3, k3, h->ctx->dev_status));
        } else {
            const std::vector<qg::TnBlock> blocks{{x, Ar, Sa + (size_t)n * k3}, {x, r, Sb + (size_t)n * k3}};
            QG_TRY(sp_upd.run(blas, st, N, N, k3, n, blocks, k3, dV));
        }
        k_place_blocks<<<n, 128, 0, st>>>(Sa, k3, n, UA, fx_d, fp_d);
        k_place_blocks<<<n, 128, 0, st>>>(Sb, k3, n, UB, fx_d, fp_d);
        QG_CUDA_TRY(cudaGetLastError());
        return QG_OK;
    }

    // After a pencil solve on the k3 x k3 pair (Sa, Sb, lower triangles, pitch k3) with
    // rotation Z (k3 x n, ld ldz; rows x, r[, p]): the pair of the rotated blocks
    // x' = [x r p] Z and p' = [r p] Z(n:, :) before normalisation,
    //   Bxx = Z^T S Z,  Bxp = Z^T S(:, n:) Z(n:, :),  Bpp = Z(n:, :)^T S(n:, n:) Z(n:, :),
    // for S = Sa (into UA) and S = Sb (into UB).
    int prepare_update(const double* Z, int ldz, int k3) {
        const double one = 1.0, zero = 0.0;
        const int kr = k3 - n;
        const size_t nn = (size_t)n * n;
        for (int w = 0; w < 2; ++w) {
            double* S = w ? Sb : Sa;
            double* U = w ? UB : UA;
            k_mirror_lower<double><<<k3, 128, 0, st>>>(S, k3, k3);
            double* T1 = Tu;
            double* T2 = Tu + (size_t)k3 * n;
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, k3, n, k3, &one, S, k3, Z, ldz, &zero, T1, k3));
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, k3, n, kr, &one, S + (size_t)n * k3, k3, Z + n, ldz,
                                    &zero, T2, k3));
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, k3, &one, Z, ldz, T1, k3, &zero, U, n));
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, k3, &one, Z, ldz, T2, k3, &zero, U + nn, n));
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, n, n, kr, &one, Z + n, ldz, T2 + n, k3, &zero,
                                    U + 2 * nn, n));
        }
        QG_CUDA_TRY(cudaGetLastError());
        return QG_OK;
    }

    int applyH(const double* in, double* out) {
        if (c == 1) return qg::apply_hamiltonian<double>(h, n, in, N, out, N, h->coef.as<double>(), st);
        return qg::apply_hamiltonian_z(h, n, in, L, out, L, h->coef.as<double>(), st);
    }

    void coldot(const double* A, const double* B, double scale, double* out) {
        k_coldot<<<n, kRedThreads, 0, st>>>(A, B, L, L, scale, out);
    }

    void scale_cols(double* A, double* B) {
        dim3 g((unsigned)std::min<long long>((L + 255) / 256, 64), n);
        k_scale_cols<<<g, 256, 0, st>>>(A, B, L, L, f_d);
    }

    // scale states of A (and B) by 1/sqrt(|A_j|^2 dV) computed from A
    void normalize(double* A, double* B) {
        coldot(A, A, 1.0, nr_d);
        k_inv_norm<<<(n + 127) / 128, 128, 0, st>>>(nr_d, dV, n, f_d);
        scale_cols(A, B);
    }

    // dst = src scaled by f_d, state by state
    void scale_copy(double* dst, const double* src) {
        dim3 g((unsigned)std::min<long long>((L + 255) / 256, 64), n);
        k_scale_copy<<<g, 256, 0, st>>>(dst, src, L, L, f_d);
    }

    // dst = src / sqrt(|src_j|^2 dV): the copy of a rotated block and its normalisation
    void normalize_from(double* dst, const double* src) {
        coldot(src, src, 1.0, nr_d);
        k_inv_norm<<<(n + 127) / 128, 128, 0, st>>>(nr_d, dV, n, f_d);
        scale_copy(dst, src);
    }

    void residual() {
        k_residual<<<n, kRedThreads, 0, st>>>(Ax, x, ev_d, r, L, L, dV, nr_d);
    }

    // C (m x nn, ldc) = alpha * A^T B, A: N x m, B: N x nn (ld N)
    int gemm_tn(int m, int nn, const double* A, const double* B, double alpha, double* C, int ldc) {
        const double beta = 0.0;
        QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, m, nn, (int)N, &alpha, A, (int)N, B, (int)N, &beta,
                                C, ldc));
        return QG_OK;
    }

    // Sa = W^T AW dV, Sb = W^T W dV over the leading m real columns. For real
    // states both are symmetric and only their lower triangles are formed, as n x n
    // blocks of one K-split batched DGEMM (qg::SplitTn; DSYRKX / DSYRK, which cost as
    // much as the full squares at these shapes, only for m not a multiple of n; the
    // eigensolvers read the lower triangle);
    // the split-complex Gram is not symmetric column by column, so it takes full DGEMMs.
    int gram(int m) {
        if (mixed) {
            QG_TRY(mg.split(x, m, 0, st));
            QG_TRY(mg.split(Ax, m, 1, st));
            QG_TRY(mg.gram(blas, st, m, false, c == 1, dV, Sa, m, h->ctx->dev_status));
            QG_TRY(mg.gram(blas, st, m, true, c == 1, dV, Sb, m, h->ctx->dev_status));
            return QG_OK;
        }
        if (c == 1 && m <= qg::kGramTsUpTo) {
            // small real pencils: K split over the GPU (cuBLAS's DSYRK took 3.5 ms per
            // iteration at 48 columns x 64k rows; complex pencils measured faster on cuBLAS)
            QG_TRY(gts.reserve(qg::gram_ts_scratch_doubles(N, 1, true) * sizeof(double)));
            return qg::gram_ts_tiled(x, N, 0, Ax, x, N, 0, N, m, m, dV, Sa, Sb, m, 0, 1, gts.as<double>(), st);
        }
        if (c == 2) {
            QG_TRY(gemm_tn(m, m, x, Ax, dV, Sa, m));
            return gemm_tn(m, m, x, x, dV, Sb, m);
        }
        if (i8) {
            // lower triangles from the int8 Ozaki products (gram_i8.cu): as accurate as DGEMM
            QG_TRY(mg.split(x, m, 0, st));
            QG_TRY(mg.split(Ax, m, 1, st));
            QG_TRY(mg.gram(blas, st, m, false, true, dV, Sa, m, h->ctx->dev_status));
            return mg.gram(blas, st, m, true, true, dV, Sb, m, h->ctx->dev_status);
        }
        if (m % n == 0) {
            // lower triangles in n x n blocks, K split over one batched DGEMM
            const int q = m / n;
            std::vector<qg::TnBlock> blocks;
            for (int j = 0; j < q; ++j)
                for (int i = j; i < q; ++i) {
                    const size_t off = (size_t)i * n + (size_t)j * n * m;
                    blocks.push_back({x + (size_t)i * n * N, Ax + (size_t)j * n * N, Sa + off});
                    blocks.push_back({x + (size_t)i * n * N, x + (size_t)j * n * N, Sb + off});
                }
            return sp_full.run(blas, st, N, N, n, n, blocks, m, dV);
        }
        const double beta = 0.0;
        QG_BLAS_TRY(cublasDsyrkx(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, m, (int)N, &dV, x, (int)N, Ax, (int)N,
                                 &beta, Sa, m));
        QG_BLAS_TRY(cublasDsyrk(blas, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, m, (int)N, &dV, x, (int)N, &beta, Sb, m));
        return QG_OK;
    }

    // C (N x nc) = A (N x k) * Z (k x nc, ldz) + beta C
    int gemm_nn(int k, int nc, const double* A, const double* Z, int ldz, double* C, double beta) {
        const double one = 1.0;
        QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)N, nc, k, &one, A, (int)N, Z, ldz, &beta, C,
                                (int)N));
        return QG_OK;
    }

    // Small generalised eigenproblem on the leading k x k block of the Gram pair
    // (row pitch k3), Jacobi-equilibrated; on success leaves the rotation matrix
    // (the first n eigenvectors, back-scaled; rows >= krows zero) in *Zout/*ldz.
    // Returns the solver's info (> 0: B not positive definite).
    int solve_pencil(int k, int k3, int krows, const double** Zout, int* ldz, int* info) {
        if (c == 1) {
            k_equilibrate<<<k, 128, 0, st>>>(Sa, Sb, k3, k, Sa2, Sb2);
            QG_SOLVER_TRY(cusolverDnDsygvd(sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                           k, Sa2, k3, Sb2, k3, w_d, work.as<double>(), lwork, info_d));
        } else {
            k_gram_to_complex<<<k, 128, 0, st>>>(Sa, Sb, 2 * k3, k, Ca, Cb, k3);
            QG_SOLVER_TRY(cusolverDnZhegvd(sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER,
                                           k, Ca, k3, Cb, k3, w_d, work.as<cuDoubleComplex>(), lwork, info_d));
        }
        QG_CUDA_TRY(cudaMemcpyAsync(info, info_d, sizeof(int), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        if (*info != 0) return QG_OK;
        if (c == 1) {
            k_rowscale<<<n, 128, 0, st>>>(Sa2, k3, k, Sb, k3);  // z = D z'
            if (krows < k3)
                QG_CUDA_TRY(cudaMemset2DAsync(Sa2 + krows, (size_t)k3 * sizeof(double), 0,
                                              (size_t)(k3 - krows) * sizeof(double), (size_t)n, st));
            *Zout = Sa2;
            *ldz = k3;
        } else {
            k_expand_rotation<<<n, 128, 0, st>>>(Ca, k3, k3, krows, Sb, 2 * k3, M, 2 * k3);
            *Zout = M;
            *ldz = 2 * k3;
        }
        return QG_OK;
    }

    // Fallback when B of the pencil is not positive definite at working precision:
    // solve on B's numerically nonsingular subspace instead of dropping P.
    //   B2 = V diag(s) V^T (eigendecomposition), keep s_i > 1e-12 max(s),
    //   T = V_kept diag(s_kept)^-1/2,  (T^T A2 T) y = lambda y,  z' = T y,  z = D z'
    // (A2, B2 the Jacobi-equilibrated pencil, D its scaling). Leaves the rotation
    // matrix like solve_pencil. Returns QG_ERR_CHOLESKY if fewer than n directions survive.
    int solve_truncated(int k, int k3, const double** Zout, int* ldz) {
        int info = 0;
        const size_t kk = (size_t)k3 * k3;
        if (c == 1) {
            double* Tm = E0;
            double* tmp = Tm + kk;
            double* Ar = tmp + kk;
            double* Zt = Ar + kk;
            k_equilibrate<<<k, 128, 0, st>>>(Sa, Sb, k3, k, Sa2, Sb2);
            k_mirror_lower<double><<<k, 128, 0, st>>>(Sa2, k3, k);
            QG_SOLVER_TRY(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k, Sb2, k3, w_d,
                                           work.as<double>(), lwork, info_d));
            QG_TRY(read_spectrum(k, &info));
            if (info != 0) return QG_ERR_LIBRARY;
            int f = 0;
            const double thr = trunc_eps * s_h[k - 1];
            while (f < k && !(s_h[f] > thr)) ++f;
            const int kp = k - f;
            if (kp < n) return QG_ERR_CHOLESKY;
            k_scaled_basis<double><<<kp, 128, 0, st>>>(Sb2, k3, k, w_d, f, Tm);
            const double one = 1.0, zero = 0.0;
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, k, kp, k, &one, Sa2, k3, Tm, k3, &zero, tmp, k3));
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_T, CUBLAS_OP_N, kp, kp, k, &one, Tm, k3, tmp, k3, &zero, Ar, k3));
            QG_SOLVER_TRY(cusolverDnDsyevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, kp, Ar, k3, w_d,
                                           work.as<double>(), lwork, info_d));
            QG_BLAS_TRY(cublasDgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, k, n, kp, &one, Tm, k3, Ar, k3, &zero, Zt, k3));
            k_rowscale<<<n, 128, 0, st>>>(Zt, k3, k, Sb, k3);  // z = D z'
            *Zout = Zt;
            *ldz = k3;
        } else {
            cuDoubleComplex* Tm = reinterpret_cast<cuDoubleComplex*>(E0);
            cuDoubleComplex* tmp = Tm + kk;
            cuDoubleComplex* Ar = tmp + kk;
            cuDoubleComplex* Zt = Ar + kk;
            k_gram_to_complex<<<k, 128, 0, st>>>(Sa, Sb, 2 * k3, k, Ca, Cb, k3);
            k_mirror_lower<cuDoubleComplex><<<k, 128, 0, st>>>(Ca, k3, k);
            QG_SOLVER_TRY(cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k, Cb, k3, w_d,
                                           work.as<cuDoubleComplex>(), lwork, info_d));
            QG_TRY(read_spectrum(k, &info));
            if (info != 0) return QG_ERR_LIBRARY;
            int f = 0;
            const double thr = trunc_eps * s_h[k - 1];
            while (f < k && !(s_h[f] > thr)) ++f;
            const int kp = k - f;
            if (kp < n) return QG_ERR_CHOLESKY;
            k_scaled_basis<cuDoubleComplex><<<kp, 128, 0, st>>>(Cb, k3, k, w_d, f, Tm);
            const cuDoubleComplex one = make_cuDoubleComplex(1.0, 0.0), zero = make_cuDoubleComplex(0.0, 0.0);
            QG_BLAS_TRY(cublasZgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, k, kp, k, &one, Ca, k3, Tm, k3, &zero, tmp, k3));
            QG_BLAS_TRY(cublasZgemm(blas, CUBLAS_OP_C, CUBLAS_OP_N, kp, kp, k, &one, Tm, k3, tmp, k3, &zero, Ar, k3));
            QG_SOLVER_TRY(cusolverDnZheevd(sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, kp, Ar, k3, w_d,
                                           work.as<cuDoubleComplex>(), lwork, info_d));
            QG_BLAS_TRY(cublasZgemm(blas, CUBLAS_OP_N, CUBLAS_OP_N, k, n, kp, &one, Tm, k3, Ar, k3, &zero, Zt, k3));
            k_expand_rotation<<<n, 128, 0, st>>>(Zt, k3, k3, k, Sb, 2 * k3, M, 2 * k3);
            *Zout = M;
            *ldz = 2 * k3;
        }
        QG_CUDA_TRY(cudaGetLastError());
        return QG_OK;
    }

    // FP64 Rayleigh-Ritz on X alone: the n x n pencil (X^T AX dV, X^T X dV) from FP64
    // products, x <- x Z, Ax = H x, Rayleigh quotients and residuals. Leaves the
    // residual norms in nr_d.
    int rayleigh_ritz_x() {
        const bool was_mixed = mixed;
        const double te = trunc_eps;
        mixed = false;
        trunc_eps = 1e-12;
        QG_TRY(gram(c * n));
        const double* Z = nullptr;
        int ldz = 0, info = 0;
        QG_TRY(solve_pencil(n, n, n, &Z, &ldz, &info));
        if (info > 0) QG_TRY(solve_truncated(n, n, &Z, &ldz));
        else if (info < 0) return QG_ERR_LIBRARY;
        QG_TRY(gemm_nn(c * n, c * n, x, Z, ldz, Tx, 0.0));
        QG_CUDA_TRY(cudaMemcpyAsync(x, Tx, (size_t)L * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        normalize(x, nullptr);
        QG_TRY(applyH(x, Ax));
        coldot(x, Ax, dV, ev_d);
        residual();
        mixed = was_mixed;
        trunc_eps = te;
        QG_CUDA_TRY(cudaGetLastError());
        return QG_OK;
    }

    // eigenvalues of B (w_d, ascending) and the solver info to the host
    int read_spectrum(int k, int* info) {
        QG_CUDA_TRY(cudaMemcpyAsync(s_h.data(), w_d, k * sizeof(double), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaMemcpyAsync(info, info_d, sizeof(int), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        return QG_OK;
    }
};

// Full Gram pencil every this many iterations in steady state (the reference recomputes
// every S_MAT_REST_LIMIT = 10, lobpcg_d_multi_mpi.h:926, :1040-1043).
constexpr int kFullGramEvery = 10;
// Largest |1 - |x'_j|^2 dV| of a rotated Ritz vector before the step is rolled back, and
// the rollbacks a solve may take before it stops (QG_ERR_CHOLESKY).
constexpr double kNormDrift = 1.0e-3;
// A step whose largest residual grew by more than this factor over the last step's is
// taken as a breakdown of the reused Gram blocks: the next Gram is a full one.
constexpr double kResidualJump = 100.0;
constexpr int kMaxRollbacks = 20;

int run_lobpcg(qg_hamiltonian h, const qg_lobpcg_options* opt, int n, int comps, double* ev, double* X_dev,
               double* P_dev, const double* X_host, double* Xout_host, const double* P_host, double* Pout_host,
               qg_lobpcg_report* rep) {
    if (!h || !opt || n <= 0 || !ev) return QG_ERR_INVALID;
    if (comps == 1 && (h->gx != 0.0 || h->gy != 0.0 || h->gz != 0.0)) return QG_ERR_INVALID;
    if (comps == 2 && h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    if (opt->precision != QG_FP64 && opt->precision != QG_MIXED_BF16X3 && opt->precision != QG_FP32 &&
        opt->precision != QG_FP64_INT8)
        return QG_ERR_UNSUPPORTED;
    if (opt->precond < 0 || opt->precond > 3) return QG_ERR_INVALID;
    if (opt->precond >= 2 && !h->learned) return QG_ERR_INVALID;
    // precond 3 (the learned block): real states and FP64 Gram products only
    const bool aug = opt->precond == 3;
    if (aug && (comps != 1 || opt->precision != QG_FP64)) return QG_ERR_UNSUPPORTED;
    const long long N = h->N();
    if ((long long)n * (aug ? 4 : 3) > N) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    Solver s;
    s.nblk = aug ? 4 : 3;
    s.h = h;
    s.n = n;
    s.c = comps;
    s.N = N;
    s.L = comps * N;
    s.dV = h->hx * h->hy * h->hz;
    s.st = h->ctx->stream;
    s.mixed = opt->precision == QG_MIXED_BF16X3 || opt->precision == QG_FP32;
    s.i8 = opt->precision == QG_FP64_INT8 && comps == 1 && qg::I8Gram::supported(N);
    s.mixed_pieces = opt->precision == QG_FP32 ? -1 : 3;
    s.trunc_eps = s.mixed ? 1e-6 : 1e-12;
    QG_TRY(qg_blas_handle(h->ctx, &s.blas));
    QG_TRY(qg_solver_handle(h->ctx, &s.sol));
    QG_TRY(s.setup());
    const size_t blk_bytes = (size_t)s.L * n * sizeof(double);
    const bool first = opt->first_call != 0;
    const double tol = opt->tol > 0 ? opt->tol : 1.0e-10;
    cudaStream_t st = s.st;
    Timer tm;
    cudaEvent_t t0, t1;
    QG_CUDA_TRY(cudaEventCreate(&t0));
    QG_CUDA_TRY(cudaEventCreate(&t1));
    QG_CUDA_TRY(cudaEventRecord(t0, st));

    // inputs
    if (X_host) QG_CUDA_TRY(cudaMemcpyAsync(s.x, X_host, blk_bytes, cudaMemcpyHostToDevice, st));
    else QG_CUDA_TRY(cudaMemcpyAsync(s.x, X_dev, blk_bytes, cudaMemcpyDeviceToDevice, st));
    if (first) {
        QG_CUDA_TRY(cudaMemsetAsync(s.p, 0, blk_bytes, st));
    } else if (P_host) {
        QG_CUDA_TRY(cudaMemcpyAsync(s.p, P_host, blk_bytes, cudaMemcpyHostToDevice, st));
    } else {
        QG_CUDA_TRY(cudaMemcpyAsync(s.p, P_dev, blk_bytes, cudaMemcpyDeviceToDevice, st));
    }

    // initial residual (lobpcg_d_multi.h:64-91)
    s.normalize(s.x, nullptr);
    QG_TRY(s.applyH(s.x, s.Ax));
    if (first) QG_CUDA_TRY(cudaMemsetAsync(s.Ap, 0, blk_bytes, st));
    else QG_TRY(s.applyH(s.p, s.Ap));
    s.coldot(s.x, s.Ax, s.dV, s.ev_d);
    s.residual();
    {
        // non-finite input states (or P): stop before any pencil is formed from them
        std::vector<double> r0(n), e0(n);
        QG_CUDA_TRY(cudaMemcpyAsync(r0.data(), s.nr_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaMemcpyAsync(e0.data(), s.ev_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        for (int j = 0; j < n; ++j)
            if (!std::isfinite(r0[j]) || !std::isfinite(e0[j])) {
                cudaEventDestroy(t0);
                cudaEventDestroy(t1);
                qg_set_last_error("run_lobpcg", "non-finite value in the initial states", __FILE__, __LINE__);
                return QG_ERR_NONFINITE;
            }
    }
    qg::KineticPrecond* pc = nullptr;
    const bool learned = opt->precond == 2;
    // w = T r (precond 1), w = T r + NN(r) (precond 2: the learned correction, learned.cu);
    // precond 3: w = T r and the network's correction as a block of its own, q = NN(r),
    // so the Rayleigh-Ritz step chooses how much of it to take (its basis [x, T r, q, p]
    // contains the kinetic method's [x, T r, p])
    auto precondition = [&]() -> int {
        if (learned || aug) QG_CUDA_TRY(cudaMemcpyAsync(s.Tx, s.r, blk_bytes, cudaMemcpyDeviceToDevice, st));
        QG_TRY(pc->apply(s.r, st));
        if (learned)
            QG_TRY(qg_learned_apply_d(h->learned, h->nx, h->ny, h->nz, comps * n, s.Tx, N, h->V_d, h->learned_vscale,
                                      s.r, N, 1));
        if (aug) {
            QG_TRY(qg_learned_apply_d(h->learned, h->nx, h->ny, h->nz, n, s.Tx, N, h->V_d, h->learned_vscale, s.q, N,
                                      0));
            s.normalize(s.q, nullptr);
        }
        s.normalize(s.r, nullptr);
        return QG_OK;
    };
    if (opt->precond >= 1) {
        // Gamma-point FD symbol on every real column (for k-point states it is an
        // approximation of the k-shifted kinetic operator, still a valid preconditioner)
        if (!h->precond) h->precond = new qg::KineticPrecond();
        pc = h->precond;
        QG_TRY(pc->setup(h, comps * n, opt->precond_shift > 0 ? opt->precond_shift : 1.0));
        QG_TRY(precondition());
    } else {
        k_inv_norm<<<(n + 127) / 128, 128, 0, st>>>(s.nr_d, 1.0, n, s.f_d);
        s.scale_cols(s.r, nullptr);
    }
    QG_CUDA_TRY(cudaGetLastError());

    std::vector<double> ev_h(n), nr_h(n);
    int it = 0;
    bool converged = false;
    double maxres = 0.0;
    int status = QG_OK;
    int restarts = 0, rollbacks = 0;
    const int c = comps;
    const int nconv = (opt->n_converge > 0 && opt->n_converge < n) ? opt->n_converge : n;
    double best_res = 1e300;
    int best_it = 0, mixed_iters = s.mixed ? opt->max_iter : 0;
    bool restart_2n = false;  // after a norm-drift rollback: the next step uses the [x r] pencil
    bool used_update = false;  // this step's pencil came from the reused Gram blocks
    double last_res = 1e300;
    for (it = 0; it < opt->max_iter; ++it) {
        tm.mark(0, st);
        QG_TRY(s.applyH(s.r, s.Ar));
        if (aug) QG_TRY(s.applyH(s.q, s.Aq));
        tm.mark(1, st);
        const bool two = (first && it == 0) || restart_2n;
        const bool after_rollback = restart_2n;
        restart_2n = false;
        // pencil columns: [x r (q) p], without p on a 2n step
        const int k3 = ((two ? 2 : 3) + (aug ? 1 : 0)) * n;
        // steady state: the x/p blocks of the pencil come from the last rotation and only
        // the r blocks are tall products; a full Gram every kFullGramEvery iterations, on a 2n
        // step, after a rank-revealing solve, on both steps after a rollback, after a step
        // whose residual jumped by kResidualJump, and in the reduced-precision phase
        const bool use_update = s.have_update && !two && !s.mixed && !aug && (it % kFullGramEvery) != 0;
        if (use_update) QG_TRY(s.gram_update(k3));
        else QG_TRY(s.gram(c * k3));
        used_update = use_update;
        s.have_update = false;
        tm.mark(2, st);
        // Jacobi-equilibrated pencil (keeps the tiny residual columns of the reference
        // iteration from ruining the Cholesky factor of B), cuSOLVER sygvd / hegvd on it;
        // if B is still not positive definite, the step is solved on B's numerically
        // nonsingular subspace (counted as a restart)
        const double* Z = nullptr;
        int ldz = 0;
        bool restarted = false;
        int solve_info = 0;
        if (s.mixed) solve_info = 1;  // the BF16x3 pencil always takes the rank-revealing solve
        else QG_TRY(s.solve_pencil(k3, k3, k3, &Z, &ldz, &solve_info));
        if (solve_info > 0) {
            restarted = true;
            const int rc = s.solve_truncated(k3, k3, &Z, &ldz);
            if (rc == QG_OK) solve_info = 0;
            else if (rc != QG_ERR_CHOLESKY) solve_info = -1;
        }
        if (solve_info != 0) {
            status = solve_info > 0 ? QG_ERR_CHOLESKY : QG_ERR_LIBRARY;
            ++it;
            break;
        }
        if (restarted && !s.mixed) ++restarts;
        tm.mark(3, st);
        // rotation: columns 0..n-1 of Z are (Cx; Cr; Cp) (c rows/columns per state)
        //   p_new = [r p] [Cr; Cp],  x_new = x Cx + p_new   (lobpcg_d_multi.h:247-300)
        // and the A-side blocks are re-applied, Ax = H x_new, Ap = H p_new, instead of
        // rotated: two memory-bound H applications cost less than the two tall DGEMMs
        // and keep Ax consistent with x for the residual.
        const bool next_update =
            h->gram_reuse && c == 1 && !s.mixed && !aug && !restarted && !after_rollback && 3 * n > qg::kGramTsUpTo;
        if (next_update) QG_TRY(s.prepare_update(Z, ldz, k3));
        QG_TRY(s.gemm_nn(c * (k3 - n), c * n, s.r, Z + c * n, ldz, s.Tp, 0.0));
        QG_CUDA_TRY(cudaMemcpyAsync(s.Tx, s.Tp, blk_bytes, cudaMemcpyDeviceToDevice, st));
        QG_TRY(s.gemm_nn(c * n, c * n, s.x, Z, ldz, s.Tx, 1.0));
        // norm drift of the rotated x (B-normalised Ritz vectors have |x'|^2 dV = 1): beyond
        // 1e-3 the step is rolled back -- x and p stay, and the next step solves the [x r]
        // pencil with a full Gram (the rollback of Eigen_d_multi_mpi, lobpcg_d_multi_mpi.h:1305-1346,
        // which keeps X and stops; here the iteration goes on from the kept X)
        s.coldot(s.Tx, s.Tx, 1.0, s.nr_d);
        QG_CUDA_TRY(cudaMemcpyAsync(nr_h.data(), s.nr_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        double drift = 0.0;
        for (int j = 0; j < n; ++j) drift = std::max(drift, std::fabs(1.0 - nr_h[j] * s.dV));
        if (!(drift <= kNormDrift) && !two) {
            ++restarts;
            ++rollbacks;
            restart_2n = true;
            s.have_update = false;
            if (opt->verbose) printf("lobpcg iter %d: |x|^2 drift %.3e, rolled back\n", it + 1, drift);
            tm.mark(-1, st);
            QG_CUDA_TRY(cudaStreamSynchronize(st));
            tm.flush();
            if (rollbacks > kMaxRollbacks) {
                status = QG_ERR_CHOLESKY;
                ++it;
                break;
            }
            continue;
        }
        tm.mark(4, st);
        k_inv_norm<<<(n + 127) / 128, 128, 0, st>>>(s.nr_d, s.dV, n, s.f_d);  // norms of x' taken above
        s.scale_copy(s.x, s.Tx);  // x = x' / |x'|, copy and scaling in one pass
        if (next_update) QG_CUDA_TRY(cudaMemcpyAsync(s.fx_d, s.f_d, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
        s.normalize_from(s.p, s.Tp);
        if (next_update) {
            QG_CUDA_TRY(cudaMemcpyAsync(s.fp_d, s.f_d, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            s.have_update = true;
        }
        tm.mark(0, st);
        QG_TRY(s.applyH(s.x, s.Ax));
        QG_TRY(s.applyH(s.p, s.Ap));
        tm.mark(4, st);
        s.coldot(s.x, s.Ax, s.dV, s.ev_d);
        s.residual();
        QG_CUDA_TRY(cudaGetLastError());
        QG_CUDA_TRY(cudaMemcpyAsync(nr_h.data(), s.nr_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (pc) QG_TRY(precondition());  // next search direction, normalised (residual norms already taken)
        tm.mark(5, st);
        tm.mark(-1, st);
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        tm.flush();
        maxres = *std::max_element(nr_h.begin(), nr_h.begin() + nconv);
        if (!std::isfinite(maxres)) {
            status = QG_ERR_NONFINITE;
            ++it;
            break;
        }
        if (s.have_update && used_update && maxres > kResidualJump * last_res) s.have_update = false;
        last_res = maxres;
        if (opt->verbose) printf("lobpcg iter %d max residual %.3e%s\n", it + 1, maxres, s.mixed ? " (bf16x3)" : "");
        if (s.mixed && maxres < tol * s.dV) {
            // the mixed iteration reached the tolerance: FP64 Rayleigh-Ritz on X and an
            // FP64 residual decide; the iteration continues with FP64 Gram products if needed
            QG_TRY(s.rayleigh_ritz_x());
            QG_CUDA_TRY(cudaMemcpyAsync(nr_h.data(), s.nr_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
            if (pc) QG_TRY(precondition());
            QG_CUDA_TRY(cudaStreamSynchronize(st));
            maxres = *std::max_element(nr_h.begin(), nr_h.begin() + nconv);
            s.mixed = false;
            s.trunc_eps = 1e-12;
            mixed_iters = it + 1;
            if (opt->verbose) printf("lobpcg FP64 Rayleigh-Ritz on X: max residual %.3e\n", maxres);
        }
        if (maxres < tol * s.dV && !s.mixed) {
            converged = true;
            ++it;
            break;
        }
        // mixed precision: hand over to FP64 Gram products once the residual is below
        // 1e-6 or has not halved over three iterations. The split-BF16 pencil is solved
        // on the span of B's eigenvectors above 1e-6 max (its error level); from about
        // that residual on, FP64 products converge the tail in fewer iterations than
        // mixed ones with either a looser or a tighter floor (216-atom cell: 19 + 13
        // iterations against 42 + 22 when the hand-over waits for a stall near 1e-9)
        if (s.mixed) {
            if (maxres < best_res * 0.5) {
                best_res = maxres;
                best_it = it;
            }
            if (maxres < 1e-6 || it - best_it >= 3) {
                s.mixed = false;
                s.trunc_eps = 1e-12;
                mixed_iters = it + 1;
            }
        }
    }
    // a solve that ends while still mixed takes a final FP64 Rayleigh-Ritz on X
    if (s.mixed && status == QG_OK) {
        s.mixed = false;
        QG_TRY(s.rayleigh_ritz_x());
        QG_CUDA_TRY(cudaMemcpyAsync(nr_h.data(), s.nr_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        maxres = *std::max_element(nr_h.begin(), nr_h.begin() + nconv);
        converged = maxres < tol * s.dV;
    }
    // outputs
    QG_CUDA_TRY(cudaMemcpyAsync(ev_h.data(), s.ev_d, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (Xout_host) QG_CUDA_TRY(cudaMemcpyAsync(Xout_host, s.x, blk_bytes, cudaMemcpyDeviceToHost, st));
    else QG_CUDA_TRY(cudaMemcpyAsync(X_dev, s.x, blk_bytes, cudaMemcpyDeviceToDevice, st));
    if (Pout_host) QG_CUDA_TRY(cudaMemcpyAsync(Pout_host, s.p, blk_bytes, cudaMemcpyDeviceToHost, st));
    else if (P_dev) QG_CUDA_TRY(cudaMemcpyAsync(P_dev, s.p, blk_bytes, cudaMemcpyDeviceToDevice, st));
    QG_CUDA_TRY(cudaEventRecord(t1, st));
    QG_CUDA_TRY(cudaStreamSynchronize(st));
    for (int j = 0; j < n; ++j) ev[j] = ev_h[j];
    float tot = 0.f;
    cudaEventElapsedTime(&tot, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rep) {
        rep->iterations = it;
        rep->converged = converged ? 1 : 0;
        rep->max_residual = maxres;
        rep->ms_total = tot;
        rep->ms_hamiltonian = tm.acc[0];
        rep->ms_gram = tm.acc[1];
        rep->ms_eigensolve = tm.acc[2];
        rep->ms_rotate = tm.acc[3];
        rep->ms_vector = tm.acc[4];
        rep->restarts = restarts;
        rep->mixed_iterations = std::min(mixed_iters, it);
    }
    const int dstat = qg_context_take_device_status(h->ctx);
    if (dstat != QG_OK) return dstat;
    if (status != QG_OK) return status;
    return converged ? QG_OK : QG_ERR_NOT_CONVERGED;
}

// Complex block LOBPCG for nk k-points at once (block-diagonal Rayleigh-Ritz).
// All nk*nb states live in the same W / AW / T blocks, k-point major ([k][s], each
// state {re[N], im[N]}), so H, norms, residuals and the preconditioner run over all
// of them in single launches (qg::apply_hamiltonian_zk for H). The Gram products
// are DGEMMs per k-point and block pair of [x r p], the rotations strided-batched
// DGEMMs over k; the small Hermitian pencils are solved k by k
// (Jacobi-equilibrated cusolverDnZhegvd, the rank-revealing solve where B is
// singular). Stops when every k-point's lowest n_converge states meet tol.
// k-points whose largest residual (sum r^2 dV, the convergence measure) is below this
// times dV take zhegvd instead of the batched Jacobi solver: on the 8-atom 40^3 cell
// (64 k-points, 16 states) the two give the same iterates down to ~1e-5 and the
// zhegvd pencils converge in 78 iterations where the Jacobi ones need 118-129
constexpr double kJacobiResidual = 1e-3;

int run_lobpcg_zk(qg_hamiltonian h, const qg_lobpcg_options* opt, int nk, const double* kv, int nb, double* ev,
                  double* X_dev, double* P_dev, qg_lobpcg_report* rep) {
    if (!h || !opt || nk <= 0 || nb <= 0 || !kv || !ev || !X_dev) return QG_ERR_INVALID;
    if (h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    if (opt->precision != QG_FP64) return QG_ERR_UNSUPPORTED;
    if (opt->precond < 0 || opt->precond > 1) return QG_ERR_INVALID;
    const long long N = h->N();
    if ((long long)nb * 3 > N) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    const int nt = nk * nb;
    Solver s;
    s.h = h;
    s.n = nt;
    s.c = 2;
    s.N = N;
    s.L = 2 * N;
    s.dV = h->hx * h->hy * h->hz;
    s.st = h->ctx->stream;
    cudaStream_t st = s.st;
    QG_TRY(qg_blas_handle(h->ctx, &s.blas));
    QG_TRY(qg_solver_handle(h->ctx, &s.sol));
    // tall blocks for all states, Gram pencils and rotations per k-point
    const size_t blk = (size_t)s.L * nt;
    QG_TRY(s.W.reserve(3 * blk * sizeof(double)));
    QG_TRY(s.AW.reserve(3 * blk * sizeof(double)));
    QG_TRY(s.T.reserve(2 * blk * sizeof(double)));
    s.x = s.W.as<double>(); s.r = s.x + blk; s.p = s.r + blk;
    s.Ax = s.AW.as<double>(); s.Ar = s.Ax + blk; s.Ap = s.Ar + blk;
    s.Tx = s.T.as<double>(); s.Tp = s.Tx + blk;
    const int k3m = 3 * nb, g3 = 2 * k3m;
    const size_t gsz = (size_t)g3 * g3, msz = (size_t)g3 * 2 * nb, kk = (size_t)k3m * k3m;
    QG_TRY(s.S.reserve((2 * nk * gsz + 4 * kk + nk * msz) * sizeof(double)));
    QG_CUDA_TRY(cudaMemsetAsync(s.S.ptr, 0, s.S.bytes, st));
    double* SaAll = s.S.as<double>();
    double* SbAll = SaAll + nk * gsz;
    s.Sa2 = SbAll + nk * gsz;
    s.Sb2 = s.Sa2 + 2 * kk;
    double* Mall = s.Sb2 + 2 * kk;
    s.Ca = reinterpret_cast<cuDoubleComplex*>(s.Sa2);
    s.Cb = reinterpret_cast<cuDoubleComplex*>(s.Sb2);
    QG_TRY(s.E.reserve(8 * kk * sizeof(double)));
    s.E0 = s.E.as<double>();
    s.s_h.resize(k3m);
    QG_TRY(s.small.reserve(((size_t)5 * 3 * nt + 16 + nk) * sizeof(double)));
    s.ev_d = s.small.as<double>(); s.nr_d = s.ev_d + 3 * nt; s.f_d = s.nr_d + 3 * nt; s.f2_d = s.f_d + 3 * nt;
    s.w_d = s.f2_d + 3 * nt;
    s.info_d = reinterpret_cast<int*>(s.w_d + 3 * nt);
    int* infos_d = s.info_d + 4;
    {
        int lw1 = 0, lw2 = 0;
        QG_SOLVER_TRY(cusolverDnZhegvd_bufferSize(s.sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                                  CUBLAS_FILL_MODE_LOWER, k3m, s.Ca, k3m, s.Cb, k3m, s.w_d, &lw1));
        QG_SOLVER_TRY(cusolverDnZheevd_bufferSize(s.sol, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, k3m, s.Cb,
                                                  k3m, s.w_d, &lw2));
        s.lwork = std::max(lw1, lw2);
        QG_TRY(s.work.reserve((size_t)std::max(s.lwork, 1) * sizeof(cuDoubleComplex)));
    }
    QG_TRY(h->coef.reserve(qg::coef_scratch_elems_z(h, nk, nb) * sizeof(double)));
    // pencils of up to kSmallHegMax rows: all k-points' Hermitian pencils in one launch
    // of the one-block Jacobi solver (small_eig.cu), cuSOLVER's zhegvd per k-point
    // otherwise and for any pencil the Jacobi solver rejects
    const bool batched_eig = k3m <= qg::kSmallHegMax;
    DevBuf& heg = s.heg;
    cuDoubleComplex *CaAll = nullptr, *CbAll = nullptr;
    double* wAll = nullptr;
    int* skip_d = nullptr;
    if (batched_eig) {
        QG_TRY(heg.reserve((2 * nk * kk) * sizeof(cuDoubleComplex) + (size_t)nk * k3m * sizeof(double) +
                           (size_t)nk * sizeof(int)));
        CaAll = heg.as<cuDoubleComplex>();
        CbAll = CaAll + nk * kk;
        wAll = reinterpret_cast<double*>(CbAll + nk * kk);
        skip_d = reinterpret_cast<int*>(wAll + (size_t)nk * k3m);
    }
    std::vector<int> skip_h(nk, 0);
    std::vector<char> near(nk, 0);
    int jacobi_fallbacks = 0;  // pencils the batched solver handed to zhegvd
    const size_t blk_bytes = blk * sizeof(double);
    const bool first = opt->first_call != 0;
    const double tol = opt->tol > 0 ? opt->tol : 1.0e-10;
    const int nconv = (opt->n_converge > 0 && opt->n_converge < nb) ? opt->n_converge : nb;
    const long long kstride = 2LL * nb * N;  // one k-point's columns within a block
    auto applyH = [&](const double* in, double* out) {
        return qg::apply_hamiltonian_zk(h, nk, kv, nb, in, s.L, (long long)nb * s.L, out, s.L, (long long)nb * s.L,
                                        h->coef.as<double>(), st);
    };
    // C_k (block (bi, bj) of the k-th pencil, ldc g) = dV * A_k^T B_k, one DGEMM per k-point:
    // cuBLAS's strided-batched DGEMM at these shapes (2nb x 2nb, K = N) returned Gram
    // matrices noticeably less accurate than its plain DGEMM (8 k-points: 208 rank-revealing
    // restarts and 95 iterations instead of 11 and 73), so the batch is a loop of DGEMMs
    auto gram_block = [&](const double* A, const double* B, double* C, int g) -> int {
        const double zero = 0.0;
        for (int k = 0; k < nk; ++k)
            QG_BLAS_TRY(cublasDgemm(s.blas, CUBLAS_OP_T, CUBLAS_OP_N, 2 * nb, 2 * nb, (int)N, &s.dV, A + k * kstride,
                                    (int)N, B + k * kstride, (int)N, &zero, C + k * gsz, g));
        return QG_OK;
    };
    auto gram_pair = [&](const double* Wi, const double* AWj, const double* Wj, double* Ca_, double* Cb_,
                         int g) -> int {
        QG_TRY(gram_block(Wi, AWj, Ca_, g));
        return gram_block(Wi, Wj, Cb_, g);
    };
    // C_k (N x 2nb) = A_k (N x 2nb) * Z_k (rows off.., ldz) + beta C_k, batched over k
    auto rot_block = [&](const double* A, const double* Z, int ldz, double* C, double beta) -> int {
        const double one = 1.0;
        QG_BLAS_TRY(cublasDgemmStridedBatched(s.blas, CUBLAS_OP_N, CUBLAS_OP_N, (int)N, 2 * nb, 2 * nb, &one, A,
                                              (int)N, kstride, Z, ldz, (long long)msz, &beta, C, (int)N, kstride, nk));
        return QG_OK;
    };
    cudaEvent_t t0, t1;
    QG_CUDA_TRY(cudaEventCreate(&t0));
    QG_CUDA_TRY(cudaEventCreate(&t1));
    QG_CUDA_TRY(cudaEventRecord(t0, st));
    QG_CUDA_TRY(cudaMemcpyAsync(s.x, X_dev, blk_bytes, cudaMemcpyDeviceToDevice, st));
    if (first || !P_dev) QG_CUDA_TRY(cudaMemsetAsync(s.p, 0, blk_bytes, st));
    else QG_CUDA_TRY(cudaMemcpyAsync(s.p, P_dev, blk_bytes, cudaMemcpyDeviceToDevice, st));
    s.normalize(s.x, nullptr);
    QG_TRY(applyH(s.x, s.Ax));
    if (first || !P_dev) QG_CUDA_TRY(cudaMemsetAsync(s.Ap, 0, blk_bytes, st));
    else QG_TRY(applyH(s.p, s.Ap));
    s.coldot(s.x, s.Ax, s.dV, s.ev_d);
    s.residual();
    qg::KineticPrecond* pc = nullptr;
    if (opt->precond == 1) {
        if (!h->precond) h->precond = new qg::KineticPrecond();
        pc = h->precond;
        QG_TRY(pc->setup(h, 2 * nt, opt->precond_shift > 0 ? opt->precond_shift : 1.0));
        QG_TRY(pc->apply(s.r, st));
        s.normalize(s.r, nullptr);
    } else {
        k_inv_norm<<<(nt + 127) / 128, 128, 0, st>>>(s.nr_d, 1.0, nt, s.f_d);
        s.scale_cols(s.r, nullptr);
    }
    QG_CUDA_TRY(cudaGetLastError());
    std::vector<double> ev_h(nt), nr_h(nt);
    std::vector<int> info_h(nk);
    // a k-point whose lowest n_converge states meet tol is frozen: its states are no
    // longer rotated and its pencil is no longer solved, so the solve ends after as
    // many iterations as the slowest k-point needs on its own
    std::vector<char> frozen(nk, 0);
    int it = 0, restarts = 0, status = QG_OK;
    bool converged = false;
    double maxres = 0.0;
    Timer tm;
    for (it = 0; it < opt->max_iter; ++it) {
        tm.mark(0, st);
        QG_TRY(applyH(s.r, s.Ar));
        tm.mark(1, st);
        const bool two = first && it == 0;
        const int k3 = (two ? 2 : 3) * nb, g = 2 * k3;
        const double* Wb[3] = {s.x, s.r, s.p};
        const double* AWb[3] = {s.Ax, s.Ar, s.Ap};
        for (int bi = 0; bi < k3 / nb; ++bi)
            for (int bj = 0; bj <= bi; ++bj) {
                const size_t off = (size_t)bi * 2 * nb + (size_t)bj * 2 * nb * g;
                QG_TRY(gram_pair(Wb[bi], AWb[bj], Wb[bj], SaAll + off, SbAll + off, g));
            }
        // Hermitian pencils k by k; solutions expanded to real rotations M_k (2k3 x 2nb)
        tm.mark(2, st);
        QG_CUDA_TRY(cudaMemsetAsync(infos_d, 0, nk * sizeof(int), st));
        if (batched_eig) {
            // the batched Jacobi solver takes the k-points still far from convergence;
            // the pencils of nearly converged k-points (residual below kJacobiResidual,
            // nearly singular B) go to zhegvd one by one, with which the iteration
            // converges in fewer steps
            for (int k = 0; k < nk; ++k) {
                double mk = it == 0 ? 1e300 : 0.0;
                if (it > 0)
                    for (int j = 0; j < nconv; ++j) mk = std::max(mk, nr_h[k * nb + j]);
                near[k] = !frozen[k] && mk < kJacobiResidual * s.dV;
                skip_h[k] = (frozen[k] || near[k]) ? 1 : 0;
            }
            QG_CUDA_TRY(cudaMemcpyAsync(skip_d, skip_h.data(), nk * sizeof(int), cudaMemcpyHostToDevice, st));
            k_gram_to_complex_b<<<dim3(k3, nk), 128, 0, st>>>(SaAll, SbAll, g, (long long)gsz, k3, CaAll, CbAll, k3,
                                                               (long long)kk, skip_d);
            QG_TRY(qg::small_heg_launch(reinterpret_cast<const double2*>(CaAll), reinterpret_cast<const double2*>(CbAll),
                                        k3, (long long)kk, k3, skip_d, reinterpret_cast<double2*>(CaAll), k3,
                                        (long long)kk, wAll, k3m, infos_d, nk, st));
            k_expand_rotation_b<<<dim3(nb, nk), 128, 0, st>>>(CaAll, k3, (long long)kk, k3, SbAll, g, (long long)gsz,
                                                               Mall, g, (long long)msz, skip_d);
            for (int k = 0; k < nk; ++k) {
                if (!near[k]) continue;
                double* Sa_k = SaAll + k * gsz;
                double* Sb_k = SbAll + k * gsz;
                k_gram_to_complex<<<k3, 128, 0, st>>>(Sa_k, Sb_k, g, k3, s.Ca, s.Cb, k3);
                QG_SOLVER_TRY(cusolverDnZhegvd(s.sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                               CUBLAS_FILL_MODE_LOWER, k3, s.Ca, k3, s.Cb, k3, s.w_d,
                                               s.work.as<cuDoubleComplex>(), s.lwork, infos_d + k));
                k_expand_rotation<<<nb, 128, 0, st>>>(s.Ca, k3, k3, k3, Sb_k, g, Mall + k * msz, g);
            }
        } else {
            for (int k = 0; k < nk; ++k) {
                double* Sa_k = SaAll + k * gsz;
                double* Sb_k = SbAll + k * gsz;
                if (frozen[k]) {
                    k_freeze_rotation<<<2 * nb, 128, 0, st>>>(Mall + k * msz, g, g);
                    continue;
                }
                k_gram_to_complex<<<k3, 128, 0, st>>>(Sa_k, Sb_k, g, k3, s.Ca, s.Cb, k3);
                QG_SOLVER_TRY(cusolverDnZhegvd(s.sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                               CUBLAS_FILL_MODE_LOWER, k3, s.Ca, k3, s.Cb, k3, s.w_d,
                                               s.work.as<cuDoubleComplex>(), s.lwork, infos_d + k));
                k_expand_rotation<<<nb, 128, 0, st>>>(s.Ca, k3, k3, k3, Sb_k, g, Mall + k * msz, g);
            }
        }
        QG_CUDA_TRY(cudaMemcpyAsync(info_h.data(), infos_d, nk * sizeof(int), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        for (int k = 0; k < nk && status == QG_OK; ++k) {
            if (batched_eig && !near[k] && info_h[k] == 2) info_h[k] = 0;  // Jacobi sweep limit: vectors kept
            if (info_h[k] == 0) continue;
            if (batched_eig && !near[k] && info_h[k] == 1) {
                // the Jacobi solver's Cholesky met a non-positive pivot: cuSOLVER's zhegvd
                // on the same pencil first (it still factors some borderline pencils,
                // which keeps the iteration of the per-k path), the rank-revealing solve
                // only if that fails too
                double* Sa_k = SaAll + k * gsz;
                double* Sb_k = SbAll + k * gsz;
                k_gram_to_complex<<<k3, 128, 0, st>>>(Sa_k, Sb_k, g, k3, s.Ca, s.Cb, k3);
                QG_SOLVER_TRY(cusolverDnZhegvd(s.sol, CUSOLVER_EIG_TYPE_1, CUSOLVER_EIG_MODE_VECTOR,
                                               CUBLAS_FILL_MODE_LOWER, k3, s.Ca, k3, s.Cb, k3, s.w_d,
                                               s.work.as<cuDoubleComplex>(), s.lwork, infos_d + k));
                int zinfo = 0;
                QG_CUDA_TRY(cudaMemcpyAsync(&zinfo, infos_d + k, sizeof(int), cudaMemcpyDeviceToHost, st));
                QG_CUDA_TRY(cudaStreamSynchronize(st));
                if (zinfo == 0) {
                    k_expand_rotation<<<nb, 128, 0, st>>>(s.Ca, k3, k3, k3, Sb_k, g, Mall + k * msz, g);
                    ++jacobi_fallbacks;
                    continue;
                }
                info_h[k] = zinfo;
            }
            if (info_h[k] < 0) {
                status = QG_ERR_LIBRARY;
                break;
            }
            ++restarts;
            s.Sa = SaAll + k * gsz;
            s.Sb = SbAll + k * gsz;
            s.M = Mall + k * msz;
            const double* Z = nullptr;
            int ldz = 0;
            s.n = nb;  // the pencil's eigenvectors kept: one k-point's states
            const int rc = s.solve_truncated(k3, k3, &Z, &ldz);
            s.n = nt;
            if (rc == QG_ERR_CHOLESKY) status = QG_ERR_CHOLESKY;
            else if (rc != QG_OK) return rc;
        }
        if (status != QG_OK) {
            ++it;
            break;
        }
        tm.mark(3, st);
        // rotation, batched over k: p_new = r Cr (+ p Cp), x_new = x Cx + p_new
        QG_TRY(rot_block(s.r, Mall + 2 * nb, g, s.Tp, 0.0));
        if (!two) QG_TRY(rot_block(s.p, Mall + 4 * nb, g, s.Tp, 1.0));
        QG_CUDA_TRY(cudaMemcpyAsync(s.Tx, s.Tp, blk_bytes, cudaMemcpyDeviceToDevice, st));
        QG_TRY(rot_block(s.x, Mall, g, s.Tx, 1.0));
        tm.mark(4, st);
        s.normalize_from(s.x, s.Tx);
        s.normalize_from(s.p, s.Tp);
        tm.mark(0, st);
        QG_TRY(applyH(s.x, s.Ax));
        QG_TRY(applyH(s.p, s.Ap));
        tm.mark(4, st);
        s.coldot(s.x, s.Ax, s.dV, s.ev_d);
        s.residual();
        QG_CUDA_TRY(cudaGetLastError());
        QG_CUDA_TRY(cudaMemcpyAsync(nr_h.data(), s.nr_d, nt * sizeof(double), cudaMemcpyDeviceToHost, st));
        if (pc) {
            QG_TRY(pc->apply(s.r, st));
            s.normalize(s.r, nullptr);
        }
        tm.mark(-1, st);
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        tm.flush();
        maxres = 0.0;
        bool all = true;
        for (int k = 0; k < nk; ++k) {
            double mk = 0.0;
            for (int j = 0; j < nconv; ++j) mk = std::max(mk, nr_h[k * nb + j]);
            if (mk < tol * s.dV) frozen[k] = 1;
            if (!frozen[k]) all = false;
            if (!frozen[k] || mk < tol * s.dV) maxres = std::max(maxres, mk);
        }
        if (!std::isfinite(maxres)) {
            status = QG_ERR_NONFINITE;
            ++it;
            break;
        }
        if (opt->verbose)
            printf("lobpcg(%d k-points) iter %d max residual %.3e (zhegvd fallbacks so far %d)\n", nk, it + 1, maxres,
                   jacobi_fallbacks);
        if (all) {
            converged = true;
            ++it;
            break;
        }
    }
    QG_CUDA_TRY(cudaMemcpyAsync(ev_h.data(), s.ev_d, nt * sizeof(double), cudaMemcpyDeviceToHost, st));
    QG_CUDA_TRY(cudaMemcpyAsync(X_dev, s.x, blk_bytes, cudaMemcpyDeviceToDevice, st));
    if (P_dev) QG_CUDA_TRY(cudaMemcpyAsync(P_dev, s.p, blk_bytes, cudaMemcpyDeviceToDevice, st));
    QG_CUDA_TRY(cudaEventRecord(t1, st));
    QG_CUDA_TRY(cudaStreamSynchronize(st));
    for (int j = 0; j < nt; ++j) ev[j] = ev_h[j];
    float tot = 0.f;
    cudaEventElapsedTime(&tot, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->iterations = it;
        rep->converged = converged ? 1 : 0;
        rep->max_residual = maxres;
        rep->ms_total = tot;
        rep->ms_hamiltonian = tm.acc[0];
        rep->ms_gram = tm.acc[1];
        rep->ms_eigensolve = tm.acc[2];
        rep->ms_rotate = tm.acc[3];
        rep->ms_vector = tm.acc[4];
        rep->restarts = restarts;
    }
    const int dstat = qg_context_take_device_status(h->ctx);
    if (dstat != QG_OK) return dstat;
    if (status != QG_OK) return status;
    return converged ? QG_OK : QG_ERR_NOT_CONVERGED;
}

}  // namespace

extern "C" {

int qg_hamiltonian_set_gram_reuse(qg_hamiltonian h, int on) {
    if (!h || (on != 0 && on != 1)) return QG_ERR_INVALID;
    h->gram_reuse = on;
    return QG_OK;
}

int qg_lobpcg_d(qg_hamiltonian h, const qg_lobpcg_options* opt, int ns, double* ev, double* X, double* P,
                qg_lobpcg_report* rep) {
    if (!X || (!P && opt && !opt->first_call)) return QG_ERR_INVALID;
    return run_lobpcg(h, opt, ns, 1, ev, nullptr, nullptr, X, X, P, P, rep);
}

int qg_lobpcg_d_device(qg_hamiltonian h, const qg_lobpcg_options* opt, int ns, double* ev, double* X, double* P,
                       qg_lobpcg_report* rep) {
    if (!X || (!P && opt && !opt->first_call)) return QG_ERR_INVALID;
    return run_lobpcg(h, opt, ns, 1, ev, X, P, nullptr, nullptr, nullptr, nullptr, rep);
}

int qg_lobpcg_cells_device(int ncells, const qg_hamiltonian* hams, const qg_lobpcg_options* opts, const int* ns,
                           double* const* ev, double* const* X, double* const* P, qg_lobpcg_report* reports,
                           int* status) {
    if (ncells <= 0 || !hams || !opts || !ns || !ev || !X) return QG_ERR_INVALID;
    for (int c = 0; c < ncells; ++c) {
        if (!hams[c] || !X[c] || !ev[c] || ns[c] <= 0) return QG_ERR_INVALID;
        if (!opts[c].first_call && (!P || !P[c])) return QG_ERR_INVALID;
        for (int d = 0; d < c; ++d)  // one context (stream and library handles) per cell
            if (hams[d]->ctx == hams[c]->ctx) return QG_ERR_INVALID;
    }
    std::vector<int> st(ncells, QG_OK);
    std::vector<std::thread> pool;
    pool.reserve(ncells);
    for (int c = 0; c < ncells; ++c)
        pool.emplace_back([&, c] {
            st[c] = run_lobpcg(hams[c], &opts[c], ns[c], 1, ev[c], X[c], P ? P[c] : nullptr, nullptr, nullptr,
                               nullptr, nullptr, reports ? &reports[c] : nullptr);
        });
    for (auto& t : pool) t.join();
    int rc = QG_OK;
    for (int c = 0; c < ncells; ++c) {
        if (status) status[c] = st[c];
        if (rc == QG_OK && st[c] != QG_OK) rc = st[c];
    }
    return rc;
}

int qg_lobpcg_z(qg_hamiltonian h, const qg_lobpcg_options* opt, int ns, double* ev, double* X, double* P,
                qg_lobpcg_report* rep) {
    if (!X || (!P && opt && !opt->first_call)) return QG_ERR_INVALID;
    return run_lobpcg(h, opt, ns, 2, ev, nullptr, nullptr, X, X, P, P, rep);
}

int qg_lobpcg_zk_device(qg_hamiltonian h, const qg_lobpcg_options* opt, int nk, const double* kvecs, int nsk,
                        double* ev, double* X, double* P, qg_lobpcg_report* rep) {
    if (!X || (!P && opt && !opt->first_call)) return QG_ERR_INVALID;
    return run_lobpcg_zk(h, opt, nk, kvecs, nsk, ev, X, P, rep);
}

int qg_lobpcg_z_device(qg_hamiltonian h, const qg_lobpcg_options* opt, int ns, double* ev, double* X, double* P,
                       qg_lobpcg_report* rep) {
    if (!X || (!P && opt && !opt->first_call)) return QG_ERR_INVALID;
    return run_lobpcg(h, opt, ns, 2, ev, X, P, nullptr, nullptr, nullptr, nullptr, rep);
}

}  // extern "C"
