// Small generalised symmetric eigensolver A z = lambda B z on the GPU, FP64,
// one thread block per problem (replaces lapack_DSYGVX, w_dsygvx.h:24-104, for
// the LOBPCG pencils of up to kSmallEigMax rows).
//
//   1. Jacobi equilibration: D = diag(B)^-1/2, A <- D A D, B <- D B D (the
//      eigenvalues are unchanged, z = D z'); it keeps the tiny residual columns
//      of the reference iteration from ruining the Cholesky factorisation;
//   2. Cholesky B = L L^T (right-looking, in shared memory);
//   3. C = L^-1 A L^-T (two triangular solves), symmetrised;
//   4. cyclic parallel Jacobi on C (round-robin pairs, all k/2 rotations of a
//      round at once), until the off-diagonal norm is below 1e-13 of the norm or
//      a bounded number of sweeps;
//   5. z = D L^-T q, eigenpairs sorted ascending.
// Only the lower triangles of A and B are read (UPLO as the reference's call).
// k_small_heg is the complex Hermitian version of the same five steps: complex
// Cholesky B = L L^H, C = L^-1 A L^-H, and Jacobi rotations that first turn the
// phase of C(p, q) away (C(p, q) = |C(p, q)| e^{i phi}; the 2 x 2 unitary is
// diag(1, e^{-i phi}) times the real rotation of the resulting real pencil).
// If B is not positive definite and the problem is an LOBPCG [x r p] pencil
// (k = 3n), the [x r] leading 2n x 2n pencil is solved instead and the rows of
// the P block are returned as zeros: the rotation then reproduces LOBPCG's
// restart without P. info: 0 ok, 1 Cholesky failure (also after the restart),
// 2 Jacobi sweep limit reached, 3 restart used (results valid).
#include <cmath>

#include "qg_internal.h"
#include "small_eig.h"

namespace qg {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxSweeps = 40;

struct SmemEig {
    double* C;   // k*k   working matrix (row-major, symmetric)
    double* C2;  // k*k   second buffer of the Jacobi rounds
    double* L;   // k*k   Cholesky factor
    double* Q;   // k*k   eigenvectors (columns)
    double* d;   // k     equilibration
    double* jd;  // k     J(i, i) of the current round
    double* jo;  // k     J(partner(i), i) of the current round
    int* part;   // k     partner of i in the current round (-1: none)
    int* rank;   // k
};

// Shared-memory layout for a k x k problem: 4 k*k matrices, 3 k-vectors, 2 k int vectors.
__device__ void layout(SmemEig& m, double* base, int k) {
    m.C = base;
    m.C2 = m.C + k * k;
    m.L = m.C2 + k * k;
    m.Q = m.L + k * k;
    m.d = m.Q + k * k;
    m.jd = m.d + k;
    m.jo = m.jd + k;
    m.part = reinterpret_cast<int*>(m.jo + k);
    m.rank = m.part + k;
}

__device__ bool factor_and_reduce(const double* __restrict__ A, const double* __restrict__ B, int lda, int k,
                                  SmemEig& m) {
    const int t = threadIdx.x, nt = blockDim.x;
    __shared__ int fail;
    __syncthreads();  // every thread is past any earlier read of `fail`
    if (t == 0) fail = 0;
    __syncthreads();
    for (int i = t; i < k; i += nt) {
        const double b = B[i + (long long)i * lda];
        m.d[i] = b > 0.0 ? 1.0 / sqrt(b) : 1.0;
        if (!(b > 0.0)) fail = 1;
    }
    __syncthreads();
    if (fail) return false;
    // lower triangles (column-major input: element (i, j), i >= j, at i + j*lda), symmetrised
    for (int e = t; e < k * k; e += nt) {
        const int i = e / k, j = e % k;
        const int r = i >= j ? i : j, c = i >= j ? j : i;
        const double s = m.d[i] * m.d[j];
        m.C[e] = A[r + (long long)c * lda] * s;
        m.L[e] = B[r + (long long)c * lda] * s;
    }
    __syncthreads();
    // Cholesky, right-looking on the lower triangle of L
    for (int j = 0; j < k; ++j) {
        if (t == 0) {
            const double v = m.L[j * k + j];
            if (!(v > 0.0) || !isfinite(v)) fail = 1;
            m.L[j * k + j] = sqrt(v);
        }
        __syncthreads();
        if (fail) return false;
        const double dj = m.L[j * k + j];
        for (int i = j + 1 + t; i < k; i += nt) m.L[i * k + j] /= dj;
        __syncthreads();
        const int rem = k - j - 1;
        for (int e = t; e < rem * rem; e += nt) {
            const int i = j + 1 + e / rem, l = j + 1 + e % rem;
            if (l <= i) m.L[i * k + l] -= m.L[i * k + j] * m.L[l * k + j];
        }
        __syncthreads();
    }
    // Y = L^-1 C (forward substitution down each column), then C = L^-1 Y^T
    for (int pass = 0; pass < 2; ++pass) {
        for (int col = t; col < k; col += nt) {
            for (int i = 0; i < k; ++i) {
                double v = m.C[i * k + col];
                for (int l = 0; l < i; ++l) v -= m.L[i * k + l] * m.C[l * k + col];
                m.C[i * k + col] = v / m.L[i * k + i];
            }
        }
        __syncthreads();
        for (int e = t; e < k * k; e += nt) {  // transpose in place (pairs)
            const int i = e / k, j = e % k;
            if (i < j) {
                const double a = m.C[i * k + j];
                m.C[i * k + j] = m.C[j * k + i];
                m.C[j * k + i] = a;
            }
        }
        __syncthreads();
    }
    for (int e = t; e < k * k; e += nt) {
        const int i = e / k, j = e % k;
        if (i < j) {
            const double a = 0.5 * (m.C[i * k + j] + m.C[j * k + i]);
            m.C[i * k + j] = a;
            m.C[j * k + i] = a;
        }
    }
    for (int e = t; e < k * k; e += nt) m.Q[e] = (e / k == e % k) ? 1.0 : 0.0;
    __syncthreads();
    return true;
}

// Cyclic parallel Jacobi on the symmetric k x k matrix m.C (m.C2 is the second
// buffer); returns false at the sweep limit. Round-robin schedule: k/2 disjoint
// pairs per round; all rotations of a round are computed from the same matrix and
// applied at once as C' = J^T C J, each new element from four old ones.
__device__ bool jacobi(int k, SmemEig& m) {
    const int t = threadIdx.x, nt = blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = nt >> 5;
    const int kk = (k + 1) & ~1;  // even number of seats (one dummy when k is odd)
    const int mm = kk - 1;
    const int npairs = kk / 2;
    __shared__ double red_off[kThreads / 32], red_tot[kThreads / 32];
    __shared__ int done;
    double* C = m.C;
    double* C2 = m.C2;
    for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
        // off-diagonal and total squared norms, reduced in a fixed order
        double so = 0.0, st = 0.0;
        for (int i = warp; i < k; i += nw)
            for (int j = lane; j < k; j += 32) {
                const double v = C[i * k + j] * C[i * k + j];
                st += v;
                if (i != j) so += v;
            }
        for (int o = 16; o > 0; o >>= 1) {
            so += __shfl_xor_sync(0xffffffffu, so, o);
            st += __shfl_xor_sync(0xffffffffu, st, o);
        }
        if (lane == 0) {
            red_off[warp] = so;
            red_tot[warp] = st;
        }
        __syncthreads();
        if (t == 0) {
            double off = 0.0, tot = 0.0;
            for (int wi = 0; wi < nw; ++wi) {
                off += red_off[wi];
                tot += red_tot[wi];
            }
            done = (off <= 1e-26 * tot || off == 0.0) ? 1 : 0;
        }
        __syncthreads();
        if (done) {
            m.C = C;
            m.C2 = C2;
            return true;
        }
        for (int round = 0; round < mm; ++round) {
            // per index: its partner and the two entries of J in its column
            for (int pi = t; pi < npairs; pi += nt) {
                const int a = (pi == 0) ? 0 : ((pi - 1 + round) % mm) + 1;
                const int b = ((kk - 2 - pi + round) % mm) + 1;
                const int p = a < b ? a : b, q = a < b ? b : a;
                double c = 1.0, sn = 0.0;
                if (q < k) {
                    const double apq = C[p * k + q];
                    if (apq != 0.0) {
                        const double th = (C[q * k + q] - C[p * k + p]) / (2.0 * apq);
                        const double tt = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(1.0 + th * th));
                        c = 1.0 / sqrt(1.0 + tt * tt);
                        sn = tt * c;
                    }
                    m.part[p] = q;
                    m.part[q] = p;
                    m.jd[p] = c;
                    m.jd[q] = c;
                    m.jo[p] = -sn;  // J(q, p)
                    m.jo[q] = sn;   // J(p, q)
                } else if (p < k) {
                    m.part[p] = -1;  // paired with the dummy seat
                    m.jd[p] = 1.0;
                    m.jo[p] = 0.0;
                }
            }
            __syncthreads();
            // C2 = J^T C J and Q <- Q J
            for (int i = warp; i < k; i += nw) {
                const int ip = m.part[i];
                const double di = m.jd[i], oi = m.jo[i];
                for (int j = lane; j < k; j += 32) {
                    const int jp = m.part[j];
                    const double dj = m.jd[j], oj = m.jo[j];
                    double v = di * dj * C[i * k + j];
                    if (ip >= 0) v += oi * dj * C[ip * k + j];
                    if (jp >= 0) v += di * oj * C[i * k + jp];
                    if (ip >= 0 && jp >= 0) v += oi * oj * C[ip * k + jp];
                    C2[i * k + j] = v;
                }
            }
            for (int i = warp; i < k; i += nw) {  // each (row, pair) updates its two columns of Q
                for (int j = lane; j < k; j += 32) {
                    const int jp = m.part[j];
                    if (jp > j || jp < 0) {
                        const double qj = m.Q[i * k + j];
                        if (jp < 0) continue;
                        const double qp = m.Q[i * k + jp];
                        m.Q[i * k + j] = m.jd[j] * qj + m.jo[j] * qp;
                        m.Q[i * k + jp] = m.jo[jp] * qj + m.jd[jp] * qp;
                    }
                }
            }
            __syncthreads();
            double* tmp = C;
            C = C2;
            C2 = tmp;
        }
    }
    m.C = C;
    m.C2 = C2;
    return false;
}

// z = D L^-T q for every column, sorted by eigenvalue; writes Z (column-major, ldz) and w.
__device__ void back_transform(int k, int kout, SmemEig& m, double* __restrict__ Z, int ldz, double* __restrict__ w,
                               int zero_rows_from, int zero_rows_to) {
    const int t = threadIdx.x, nt = blockDim.x;
    for (int col = t; col < k; col += nt) {  // solve L^T y = q (backward)
        for (int i = k - 1; i >= 0; --i) {
            double v = m.Q[i * k + col];
            for (int l = i + 1; l < k; ++l) v -= m.L[l * k + i] * m.Q[l * k + col];
            m.Q[i * k + col] = v / m.L[i * k + i];
        }
    }
    for (int i = t; i < k; i += nt) {
        const double li = m.C[i * k + i];
        int r = 0;
        for (int j = 0; j < k; ++j) {
            const double lj = m.C[j * k + j];
            if (lj < li || (lj == li && j < i)) ++r;
        }
        m.rank[i] = r;
    }
    __syncthreads();
    for (int e = t; e < k * k; e += nt) {
        const int row = e / k, col = e % k;
        const int r = m.rank[col];
        Z[row + (long long)r * ldz] = m.d[row] * m.Q[row * k + col];
    }
    for (int i = t; i < k; i += nt) w[m.rank[i]] = m.C[i * k + i];
    for (int e = t; e < (zero_rows_to - zero_rows_from) * k; e += nt) {
        const int row = zero_rows_from + e / k, col = e % k;
        Z[row + (long long)col * ldz] = 0.0;
    }
}

__global__ void __launch_bounds__(kThreads) k_small_eig(const double* __restrict__ A, const double* __restrict__ B,
                                                         int lda, long long stride_ab, int k, int n_restart,
                                                         double* __restrict__ Z, int ldz, long long stride_z,
                                                         double* __restrict__ w, long long stride_w,
                                                         int* __restrict__ info) {
    extern __shared__ __align__(16) double sm_eig[];
    const long long bid = blockIdx.x;
    A += bid * stride_ab;
    B += bid * stride_ab;
    Z += bid * stride_z;
    w += bid * stride_w;
    int kk = k;
    SmemEig m;
    layout(m, sm_eig, k);
    int status = 0;
    bool ok = factor_and_reduce(A, B, lda, kk, m);
    if (!ok && n_restart > 0 && n_restart < k) {
        kk = n_restart;  // [x r] pencil: the leading n_restart rows and columns
        layout(m, sm_eig, kk);
        ok = factor_and_reduce(A, B, lda, kk, m);
        status = 3;
    }
    if (!ok) {
        if (threadIdx.x == 0) info[bid] = 1;
        return;
    }
    if (!jacobi(kk, m)) status = 2;
    back_transform(kk, kk, m, Z, ldz, w, kk, k);
    if (threadIdx.x == 0) info[bid] = status;
}

// ---------------------------------------------------------------------------
// Complex Hermitian pencils (double2 = {re, im}).

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b) {  // conj(a) * b
    return make_double2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }

struct SmemHeg {
    double2* C;   // k*k working matrix (row-major, Hermitian)
    double2* C2;  // k*k second buffer of the Jacobi rounds
    double2* L;   // k*k Cholesky factor (lower)
    double2* Q;   // k*k eigenvectors (columns)
    double2* jd;  // k    U(i, i) of the current round
    double2* jo;  // k    U(partner(i), i)
    double* d;    // k    equilibration
    int* part;    // k
    int* rank;    // k
};

__device__ void layout_heg(SmemHeg& m, double2* base, int k) {
    m.C = base;
    m.C2 = m.C + k * k;
    m.L = m.C2 + k * k;
    m.Q = m.L + k * k;
    m.jd = m.Q + k * k;
    m.jo = m.jd + k;
    m.d = reinterpret_cast<double*>(m.jo + k);
    m.part = reinterpret_cast<int*>(m.d + k);
    m.rank = m.part + k;
}

// Loads the lower triangles of A and B (column-major, lda), equilibrates with
// D = diag(B)^-1/2, factors B = L L^H and forms C = L^-1 A L^-H (Hermitian).
__device__ bool heg_factor_and_reduce(const double2* __restrict__ A, const double2* __restrict__ B, int lda, int k,
                                      SmemHeg& m, double pivot_floor) {
    const int t = threadIdx.x, nt = blockDim.x;
    __shared__ int fail;
    __syncthreads();
    if (t == 0) fail = 0;
    __syncthreads();
    for (int i = t; i < k; i += nt) {
        const double b = B[i + (long long)i * lda].x;
        m.d[i] = b > 0.0 ? 1.0 / sqrt(b) : 1.0;
        if (!(b > 0.0)) fail = 1;
    }
    __syncthreads();
    if (fail) return false;
    for (int e = t; e < k * k; e += nt) {
        const int i = e / k, j = e % k;
        const double s = m.d[i] * m.d[j];
        double2 a, b;
        if (i >= j) {
            a = A[i + (long long)j * lda];
            b = B[i + (long long)j * lda];
        } else {
            a = cconj(A[j + (long long)i * lda]);
            b = cconj(B[j + (long long)i * lda]);
        }
        if (i == j) a.y = b.y = 0.0;
        m.C[e] = cscale(a, s);
        m.L[e] = cscale(b, s);
    }
    __syncthreads();
    // Cholesky B = L L^H, right-looking on the lower triangle
    for (int j = 0; j < k; ++j) {
        if (t == 0) {
            const double v = m.L[j * k + j].x;
            if (!(v > pivot_floor) || !(v > 0.0) || !isfinite(v)) fail = 1;
            m.L[j * k + j] = make_double2(sqrt(v), 0.0);
        }
        __syncthreads();
        if (fail) return false;
        const double dj = m.L[j * k + j].x;
        for (int i = j + 1 + t; i < k; i += nt) m.L[i * k + j] = cscale(m.L[i * k + j], 1.0 / dj);
        __syncthreads();
        const int rem = k - j - 1;
        for (int e = t; e < rem * rem; e += nt) {
            const int i = j + 1 + e / rem, l = j + 1 + e % rem;
            if (l <= i) m.L[i * k + l] = csub(m.L[i * k + l], cmul(m.L[i * k + j], cconj(m.L[l * k + j])));
        }
        __syncthreads();
    }
    // Y = L^-1 C, then Y^H; twice: (L^-1 (L^-1 C)^H)^H = L^-1 C L^-H
    for (int pass = 0; pass < 2; ++pass) {
        for (int col = t; col < k; col += nt) {
            for (int i = 0; i < k; ++i) {
                double2 v = m.C[i * k + col];
                for (int l = 0; l < i; ++l) v = csub(v, cmul(m.L[i * k + l], m.C[l * k + col]));
                m.C[i * k + col] = cscale(v, 1.0 / m.L[i * k + i].x);
            }
        }
        __syncthreads();
        for (int e = t; e < k * k; e += nt) {  // conjugate transpose in place
            const int i = e / k, j = e % k;
            if (i < j) {
                const double2 a = m.C[i * k + j];
                m.C[i * k + j] = cconj(m.C[j * k + i]);
                m.C[j * k + i] = cconj(a);
            } else if (i == j) {
                m.C[e] = cconj(m.C[e]);
            }
        }
        __syncthreads();
    }
    for (int e = t; e < k * k; e += nt) {  // Hermitian part
        const int i = e / k, j = e % k;
        if (i < j) {
            const double2 a = cscale(cadd(m.C[i * k + j], cconj(m.C[j * k + i])), 0.5);
            m.C[i * k + j] = a;
            m.C[j * k + i] = cconj(a);
        } else if (i == j) {
            m.C[e].y = 0.0;
        }
    }
    for (int e = t; e < k * k; e += nt) m.Q[e] = make_double2((e / k == e % k) ? 1.0 : 0.0, 0.0);
    __syncthreads();
    return true;
}

// Cyclic parallel Jacobi on the Hermitian matrix m.C: round-robin pairs, all
// rotations of a round applied at once as C' = U^H C U (each new element from four
// old ones); Q <- Q U. Returns false at the sweep limit.
__device__ bool heg_jacobi(int k, SmemHeg& m) {
    const int t = threadIdx.x, nt = blockDim.x;
    const int lane = t & 31, warp = t >> 5, nw = nt >> 5;
    const int kk = (k + 1) & ~1;
    const int mm = kk - 1;
    const int npairs = kk / 2;
    __shared__ double red_off[kThreads / 32], red_tot[kThreads / 32];
    __shared__ int done;
    double2* C = m.C;
    double2* C2 = m.C2;
    for (int sweep = 0; sweep < kMaxSweeps; ++sweep) {
        double so = 0.0, st = 0.0;
        for (int i = warp; i < k; i += nw)
            for (int j = lane; j < k; j += 32) {
                const double2 c = C[i * k + j];
                const double v = c.x * c.x + c.y * c.y;
                st += v;
                if (i != j) so += v;
            }
        for (int o = 16; o > 0; o >>= 1) {
            so += __shfl_xor_sync(0xffffffffu, so, o);
            st += __shfl_xor_sync(0xffffffffu, st, o);
        }
        if (lane == 0) {
            red_off[warp] = so;
            red_tot[warp] = st;
        }
        __syncthreads();
        if (t == 0) {
            double off = 0.0, tot = 0.0;
            for (int wi = 0; wi < nw; ++wi) {
                off += red_off[wi];
                tot += red_tot[wi];
            }
            done = (off <= 1e-26 * tot || off == 0.0) ? 1 : 0;
        }
        __syncthreads();
        if (done) {
            m.C = C;
            m.C2 = C2;
            return true;
        }
        for (int round = 0; round < mm; ++round) {
            for (int pi = t; pi < npairs; pi += nt) {
                const int a = (pi == 0) ? 0 : ((pi - 1 + round) % mm) + 1;
                const int b = ((kk - 2 - pi + round) % mm) + 1;
                const int p = a < b ? a : b, q = a < b ? b : a;
                if (q < k) {
                    double c = 1.0, sn = 0.0;
                    double2 ph = make_double2(1.0, 0.0);  // e^{-i phi}
                    const double2 cpq = C[p * k + q];
                    const double apq = hypot(cpq.x, cpq.y);
                    if (apq != 0.0) {
                        ph = make_double2(cpq.x / apq, -cpq.y / apq);
                        const double th = (C[q * k + q].x - C[p * k + p].x) / (2.0 * apq);
                        const double tt = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(1.0 + th * th));
                        c = 1.0 / sqrt(1.0 + tt * tt);
                        sn = tt * c;
                    }
                    // U = diag(1, e^{-i phi}) J, J = [[c, s], [-s, c]] on (p, q)
                    m.part[p] = q;
                    m.part[q] = p;
                    m.jd[p] = make_double2(c, 0.0);    // U(p, p)
                    m.jo[p] = cscale(ph, -sn);         // U(q, p)
                    m.jd[q] = cscale(ph, c);           // U(q, q)
                    m.jo[q] = make_double2(sn, 0.0);   // U(p, q)
                } else if (p < k) {
                    m.part[p] = -1;
                    m.jd[p] = make_double2(1.0, 0.0);
                    m.jo[p] = make_double2(0.0, 0.0);
                }
            }
            __syncthreads();
            // C2(i, j) = sum_{a in {i, ip}, b in {j, jp}} conj(U(a, i)) C(a, b) U(b, j)
            for (int i = warp; i < k; i += nw) {
                const int ip = m.part[i];
                const double2 di = m.jd[i], oi = m.jo[i];
                for (int j = lane; j < k; j += 32) {
                    const int jp = m.part[j];
                    const double2 dj = m.jd[j], oj = m.jo[j];
                    double2 v = cmulc(di, cmul(C[i * k + j], dj));
                    if (ip >= 0) v = cadd(v, cmulc(oi, cmul(C[ip * k + j], dj)));
                    if (jp >= 0) v = cadd(v, cmulc(di, cmul(C[i * k + jp], oj)));
                    if (ip >= 0 && jp >= 0) v = cadd(v, cmulc(oi, cmul(C[ip * k + jp], oj)));
                    C2[i * k + j] = v;
                }
            }
            // Q(r, j) <- Q(r, j) U(j, j) + Q(r, jp) U(jp, j), both columns of a pair together
            for (int i = warp; i < k; i += nw) {
                for (int j = lane; j < k; j += 32) {
                    const int jp = m.part[j];
                    if (jp > j) {
                        const double2 qj = m.Q[i * k + j], qp = m.Q[i * k + jp];
                        m.Q[i * k + j] = cadd(cmul(qj, m.jd[j]), cmul(qp, m.jo[j]));
                        m.Q[i * k + jp] = cadd(cmul(qj, m.jo[jp]), cmul(qp, m.jd[jp]));
                    }
                }
            }
            __syncthreads();
            double2* tmp = C;
            C = C2;
            C2 = tmp;
        }
    }
    m.C = C;
    m.C2 = C2;
    return false;
}

// z = D L^-H q for every column, sorted by eigenvalue.
__device__ void heg_back_transform(int k, SmemHeg& m, double2* __restrict__ Z, int ldz, double* __restrict__ w) {
    const int t = threadIdx.x, nt = blockDim.x;
    for (int col = t; col < k; col += nt) {  // L^H y = q, backward
        for (int i = k - 1; i >= 0; --i) {
            double2 v = m.Q[i * k + col];
            for (int l = i + 1; l < k; ++l) v = csub(v, cmulc(m.L[l * k + i], m.Q[l * k + col]));
            m.Q[i * k + col] = cscale(v, 1.0 / m.L[i * k + i].x);
        }
    }
    for (int i = t; i < k; i += nt) {
        const double li = m.C[i * k + i].x;
        int r = 0;
        for (int j = 0; j < k; ++j) {
            const double lj = m.C[j * k + j].x;
            if (lj < li || (lj == li && j < i)) ++r;
        }
        m.rank[i] = r;
    }
    __syncthreads();
    for (int e = t; e < k * k; e += nt) {
        const int row = e / k, col = e % k;
        Z[row + (long long)m.rank[col] * ldz] = cscale(m.Q[row * k + col], m.d[row]);
    }
    for (int i = t; i < k; i += nt) w[m.rank[i]] = m.C[i * k + i].x;
}

__global__ void __launch_bounds__(kThreads) k_small_heg(const double2* __restrict__ A, const double2* __restrict__ B,
                                                         int lda, long long stride_ab, int k,
                                                         const int* __restrict__ skip, double2* Z, int ldz,
                                                         long long stride_z, double* __restrict__ w,
                                                         long long stride_w, int* __restrict__ info,
                                                         double pivot_floor) {
    extern __shared__ __align__(16) double2 sm_heg[];
    const long long bid = blockIdx.x;
    if (skip && skip[bid]) {
        if (threadIdx.x == 0) info[bid] = 0;
        return;
    }
    A += bid * stride_ab;
    B += bid * stride_ab;
    Z += bid * stride_z;
    w += bid * stride_w;
    SmemHeg m;
    layout_heg(m, sm_heg, k);
    if (!heg_factor_and_reduce(A, B, lda, k, m, pivot_floor)) {
        if (threadIdx.x == 0) info[bid] = 1;
        return;
    }
    const int status = heg_jacobi(k, m) ? 0 : 2;
    heg_back_transform(k, m, Z, ldz, w);
    if (threadIdx.x == 0) info[bid] = status;
}

}  // namespace

size_t small_heg_smem(int k) {
    return (size_t)(4 * k * k + 2 * k) * sizeof(double2) + (size_t)k * sizeof(double) + (size_t)2 * k * sizeof(int);
}

int small_heg_launch(const double2* A, const double2* B, int lda, long long stride_ab, int k, const int* skip,
                     double2* Z, int ldz, long long stride_z, double* w, long long stride_w, int* info, int batch,
                     cudaStream_t st, double pivot_floor) {
    if (k <= 0 || k > kSmallHegMax || batch <= 0) return QG_ERR_UNSUPPORTED;
    const size_t smem = small_heg_smem(k);
    if (smem > 48 * 1024)
        QG_CUDA_TRY(allow_max_dynamic_smem(k_small_heg));
    k_small_heg<<<batch, kThreads, smem, st>>>(A, B, lda, stride_ab, k, skip, Z, ldz, stride_z, w, stride_w, info,
                                               pivot_floor);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

namespace {
}  // namespace

size_t small_eig_smem(int k) { return (size_t)(4 * k * k + 4 * k + 2) * sizeof(double); }

int small_eig_launch(const double* A, const double* B, int lda, long long stride_ab, int k, int n_restart, double* Z,
                     int ldz, long long stride_z, double* w, long long stride_w, int* info, int batch,
                     cudaStream_t st) {
    if (k <= 0 || k > kSmallEigMax || batch <= 0) return QG_ERR_UNSUPPORTED;
    const size_t smem = small_eig_smem(k);
    if (smem > 48 * 1024) {
        QG_CUDA_TRY(allow_max_dynamic_smem(k_small_eig));
    }
    k_small_eig<<<batch, kThreads, smem, st>>>(A, B, lda, stride_ab, k, n_restart, Z, ldz, stride_z, w, stride_w,
                                               info);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

}  // namespace qg

extern "C" int qg_sygv_small_batched_d(qg_context ctx, int batch, int k, const double* A, const double* B, int lda,
                                       long long stride, double* w, double* Z, int* info) {
    if (!ctx || batch <= 0 || k <= 0 || lda < k || !A || !B || !w || !Z) return QG_ERR_INVALID;
    if (k > qg::kSmallEigMax) return QG_ERR_UNSUPPORTED;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    int* info_d = nullptr;
    QG_CUDA_TRY(cudaMallocAsync(&info_d, sizeof(int) * batch, ctx->stream));
    int rc = qg::small_eig_launch(A, B, lda, stride, k, 0, Z, k, (long long)k * k, w, k, info_d, batch, ctx->stream);
    if (rc == QG_OK && info) {
        if (cudaMemcpyAsync(info, info_d, sizeof(int) * batch, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            rc = QG_ERR_CUDA;
        for (int b = 0; rc == QG_OK && b < batch; ++b)
            if (info[b] == 2) info[b] = 0;  // sweep limit: result kept
    }
    cudaFreeAsync(info_d, ctx->stream);
    return rc;
}

extern "C" int qg_hegv_small_batched_z(qg_context ctx, int batch, int k, const double* A, const double* B, int lda,
                                       long long stride, double* w, double* Z, int* info) {
    if (!ctx || batch <= 0 || k <= 0 || lda < k || !A || !B || !w || !Z) return QG_ERR_INVALID;
    if (k > qg::kSmallHegMax) return QG_ERR_UNSUPPORTED;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    int* info_d = nullptr;
    QG_CUDA_TRY(cudaMallocAsync(&info_d, sizeof(int) * batch, ctx->stream));
    int rc = qg::small_heg_launch(reinterpret_cast<const double2*>(A), reinterpret_cast<const double2*>(B), lda,
                                  stride, k, nullptr, reinterpret_cast<double2*>(Z), k, (long long)k * k, w, k, info_d,
                                  batch, ctx->stream);
    if (rc == QG_OK && info) {
        if (cudaMemcpyAsync(info, info_d, sizeof(int) * batch, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
            cudaStreamSynchronize(ctx->stream) != cudaSuccess)
            rc = QG_ERR_CUDA;
        for (int b = 0; rc == QG_OK && b < batch; ++b)
            if (info[b] == 2) info[b] = 0;  // sweep limit: result kept
    }
    cudaFreeAsync(info_d, ctx->stream);
    return rc;
}
