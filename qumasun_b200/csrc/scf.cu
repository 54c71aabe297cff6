// The SCF-step neighbours of the eigensolver on the device:
//  * electron density rho = sum_s f_s |psi_s|^2 (mSetDensityOne,
//    qumasun_single.density.h:10-27; complex: qumasun_kpoint.density.h:11-33);
//  * Fermi occupations by bisection on the chemical potential (SetOccupancy.h:7-18 inside
//    mSetOccupancySpinOff / SpinOn, qumasun_single.occupancy.h:19-109) -- host scalar work;
//  * Hartree potential by the FFT Poisson solve plus LDA (Perdew-Zunger 81) exchange and
//    correlation, V_tot = V_ext + V_hart + V_x + V_c (mSetPotential for KohnSham_PP,
//    qumasun_single.potential.h:33-43; SetPotentialByPoissonFFT, poisson_fft.h:14-128;
//    Calc_XC_LDA, Vxc.h:41-70);
//  * one fourth-order Taylor step of the time-dependent propagation (QUMASUN::TimeEvoH4,
//    qumasun_td.time_evo_H4.h:13-60), batched over all states;
//  * nonlocal energy and forces (QUMASUN_MPI::mGetForcePseudoNonlocal,
//    qumasun_mpi.force.h:227-254, PseudoPotIntegrator_mpi::ForceNonlocal,
//    PseudoPotOperator_mpi_v2.h:905-1010; k-point form PseudoPotOperator_kpoint_v2.h:2760-2866).
#include <cufft.h>

#include <cmath>
#include <vector>

#include "qg_internal.h"

namespace qg {
namespace {

constexpr int kThreads = 256;

int grid_for(long long n, int per_sm = 8) {
    const long long b = (n + kThreads - 1) / kThreads;
    return (int)std::max<long long>(1, std::min<long long>(b, 148LL * per_sm));
}

// rho[i] (+)= sum_j f[j] * |psi_{idx[j]}[i]|^2, the listed states in order, each term
// rounded as the reference forms it: ((p*p) [+ q*q]) * f added to rho (no fused
// multiply-add), so the sums match the reference's bit for bit on the same inputs.
template <bool CPLX>
__global__ void __launch_bounds__(kThreads) k_density(long long N, int nocc, const int* __restrict__ idx,
                                                      const double* __restrict__ f, const double* __restrict__ X,
                                                      long long ldx, double* __restrict__ rho, int accumulate) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double r = accumulate ? rho[i] : 0.0;
        int j = 0;
        for (; j + 4 <= nocc; j += 4) {
            double t[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const double* xs = X + (long long)__ldg(&idx[j + u]) * ldx;
                const double p = xs[i];
                t[u] = __dmul_rn(p, p);
                if constexpr (CPLX) {
                    const double q = xs[N + i];
                    t[u] = __dadd_rn(t[u], __dmul_rn(q, q));
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) r = __dadd_rn(r, __dmul_rn(t[u], __ldg(&f[j + u])));
        }
        for (; j < nocc; ++j) {
            const double* xs = X + (long long)__ldg(&idx[j]) * ldx;
            const double p = xs[i];
            double t = __dmul_rn(p, p);
            if constexpr (CPLX) {
                const double q = xs[N + i];
                t = __dadd_rn(t, __dmul_rn(q, q));
            }
            r = __dadd_rn(r, __dmul_rn(t, __ldg(&f[j])));
        }
        rho[i] = r;
    }
}

template <bool CPLX>
int density(qg_context c, long long N, int ns, const double* X, long long ldx, const double* occ, double* rho,
            int accumulate) {
    if (!c || N <= 0 || ns < 0 || !rho || (ns > 0 && (!X || !occ))) return QG_ERR_INVALID;
    if (ldx < (CPLX ? 2 * N : N)) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(c->device));
    // states with a positive occupation, in order (the reference skips the others)
    std::vector<int> idx;
    std::vector<double> f;
    for (int s = 0; s < ns; ++s)
        if (occ[s] > 0.0) {
            idx.push_back(s);
            f.push_back(occ[s]);
        }
    const int nocc = (int)idx.size();
    if (nocc == 0) {
        if (!accumulate) QG_CUDA_TRY(cudaMemsetAsync(rho, 0, (size_t)N * sizeof(double), c->stream));
        return QG_OK;
    }
    QG_CUDA_TRY(cudaStreamSynchronize(c->stream));  // the list buffer may still be read by the last call
    QG_TRY(c->small.reserve((size_t)nocc * (sizeof(double) + sizeof(int))));
    double* fd = c->small.as<double>();
    int* id = reinterpret_cast<int*>(fd + nocc);
    QG_CUDA_TRY(cudaMemcpyAsync(fd, f.data(), nocc * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    QG_CUDA_TRY(cudaMemcpyAsync(id, idx.data(), nocc * sizeof(int), cudaMemcpyHostToDevice, c->stream));
    k_density<CPLX><<<grid_for(N), kThreads, 0, c->stream>>>(N, nocc, id, fd, X, ldx, rho, accumulate);
    QG_CUDA_TRY(cudaGetLastError());
    QG_CUDA_TRY(cudaStreamSynchronize(c->stream));  // the host lists go out of scope
    return QG_OK;
}

// Fermi occupations at chemical potential mu (SetOccupancy.h:7-18); returns their sum.
double fermi(double coef, double kbT, int n, const double* ev, double mu, double* occ) {
    constexpr double PMAX = 80.0;
    const double beta = 1.0 / kbT;
    double sum = 0.0;
    for (int s = 0; s < n; ++s) {
        const double p = std::min(beta * (ev[s] - mu), PMAX);
        occ[s] = coef / (std::exp(p) + 1.0);
        sum += occ[s];
    }
    return sum;
}

// ---------------------------------------------------------------- Poisson + LDA

// Perdew-Zunger 1981 LDA exchange and correlation potentials at density rho (the
// unpolarised branch of the published parametrisation, as Calc_XC_LDA uses it:
// gamma, beta1, beta2 for rs >= 1; A, B, C, D for rs < 1).
struct LdaConst {
    double c2, c3;  // (3/(4 pi))^(1/3), -(3/(4 pi)) (9 pi/4)^(1/3)
};

__device__ __forceinline__ void lda_pz81(double rho, const LdaConst& k, double& vx, double& vc) {
    if (rho < 1.0e-8) {
        vx = 0.0;
        vc = 0.0;
        return;
    }
    const double rs = k.c2 / cbrt(rho);
    const double ex0 = k.c3 / rs;
    const double ndex0 = ex0 / 3.0;
    double ec, ndec;
    if (rs >= 1.0) {
        const double gamma = -0.1423, b1 = 1.0529, b2 = 0.3334;
        const double sq = sqrt(rs);
        ec = gamma / (1.0 + b1 * sq + b2 * rs);
        ndec = ec * ec * (b1 * 0.5 * sq + b2 * rs) / (3.0 * gamma);
    } else {
        const double A = 0.0311, B = -0.0480, C = 0.0020, D = -0.0116;
        const double lr = log(rs);
        ec = B + A * lr + D * rs + C * rs * lr;
        ndec = -(A + (D + C) * rs + C * rs * lr) / 3.0;
    }
    vx = ex0 + ndex0;
    vc = ec + ndec;
}

__global__ void __launch_bounds__(kThreads) k_pack_complex(long long N, const double* __restrict__ rho,
                                                           cufftDoubleComplex* __restrict__ buf) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
        buf[i] = make_cuDoubleComplex(rho[i], 0.0);
}

// rho(k) *= 4 pi / |k|^2 with the folded wave numbers of the reference (k = 0 dropped).
__global__ void __launch_bounds__(kThreads) k_poisson_scale(int nx, int ny, int nz, double c1x, double c1y, double c1z,
                                                            cufftDoubleComplex* __restrict__ buf) {
    const long long N = (long long)nx * ny * nz;
    const double four_pi = 4.0 * 3.14159265358979323846;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const int kx = (int)(i % nx);
        const int ky = (int)((i / nx) % ny);
        const int kz = (int)(i / ((long long)nx * ny));
        if (i == 0) {
            buf[i] = make_cuDoubleComplex(0.0, 0.0);
            continue;
        }
        const double fx = c1x * (double)(kx < nx / 2 ? kx : kx - nx);
        const double fy = c1y * (double)(ky < ny / 2 ? ky : ky - ny);
        const double fz = c1z * (double)(kz < nz / 2 ? kz : kz - nz);
        const double s = four_pi / (fx * fx + fy * fy + fz * fz);
        buf[i] = make_cuDoubleComplex(buf[i].x * s, buf[i].y * s);
    }
}

__global__ void __launch_bounds__(kThreads) k_potential_finish(long long N, double invN,
                                                               const cufftDoubleComplex* __restrict__ buf,
                                                               const double* __restrict__ rho,
                                                               const double* __restrict__ pcc,
                                                               const double* __restrict__ vext, LdaConst k,
                                                               double* __restrict__ vtot, double* __restrict__ vhart,
                                                               double* __restrict__ vxo, double* __restrict__ vco) {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        const double vh = buf[i].x * invN;
        double vx, vc;
        lda_pz81(rho[i] + (pcc ? pcc[i] : 0.0), k, vx, vc);
        if (vhart) vhart[i] = vh;
        if (vxo) vxo[i] = vx;
        if (vco) vco[i] = vc;
        vtot[i] = ((vext[i] + vh) + vx) + vc;
    }
}

// ---------------------------------------------------------------- Taylor-4 propagation

// X += a * W for both parts (REAL_STEP), or X.re += a * W.im, X.im += b * W.re; each
// product rounded before the add, as the reference's separate loops form them.
template <bool REAL_STEP>
__global__ void __launch_bounds__(kThreads) k_td_update(int ns, long long N, double* __restrict__ X, long long ldx,
                                                        const double* __restrict__ W, long long ldw, double a, double b) {
    const long long total = (long long)ns * N;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const long long s = t / N, i = t - s * N;
        double* xr = X + s * ldx + i;
        double* xi = xr + N;
        const double* wr = W + s * ldw + i;
        const double* wi = wr + N;
        if constexpr (REAL_STEP) {
            *xr = __dadd_rn(*xr, __dmul_rn(a, *wr));
            *xi = __dadd_rn(*xi, __dmul_rn(a, *wi));
        } else {
            const double re = *wr, im = *wi;
            *xr = __dadd_rn(*xr, __dmul_rn(a, im));
            *xi = __dadd_rn(*xi, __dmul_rn(b, re));
        }
    }
}

// ---------------------------------------------------------------- nonlocal forces

// out_d[c][i] = coef_c * d psi_c / d axis at i, 8th order, periodic; cf[c*12 + 4*axis + (0..3)]
// holds (c1, c2, c3, c4) * coef_c / (840 h) with (672, -168, 32, -3), summed from the
// outermost pair inwards as Gradient8th_{x,y,z}_halo_f (GridGradient8th.h:19-190) does.
__global__ void __launch_bounds__(kThreads) k_gradient8(int nx, int ny, int nz, int nc, const double* __restrict__ X,
                                                        long long ldx, const int* __restrict__ sidx,
                                                        const double* __restrict__ cf, double* __restrict__ out,
                                                        long long ldo) {
    const long long N = (long long)nx * ny * nz;
    const long long total = (long long)nc * N;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / N);
        const long long i = t - (long long)c * N;
        const int ix = (int)(i % nx), iy = (int)((i / nx) % ny), iz = (int)(i / ((long long)nx * ny));
        const double* p = X + (long long)sidx[c] * ldx;
        const double* k = cf + c * 12;
        double g[3];
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
            double d[5];  // p(+s) - p(-s), s = 1..4
#pragma unroll
            for (int s = 1; s <= 4; ++s) {
                long long ip, im;
                if (ax == 0) {
                    ip = i - ix + (ix + s) % nx;
                    im = i - ix + (ix - s + nx) % nx;
                } else if (ax == 1) {
                    ip = i + (long long)(((iy + s) % ny) - iy) * nx;
                    im = i + (long long)(((iy - s + ny) % ny) - iy) * nx;
                } else {
                    ip = i + (long long)(((iz + s) % nz) - iz) * nx * ny;
                    im = i + (long long)(((iz - s + nz) % nz) - iz) * nx * ny;
                }
                d[s] = p[ip] - p[im];
            }
            g[ax] = k[4 * ax + 3] * d[4] + k[4 * ax + 2] * d[3] + k[4 * ax + 1] * d[2] + k[4 * ax + 0] * d[1];
        }
        out[(long long)c * ldo + i] = g[0];
        out[(long long)(nc + c) * ldo + i] = g[1];
        out[(long long)(2 * nc + c) * ldo + i] = g[2];
    }
}

// Per chunk of nc states: e[c] = sum_{a,ch} E inner^2 and, for every atom,
// f[3a + d] += sum_c sum_ch E inner dinner_d (states in order, channels in order).
__global__ void __launch_bounds__(kThreads) k_force_reduce(int na, int nch, int nc, long long ldc,
                                                           const double* __restrict__ inner,
                                                           const double* __restrict__ dinner,  // [3][na*nch][ldc]
                                                           const double* __restrict__ chE, const int* __restrict__ use,
                                                           double* __restrict__ forces, double* __restrict__ e_out) {
    const long long plane = (long long)na * nch * ldc;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < na + nc; t += gridDim.x * blockDim.x) {
        if (t < na) {
            const int a = t;
            double f[3] = {forces[3 * a], forces[3 * a + 1], forces[3 * a + 2]};
            for (int c = 0; c < nc; ++c) {
                if (!use[c]) continue;
                double fi[3] = {0.0, 0.0, 0.0};
                for (int ch = 0; ch < nch; ++ch) {
                    const long long q = (long long)(a * nch + ch) * ldc + c;
                    const double E = chE[a * nch + ch];
                    const double in = inner[q];
#pragma unroll
                    for (int d = 0; d < 3; ++d) fi[d] += dinner[d * plane + q] * in * E;
                }
#pragma unroll
                for (int d = 0; d < 3; ++d) f[d] += fi[d];
            }
            forces[3 * a] = f[0];
            forces[3 * a + 1] = f[1];
            forces[3 * a + 2] = f[2];
        } else {
            const int c = t - na;
            double e = 0.0;
            for (int q = 0; q < na * nch; ++q) {
                const double in = inner[(long long)q * ldc + c];
                e += in * in * chE[q];
            }
            e_out[c] = e;
        }
    }
}

}  // namespace
}  // namespace qg

struct qg_poisson_s {
    qg_context ctx = nullptr;
    int nx = 0, ny = 0, nz = 0;
    double hx = 0, hy = 0, hz = 0;
    cufftHandle plan = 0;
    bool plan_ok = false;
    cufftDoubleComplex* buf = nullptr;
};

extern "C" {

int qg_density_d(qg_context ctx, long long N, int ns, const double* X, long long ldx, const double* occ, double* rho,
                 int accumulate) {
    return qg::density<false>(ctx, N, ns, X, ldx, occ, rho, accumulate);
}

int qg_density_z(qg_context ctx, long long N, int ns, const double* X, long long ldx, const double* occ, double* rho,
                 int accumulate) {
    return qg::density<true>(ctx, N, ns, X, ldx, occ, rho, accumulate);
}

int qg_occupancy(double kbT, int n, const double* ev, int n_electrons, double* occ, double* mu_out) {
    if (n <= 0 || !ev || !occ || !(kbT > 0.0) || n_electrons < 0) return QG_ERR_INVALID;
    const double ne = (double)n_electrons;
    double mu_min = ev[0];
    double mu_max = ev[n - 1];
    mu_max = (mu_max > 0.0) ? mu_max * 16.0 : std::fabs(mu_max) + 16.0;
    if ((n_electrons + 1) / 2 >= n) mu_max *= 10.0;
    double mu = (mu_min + mu_max) / 2.0;
    constexpr double THRESHOLD_MU = 1.0e-9;
    while (std::fabs(mu_max - mu_min) > THRESHOLD_MU) {
        const double num_e = qg::fermi(2.0, kbT, n, ev, mu, occ);
        if (num_e < ne) mu_min = mu;
        else if (num_e > ne) mu_max = mu;
        else break;
        mu = (mu_min + mu_max) / 2.0;
    }
    if (mu_out) *mu_out = mu;
    return QG_OK;
}

int qg_occupancy_spin(double kbT, int n, const double* ev_up, const double* ev_dn, int n_electrons, double* occ_up,
                      double* occ_dn, double* mu_out) {
    if (n <= 0 || !ev_up || !ev_dn || !occ_up || !occ_dn || !(kbT > 0.0) || n_electrons < 0) return QG_ERR_INVALID;
    const double ne = (double)n_electrons;
    double mu_min = std::min(ev_up[0], ev_dn[0]);
    double mu_max = std::max(ev_up[n - 1], ev_dn[n - 1]);
    mu_max = (mu_max > 0.0) ? mu_max * 16.0 : std::fabs(mu_max) + 16.0;
    if ((n_electrons + 1) / 2 >= n) mu_max *= 10.0;
    double mu = (mu_min + mu_max) / 2.0;
    constexpr double THRESHOLD_MU = 1.0e-9;
    while (std::fabs(mu_max - mu_min) > THRESHOLD_MU) {
        const double up = qg::fermi(1.0, kbT, n, ev_up, mu, occ_up);
        const double dn = qg::fermi(1.0, kbT, n, ev_dn, mu, occ_dn);
        const double num_e = up + dn;
        if (num_e < ne) mu_min = mu;
        else if (num_e > ne) mu_max = mu;
        else break;
        mu = (mu_min + mu_max) / 2.0;
    }
    if (mu_out) *mu_out = mu;
    return QG_OK;
}

int qg_poisson_create(qg_context ctx, int nx, int ny, int nz, double hx, double hy, double hz, qg_poisson* out) {
    if (!ctx || !out || nx <= 0 || ny <= 0 || nz <= 0 || !(hx > 0) || !(hy > 0) || !(hz > 0)) return QG_ERR_INVALID;
    *out = nullptr;
    QG_CUDA_TRY(cudaSetDevice(ctx->device));
    qg_poisson p = new qg_poisson_s;
    p->ctx = ctx;
    p->nx = nx; p->ny = ny; p->nz = nz;
    p->hx = hx; p->hy = hy; p->hz = hz;
    const long long N = (long long)nx * ny * nz;
    if (cudaMalloc(&p->buf, (size_t)N * sizeof(cufftDoubleComplex)) != cudaSuccess) {
        delete p;
        return QG_ERR_NOMEM;
    }
    if (cufftPlan3d(&p->plan, nz, ny, nx, CUFFT_Z2Z) != CUFFT_SUCCESS) {
        cudaFree(p->buf);
        delete p;
        qg_set_last_error("cufftPlan3d", "plan creation failed", __FILE__, __LINE__);
        return QG_ERR_LIBRARY;
    }
    p->plan_ok = true;
    ++ctx->live_hamiltonians;  // the context outlives the solver
    *out = p;
    return QG_OK;
}

int qg_poisson_destroy(qg_poisson p) {
    if (!p) return QG_ERR_INVALID;
    cudaSetDevice(p->ctx->device);
    cudaStreamSynchronize(p->ctx->stream);
    if (p->plan_ok) cufftDestroy(p->plan);
    cudaFree(p->buf);
    --p->ctx->live_hamiltonians;
    delete p;
    return QG_OK;
}

int qg_potential_lda_d(qg_poisson p, const double* rho, const double* pcc, const double* vext, double* vtot,
                       double* vhart, double* vx, double* vc) {
    if (!p || !rho || !vext || !vtot) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(p->ctx->device));
    cudaStream_t st = p->ctx->stream;
    const long long N = (long long)p->nx * p->ny * p->nz;
    if (cufftSetStream(p->plan, st) != CUFFT_SUCCESS) return QG_ERR_LIBRARY;
    qg::k_pack_complex<<<qg::grid_for(N), qg::kThreads, 0, st>>>(N, rho, p->buf);
    if (cufftExecZ2Z(p->plan, p->buf, p->buf, CUFFT_FORWARD) != CUFFT_SUCCESS) return QG_ERR_LIBRARY;
    const double PI = 3.14159265358979323846;
    const double c1x = 2.0 * PI / (p->hx * (double)p->nx);
    const double c1y = 2.0 * PI / (p->hy * (double)p->ny);
    const double c1z = 2.0 * PI / (p->hz * (double)p->nz);
    qg::k_poisson_scale<<<qg::grid_for(N), qg::kThreads, 0, st>>>(p->nx, p->ny, p->nz, c1x, c1y, c1z, p->buf);
    if (cufftExecZ2Z(p->plan, p->buf, p->buf, CUFFT_INVERSE) != CUFFT_SUCCESS) return QG_ERR_LIBRARY;
    qg::LdaConst k;
    k.c2 = std::cbrt(3.0 / (4.0 * PI));
    k.c3 = -(3.0 / (4.0 * PI)) * std::cbrt(9.0 * PI / 4.0);
    qg::k_potential_finish<<<qg::grid_for(N), qg::kThreads, 0, st>>>(N, 1.0 / (double)N, p->buf, rho, pcc, vext, k,
                                                                     vtot, vhart, vx, vc);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int qg_td_taylor4_z(qg_hamiltonian h, int ns, double dt, double* X, long long ldx) {
    if (!h || ns < 0 || (ns > 0 && !X)) return QG_ERR_INVALID;
    if (ns == 0) return QG_OK;
    const long long N = h->N();
    if (ldx < 2 * N) return QG_ERR_INVALID;
    if (h->order != 2 && h->order != 6 && h->order != 8) return QG_ERR_UNSUPPORTED;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    cudaStream_t st = h->ctx->stream;
    const long long ldw = 2 * N;
    QG_TRY(h->scf_work.reserve((size_t)2 * ns * ldw * sizeof(double)));
    double* W1 = h->scf_work.as<double>();
    double* W2 = W1 + (size_t)ns * ldw;
    double* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems_z(h, 1, ns) * sizeof(double)));
        coef = h->coef.as<double>();
    }
    const int g = qg::grid_for((long long)ns * N);
    const double c2 = dt * dt / 2.0;
    const double c3 = c2 * dt / 3.0;
    const double c4 = c3 * dt / 4.0;
    // x += -i dt H x
    QG_TRY(qg::apply_hamiltonian_z<double>(h, ns, X, ldx, W1, ldw, coef, st));
    qg::k_td_update<false><<<g, qg::kThreads, 0, st>>>(ns, N, X, ldx, W1, ldw, dt, -dt);
    // x += -(dt^2/2) H^2 x
    QG_TRY(qg::apply_hamiltonian_z<double>(h, ns, W1, ldw, W2, ldw, coef, st));
    qg::k_td_update<true><<<g, qg::kThreads, 0, st>>>(ns, N, X, ldx, W2, ldw, -c2, 0.0);
    // x += i (dt^3/6) H^3 x
    QG_TRY(qg::apply_hamiltonian_z<double>(h, ns, W2, ldw, W1, ldw, coef, st));
    qg::k_td_update<false><<<g, qg::kThreads, 0, st>>>(ns, N, X, ldx, W1, ldw, -c3, c3);
    // x += (dt^4/24) H^4 x
    QG_TRY(qg::apply_hamiltonian_z<double>(h, ns, W1, ldw, W2, ldw, coef, st));
    qg::k_td_update<true><<<g, qg::kThreads, 0, st>>>(ns, N, X, ldx, W2, ldw, c4, 0.0);
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

int qg_nonlocal_force_d(qg_hamiltonian h, int ns, const double* X, long long ldx, const double* occ, double* forces,
                        double* e_state, double* ev_sum) {
    if (!h || ns < 0 || (ns > 0 && (!X || !occ || !forces))) return QG_ERR_INVALID;
    const long long N = h->N();
    if (ldx < N) return QG_ERR_INVALID;
    if (ev_sum) *ev_sum = 0.0;
    const int na = h->pj.na, nch = h->pj.nch;
    if (ns == 0 || na <= 0 || nch <= 0) {
        if (e_state)
            for (int s = 0; s < ns; ++s) e_state[s] = 0.0;
        return QG_OK;
    }
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    cudaStream_t st = h->ctx->stream;
    // chunk of states whose three gradients fit ~1 GiB
    const int nc_max = (int)std::max<long long>(1, std::min<long long>(ns, (1LL << 30) / (3 * N * 8)));
    const long long ldc = qg::coef_ld(nc_max);
    const size_t grad_elems = (size_t)3 * nc_max * N;
    const size_t inner_elems = (size_t)4 * na * nch * ldc;
    const size_t meta = (size_t)nc_max * (12 + 1) + 3 * (size_t)na + nc_max;  // coefficients, flags, forces, energies
    QG_TRY(h->scf_work.reserve((grad_elems + inner_elems + meta) * sizeof(double) + (size_t)2 * nc_max * sizeof(int)));
    double* grad = h->scf_work.as<double>();
    double* inner = grad + grad_elems;
    double* dinner = inner + (size_t)na * nch * ldc;
    double* cf = inner + inner_elems;
    double* fdev = cf + (size_t)nc_max * 12;
    double* edev = fdev + 3 * (size_t)na;
    int* sidx = reinterpret_cast<int*>(edev + nc_max);
    int* use = sidx + nc_max;
    QG_CUDA_TRY(cudaMemcpyAsync(fdev, forces, 3 * (size_t)na * sizeof(double), cudaMemcpyHostToDevice, st));
    const double h3[3] = {h->hx, h->hy, h->hz};
    const double kk[4] = {672.0, -168.0, 32.0, -3.0};
    double ev = 0.0;
    std::vector<double> e_chunk(nc_max), cf_h((size_t)nc_max * 12);
    std::vector<int> sidx_h(nc_max), use_h(nc_max);
    for (int s0 = 0; s0 < ns; s0 += nc_max) {
        const int nc = std::min(nc_max, ns - s0);
        for (int c = 0; c < nc; ++c) {
            const double o = occ[s0 + c];
            const double coef = o > 0.0 ? -2.0 * o : 1.0;  // energies of unoccupied states too
            sidx_h[c] = s0 + c;
            use_h[c] = o > 0.0;
            for (int ax = 0; ax < 3; ++ax)
                for (int j = 0; j < 4; ++j) cf_h[(size_t)c * 12 + 4 * ax + j] = kk[j] * coef / (840.0 * h3[ax]);
        }
        QG_CUDA_TRY(cudaMemcpyAsync(cf, cf_h.data(), (size_t)nc * 12 * sizeof(double), cudaMemcpyHostToDevice, st));
        QG_CUDA_TRY(cudaMemcpyAsync(sidx, sidx_h.data(), nc * sizeof(int), cudaMemcpyHostToDevice, st));
        QG_CUDA_TRY(cudaMemcpyAsync(use, use_h.data(), nc * sizeof(int), cudaMemcpyHostToDevice, st));
        qg::k_gradient8<<<qg::grid_for((long long)nc * N), qg::kThreads, 0, st>>>(h->nx, h->ny, h->nz, nc, X, ldx, sidx,
                                                                                 cf, grad, N);
        QG_TRY(qg::project_inner_d(h, nc, X + (long long)s0 * ldx, ldx, inner, ldc, st));
        for (int d = 0; d < 3; ++d)
            QG_TRY(qg::project_inner_d(h, nc, grad + (size_t)d * nc * N, N, dinner + (size_t)d * na * nch * ldc, ldc,
                                       st));
        qg::k_force_reduce<<<(na + nc + qg::kThreads - 1) / qg::kThreads, qg::kThreads, 0, st>>>(
            na, nch, nc, ldc, inner, dinner, h->pj.ch_E, use, fdev, edev);
        QG_CUDA_TRY(cudaGetLastError());
        QG_CUDA_TRY(cudaMemcpyAsync(e_chunk.data(), edev, nc * sizeof(double), cudaMemcpyDeviceToHost, st));
        QG_CUDA_TRY(cudaStreamSynchronize(st));
        for (int c = 0; c < nc; ++c) {
            // the unoccupied states' gradients were formed with coef 1: their energy is
            // still E inner^2, they add no force (use = 0) and nothing to EV
            if (e_state) e_state[s0 + c] = e_chunk[c];
            if (use_h[c]) ev += e_chunk[c] * occ[s0 + c];
        }
    }
    QG_CUDA_TRY(cudaMemcpyAsync(forces, fdev, 3 * (size_t)na * sizeof(double), cudaMemcpyDeviceToHost, st));
    QG_CUDA_TRY(cudaStreamSynchronize(st));
    if (ev_sum) *ev_sum = ev;
    return QG_OK;
}

}  // extern "C"
