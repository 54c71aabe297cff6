// Kinetic preconditioner for LOBPCG: w = (-1/2 Lap_FD + sigma)^-1 r.
//
// The reference solvers are unpreconditioned (r is used as is,
// lobpcg_d_multi.h:77, :510). This is the plain preconditioner the engine adds:
// the inverse of the shifted kinetic operator, applied in Fourier space with
// the exact symbol of the same finite-difference stencil the Hamiltonian uses,
//   Lap_FD(k) = sum_axis [ c0_axis + 2 sum_s c_s cos(2 pi k s / n_axis) ],
// so T is a positive definite approximation of (H - eps)^-1 that is exact for
// the kinetic part. Batched double-precision R2C / C2R transforms (cuFFT).
#include <cufft.h>

#include <cmath>
#include <vector>

#include "precond.h"
#include "qg_internal.h"

namespace qg {

namespace {

// per-axis FD symbol of Lap (without the -1/2) for wavenumber index k of n points
double axis_symbol(int order, double h, int k, int n) {
    const double th = 2.0 * M_PI * (double)k / (double)n;
    switch (order) {
        case 2:
            return (2.0 * cos(th) - 2.0) / (h * h);
        case 4: {  // composed 7-point stencil (1, -54, 783, -1460) / (24 h)^2
            const double s = 1.0 / ((24.0 * h) * (24.0 * h));
            return s * (2.0 * cos(3 * th) - 54.0 * 2.0 * cos(2 * th) + 783.0 * 2.0 * cos(th) - 1460.0);
        }
        case 6: {
            const double s = 1.0 / (90.0 * h * h);
            return s * (2.0 * cos(3 * th) - 13.5 * 2.0 * cos(2 * th) + 135.0 * 2.0 * cos(th) - 245.0);
        }
        default: {
            const double s = 1.0 / (5040.0 * h * h);
            return s * (-9.0 * 2.0 * cos(4 * th) + 128.0 * 2.0 * cos(3 * th) - 1008.0 * 2.0 * cos(2 * th) +
                        8064.0 * 2.0 * cos(th) - 14350.0);
        }
    }
}

__global__ void k_apply_symbol(cufftDoubleComplex* __restrict__ F, const double* __restrict__ sym, long long nc,
                               int batch) {
    const long long total = nc * batch;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        const double w = sym[i % nc];
        F[i].x *= w;
        F[i].y *= w;
    }
}

}  // namespace

KineticPrecond::~KineticPrecond() { release(); }

void KineticPrecond::release() {
    if (plan_fwd) cufftDestroy(plan_fwd);
    if (plan_inv) cufftDestroy(plan_inv);
    plan_fwd = plan_inv = 0;
    if (sym) cudaFree(sym);
    if (buf) cudaFree(buf);
    sym = nullptr;
    buf = nullptr;
    batch = 0;
}

int KineticPrecond::setup(qg_hamiltonian h, int nbatch, double shift) {
    if (batch == nbatch && shift == sigma && sym) return QG_OK;
    release();
    const int nx = h->nx, ny = h->ny, nz = h->nz;
    const int nxc = nx / 2 + 1;
    nc = (long long)nz * ny * nxc;
    const long long N = h->N();
    std::vector<double> s(nc);
    for (int kz = 0; kz < nz; ++kz) {
        const double sz = axis_symbol(h->order, h->hz, kz, nz);
        for (int ky = 0; ky < ny; ++ky) {
            const double sy = axis_symbol(h->order, h->hy, ky, ny);
            for (int kx = 0; kx < nxc; ++kx) {
                const double sx = axis_symbol(h->order, h->hx, kx, nx);
                const double kin = -0.5 * (sx + sy + sz);  // >= 0
                s[(size_t)kx + (size_t)nxc * (ky + (size_t)ny * kz)] = 1.0 / ((kin + shift) * (double)N);
            }
        }
    }
    QG_CUDA_TRY(cudaMalloc(&sym, nc * sizeof(double)));
    QG_CUDA_TRY(cudaMemcpy(sym, s.data(), nc * sizeof(double), cudaMemcpyHostToDevice));
    QG_CUDA_TRY(cudaMalloc(&buf, (size_t)nc * nbatch * sizeof(cufftDoubleComplex)));
    int dims[3] = {nz, ny, nx};
    if (cufftPlanMany(&plan_fwd, 3, dims, nullptr, 1, (int)N, nullptr, 1, (int)nc, CUFFT_D2Z, nbatch) !=
            CUFFT_SUCCESS ||
        cufftPlanMany(&plan_inv, 3, dims, nullptr, 1, (int)nc, nullptr, 1, (int)N, CUFFT_Z2D, nbatch) !=
            CUFFT_SUCCESS) {
        release();
        return QG_ERR_LIBRARY;
    }
    batch = nbatch;
    sigma = shift;
    return QG_OK;
}

// R (N x batch, ld N) <- T R, in place.
int KineticPrecond::apply(double* R, cudaStream_t st) {
    if (cufftSetStream(plan_fwd, st) != CUFFT_SUCCESS || cufftSetStream(plan_inv, st) != CUFFT_SUCCESS)
        return QG_ERR_LIBRARY;
    if (cufftExecD2Z(plan_fwd, R, buf) != CUFFT_SUCCESS) return QG_ERR_LIBRARY;
    k_apply_symbol<<<1184, 256, 0, st>>>(buf, sym, nc, batch);
    if (cufftExecZ2D(plan_inv, buf, R) != CUFFT_SUCCESS) return QG_ERR_LIBRARY;
    QG_CUDA_TRY(cudaGetLastError());
    return QG_OK;
}

}  // namespace qg

extern "C" int qg_hamiltonian_precondition_d(qg_hamiltonian h, int ns, double* R, long long ldr, double shift) {
    if (!h || ns <= 0 || !R || ldr != h->N() || !(shift > 0)) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    if (!h->precond) h->precond = new qg::KineticPrecond();
    QG_TRY(h->precond->setup(h, ns, shift));
    return h->precond->apply(R, h->ctx->stream);
}
