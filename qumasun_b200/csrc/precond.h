// Kinetic preconditioner (precond.cu).
#pragma once
#include <cufft.h>

#include "qg_internal.h"

namespace qg {

struct KineticPrecond {
    cufftHandle plan_fwd = 0, plan_inv = 0;
    double* sym = nullptr;             // [nz][ny][nx/2+1] 1 / ((-1/2 Lap_FD(k) + sigma) N)
    cufftDoubleComplex* buf = nullptr; // [batch][nc]
    long long nc = 0;
    int batch = 0;
    double sigma = 0.0;
    ~KineticPrecond();
    void release();
    int setup(qg_hamiltonian h, int nbatch, double shift);
    int apply(double* R, cudaStream_t st);  // R (N x batch) <- T R in place
};

}  // namespace qg
