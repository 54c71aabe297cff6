// Autotuner of the real-state H|psi> apply.
//
// Times, on the caller's own block of states, the launch shapes the engine can choose
// without changing a single bit of the result: the stencil kernel (one-plane ring,
// two-plane ring, two rows per thread with V in the ring or from global memory; all give
// the same sums in the same order), the
// states per projection block (1-16) and the states per scatter group (4, 8). The split
// of each atom's projector points over blocks is NOT tuned: it changes the summation
// order, and results must not depend on the tuning or on the batch. Each phase is
// timed with CUDA events on the context stream (phase timer of qg_hamiltonian_apply_timed_d:
// projection, stencil + V, scatter), the best of `reps` applies per candidate; the
// phases are independent, so each dimension is swept with the others at the engine's
// choice. The winner is stored in the operator and used by every later apply.
#include <algorithm>
#include <cfloat>
#include <vector>

#include "qg_internal.h"
#include "stencil_common.cuh"

namespace {

template <typename T>
int timed_phases(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx, int reps,
                 float best[3]) {
    best[0] = best[1] = best[2] = FLT_MAX;
    T* coef = nullptr;
    if (h->pj.na > 0) {
        QG_TRY(h->coef.reserve(qg::coef_scratch_elems(h, ns) * sizeof(T)));
        coef = h->coef.as<T>();
    }
    for (int r = 0; r < reps + 1; ++r) {  // the first apply warms caches and the instruction path
        qg::PhaseTimer pt;
        QG_TRY(qg::apply_hamiltonian<T>(h, ns, X, ldx, HX, ldhx, coef, h->ctx->stream, &pt));
        float ms[3];
        pt.totals(ms);
        QG_CUDA_TRY(cudaGetLastError());
        if (r == 0) continue;
        for (int p = 0; p < 3; ++p) best[p] = std::min(best[p], ms[p]);
    }
    return QG_OK;
}

template <typename T>
int autotune(qg_hamiltonian h, int ns, const T* X, long long ldx, T* HX, long long ldhx, int* choice,
             float* ms_out) {
    if (!h || ns <= 0 || !X || !HX) return QG_ERR_INVALID;
    const long long N = h->N();
    if (ldx < N || ldhx < N) return QG_ERR_INVALID;
    QG_CUDA_TRY(cudaSetDevice(h->ctx->device));
    const int reps = 3;
    const int keep_v = h->stencil_variant;
    float ms[3];
    // stencil kernel (phase 1)
    int best_v = 0;
    float best_t = FLT_MAX;
    for (int v : {2, 3, 4, 5}) {
        h->stencil_variant = v;
        const int rc = timed_phases<T>(h, ns, X, ldx, HX, ldhx, reps, ms);
        if (rc != QG_OK) {
            h->stencil_variant = keep_v;
            return rc;
        }
        if (ms[1] < best_t) {
            best_t = ms[1];
            best_v = v;
        }
    }
    h->stencil_variant = best_v;
    const bool nonlocal = h->pj.na > 0 && h->pj.nch > 0;
    int best_sb = 0, best_sg = 0;
    if (nonlocal) {
        best_t = FLT_MAX;
        for (int sb : {2, 4, 8, 16}) {  // projection (phase 0)
            h->proj_sb = sb;
            QG_TRY(timed_phases<T>(h, ns, X, ldx, HX, ldhx, reps, ms));
            if (ms[0] < best_t) {
                best_t = ms[0];
                best_sb = sb;
            }
        }
        h->proj_sb = best_sb;
        best_t = FLT_MAX;
        for (int sg : {4, 8}) {  // scatter (phase 2)
            h->scatter_sg = sg;
            QG_TRY(timed_phases<T>(h, ns, X, ldx, HX, ldhx, reps, ms));
            if (ms[2] < best_t) {
                best_t = ms[2];
                best_sg = sg;
            }
        }
        h->scatter_sg = best_sg;
    }
    // the chosen configuration once more, for the reported phase times
    QG_TRY(timed_phases<T>(h, ns, X, ldx, HX, ldhx, reps, ms));
    if (choice) {
        choice[0] = h->stencil_variant;
        choice[1] = h->proj_sb;
        choice[2] = h->scatter_sg;
    }
    if (ms_out) {
        ms_out[0] = nonlocal ? ms[0] : 0.f;
        ms_out[1] = ms[1];
        ms_out[2] = nonlocal ? ms[2] : 0.f;
    }
    return QG_OK;
}

}  // namespace

extern "C" {

int qg_hamiltonian_autotune_d(qg_hamiltonian h, int ns, const double* X, long long ldx, double* HX, long long ldhx,
                              int* choice, float* ms_phases) {
    return autotune<double>(h, ns, X, ldx, HX, ldhx, choice, ms_phases);
}

int qg_hamiltonian_autotune_f(qg_hamiltonian h, int ns, const float* X, long long ldx, float* HX, long long ldhx,
                              int* choice, float* ms_phases) {
    return autotune<float>(h, ns, X, ldx, HX, ldhx, choice, ms_phases);
}

}  // extern "C"
