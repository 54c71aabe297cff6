/*
 * ref_harness.cpp -- C entry points around the reference's own CPU code.
 *
 * TEST INFRASTRUCTURE ONLY. This file is compiled by oracle/Makefile against
 * the reference's headers where they lie (QUMASUN source/), into
 * oracle/_ref/libqumasun_ref.so. Only tests/, __graft_entry__.smoke() and the
 * CPU-baseline legs of bench.py load it, as the checker and the timed CPU
 * baseline. Nothing in the product links or calls it.
 *
 * Each entry point drives one reference function unchanged:
 *   ref_laplacian          -> Laplasian{2nd,4th,6th,8th}_halo
 *                             (GridDifference2nd.h:1052, 4th.h:544, 6th.h:440, 8th.h:153)
 *   ref_laplacian_kpoint8  -> LaplasianKpoint8th_halo<KX,KY,KZ> (GridDifferenceKpoint8th.h:124),
 *                             dispatched on |g| < 1e-8 like LaplasianKpoint8th_ddm (:325-368)
 *   ref_hamiltonian_apply  -> mHamiltonianMatrix_ddm order (qumasun_mpi.matrix.h:20-43):
 *                             zero, mPotentialMatrix (V*psi), ProjectionPP
 *                             (PseudoPotOperator.h:740-772), kinetic Laplacian (coef -1/2)
 *   ref_lobpcg_d_multi     -> EigenLOBPCG_d_multi (lobpcg_d_multi.h:23-545)
 *   ref_lobpcg_z_multi     -> LOBPCG::Eigen_z_multi_mpi (lobpcg_z_multi_mpi.h:988-1800), one rank,
 *                             with the reference k-point H as OpeA
 *   ref_grid_for_sphere    -> GridForSphere (GridSubgrid.h:482-492)
 *   ref_ylm_cube           -> SetYlmAround<L,M> (PseudoPotOperator.h:58-71)
 *   ref_hamiltonian_kpoint_apply
 *                          -> mHamiltonianMatrix_ddm of QUMASUN_KPOINT (qumasun_kpoint.matrix.h:25-50):
 *                             zero, V on re and im, PseudoPotIntegrator_kpoint::ProjectionPP
 *                             (PseudoPotOperator_kpoint_v2.h:2581-2700, its Gamma branch included),
 *                             LaplasianKpoint8th (coef -1/2)
 *
 * The projector tables are injected in the reference's own cube form
 * (PP_nonlocal_each_atom: one SubspaceField per projector w_k and per Y_lm),
 * so the reference's ProjectionPP runs on exactly the arrays the GPU receives.
 */
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <cstdint>
#include <vector>
#include <map>
#include <string>
#include <complex>
#include <algorithm>
#include <random>
#include <locale>
#include <type_traits>
#include <unistd.h>
#include <fcntl.h>

#include "GridRange.h"
#include "GridDifference2nd.h"
#include "GridDifference4th.h"
#include "GridDifference6th.h"
#include "GridDifference8th.h"
#include "GridDifferenceKpoint8th.h"
#include "GridDifferenceKpoint2nd.h"
#include "GridDifferenceKpoint6th.h"
#include "w_dsygvx.h"

/* lobpcg_d_multi.h:209 and :284 call lapack_DSYGVX with six arguments while
 * w_dsygvx.h:25 declares five; the fifth (a factor workspace) is unused by
 * the solve. This adapter must be declared before the template is parsed. */
inline int lapack_DSYGVX(double* A, double* B, double* ev, double* evec, double* /*factors*/, int N) {
    return lapack_DSYGVX(A, B, ev, evec, N);
}
#include "lobpcg_d_multi.h"
#include "debug_print.h"
#include "lobpcg_z_multi_mpi.h"
#include "lobpcg_d_multi_mpi.h"

/* PseudoPotIntegrator_single keeps its per-atom tables private; the harness
 * fills them directly instead of going through the .vps radial loader. */
#define private public
#define protected public
#include "PseudoPotOperator.h"
#include "PseudoPotOperator_kpoint_v2.h"
#undef private
#undef protected

/* SCF-step neighbours of the eigensolver: the FFT Poisson solve (poisson_fft.h, FFTW
 * provided by shims/fftw3.h), LDA exchange-correlation (Vxc.h), Fermi occupations
 * (SetOccupancy.h), the 8th-order gradient (GridGradient8th.h) and the Taylor-4
 * propagator (qumasun_td.time_evo_H4.h, which brings in the QUMASUN_TD class). */
#include "poisson_fft.h"
#include "Vxc.h"
#include "SetOccupancy.h"
#include "GridGradient8th.h"
#include "qumasun_td.time_evo_H4.h"

namespace {

struct NullWatch {
    void Record(int) {}
    void Record(int, int) {}
};

double wall_now() {
    timespec t;
    clock_gettime(CLOCK_MONOTONIC, &t);
    return t.tv_sec + 1e-9 * t.tv_nsec;
}

/* The reference's watch protocol: Record(id) closes a section that began at the
 * previous Record. Each section's time goes to its id, less the H applications
 * (OpeA) that ran inside it, which are counted apart. */
struct PhaseWatch {
    double last = wall_now();
    double acc[32] = {};
    double h_total = 0.0, h_since = 0.0;
    void Record(int id) {
        const double t = wall_now();
        if (id >= 0 && id < 32) acc[id] += (t - last) - h_since;
        last = t;
        h_since = 0.0;
    }
    void Record(int id, int) { Record(id); }
    void add_h(double dt) {
        h_total += dt;
        h_since += dt;
    }
};

struct QuietStdout {
    int saved = -1;
    explicit QuietStdout(bool on) {
        if (!on) return;
        fflush(stdout);
        saved = dup(1);
        int devnull = open("/dev/null", O_WRONLY);
        dup2(devnull, 1);
        close(devnull);
    }
    ~QuietStdout() {
        if (saved < 0) return;
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

}  // namespace

extern "C" {

/* Hamiltonian description passed from Python (flat arrays, FP64). */
typedef struct ref_ham_desc {
    int nx, ny, nz;
    double hx, hy, hz;
    int fd_order;            /* 2, 4 (the reference's composed 7-point stencil), 6, 8 */
    const double* V;         /* nx*ny*nz local potential */
    int n_atoms;
    const double* atom_pos;  /* 3*n_atoms */
    int n_proj;              /* projectors per atom */
    const int* proj_l;       /* n_proj */
    const double* proj_E;    /* n_proj */
    const int* cube;         /* n_atoms*n_proj*6: begin xyz, size xyz of projector k's cube */
    const double* w_data;    /* concatenated w cubes */
    const long long* w_off;  /* n_atoms*n_proj offsets into w_data */
    int n_lm;                /* (lmax+1)^2 */
    const double* ylm_data;  /* concatenated Y_lm cubes (cube of the first projector with that l) */
    const long long* ylm_off;/* n_atoms*n_lm offsets */
} ref_ham_desc;

int ref_grid_for_sphere(double Rx, double Ry, double Rz, double rc, double hx, double hy, double hz,
                        int* out6) {
    GridRange g = GridForSphere(Rx, Ry, Rz, rc, hx, hy, hz);
    out6[0] = g.begin_x; out6[1] = g.begin_y; out6[2] = g.begin_z;
    out6[3] = g.end_x;   out6[4] = g.end_y;   out6[5] = g.end_z;
    return 0;
}

int ref_ylm_cube(int l, int m, const int* begin3, const int* size3, const double* R3,
                 const double* h3, double* out) {
#define QG_YLM_CASE(L, M)                                                                   \
    if (l == L && m == M) {                                                                 \
        SetYlmAround<L, M>(out, begin3[0], begin3[1], begin3[2], size3[0], size3[1], size3[2], \
                           R3[0], R3[1], R3[2], h3[0], h3[1], h3[2]);                         \
        return 0;                                                                           \
    }
    QG_YLM_CASE(0, 0)
    QG_YLM_CASE(1, -1) QG_YLM_CASE(1, 0) QG_YLM_CASE(1, 1)
    QG_YLM_CASE(2, -2) QG_YLM_CASE(2, -1) QG_YLM_CASE(2, 0) QG_YLM_CASE(2, 1) QG_YLM_CASE(2, 2)
#undef QG_YLM_CASE
    return -1;
}

/* out += coef * Laplacian(in), periodic, one state. */
int ref_laplacian(int order, int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                  const double* in, double* out) {
    GridRange grid{0, 0, 0, nx, ny, nz};
    int mw = (order == 2) ? 1 : (order == 8) ? 4 : 3;
    std::vector<double> buf((size_t)(nx + 2 * mw) * (ny + 2 * mw) * (nz + 2 * mw));
    switch (order) {
        case 2: Laplasian2nd_halo(grid, out, in, buf.data(), coef, hx, hy, hz); break;
        case 4: Laplasian4th_halo(grid, out, in, buf.data(), coef, hx, hy, hz); break;
        case 6: Laplasian6th_halo(grid, out, in, buf.data(), coef, hx, hy, hz); break;
        case 8: Laplasian8th_halo(grid, out, in, buf.data(), coef, hx, hy, hz); break;
        default: return -1;
    }
    return 0;
}

/* out += -(1/2)(nabla^2 + 2 i g.nabla - g^2) psi on split re/im arrays (coef = -1/2). */
int ref_laplacian_kpoint8(int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                          double gx, double gy, double gz, const double* re, const double* im,
                          double* out_re, double* out_im) {
    GridRange grid{0, 0, 0, nx, ny, nz};
    std::vector<double> bre((size_t)(nx + 8) * (ny + 8) * (nz + 8));
    std::vector<double> bim(bre.size());
    SoAComplex out{out_re, out_im};
    SoAComplex src{const_cast<double*>(re), const_cast<double*>(im)};
    const double th = 1.0e-8;
    const int kx = fabs(gx) >= th, ky = fabs(gy) >= th, kz = fabs(gz) >= th;
    const int sel = kx * 4 + ky * 2 + kz;
#define QG_KP(A, B, C)                                                                        \
    case A * 4 + B * 2 + C:                                                                   \
        LaplasianKpoint8th_halo<A, B, C>(grid, out, src, bre.data(), bim.data(), coef, hx, hy, hz, \
                                         gx, gy, gz);                                         \
        break;
    switch (sel) {
        QG_KP(0, 0, 0) QG_KP(0, 0, 1) QG_KP(0, 1, 0) QG_KP(0, 1, 1)
        QG_KP(1, 0, 0) QG_KP(1, 0, 1) QG_KP(1, 1, 0) QG_KP(1, 1, 1)
    }
#undef QG_KP
    return 0;
}

/* The same for FD order 2 (LaplasianKpoint2nd_halo, GridDifferenceKpoint2nd.h:97-130), 6
 * (LaplasianKpoint6th_halo, GridDifferenceKpoint6th.h:108-142) or 8. */
int ref_laplacian_kpoint(int order, int nx, int ny, int nz, double hx, double hy, double hz, double coef,
                         double gx, double gy, double gz, const double* re, const double* im,
                         double* out_re, double* out_im) {
    if (order == 8) return ref_laplacian_kpoint8(nx, ny, nz, hx, hy, hz, coef, gx, gy, gz, re, im, out_re, out_im);
    if (order != 2 && order != 6) return -1;
    GridRange grid{0, 0, 0, nx, ny, nz};
    std::vector<double> bre((size_t)(nx + 8) * (ny + 8) * (nz + 8));
    std::vector<double> bim(bre.size());
    SoAComplex out{out_re, out_im};
    SoAComplex src{const_cast<double*>(re), const_cast<double*>(im)};
    const double th = 1.0e-8;
    const int kx = fabs(gx) >= th, ky = fabs(gy) >= th, kz = fabs(gz) >= th;
    const int sel = kx * 4 + ky * 2 + kz;
#define QG_KP(A, B, C)                                                                                     \
    case A * 4 + B * 2 + C:                                                                                \
        if (order == 2)                                                                                    \
            LaplasianKpoint2nd_halo<A, B, C>(grid, out, src, bre.data(), bim.data(), coef, hx, hy, hz, gx, gy, gz); \
        else                                                                                               \
            LaplasianKpoint6th_halo<A, B, C>(grid, out, src, bre.data(), bim.data(), coef, hx, hy, hz, gx, gy, gz); \
        break;
    switch (sel) {
        QG_KP(0, 0, 0) QG_KP(0, 0, 1) QG_KP(0, 1, 0) QG_KP(0, 1, 1)
        QG_KP(1, 0, 0) QG_KP(1, 0, 1) QG_KP(1, 1, 0) QG_KP(1, 1, 1)
    }
#undef QG_KP
    return 0;
}

}  // extern "C"

namespace {

/* Owns a PseudoPotIntegrator_single whose tables come from a ref_ham_desc. */
struct RefHamiltonian {
    const ref_ham_desc* d;
    PseudoPotIntegrator_single pp;
    std::vector<Nucleus> nuclei;
    std::vector<double> halo;

    explicit RefHamiltonian(const ref_ham_desc* desc) : d(desc) {
        GridInfo gi;
        gi.size_x = d->nx; gi.size_y = d->ny; gi.size_z = d->nz;
        gi.size_3d = (size_t)d->nx * d->ny * d->nz;
        pp.InitializeGrid(gi, d->hx, d->hy, d->hz);
        const int Z = 6;
        if (d->n_atoms > 0 && d->n_proj > 0) {
            PseudoPot_MBK* mbk = new PseudoPot_MBK();
            mbk->num_projectors = d->n_proj;
            mbk->projector_quantum_l = new int[d->n_proj];
            mbk->projector_energy_up = new double[d->n_proj];
            for (int k = 0; k < d->n_proj; ++k) {
                mbk->projector_quantum_l[k] = d->proj_l[k];
                mbk->projector_energy_up[k] = d->proj_E[k];
            }
            pp.m_pp_list.emplace(Z, mbk);
        }
        pp.m_pp_by_atom.resize(d->n_atoms);
        for (int a = 0; a < d->n_atoms; ++a) {
            nuclei.push_back(Nucleus{Z, d->atom_pos[3 * a], d->atom_pos[3 * a + 1], d->atom_pos[3 * a + 2]});
            PP_nonlocal_each_atom& at = pp.m_pp_by_atom[a];
            for (int k = 0; k < d->n_proj; ++k) {
                const int* c = d->cube + 6 * ((size_t)a * d->n_proj + k);
                at.projector.emplace_back(c[0], c[1], c[2], c[3], c[4], c[5]);
                double* buf = at.projector.back().Reserve();
                std::memcpy(buf, d->w_data + d->w_off[(size_t)a * d->n_proj + k],
                            sizeof(double) * at.projector.back().num_total_grid);
            }
            for (int lm = 0; lm < d->n_lm; ++lm) {
                int l = (int)std::floor(std::sqrt((double)lm) + 1e-9);
                int kfirst = -1;
                for (int k = 0; k < d->n_proj; ++k) if (d->proj_l[k] == l) { kfirst = k; break; }
                const int* c = d->cube + 6 * ((size_t)a * d->n_proj + (kfirst < 0 ? 0 : kfirst));
                at.Ylm.emplace_back(c[0], c[1], c[2], c[3], c[4], c[5]);
                double* buf = at.Ylm.back().Reserve();
                std::memcpy(buf, d->ylm_data + d->ylm_off[(size_t)a * d->n_lm + lm],
                            sizeof(double) * at.Ylm.back().num_total_grid);
            }
        }
        int mw = (d->fd_order == 2) ? 1 : (d->fd_order == 8) ? 4 : 3;
        halo.resize((size_t)(d->nx + 2 * mw) * (d->ny + 2 * mw) * (d->nz + 2 * mw));
    }

    ~RefHamiltonian() {
        for (auto& at : pp.m_pp_by_atom) {
            for (auto& f : at.projector) f.Release();
            for (auto& f : at.Ylm) f.Release();
        }
    }

    /* One state, in the order of mHamiltonianMatrix_ddm (qumasun_mpi.matrix.h:20-43). */
    void Apply(double* Hp, const double* phi) {
        const size_t N = (size_t)d->nx * d->ny * d->nz;
        vecmath::SetZero<double>(Hp, N);
        for (size_t i = 0; i < N; ++i) Hp[i] = d->V[i] * phi[i];
        if (d->n_atoms > 0 && d->n_proj > 0) {
            RspaceFunc<double> hp(Hp);
            RspaceFunc<double> ps(const_cast<double*>(phi));
            pp.ProjectionPP(hp, ps, nuclei.data(), (int)nuclei.size());
        }
        GridRange grid{0, 0, 0, d->nx, d->ny, d->nz};
        switch (d->fd_order) {
            case 2: Laplasian2nd_halo(grid, Hp, phi, halo.data(), -0.5, d->hx, d->hy, d->hz); break;
            case 4: Laplasian4th_halo(grid, Hp, phi, halo.data(), -0.5, d->hx, d->hy, d->hz); break;
            case 6: Laplasian6th_halo(grid, Hp, phi, halo.data(), -0.5, d->hx, d->hy, d->hz); break;
            default: Laplasian8th_halo(grid, Hp, phi, halo.data(), -0.5, d->hx, d->hy, d->hz); break;
        }
    }
};

}  // namespace

extern "C" {

/* HX[s] = H X[s] for ns states, state-major (X[s*N + i]). */
int ref_hamiltonian_apply(const ref_ham_desc* d, int ns, const double* X, double* HX) {
    if (d->fd_order != 2 && d->fd_order != 4 && d->fd_order != 6 && d->fd_order != 8) return -1;
    RefHamiltonian H(d);
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    for (int s = 0; s < ns; ++s) H.Apply(HX + (size_t)s * N, X + (size_t)s * N);
    return 0;
}

/* The reference's serial block LOBPCG, run unchanged with the reference H as OpeA.
 * X (ns*N) in/out, P (ns*N) in/out (the "keep" block), ev (ns) out.
 * *iters receives the number of LOBPCG iterations taken (counted from OpeA calls). */
int ref_lobpcg_d_multi(const ref_ham_desc* d, int ns, int iter_max, double* ev, double* X,
                       double* P, int is_first_time, int quiet, int* iters) {
    RefHamiltonian H(d);
    const int N = d->nx * d->ny * d->nz;
    const double dV = d->hx * d->hy * d->hz;
    std::vector<double> work(WorkSizeLOBPCG_d_multi(N, ns));
    long long calls = 0;
    auto OpeA = [&](double* Ax, double* x) { ++calls; H.Apply(Ax, x); };
    NullWatch watch;
    {
        QuietStdout q(quiet != 0);
        EigenLOBPCG_d_multi(N, dV, ns, iter_max, ev, X, P, work.data(), is_first_time != 0, OpeA, watch);
    }
    if (iters) *iters = (int)((calls - 2LL * ns) / ns);
    return 0;
}

}  // extern "C"

namespace {

/* Owns a PseudoPotIntegrator_kpoint set up by the reference's own routines:
 * per-l blocks from GridForSphere + GetOverlapPeriodic (the two calls of
 * UpdatePositionLocal, PseudoPotOperator_vlocal.h:155-165), projector counts
 * (CountNonlocalProjector, mSetNonlocalProjectorInfo), Y_lm on the blocks
 * (tCreateProjectorYlmOnBlock) and the Bloch phases (UpdateNonlocalBlock ->
 * mCreateProjectorRadialOnBlock[_gamma], PseudoPotOperator_kpoint_v2.h:287-420).
 * The radial table handed to the reference is the constant 1 (every point lies
 * inside radius[0], so the reference takes p = projector[2k][0] = 1 without
 * interpolation); the harness then multiplies each block value by the
 * analytic w_k of the matching cube point, so projector_expikx ends up as
 * w_k(r) * exp(i g.r) with the reference's own phases and block layout. */
struct RefKpointHamiltonian {
    const ref_ham_desc* d;
    double g[3];
    PseudoPotIntegrator_kpoint pp;
    std::vector<Nucleus> nuclei;
    GridRangeMPI grid;
    int status = 0;

    RefKpointHamiltonian(const ref_ham_desc* desc, double gx, double gy, double gz, double rc) : d(desc) {
        g[0] = gx; g[1] = gy; g[2] = gz;
        std::memset(static_cast<void*>(&grid), 0, sizeof(grid));
        grid.begin_x = 0; grid.begin_y = 0; grid.begin_z = 0;
        grid.end_x = d->nx; grid.end_y = d->ny; grid.end_z = d->nz;
        grid.mpi_comm = MPI_COMM_WORLD;
        GridInfo gi;
        gi.size_x = d->nx; gi.size_y = d->ny; gi.size_z = d->nz;
        gi.size_3d = (size_t)d->nx * d->ny * d->nz;
        pp.InitializeGrid(gi, d->hx, d->hy, d->hz);
        const int Z = 6;
        for (int a = 0; a < d->n_atoms; ++a)
            nuclei.push_back(Nucleus{Z, d->atom_pos[3 * a], d->atom_pos[3 * a + 1], d->atom_pos[3 * a + 2]});
        if (d->n_atoms <= 0 || d->n_proj <= 0) return;
        const int np = d->n_proj;
        PseudoPot_MBK* mbk = new PseudoPot_MBK();
        mbk->num_projectors = np;
        mbk->projector_quantum_l = new int[np];
        mbk->projector_energy_up = new double[np];
        for (int k = 0; k < np; ++k) {
            mbk->projector_quantum_l[k] = d->proj_l[k];
            mbk->projector_energy_up[k] = d->proj_E[k];
        }
        mbk->num_radial_grids = 2;
        mbk->buffer_all = new double[2 + 4 * np];
        mbk->radius = mbk->buffer_all;
        mbk->radius[0] = 1.0e6;
        mbk->radius[1] = 2.0e6;
        for (int j = 0; j < 2 * np; ++j) {
            double* pr = mbk->buffer_all + 2 + 2 * j;
            pr[0] = 1.0;
            pr[1] = 1.0;
            mbk->projector.push_back(pr);
        }
        mbk->xi_min = 0.0;
        mbk->xi_delta = 1.0;
        for (int l = 0; l < 4; ++l) mbk->cutoff_r[l] = rc;
        pp.m_pp_list.emplace(Z, mbk);

        const int max_l = mbk->MaxProjectorL();
        pp.m_nonlocal_blocks.resize(d->n_atoms);
        size_t max_grid = 0;
        for (int a = 0; a < d->n_atoms; ++a) {
            auto& blocks = pp.m_nonlocal_blocks[a];
            blocks.resize(max_l + 1);
            for (int l = 0; l <= max_l; ++l) {
                blocks[l].cutoff = rc;
                GridRange sub = GridForSphere(nuclei[a].Rx, nuclei[a].Ry, nuclei[a].Rz, rc, d->hx, d->hy, d->hz);
                /* the injected w cubes must sit on exactly this subgrid */
                for (int k = 0; k < np; ++k) {
                    if (d->proj_l[k] != l) continue;
                    const int* c = d->cube + 6 * ((size_t)a * np + k);
                    if (c[0] != sub.begin_x || c[1] != sub.begin_y || c[2] != sub.begin_z ||
                        c[3] != sub.end_x - sub.begin_x || c[4] != sub.end_y - sub.begin_y ||
                        c[5] != sub.end_z - sub.begin_z)
                        status = -2;
                }
                blocks[l].grid_sizes = GetOverlapPeriodic(grid, sub, d->nx, d->ny, d->nz, blocks[l].range_blocks,
                                                          blocks[l].shifted_grids);
                max_grid = std::max(max_grid, (size_t)blocks[l].grid_sizes);
            }
        }
        if (status) return;
        pp.m_max_grid_size = max_grid;
        pp.CountNonlocalProjector(nuclei.data(), d->n_atoms);
        pp.m_nonlocal_projectors.clear();
        pp.m_nonlocal_projectors.resize(d->n_atoms);
        for (int a = 0; a < d->n_atoms; ++a) {
            pp.mSetNonlocalProjectorInfo(pp.m_nonlocal_projectors[a], nuclei[a]);
            tCreateProjectorYlmOnBlock(pp.m_nonlocal_blocks[a], pp.m_nonlocal_projectors[a], nuclei[a], d->hx, d->hy,
                                       d->hz, grid);
        }
        pp.m_comm4atoms.comm_4_nuclei.assign(d->n_atoms, MPI_COMM_WORLD);
        pp.m_request4atoms.resize(d->n_atoms);
        pp.m_status4atoms.resize(d->n_atoms);
        pp.UpdateNonlocalBlock(nuclei.data(), d->n_atoms, grid, 0, gx * d->hx, gy * d->hy, gz * d->hz);
        /* w_k onto the blocks (same point order as mCreateProjectorRadialOnBlock) */
        for (int a = 0; a < d->n_atoms; ++a) {
            auto& proj = pp.m_nonlocal_projectors[a];
            for (int k = 0; k < np; ++k) {
                const int l = d->proj_l[k];
                const auto& blk = pp.m_nonlocal_blocks[a][l];
                const int* c = d->cube + 6 * ((size_t)a * np + k);
                const double* w = d->w_data + d->w_off[(size_t)a * np + k];
                SoAComplex& pb = proj.projector_expikx[0][k];
                int off = 0;
                for (size_t ib = 0; ib < blk.range_blocks.size(); ++ib) {
                    const GridRange& r = blk.range_blocks[ib];
                    const auto& sh = blk.shifted_grids[ib];
                    const int sx = r.end_x - r.begin_x, sy = r.end_y - r.begin_y;
                    for (int iz = r.begin_z; iz < r.end_z; ++iz)
                        for (int iy = r.begin_y; iy < r.end_y; ++iy)
                            for (int ix = r.begin_x; ix < r.end_x; ++ix) {
                                const int i = off + (ix - r.begin_x) + sx * ((iy - r.begin_y) + sy * (iz - r.begin_z));
                                const int qx = ix - sh.x - c[0], qy = iy - sh.y - c[1], qz = iz - sh.z - c[2];
                                const double wv = w[qx + (size_t)c[3] * (qy + (size_t)c[4] * qz)];
                                pb.re[i] *= wv;
                                if (pb.im) pb.im[i] *= wv;
                            }
                    off += r.Size3D();
                }
            }
        }
#ifdef EXPAND_PROJECTOR_YLM_Z
        /* UpdateNonlocalBlock also expanded projector * Y_lm into projector_RY_expikx (the
         * table the force inner products read, mInnerNonlocalPsi_b3*) while the radial part
         * was still 1: expand again now that projector_expikx carries w_k. */
        for (int a = 0; a < d->n_atoms; ++a) {
            auto& proj = pp.m_nonlocal_projectors[a];
            for (auto* b : proj.projector_RY_expikx) delete[] b;
            proj.projector_RY_expikx.clear();
            pp.mExpandProjectorYlm(pp.m_nonlocal_blocks[a], proj, 0);
        }
#endif
    }

    /* One {re, im} state, in the order of mHamiltonianMatrix_ddm (qumasun_kpoint.matrix.h:25-50). */
    void Apply(double* ore, double* oim, const double* re, const double* im) {
        const size_t N = (size_t)d->nx * d->ny * d->nz;
        for (size_t i = 0; i < N; ++i) { ore[i] = 0.0; oim[i] = 0.0; }
        for (size_t i = 0; i < N; ++i) ore[i] = d->V[i] * re[i];
        for (size_t i = 0; i < N; ++i) oim[i] = d->V[i] * im[i];
        if (d->n_atoms > 0 && d->n_proj > 0) {
            SoAComplex hp{ore, oim};
            SoAComplex ps{const_cast<double*>(re), const_cast<double*>(im)};
            pp.ProjectionPP(hp, ps, grid, nuclei.data(), d->n_atoms, 0);
        }
        ref_laplacian_kpoint(d->fd_order, d->nx, d->ny, d->nz, d->hx, d->hy, d->hz, -0.5, g[0], g[1], g[2], re, im,
                             ore, oim);
    }
};

}  // namespace

extern "C" {

/* HX[s] = H_k X[s] for ns complex states, each {re[N], im[N]} contiguous (X[s*2N + i],
 * X[s*2N + N + i]); g = Bloch vector (bohr^-1); rc = projector cutoff radius that made
 * the cubes in d. Returns -2 if a cube differs from GridForSphere(R, rc). */
int ref_hamiltonian_kpoint_apply(const ref_ham_desc* d, double gx, double gy, double gz, double rc, int ns,
                                 const double* X, double* HX) {
    if (d->fd_order != 2 && d->fd_order != 6 && d->fd_order != 8) return -1;
    RefKpointHamiltonian H(d, gx, gy, gz, rc);
    if (H.status) return H.status;
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    for (int s = 0; s < ns; ++s)
        H.Apply(HX + (size_t)s * 2 * N, HX + (size_t)s * 2 * N + N, X + (size_t)s * 2 * N, X + (size_t)s * 2 * N + N);
    return 0;
}

}  // extern "C"

extern "C" {

/* The reference's distributed real LOBPCG (LOBPCG::Eigen_d_multi_mpi,
 * lobpcg_d_multi_mpi.h:882-1572) on one rank with the reference H as OpeA (one state
 * per call, no OPERATION_BUNDLE), SCF_step 0 (P starts from zero), no kept S matrix,
 * DGEMMs on `threads` OpenBLAS threads, iter_max iterations. X (ns*N) in/out, ev (ns)
 * out. phase_s[7] receives seconds: [0] H (every OpeA call), [1] Gram (the GEMM1
 * section, watch id 17, without its H calls), [2] rotation (GEMM2, id 16), [3] n x n
 * GEMMs (GEMM3, id 19), [4] small eigensolve (LAPACK, id 15), [5] the rest (ids 10, 14),
 * [6] the whole call; iter_s[iter_max] (may be null) the seconds of each iteration, from
 * its first H application to the next one's. *iters receives the iterations taken
 * (from OpeA calls). */
int ref_lobpcg_d_mpi(const ref_ham_desc* d, int ns, int iter_max, int threads, double* ev, double* X, int quiet,
                     double* phase_s, double* iter_s, int* iters) {
    RefHamiltonian H(d);
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    const double dV = d->hx * d->hy * d->hz;
    GridRangeMPI grid;
    std::memset(static_cast<void*>(&grid), 0, sizeof(grid));
    grid.end_x = d->nx; grid.end_y = d->ny; grid.end_z = d->nz;
    grid.mpi_comm = MPI_COMM_WORLD;
    if (threads > 0) scipy_openblas_set_num_threads(threads);
    std::vector<double> keep((size_t)ns * N, 0.0);
    std::vector<double> work((size_t)5 * ns * N, 0.0);
    long long calls = 0;
    PhaseWatch watch;
    std::vector<double> batch_start;  // wall time of the first OpeA call of every ns-state batch
    auto OpeA = [&](double* Ax, double* x) {
        ++calls;
        const double t0 = wall_now();
        if ((calls - 1) % ns == 0) batch_start.push_back(t0);
        H.Apply(Ax, x);
        watch.add_h(wall_now() - t0);
    };
    const double t0 = wall_now();
    {
        QuietStdout q(quiet != 0);
        LOBPCG::Eigen_d_multi_mpi(grid, dV, ns, iter_max, ev, X, keep.data(), work.data(), (double*)nullptr, 0,
                                  OpeA, watch);
    }
    const double t_end = wall_now();
    if (iter_s) {
        // batches 0 and 1 are the initial A x and A p; iteration i starts with batch 2 + i
        for (int i = 0; i < iter_max; ++i) {
            const size_t b = 2 + (size_t)i;
            iter_s[i] = b < batch_start.size()
                            ? (b + 1 < batch_start.size() ? batch_start[b + 1] : t_end) - batch_start[b]
                            : 0.0;
        }
    }
    if (phase_s) {
        phase_s[0] = watch.h_total;
        phase_s[1] = watch.acc[17];
        phase_s[2] = watch.acc[16];
        phase_s[3] = watch.acc[19];
        phase_s[4] = watch.acc[15];
        phase_s[5] = watch.acc[10] + watch.acc[14];
        phase_s[6] = t_end - t0;
    }
    if (iters) *iters = (int)((calls - 2LL * ns) / ns);
    return 0;
}

/* The reference's complex block LOBPCG (Eigen_z_multi_mpi) on one rank with the
 * reference k-point Hamiltonian as OpeA, SCF_step 0 (P starts from zero), run
 * until its residual escape (max |r|^2 < LIMIT_Z_NORM_R_FOR_ESCAPE) or iter_max.
 * X (ns * 2N, {re, im} per state) in/out, ev (ns) out; *iters receives the
 * iterations taken (counted from OpeA calls). */
int ref_lobpcg_z_multi(const ref_ham_desc* d, double gx, double gy, double gz, double rc, int ns, int iter_max,
                       double* ev, double* X, int quiet, int* iters) {
    if (d->fd_order != 8) return -1;
    RefKpointHamiltonian H(d, gx, gy, gz, rc);
    if (H.status) return H.status;
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    const double dV = d->hx * d->hy * d->hz;
    std::vector<SoAComplex> evec(ns);
    for (int s = 0; s < ns; ++s) {
        evec[s].re = X + (size_t)s * 2 * N;
        evec[s].im = X + (size_t)s * 2 * N + N;
    }
    std::vector<double> keep((size_t)ns * 2 * N, 0.0);
    std::vector<double> work((size_t)5 * ns * 2 * N, 0.0);
    long long calls = 0;
    auto OpeA = [&](SoAComplex& Ax, const SoAComplex& x) {
        ++calls;
        H.Apply(Ax.re, Ax.im, x.re, x.im);
    };
    NullWatch watch;
    {
        QuietStdout q(quiet != 0);
        LOBPCG::Eigen_z_multi_mpi(H.grid, dV, ns, iter_max, ev, evec.data(), keep.data(), work.data(),
                                  (OneComplex*)nullptr, 0, 0, OpeA, watch);
    }
    if (iters) *iters = (int)((calls - 2LL * ns) / ns);
    return 0;
}

}  // extern "C"

extern "C" {

/* V_tot = V_ext + V_hart + V_x + V_c as QUMASUN_SINGLE::mSetPotential forms it for
 * KohnSham_PP without spin (qumasun_single.potential.h:33-43): V_hart by
 * SetPotentialByPoissonFFT (poisson_fft.h:14-128, the free-function form of
 * mSetPotentialVhart, :101-200), V_x and V_c by Calc_XC_LDA(rho + pcc) per point
 * (mSetPotentialVxc, :311-317; Vxc.h:41-70). pcc may be NULL (zero). */
int ref_potential_lda(int nx, int ny, int nz, double hx, double hy, double hz, const double* rho, const double* pcc,
                      const double* vext, double* vtot, double* vhart, double* vx, double* vc) {
    const size_t N = (size_t)nx * ny * nz;
    std::vector<double> work(N * 4);
    SetPotentialByPoissonFFT(vhart, rho, nx, ny, nz, hx, hy, hz, work.data());
    for (size_t i = 0; i < N; ++i) {
        const Return_XC r = Calc_XC_LDA(rho[i] + (pcc ? pcc[i] : 0.0));
        vx[i] = r.V_x;
        vc[i] = r.V_c;
    }
    for (size_t i = 0; i < N; ++i) vtot[i] = vext[i] + vhart[i] + vx[i] + vc[i];
    return 0;
}

/* Fermi occupations at a given chemical potential (SetOccupancy.h:7-18); returns the sum. */
double ref_set_occupancy(double coef, double kbT, int n, const double* ev, double mu, double* occ) {
    return SetOccupancy(coef, kbT, n, ev, mu, occ);
}

/* out_{x,y,z} = coef * grad psi, 8th order, periodic (Gradient8th, GridGradient8th.h:219-235). */
int ref_gradient8(int nx, int ny, int nz, double hx, double hy, double hz, double coef, const double* psi,
                  double* gx_out, double* gy_out, double* gz_out) {
    GridRange grid{0, 0, 0, nx, ny, nz};
    Gradient8th(grid, gx_out, gy_out, gz_out, psi, coef, hx, hy, hz);
    return 0;
}

/* One Taylor-4 step of ns complex states ({re, im} per state, X[s*2N ..]) with the
 * reference k-point H at Bloch vector g: QUMASUN::TimeEvoH4 (qumasun_td.time_evo_H4.h:13-60)
 * run unchanged on one rank. */
int ref_td_taylor4(const ref_ham_desc* d, double gx, double gy, double gz, double rc, double dt, int ns,
                   double* X) {
    if (d->fd_order != 8) return -1;
    RefKpointHamiltonian H(d, gx, gy, gz, rc);
    if (H.status) return H.status;
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    const double dV = d->hx * d->hy * d->hz;
    std::vector<SoAComplex> xs(ns);
    for (int s = 0; s < ns; ++s) {
        xs[s].re = X + (size_t)s * 2 * N;
        xs[s].im = X + (size_t)s * 2 * N + N;
    }
    auto OpeA = [&](SoAComplex& Ax, const SoAComplex& x) { H.Apply(Ax.re, Ax.im, x.re, x.im); };
    NullWatch watch;
    QUMASUN::TimeEvoH4(H.grid, dV, dt, ns, xs.data(), OpeA, watch);
    return 0;
}

/* Nonlocal energy and forces of ns complex states at Bloch vector g, as
 * QUMASUN_KPOINT::mGetForcePseudoNonlocal forms them (qumasun_kpoint.force.h:238-258):
 * for each state with occ > 0, dpsi = -2 occ grad psi (Gradient8th on re and im) and
 * PseudoPotIntegrator_kpoint::ForceNonlocal (PseudoPotOperator_kpoint_v2.h:2760-2866)
 * with g scaled by -2 occ. forces (3 per atom) accumulate; e_state[s] receives the
 * state's nonlocal energy (0 for occ <= 0); *ev_sum = sum_s occ_s e_state[s].
 * At g = 0 with zero imaginary parts this is the Gamma-point real-state force of
 * QUMASUN_MPI::mGetForcePseudoNonlocal (qumasun_mpi.force.h:227-254). */
int ref_nonlocal_force_z(const ref_ham_desc* d, double gx, double gy, double gz, double rc, int ns,
                         const double* X, const double* occ, double* forces, double* e_state, double* ev_sum) {
    if (d->fd_order != 8) return -1;
    RefKpointHamiltonian H(d, gx, gy, gz, rc);
    if (H.status) return H.status;
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    std::vector<double> buf(6 * N);
    SoAComplex dx{buf.data(), buf.data() + N}, dy{buf.data() + 2 * N, buf.data() + 3 * N},
        dz{buf.data() + 4 * N, buf.data() + 5 * N};
    GridRange grid{0, 0, 0, d->nx, d->ny, d->nz};
    double ev = 0.0;
    for (int s = 0; s < ns; ++s) {
        e_state[s] = 0.0;
        if (occ[s] <= 0.0) continue;
        const double coef = -2.0 * occ[s];
        SoAComplex psi{const_cast<double*>(X + (size_t)s * 2 * N), const_cast<double*>(X + (size_t)s * 2 * N + N)};
        Gradient8th(grid, dx.re, dy.re, dz.re, psi.re, coef, d->hx, d->hy, d->hz);
        Gradient8th(grid, dx.im, dy.im, dz.im, psi.im, coef, d->hx, d->hy, d->hz);
        const double e = H.pp.ForceNonlocal(forces, psi, dx, dy, dz, H.grid, H.nuclei.data(), d->n_atoms, 0,
                                            gx * coef, gy * coef, gz * coef);
        e_state[s] = e;
        ev += e * occ[s];
    }
    if (ev_sum) *ev_sum = ev;
    return 0;
}

/* Nonlocal energy of each real state (PseudoPotIntegrator_single::EnergyPPnonlocal,
 * PseudoPotOperator.h:775-816), X state-major (ns * N). */
int ref_nonlocal_energy_d(const ref_ham_desc* d, int ns, const double* X, double* e_state) {
    RefHamiltonian H(d);
    const size_t N = (size_t)d->nx * d->ny * d->nz;
    for (int s = 0; s < ns; ++s) {
        RspaceFunc<double> psi(const_cast<double*>(X + (size_t)s * N));
        e_state[s] = H.pp.EnergyPPnonlocal(psi, H.nuclei.data(), d->n_atoms);
    }
    return 0;
}

}  // extern "C"
