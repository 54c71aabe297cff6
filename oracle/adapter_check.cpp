/*
 * Checks of the header-only C++ adapter (include/qumasun_b200_adapter.hpp) against
 * the reference's own code -- TEST INFRASTRUCTURE ONLY, built by oracle/Makefile into
 * oracle/_ref/libadapter_check.so where the reference tree exists, linked against the
 * engine library.
 *
 * The reference integrator here is set up the way QUMASUN sets it up: a PseudoPot_MBK
 * whose radial tables sample w_l(r) = r^l exp(-r^2 / (2 sigma^2)) on a logarithmic
 * grid, then PseudoPotIntegrator_single::UpdatePosition (PseudoPotOperator.h:453-466)
 * tabulates the per-atom cubes (mMakeSubspacePPnonlocal_Radial / _Ylm). The adapter
 * flattens exactly those cubes into the engine's descriptor; the reference applies H
 * with the same integrator (V psi, ProjectionPP, Laplasian8th), and the serial solver
 * EigenLOBPCG_d_multi runs both with the reference's lambda and, unchanged, with the
 * adapter's GpuOperator in its place.
 *
 * PseudoPotIntegrator_single keeps m_pp_by_atom private; this checker opens it by
 * compiling the header with private/protected mapped to public. An integration into
 * QUMASUN adds a const accessor instead (INTEGRATION.md shows it).
 */
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <unistd.h>
#include <fcntl.h>

#include "GridRange.h"
#include "GridDifference2nd.h"
#include "GridDifference4th.h"
#include "GridDifference6th.h"
#include "GridDifference8th.h"
#include "w_dsygvx.h"
inline int lapack_DSYGVX(double* A, double* B, double* ev, double* evec, double* /*factors*/, int N) {
    return lapack_DSYGVX(A, B, ev, evec, N);
}
#include "lobpcg_d_multi.h"

#define private public
#define protected public
#include "PseudoPotOperator.h"
#undef private
#undef protected

#include "qumasun_b200_adapter.hpp"

namespace {

struct NullWatch {
    void Record(int) {}
    void Record(int, int) {}
};

struct Quiet {
    int saved = -1;
    Quiet() {
        fflush(stdout);
        saved = dup(1);
        int dn = open("/dev/null", O_WRONLY);
        dup2(dn, 1);
        close(dn);
    }
    ~Quiet() {
        fflush(stdout);
        dup2(saved, 1);
        close(saved);
    }
};

/* A reference integrator for n_atoms carbon-like atoms with projectors l = proj_l[k],
 * energies proj_E[k], radial w_l(r) = r^l exp(-r^2/(2 sigma^2)) up to cutoff rc. */
struct RefSetup {
    int nx, ny, nz;
    double hx, hy, hz;
    PseudoPotIntegrator_single pp;
    std::vector<Nucleus> nuclei;
    std::vector<int> proj_l;
    std::vector<double> proj_E;
    std::vector<double> halo;

    RefSetup(int nx_, int ny_, int nz_, double hx_, double hy_, double hz_, int na, const double* pos, int np,
             const int* pl, const double* pe, double rc, double sigma)
        : nx(nx_), ny(ny_), nz(nz_), hx(hx_), hy(hy_), hz(hz_), proj_l(pl, pl + np), proj_E(pe, pe + np) {
        GridInfo gi;
        gi.size_x = nx; gi.size_y = ny; gi.size_z = nz;
        gi.size_3d = (size_t)nx * ny * nz;
        pp.InitializeGrid(gi, hx, hy, hz);
        const int Z = 6;
        PseudoPot_MBK* mbk = new PseudoPot_MBK();
        mbk->num_projectors = np;
        mbk->projector_quantum_l = new int[np];
        mbk->projector_energy_up = new double[np];
        for (int k = 0; k < np; ++k) {
            mbk->projector_quantum_l[k] = pl[k];
            mbk->projector_energy_up[k] = pe[k];
        }
        const int nr = 600;
        const double r0 = 1.0e-4, r1 = 2.0 * rc;
        mbk->num_radial_grids = nr;
        mbk->xi_min = std::log(r0);
        mbk->xi_delta = (std::log(r1) - std::log(r0)) / (nr - 1);
        mbk->buffer_all = new double[(size_t)nr * (1 + 2 * np)];
        mbk->radius = mbk->buffer_all;
        for (int i = 0; i < nr; ++i) mbk->radius[i] = std::exp(mbk->xi_min + i * mbk->xi_delta);
        for (int j = 0; j < 2 * np; ++j) {
            double* w = mbk->buffer_all + (size_t)nr * (1 + j);
            const int l = pl[j / 2];
            for (int i = 0; i < nr; ++i) {
                const double r = mbk->radius[i];
                w[i] = std::pow(r, l) * std::exp(-r * r / (2.0 * sigma * sigma));
            }
            mbk->projector.push_back(w);
        }
        for (int l = 0; l < 4; ++l) mbk->cutoff_r[l] = rc;
        pp.m_pp_list.emplace(Z, mbk);
        for (int a = 0; a < na; ++a) nuclei.push_back(Nucleus{Z, pos[3 * a], pos[3 * a + 1], pos[3 * a + 2]});
        {
            Quiet q;
            pp.UpdatePosition(nuclei.data(), na);
        }
        halo.resize((size_t)(nx + 8) * (ny + 8) * (nz + 8));
    }

    qumasun_b200::HamiltonianTables tables(const double* V) const {
        return qumasun_b200::flatten_projectors(nx, ny, nz, hx, hy, hz, 8, V, pp.m_pp_by_atom, nuclei.data(),
                                                proj_l, proj_E);
    }

    /* H psi for one state in the order of mHamiltonianMatrix_ddm (qumasun_mpi.matrix.h:20-43). */
    void apply(const double* V, double* Hp, const double* phi) {
        const size_t N = (size_t)nx * ny * nz;
        for (size_t i = 0; i < N; ++i) Hp[i] = V[i] * phi[i];
        RspaceFunc<double> hp(Hp);
        RspaceFunc<double> ps(const_cast<double*>(phi));
        pp.ProjectionPP(hp, ps, nuclei.data(), (int)nuclei.size());
        GridRange grid{0, 0, 0, nx, ny, nz};
        Laplasian8th_halo(grid, Hp, phi, halo.data(), -0.5, hx, hy, hz);
    }
};

}  // namespace

extern "C" {

/* Flattens a reference integrator's tables (no GPU): returns the number of atoms,
 * projector cubes and Y_lm cubes read, and the table sums, so a test can check the
 * flattened descriptor against the reference's own cubes. */
int adapter_flatten_stats(int nx, int ny, int nz, double hx, double hy, double hz, int na, const double* pos,
                          int np, const int* pl, const double* pe, double rc, double sigma, const double* V,
                          int* cube_out, double* sums_out) {
    RefSetup r(nx, ny, nz, hx, hy, hz, na, pos, np, pl, pe, rc, sigma);
    const qumasun_b200::HamiltonianTables t = r.tables(V);
    std::memcpy(cube_out, t.cube.data(), t.cube.size() * sizeof(int));
    double sw = 0.0, sy = 0.0, direct_w = 0.0, direct_y = 0.0;
    for (double v : t.w_data) sw += v;
    for (double v : t.ylm_data) sy += v;
    for (const auto& at : r.pp.m_pp_by_atom) {
        for (const auto& f : at.projector)
            for (size_t i = 0; i < f.num_total_grid; ++i) direct_w += f.GetGridPointer()[i];
        for (const auto& f : at.Ylm)
            for (size_t i = 0; i < f.num_total_grid; ++i) direct_y += f.GetGridPointer()[i];
    }
    sums_out[0] = sw;
    sums_out[1] = direct_w;
    sums_out[2] = sy;
    sums_out[3] = direct_y;
    return t.n_atoms * 1000000 + t.n_proj * 1000 + t.n_lm;
}

/* GPU: H X through the adapter (flattened reference tables -> qumasun_b200::Operator)
 * and through the reference integrator; HX_gpu, HX_ref (ns * N) out. */
int adapter_apply_check(int nx, int ny, int nz, double hx, double hy, double hz, int na, const double* pos, int np,
                        const int* pl, const double* pe, double rc, double sigma, const double* V, int ns,
                        const double* X, double* HX_gpu, double* HX_ref) {
    try {
        RefSetup r(nx, ny, nz, hx, hy, hz, na, pos, np, pl, pe, rc, sigma);
        const qumasun_b200::HamiltonianTables t = r.tables(V);
        qumasun_b200::Context ctx(0);
        qumasun_b200::Operator op(ctx, t);
        op.apply(ns, X, HX_gpu);
        const size_t N = (size_t)nx * ny * nz;
        for (int s = 0; s < ns; ++s) r.apply(V, HX_ref + s * N, X + s * N);
    } catch (const std::exception& e) {
        fprintf(stderr, "adapter_apply_check: %s\n", e.what());
        return -1;
    }
    return 0;
}

/* GPU: the reference's call site, EigenLOBPCG_d_multi(N, dVol, ns, iter_max, ev, X, P,
 * work, true, OpeA, watch), once with the reference's lambda and once, unchanged, with
 * the adapter's GpuOperator. ev_ref / ev_gpu (ns) out; iters_ref receives the reference's
 * iteration count (from its OpeA calls). */
int adapter_lobpcg_check(int nx, int ny, int nz, double hx, double hy, double hz, int na, const double* pos, int np,
                         const int* pl, const double* pe, double rc, double sigma, const double* V, int ns,
                         int iter_max, const double* X0, double* ev_ref, double* ev_gpu, int* iters_ref) {
    try {
        RefSetup r(nx, ny, nz, hx, hy, hz, na, pos, np, pl, pe, rc, sigma);
        const int N = nx * ny * nz;
        const double dV = hx * hy * hz;
        std::vector<double> X(X0, X0 + (size_t)ns * N), P((size_t)ns * N, 0.0);
        std::vector<double> work(WorkSizeLOBPCG_d_multi(N, ns));
        long long calls = 0;
        auto OpeA = [&](double* Ax, double* x) {
            ++calls;
            r.apply(V, Ax, x);
        };
        NullWatch watch;
        {
            Quiet q;
            EigenLOBPCG_d_multi(N, dV, ns, iter_max, ev_ref, X.data(), P.data(), work.data(), true, OpeA, watch);
        }
        *iters_ref = (int)((calls - 2LL * ns) / ns);

        const qumasun_b200::HamiltonianTables t = r.tables(V);
        qumasun_b200::Context ctx(0);
        qumasun_b200::Operator op(ctx, t);
        qumasun_b200::GpuOperator gop(op);
        std::vector<double> Xg(X0, X0 + (size_t)ns * N), Pg((size_t)ns * N, 0.0);
        EigenLOBPCG_d_multi(N, dV, ns, iter_max, ev_gpu, Xg.data(), Pg.data(), work.data(), true, gop, watch);
    } catch (const std::exception& e) {
        fprintf(stderr, "adapter_lobpcg_check: %s\n", e.what());
        return -1;
    }
    return 0;
}

}  // extern "C"
