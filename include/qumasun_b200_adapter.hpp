/*
 * qumasun_b200_adapter.hpp -- header-only C++ adapter over the C ABI of
 * qumasun_b200.h, for the reference's own call sites.
 *
 * QUMASUN calls its eigensolvers as templates over a host callback that applies H
 * to one state:
 *   EigenLOBPCG_d_multi(N, dVol, ns, iter_max, ev, evec, keep, work, is_first_time,
 *                       OpeA, watch)                         (lobpcg_d_multi.h:23-27)
 * called from qumasun_single.lobpcg.h:17-23, and
 *   LOBPCG::Eigen_z_multi_mpi(l_grid, dVol, ns, iter_max, ev, evec, keep_P, work,
 *                             keep_S_matrix, SCF_step, sk, OpeA, watch)
 *                                                             (lobpcg_z_multi_mpi.h:988-996)
 * called from qumasun_kpoint.lobpcg.h:32-41. A host callback cannot run on the GPU, so
 * the engine takes the Hamiltonian as data. This header supplies:
 *  - flatten_projectors(): the per-atom cube tables of PseudoPotIntegrator_single
 *    (PP_nonlocal_each_atom: one SubspaceField per projector w_k and per Y_lm,
 *    PseudoPotOperator.h:21-24, as UpdatePosition tabulates them, :453-466) flattened
 *    into a qg_hamiltonian_desc;
 *  - Context / Operator: RAII owners of qg_context / qg_hamiltonian;
 *  - GpuOperator: a tag type passed where the reference passes OpeA; overloads of
 *    EigenLOBPCG_d_multi (and, with QUMASUN_B200_ADAPTER_KPOINT defined after the
 *    reference's lobpcg_z_multi_mpi.h, LOBPCG::Eigen_z_multi_mpi) taking it are more
 *    specialised than the reference's templates, so an unchanged call site with a
 *    GpuOperator in place of the lambda runs the GPU solver.
 * Errors throw std::runtime_error carrying the engine's status and message; reaching
 * iter_max is not an error (the reference returns after iter_max too).
 */
#pragma once

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "qumasun_b200.h"

namespace qumasun_b200 {

inline void check(int status, const char* where) {
    if (status == QG_OK) return;
    std::string msg = std::string(where) + ": " + qg_status_string(status);
    const char* detail = qg_last_error();
    if (detail && *detail) msg += std::string(" (") + detail + ")";
    throw std::runtime_error(msg);
}

/* Owns the flat arrays a qg_hamiltonian_desc points into. */
struct HamiltonianTables {
    int nx = 0, ny = 0, nz = 0;
    double hx = 0, hy = 0, hz = 0;
    int fd_order = 8;
    int n_atoms = 0, n_proj = 0, n_lm = 0;
    double gx = 0, gy = 0, gz = 0;
    std::vector<double> V, atom_pos, proj_E, w_data, ylm_data;
    std::vector<int> proj_l, cube;
    std::vector<long long> w_off, ylm_off;

    /* The descriptor; valid while this object lives and is not modified. */
    qg_hamiltonian_desc desc() const {
        qg_hamiltonian_desc d;
        std::memset(&d, 0, sizeof(d));
        d.nx = nx; d.ny = ny; d.nz = nz;
        d.hx = hx; d.hy = hy; d.hz = hz;
        d.fd_order = fd_order;
        d.V = V.data();
        d.n_atoms = n_atoms;
        d.atom_pos = atom_pos.data();
        d.n_proj = n_proj;
        d.proj_l = proj_l.data();
        d.proj_E = proj_E.data();
        d.cube = cube.data();
        d.w_data = w_data.data();
        d.w_off = w_off.data();
        d.n_lm = n_lm;
        d.ylm_data = ylm_data.data();
        d.ylm_off = ylm_off.data();
        d.gx = gx; d.gy = gy; d.gz = gz;
        return d;
    }
};

/* Flattens the reference's per-atom projector tables.
 *  per_atom[a].projector[k]: the w_k cube of atom a (SubspaceField: begin_grid_{x,y,z},
 *      num_grid_{x,y,z}, num_total_grid, GetGridPointer(), x fastest);
 *  per_atom[a].Ylm[lm]: Y_lm on the cube of the first projector with that l,
 *      lm = l*l + (m + l) (mMakeSubspacePPnonlocal_Ylm, PseudoPotOperator.h:567-727);
 *  positions[a].Rx/Ry/Rz: the nuclei (Nucleus);
 *  proj_l / proj_E: each projector's l and energy (PseudoPot_MBK::projector_quantum_l,
 *      projector_energy_up), the same for every atom (one species).
 * V (nx*ny*nz values) is copied. Atoms whose table lists are empty carry no projector;
 * then n_atoms is 0 only if every list is empty. */
template <class EachAtom, class Pos>
HamiltonianTables flatten_projectors(int nx, int ny, int nz, double hx, double hy, double hz, int fd_order,
                                     const double* V, const std::vector<EachAtom>& per_atom, const Pos* positions,
                                     const std::vector<int>& proj_l, const std::vector<double>& proj_E) {
    HamiltonianTables t;
    t.nx = nx; t.ny = ny; t.nz = nz;
    t.hx = hx; t.hy = hy; t.hz = hz;
    t.fd_order = fd_order;
    t.V.assign(V, V + (size_t)nx * ny * nz);
    const int na = (int)per_atom.size();
    const int np = (int)proj_l.size();
    int lmax = -1;
    for (int l : proj_l) lmax = l > lmax ? l : lmax;
    const int nlm = (lmax + 1) * (lmax + 1);
    bool any = false;
    for (const auto& at : per_atom) any = any || !at.projector.empty();
    if (!any || np == 0) {
        t.n_atoms = 0;
        return t;
    }
    if (proj_E.size() != proj_l.size()) throw std::runtime_error("flatten_projectors: proj_l / proj_E sizes differ");
    t.n_atoms = na;
    t.n_proj = np;
    t.n_lm = nlm;
    t.proj_l = proj_l;
    t.proj_E = proj_E;
    t.cube.resize((size_t)na * np * 6);
    t.w_off.resize((size_t)na * np);
    t.ylm_off.resize((size_t)na * nlm);
    for (int a = 0; a < na; ++a) {
        t.atom_pos.push_back(positions[a].Rx);
        t.atom_pos.push_back(positions[a].Ry);
        t.atom_pos.push_back(positions[a].Rz);
        const auto& at = per_atom[a];
        if ((int)at.projector.size() != np || (int)at.Ylm.size() < nlm)
            throw std::runtime_error("flatten_projectors: atom tables do not match proj_l");
        for (int k = 0; k < np; ++k) {
            const auto& f = at.projector[k];
            int* c = &t.cube[((size_t)a * np + k) * 6];
            c[0] = f.begin_grid_x; c[1] = f.begin_grid_y; c[2] = f.begin_grid_z;
            c[3] = f.num_grid_x; c[4] = f.num_grid_y; c[5] = f.num_grid_z;
            t.w_off[(size_t)a * np + k] = (long long)t.w_data.size();
            const double* p = f.GetGridPointer();
            t.w_data.insert(t.w_data.end(), p, p + f.num_total_grid);
        }
        for (int lm = 0; lm < nlm; ++lm) {
            const auto& f = at.Ylm[lm];
            t.ylm_off[(size_t)a * nlm + lm] = (long long)t.ylm_data.size();
            const double* p = f.GetGridPointer();
            t.ylm_data.insert(t.ylm_data.end(), p, p + f.num_total_grid);
        }
    }
    return t;
}

/* RAII owner of a qg_context. */
class Context {
public:
    explicit Context(int device = 0) { check(qg_context_create(device, &h_), "qg_context_create"); }
    ~Context() { if (h_) qg_context_destroy(h_); }
    Context(const Context&) = delete;
    Context& operator=(const Context&) = delete;
    qg_context get() const { return h_; }

private:
    qg_context h_ = nullptr;
};

/* RAII owner of a qg_hamiltonian built from tables (copied by the library). */
class Operator {
public:
    Operator(const Context& ctx, const HamiltonianTables& t) : N_((long long)t.nx * t.ny * t.nz) {
        const qg_hamiltonian_desc d = t.desc();
        check(qg_hamiltonian_create(ctx.get(), &d, &h_), "qg_hamiltonian_create");
    }
    ~Operator() { if (h_) qg_hamiltonian_destroy(h_); }
    Operator(const Operator&) = delete;
    Operator& operator=(const Operator&) = delete;
    qg_hamiltonian get() const { return h_; }
    long long N() const { return N_; }
    /* HX = H X for ns host states (state-major, N each). */
    void apply(int ns, const double* X, double* HX) const {
        check(qg_hamiltonian_apply_host_d(h_, ns, X, HX), "qg_hamiltonian_apply_host_d");
    }

private:
    qg_hamiltonian h_ = nullptr;
    long long N_ = 0;
};

/* Passed where the reference passes OpeA. tol follows the serial solver's stopping rule
 * (max_j |r_j|^2 dV < tol dV); precond 0 reproduces the reference's unpreconditioned
 * iteration, 1 uses the kinetic preconditioner. */
struct GpuOperator {
    qg_hamiltonian ham = nullptr;
    int precond = 0;
    double precond_shift = 1.0;
    qg_precision precision = QG_FP64;
    double tol = 1.0e-10;
    int n_converge = 0;
    qg_lobpcg_report* report = nullptr;  // optional: receives the solve's report

    explicit GpuOperator(const Operator& op) : ham(op.get()) {}
    explicit GpuOperator(qg_hamiltonian h) : ham(h) {}

    qg_lobpcg_options options(int iter_max, bool first) const {
        qg_lobpcg_options o;
        std::memset(&o, 0, sizeof(o));
        o.max_iter = iter_max;
        o.tol = tol;
        o.first_call = first ? 1 : 0;
        o.precision = precision;
        o.verbose = 0;
        o.precond = precond;
        o.precond_shift = precond_shift;
        o.n_converge = n_converge;
        return o;
    }
};

}  // namespace qumasun_b200

/* The GPU form of the reference's serial block LOBPCG (lobpcg_d_multi.h:23-545):
 * eigen_vectors (ns*N, in/out) and keep (the P block, ns*N, in/out) are the reference's
 * host buffers, state-major; eigen_values (ns) out; work is not used (the GPU keeps its
 * own); watch is not used. dVol must be the operator's hx*hy*hz and N its point count. */
template <class W>
inline void EigenLOBPCG_d_multi(int N, double dVol, int ns, int iter_max, double* eigen_values,
                                double* eigen_vectors, double* keep, double* /*work*/, bool is_first_time,
                                qumasun_b200::GpuOperator OpeA, W& /*watch*/) {
    (void)dVol;
    (void)N;
    const qg_lobpcg_options o = OpeA.options(iter_max, is_first_time);
    qg_lobpcg_report rep;
    std::memset(&rep, 0, sizeof(rep));
    const int st = qg_lobpcg_d(OpeA.ham, &o, ns, eigen_values, eigen_vectors, keep, &rep);
    if (OpeA.report) *OpeA.report = rep;
    if (st != QG_ERR_NOT_CONVERGED) qumasun_b200::check(st, "qg_lobpcg_d");
}

#ifdef QUMASUN_B200_ADAPTER_KPOINT
/* The GPU form of LOBPCG::Eigen_z_multi_mpi (lobpcg_z_multi_mpi.h:988-1800) on one rank:
 * eigen_vectors[s] = {re, im} of state s; keep_P (ns*2N, {re, im} per state) in/out;
 * SCF_step == 0 starts P from zero (first call). keep_S_matrix, work, sk, watch and the
 * grid's communicator are not used; the grid must cover the whole cell (one rank). The
 * states are packed into {re[N], im[N]} blocks around the call unless they already lie
 * that way. Include this header after the reference's lobpcg_z_multi_mpi.h. */
namespace LOBPCG {
template <class W>
inline void Eigen_z_multi_mpi(const GridRangeMPI& l_grid, const double dVol, const int num_solution,
                              const int iter_max, double* eigen_values, SoAComplex* eigen_vectors, double* keep_P,
                              double* /*work*/, OneComplex* /*keep_S_matrix*/, int SCF_step, int /*sk*/,
                              qumasun_b200::GpuOperator OpeA, W& /*watch*/) {
    (void)dVol;
    const size_t N = l_grid.Size3D();
    bool packed = true;
    for (int s = 0; s < num_solution; ++s)
        packed = packed && eigen_vectors[s].re == eigen_vectors[0].re + 2 * N * (size_t)s &&
                 eigen_vectors[s].im == eigen_vectors[s].re + N;
    std::vector<double> X;
    double* xp = eigen_vectors[0].re;
    if (!packed) {
        X.resize(2 * N * (size_t)num_solution);
        for (int s = 0; s < num_solution; ++s) {
            std::memcpy(&X[2 * N * s], eigen_vectors[s].re, N * sizeof(double));
            std::memcpy(&X[2 * N * s + N], eigen_vectors[s].im, N * sizeof(double));
        }
        xp = X.data();
    }
    const qg_lobpcg_options o = OpeA.options(iter_max, SCF_step == 0);
    qg_lobpcg_report rep;
    std::memset(&rep, 0, sizeof(rep));
    const int st = qg_lobpcg_z(OpeA.ham, &o, num_solution, eigen_values, xp, keep_P, &rep);
    if (OpeA.report) *OpeA.report = rep;
    if (!packed)
        for (int s = 0; s < num_solution; ++s) {
            std::memcpy(eigen_vectors[s].re, &X[2 * N * s], N * sizeof(double));
            std::memcpy(eigen_vectors[s].im, &X[2 * N * s + N], N * sizeof(double));
        }
    if (st != QG_ERR_NOT_CONVERGED) qumasun_b200::check(st, "qg_lobpcg_z");
}
}  // namespace LOBPCG
#endif
