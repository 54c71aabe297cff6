"""Generates tests/golden/*.npz from the reference's own code (oracle/_ref).

Run where the reference tree exists and `make -C oracle` has built
oracle/_ref/libqumasun_ref.so:  python tests/golden/make_golden.py
Every array comes from the reference functions driven by oracle/ref_harness.cpp:
Laplasian{2,4,6,8}th_halo, LaplasianKpoint8th_halo, the reference Hamiltonian
(V, ProjectionPP, kinetic), the reference k-point Hamiltonian (V,
PseudoPotIntegrator_kpoint::ProjectionPP, LaplasianKpoint8th; `--kpoint` writes
only ham_kpoint.npz) and GridForSphere / SetYlmAround tables. `--scf` writes
scf.npz: the FFT Poisson + LDA potential (SetPotentialByPoissonFFT, Calc_XC_LDA),
Fermi occupations (SetOccupancy), the 8th-order gradient (Gradient8th), one Taylor-4
step (QUMASUN::TimeEvoH4) and nonlocal energies and forces
(PseudoPotIntegrator_kpoint::ForceNonlocal, PseudoPotIntegrator_single::EnergyPPnonlocal).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle as O  # noqa: E402
from qumasun_b200.cell import build_cell, initial_states  # noqa: E402

# small cells: (name, build_cell kwargs). "wrap" has projector cubes larger than
# the cell, so a grid point is covered by several periodic images of one atom.
CASES = [
    ("noncubic", dict(grid=(20, 16, 24))),
    ("wrap", dict(grid=(12, 12, 12), a0=4.4)),
]


def main():
    for name, kw in CASES:
        cell = build_cell(**kw)
        X = initial_states(2, cell.N, seed=7)
        out = dict(X=X, grid=np.array([cell.nx, cell.ny, cell.nz]),
                   h=np.array([cell.hx, cell.hy, cell.hz]), V=cell.V,
                   positions=cell.positions)
        for order in (2, 4, 6, 8):
            out[f"HX{order}"] = O.hamiltonian_apply(cell, X, impl="ref", fd_order=order)
            out[f"LAP{order}"] = O.laplacian(order, (cell.nx, cell.ny, cell.nz),
                                             (cell.hx, cell.hy, cell.hz), -0.5, X[0], impl="ref")
        g = (0.31, -0.17, 0.05)
        ore, oim = O.laplacian_kpoint8((cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz),
                                       -0.5, g, X[0], X[1], impl="ref")
        out["kp_g"] = np.array(g)
        out["KP_re"], out["KP_im"] = ore, oim
        # the reference's own projector-cube geometry and Y_lm tables for atom 0
        lib = O.ref_lib()
        import ctypes as C
        R = cell.positions[0]
        c6 = (C.c_int * 6)()
        lib.ref_grid_for_sphere(R[0], R[1], R[2], cell.cutoff, cell.hx, cell.hy, cell.hz, c6)
        b = np.array(c6[:3], dtype=np.int32)
        s = np.array([c6[3] - c6[0], c6[4] - c6[1], c6[5] - c6[2]], dtype=np.int32)
        out["cube0"] = np.concatenate([b, s])
        for lm, (l, m) in enumerate([(0, 0), (1, -1), (1, 0), (1, 1)]):
            buf = np.zeros(int(np.prod(s)))
            Rv = np.ascontiguousarray(R, dtype=np.float64)
            hv = np.array([cell.hx, cell.hy, cell.hz])
            lib.ref_ylm_cube(l, m, b.ctypes.data_as(C.POINTER(C.c_int)), s.ctypes.data_as(C.POINTER(C.c_int)),
                             Rv.ctypes.data_as(C.POINTER(C.c_double)), hv.ctypes.data_as(C.POINTER(C.c_double)),
                             buf.ctypes.data_as(C.POINTER(C.c_double)))
            out[f"Y{lm}"] = buf
        np.savez_compressed(os.path.join(HERE, f"ham_{name}.npz"), **out)
        print("wrote", name)
    # the reference's serial block LOBPCG (EigenLOBPCG_d_multi) on a small cell
    cell = build_cell(grid=(16, 16, 16))
    X0 = initial_states(6, cell.N, seed=11)
    r = O.ref_lobpcg_d_multi(cell, X0, 2000)
    np.savez_compressed(os.path.join(HERE, "lobpcg_small.npz"), grid=np.array([16, 16, 16]),
                        ns=6, seed=11, ev=r["ev"], iters=r["iters"])
    print("wrote lobpcg_small", r["iters"], r["ev"])


def smooth_state(cell):
    """{re, im} of one smooth state: Gaussians (width 1.2 bohr) centred on atoms 0 and 1."""
    out = []
    for a in (0, 1):
        R = cell.positions[a]
        x = cell.hx * np.arange(cell.nx) - R[0]
        y = cell.hy * np.arange(cell.ny) - R[1]
        z = cell.hz * np.arange(cell.nz) - R[2]
        rr = z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2
        out.append(np.exp(-rr / (2 * 1.2 ** 2)).reshape(-1))
    return np.concatenate(out)


# k-point cases: Gamma, a commensurate k (a quarter and a half of the cell's
# reciprocal vectors) and a general k; "wrap" cubes exceed the cell, so one grid
# point carries several periodic images of an atom with different Bloch phases.
KPOINT_CASES = [
    ("noncubic", dict(grid=(20, 16, 24), displacement=0.05, seed=3)),
    ("wrap", dict(grid=(12, 12, 12), a0=4.4)),
]


def make_kpoint():
    out = {}
    for name, kw in KPOINT_CASES:
        cell = build_cell(**kw)
        X = np.stack([initial_states(1, 2 * cell.N, seed=13)[0], smooth_state(cell)])
        L = np.array([cell.nx * cell.hx, cell.ny * cell.hy, cell.nz * cell.hz])
        gs = [(0.0, 0.0, 0.0), tuple(2 * np.pi / L * np.array([0.25, -0.5, 0.25])), (0.31, -0.17, 0.05)]
        out[f"{name}_X"] = X
        out[f"{name}_g"] = np.array(gs)
        for i, g in enumerate(gs):
            out[f"{name}_HX{i}"] = O.hamiltonian_kpoint_apply(cell, g, X, impl="ref")
            # FD orders 2 and 6 (LaplasianKpoint2nd / 6th) at the general k-vector too
            if i == 2:
                for order in (2, 6):
                    out[f"{name}_HX{i}_o{order}"] = O.hamiltonian_kpoint_apply(cell, g, X, impl="ref",
                                                                            fd_order=order)
    np.savez_compressed(os.path.join(HERE, "ham_kpoint.npz"), **out)
    print("wrote ham_kpoint")


def make_lobpcg_kpoint():
    """The reference's complex LOBPCG (Eigen_z_multi_mpi) at a general k on the
    12^3 "wrap" cell (checked against a dense eigensolve of the same operator)
    and at a 4x4x4 Monkhorst-Pack point of the 8-atom 40^3 cell. The reference
    solver's residual escape does not fire on these cells, so it runs a fixed
    iteration count; the count is large enough that the eigenvalues no longer
    move (checked against a run 200 iterations shorter). On the 40^3 cell the
    reference solver leaves its 16th eigenvalue 8e-8 Ha above the Lanczos value
    (d8_lanczos) while the lower 15 agree to 1e-10."""
    out = {}
    cell = build_cell(grid=(12, 12, 12), a0=4.4)
    g = (0.31, -0.17, 0.05)
    X0 = initial_states(6, 2 * cell.N, seed=3)
    r = O.ref_lobpcg_z_multi(cell, g, X0, 600)
    dense = np.linalg.eigvalsh(O.dense_kpoint_hamiltonian(cell, g))[:8]
    assert np.abs(np.sort(r["ev"]) - dense[:6]).max() < 1e-10
    out.update(small_g=np.array(g), small_ns=6, small_seed=3, small_ev=r["ev"], small_iters=r["iters"],
               small_dense=dense)
    cell = build_cell()
    g = tuple(2 * np.pi / 6.74 * np.array([1 / 8, 3 / 8, -1 / 8]))
    X0 = initial_states(16, 2 * cell.N, seed=1234)
    r = O.ref_lobpcg_z_multi(cell, g, X0, 1000)
    r2 = O.ref_lobpcg_z_multi(cell, g, X0, 800)
    assert np.abs(r["ev"] - r2["ev"]).max() < 1e-10
    # an independent check of the same spectrum: implicitly restarted Lanczos (ARPACK)
    # on the oracle operator, 20 lowest eigenvalues
    import scipy.sparse.linalg as sla
    N = cell.N

    def mv(v):
        v = np.asarray(v).reshape(-1)
        HX = O.hamiltonian_kpoint_apply(cell, g, np.concatenate([v.real, v.imag])[None])[0]
        return HX[:N] + 1j * HX[N:]

    op = sla.LinearOperator((N, N), matvec=mv, dtype=np.complex128)
    lanczos = np.sort(sla.eigsh(op, k=20, which="SA", tol=1e-13, ncv=60, return_eigenvectors=False))
    out.update(d8_g=np.array(g), d8_ns=16, d8_seed=1234, d8_ev=r["ev"], d8_iters=r["iters"],
               d8_seconds=r["seconds"], d8_lanczos=lanczos)
    np.savez_compressed(os.path.join(HERE, "lobpcg_kpoint.npz"), **out)
    print("wrote lobpcg_kpoint", out["small_ev"], out["d8_ev"])


def make_scf():
    """Reference outputs of the SCF-step neighbours on the non-cubic 20x16x24 cell."""
    cell = build_cell(grid=(20, 16, 24))
    grid = (cell.nx, cell.ny, cell.nz)
    h = (cell.hx, cell.hy, cell.hz)
    X = initial_states(3, cell.N, seed=41)
    occ = np.array([2.0, 1.5, 0.0])
    rng = np.random.default_rng(42)
    # a density spanning both LDA branches (rs < 1 and rs >= 1) and the 1e-8 cut-off
    rho = 0.6 * O.density(X, occ)
    rho[::97] = 0.0
    pcc = 0.05 * np.exp(-((np.arange(cell.N) % 37) / 9.0) ** 2)
    vt, vh, vx, vc = O.potential_lda(grid, h, rho, cell.V, pcc=pcc, impl="ref")
    ev = np.sort(rng.uniform(-0.9, 0.4, 24))
    occ_mu, tot_mu = O.fermi(2.0, 0.01, ev, -0.2, impl="ref")
    occ_b, mu_b = O.occupancy(0.01, ev, 30, impl="ref")
    gx, gy, gz = O.gradient8(grid, h, -3.0, X[0], impl="ref")
    Z = np.ascontiguousarray(np.concatenate([X[:2], 0.4 * X[1:3][::-1]], axis=1))
    g = (0.31, -0.17, 0.05)
    Zt = O.td_taylor4(cell, g, 0.02, Z, impl="ref")
    f_r, e_r, ev_r = O.nonlocal_force(cell, X, occ, impl="ref")
    f_z, e_z, ev_z = O.nonlocal_force(cell, Z, occ[:2], g=g, impl="ref")
    e_single = O.nonlocal_energy(cell, X)
    np.savez_compressed(os.path.join(HERE, "scf.npz"), grid=np.array(grid), h=np.array(h), X=X, occ=occ,
                        rho=rho, pcc=pcc, vtot=vt, vhart=vh, vx=vx, vc=vc, ev=ev, occ_mu=occ_mu, tot_mu=tot_mu,
                        occ_bisect=occ_b, mu_bisect=mu_b, grad=np.stack([gx, gy, gz]), Z=Z, g=np.array(g),
                        dt=0.02, Z_taylor4=Zt, force_real=f_r, e_real=e_r, ev_real=ev_r, force_z=f_z, e_z=e_z,
                        ev_z=ev_z, e_single=e_single)
    print("wrote scf", ev_r, ev_z, mu_b)


if __name__ == "__main__" and "--scf" in sys.argv:
    make_scf()
elif __name__ == "__main__" and "--lobpcg-kpoint" in sys.argv:
    make_lobpcg_kpoint()
elif __name__ == "__main__" and "--kpoint" in sys.argv:
    make_kpoint()
elif __name__ == "__main__" and "--diamond8" not in sys.argv:
    main()
    make_kpoint()

# lobpcg_diamond8.npz (the 8-atom 40^3 cell, 16 states, seed 1234, FD order 8) is
# the output of oracle.ref_lobpcg_d_multi(build_cell(), initial_states(16, 64000,
# seed=1234), 3000): 435 iterations, about 3 minutes on one core. Regenerate with
#   python tests/golden/make_golden.py --diamond8
if __name__ == "__main__" and "--diamond8" in sys.argv:
    cell = build_cell()
    r = O.ref_lobpcg_d_multi(cell, initial_states(16, cell.N, seed=1234), 3000)
    np.savez_compressed(os.path.join(HERE, "lobpcg_diamond8.npz"), ev=r["ev"], iters=r["iters"], ns=16,
                        seed=1234, seconds=r["seconds"])
