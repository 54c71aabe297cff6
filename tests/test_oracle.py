"""The CPU oracle against the reference's own outputs (golden fixtures made by
tests/golden/make_golden.py from oracle/_ref, i.e. the reference headers)."""
import os

import numpy as np
import pytest

import oracle as O
from qumasun_b200.cell import build_cell, grid_for_sphere, initial_states

GOLD = os.path.join(os.path.dirname(__file__), "golden")
CASES = {"noncubic": dict(grid=(20, 16, 24)), "wrap": dict(grid=(12, 12, 12), a0=4.4)}


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    name = request.param
    g = np.load(os.path.join(GOLD, f"ham_{name}.npz"))
    return name, build_cell(**CASES[name]), g


def test_cell_builder_reproduces_fixture_inputs(case):
    _, cell, g = case
    assert tuple(g["grid"]) == (cell.nx, cell.ny, cell.nz)
    np.testing.assert_array_equal(g["V"], cell.V)
    np.testing.assert_array_equal(g["positions"], cell.positions)
    np.testing.assert_array_equal(g["X"], initial_states(2, cell.N, seed=7))


def test_projector_tables_match_reference_tabulation(case):
    # GridForSphere (GridSubgrid.h:482-492) and SetYlmAround<L,M> (PseudoPotOperator.h:58-71)
    _, cell, g = case
    R = cell.positions[0]
    b, e = grid_for_sphere(R, cell.cutoff, (cell.hx, cell.hy, cell.hz))
    np.testing.assert_array_equal(g["cube0"], np.array(b + [e[i] - b[i] for i in range(3)]))
    for lm in range(4):
        np.testing.assert_allclose(cell.ylm_tabs[0][lm], g[f"Y{lm}"], rtol=0, atol=2e-16)


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_port_laplacian_matches_reference(case, order):
    _, cell, g = case
    lap = O.laplacian(order, (cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz), -0.5, g["X"][0])
    assert rel(lap, g[f"LAP{order}"]) < 1e-15


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_port_hamiltonian_matches_reference(case, order):
    _, cell, g = case
    HX = O.hamiltonian_apply(cell, g["X"], impl="port", fd_order=order)
    for s in range(2):
        assert rel(HX[s], g[f"HX{order}"][s]) < 1e-14


def test_port_kpoint_laplacian_matches_reference(case):
    _, cell, g = case
    ore, oim = O.laplacian_kpoint8((cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz), -0.5,
                                   tuple(g["kp_g"]), g["X"][0], g["X"][1])
    np.testing.assert_array_equal(ore, g["KP_re"])
    np.testing.assert_array_equal(oim, g["KP_im"])


def test_port_lobpcg_matches_reference_eigenvalues_and_iterations():
    g = np.load(os.path.join(GOLD, "lobpcg_small.npz"))
    cell = build_cell(grid=tuple(g["grid"]))
    X0 = initial_states(int(g["ns"]), cell.N, seed=int(g["seed"]))
    r = O.lobpcg_d_multi(lambda X: O.hamiltonian_apply(cell, X), X0, cell.dV, 2000)
    assert r["iters"] == int(g["iters"])
    np.testing.assert_allclose(r["ev"], g["ev"], rtol=0, atol=1e-10)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_port_matches_live_reference_on_fresh_cell():
    cell = build_cell(grid=(16, 20, 12), displacement=0.2, seed=3)
    X = initial_states(3, cell.N, seed=99)
    a = O.hamiltonian_apply(cell, X, impl="port")
    b = O.hamiltonian_apply(cell, X, impl="ref")
    assert max(rel(a[s], b[s]) for s in range(3)) < 1e-14


# ---------------------------------------------------------------- k-point H
KPOINT_CASES = {"noncubic": dict(grid=(20, 16, 24), displacement=0.05, seed=3),
                "wrap": dict(grid=(12, 12, 12), a0=4.4)}


@pytest.fixture(scope="module")
def kpoint_gold():
    return np.load(os.path.join(GOLD, "ham_kpoint.npz"))


@pytest.mark.parametrize("name", sorted(KPOINT_CASES))
def test_port_kpoint_hamiltonian_matches_reference(kpoint_gold, name):
    # PseudoPotIntegrator_kpoint::ProjectionPP + LaplasianKpoint8th (qumasun_kpoint.matrix.h:25-50)
    cell = build_cell(**KPOINT_CASES[name])
    X = kpoint_gold[f"{name}_X"]
    for i, g in enumerate(kpoint_gold[f"{name}_g"]):
        ref = kpoint_gold[f"{name}_HX{i}"]
        HX = O.hamiltonian_kpoint_apply(cell, tuple(g), X)
        loc = O.hamiltonian_kpoint_local(cell, tuple(g), X)
        for s in range(2):
            assert rel(HX[s], ref[s]) < 1e-14
            # the nonlocal part alone, relative to its own size (for the random state it is
            # ~4e-4 of the total, so the subtraction costs about three digits)
            assert rel(HX[s] - loc[s], ref[s] - loc[s]) < 1e-12


@pytest.mark.parametrize("order", [2, 6])
@pytest.mark.parametrize("name", sorted(KPOINT_CASES))
def test_port_kpoint_fd_orders_2_6_match_reference(kpoint_gold, name, order):
    # LaplasianKpoint2nd / LaplasianKpoint6th (GridDifferenceKpoint2nd.h, 6th.h) in the k-point H
    cell = build_cell(**KPOINT_CASES[name])
    X = kpoint_gold[f"{name}_X"]
    g = tuple(kpoint_gold[f"{name}_g"][2])
    HX = O.hamiltonian_kpoint_apply(cell, g, X, fd_order=order)
    ref = kpoint_gold[f"{name}_HX2_o{order}"]
    for s in range(2):
        assert rel(HX[s], ref[s]) < 1e-14
    # and the stencil alone is the reference's to the bit
    re, im = X[0, :cell.N], X[0, cell.N:]
    a = O.laplacian_kpoint(order, (cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz), -0.5, g, re, im)
    b = O.laplacian_kpoint(order, (cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz), -0.5, g, re, im,
                           impl="ref") if O.ref_available() else a
    np.testing.assert_array_equal(a[0], b[0])
    np.testing.assert_array_equal(a[1], b[1])


def test_port_kpoint_nonlocal_is_gauge_covariant_for_commensurate_k():
    # For g a reciprocal vector of the cell the Bloch phase is periodic on the
    # grid, so V_NL(g) u = exp(-i g.r) V_NL(0) (exp(i g.r) u) holds exactly.
    cell = build_cell(grid=(20, 16, 24), displacement=0.05, seed=3)
    N = cell.N
    L = np.array([cell.nx * cell.hx, cell.ny * cell.hy, cell.nz * cell.hz])
    g = 2 * np.pi / L * np.array([1.0, -2.0, 1.0])
    u = initial_states(1, 2 * N, seed=21)[0]
    uc = u[:N] + 1j * u[N:]
    ix = np.arange(cell.nx) * cell.hx
    iy = np.arange(cell.ny) * cell.hy
    iz = np.arange(cell.nz) * cell.hz
    phase = np.exp(1j * (g[2] * iz[:, None, None] + g[1] * iy[None, :, None] + g[0] * ix[None, None, :])).reshape(-1)

    def nl(gv, vec):
        X = np.concatenate([vec.real, vec.imag])[None]
        out = O.hamiltonian_kpoint_apply(cell, tuple(gv), X) - O.hamiltonian_kpoint_local(cell, tuple(gv), X)
        return out[0, :N] + 1j * out[0, N:]

    lhs = nl(g, uc)
    rhs = np.conj(phase) * nl((0.0, 0.0, 0.0), phase * uc)
    assert np.linalg.norm(lhs - rhs) / np.linalg.norm(lhs) < 1e-12


def test_port_kpoint_hamiltonian_is_hermitian():
    cell = build_cell(grid=(20, 16, 24), displacement=0.05, seed=3)
    N = cell.N
    g = (0.31, -0.17, 0.05)
    X = initial_states(2, 2 * N, seed=17)
    HX = O.hamiltonian_kpoint_apply(cell, g, X)
    z = X[:, :N] + 1j * X[:, N:]
    hz = HX[:, :N] + 1j * HX[:, N:]
    a = np.vdot(z[0], hz[1])
    b = np.conj(np.vdot(z[1], hz[0]))
    assert abs(a - b) < 1e-12 * abs(a)


@pytest.mark.skipif(not O.ref_available(), reason="oracle/_ref not built here")
def test_port_kpoint_matches_live_reference_on_fresh_cell():
    cell = build_cell(grid=(16, 20, 12), displacement=0.2, seed=4)
    X = initial_states(2, 2 * cell.N, seed=98)
    g = (-0.2, 0.45, 0.1)
    a = O.hamiltonian_kpoint_apply(cell, g, X, impl="port")
    b = O.hamiltonian_kpoint_apply(cell, g, X, impl="ref")
    assert rel(a, b) < 1e-14


def test_port_dense_kpoint_spectrum_matches_reference_complex_solver():
    # eigenvalues of the port's k-point operator (dense) against the reference's
    # own Eigen_z_multi_mpi run on the reference operator (golden fixture)
    g = np.load(os.path.join(GOLD, "lobpcg_kpoint.npz"))
    cell = build_cell(grid=(12, 12, 12), a0=4.4)
    w = np.linalg.eigvalsh(O.dense_kpoint_hamiltonian(cell, tuple(g["small_g"])))
    np.testing.assert_allclose(w[:6], np.sort(g["small_ev"]), rtol=0, atol=1e-10)
