"""SCF-step neighbours of the eigensolver on the B200 against the reference's outputs
(tests/golden/scf.npz, made by oracle/_ref) and the CPU oracle:

* density (qg_density_d / _z): the same sums in the same order with the same rounding
  as mSetDensityOne, so equal to the bit, at the fixture size and on the 64-atom 80^3
  cell with 256 states;
* Poisson + LDA potential (qg_potential_lda_d): 1e-12 relative to the reference
  (cuFFT against FFTW-order sums);
* Taylor-4 step (qg_td_taylor4_z): 1e-12 relative per state to QUMASUN::TimeEvoH4
  with the reference k-point H; on smooth states a step conserves the norm to O(dt^5);
* nonlocal energies and forces (qg_nonlocal_force_d): 1e-10 relative to the largest
  force / energy of the reference (ForceNonlocal, EnergyPPnonlocal)."""
import os

import numpy as np
import pytest

import oracle as O
from qumasun_b200.cell import build_cell, initial_states

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden", "scf.npz")


@pytest.fixture(scope="module")
def gold():
    return np.load(GOLD)


@pytest.fixture(scope="module")
def cell(gold):
    return build_cell(grid=tuple(int(v) for v in gold["grid"]))


def rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max()


def test_density_bit_exact(cuda_ctx, gold):
    import torch
    from qumasun_b200 import density
    X, occ = gold["X"], gold["occ"]
    rho = density(cuda_ctx, torch.from_numpy(X).cuda(), occ)
    np.testing.assert_array_equal(rho.cpu().numpy(), O.density(X, occ))
    # accumulate onto an existing density, complex states
    Z = gold["Z"]
    rz = density(cuda_ctx, torch.from_numpy(Z).cuda(), occ[:2], rho=rho.clone(), accumulate=True,
                 complex_states=True)
    np.testing.assert_array_equal(rz.cpu().numpy(), O.density_z(Z, occ[:2], rho0=O.density(X, occ)))
    # no occupied state: zeroed, or left as it is when accumulating
    r0 = density(cuda_ctx, torch.from_numpy(X).cuda(), np.zeros(3), rho=torch.ones(X.shape[1], dtype=torch.float64,
                                                                                       device="cuda"))
    assert float(r0.abs().max()) == 0.0


def test_density_full_size_bit_exact(cuda_ctx):
    """256 states of the 64-atom 80^3 cell with Fermi-like occupations (some zero)."""
    import torch
    from qumasun_b200 import density
    cell = build_cell(reps=(2, 2, 2))
    g = torch.Generator(device="cuda").manual_seed(3)
    X = torch.rand(256, cell.N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    occ = np.where(np.arange(256) < 200, 2.0 / (1.0 + np.exp((np.arange(256) - 180) / 7.0)), 0.0)
    rho = density(cuda_ctx, X, occ).cpu().numpy()
    np.testing.assert_array_equal(rho, O.density(X.cpu().numpy(), occ))


def test_potential_matches_reference(cuda_ctx, gold, cell):
    import torch
    from qumasun_b200 import Poisson
    P = Poisson(cuda_ctx, tuple(int(v) for v in gold["grid"]), tuple(gold["h"]))
    d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    vt, vh, vx, vc = P.potential(d(gold["rho"]), d(cell.V), pcc=d(gold["pcc"]), parts=True)
    torch.cuda.synchronize()
    assert rel(vh.cpu().numpy(), gold["vhart"]) < 1e-12
    assert rel(vx.cpu().numpy(), gold["vx"]) < 1e-13
    assert rel(vc.cpu().numpy(), gold["vc"]) < 1e-13
    assert rel(vt.cpu().numpy(), gold["vtot"]) < 1e-12
    # without core charge, only V_tot returned; against the port
    vt2 = P.potential(d(gold["rho"]), d(cell.V)).cpu().numpy()
    ref2 = O.potential_lda(tuple(int(v) for v in gold["grid"]), tuple(gold["h"]), gold["rho"], cell.V,
                           impl="port")[0]
    assert rel(vt2, ref2) < 1e-12
    P.close()


def test_potential_80cube_matches_port(cuda_ctx):
    import torch
    from qumasun_b200 import Poisson
    cell = build_cell(reps=(2, 2, 2))
    rho = 0.02 + 0.3 * np.exp(cell.V / 4.0)  # smooth, both LDA branches
    P = Poisson(cuda_ctx, (cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz))
    vt = P.potential(torch.from_numpy(rho).cuda(), torch.from_numpy(cell.V).cuda()).cpu().numpy()
    ref = O.potential_lda((cell.nx, cell.ny, cell.nz), (cell.hx, cell.hy, cell.hz), rho, cell.V, impl="port")[0]
    assert rel(vt, ref) < 1e-12
    P.close()


def test_taylor4_matches_reference(cuda_ctx, gold, cell):
    import torch
    from qumasun_b200 import Hamiltonian
    H = Hamiltonian(cuda_ctx, cell, kvec=tuple(gold["g"]))
    Z = torch.from_numpy(np.ascontiguousarray(gold["Z"])).cuda()
    H.td_taylor4(Z, float(gold["dt"]))
    out = Z.cpu().numpy()
    ref = gold["Z_taylor4"]
    err = np.linalg.norm(out - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert err.max() < 1e-12, err
    assert cuda_ctx.take_device_status() == 0
    H.close()


def test_taylor4_conserves_norm_on_smooth_states(cuda_ctx):
    """Low-frequency Bloch states of the 8-atom cell: twenty steps of dt = 0.002 keep the
    norm to 1e-9. A Taylor-4 step scales a component of energy E by
    |T4(-i dt E)|^2 = 1 - (dt E)^6/72 + (dt E)^8/576, which grows past dt E = 2.8; the FD
    spectrum of the 40^3 grid reaches ~700 Ha, so dt stays below 2.8/700."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell()
    N = cell.N
    x = np.arange(cell.nx) * cell.hx
    L = cell.nx * cell.hx
    X = np.zeros((3, 2 * N))
    z, y, xx = np.meshgrid(x, x, x, indexing="ij")
    for s, (kx, ky, kz) in enumerate(((1, 0, 0), (0, 1, 1), (1, 1, 0))):
        th = 2 * np.pi * (kx * xx + ky * y + kz * z) / L
        X[s, :N] = np.cos(th).reshape(-1)
        X[s, N:] = np.sin(th).reshape(-1)
    H = Hamiltonian(cuda_ctx, cell, kvec=(0.05, 0.0, 0.0))
    Xd = torch.from_numpy(X).cuda()
    n0 = (Xd ** 2).sum(dim=1)
    for _ in range(20):
        H.td_taylor4(Xd, 0.002)
    n1 = (Xd ** 2).sum(dim=1)
    assert float((n1 / n0 - 1.0).abs().max()) < 1e-9
    H.close()


def test_nonlocal_force_matches_reference(cuda_ctx, gold, cell):
    import torch
    from qumasun_b200 import Hamiltonian
    H = Hamiltonian(cuda_ctx, cell)
    f, e, ev = H.nonlocal_force(torch.from_numpy(gold["X"]).cuda(), gold["occ"])
    assert rel(f, gold["force_real"]) < 1e-10
    assert rel(e, gold["e_single"]) < 1e-10
    assert abs(ev - float(gold["ev_real"])) < 1e-10 * abs(float(gold["ev_real"]))
    # forces accumulate onto what the caller passes in
    f2, _, _ = H.nonlocal_force(torch.from_numpy(gold["X"]).cuda(), gold["occ"], forces=f)
    assert rel(f2, 2.0 * gold["force_real"]) < 1e-10
    H.close()


def test_nonlocal_force_64_atoms_matches_port(cuda_ctx):
    """64-atom 80^3 cell with displaced atoms, 6 states (two unoccupied), several chunks."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(2, 2, 2), displacement=0.05, seed=4)
    X = initial_states(6, cell.N, seed=8)
    occ = np.array([2.0, 2.0, 1.0, 0.5, 0.0, 0.0])
    H = Hamiltonian(cuda_ctx, cell)
    f, e, ev = H.nonlocal_force(torch.from_numpy(X).cuda(), occ)
    fr, er, evr = O.nonlocal_force(cell, X, occ, impl="port")
    assert rel(f, fr) < 1e-10 and rel(e, er) < 1e-10 and abs(ev - evr) < 1e-10 * abs(evr)
    H.close()
