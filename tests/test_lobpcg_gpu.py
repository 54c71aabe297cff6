"""GPU block LOBPCG (qg_lobpcg_d) against the reference's EigenLOBPCG_d_multi.

Tolerance: eigenvalues within 1e-8 Ha of the reference's (golden fixtures made
from oracle/_ref, i.e. the reference's own solver and Hamiltonian)."""
import os

import numpy as np
import pytest

import oracle as O
from qumasun_b200.cell import build_cell, initial_states

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
EV_TOL = 1e-8


def test_small_cell_matches_reference_solver(cuda_ctx):
    from qumasun_b200 import Hamiltonian
    g = np.load(os.path.join(GOLD, "lobpcg_small.npz"))
    cell = build_cell(grid=tuple(g["grid"]))
    X0 = initial_states(int(g["ns"]), cell.N, seed=int(g["seed"]))
    H = Hamiltonian(cuda_ctx, cell)
    r = H.lobpcg(X0, max_iter=2000)
    H.close()
    assert r["status"] == 0 and r["report"]["converged"] == 1
    np.testing.assert_allclose(r["ev"], g["ev"], rtol=0, atol=EV_TOL)
    assert abs(r["report"]["iterations"] - int(g["iters"])) <= 5


def test_diamond8_matches_reference_solver(cuda_ctx):
    """8 atoms, 40^3, FD order 8, 16 states from seeded uniform(-0.5, 0.5)."""
    from qumasun_b200 import Hamiltonian
    g = np.load(os.path.join(GOLD, "lobpcg_diamond8.npz"))
    cell = build_cell()
    X0 = initial_states(int(g["ns"]), cell.N, seed=int(g["seed"]))
    H = Hamiltonian(cuda_ctx, cell)
    r = H.lobpcg(X0, max_iter=3000)
    assert r["status"] == 0 and r["report"]["converged"] == 1
    np.testing.assert_allclose(r["ev"], g["ev"], rtol=0, atol=EV_TOL)
    # the returned vectors are eigenvectors: H x = lambda x with the CPU oracle's H
    X = r["X"]
    HX = O.hamiltonian_apply(cell, X)
    res = np.sqrt(((HX - r["ev"][:, None] * X) ** 2).sum(axis=1) * cell.dV)
    assert res.max() < 1e-5
    G = X @ X.T * cell.dV
    assert np.abs(G - np.eye(len(X))).max() < 1e-6
    H.close()


def test_iteration_limit_reports_not_converged(cuda_ctx):
    from qumasun_b200 import Hamiltonian
    cell = build_cell(grid=(16, 16, 16))
    X0 = initial_states(4, cell.N, seed=3)
    H = Hamiltonian(cuda_ctx, cell)
    r = H.lobpcg(X0, max_iter=3)
    assert r["status"] == -9 and r["report"]["iterations"] == 3 and r["report"]["converged"] == 0
    # continuing from the returned X and P (not a first call) keeps improving the residual
    r2 = H.lobpcg(r["X"], max_iter=200, P0=r["P"], first=False)
    assert r2["report"]["max_residual"] < r["report"]["max_residual"]
    H.close()


def test_kinetic_preconditioner_same_eigenpairs_fewer_iterations(cuda_ctx):
    """The plain kinetic preconditioner (not in the reference) reaches the reference's
    eigenvalues in far fewer iterations."""
    from qumasun_b200 import Hamiltonian
    g = np.load(os.path.join(GOLD, "lobpcg_diamond8.npz"))
    cell = build_cell()
    X0 = initial_states(int(g["ns"]), cell.N, seed=int(g["seed"]))
    H = Hamiltonian(cuda_ctx, cell)
    r = H.lobpcg(X0, max_iter=3000, precond=1, shift=1.0)
    H.close()
    assert r["status"] == 0 and r["report"]["converged"] == 1
    np.testing.assert_allclose(r["ev"], g["ev"], rtol=0, atol=EV_TOL)
    assert r["report"]["iterations"] < int(g["iters"]) // 3


@pytest.mark.parametrize("precision", [2, 1], ids=["bf16x3", "fp32"])
def test_mixed_precision_gram_reaches_fp64_eigenvalues(cuda_ctx, precision):
    """Split-BF16x3 (QG_MIXED_BF16X3) or FP32 (QG_FP32) Gram products with the FP64
    residual and the final FP64 Rayleigh-Ritz: the same 16 eigenvalues as the
    reference solver to 1e-8 Ha on the 8-atom 40^3 cell."""
    import torch
    from qumasun_b200 import Hamiltonian
    g = np.load(os.path.join(GOLD, "lobpcg_diamond8.npz"))
    cell = build_cell()
    X0 = initial_states(int(g["ns"]), cell.N, seed=int(g["seed"]))
    H = Hamiltonian(cuda_ctx, cell)
    X = torch.from_numpy(X0).cuda()
    r = H.lobpcg_device(X, None, max_iter=400, precond=1, precision=precision)
    H.close()
    assert r["status"] == 0 and r["report"]["converged"] == 1
    assert r["report"]["mixed_iterations"] > 0
    np.testing.assert_allclose(np.sort(r["ev"]), np.sort(g["ev"]), rtol=0, atol=1e-8)


def test_cells_solved_together_match_one_by_one(cuda_ctx):
    """qg_lobpcg_cells_device: three cells of different grids (the 8-atom 40^3 cell of
    the reference fixture, a displaced 16-atom 80x40x40 cell and a small 24x20x16 cell),
    each on its own context and stream, solved concurrently, give the eigenvalues of
    solving them one by one, and the 8-atom cell the reference solver's."""
    import torch
    from qumasun_b200 import Context, Hamiltonian
    from qumasun_b200.engine import lobpcg_cells
    g = np.load(os.path.join(GOLD, "lobpcg_diamond8.npz"))
    cells = [build_cell(), build_cell(reps=(2, 1, 1), displacement=0.05, seed=7), build_cell(grid=(24, 20, 16))]
    ns = [int(g["ns"]), 34, 6]
    nconv = [int(g["ns"]), 32, 6]
    X0 = [initial_states(ns[0], cells[0].N, seed=int(g["seed"])), initial_states(ns[1], cells[1].N, seed=8),
          initial_states(ns[2], cells[2].N, seed=9)]
    ctxs = [Context(0) for _ in cells]
    hams = [Hamiltonian(c, cell) for c, cell in zip(ctxs, cells)]
    Xs = [torch.from_numpy(x).cuda() for x in X0]
    out, rc = lobpcg_cells(hams, Xs, max_iter=3000, precond=1, n_converge=nconv)
    assert rc == 0 and all(o["status"] == 0 and o["report"]["converged"] == 1 for o in out)
    for c in range(3):
        one = hams[c].lobpcg_device(torch.from_numpy(X0[c]).cuda(), None, max_iter=3000, precond=1,
                                    n_converge=nconv[c])
        np.testing.assert_allclose(out[c]["ev"][:nconv[c]], one["ev"][:nconv[c]], rtol=0, atol=1e-10)
    np.testing.assert_allclose(np.sort(out[0]["ev"]), g["ev"], rtol=0, atol=EV_TOL)
    with pytest.raises(AssertionError):
        lobpcg_cells([hams[0], hams[0]], [Xs[0], Xs[0]])  # one context per cell
    for h in hams:
        h.close()
    for c in ctxs:
        c.close()


def test_gram_reuse_reaches_the_full_gram_eigenpairs(cuda_ctx):
    """More than 128 Gram columns (64-atom 80^3 cell, 60 states, 48 judged): the steady-state
    pencil from the last rotation (direct update, full Gram every 10 iterations) reaches
    the eigenvalues of the full-Gram iteration to 1e-9 Ha, both converged."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(2, 2, 2), displacement=0.05, seed=11)
    X0 = initial_states(60, cell.N, seed=12)
    H = Hamiltonian(cuda_ctx, cell)
    out = {}
    for reuse in (True, False):
        H.set_gram_reuse(reuse)
        X = torch.from_numpy(X0).cuda()
        r = H.lobpcg_device(X, None, max_iter=400, precond=1, n_converge=48)
        assert r["status"] == 0 and r["report"]["converged"] == 1, (reuse, r["report"])
        out[reuse] = r
    d = np.abs(out[True]["ev"][:48] - out[False]["ev"][:48]).max()
    assert d < 1e-9, d
    it_r, it_f = out[True]["report"]["iterations"], out[False]["report"]["iterations"]
    assert it_r <= it_f + 10, (it_r, it_f)
    H.set_gram_reuse(True)
    H.close()


def test_nonfinite_start_reports_nonfinite(cuda_ctx):
    from qumasun_b200 import Hamiltonian, QGError
    cell = build_cell(grid=(16, 16, 16))
    X0 = initial_states(4, cell.N, seed=3)
    X0[2, 100] = np.nan
    H = Hamiltonian(cuda_ctx, cell)
    with pytest.raises(QGError) as e:
        H.lobpcg(X0, max_iter=50)
    assert e.value.status == -6  # QG_ERR_NONFINITE
    # the operator and context stay usable
    r = H.lobpcg(initial_states(4, cell.N, seed=3), max_iter=500)
    assert r["status"] == 0
    H.close()


def test_rank_deficient_start_reports_cholesky(cuda_ctx):
    """Every starting state the same vector: [x r p] spans one direction per block, fewer
    than ns independent directions remain in the pencil."""
    from qumasun_b200 import Hamiltonian, QGError
    cell = build_cell(grid=(16, 16, 16))
    X0 = np.repeat(initial_states(1, cell.N, seed=5), 4, axis=0)
    H = Hamiltonian(cuda_ctx, cell)
    with pytest.raises(QGError) as e:
        H.lobpcg(X0, max_iter=50)
    assert e.value.status == -4  # QG_ERR_CHOLESKY
    H.close()


def test_bounded_stencil_wait_reports_timeout_and_context_survives(cuda_ctx):
    """The test hook keeps the ring stencil's producer from issuing any copy: every consumer
    wait runs out (about 2^31 SM clocks), the kernel winds down and records
    QG_ERR_TIMEOUT; after the hook is cleared the same operator gives the oracle's H|psi>."""
    import torch
    from qumasun_b200 import Hamiltonian, lib
    cell = build_cell(grid=(24, 24, 24))
    X = initial_states(3, cell.N, seed=4)
    H = Hamiltonian(cuda_ctx, cell)
    Xd = torch.from_numpy(X).cuda()
    assert lib().qg_hamiltonian_test_stall(H.h, 1) == 0
    H.apply(Xd)
    torch.cuda.synchronize()
    assert cuda_ctx.take_device_status() == -5  # QG_ERR_TIMEOUT
    assert lib().qg_hamiltonian_test_stall(H.h, 0) == 0
    out = H.apply(Xd).cpu().numpy()
    ref = O.hamiltonian_apply(cell, X)
    assert (np.linalg.norm(out - ref, axis=1) / np.linalg.norm(ref, axis=1)).max() < 1e-12
    assert cuda_ctx.take_device_status() == 0
    H.close()


def test_config2_cell_mixed_precision_matches_fp64(cuda_ctx):
    """The mixed-precision configuration's cell (216 atoms, 120^3, sigma 0.05 bohr): 64
    states (the lowest 48 judged, a 16-state guard band), kinetic preconditioner, FP64
    against split-BF16x3 and FP32 Gram products -- the same 48 eigenvalues to 1e-8 Ha,
    all converged, the reduced precisions having run some iterations."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(3, 3, 3), displacement=0.05, seed=2024)
    gen = torch.Generator(device="cuda").manual_seed(7)
    X0 = torch.rand(64, cell.N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    H = Hamiltonian(cuda_ctx, cell)
    ev = {}
    for prec in (0, 2, 1):
        X = X0.clone()
        r = H.lobpcg_device(X, None, max_iter=300, precond=1, n_converge=48, precision=prec)
        assert r["status"] == 0 and r["report"]["converged"] == 1, (prec, r["report"])
        if prec:
            assert r["report"]["mixed_iterations"] > 0
        ev[prec] = r["ev"][:48]
        del X
    H.close()
    for prec in (2, 1):
        assert np.abs(ev[prec] - ev[0]).max() < 1e-8, (prec, np.abs(ev[prec] - ev[0]).max())


def test_config2_cell_int8_gram_matches_fp64(cuda_ctx):
    """QG_FP64_INT8 (Gram products as int8 slice products on the tensor cores, as
    accurate as DGEMM) on the config-2 cell, 64 states (48 judged): converges like the
    FP64 solve, to the same 48 eigenvalues within 1e-10 Ha."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(3, 3, 3), displacement=0.05, seed=2024)
    gen = torch.Generator(device="cuda").manual_seed(7)
    X0 = torch.rand(64, cell.N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    H = Hamiltonian(cuda_ctx, cell)
    ev, its = {}, {}
    for prec in (0, 3):
        X = X0.clone()
        r = H.lobpcg_device(X, None, max_iter=300, precond=1, n_converge=48, precision=prec)
        assert r["status"] == 0 and r["report"]["converged"] == 1, (prec, r["report"])
        ev[prec] = r["ev"][:48]
        its[prec] = r["report"]["iterations"]
        del X
    assert cuda_ctx.take_device_status() == 0
    H.close()
    assert np.abs(ev[3] - ev[0]).max() < 1e-10, np.abs(ev[3] - ev[0]).max()
    assert its[3] <= its[0] + 3, its
