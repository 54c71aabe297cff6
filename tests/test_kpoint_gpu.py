"""Complex k-point H|psi> on the B200 against the reference's golden fixture
(PseudoPotIntegrator_kpoint::ProjectionPP + LaplasianKpoint8th, run through
oracle/_ref) and the CPU oracle. Tolerance: FP64 1e-12 relative per state
(norm-wise) for the whole operator, and 1e-10 for the nonlocal part alone
relative to its own size (it is ~4e-4 of the total on random states, so the
subtraction of the local part costs about four digits)."""
import os

import numpy as np
import pytest

import oracle as O
from qumasun_b200.cell import build_cell, initial_states

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-12
KPOINT_CASES = {"noncubic": dict(grid=(20, 16, 24), displacement=0.05, seed=3),
                "wrap": dict(grid=(12, 12, 12), a0=4.4)}


def rel_per_state(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def gpu_apply_z(ctx, cell, X, g, plain=False):
    import torch
    from qumasun_b200 import Hamiltonian
    H = Hamiltonian(ctx, cell, kvec=tuple(g))
    H.set_stencil_kernel(plain)
    Xd = torch.from_numpy(np.ascontiguousarray(X)).to("cuda", torch.float64)
    out = H.apply_z(Xd)
    torch.cuda.synchronize()
    H.close()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def gold():
    return np.load(os.path.join(GOLD, "ham_kpoint.npz"))


@pytest.mark.parametrize("plain", [False, True], ids=["tma", "plain"])
@pytest.mark.parametrize("name", sorted(KPOINT_CASES))
def test_kpoint_matches_reference_golden(cuda_ctx, gold, name, plain):
    cell = build_cell(**KPOINT_CASES[name])
    X = gold[f"{name}_X"]
    for i, g in enumerate(gold[f"{name}_g"]):
        ref = gold[f"{name}_HX{i}"]
        HX = gpu_apply_z(cuda_ctx, cell, X, g, plain)
        assert rel_per_state(HX, ref).max() < TOL64, (name, i)
        loc = O.hamiltonian_kpoint_local(cell, tuple(g), X)
        assert rel_per_state(HX - loc, ref - loc).max() < 1e-10, (name, i)


@pytest.mark.parametrize("plain", [False, True], ids=["tma", "plain"])
@pytest.mark.parametrize("order", [2, 6])
@pytest.mark.parametrize("name", sorted(KPOINT_CASES))
def test_kpoint_fd_orders_2_6_match_reference_golden(cuda_ctx, gold, name, order, plain):
    """FD orders 2 and 6 of the k-point operator (LaplasianKpoint2nd / 6th of the
    reference, KINETIC_2ND / KINETIC_6TH in qumasun_kpoint.matrix.h) at the general
    k-vector, both stencil kernels."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(**KPOINT_CASES[name])
    X = gold[f"{name}_X"]
    g = gold[f"{name}_g"][2]
    H = Hamiltonian(cuda_ctx, cell, fd_order=order, kvec=tuple(g))
    H.set_stencil_kernel(plain)
    HX = H.apply_z(torch.from_numpy(np.ascontiguousarray(X)).cuda()).cpu().numpy()
    H.close()
    assert rel_per_state(HX, gold[f"{name}_HX2_o{order}"]).max() < TOL64


def test_kpoint_diamond8_general_k_and_kvector_switch(cuda_ctx):
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell()  # 8 atoms, 40^3
    X = initial_states(6, 2 * cell.N, seed=31)
    g1 = (0.233, -0.466, 0.116)
    g2 = (0.0, 0.233, 0.0)  # two components below the 1e-8 skip threshold
    H = Hamiltonian(cuda_ctx, cell, kvec=g1)
    Xd = torch.from_numpy(X).cuda()
    a = H.apply_z(Xd).cpu().numpy()
    H.set_kvector(g2)
    b = H.apply_z(Xd).cpu().numpy()
    hb = H.apply_host_z(X)
    H.close()
    assert rel_per_state(a, O.hamiltonian_kpoint_apply(cell, g1, X)).max() < TOL64
    assert rel_per_state(b, O.hamiltonian_kpoint_apply(cell, g2, X)).max() < TOL64
    np.testing.assert_array_equal(hb, b)


def test_kpoint_gamma_equals_real_operator(cuda_ctx):
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(grid=(24, 20, 16), displacement=0.1, seed=2)
    N = cell.N
    X = initial_states(3, 2 * N, seed=4)
    H = Hamiltonian(cuda_ctx, cell)
    z = H.apply_z(torch.from_numpy(X).cuda()).cpu().numpy()
    r = H.apply(torch.from_numpy(X.reshape(6, N)).cuda()).cpu().numpy().reshape(3, 2 * N)
    H.close()
    assert rel_per_state(z, r).max() < 1e-14


def test_kpoint_operator_is_hermitian_on_device(cuda_ctx):
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell()
    N = cell.N
    X = initial_states(2, 2 * N, seed=5)
    H = Hamiltonian(cuda_ctx, cell, kvec=(0.3, 0.2, -0.1))
    HX = H.apply_z(torch.from_numpy(X).cuda()).cpu().numpy()
    H.close()
    z = X[:, :N] + 1j * X[:, N:]
    hz = HX[:, :N] + 1j * HX[:, N:]
    a = np.vdot(z[0], hz[1])
    b = np.conj(np.vdot(z[1], hz[0]))
    assert abs(a - b) < 1e-12 * abs(a)


def test_kpoint_invalid_arguments(cuda_ctx):
    import ctypes as C
    import torch
    from qumasun_b200 import Hamiltonian
    from qumasun_b200.engine import lib
    cell = build_cell(grid=(16, 16, 16))
    H = Hamiltonian(cuda_ctx, cell, kvec=(0.1, 0.0, 0.0))
    X = torch.zeros((2, 2 * cell.N), dtype=torch.float64, device="cuda")
    Y = torch.empty_like(X)
    assert lib().qg_hamiltonian_apply_z(H.h, 2, C.c_void_p(X.data_ptr()), cell.N, C.c_void_p(Y.data_ptr()),
                                        2 * cell.N) == -1
    # the real entry point refuses a nonzero Bloch vector
    assert lib().qg_hamiltonian_apply_d(H.h, 2, C.c_void_p(X.data_ptr()), cell.N, C.c_void_p(Y.data_ptr()),
                                        cell.N) == -1
    H.close()
    # the reference has no 4th-order k-point stencil: QG_ERR_UNSUPPORTED
    H4 = Hamiltonian(cuda_ctx, cell, fd_order=4, kvec=(0.1, 0.0, 0.0))
    assert lib().qg_hamiltonian_apply_z(H4.h, 2, C.c_void_p(X.data_ptr()), 2 * cell.N, C.c_void_p(Y.data_ptr()),
                                        2 * cell.N) == -7
    H4.close()


@pytest.mark.parametrize("plain", [False, True], ids=["tma", "plain"])
def test_multi_kpoint_apply_in_one_pass(cuda_ctx, plain):
    """qg_hamiltonian_apply_zk over 5 Monkhorst-Pack k-points x 3 states equals the
    single-k operator applied k-point by k-point, and the oracle."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(grid=(24, 20, 16), displacement=0.05, seed=3)
    N = cell.N
    b = 2 * np.pi / (cell.nx * cell.hx)
    kv = np.array([[0.125, 0.375, -0.125], [0.0, 0.0, 0.0], [-0.375, 0.125, 0.375], [0.25, 0.25, 0.25],
                   [0.5, -0.5, 0.0]]) * b
    X = initial_states(15, 2 * N, seed=41).reshape(5, 3, 2 * N)
    H = Hamiltonian(cuda_ctx, cell)
    H.set_stencil_kernel(plain)
    Xd = torch.from_numpy(X).cuda()
    many = H.apply_zk(kv, Xd).cpu().numpy()
    for k in range(5):
        H.set_kvector(kv[k])
        one = H.apply_z(Xd[k]).cpu().numpy()
        np.testing.assert_array_equal(many[k], one)
        ref = O.hamiltonian_kpoint_apply(cell, tuple(kv[k]), X[k])
        assert rel_per_state(many[k], ref).max() < TOL64
    H.close()


@pytest.mark.parametrize("plain", [False, True], ids=["tma", "plain"])
def test_complex64_states_match_oracle(cuda_ctx, plain):
    """Complex64 Bloch states (FP32 split complex) on the 8-atom 40^3 cell and a
    non-cubic cell: within 2e-6 relative per state of the FP64 oracle; the multi-k
    FP32 apply equals the single-k FP32 apply bit for bit."""
    import torch
    from qumasun_b200 import Hamiltonian
    for cell, g in ((build_cell(), (0.233, -0.466, 0.116)),
                    (build_cell(grid=(24, 20, 16), displacement=0.05, seed=3), (0.1, 0.0, -0.3))):
        X = initial_states(6, 2 * cell.N, seed=51)
        H = Hamiltonian(cuda_ctx, cell, kvec=g)
        H.set_stencil_kernel(plain)
        out = H.apply_z(torch.from_numpy(X.astype(np.float32)).cuda()).double().cpu().numpy()
        ref = O.hamiltonian_kpoint_apply(cell, g, X)
        assert rel_per_state(out, ref).max() < 2e-6
        kv = np.array([g, (0.0, 0.0, 0.0), (-0.2, 0.15, 0.05)])
        Xk = torch.from_numpy(np.stack([X] * 3).astype(np.float32)).cuda()
        many = H.apply_zk(kv, Xk).cpu().numpy()
        for k in range(3):
            H.set_kvector(kv[k])
            np.testing.assert_array_equal(many[k], H.apply_z(Xk[k]).cpu().numpy())
        H.close()
