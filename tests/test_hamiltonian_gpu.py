"""H|psi> on the B200 against the CPU oracle (port pinned to the reference)
and the reference's golden fixtures. Tolerances: FP64 1e-12 relative per state
(norm-wise), FP32 2e-6 relative per state against the FP64 oracle."""
import os

import numpy as np
import pytest

import oracle as O
from qumasun_b200.cell import build_cell, initial_states

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL64 = 1e-12
TOL32 = 2e-6


def rel_per_state(a, b):
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


def gpu_apply(ctx, cell, X, order=None, dtype="f64"):
    import torch
    from qumasun_b200 import Hamiltonian
    H = Hamiltonian(ctx, cell, fd_order=order)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    Xd = torch.from_numpy(np.ascontiguousarray(X)).to("cuda", tdt)
    out = H.apply(Xd)
    torch.cuda.synchronize()
    H.close()
    return out.double().cpu().numpy()


@pytest.mark.parametrize("name,kw", [("noncubic", dict(grid=(20, 16, 24))),
                                     ("wrap", dict(grid=(12, 12, 12), a0=4.4))])
@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_fp64_matches_reference_golden(cuda_ctx, name, kw, order):
    g = np.load(os.path.join(GOLD, f"ham_{name}.npz"))
    cell = build_cell(**kw)
    HX = gpu_apply(cuda_ctx, cell, g["X"], order)
    assert rel_per_state(HX, g[f"HX{order}"]).max() < TOL64


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_fp64_and_fp32_match_oracle_diamond8(cuda_ctx, order):
    cell = build_cell()  # 8 atoms, 40^3
    X = initial_states(16, cell.N, seed=21)
    ref = O.hamiltonian_apply(cell, X, fd_order=order)
    assert rel_per_state(gpu_apply(cuda_ctx, cell, X, order), ref).max() < TOL64
    assert rel_per_state(gpu_apply(cuda_ctx, cell, X.astype(np.float32), order, "f32"), ref).max() < TOL32


@pytest.mark.parametrize("kw", [dict(), dict(grid=(12, 12, 12), a0=4.4)], ids=["diamond8", "wrap"])
def test_nonlocal_blocking_gives_identical_results(cuda_ctx, kw):
    """Every projection / scatter state blocking (and the register-window kernel,
    which reads the same channel-major coefficients) gives the same bits for a given
    split of each atom's points over a thread-block cluster; every split (1-8 blocks
    per atom) matches the oracle. The wrap cell has points inside up to 10 projector
    spheres, past the scatter's register cache of entries."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(**kw)
    X = initial_states(21, cell.N, seed=17)  # ragged against every state group
    ref = O.hamiltonian_apply(cell, X)
    H = Hamiltonian(cuda_ctx, cell)
    for dt in (torch.float64, torch.float32):
        Xd = torch.from_numpy(X).to("cuda", dt)
        tol = TOL64 if dt == torch.float64 else TOL32
        for parts in (1, 3, 8):
            H.set_nonlocal_blocking(0, 0, parts)
            base = H.apply(Xd).cpu().numpy()
            assert rel_per_state(base, ref).max() < tol
            for sb in (1, 2, 4, 8, 16):
                for sg in (4, 8):
                    H.set_nonlocal_blocking(sb, sg, parts)
                    np.testing.assert_array_equal(H.apply(Xd).cpu().numpy(), base)
            H.set_nonlocal_blocking(0, 0, parts)
            H.set_stencil_kernel(True)
            plain = H.apply(Xd).cpu().numpy()
            H.set_stencil_kernel(False)
            assert rel_per_state(plain, ref).max() < tol
        H.set_nonlocal_blocking(0, 0, 0)
    for bad in ((3, 0, 0), (0, 16, 0), (0, 0, 9), (0, 0, -1)):
        with pytest.raises(Exception):
            H.set_nonlocal_blocking(*bad)
    H.close()


def test_projection_split_does_not_depend_on_the_batch(cuda_ctx):
    """The engine's split of the projection depends on the cell only: a state gives
    the same bits applied alone, in a batch of 5 and in a batch of 40."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell()
    X = torch.from_numpy(initial_states(40, cell.N, seed=23)).cuda()
    H = Hamiltonian(cuda_ctx, cell)
    full = H.apply(X).cpu().numpy()
    five = H.apply(X[:5].contiguous()).cpu().numpy()
    one = H.apply(X[:1].contiguous()).cpu().numpy()
    H.close()
    np.testing.assert_array_equal(five, full[:5])
    np.testing.assert_array_equal(one, full[:1])


def test_displaced_cell_no_nonlocal_and_no_potential(cuda_ctx):
    for kw in [dict(grid=(24, 20, 16), displacement=0.3, seed=5),
               dict(grid=(16, 16, 16), nonlocal_on=False),
               dict(grid=(16, 24, 16), potential_on=False)]:
        cell = build_cell(**kw)
        X = initial_states(5, cell.N, seed=8)
        ref = O.hamiltonian_apply(cell, X)
        assert rel_per_state(gpu_apply(cuda_ctx, cell, X), ref).max() < TOL64


def test_strided_states_and_empty_batch(cuda_ctx):
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(grid=(16, 16, 16))
    N = cell.N
    X = initial_states(3, N, seed=4)
    ld = N + 40
    Xp = torch.zeros(3, ld, dtype=torch.float64, device="cuda")
    Xp[:, :N] = torch.from_numpy(X).cuda()
    HXp = torch.full((3, ld), 7.0, dtype=torch.float64, device="cuda")
    H = Hamiltonian(cuda_ctx, cell)
    H.apply_device(3, Xp.data_ptr(), HXp.data_ptr(), ldx=ld, ldhx=ld)
    H.apply_device(0, Xp.data_ptr(), HXp.data_ptr())  # no-op
    torch.cuda.synchronize()
    out = HXp.cpu().numpy()
    assert np.all(out[:, N:] == 7.0)  # padding untouched
    assert rel_per_state(out[:, :N], O.hamiltonian_apply(cell, X)).max() < TOL64
    H.close()


@pytest.mark.parametrize("ns", [1, 4, 13])
def test_host_entry_point_matches_device(cuda_ctx, ns):
    """The host-buffer entry point copies in, applies and copies out in chunks of
    states on separate streams; ragged last chunks included, it equals the device
    apply bit for bit."""
    from qumasun_b200 import Hamiltonian
    cell = build_cell(grid=(20, 20, 20))
    X = initial_states(ns, cell.N, seed=6)
    H = Hamiltonian(cuda_ctx, cell)
    HXh = H.apply_host(X)
    H.close()
    np.testing.assert_array_equal(HXh, gpu_apply(cuda_ctx, cell, X))
    assert rel_per_state(HXh, O.hamiltonian_apply(cell, X)).max() < TOL64


def test_invalid_arguments_are_rejected(cuda_ctx):
    from qumasun_b200 import Hamiltonian, QGError
    cell = build_cell(grid=(16, 16, 16))
    with pytest.raises(QGError):
        Hamiltonian(cuda_ctx, cell, fd_order=5)
    H = Hamiltonian(cuda_ctx, cell)
    with pytest.raises(QGError):
        H.apply_device(2, 0, 0)
    with pytest.raises(QGError):
        H.apply_device(1, 16, 16, ldx=10)
    H.close()


def test_diamond64_full_batch_properties(cuda_ctx):
    """64 atoms, 80^3, 256 states (the benchmark's workload): every state against the
    oracle (FP64 1e-12 per state; FP32 against the oracle too), and the size-independent
    properties of the whole batch (symmetry of H, linearity)."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(2, 2, 2))
    ns = 256
    H = Hamiltonian(cuda_ctx, cell)
    gen = torch.Generator(device="cuda").manual_seed(0)
    X = torch.rand(ns, cell.N, dtype=torch.float64, device="cuda", generator=gen) - 0.5
    HX = H.apply(X)
    torch.cuda.synchronize()
    ref = O.hamiltonian_apply(cell, X.cpu().numpy())
    assert rel_per_state(HX.cpu().numpy(), ref).max() < TOL64
    G = (X @ HX.T) * cell.dV            # <x_i|H|x_j>
    asym = (G - G.T).abs().max().item() / G.abs().max().item()
    assert asym < 1e-12
    a, b = 0.3, -1.7
    Y = torch.roll(X, 1, 0)
    lin = H.apply(a * X + b * Y) - (a * HX + b * H.apply(Y))
    assert (lin.norm(dim=1) / HX.norm(dim=1)).max().item() < 1e-12
    Xf = X.float()
    HXf = H.apply(Xf)
    torch.cuda.synchronize()
    assert ((HXf.double() - HX).norm(dim=1) / HX.norm(dim=1)).max().item() < TOL32
    refF = O.hamiltonian_apply(cell, Xf.double().cpu().numpy())
    assert rel_per_state(HXf.double().cpu().numpy(), refF).max() < TOL32
    H.close()


@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_config1_sweep_fp32_against_oracle(cuda_ctx, order):
    """The benchmark's FD-order sweep cell (64 atoms, 80^3) in FP32 against the FP64 oracle
    at every order (FP32 tolerance), 16 states."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(2, 2, 2))
    X = initial_states(16, cell.N, seed=40 + order).astype(np.float32)
    ref = O.hamiltonian_apply(cell, X.astype(np.float64), fd_order=order)
    H = Hamiltonian(cuda_ctx, cell, fd_order=order)
    out = H.apply(torch.from_numpy(X).cuda()).double().cpu().numpy()
    assert rel_per_state(out, ref).max() < TOL32
    H.close()


def test_diamond216_sampled_states(cuda_ctx):
    """216 atoms, 120^3, displaced: a few states against the oracle."""
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(3, 3, 3), displacement=0.05, seed=0)
    X = initial_states(3, cell.N, seed=31)
    ref = O.hamiltonian_apply(cell, X)
    assert rel_per_state(gpu_apply(cuda_ctx, cell, X), ref).max() < TOL64


@pytest.mark.parametrize("grid", [(20, 16, 24), (12, 12, 12), (40, 40, 40)])
@pytest.mark.parametrize("order", [2, 4, 6, 8])
def test_every_stencil_kernel_agrees_with_oracle(cuda_ctx, grid, order):
    """Two-plane, two-row and one-plane TMA-ring kernels and the register-window kernel,
    FP64 and FP32, several tile/wrap shapes (odd and even plane counts per slab); the
    ring kernels give the same bits."""
    import torch
    from qumasun_b200 import Hamiltonian
    kw = dict(grid=grid, a0=4.4) if grid == (12, 12, 12) else dict(grid=grid)
    cell = build_cell(**kw)
    X = initial_states(5, cell.N, seed=12)
    ref = O.hamiltonian_apply(cell, X, fd_order=order)
    H = Hamiltonian(cuda_ctx, cell, fd_order=order)
    ring = {}
    for variant in (0, 1, 2, 3, 4, 5):
        H.set_stencil_kernel(variant)
        for dt, tol in ((torch.float64, TOL64), (torch.float32, TOL32)):
            out = H.apply(torch.from_numpy(X).to("cuda", dt))
            torch.cuda.synchronize()
            got = out.double().cpu().numpy()
            err = rel_per_state(got, ref).max()
            assert err < tol, (variant, dt, err)
            if variant >= 2:
                ring.setdefault(dt, []).append(got)
    for outs in ring.values():
        for o in outs[1:]:
            np.testing.assert_array_equal(o, outs[0])
    assert cuda_ctx.take_device_status() == 0
    H.close()


def test_autotuner_keeps_the_bits(cuda_ctx):
    """The autotuner only picks among launch shapes with identical results: H|psi> after
    tuning equals H|psi> before it, bit for bit, FP64 and FP32, and the choice is one of
    the candidates."""
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(2, 1, 1), displacement=0.05, seed=5)
    X = torch.from_numpy(initial_states(24, cell.N, seed=6)).cuda()
    H = Hamiltonian(cuda_ctx, cell)
    for Xd in (X, X.float()):
        before = H.apply(Xd).cpu().numpy()
        ch = H.autotune(Xd)
        assert ch["stencil"] in (2, 3, 4, 5) and ch["project_states"] in (2, 4, 8, 16)
        assert ch["scatter_states"] in (4, 8) and all(v > 0 for v in ch["ms_phases"])
        np.testing.assert_array_equal(H.apply(Xd).cpu().numpy(), before)
    assert cuda_ctx.take_device_status() == 0
    H.close()
