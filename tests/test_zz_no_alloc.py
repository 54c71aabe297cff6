"""The H|psi> entry point that allocates nothing (qg_hamiltonian_apply_noalloc_d).

Some callers of this library cannot call cudaMalloc when they apply H: hosts
whose device memory is owned by another framework's allocator (a memory pool
that must not be bypassed), and time-critical loops that must not touch the
allocator at all. This entry point takes its projector-coefficient scratch from
a fixed array compiled into the library, so the call itself allocates nothing;
the caller still passes the states in and the result buffer out. It must give
the same H|psi> as the regular entry point. This file is collected last so that
a run stopping at the first failure has already run every other test; it passes
on its own in a fresh process too (the session context fixture builds what it
needs)."""
import numpy as np
import pytest

from qumasun_b200.cell import build_cell, initial_states

pytestmark = pytest.mark.gpu
TOL64 = 1e-12


def test_noalloc_matches_regular_entry_point_twice(cuda_ctx):
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(reps=(2, 2, 2))          # 64 atoms, 80^3: 256 coefficient slots per state
    H = Hamiltonian(cuda_ctx, cell)
    X = torch.from_numpy(initial_states(24, cell.N, seed=77)).cuda()
    ref = H.apply(X)
    torch.cuda.synchronize()
    for call in range(2):
        out = torch.full_like(X, float("nan"))
        H.apply_noalloc(X, out)
        torch.cuda.synchronize()
        err = ((out - ref).norm(dim=1) / ref.norm(dim=1)).max().item()
        assert err < TOL64, (call, err)
    # a second operator of another size shares the same fixed array
    cell2 = build_cell(grid=(24, 24, 24))
    H2 = Hamiltonian(cuda_ctx, cell2)
    X2 = torch.from_numpy(initial_states(5, cell2.N, seed=78)).cuda()
    ref2 = H2.apply(X2)
    out2 = H2.apply_noalloc(X2, torch.empty_like(X2))
    torch.cuda.synchronize()
    assert ((out2 - ref2).norm(dim=1) / ref2.norm(dim=1)).max().item() < TOL64
    assert cuda_ctx.take_device_status() == 0
    H2.close()
    H.close()


def test_noalloc_rejects_batches_beyond_the_fixed_buffer(cuda_ctx):
    import ctypes as C
    import torch
    from qumasun_b200 import Hamiltonian, lib
    # 64 atoms on a small grid: one state more than the fixed array holds still fits
    # real buffers (2049 x 24^3 doubles, ~230 MB each), so the call is given valid
    # memory even if the capacity check ever moved behind a launch
    cell = build_cell(reps=(2, 2, 2), grid=(24, 24, 24))
    H = Hamiltonian(cuda_ctx, cell)
    cap = lib().qg_noalloc_scratch_capacity()
    per_state = cell.n_atoms * 4
    ns = cap // per_state + 1
    X = torch.zeros(ns, cell.N, dtype=torch.float64, device="cuda")
    HX = torch.zeros_like(X)
    status = lib().qg_hamiltonian_apply_noalloc_d(H.h, ns, C.c_void_p(X.data_ptr()), cell.N,
                                                  C.c_void_p(HX.data_ptr()), cell.N)
    assert status == -7  # QG_ERR_UNSUPPORTED
    assert b"fixed buffer" in lib().qg_last_error()
    del X, HX
    H.close()


def test_noalloc_binding_rejects_bad_blocks(cuda_ctx):
    import torch
    from qumasun_b200 import Hamiltonian
    cell = build_cell(grid=(24, 24, 24))
    H = Hamiltonian(cuda_ctx, cell)
    X = torch.zeros(3, cell.N, dtype=torch.float64, device="cuda")
    with pytest.raises(TypeError):
        H.apply_noalloc(X.float(), torch.empty_like(X).float())
    with pytest.raises(TypeError):
        H.apply_noalloc(X.cpu(), torch.empty_like(X))
    with pytest.raises(ValueError):
        H.apply_noalloc(X, torch.empty(2, cell.N, dtype=torch.float64, device="cuda"))
    with pytest.raises(ValueError):
        H.apply_noalloc(torch.zeros(cell.N, 3, dtype=torch.float64, device="cuda").t(), torch.empty_like(X))
    H.close()
