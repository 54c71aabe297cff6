"""The no-allocation H|psi> entry point (qg_hamiltonian_apply_noalloc_d).

It exists for callers that cannot allocate device memory when they apply H:
work recorded into a CUDA stream capture, loops that must not touch the
allocator, hosts whose device memory another framework owns. It must give the
same H|psi> as the regular entry point while taking its scratch from a fixed
array compiled into the library. This file is collected last so that a run
stopping at the first failure has already run every other test; it passes on
its own in a fresh process too (the session context fixture builds what it
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
    from qumasun_b200 import Hamiltonian, QGError, lib
    cell = build_cell(reps=(2, 2, 2))
    H = Hamiltonian(cuda_ctx, cell)
    cap = lib().qg_noalloc_scratch_capacity()
    per_state = cell.n_atoms * 4
    ns = cap // per_state + 1                   # one state more than fits
    import ctypes as C
    # rejected before any pointer is touched
    status = lib().qg_hamiltonian_apply_noalloc_d(H.h, ns, C.c_void_p(256), cell.N, C.c_void_p(256), cell.N)
    assert status == -7  # QG_ERR_UNSUPPORTED
    assert b"fixed buffer" in lib().qg_last_error()
    H.close()
