"""The header-only C++ adapter (include/qumasun_b200_adapter.hpp) at the reference's own
call sites, through oracle/_ref/libadapter_check.so (oracle/adapter_check.cpp):

* flatten_projectors() reads PseudoPotIntegrator_single's cube tables, as the reference's
  UpdatePosition tabulates them from a radial table (PseudoPotOperator.h:453-727), into
  the engine's descriptor without changing a value (CPU);
* the GPU operator built from those tables applies the reference's H (V psi,
  ProjectionPP, Laplasian8th) to 1e-12 relative per state (GPU);
* EigenLOBPCG_d_multi(..., OpeA, watch) -- the call of qumasun_single.lobpcg.h:17-23 --
  with the adapter's GpuOperator in place of the lambda reaches the reference solver's
  eigenvalues to 1e-8 Ha (GPU).
Skipped where the checker library was not built (it needs the reference tree)."""
import numpy as np
import pytest

import oracle as O
from qumasun_b200.cell import PROJ_SIGMA, build_cell, initial_states

needs_adapter = pytest.mark.skipif(not O.adapter_available(), reason="oracle/_ref/libadapter_check.so not built")


@needs_adapter
def test_flatten_reads_the_reference_cubes():
    cell = build_cell(grid=(20, 16, 24), displacement=0.05, seed=2)
    code, cubes, sums = O.adapter_flatten_stats(cell, PROJ_SIGMA)
    assert code == cell.n_atoms * 1000000 + 2 * 1000 + 4   # 8 atoms, 2 projectors, 4 lm
    assert sums[0] == sums[1] and sums[2] == sums[3] and sums[0] != 0.0
    # every cube is the reference's GridForSphere of its atom
    import ctypes as C
    lib = O.ref_lib()
    for a in range(cell.n_atoms):
        R = cell.positions[a]
        c6 = (C.c_int * 6)()
        lib.ref_grid_for_sphere(R[0], R[1], R[2], cell.cutoff, cell.hx, cell.hy, cell.hz, c6)
        want = [c6[0], c6[1], c6[2], c6[3] - c6[0], c6[4] - c6[1], c6[5] - c6[2]]
        for k in range(2):
            assert list(cubes[a * 2 + k]) == want


@needs_adapter
@pytest.mark.gpu
def test_adapter_operator_applies_the_reference_h(cuda_ctx):
    cell = build_cell(grid=(20, 16, 24), displacement=0.05, seed=2)
    X = initial_states(4, cell.N, seed=9)
    hg, hr = O.adapter_apply(cell, PROJ_SIGMA, X)
    err = np.linalg.norm(hg - hr, axis=1) / np.linalg.norm(hr, axis=1)
    assert err.max() < 1e-12, err


@needs_adapter
@pytest.mark.gpu
def test_adapter_lobpcg_call_site_reaches_reference_eigenvalues(cuda_ctx):
    cell = build_cell(grid=(16, 16, 16))
    X0 = initial_states(8, cell.N, seed=21)
    er, eg, it = O.adapter_lobpcg(cell, PROJ_SIGMA, X0, 2000)
    assert it < 2000
    assert np.abs(np.sort(eg) - np.sort(er)).max() < 1e-8, (er, eg)
