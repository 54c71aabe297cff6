"""Split-BF16 Gram products (qg_gram_mixed_d) against FP64 DGEMM on the device.
pieces = 3 and 2 run the library's tcgen05 kernel (FP32 accumulation over one
64-row K block, FP64 across blocks); pieces = 0 the cuBLAS BF16 hi/lo path with
1024-row FP32 chunks. Bounds (max abs error on unit-norm columns): products of
unrelated columns (A^T B) 5e-8 with 3 pieces; norm-like entries (A^T A, same-sign
sums) carry the tensor cores' FP32 accumulation drift, ~7 ulp of the K block's
partial sum, so 2e-6 with 3 pieces; 2 pieces (a_lo b_lo dropped, ~2^-18 on
norm-like entries) and the cuBLAS path 1e-5; pieces = -1 (FP32 copies, FP32 GEMMs over
1024-row chunks, the Gram of QG_FP32) 1e-6; pieces = 7 (the int8 slice products of
QG_FP64_INT8, exact int32 sums) 1e-13, DGEMM's level."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
BOUND = {3: (5e-8, 2e-6), 2: (1e-5, 1e-5), 0: (1e-5, 1e-5), -1: (1e-6, 1e-6), 7: (1e-13, 1e-13)}


def run_gram(ctx, A, B, pieces):
    import torch
    from qumasun_b200.engine import lib
    m, N = A.shape
    C64 = torch.zeros(m, m, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    rc = lib().qg_gram_mixed_d(ctx.h, N, m, C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), 1.0,
                               C.c_void_p(C64.data_ptr()), pieces)
    assert rc == 0
    return C64


@pytest.mark.parametrize("pieces", [3, 2, 0, -1, 7])
@pytest.mark.parametrize("N,m", [(64_000, 300), (200_000, 96), (1_728_000, 64)])
def test_gram_mixed_matches_fp64(cuda_ctx, N, m, pieces):
    import torch
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.rand(m, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    B = torch.rand(m, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    A /= A.norm(dim=1, keepdim=True)
    B /= B.norm(dim=1, keepdim=True)
    for case, Bt in enumerate((B, A)):
        C64 = run_gram(cuda_ctx, A, Bt, pieces)
        ref = (A @ Bt.T).T  # column-major C(i, j) = a_i . b_j is C64[j, i] in row-major torch
        err = (C64 - ref).abs().max().item()
        print(N, m, pieces, "max abs error", err)
        assert err < BOUND[pieces][case]


def test_gram_cublas_path_takes_any_row_count(cuda_ctx):
    import torch
    N, m = 13_824 * 3 + 517, 40
    g = torch.Generator(device="cuda").manual_seed(9)
    A = torch.rand(m, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    A /= A.norm(dim=1, keepdim=True)
    C64 = run_gram(cuda_ctx, A, A, 0)
    assert (C64 - A @ A.T).abs().max().item() < 1e-5
