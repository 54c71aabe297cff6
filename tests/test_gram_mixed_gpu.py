"""Split-BF16x3 Gram products (qg_gram_mixed_d) against FP64 DGEMM on the
device: the error per entry stays at the level the split representation and
the chunked FP32 accumulation allow (about 1e-6 of |a||b|)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,m", [(200_000, 96), (1_728_000, 64), (13_824 * 3 + 517, 40)])
def test_gram_mixed_matches_fp64(cuda_ctx, N, m):
    import torch
    from qumasun_b200.engine import lib
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.rand(m, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    B = torch.rand(m, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    A /= A.norm(dim=1, keepdim=True)
    B /= B.norm(dim=1, keepdim=True)
    C64 = torch.empty(m, m, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    for Bt in (B, A):
        rc = lib().qg_gram_mixed_d(cuda_ctx.h, N, m, C.c_void_p(A.data_ptr()), C.c_void_p(Bt.data_ptr()), 1.0,
                                   C.c_void_p(C64.data_ptr()))
        assert rc == 0
        ref = (A @ Bt.T).T  # column-major C(i, j) = a_i . b_j is C64[j, i] in row-major torch
        err = (C64 - ref).abs().max().item()
        print(N, m, "max abs error", err)
        assert err < 1e-5
