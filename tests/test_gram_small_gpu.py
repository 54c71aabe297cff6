"""The tall-skinny Gram kernel of the real LOBPCG's small pencils (qg_gram_small_d:
K split over the GPU, partial sums in a fixed order) against torch's FP64 matmul:
1e-13 relative to the largest entry, any column counts (tiles of 64), ragged row
counts, and the same bits on repeated calls."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def gram_small(ctx, A, B, alpha=1.0):
    import torch
    from qumasun_b200.engine import check, lib
    ma, N = A.shape
    mb = B.shape[0]
    Cm = torch.empty(mb, ma, dtype=torch.float64, device="cuda")  # column-major ma x mb
    torch.cuda.synchronize()
    check(lib().qg_gram_small_d(ctx.h, N, ma, mb, C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), alpha,
                                C.c_void_p(Cm.data_ptr())), "qg_gram_small_d")
    return Cm.T  # (ma, mb)


@pytest.mark.parametrize("N,ma,mb", [(64_000, 48, 48), (1000, 7, 5), (200_003, 64, 30), (77_777, 96, 128)])
def test_gram_small_matches_fp64_matmul(cuda_ctx, N, ma, mb):
    import torch
    g = torch.Generator(device="cuda").manual_seed(N + ma)
    A = torch.rand(ma, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    B = torch.rand(mb, N, dtype=torch.float64, device="cuda", generator=g) - 0.5
    got = gram_small(cuda_ctx, A, B, 0.25)
    ref = 0.25 * (A @ B.T)
    assert (got - ref).abs().max().item() <= 1e-13 * ref.abs().max().item() * 10
    again = gram_small(cuda_ctx, A, B, 0.25)
    assert torch.equal(got, again)
