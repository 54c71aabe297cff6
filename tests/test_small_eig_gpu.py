"""The library's batched small generalised eigensolvers (qg_sygv_small_batched_d,
qg_hegv_small_batched_z) against LAPACK (scipy.linalg.eigh, the same ITYPE 1 problems
DSYGVX / ZHEGVX solve): eigenvalues, residuals and B-orthonormality to 1e-8."""
import numpy as np
import pytest
import scipy.linalg as sl

pytestmark = pytest.mark.gpu


def spd_pencil(k, rng, cond=1e6):
    M = rng.standard_normal((k, k))
    A = (M + M.T) / 2
    U, _ = np.linalg.qr(rng.standard_normal((k, k)))
    s = np.logspace(0, -np.log10(cond), k)
    B = (U * s) @ U.T
    scale = rng.uniform(1e-3, 1e3, k)           # badly scaled rows/columns, like tiny residual blocks
    S = np.outer(scale, scale)
    # the scaled pencil has the same eigenvalues as the unscaled one (a congruence)
    return A * S, B * S, sl.eigh(A, B, eigvals_only=True)


@pytest.mark.parametrize("k", [1, 7, 47, 48, 80])
def test_matches_lapack(cuda_ctx, k):
    import torch
    from qumasun_b200.engine import sygv_small_batched
    rng = np.random.default_rng(k)
    As, Bs, Ws = zip(*[spd_pencil(k, rng) for _ in range(5)])
    A = torch.tensor(np.array(As)).cuda()
    B = torch.tensor(np.array(Bs)).cuda()
    w, Z, info = sygv_small_batched(cuda_ctx, A, B)
    torch.cuda.synchronize()
    assert (info == 0).all()
    w, Z = w.cpu().numpy(), Z.cpu().numpy()
    for b in range(5):
        wr = Ws[b]
        assert np.abs(w[b] - wr).max() <= 1e-8 * max(1.0, np.abs(wr).max())
        # residual and B-orthonormality of the returned vectors
        R = As[b] @ Z[b] - Bs[b] @ Z[b] * w[b]
        assert np.linalg.norm(R) <= 1e-8 * np.linalg.norm(As[b]) * np.linalg.norm(Z[b])
        G = Z[b].T @ Bs[b] @ Z[b]
        assert np.abs(G - np.eye(k)).max() < 1e-8


def test_indefinite_b_is_reported(cuda_ctx):
    import torch
    from qumasun_b200.engine import sygv_small_batched
    k = 12
    A = torch.eye(k, dtype=torch.float64).unsqueeze(0).cuda()
    B = torch.eye(k, dtype=torch.float64)
    B[3, 3] = -1.0
    w, Z, info = sygv_small_batched(cuda_ctx, A, B.unsqueeze(0).cuda())
    assert info[0] == 1


def hpd_pencil(k, rng, cond=1e6):
    M = rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k))
    A = (M + M.conj().T) / 2
    U, _ = np.linalg.qr(rng.standard_normal((k, k)) + 1j * rng.standard_normal((k, k)))
    s = np.logspace(0, -np.log10(cond), k)
    B = (U * s) @ U.conj().T
    B = (B + B.conj().T) / 2
    scale = rng.uniform(1e-3, 1e3, k)
    S = np.outer(scale, scale)
    return A * S, B * S, sl.eigh(A, B, eigvals_only=True)


@pytest.mark.parametrize("k", [1, 6, 32, 48, 56])
def test_hermitian_matches_lapack(cuda_ctx, k):
    import torch
    from qumasun_b200.engine import hegv_small_batched
    rng = np.random.default_rng(100 + k)
    As, Bs, Ws = zip(*[hpd_pencil(k, rng) for _ in range(4)])
    A = torch.tensor(np.array(As)).cuda()
    B = torch.tensor(np.array(Bs)).cuda()
    w, Z, info = hegv_small_batched(cuda_ctx, A, B)
    torch.cuda.synchronize()
    assert (info == 0).all()
    w, Z = w.cpu().numpy(), Z.cpu().numpy()
    for b in range(4):
        wr = Ws[b]
        assert np.abs(w[b] - wr).max() <= 1e-8 * max(1.0, np.abs(wr).max())
        R = As[b] @ Z[b] - Bs[b] @ Z[b] * w[b]
        assert np.linalg.norm(R) <= 1e-8 * np.linalg.norm(As[b]) * np.linalg.norm(Z[b])
        G = Z[b].conj().T @ Bs[b] @ Z[b]
        assert np.abs(G - np.eye(k)).max() < 1e-8


def test_hermitian_indefinite_b_and_size_limit(cuda_ctx):
    import torch
    from qumasun_b200.engine import hegv_small_batched
    k = 10
    A = torch.eye(k, dtype=torch.complex128).unsqueeze(0).cuda()
    B = torch.eye(k, dtype=torch.complex128)
    B[4, 4] = -2.0
    _, _, info = hegv_small_batched(cuda_ctx, A, B.unsqueeze(0).cuda())
    assert info[0] == 1
    big = torch.eye(57, dtype=torch.complex128).unsqueeze(0).cuda()
    with pytest.raises(Exception):
        hegv_small_batched(cuda_ctx, big, big)
