"""Randomized range finder and SVD built on the SHGEMM sketch (shgemm_b200.randnla):
subspace and singular values of a decaying-spectrum matrix against an FP64 SVD."""
import pytest

pytestmark = pytest.mark.gpu


def _lowrank(m, k, seed):
    import torch

    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    r = 60
    U = torch.linalg.qr(torch.randn(m, r, device="cuda", generator=g, dtype=torch.float64))[0]
    V = torch.linalg.qr(torch.randn(k, r, device="cuda", generator=g, dtype=torch.float64))[0]
    sig = torch.arange(1, r + 1, device="cuda", dtype=torch.float64).pow(-2.0)
    A64 = (U * sig) @ V.T + 1e-7 * torch.randn(m, k, device="cuda", generator=g, dtype=torch.float64)
    lda = (m + 3) // 4 * 4
    Abuf = torch.zeros(k, lda, device="cuda", dtype=torch.float32)  # column-major m x k
    Abuf[:, :m] = A64.T.float()
    return A64, Abuf.reshape(-1), lda


@pytest.mark.parametrize("tc", [0, 1])
def test_rsvd_matches_fp64_svd(cuda_device, tc):
    import torch

    import shgemm_b200 as sg
    from shgemm_b200 import randnla

    m, k, rank = 3000, 2000, 12
    A64, A, lda = _lowrank(m, k, seed=3 + tc)
    h = sg.Handle(0)
    try:
        U, S, V = randnla.rsvd(h, A, m, k, lda, rank, oversample=10, power_iters=1, compute_type=tc)
        Q = randnla.range_finder(h, A, m, k, lda, rank, oversample=10, power_iters=0, compute_type=tc, seed=5)
        torch.cuda.synchronize()
        assert h.check_error() == 0
    finally:
        h.close()
    s_true = torch.linalg.svdvals(A64)
    rel = ((S.double() - s_true[:rank]).abs() / s_true[:rank]).max().item()
    assert rel < 5e-3, rel
    # the rank-12 reconstruction is as good as the best rank-12 approximation (Eckart-Young)
    A32 = A64.float()
    err = torch.linalg.norm(A32 - (U * S) @ V.T).item()
    best = s_true[rank:].pow(2).sum().sqrt().item()
    assert err <= 1.5 * best + 1e-5 * torch.linalg.norm(A32).item(), (err, best)
    # Q captures the range: || A - Q Q^T A || close to the tail beyond l = rank + oversample
    resid = torch.linalg.norm(A32 - Q @ (Q.T @ A32)).item()
    assert resid <= 5 * s_true[rank + 10 - 2:].pow(2).sum().sqrt().item() + 1e-5 * torch.linalg.norm(A32).item()
    assert torch.allclose(Q.T @ Q, torch.eye(Q.shape[1], device="cuda"), atol=1e-4)
