"""GPU: gradients of the differentiable solve against dense autograd and
central finite differences (the config-3 check: batch 256, N=128, n=16, m=1,
loss sum(w * x), 64 random directions, h=1e-6, rel. err <= 1e-8)."""
import numpy as np
import pytest
import torch

from oracle import generators
from socu_b200.autograd import block_tridiag_solve

pytestmark = pytest.mark.gpu
DEV = "cuda"


def dense_psi(D, E):
    """Psi from lower(D_i) and E_i = Psi_{i+1,i} with differentiable torch ops."""
    B, N, n = D.shape[:3]
    Dl = torch.tril(D)
    Dsym = Dl + torch.tril(D, -1).transpose(-1, -2)
    A = torch.zeros(B, N * n, N * n, dtype=D.dtype, device=D.device)
    rows = []
    for i in range(N):
        blocks = []
        for j in range(N):
            if i == j:
                blocks.append(Dsym[:, i])
            elif i == j + 1:
                blocks.append(E[:, j])
            elif j == i + 1:
                blocks.append(E[:, i].transpose(-1, -2))
            else:
                blocks.append(torch.zeros(B, n, n, dtype=D.dtype, device=D.device))
        rows.append(torch.cat(blocks, dim=-1))
    return torch.cat(rows, dim=-2)


def problem(B, N, n, m, seed):
    Ls, Es, bs = [], [], []
    for k in range(B):
        L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=seed + k, storage=False)
        Ls.append(L); Es.append(E); bs.append(b)
    t = lambda a: torch.tensor(np.stack(a), dtype=torch.float64, device=DEV)
    return t(Ls), t(Es), t(bs)


@pytest.mark.parametrize("B,N,n,m", [(2, 5, 4, 2), (1, 9, 10, 1), (3, 4, 17, 3), (1, 1, 6, 2)])
def test_gradients_match_dense_autograd(B, N, n, m):
    D, E, b = problem(B, N, n, m, seed=3)
    # give the upper triangles of D junk: only the lower triangle may matter
    D = D + torch.triu(torch.full_like(D, 0.3), 1)
    w = torch.randn(B, N, n, m, dtype=torch.float64, device=DEV)
    D1, E1, b1 = (a.clone().requires_grad_(True) for a in (D, E, b))
    x = block_tridiag_solve(D1, E1, b1)
    (w * x).sum().backward()
    D2, E2, b2 = (a.clone().requires_grad_(True) for a in (D, E, b))
    psi = dense_psi(D2, E2)
    x2 = torch.linalg.solve(psi, b2.reshape(B, N * n, m)).reshape(B, N, n, m)
    (w * x2).sum().backward()
    assert torch.allclose(x, x2, rtol=1e-10, atol=1e-12)
    for g1, g2 in ((D1.grad, D2.grad), (E1.grad, E2.grad), (b1.grad, b2.grad)):
        if g2 is None:   # N = 1: no off-diagonal blocks
            assert g1.numel() == 0
            continue
        scale = float(g2.abs().max())
        assert float((g1 - g2).abs().max()) <= 1e-8 * scale
    assert float(torch.triu(D1.grad, 1).abs().max()) == 0.0


@pytest.mark.parametrize("h,bar", [(1e-6, 1e-7), (1e-5, 1e-8)])
def test_gradients_central_differences_config3(h, bar):
    # h = 1e-6 sits at the round-off floor of central differences for these
    # systems (forward error of each solve ~ cond * eps, divided by 2h ~ 1e-8);
    # h = 1e-5 keeps truncation negligible and meets 1e-8.
    B, N, n, m = 256, 128, 16, 1
    D, E, b = problem(B, N, n, m, seed=100)
    w = torch.randn(B, N, n, m, dtype=torch.float64, device=DEV, generator=torch.Generator(DEV).manual_seed(0))
    D1, E1, b1 = (a.clone().requires_grad_(True) for a in (D, E, b))
    (w * block_tridiag_solve(D1, E1, b1)).sum().backward()
    solve = lambda Dp, Ep, bp: block_tridiag_solve(Dp, Ep, bp)
    gen = torch.Generator(DEV).manual_seed(1)
    worst = 0.0
    for _ in range(64):
        VD = torch.tril(torch.randn(D.shape, dtype=torch.float64, device=DEV, generator=gen))
        VE = torch.randn(E.shape, dtype=torch.float64, device=DEV, generator=gen)
        Vb = torch.randn(b.shape, dtype=torch.float64, device=DEV, generator=gen)
        # difference the solutions first, then weight: avoids cancelling two large sums
        dx = solve(D + h * VD, E + h * VE, b + h * Vb) - solve(D - h * VD, E - h * VE, b - h * Vb)
        fd = float((w * dx).sum()) / (2 * h)
        an = float((D1.grad * VD).sum() + (E1.grad * VE).sum() + (b1.grad * Vb).sum())
        worst = max(worst, abs(fd - an) / max(abs(an), 1e-300))
    assert worst <= bar, worst
