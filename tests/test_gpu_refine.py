"""GPU: mixed-precision factor + FP64 refinement and the FP64 residual kernel."""
import numpy as np
import pytest
import torch

from oracle import generators, nd_cholesky as nd
from socu_b200.mixed import backward_error, block_tridiag_residual, create_cholesky_refined_solve_launch

pytestmark = pytest.mark.gpu
DEV = "cuda"


def t(a):
    return torch.tensor(a, dtype=torch.float64, device=DEV)


@pytest.mark.parametrize("N,n,m", [(1, 8, 1), (7, 10, 2), (64, 32, 4), (100, 36, 1), (33, 64, 8), (9, 128, 3),
                                   (20, 13, 11), (5, 64, 17), (3, 1, 9), (2, 7, 8)])
def test_residual_matches_oracle(N, n, m):
    L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=N + n)
    x = np.random.default_rng(1).standard_normal(b.shape)
    r = block_tridiag_residual(t(L), t(E), t(x), t(b)).cpu().numpy()
    ref = b - nd.block_tridiag_matmul(L, E, x)[0]
    assert np.abs(r - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())
    eta = backward_error(t(L), t(E), t(x), t(b)).cpu().numpy()
    assert np.allclose(eta, nd.backward_error(L, E, x, b), rtol=1e-10)


@pytest.mark.parametrize("N,n,m,B", [(100, 32, 1, 1), (64, 16, 4, 3), (37, 64, 8, 2), (1, 12, 2, 2), (20, 68, 1, 1)])
@pytest.mark.parametrize("graph", [False, True])
def test_refined_solve_reaches_fp64_backward_error(N, n, m, B, graph):
    L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=5)
    Lb, Eb, bb = (np.tile(a, (B, 1, 1, 1)) for a in (L, E, b))
    Lt, Et, bt = t(Lb), t(Eb), t(bb)
    x = torch.full_like(bt, float("nan"))
    run = create_cholesky_refined_solve_launch(Lt, Et, bt, x, tol=1e-12, max_iter=10, use_cuda_graph=graph)
    run()
    torch.cuda.synchronize()
    eta = run.eta.cpu().numpy()
    it = run.iterations.cpu().numpy()
    assert (eta <= 1e-12).all(), (eta, it)
    assert (it >= 1).all() and (it <= 10).all()
    _, _, x_ref = nd.nd_factor_and_solve(L, E, b)
    xs = x.cpu().numpy()
    # forward error is bounded by cond(Psi) times the backward error
    kappa = np.linalg.cond(generators.dense_from_blocks(L, E))
    for k in range(B):
        err = np.abs(xs[k] - x_ref[0]).max() / max(1e-300, np.abs(x_ref).max())
        assert err <= 20 * kappa * 1e-12 + 1e-14, (err, kappa)
    # inputs untouched
    assert torch.equal(Lt, t(Lb)) and torch.equal(Et, t(Eb)) and torch.equal(bt, t(bb))
    # oracle backward error of the result
    assert nd.backward_error(L, E, xs[0], b)[0] <= 1e-12


def test_refined_solve_mask_and_rerun():
    N, n, m, B = 50, 24, 2, 4
    L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=9)
    Lt, Et, bt = (t(np.tile(a, (B, 1, 1, 1))) for a in (L, E, b))
    x = torch.full_like(bt, 7.0)
    mask = torch.tensor([True, False, True, False], device=DEV)
    run = create_cholesky_refined_solve_launch(Lt, Et, bt, x, mask=mask)
    run()
    torch.cuda.synchronize()
    assert (x[1] == 7.0).all() and (x[3] == 7.0).all()
    assert (run.eta[[0, 2]] <= 1e-12).all()
    mask.copy_(torch.tensor([False, True, False, True]))
    x.fill_(3.0)
    run()   # the mask is read at run time, also under the captured graph
    torch.cuda.synchronize()
    assert (x[0] == 3.0).all() and (x[2] == 3.0).all()
    assert (run.eta[[1, 3]] <= 1e-12).all()


def test_refined_solve_reports_breakdown_without_crashing():
    # shift 0.1: tril(randn) + 0.1 I blocks are numerically singular, Psi is
    # numerically indefinite and no Cholesky can factor it
    N, n, m = 16, 64, 1
    L, E, b = generators.readme_problem(N, n, m, shift=0.1, seed=0)
    x = torch.zeros_like(t(b))
    run = create_cholesky_refined_solve_launch(t(L), t(E), t(b), x, tol=1e-12, max_iter=5)
    run()
    torch.cuda.synchronize()
    eta = float(run.eta[0])
    it = int(run.iterations[0])
    assert it < 0 or not (eta <= 1e-12)
