"""GPU: factors that keep their diagonal inverses, and the matvec sweeps on them
(extension ops SOCU_OP_FACTOR_INV / *_INV; factor reuse over many right-hand sides)."""
import numpy as np
import pytest
import torch

from oracle import generators, nd_cholesky as nd
from socu_b200.block_tridiag_solver import (
    create_cholesky_backward_substitution_launch,
    create_cholesky_factor_and_solve_launch,
    create_cholesky_factor_launch,
    create_cholesky_forward_substitution_launch,
    create_cholesky_solve_launch,
)

pytestmark = pytest.mark.gpu
DEV = "cuda"
TOL = {torch.float32: 1e-4, torch.float64: 1e-10}


@pytest.mark.parametrize("N,n,m", [(1, 1, 1), (7, 10, 2), (100, 32, 1), (20, 64, 8), (33, 17, 40)])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("graph", [False, True])
def test_factor_once_solve_many(N, n, m, dtype, graph):
    L0, E0, b0 = generators.readme_problem(N, n, m, shift=10.0, seed=N + n)
    L, E = (torch.tensor(a, dtype=dtype, device=DEV) for a in (L0, E0))
    Lp, Ep = L.clone(), E.clone()
    create_cholesky_factor_launch(L, E, dtype=dtype, use_cuda_graph=graph, keep_inverse=True)()
    create_cholesky_factor_launch(Lp, Ep, dtype=dtype, use_cuda_graph=graph)()
    torch.cuda.synchronize()
    # the factor itself is the plain factor (lower triangles, all of E), bit for bit
    assert torch.equal(torch.tril(L), torch.tril(Lp)) and torch.equal(E, Ep)
    x_ref = nd.nd_factor_and_solve(L0, E0, b0)[2][0]
    scale = max(1.0, float(np.abs(x_ref).max()))
    x = torch.tensor(b0, dtype=dtype, device=DEV)
    run = create_cholesky_solve_launch(L, E, x, dtype=dtype, use_cuda_graph=graph, factor_has_inverse=True)
    for rep in range(3):   # the same factor, several right-hand sides
        x.copy_(torch.tensor(b0 * (rep + 1), dtype=dtype, device=DEV))
        run()
        torch.cuda.synchronize()
        err = np.abs(x.double().cpu().numpy() - (rep + 1) * x_ref).max()
        assert err <= TOL[dtype] * (rep + 1) * scale, (rep, err)
    # forward then backward on the inverse-carrying factor == solve
    y = torch.tensor(b0, dtype=dtype, device=DEV)
    create_cholesky_forward_substitution_launch(L, E, y, dtype=dtype, factor_has_inverse=True)()
    create_cholesky_backward_substitution_launch(L, E, y, dtype=dtype, factor_has_inverse=True)()
    torch.cuda.synchronize()
    assert np.abs(y.double().cpu().numpy() - x_ref).max() <= TOL[dtype] * scale


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_factor_and_solve_factor_carries_inverse(dtype):
    N, n, m = 40, 24, 3
    L0, E0, b0 = generators.readme_problem(N, n, m, shift=10.0, seed=3)
    L, E, x = (torch.tensor(a, dtype=dtype, device=DEV) for a in (L0, E0, b0))
    create_cholesky_factor_and_solve_launch(L, E, x, dtype=dtype)()
    x2 = torch.tensor(b0, dtype=dtype, device=DEV)
    create_cholesky_solve_launch(L, E, x2, dtype=dtype, factor_has_inverse=True)()
    torch.cuda.synchronize()
    scale = max(1.0, float(x.abs().max()))
    assert float((x - x2).abs().max()) <= TOL[dtype] * scale


def test_inverse_ops_reject_large_blocks():
    N, n = 4, 68
    L = torch.eye(n, dtype=torch.float64, device=DEV).repeat(N, 1, 1)
    E = torch.zeros(N, n, n, dtype=torch.float64, device=DEV)
    with pytest.raises(RuntimeError, match="unsupported"):
        create_cholesky_factor_launch(L, E, keep_inverse=True)


def _wide_batch(B=8, N=128, n=32, m=4):
    probs = [generators.readme_problem(N, n, m, shift=10.0, seed=50 + k) for k in range(B)]
    return tuple(np.stack([p[j] for p in probs]) for j in range(3))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("graph", [False, True])
def test_inverse_sweeps_on_launches_wider_than_resident(dtype, graph):
    """8 instances of N = 128: the level-0 sweep launches have 512 CTAs, more
    than three per SM on a 148-SM B200, where the FP32 sweeps switch from the
    SIMT products to the FP64 tensor-core ones (narrower levels keep SIMT);
    every path must agree with the oracle."""
    L0, E0, b0 = _wide_batch()
    x_ref = nd.nd_factor_and_solve(L0, E0, b0)[2]
    scale = max(1.0, float(np.abs(x_ref).max()))
    L, E, x = (torch.tensor(a, dtype=dtype, device=DEV) for a in (L0, E0, b0))
    create_cholesky_factor_and_solve_launch(L, E, x, dtype=dtype, use_cuda_graph=graph)()
    torch.cuda.synchronize()
    assert np.abs(x.double().cpu().numpy() - x_ref).max() <= TOL[dtype] * scale
    # forward + backward sweeps on the inverse-carrying factor, all levels
    x2 = torch.tensor(b0, dtype=dtype, device=DEV)
    create_cholesky_solve_launch(L, E, x2, dtype=dtype, use_cuda_graph=graph, factor_has_inverse=True)()
    torch.cuda.synchronize()
    assert np.abs(x2.double().cpu().numpy() - x_ref).max() <= TOL[dtype] * scale


def test_refined_solve_on_launches_wider_than_resident():
    """The mixed solve's float sweeps on the same wide batch: FP64 backward error."""
    from socu_b200.mixed import create_cholesky_refined_solve_launch
    L0, E0, b0 = _wide_batch()
    L, E, b = (torch.tensor(a, device=DEV) for a in (L0, E0, b0))
    x = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, x, tol=1e-12)
    run()
    torch.cuda.synchronize()
    assert float(run.eta.max()) <= 1e-12, run.eta
    eta = nd.backward_error(L0, E0, x.cpu().numpy(), b0)
    assert float(np.max(eta)) <= 1e-12
