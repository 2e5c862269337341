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
