"""GPU: the large stress shape (N=16384, n=128, m=32; ~7 GB of FP64 blocks).

At the README construction's shift 0.05 the diagonal factor blocks are
numerically singular, so the system is indefinite and no Cholesky factors it;
there the solver must report the breakdown (non-finite eta, iterations < 0)
instead of returning a wrong answer.  With n = 128 the coupling blocks
(||E_chol|| ~ 2 sqrt(n)) also outgrow a shift of 10 along long horizons (the
oracle's FP64 Cholesky fails at N = 64 already); from shift 16 on the shape is
positive definite, and at shift 24 both paths must reach the FP64
backward-error bound.
"""
import pytest
import torch

from socu_b200.block_tridiag_solver import create_cholesky_factor_and_solve_launch
from socu_b200.mixed import backward_error, create_cholesky_refined_solve_launch
from socu_b200.problems import readme_blocks

pytestmark = pytest.mark.gpu
N, n, m = 16384, 128, 32


def test_stress_shape_well_conditioned():
    L, E, b = readme_blocks(N, n, m, shift=24.0, seed=4, device="cuda")
    x = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, x, tol=1e-12, max_iter=10)
    run()
    torch.cuda.synchronize()
    assert float(run.eta.max()) <= 1e-12 and int(run.iterations.min()) >= 1
    assert float(backward_error(L, E, x, b).max()) <= 1e-12
    Lw, Ew, xw = L.clone(), E.clone(), b.clone()
    create_cholesky_factor_and_solve_launch(Lw, Ew, xw)()
    torch.cuda.synchronize()
    del Lw, Ew
    assert float(backward_error(L, E, xw, b).max()) <= 1e-13
    assert float((x - xw).abs().max()) <= 1e-6 * float(xw.abs().max())


def test_stress_shape_indefinite_is_reported():
    L, E, b = readme_blocks(N, n, m, shift=0.05, seed=4, device="cuda")
    x = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, x, tol=1e-12, max_iter=10)
    run()
    torch.cuda.synchronize()
    eta, it = float(run.eta.max()), int(run.iterations.min())
    # either the float factor broke down (reported) or refinement could not reach the bound
    assert it < 0 or not eta <= 1e-12, (eta, it)
