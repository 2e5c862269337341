"""GPU: the mixed solve's FP64 fallback (graph-captured; IF node after the refinement loop)."""
import numpy as np
import pytest
import torch

from oracle import nd_cholesky as nd
from oracle.nd_cholesky import off_diag_storage_len
from socu_b200.block_tridiag_solver import create_cholesky_factor_and_solve_launch
from socu_b200.mixed import create_cholesky_refined_solve_launch

pytestmark = pytest.mark.gpu
DEV = "cuda"


def _problem(N, n, m, seed, tiny=None):
    """README construction Psi = C C^T; with `tiny`, the last diagonal entry of
    the first diagonal factor block is `tiny`: the float Cholesky then loses
    that pivot to rounding, FP64 still resolves it."""
    rng = np.random.default_rng(seed)
    Dc = np.tril(rng.standard_normal((N, n, n))) + 10.0 * np.eye(n)
    if tiny is not None:
        Dc[0, n - 1, n - 1] = tiny
    Ec = rng.standard_normal((N - 1, n, n))
    L = Dc @ np.swapaxes(Dc, -1, -2)
    L[1:] += Ec @ np.swapaxes(Ec, -1, -2)
    E = np.zeros((off_diag_storage_len(N), n, n))
    E[:N - 1] = Ec @ np.swapaxes(Dc[:N - 1], -1, -2)
    b = rng.standard_normal((N, n, m))
    return L, E, b


def _batch(probs):
    return (torch.tensor(np.stack([p[k] for p in probs]), device=DEV) for k in range(3))


def test_fallback_solves_the_instance_the_float_factor_cannot():
    N, n, m = 40, 32, 2
    probs = [_problem(N, n, m, 1), _problem(N, n, m, 2, tiny=1e-5), _problem(N, n, m, 3)]
    L, E, b = _batch(probs)
    L0, E0, b0 = L.clone(), E.clone(), b.clone()
    x = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, x, tol=1e-12, max_iter=8, fp64_fallback=True)
    # without the fallback the middle instance does not reach the bound
    x_plain_mixed = torch.zeros_like(b)
    run_nf = create_cholesky_refined_solve_launch(L, E, b, x_plain_mixed, tol=1e-12, max_iter=8)
    for _ in range(2):   # twice: the IF stage and its flag must reset between runs
        run()
        run_nf()
        torch.cuda.synchronize()
        assert run.used_fp64.tolist() == [0, 1, 0]
        assert float(run.eta.max()) <= 1e-12, run.eta
        assert not float(run_nf.eta[1]) <= 1e-12
    # inputs untouched
    assert torch.equal(L, L0) and torch.equal(E, E0) and torch.equal(b, b0)
    # the good instances are the refined solution, the bad one the plain FP64 solution
    assert torch.equal(x[0], x_plain_mixed[0]) and torch.equal(x[2], x_plain_mixed[2])
    Lw, Ew, xw = L[1:2].clone(), E[1:2].clone(), b[1:2].clone()
    create_cholesky_factor_and_solve_launch(Lw, Ew, xw)()
    torch.cuda.synchronize()
    scale = float(xw.abs().max())
    assert float((x[1] - xw[0]).abs().max()) <= 1e-12 * scale
    # and the oracle agrees on its backward error
    assert nd.backward_error(probs[1][0], probs[1][1], x[1].cpu().numpy(), probs[1][2])[0] <= 1e-12


def test_fallback_idle_on_well_conditioned_batch_and_respects_mask():
    N, n, m = 64, 24, 3
    probs = [_problem(N, n, m, 10 + k) for k in range(4)]
    L, E, b = _batch(probs)
    mask = torch.tensor([True, False, True, True], device=DEV)
    x = torch.full_like(b, 7.0)
    run = create_cholesky_refined_solve_launch(L, E, b, x, mask=mask, tol=1e-12, fp64_fallback=True)
    x_ref = torch.full_like(b, 7.0)
    ref = create_cholesky_refined_solve_launch(L, E, b, x_ref, mask=mask, tol=1e-12)
    run(); ref()
    torch.cuda.synchronize()
    assert run.used_fp64.tolist() == [0, 0, 0, 0]
    assert torch.equal(x, x_ref)
    assert torch.equal(x[1], torch.full_like(x[1], 7.0))   # masked-off instance untouched
    assert float(run.eta[mask].max()) <= 1e-12


def test_fallback_needs_the_graph():
    L, E, b = _batch([_problem(8, 4, 1, 0)])
    with pytest.raises(ValueError, match="use_cuda_graph"):
        create_cholesky_refined_solve_launch(L, E, b, torch.zeros_like(b), use_cuda_graph=False, fp64_fallback=True)
