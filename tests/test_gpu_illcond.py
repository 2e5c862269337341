"""FP64 factor and solves on ill-conditioned diagonal factor blocks (needs a B200).

For blocks n <= 64 the FP64 node kernel forms the explicit inverse
W_i = C_i^{-1} of each diagonal factor block and applies it by matrix products
(F = R W^T, G = W Lf, y = W y, and x = W^T x in the backward sweep of
factor_and_solve), where the reference runs triangular solves
(socu/blas/trsm.py:95-120, 203-228, 315-340).  An explicit inverse can lose
accuracy as kappa(C_i) grows, which well-conditioned test problems cannot show.

These cases use oracle.generators.illcond_problem, whose factor blocks have
kappa(C_i) ~ 1e4, 1e6, 1e8 at every level while Psi stays positive definite in
FP64.  Every FP64 method then carries factor errors of order kappa^2 * 1e-16
(at kappa 1e8 that is the whole factor), so two FP64 results are not compared
with each other at a fixed 1e-10; each is compared with the long-double
restatement (oracle.extended) instead:
  * factor blocks (lower(L), every E slot): GPU error <= 10 x the error of the
    FP64 oracle, which uses the reference's triangular solves;
  * solutions of factor_and_solve, factor + solve and the inverse-carrying
    factor + solve: normwise backward error <= 1e-15 (the reference's
    algorithm gives ~2e-17 here) and forward error <= 10 x the FP64 oracle's.
"""
import functools

import numpy as np
import pytest
import torch

from oracle import extended, generators, nd_cholesky as nd
from socu_b200.block_tridiag_solver import (create_cholesky_factor_and_solve_launch, create_cholesky_factor_launch,
                                            create_cholesky_solve_launch)

pytestmark = pytest.mark.gpu
DEV = "cuda"
CASES = [(kappa, N, n) for kappa in (1e4, 1e6, 1e8) for (N, n) in ((20, 32), (100, 64))]


@functools.lru_cache(maxsize=None)
def problem(kappa, N, n, m=3):
    L, E, b = generators.illcond_problem(N, n, m, kappa=kappa, seed=int(np.log10(kappa)) + N)
    truth = extended.nd_factor_and_solve(L, E, b)
    Lo, Eo, xo = nd.nd_factor_and_solve(L, E, b)
    return L, E, b, truth, (np.tril(Lo[0]), Eo[0], xo[0])


def t(a):
    return torch.tensor(a, dtype=torch.float64, device=DEV)


@pytest.mark.parametrize("kappa,N,n", CASES)
def test_factor_blocks_as_accurate_as_triangular_solves(kappa, N, n):
    L, E, _, (Lt, Et, _), (Lo, Eo, _) = problem(kappa, N, n)
    Lg, Eg = t(L), t(E)
    create_cholesky_factor_launch(Lg, Eg)()
    Lgpu, Egpu = np.tril(Lg.cpu().numpy()), Eg.cpu().numpy()
    for got, ora, tru in ((Lgpu, Lo, Lt), (Egpu, Eo, Et)):
        e_gpu, e_ora = extended.rel_error(got, tru), extended.rel_error(ora, tru)
        assert e_gpu <= 10.0 * e_ora + 1e-15, (e_gpu, e_ora)


@pytest.mark.parametrize("kappa,N,n", CASES)
@pytest.mark.parametrize("sequence", ["factor_and_solve", "factor+solve", "factor(keep_inverse)+solve"])
def test_solutions_backward_stable(kappa, N, n, sequence):
    L, E, b, (_, _, xt), (_, _, xo) = problem(kappa, N, n)
    Lg, Eg, xg = t(L), t(E), t(b)
    if sequence == "factor_and_solve":
        create_cholesky_factor_and_solve_launch(Lg, Eg, xg)()
    elif sequence == "factor+solve":
        create_cholesky_factor_launch(Lg, Eg)()
        create_cholesky_solve_launch(Lg, Eg, xg)()
    else:
        create_cholesky_factor_launch(Lg, Eg, keep_inverse=True)()
        create_cholesky_solve_launch(Lg, Eg, xg, factor_has_inverse=True)()
    x = xg.cpu().numpy()
    eta = float(nd.backward_error(L, E, x, b)[0])
    assert eta <= 1e-15, eta
    f_gpu, f_ora = extended.rel_error(x, xt), extended.rel_error(xo, xt)
    assert f_gpu <= 10.0 * f_ora + 1e-15, (f_gpu, f_ora)
