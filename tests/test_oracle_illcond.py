"""The oracle on ill-conditioned diagonal factor blocks (CPU only).

The generator (oracle.generators.illcond_problem) must give factor blocks
with the requested condition number at every level and a matrix that FP64
dense Cholesky (the reference tests' oracle) still factors.  The FP64 oracle
is then checked against the long-double restatement (oracle.extended): its
factor error must stay within the first-order bound kappa^2 * u of any FP64
Cholesky-based method, and its solution must be backward stable.
"""
import numpy as np
import pytest
import scipy.linalg as la

from oracle import extended, generators, nd_cholesky as nd

U64 = 2.0 ** -53


@pytest.mark.parametrize("kappa", [1e4, 1e6, 1e8])
def test_generator_gives_requested_block_conditioning(kappa):
    N, n = 12, 16
    L, E, b = generators.illcond_problem(N, n, 2, kappa=kappa, seed=3)
    la.cholesky(generators.dense_from_blocks(L, E), lower=True)   # SPD in FP64
    Lt, _, _ = extended.nd_factor_and_solve(L, E, b)
    conds = [np.linalg.cond(Lt[i].astype(np.float64)) for i in range(N)]
    assert 0.3 * kappa <= min(conds) and max(conds) <= 3.0 * kappa


@pytest.mark.parametrize("kappa", [1e4, 1e6, 1e8])
def test_fp64_oracle_against_long_double_truth(kappa):
    N, n, m = 20, 16, 2
    L, E, b = generators.illcond_problem(N, n, m, kappa=kappa, seed=5)
    Lt, Et, xt = extended.nd_factor_and_solve(L, E, b)
    Lo, Eo, xo = nd.nd_factor_and_solve(L, E, b)
    bound = 50.0 * n * kappa ** 2 * U64
    assert extended.rel_error(np.tril(Lo[0]), Lt) <= bound
    assert extended.rel_error(Eo[0], Et) <= bound
    assert nd.backward_error(L, E, xo[0], b)[0] <= 1e-15


def test_long_double_truth_matches_oracle_on_well_conditioned_input():
    N, n, m = 17, 5, 2
    L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=1)
    Lt, Et, xt = extended.nd_factor_and_solve(L, E, b)
    Lo, Eo, xo = nd.nd_factor_and_solve(L, E, b)
    assert extended.rel_error(np.tril(Lo[0]), Lt) <= 1e-14
    assert extended.rel_error(Eo[0][:N - 1], Et[:N - 1]) <= 1e-14
    assert extended.rel_error(xo[0], xt) <= 1e-13
