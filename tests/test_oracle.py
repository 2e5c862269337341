"""The oracle against the reference tests' known answers (CPU only).

Pins the NumPy restatement (oracle/nd_cholesky.py) against
  * SciPy dense Cholesky on the reference test generator at the reference
    tolerance 1e-10 (tests/test_block_tridiag_solver.py:9-12, 82-130 of socu),
  * the committed golden fixtures (tests/golden/*.npz), including the exact
    in-place (L, E[storage_len]) factor layout.
"""
import glob
import os

import numpy as np
import pytest

from oracle import dense, generators, nd_cholesky as nd

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
TOL = 1e-10


def test_storage_len_matches_reference_examples():
    # values quoted for the configs and edge cases
    assert nd.off_diag_storage_len(1) == 0
    assert nd.off_diag_storage_len(2) == 1
    assert nd.off_diag_storage_len(100) == 190
    assert nd.off_diag_storage_len(1024) == 2036
    assert nd.off_diag_storage_len(128) == 247
    assert nd.off_diag_storage_len(16384) == 32752
    assert nd.recursive_iterations(1) == 1 and nd.recursive_iterations(1024) == 11


def test_every_node_eliminated_once():
    for N in [1, 2, 3, 7, 8, 20, 100, 257]:
        seen = sorted(int(i) for *_, nodes in nd.level_schedule(N) for i in nodes)
        assert seen == list(range(N))


@pytest.mark.parametrize("N", [1, 2, 3, 4, 7, 8, 20, 100])
@pytest.mark.parametrize("n", [1, 10, 32, 36])
def test_oracle_matches_dense_on_reference_grid(n, N):
    if n * N > 2000:
        pytest.skip("dense reference too large for the CPU suite")
    A, L, E, b = generators.reference_test_problem(n, N)
    x_ref = dense.reference_solution(A, b)
    bb = b.reshape(N, n, 1)
    Lf, Ef = nd.nd_factor(L, E)
    x = nd.nd_solve(Lf, Ef, bb)
    assert np.linalg.norm(x.ravel() - x_ref) < TOL
    assert np.linalg.norm(b - A @ x.ravel()) < TOL
    Lc, Ec, xc = nd.nd_factor_and_solve(L, E, bb)
    assert np.linalg.norm(xc.ravel() - x_ref) < TOL
    y = nd.nd_forward(Lf, Ef, bb)
    xs = nd.nd_backward(Lf, Ef, y)
    assert np.linalg.norm(xs.ravel() - x.ravel()) < TOL


@pytest.mark.parametrize("path", sorted(glob.glob(os.path.join(GOLDEN, "*.npz"))))
def test_oracle_matches_golden(path):
    g = np.load(path)
    L, E, b, x_ref = g["L"], g["E"], g["b"], g["x_ref"]
    N, n = L.shape[0], L.shape[1]
    bb = b.reshape(N, n, -1)
    Lf, Ef, x = nd.nd_factor_and_solve(L, E, bb)
    scale = max(1.0, np.abs(x_ref).max())
    assert np.abs(x.reshape(x_ref.shape) - x_ref).max() / scale < TOL
    # exact storage layout of the factor (lower triangles of L, all of E)
    lf = np.tril(Lf[0])
    assert np.abs(lf - g["L_fac"]).max() <= TOL * max(1.0, np.abs(g["L_fac"]).max())
    if Ef.shape[1]:
        assert np.abs(Ef[0] - g["E_fac"]).max() <= TOL * max(1.0, np.abs(g["E_fac"]).max())


def test_golden_inputs_regenerate_bit_identically():
    g = np.load(os.path.join(GOLDEN, "ref_n10_N8.npz"))
    _, L, E, b = generators.reference_test_problem(10, 8)
    assert np.array_equal(L, g["L"]) and np.array_equal(E, g["E"]) and np.array_equal(b, g["b"])


def test_mask_leaves_inactive_entries_untouched():
    _, L, E, b = generators.reference_test_problem(10, 7)
    B = 4
    Lb, Eb = np.tile(L, (B, 1, 1, 1)), np.tile(E, (B, 1, 1, 1))
    bb = np.tile(b.reshape(7, 10, 1), (B, 1, 1, 1))
    mask = np.array([True, False, True, False])
    Lf, Ef, x = nd.nd_factor_and_solve(Lb, Eb, bb, mask=mask)
    for k in range(B):
        if not mask[k]:
            assert np.array_equal(Lf[k], Lb[k]) and np.array_equal(Ef[k], Eb[k]) and np.array_equal(x[k], bb[k])
    assert np.allclose(x[0], x[2])


def test_backward_error_of_exact_solution_is_tiny():
    L, E, b = generators.readme_problem(64, 8, 2, shift=10.0, seed=3)
    A = generators.dense_from_blocks(L, E)
    x = np.linalg.solve(A, b.reshape(-1, 2)).reshape(b.shape)
    assert nd.backward_error(L, E, x, b)[0] < 1e-15
    assert np.allclose(nd.block_tridiag_matmul(L, E, x)[0], b)


def test_readme_generator_low_shift_is_numerically_singular():
    # the diagonal Cholesky blocks tril(randn) + s I are exponentially
    # ill-conditioned for s <= 1: no Cholesky can factor the shifted configs
    rng = np.random.default_rng(0)
    D = np.tril(rng.standard_normal((64, 64))) + 0.1 * np.eye(64)
    assert np.linalg.cond(D) > 1e12
