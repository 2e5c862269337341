"""Seeded input generators (TEST INFRASTRUCTURE ONLY).

* ``reference_test_problem`` restates the generator of the reference tests
  (tests/test_block_tridiag_solver.py:45-80, identical in tests/test_jax.py:29-69):
  legacy ``np.random.seed(42)``, diagonal factor blocks ``tril(rand) + 10 I``,
  sub-diagonal factor blocks ``rand``, Psi = Lfull Lfull^T, b = rand(N n) after
  re-seeding with 42.  Inputs are bit-identical to the reference's.
* ``readme_problem`` is the README generator (README.md:100-121) with the
  diagonal shift ``s`` as a parameter and a ``numpy.random.default_rng(seed)``
  stream: D_chol = tril(randn) + s I, E_chol = randn, L_i = D_chol D_chol^T
  (+ E_chol,i-1 E_chol,i-1^T), E_i = E_chol,i D_chol,i^T, b = randn(N, n, m).
"""
from __future__ import annotations

import numpy as np

from .nd_cholesky import off_diag_storage_len


def reference_test_problem(n: int, N: int, seed: int = 42):
    """Returns (A dense, L (N,n,n), E (S,n,n), b (N*n,)) exactly as the reference tests."""
    np.random.seed(seed)
    Lfull = np.zeros((N * n, N * n))
    for i in range(N):
        Lfull[i * n:(i + 1) * n, i * n:(i + 1) * n] = np.tril(np.random.rand(n, n)) + 10 * np.eye(n)
        if i < N - 1:
            Lfull[(i + 1) * n:(i + 2) * n, i * n:(i + 1) * n] = np.random.rand(n, n)
    A = Lfull @ Lfull.T
    L = np.zeros((N, n, n))
    for i in range(N):
        L[i] = A[i * n:(i + 1) * n, i * n:(i + 1) * n]
    E = np.zeros((off_diag_storage_len(N), n, n))
    for i in range(N - 1):
        E[i] = A[(i + 1) * n:(i + 2) * n, i * n:(i + 1) * n]
    np.random.seed(seed)
    b = np.random.rand(N * n)
    return A, L, E, b


def readme_problem(N: int, n: int, m: int = 1, shift: float = 10.0, seed: int = 0,
                   storage: bool = True):
    """README generator with diagonal shift; returns (L (N,n,n), E (S or N-1,n,n), b (N,n,m))."""
    rng = np.random.default_rng(seed)
    Dc = np.tril(rng.standard_normal((N, n, n))) + shift * np.eye(n)
    Ec = rng.standard_normal((max(N - 1, 0), n, n))
    L = Dc @ np.swapaxes(Dc, -1, -2)
    if N > 1:
        L[1:] += Ec @ np.swapaxes(Ec, -1, -2)
    S = off_diag_storage_len(N) if storage else max(N - 1, 0)
    E = np.zeros((S, n, n))
    if N > 1:
        E[:N - 1] = Ec @ np.swapaxes(Dc[:N - 1], -1, -2)
    b = rng.standard_normal((N, n, m))
    return L, E, b


def illcond_problem(N: int, n: int, m: int = 2, kappa: float = 1e6, alpha: float = 0.3, seed: int = 0):
    """SPD block-tridiagonal system whose diagonal factor blocks have condition
    number ~kappa at every separator level; returns (L (N,n,n), E (S,n,n), b (N,n,m)).

    Psi = A^{1/2} M A^{1/2} with A = blockdiag(A_i), A_i = U_i diag(sigma^2) U_i^T
    (U_i random orthogonal, sigma from 1 down to 1/kappa) and M the block
    tridiagonal matrix with identity diagonal blocks and alpha * Q_i (Q_i random
    orthogonal) off the diagonal.  M is well conditioned for alpha < 1/2
    (eigenvalues in [1 - 2 alpha, 1 + 2 alpha]), so every Schur complement of Psi
    is A^{1/2}-congruent to one of M: each diagonal factor block C_i is
    A_i^{1/2} times a well-conditioned matrix and kappa(C_i) ~ kappa, while
    kappa(Psi) ~ kappa^2 (still positive definite in FP64 up to kappa ~ 1e8).
    The blocks are genuinely ill conditioned, not merely badly scaled (a
    diagonal scaling would leave every Cholesky-based method's relative
    errors unchanged).
    """
    rng = np.random.default_rng(seed)
    sig = np.geomspace(1.0, 1.0 / kappa, n)
    roots = []
    for _ in range(N):
        U, _ = np.linalg.qr(rng.standard_normal((n, n)))
        roots.append((U * sig) @ U.T)
    L = np.stack([r @ r for r in roots])
    L = 0.5 * (L + np.swapaxes(L, -1, -2))
    E = np.zeros((off_diag_storage_len(N), n, n))
    for i in range(N - 1):
        Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
        E[i] = alpha * roots[i + 1] @ Q @ roots[i]
    b = rng.standard_normal((N, n, m))
    return L, E, b


def ragged_instance(seed: int, instance: int):
    """One instance of the ragged MPC-style batch: N ~ U{8..256}, n in {8,16,32,48},
    m in {1,4}, README generator with shift 10, seeded by seed + instance id."""
    rng = np.random.default_rng(seed + instance)
    N = int(rng.integers(8, 257))
    n = int(rng.choice([8, 16, 32, 48]))
    m = int(rng.choice([1, 4]))
    return (N, n, m) + readme_problem(N, n, m, shift=10.0, seed=seed + instance)


def dense_from_blocks(L, E):
    """Dense Psi from lower(L_i) and level-0 slots E_i = Psi_{i+1,i}."""
    N, n = L.shape[0], L.shape[1]
    A = np.zeros((N * n, N * n))
    for i in range(N):
        lo = np.tril(L[i])
        A[i * n:(i + 1) * n, i * n:(i + 1) * n] = lo + np.tril(L[i], -1).T
        if i < N - 1:
            A[(i + 1) * n:(i + 2) * n, i * n:(i + 1) * n] = E[i]
            A[i * n:(i + 1) * n, (i + 1) * n:(i + 2) * n] = E[i].T
    return A
