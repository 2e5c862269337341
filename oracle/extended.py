"""Extended-precision (x87 80-bit ``numpy.longdouble``) restatement of the
nested-dissection factor and solve.

TEST INFRASTRUCTURE ONLY: the "truth" against which FP64 results on
ill-conditioned inputs are judged.  The level schedule, slot orientation and
per-node math are those of ``oracle.nd_cholesky`` (socu/block_tridiag_solver.py
:63-150 factor, :425-485 forward, :581-643 backward, blocked kernels K2-K7
:197-377); only the arithmetic is carried in long double (64-bit significand,
unit roundoff 5.4e-20), with a column Cholesky and substitution loops written
here because LAPACK has no long-double path.

On inputs whose diagonal factor blocks have condition number kappa, every FP64
implementation (the reference's included) carries factor errors of order
kappa^2 * 1e-16; comparing two FP64 results with each other therefore says
little.  Comparing each with this truth does: an implementation is as
accurate as the reference's algorithm when its error is of the same size as
the FP64 oracle's.
"""
from __future__ import annotations

import numpy as np

from .nd_cholesky import level_schedule, off_diag_storage_len

LD = np.longdouble


def _T(A):
    return np.swapaxes(A, -1, -2)


def _chol(A):
    """Batched lower Cholesky of the symmetric matrices A (lower triangle read)."""
    A = np.array(A, dtype=LD)
    n = A.shape[-1]
    C = np.zeros_like(A)
    for j in range(n):
        d = A[..., j, j] - np.einsum("...k,...k->...", C[..., j, :j], C[..., j, :j])
        C[..., j, j] = np.sqrt(d)
        if j + 1 < n:
            C[..., j + 1:, j] = (A[..., j + 1:, j] - np.einsum("...ik,...k->...i", C[..., j + 1:, :j],
                                                               C[..., j, :j])) / C[..., j, j][..., None]
    return C


def _lower_solve(C, X):
    """C^{-1} X, forward substitution (trsm LLNN, socu/blas/trsm.py:203-228)."""
    X = np.array(X, dtype=LD)
    n = C.shape[-1]
    for r in range(n):
        if r:
            X[..., r, :] -= np.einsum("...k,...km->...m", C[..., r, :r], X[..., :r, :])
        X[..., r, :] /= C[..., r, r][..., None]
    return X


def _upper_solve_t(C, X):
    """C^{-T} X, backward substitution (trsm LLTN, socu/blas/trsm.py:315-340)."""
    X = np.array(X, dtype=LD)
    n = C.shape[-1]
    for r in range(n - 1, -1, -1):
        if r < n - 1:
            X[..., r, :] -= np.einsum("...k,...km->...m", C[..., r + 1:, r], X[..., r + 1:, :])
        X[..., r, :] /= C[..., r, r][..., None]
    return X


def nd_factor_and_solve(L, E, b):
    """(L, E, x) in long double for one system: L (N,n,n), E (S,n,n), b (N,n,m)."""
    L = np.array(L, dtype=LD)
    E = np.array(E, dtype=LD)
    y = np.array(b, dtype=LD)
    N = L.shape[0]
    assert E.shape[0] == off_diag_storage_len(N)
    sched = level_schedule(N)
    for s, curr, nxt, nodes in sched:
        A = np.tril(L[nodes]) + _T(np.tril(L[nodes], -1))
        C = _chol(A)
        L[nodes] = C
        y[nodes] = _lower_solve(C, y[nodes])
        right = nodes + s < N
        left = nodes >= s
        F = G = None
        if right.any():
            ir = nodes[right]
            F = _T(_lower_solve(C[right], _T(E[curr + ir // s])))
            E[curr + ir // s] = F
            y[ir + s] -= F @ y[ir]
        if left.any():
            il = nodes[left]
            G = _lower_solve(C[left], E[curr + (il - s) // s])
            E[curr + (il - s) // s] = G
            y[il - s] -= _T(G) @ y[il]
        if right.any():
            L[nodes[right] + s] -= F @ _T(F)
        if left.any():
            L[nodes[left] - s] -= _T(G) @ G
        both = right & left
        if both.any():
            ib = nodes[both]
            E[nxt + (ib - s) // (2 * s)] -= F[both[right]] @ G[both[left]]
    x = y
    for s, curr, _, nodes in reversed(sched):
        right = nodes + s < N
        left = nodes >= s
        xi = x[nodes].copy()
        if right.any():
            ir = nodes[right]
            xi[right] -= _T(E[curr + ir // s]) @ x[ir + s]
        if left.any():
            il = nodes[left]
            xi[left] -= E[curr + (il - s) // s] @ x[il - s]
        x[nodes] = _upper_solve_t(np.tril(L[nodes]), xi)
    return np.tril(L), E, x


def rel_error(a, truth):
    """Normwise relative error ||a - truth||_F / ||truth||_F, computed in long double."""
    a = np.asarray(a, dtype=LD)
    t = np.asarray(truth, dtype=LD)
    den = np.sqrt(np.sum(t * t))
    return float(np.sqrt(np.sum((a - t) * (a - t))) / den) if den > 0 else float(np.sqrt(np.sum(a * a)))
