"""Dense SciPy checks (TEST INFRASTRUCTURE ONLY).

``reference_solution`` is the reference tests' own oracle
(tests/test_block_tridiag_solver.py:75-78): dense lower Cholesky followed by
two triangular solves.

``permuted_factor`` pins the exact factor storage.  Ordering the block
unknowns by nested-dissection level (node i is eliminated at level
ctz(i+1), socu/block_tridiag_solver.py:174) gives P Psi P^T = LL LL^T.  By
uniqueness of the Cholesky factor the reference's in-place outputs are blocks
of LL: L[i] = LL[i,i]; a level-l slot k couples p=(k+1)2^l-1 and q=p+2^l; for
even k (p eliminated at level l) it stores LL[q,p] (E C^{-T}, trsm_rltn); for
odd k (q eliminated at level l) it stores LL[p,q]^T (C^{-1} E, trsm_llnn).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as la

from .generators import dense_from_blocks
from .nd_cholesky import level_schedule, off_diag_storage_len


def reference_solution(A, b):
    Lc = la.cholesky(A, lower=True)
    y = la.solve_triangular(Lc, b, lower=True)
    return la.solve_triangular(Lc.T, y, lower=False)


def nd_order(N: int):
    """Block order of the permuted matrix: nodes by (level, index)."""
    order = []
    for _, _, _, nodes in level_schedule(N):
        order.extend(int(i) for i in nodes)
    return order


def permuted_factor(L, E):
    """Expected (L, E[S]) factor blocks from the dense Cholesky of P Psi P^T."""
    N, n = L.shape[0], L.shape[1]
    A = dense_from_blocks(L, E)
    order = nd_order(N)
    pos = {node: k for k, node in enumerate(order)}
    perm = np.concatenate([np.arange(i * n, (i + 1) * n) for i in order]) if N else np.zeros(0, int)
    LL = la.cholesky(A[np.ix_(perm, perm)], lower=True)

    def blk(r, c):
        return LL[pos[r] * n:(pos[r] + 1) * n, pos[c] * n:(pos[c] + 1) * n]

    Lx = np.stack([blk(i, i) for i in range(N)])
    Ex = np.zeros((off_diag_storage_len(N), n, n))
    for s, curr, _, _ in level_schedule(N):
        for k in range(N // s - 1):
            p = (k + 1) * s - 1
            q = p + s
            Ex[curr + k] = blk(q, p) if k % 2 == 0 else blk(p, q).T
    return Lx, Ex
