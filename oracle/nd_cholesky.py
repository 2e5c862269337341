"""NumPy restatement of socu's nested-dissection block-tridiagonal Cholesky.

TEST INFRASTRUCTURE ONLY (checker and CPU baseline); never imported by the
product package.

Every function follows the reference file:line it cites.  All arithmetic is
float64 regardless of the input dtype.  Arrays are batched:
  L (B, N, n, n)   diagonal blocks; only the lower triangle is read
  E (B, S, n, n)   off-diagonal storage, S = off_diag_storage_len(N); slots
                   >= N-1 must be zero on input (fill-in is accumulated)
  x (B, N, n, m)   right-hand side in, solution (or y) out
Work is vectorised over the batch and over the independent nodes of one
nested-dissection level, which is exactly the parallelism the reference's
per-level kernels expose (socu/block_tridiag_solver.py:169-174).
"""
from __future__ import annotations

import numpy as np


# ---------------------------------------------------------------------------
# schedule and storage (socu/block_tridiag_solver.py:12-23, 792-813)
# ---------------------------------------------------------------------------

def recursive_iterations(horizon: int) -> int:
    """K = floor(log2 N) + 1 (socu/block_tridiag_solver.py:12-15)."""
    assert horizon > 0
    return int(horizon).bit_length()


def off_diag_storage_len(horizon: int) -> int:
    """S = sum_{l<K} (N // 2^l - 1) (socu/block_tridiag_solver.py:18-23)."""
    return sum(horizon // (2 ** l) - 1 for l in range(recursive_iterations(horizon)))


def level_schedule(horizon: int):
    """Per-level (stride, curr_offset, next_offset, nodes).

    Follows the host loop of socu/block_tridiag_solver.py:869-914: stride
    s = 2^l, level-l nodes i = s-1 + 2s*t for t < (N+s)//(2s), offsets
    o_0 = 0 and o_{l+1} = o_l + N//2^l - 1.
    """
    out = []
    s, curr, nxt = 1, 0, horizon - 1
    for _ in range(recursive_iterations(horizon)):
        d = (horizon + s) // (2 * s)
        nodes = s - 1 + 2 * s * np.arange(d)
        out.append((s, curr, nxt, nodes))
        s *= 2
        curr = nxt
        nxt += horizon // s - 1
    return out


# ---------------------------------------------------------------------------
# small batched dense kernels
# ---------------------------------------------------------------------------

def _sym_lower(A):
    """Symmetric matrix built from the lower triangle (potrf.py:101-102: only
    the lower triangle is used)."""
    lo = np.tril(A)
    return lo + np.swapaxes(np.tril(A, -1), -1, -2)


def _lower_solve(C, X):
    """C^{-1} X for lower-triangular C by forward substitution, batched."""
    X = np.array(X, dtype=np.float64, copy=True)
    n = C.shape[-1]
    for r in range(n):
        if r:
            X[..., r, :] -= np.einsum("...k,...km->...m", C[..., r, :r], X[..., :r, :])
        X[..., r, :] /= C[..., r, r][..., None]
    return X


def _upper_solve_t(C, X):
    """C^{-T} X for lower-triangular C by backward substitution, batched."""
    X = np.array(X, dtype=np.float64, copy=True)
    n = C.shape[-1]
    for r in range(n - 1, -1, -1):
        if r < n - 1:
            X[..., r, :] -= np.einsum("...k,...km->...m", C[..., r + 1:, r], X[..., r + 1:, :])
        X[..., r, :] /= C[..., r, r][..., None]
    return X


def _T(A):
    return np.swapaxes(A, -1, -2)


def _as_batched(*arrays):
    out = []
    for a in arrays:
        out.append(None if a is None else (a[None] if a.ndim == 3 else a))
    return out


def _active(mask, B):
    if mask is None:
        return np.arange(B)
    return np.nonzero(np.asarray(mask, dtype=bool))[0]


# ---------------------------------------------------------------------------
# factor (socu/block_tridiag_solver.py:739-923; blocked kernels K2-K7 at
# :197-377 and socu/blas/{potrf,trsm,syrk,gemm}.py)
# ---------------------------------------------------------------------------

def _factor_level(L, E, y, s, curr, nxt, nodes, N):
    b = L.shape[0]
    # K2: in-place lower Cholesky of every level node (potrf.py:97-117)
    C = np.linalg.cholesky(_sym_lower(L[:, nodes]))
    L[:, nodes] = C
    if y is not None:
        # fused forward step, block_tridiag_solver.py:108-110
        y[:, nodes] = _lower_solve(C, y[:, nodes])
    right = nodes + s < N
    left = nodes >= s
    F = G = None
    if right.any():
        ir = nodes[right]
        slot = curr + ir // s
        # K3: E_right <- E_right C^{-T} (trsm_rltn, block_tridiag_solver.py:219-248)
        F = _T(_lower_solve(C[:, right], _T(E[:, slot])))
        E[:, slot] = F
    if left.any():
        il = nodes[left]
        slot = curr + (il - s) // s
        # K4: E_left <- C^{-1} E_left (trsm_llnn, block_tridiag_solver.py:251-279)
        G = _lower_solve(C[:, left], E[:, slot])
        E[:, slot] = G
    if y is not None:
        # forward coupling updates (block_tridiag_solver.py:124-126, 138-141)
        if right.any():
            ir = nodes[right]
            y[:, ir + s] -= F @ y[:, ir]
        if left.any():
            il = nodes[left]
            y[:, il - s] -= _T(G) @ y[:, il]
    # K5/K6: Schur updates of the two neighbours (syrk_ln / syrk_lt,
    # block_tridiag_solver.py:282-342).  Targets i+s of a right coupling and
    # i-s of a left coupling can coincide (nodes i and i+2s); the reference
    # accumulates both with atomics, here they are applied one after the other.
    if right.any():
        ir = nodes[right]
        L[:, ir + s] -= F @ _T(F)
    if left.any():
        il = nodes[left]
        L[:, il - s] -= _T(G) @ G
    # K7: fill-in coupling i-s <-> i+s (gemm_nn, block_tridiag_solver.py:345-377)
    both = right & left
    if both.any():
        ib = nodes[both]
        Fb = F[:, both[right]]
        Gb = G[:, both[left]]
        E[:, nxt + (ib - s) // (2 * s)] -= Fb @ Gb


def nd_factor(L, E, mask=None, y=None):
    """In-place ND Cholesky factor (and optional fused forward substitution).

    Returns (L, E[, y]) as float64 copies; the inputs are not modified.
    Upper triangles of the returned L blocks are zero.
    """
    L, E, y = _as_batched(np.asarray(L, np.float64), np.asarray(E, np.float64),
                          None if y is None else np.asarray(y, np.float64))
    B, N, n, _ = L.shape
    assert E.shape[1] == off_diag_storage_len(N)
    act = _active(mask, B)
    Lw, Ew = L[act].copy(), E[act].copy()
    yw = None if y is None else y[act].copy()
    for s, curr, nxt, nodes in level_schedule(N):
        _factor_level(Lw, Ew, yw, s, curr, nxt, nodes, N)
    Lo, Eo = L.copy(), E.copy()
    Lo[act], Eo[act] = Lw, Ew
    if y is None:
        return Lo, Eo
    yo = y.copy()
    yo[act] = yw
    return Lo, Eo, yo


# ---------------------------------------------------------------------------
# substitution sweeps (K9 socu/block_tridiag_solver.py:425-485,
# K13 :581-643; launch loops :1294-1309 and :1435-1451)
# ---------------------------------------------------------------------------

def nd_forward(L, E, x, mask=None):
    """y <- (ND factor)^{-1} b, levels ascending."""
    L, E, x = _as_batched(np.asarray(L, np.float64), np.asarray(E, np.float64),
                          np.asarray(x, np.float64))
    B, N = L.shape[:2]
    act = _active(mask, B)
    y = x.copy()
    yw = y[act]
    Lw, Ew = L[act], E[act]
    for s, curr, _, nodes in level_schedule(N):
        C = np.tril(Lw[:, nodes])
        yw[:, nodes] = _lower_solve(C, yw[:, nodes])
        right = nodes + s < N
        left = nodes >= s
        if right.any():
            ir = nodes[right]
            yw[:, ir + s] -= Ew[:, curr + ir // s] @ yw[:, ir]
        if left.any():
            il = nodes[left]
            yw[:, il - s] -= _T(Ew[:, curr + (il - s) // s]) @ yw[:, il]
    y[act] = yw
    return y


def nd_backward(L, E, y, mask=None):
    """x <- (ND factor)^{-T} y, levels descending."""
    L, E, y = _as_batched(np.asarray(L, np.float64), np.asarray(E, np.float64),
                          np.asarray(y, np.float64))
    B, N = L.shape[:2]
    act = _active(mask, B)
    x = y.copy()
    xw = x[act]
    Lw, Ew = L[act], E[act]
    for s, curr, _, nodes in reversed(level_schedule(N)):
        right = nodes + s < N
        left = nodes >= s
        xi = xw[:, nodes].copy()
        if right.any():
            ir = nodes[right]
            xi[:, right] -= _T(Ew[:, curr + ir // s]) @ xw[:, ir + s]
        if left.any():
            il = nodes[left]
            xi[:, left] -= Ew[:, curr + (il - s) // s] @ xw[:, il - s]
        xw[:, nodes] = _upper_solve_t(np.tril(Lw[:, nodes]), xi)
    x[act] = xw
    return x


def nd_solve(L, E, b, mask=None):
    """Forward then backward sweep on a stored factor (create_cholesky_solve_launch)."""
    return nd_backward(L, E, nd_forward(L, E, b, mask), mask)


def nd_factor_and_solve(L, E, b, mask=None):
    """Fused factor + forward, then backward (create_cholesky_factor_and_solve_launch)."""
    Lf, Ef, y = nd_factor(L, E, mask=mask, y=b)
    return Lf, Ef, nd_backward(Lf, Ef, y, mask)


# ---------------------------------------------------------------------------
# residual and backward error against the ORIGINAL blocks
# ---------------------------------------------------------------------------

def block_tridiag_matmul(D, E, x):
    """Psi x for Psi built from lower(D_i) and the level-0 slots E_i = Psi_{i+1,i}."""
    D, E, x = _as_batched(np.asarray(D, np.float64), np.asarray(E, np.float64),
                          np.asarray(x, np.float64))
    N = D.shape[1]
    out = _sym_lower(D) @ x
    if N > 1:
        E0 = E[:, :N - 1]
        out[:, 1:] += E0 @ x[:, :-1]
        out[:, :-1] += _T(E0) @ x[:, 1:]
    return out


def psi_inf_norm(D, E):
    """||Psi||_inf per batch entry (max absolute row sum)."""
    D, E = _as_batched(np.asarray(D, np.float64), np.asarray(E, np.float64))
    N = D.shape[1]
    rows = np.abs(_sym_lower(D)).sum(-1)
    if N > 1:
        E0 = np.abs(E[:, :N - 1])
        rows[:, 1:] += E0.sum(-1)
        rows[:, :-1] += E0.sum(-2)
    return rows.reshape(rows.shape[0], -1).max(-1)


def backward_error(D, E, x, b):
    """eta = ||b - Psi x||_inf / (||Psi||_inf ||x||_inf + ||b||_inf) per batch entry."""
    D, E, x, b = _as_batched(np.asarray(D, np.float64), np.asarray(E, np.float64),
                             np.asarray(x, np.float64), np.asarray(b, np.float64))
    r = b - block_tridiag_matmul(D, E, x)
    Bn = r.shape[0]
    rn = np.abs(r).reshape(Bn, -1).max(-1)
    xn = np.abs(x).reshape(Bn, -1).max(-1)
    bn = np.abs(b).reshape(Bn, -1).max(-1)
    return rn / (psi_inf_norm(D, E) * xn + bn)
