"""Differentiable block-tridiagonal solve (no counterpart in the reference,
whose Warp kernels are built with enable_backward=False and whose JAX entry
points define no VJP, socu/block_tridiag_solver.py:157 and socu/jax.py).

    x = block_tridiag_solve(D, E, b)

D (B,N,n,n) diagonal blocks (only the lower triangle is read, as by the
solver), E (B,N-1,n,n) or (B,S,n,n) off-diagonal blocks E_i = Psi_{i+1,i}
(only the first N-1 are read), b (B,N,n,m); 3-D inputs without the batch axis
work too.  The forward factors copies of (D, E) with the ND Cholesky
(factor_and_solve); the backward reuses that factor to solve Psi g = dloss/dx
and forms dloss/dPsi = -g x^T on the D/E block pattern in one fused kernel
(lower-triangle convention for D: the gradient of an entry below the diagonal
collects both of its positions in Psi).
"""
from __future__ import annotations

import torch

from . import _lib
from .block_tridiag_solver import calculate_off_diag_storage_len

__all__ = ["block_tridiag_solve"]


def _dt(t):
    if t.dtype == torch.float64:
        return _lib.FLOAT64
    if t.dtype == torch.float32:
        return _lib.FLOAT32
    raise ValueError("dtype must be float32 or float64")


class _Solve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, D, E, b):
        lib = _lib.load()
        B, N, n = D.shape[0], D.shape[1], D.shape[2]
        m = b.shape[3]
        S = calculate_off_diag_storage_len(N)
        L = D.detach().contiguous().clone()
        Es = torch.zeros((B, S, n, n), dtype=D.dtype, device=D.device)
        if N > 1:
            Es[:, :N - 1] = E.detach()[:, :N - 1]
        x = b.detach().contiguous().clone()
        with torch.cuda.device(D.device):
            st = lib.socu_cholesky_factor_and_solve(_dt(D), L.data_ptr(), Es.data_ptr() if S else None,
                                                    x.data_ptr(), None, B, N, n, m,
                                                    torch.cuda.current_stream(D.device).cuda_stream)
        _lib.check(st, "socu_cholesky_factor_and_solve")
        ctx.factor = (L, Es)
        ctx.e_blocks = E.shape[1]
        ctx.save_for_backward(x)
        return x

    @staticmethod
    def backward(ctx, gx):
        lib = _lib.load()
        (x,) = ctx.saved_tensors
        L, Es = ctx.factor
        B, N, n, m = x.shape
        S = Es.shape[1]
        g = gx.contiguous().clone()
        dD = torch.empty_like(L)
        dE = torch.empty((B, ctx.e_blocks, n, n), dtype=x.dtype, device=x.device)
        with torch.cuda.device(x.device):
            s = torch.cuda.current_stream(x.device).cuda_stream
            st = lib.socu_cholesky_solve(_dt(x), L.data_ptr(), Es.data_ptr() if S else None, g.data_ptr(), None,
                                         B, N, n, m, s)
            _lib.check(st, "socu_cholesky_solve")
            st = lib.socu_block_tridiag_grad(_dt(x), x.data_ptr(), g.data_ptr(), dD.data_ptr(),
                                             dE.data_ptr() if dE.numel() else None, B, N, n, m, ctx.e_blocks, s)
            _lib.check(st, "socu_block_tridiag_grad")
        return dD, dE, g


def block_tridiag_solve(D, E, b):
    """x = Psi^{-1} b, differentiable with respect to D, E and b."""
    squeeze = D.ndim == 3
    if squeeze:
        D, E, b = D[None], E[None], b[None]
    assert D.ndim == 4 and E.ndim == 4 and b.ndim == 4, "D, E and b must be 3- or 4-dimensional"
    B, N, n = D.shape[0], D.shape[1], D.shape[2]
    assert D.shape[3] == n and E.shape[0] == B and E.shape[2:] == (n, n), "inconsistent block shapes"
    assert E.shape[1] >= N - 1, "E must hold at least N-1 blocks"
    assert b.shape[:3] == (B, N, n), "b must have shape (B, N, n, m)"
    assert D.dtype == E.dtype == b.dtype, "D, E and b must share a dtype"
    for t, name in ((D, "D"), (E, "E"), (b, "b")):
        if t.device.type != "cuda":
            raise ValueError(f"socu_b200 runs on CUDA devices only; {name} is on {t.device}")
    x = _Solve.apply(D, E, b)
    return x[0] if squeeze else x
