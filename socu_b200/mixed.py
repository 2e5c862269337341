"""Mixed-precision factorisation with FP64 iterative refinement.

No counterpart in the reference (socu has plain f32 and f64 paths only,
socu/block_tridiag_solver.py:26-60).  A float copy of (L, E) is factored with
the same nested-dissection kernels as the drop-in API; the solution is then
refined in FP64 against the original blocks until the normwise backward error

    eta = ||b - Psi x||_inf / (||Psi||_inf ||x||_inf + ||b||_inf) <= tol

per instance (or max_iter corrections).  Converged instances drop out of all
later kernels.  Inputs are FP64 CUDA tensors in the reference layouts
(L (B,N,n,n), E (B,S,n,n) with S = calculate_off_diag_storage_len(N),
b and x (B,N,n,m); 3-D inputs without the batch axis are accepted) and are not
modified, except x (the solution).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .block_tridiag_solver import _LaunchHandle, _as_tensor, _profiler, _stream_handle, _validate

__all__ = ["create_cholesky_refined_solve_launch", "block_tridiag_residual", "backward_error"]


def _check_f64(**arrays):
    for name, a in arrays.items():
        if a.device.type != "cuda":
            raise ValueError(f"socu_b200 runs on CUDA devices only; {name} is on {a.device}")
        assert a.dtype == torch.float64, f"{name} must be float64"
        assert a.is_contiguous(), f"{name} must be contiguous"


def create_cholesky_refined_solve_launch(L, E, b, x, mask=None, tol=1e-12, max_iter=10, stream=None,
                                         use_cuda_graph=True, fp64_fallback=False):
    """Returns a zero-argument callable solving Psi x = b (float factor + FP64
    refinement).  After each call, ``callback.eta`` (B,) holds the final
    backward errors and ``callback.iterations`` (B,) the corrections applied
    (negative: the float factor broke down after that many steps).

    fp64_fallback (graph only): instances whose refinement does not reach tol
    (stalled, out of rounds, or broken down) are solved again by the plain
    FP64 factor_and_solve inside the same graph; ``callback.used_fp64`` (B,)
    marks them and ``callback.eta`` then holds the FP64 solution's backward
    error.  Needs a workspace with FP64 copies of L and E."""
    if fp64_fallback and not use_cuda_graph:
        raise ValueError("fp64_fallback runs inside the CUDA graph; use_cuda_graph must be True")
    L, E, b, x = (_as_tensor(a) for a in (L, E, b, x))
    mask = _as_tensor(mask) if mask is not None else None
    assert b.shape == x.shape, "b and x must have the same shape"
    L4, E4, x4, B, N, n, m = _validate(L, E, x, mask, True)
    b4 = b.reshape(x4.shape)
    _check_f64(L=L4, E=E4, b=b4, x=x4)
    dev = L4.device
    lib = _lib.load()
    ws_bytes = int(lib.socu_refine_fallback_workspace_bytes(B, N, n, m) if fp64_fallback
                   else lib.socu_refine_workspace_bytes(B, N, n, m))
    ws = torch.empty(max(ws_bytes, 256) + 256, dtype=torch.uint8, device=dev)
    ws_ptr = (ws.data_ptr() + 255) // 256 * 256
    eta = torch.zeros(B, dtype=torch.float64, device=dev)
    iters = torch.zeros(B, dtype=torch.int32, device=dev)
    sh = _stream_handle(stream, dev)
    handle = ctypes.c_void_p()
    used = torch.zeros(B, dtype=torch.uint8, device=dev)
    with torch.cuda.device(dev):
        cap_stream = sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream
        E_ptr = E4.data_ptr() if E4.numel() else None
        mask_ptr = mask.data_ptr() if mask is not None else None
        if fp64_fallback:
            status = lib.socu_refine_fallback_launch_create(
                ctypes.byref(handle), L4.data_ptr(), E_ptr, b4.data_ptr(), x4.data_ptr(), mask_ptr, B, N, n, m,
                int(max_iter), float(tol), ws_ptr, ws_bytes, eta.data_ptr(), iters.data_ptr(), used.data_ptr(),
                cap_stream)
        else:
            status = lib.socu_refine_launch_create(
                ctypes.byref(handle), L4.data_ptr(), E_ptr, b4.data_ptr(), x4.data_ptr(), mask_ptr, B, N, n, m,
                int(max_iter), float(tol), ws_ptr, ws_bytes, eta.data_ptr(), iters.data_ptr(),
                int(bool(use_cuda_graph)), cap_stream)
    _lib.check(status, "socu_refine_fallback_launch_create" if fp64_fallback else "socu_refine_launch_create")
    h = handle.value

    def callback():
        s = sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.socu_launch_run(h, s), "socu_launch_run")

    callback._socu_arrays = (L4, E4, b4, x4, mask, ws)
    callback.eta = eta
    callback.iterations = iters
    callback.used_fp64 = used
    callback.workspace_bytes = ws_bytes
    callback.kernel_count = int(lib.socu_launch_kernel_count(h))
    # graph mode: the refinement rounds run in a conditional WHILE node
    callback.round_kernel_count = int(lib.socu_launch_round_kernel_count(h))
    # eager run with per-kernel events (all max_iter rounds; not the graph)
    handle = _LaunchHandle(lib, h, callback._socu_arrays)
    callback._handle = handle
    callback.profile = _profiler(lib, handle, sh, dev)
    return callback


def block_tridiag_residual(L, E, x, b, out=None):
    """r = b - Psi x in FP64 (Psi from lower(L_i) and the level-0 slots of E)."""
    L, E, x, b = (_as_tensor(a) for a in (L, E, x, b))
    L4, E4, x4, B, N, n, m = _validate(L, E, x, None, True)
    b4 = b.reshape(x4.shape)
    _check_f64(L=L4, E=E4, x=x4, b=b4)
    r = torch.empty_like(x4) if out is None else out.reshape(x4.shape)
    lib = _lib.load()
    with torch.cuda.device(L4.device):
        st = lib.socu_block_tridiag_residual(L4.data_ptr(), E4.data_ptr() if E4.numel() else None, x4.data_ptr(),
                                             b4.data_ptr(), r.data_ptr(), B, N, n, m,
                                             torch.cuda.current_stream(L4.device).cuda_stream)
    _lib.check(st, "socu_block_tridiag_residual")
    return r.reshape(x.shape)


def backward_error(L, E, x, b):
    """Per-instance eta = ||b - Psi x||_inf / (||Psi||_inf ||x||_inf + ||b||_inf), FP64 on the GPU."""
    L, E, x, b = (_as_tensor(a) for a in (L, E, x, b))
    r = block_tridiag_residual(L, E, x, b)
    L4 = L if L.ndim == 4 else L[None]
    E4 = E if E.ndim == 4 else E[None]
    B, N = L4.shape[:2]
    lo = torch.tril(L4)
    D = lo + torch.tril(L4, -1).transpose(-1, -2)
    rows = D.abs().sum(-1)
    if N > 1:
        E0 = E4[:, :N - 1].abs()
        rows[:, 1:] += E0.sum(-1)
        rows[:, :-1] += E0.sum(-2)
    psi = rows.reshape(B, -1).amax(-1)
    rr = r.reshape(B, -1).abs().amax(-1)
    xx = x.reshape(B, -1).abs().amax(-1)
    bb = b.reshape(B, -1).abs().amax(-1)
    return rr / (psi * xx + bb)
