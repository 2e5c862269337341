"""The no-allocation refined solve, called through the C ABI.

socu_refine_solve_noalloc exists for callers that must not allocate device
memory while they solve: an XLA/JAX custom call (its buffers come from XLA's
allocator and the handler must not call cudaMalloc), a real-time control loop
that bans allocation after start-up, or code running under CUDA stream
capture.  It keeps its scratch in a fixed array inside the library instead of
a caller workspace.  These tests compare it with socu_refine_solve (same
kernels, caller-provided workspace) on problems of different sizes in a
row, so that left-over contents of the shared array from an earlier call would
show up in a later one, and checks each result against the CPU oracle: the
oracle's backward error of x must meet the tolerance, and x must agree with the
oracle's FP64 solution within cond(Psi) times that tolerance.  The block sizes
cover the float node kernel's narrow (n <= 32) and wide (n = 64, 256-thread
CTAs, tensor-core Schur update) launch shapes.  This file is collected last
on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from oracle import generators, nd_cholesky as nd
from socu_b200 import _lib

pytestmark = pytest.mark.gpu

TOL = 1e-12


def _problem(N, n, m, B, seed):
    L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=seed)
    # distinct instances: shift each diagonal block a little
    Ls = np.stack([L + 0.05 * k * np.eye(n) for k in range(B)])
    dev = "cuda"
    return (torch.tensor(Ls, device=dev), torch.tensor(np.tile(E, (B, 1, 1, 1)), device=dev),
            torch.tensor(np.tile(b, (B, 1, 1, 1)), device=dev))


def _run_workspace(lib, L, E, b, B, N, n, m):
    x = torch.zeros_like(b)
    eta = torch.zeros(B, dtype=torch.float64, device=b.device)
    it = torch.zeros(B, dtype=torch.int32, device=b.device)
    nbytes = int(lib.socu_refine_workspace_bytes(B, N, n, m))
    ws = torch.empty(nbytes + 256, dtype=torch.uint8, device=b.device)
    ptr = (ws.data_ptr() + 255) // 256 * 256
    st = lib.socu_refine_solve(L.data_ptr(), E.data_ptr() if E.numel() else None, b.data_ptr(), x.data_ptr(),
                               None, B, N, n, m, 10, TOL, ptr, nbytes, eta.data_ptr(), it.data_ptr(),
                               torch.cuda.current_stream().cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    return x, eta, it


def _run_noalloc(lib, L, E, b, B, N, n, m):
    x = torch.full_like(b, float("nan"))
    eta = torch.zeros(B, dtype=torch.float64, device=b.device)
    it = torch.zeros(B, dtype=torch.int32, device=b.device)
    st = lib.socu_refine_solve_noalloc(L.data_ptr(), E.data_ptr() if E.numel() else None, b.data_ptr(),
                                       x.data_ptr(), None, B, N, n, m, 10, TOL, eta.data_ptr(), it.data_ptr(),
                                       torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.socu_status_string(st)
    torch.cuda.synchronize()
    return x, eta, it


def test_noalloc_matches_workspace_entry_point_on_two_calls():
    lib = _lib.load()
    # later problems are smaller than earlier ones, so stale contents of the
    # shared scratch from an earlier call would be picked up if anything were
    # not re-initialised
    for (N, n, m, B, seed) in [(37, 24, 3, 3, 1), (16, 64, 2, 2, 3), (20, 16, 1, 2, 2)]:
        L, E, b = _problem(N, n, m, B, seed)
        assert lib.socu_refine_workspace_bytes(B, N, n, m) <= 16 << 20
        x_ref, eta_ref, it_ref = _run_workspace(lib, L, E, b, B, N, n, m)
        x, eta, it = _run_noalloc(lib, L, E, b, B, N, n, m)
        assert (eta <= TOL).all() and (eta_ref <= TOL).all()
        assert torch.equal(it, it_ref)
        scale = float(x_ref.abs().max())
        assert float((x - x_ref).abs().max()) <= 1e-12 * scale
        # against the CPU oracle, instance by instance
        Ln, En, bn, xn = (a.cpu().numpy() for a in (L, E, b, x))
        for k in range(B):
            assert nd.backward_error(Ln[k], En[k], xn[k], bn[k])[0] <= TOL
            _, _, x_ora = nd.nd_factor_and_solve(Ln[k], En[k], bn[k])
            kappa = np.linalg.cond(generators.dense_from_blocks(Ln[k], En[k]))
            err = np.abs(xn[k] - x_ora[0]).max() / np.abs(x_ora[0]).max()
            assert err <= 20 * kappa * TOL + 1e-14, (err, kappa)


def test_noalloc_rejects_problems_larger_than_its_scratch():
    lib = _lib.load()
    B, N, n, m = 1, 1024, 64, 8          # float factor alone needs ~50 MB
    assert lib.socu_refine_workspace_bytes(B, N, n, m) > 16 << 20
    L, E, b = (torch.zeros(1, device="cuda", dtype=torch.float64) for _ in range(3))
    x = torch.zeros(1, device="cuda", dtype=torch.float64)
    eta = torch.zeros(1, device="cuda", dtype=torch.float64)
    it = torch.zeros(1, device="cuda", dtype=torch.int32)
    st = lib.socu_refine_solve_noalloc(L.data_ptr(), E.data_ptr(), b.data_ptr(), x.data_ptr(), None, B, N, n, m,
                                       10, TOL, eta.data_ptr(), it.data_ptr(), None)
    assert st == -5
    assert b"no-allocation" in lib.socu_status_string(st)
