"""Ragged batches: thousands of independent systems of different horizon N,
block size n and right-hand-side count m, solved by one persistent kernel.

No counterpart in the reference: every socu launch takes a single (N, n, m)
shape for its whole batch (socu/block_tridiag_solver.py:763-800), so a set of
uneven MPC problems needs one launch object per shape.  Here the systems are
packed back to back in three flat arrays (L, E, x); instance i keeps the
reference layouts inside its slice:

    L[off_L[i] : ...]  (N_i, n_i, n_i)            diagonal blocks (lower read)
    E[off_E[i] : ...]  (S_i, n_i, n_i)            S_i = calculate_off_diag_storage_len(N_i)
    x[off_x[i] : ...]  (N_i, n_i, m_i)            right-hand sides in, solution out

and gets exactly the results of ``create_cholesky_factor_and_solve_launch``
on that slice (factor in L/E, solution in x).  The mixed path
(``create_ragged_refined_solve_launch``) leaves L, E, b untouched and refines
every instance in FP64 until its own backward error reaches ``tol``.
"""
from __future__ import annotations

import ctypes
import weakref

import numpy as np
import torch

from . import _lib
from .block_tridiag_solver import _LaunchHandle, _profiler, _stream_handle

__all__ = ["RaggedBatch", "ragged_layout", "shard_instances", "create_ragged_factor_and_solve_launch",
           "create_ragged_refined_solve_launch"]

MAX_BLOCK_SIZE = 64


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64).reshape(-1))


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def ragged_layout(horizons, block_sizes, n_rhs):
    """Packed offsets (elements) and totals of a ragged batch, computed by the
    native library: returns (off_L, off_E, off_x, totals) as int64 arrays."""
    N, n, m = _i64(horizons), _i64(block_sizes), _i64(n_rhs)
    assert N.shape == n.shape == m.shape, "horizons, block_sizes and n_rhs must have the same length"
    count = N.shape[0]
    off = [np.zeros(count, dtype=np.int64) for _ in range(3)]
    tot = np.zeros(3, dtype=np.int64)
    lib = _lib.load()
    _lib.check(lib.socu_ragged_layout(_ptr(N), _ptr(n), _ptr(m), count, _ptr(off[0]), _ptr(off[1]),
                                      _ptr(off[2]), _ptr(tot)), "socu_ragged_layout")
    return off[0], off[1], off[2], tot


def shard_instances(horizons, block_sizes, world_size, rank):
    """Contiguous instance range [lo, hi) for `rank` when a ragged batch is
    split over `world_size` GPUs (one process each), balanced by the factor
    work N * n^3 of every instance.  Instances are independent, so the shards
    need no exchange; each rank builds a RaggedBatch from its own range."""
    assert world_size >= 1 and 0 <= rank < world_size, "rank must lie in [0, world_size)"
    w = _i64(horizons).astype(np.float64) * _i64(block_sizes).astype(np.float64) ** 3
    cum = np.concatenate([[0.0], np.cumsum(w)])
    targets = cum[-1] * np.arange(world_size + 1) / world_size
    bounds = np.searchsorted(cum, targets, side="left")
    bounds[0], bounds[-1] = 0, len(w)
    bounds = np.maximum.accumulate(bounds)
    return int(bounds[rank]), int(bounds[rank + 1])


class RaggedBatch:
    """Shapes, packed layout and device plan (work queue, descriptors, and for
    ``refine=True`` the float workspace) of a ragged batch.

    ``dtype`` is the arithmetic type of the plain path (float32/float64);
    ``refine=True`` selects the mixed path, which takes FP64 arrays."""

    def __init__(self, horizons, block_sizes, n_rhs, dtype=torch.float64, device="cuda", refine=False,
                 max_iter=10):
        self.horizons, self.block_sizes, self.n_rhs = _i64(horizons), _i64(block_sizes), _i64(n_rhs)
        self.count = int(self.horizons.shape[0])
        self.off_L, self.off_E, self.off_x, tot = ragged_layout(self.horizons, self.block_sizes, self.n_rhs)
        self.total_L, self.total_E, self.total_x = (int(t) for t in tot)
        self.storage_len = np.array([_storage_len(int(N)) for N in self.horizons], dtype=np.int64)
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise ValueError(f"socu_b200 runs on CUDA devices only; got device {self.device}")
        if refine and dtype != torch.float64:
            raise ValueError("the refined ragged solve takes float64 arrays")
        assert dtype in (torch.float32, torch.float64), "dtype must be float32 or float64"
        self.dtype = dtype
        self.refine = bool(refine)
        self.max_iter = int(max_iter)
        lib = _lib.load()
        handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            status = lib.socu_ragged_create(
                ctypes.byref(handle), _lib.FLOAT64 if dtype == torch.float64 else _lib.FLOAT32, int(self.refine),
                _ptr(self.horizons), _ptr(self.block_sizes), _ptr(self.n_rhs), self.count, self.max_iter)
        _lib.check(status, "socu_ragged_create")
        self._handle = handle.value
        self._finalizer = weakref.finalize(self, lib.socu_ragged_destroy, self._handle)

    # packed arrays ---------------------------------------------------------
    def empty(self):
        """Uninitialised packed (L, E, x) arrays on the batch's device."""
        kw = dict(dtype=self.dtype, device=self.device)
        return (torch.empty(self.total_L, **kw), torch.empty(self.total_E, **kw), torch.empty(self.total_x, **kw))

    def L_view(self, L, i):
        N, n = int(self.horizons[i]), int(self.block_sizes[i])
        o = int(self.off_L[i])
        return L[o:o + N * n * n].view(N, n, n)

    def E_view(self, E, i):
        S, n = int(self.storage_len[i]), int(self.block_sizes[i])
        o = int(self.off_E[i])
        return E[o:o + S * n * n].view(S, n, n)

    def x_view(self, x, i):
        N, n, m = int(self.horizons[i]), int(self.block_sizes[i]), int(self.n_rhs[i])
        o = int(self.off_x[i])
        return x[o:o + N * n * m].view(N, n, m)

    def pack(self, Ls, Es, xs):
        """Pack per-instance arrays (lists of (N,n,n), (S or N-1,n,n), (N,n,m)
        tensors or numpy arrays) into new device arrays.  E blocks beyond the
        given ones are zero (the storage tail is scratch)."""
        L, E, x = self.empty()
        E.zero_()
        for i in range(self.count):
            self.L_view(L, i).copy_(torch.as_tensor(Ls[i]))
            Ei = torch.as_tensor(Es[i])
            if Ei.shape[0]:
                self.E_view(E, i)[:Ei.shape[0]].copy_(Ei)
            self.x_view(x, i).copy_(torch.as_tensor(xs[i]))
        return L, E, x

    def error_flag(self):
        """Error word of the last finished solve (synchronises): 0 ok,
        1 a queue wait exceeded its time bound, 2 queue overflow."""
        flag = ctypes.c_int(0)
        _lib.check(_lib.load().socu_ragged_error(self._handle, ctypes.byref(flag)), "socu_ragged_error")
        return flag.value

    @property
    def grid(self):
        """CTAs of the persistent kernel."""
        return int(_lib.load().socu_ragged_grid(self._handle))

    def set_wait_limit(self, seconds):
        """Bound of one device-side queue wait without queue progress (default
        4 s).  A wait that runs out sets error word 1 and ends its CTA, so a
        stalled queue ends the launch instead of hanging the GPU."""
        ns = int(round(float(seconds) * 1e9))
        _lib.check(_lib.load().socu_ragged_set_wait_limit(self._handle, ns), "socu_ragged_set_wait_limit")

    def withhold_instance(self, i):
        """Failure injection for tests (host side): leave instance i's first
        tasks out of the queue, so the next solve stalls and must end through
        the wait limit with error word 1."""
        _lib.check(_lib.load().socu_ragged_withhold_instance(self._handle, int(i)), "socu_ragged_withhold_instance")


def _storage_len(N):
    return int(_lib.load().socu_off_diag_storage_len(N))


def _check_packed(batch, name, a, total, dtype):
    assert isinstance(a, torch.Tensor), f"{name} must be a torch tensor"
    if a.device.type != "cuda":
        raise ValueError(f"socu_b200 runs on CUDA devices only; {name} is on {a.device}")
    assert a.dtype == dtype, f"{name} must be {dtype}"
    assert a.is_contiguous(), f"{name} must be contiguous"
    assert a.numel() == total, f"{name} must hold {total} elements (packed ragged layout), got {a.numel()}"


def _launch(batch, L, E, b, x, tol, eta, iters, stream, use_cuda_graph):
    lib = _lib.load()
    dev = batch.device
    sh = _stream_handle(stream, dev)
    handle = ctypes.c_void_p()
    with torch.cuda.device(dev):
        status = lib.socu_ragged_launch_create(
            ctypes.byref(handle), batch._handle, L.data_ptr(), E.data_ptr() if E.numel() else None,
            b.data_ptr() if b is not None else None, x.data_ptr(), float(tol),
            eta.data_ptr() if eta is not None else None, iters.data_ptr() if iters is not None else None,
            int(bool(use_cuda_graph)), sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream)
    _lib.check(status, "socu_ragged_launch_create")
    h = handle.value

    def callback():
        s = sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.socu_launch_run(h, s), "socu_launch_run")

    callback._socu_arrays = (batch, L, E, b, x, eta, iters)
    callback.kernel_count = int(lib.socu_launch_kernel_count(h))
    callback.batch = batch
    handle = _LaunchHandle(lib, h, callback._socu_arrays)
    callback._handle = handle
    callback.profile = _profiler(lib, handle, sh, dev)
    return callback


def create_ragged_factor_and_solve_launch(batch: RaggedBatch, L, E, x, stream=None, use_cuda_graph=True):
    """Factor every instance in place and overwrite x (right-hand sides) with
    the solutions, in one persistent launch (plus a queue reset)."""
    assert not batch.refine, "batch was created for the refined solve"
    _check_packed(batch, "L", L, batch.total_L, batch.dtype)
    _check_packed(batch, "E", E, batch.total_E, batch.dtype)
    _check_packed(batch, "x", x, batch.total_x, batch.dtype)
    return _launch(batch, L, E, None, x, 0.0, None, None, stream, use_cuda_graph)


def create_ragged_refined_solve_launch(batch: RaggedBatch, L, E, b, x, tol=1e-12, stream=None, use_cuda_graph=True):
    """Float factor + FP64 refinement of every instance (L, E, b untouched).
    After each call ``callback.eta`` (count,) holds the backward errors and
    ``callback.iterations`` (count,) the corrections applied (negative: the
    float factor broke down)."""
    assert batch.refine, "batch was created for the plain solve"
    for name, a, total in (("L", L, batch.total_L), ("E", E, batch.total_E), ("b", b, batch.total_x),
                           ("x", x, batch.total_x)):
        _check_packed(batch, name, a, total, torch.float64)
    eta = torch.zeros(batch.count, dtype=torch.float64, device=batch.device)
    iters = torch.zeros(batch.count, dtype=torch.int32, device=batch.device)
    cb = _launch(batch, L, E, b, x, tol, eta, iters, stream, use_cuda_graph)
    cb.eta = eta
    cb.iterations = iters
    return cb
