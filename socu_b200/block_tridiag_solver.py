"""Drop-in replacement of ``socu.block_tridiag_solver`` on B200 (sm_100a).

Same function names, keyword arguments, array layouts, mask semantics and
error behaviour as the reference (socu/block_tridiag_solver.py:12-60 and
:739-1727).  Arrays are PyTorch CUDA tensors (or any object exposing
``__cuda_array_interface__``, e.g. a Warp array, which is wrapped without a
copy).  Each ``create_*_launch`` validates its arguments, binds the buffers
and returns a zero-argument callable that enqueues the hand-written CUDA
kernels of ``libsocu_b200.so`` on the chosen stream; ``use_cuda_graph=True``
captures them once, natively, into a CUDA graph.

There is no CPU path: CPU tensors are rejected with ``ValueError`` after the
shape checks (the reference would run them through Warp's CPU backend).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib

__all__ = [
    "calculate_recursive_iterations",
    "calculate_off_diag_storage_len",
    "optimal_problem_settings",
    "create_cholesky_factor_launch",
    "create_cholesky_factor_and_solve_launch",
    "create_cholesky_forward_substitution_launch",
    "create_cholesky_backward_substitution_launch",
    "create_cholesky_solve_launch",
]


def calculate_recursive_iterations(horizon: int) -> int:
    """floor(log2(horizon)) + 1 (socu/block_tridiag_solver.py:12-15)."""
    assert horizon > 0
    return int(horizon).bit_length()


def calculate_off_diag_storage_len(horizon: int) -> int:
    """Number of off-diagonal blocks E must hold (socu/block_tridiag_solver.py:18-23)."""
    iterations = calculate_recursive_iterations(horizon)
    return sum(horizon // (2 ** i) - 1 for i in range(iterations))


def _dtype_name(dtype) -> str:
    """Accepts torch dtypes, numpy dtypes, strings and Warp scalar types."""
    if dtype is None:
        return "float64"
    if isinstance(dtype, torch.dtype):
        return {torch.float64: "float64", torch.float32: "float32"}.get(dtype, str(dtype))
    name = getattr(dtype, "__name__", None) or getattr(dtype, "name", None) or str(dtype)
    name = str(name).rsplit(".", 1)[-1]
    return {"double": "float64", "float": "float32"}.get(name, name)


def _torch_dtype(dtype):
    name = _dtype_name(dtype)
    if name == "float64":
        return torch.float64
    if name == "float32":
        return torch.float32
    raise ValueError("dtype must be wp.float64 or wp.float32")


def optimal_problem_settings(n: int, dtype):
    """Same keys and values as the reference (socu/block_tridiag_solver.py:26-60).

    These are the reference's defaults, reported for compatibility; the B200
    kernels take their launch settings from built-in heuristics or the tuned
    table (socu_b200.autotune) unless ``block_dim`` / ``block_size`` are
    passed to a factory explicitly.  ``pad_multiple`` drives the JAX
    frontend's padding.
    """
    name = _dtype_name(dtype)
    if name == "float64":
        factor_fuse_threshold, solve_fuse_threshold = 16, 32
        pad_multiple_fuse, pad_multiple_blocked = 2, 8
    elif name == "float32":
        factor_fuse_threshold, solve_fuse_threshold = 32, 32
        pad_multiple_fuse, pad_multiple_blocked = 4, 16
    else:
        raise ValueError("dtype must be wp.float64 or wp.float32")
    settings = {
        "block_dim": {"factor": 64, "solve": 64},
        "block_size": {
            "factor": 32 if n % 32 == 0 else 16,
            "solve": 32 if n % 32 == 0 else 16,
        },
        "pad_multiple": {
            "factor": pad_multiple_fuse if n < factor_fuse_threshold else pad_multiple_blocked,
            "solve": pad_multiple_fuse if n < solve_fuse_threshold else pad_multiple_blocked,
        },
    }
    if n < factor_fuse_threshold:
        settings["block_size"]["factor"] = factor_fuse_threshold
    if n < solve_fuse_threshold:
        settings["block_size"]["solve"] = solve_fuse_threshold
    return settings


# ---------------------------------------------------------------------------
# argument handling
# ---------------------------------------------------------------------------

def _as_tensor(a):
    if isinstance(a, torch.Tensor):
        return a
    if hasattr(a, "__cuda_array_interface__"):
        return torch.as_tensor(a, device="cuda")
    raise TypeError(f"expected a torch.Tensor or a __cuda_array_interface__ array, got {type(a)!r}")


def _is_bool(mask) -> bool:
    if isinstance(mask, torch.Tensor):
        return mask.dtype == torch.bool
    dt = getattr(mask, "dtype", None)
    return _dtype_name(dt) in ("bool", "bool_")


def _stream_handle(stream, device):
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    if hasattr(stream, "cuda_stream"):
        return int(stream.cuda_stream)
    raise TypeError(f"unsupported stream object {type(stream)!r}")


def _validate(L, E, x, mask, with_x: bool):
    """Shape checks in the reference's order and with its messages
    (socu/block_tridiag_solver.py:749-774 and :937-966)."""
    if with_x:
        assert E.ndim == L.ndim and x.ndim == L.ndim, "L, E, and x must have the same number of dimensions"
    else:
        assert E.ndim == L.ndim, "L and E must have the same number of dimensions"
    if L.ndim == 4:
        batch_dim = L.shape[0]
    elif L.ndim == 3:
        batch_dim = 1
        L = L.reshape((1, *L.shape))
        E = E.reshape((1, *E.shape))
        if with_x:
            x = x.reshape((1, *x.shape))
    else:
        raise ValueError("L must have 4 or 3 dimensions")
    if with_x:
        assert E.shape[0] == batch_dim and x.shape[0] == batch_dim, "L, E, and x must have same batch dimension"
    else:
        assert E.shape[0] == batch_dim, "L and E must have same batch dimension"
    horizon = L.shape[1]
    n = L.shape[2]
    assert L.shape[3] == n, "The last two dimensions of L must be the same"
    assert E.shape[2] == n and E.shape[3] == n, "L and E must have same block size"
    n_E = calculate_off_diag_storage_len(horizon)
    assert E.shape[1] == n_E, "E has incorrect size, use calculate_off_diag_storage_len to calculate the correct number of blocks"
    n_rhs = 0
    if with_x:
        n_rhs = x.shape[3]
        assert x.shape[1] == horizon and x.shape[2] == n, "x has incorrect dimensions"
    if mask is not None:
        assert mask.ndim == 1 and mask.shape[0] == batch_dim, "mask must have shape (batch_dim,)"
        assert _is_bool(mask), "mask must be a wp.bool array"
    return L, E, x, batch_dim, horizon, n, n_rhs


def _settings(block_dim, block_size):
    """Per-launch settings from the reference's tiling arguments: block_dim
    (threads per tile block) sets the threads per CTA of the node, update and
    sweep kernels, rounded up to 64, 128 or 256; block_size (tile size of the
    blocked kernels) sets the output tile of the blocked Schur update, used for
    n > 64 (16 if block_size <= 16, else 32).  None leaves a setting to the
    tuned table / heuristics."""
    out = {}
    if block_dim is not None:
        bd = int(block_dim)
        assert bd > 0, "block_dim must be positive"
        out["node_threads"] = out["update_threads"] = out["sweep_threads"] = 64 if bd <= 64 else (
            128 if bd <= 128 else 256)
    if block_size is not None:
        bs = int(block_size)
        assert bs > 0, "block_size must be positive"
        out["update_tile"] = 16 if bs <= 16 else 32
    return out or None


class _LaunchHandle:
    """Owns one native launch object; destroyed when the last holder (the
    launch callable and its profile()) goes away."""

    def __init__(self, lib, h, keep=None):
        self.lib, self.h = lib, h
        self.keep = keep   # objects the native launch refers to (buffers, a ragged batch)

    def __del__(self):
        if self.h is not None:
            self.lib.socu_launch_destroy(self.h)
            self.h = None


def _profiler(lib, handle, sh, dev):
    """profile() of a launch object: device time per kernel kind of one eager
    run (CUDA events around every kernel; synchronises), as
    {kind: (ms, launches)} for the kinds that ran.  Holds the handle, so it
    stays valid even if the launch callable itself is dropped."""
    h = handle.h

    def profile():
        assert handle.h is not None
        ms = (ctypes.c_double * _lib.KIND_COUNT)()
        cnt = (ctypes.c_int64 * _lib.KIND_COUNT)()
        s = sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream
        with torch.cuda.device(dev):
            status = lib.socu_launch_profile(h, s, ms, cnt)
        if status != _lib.SOCU_OK:
            kind, where = ctypes.c_int(-1), ctypes.c_int(-1)
            lib.socu_profile_error(ctypes.byref(kind), ctypes.byref(where))
            name = _lib.KIND_NAMES[kind.value] if 0 <= kind.value < _lib.KIND_COUNT else "none"
            places = {0: "pending before a launch", 1: "raised by a launch", 2: "recording a timing event",
                      3: "in a non-launch call of the op", 4: "reading the timing events"}
            _lib.check(status, f"socu_launch_profile ({places.get(where.value, 'unknown')}, kernel kind {name})")
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(_lib.KIND_NAMES) if cnt[i]}
    return profile


def _check_info(info, batch, dev):
    assert isinstance(info, torch.Tensor), "info must be a torch tensor"
    assert info.dtype == torch.int32 and info.ndim == 1 and info.shape[0] == batch, \
        "info must be an int32 tensor of shape (batch_dim,)"
    assert info.device == dev and info.is_contiguous(), "info must be a contiguous tensor on the solver's device"


def _create(op, L, E, x, mask, dtype, device, stream, use_cuda_graph, with_x, settings=None, info=None):
    L, E = _as_tensor(L), _as_tensor(E)
    x = _as_tensor(x) if with_x else None
    mask = _as_tensor(mask) if mask is not None else None
    L, E, x, batch, horizon, n, n_rhs = _validate(L, E, x, mask, with_x)
    tdt = _torch_dtype(dtype)
    optimal_problem_settings(n, dtype)  # dtype check, as the reference does
    arrays = [("L", L), ("E", E)] + ([("x", x)] if with_x else [])
    for name, a in arrays:
        if a.device.type != "cuda":
            if use_cuda_graph:
                raise ValueError("use_cuda_graph=True requires a CUDA device")
            raise ValueError(f"socu_b200 runs on CUDA devices only; {name} is on {a.device}")
        assert a.dtype == tdt, f"{name} must have dtype {tdt}, got {a.dtype}"
        assert a.is_contiguous(), f"{name} must be contiguous"
    if device is not None and torch.device(device).type != "cuda":
        raise ValueError("socu_b200 runs on CUDA devices only")
    dev = L.device
    for name, a in arrays[1:]:
        assert a.device == dev, f"{name} must be on {dev}"
    if mask is not None:
        assert mask.device == dev and mask.is_contiguous(), "mask must be a contiguous array on the solver's device"
    if info is not None:
        _check_info(info, batch, dev)

    lib = _lib.load()
    from . import autotune
    autotune.maybe_autotune(tdt, n, n_rhs, dev)
    dt = _lib.FLOAT64 if tdt == torch.float64 else _lib.FLOAT32
    sh = _stream_handle(stream, dev)
    handle = ctypes.c_void_p()
    tuning = _lib.Tuning.from_dict(settings) if settings else None
    with torch.cuda.device(dev):
        cap_stream = sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream
        status = lib.socu_launch_create_ex(
            ctypes.byref(handle), op, dt,
            L.data_ptr(), E.data_ptr() if E.numel() else None,
            x.data_ptr() if with_x else None,
            mask.data_ptr() if mask is not None else None,
            info.data_ptr() if info is not None else None,
            batch, horizon, n, n_rhs, int(bool(use_cuda_graph)),
            ctypes.byref(tuning) if tuning is not None else None, cap_stream)
    _lib.check(status, "socu_launch_create")
    keep = (L, E, x, mask, info)
    h = handle.value

    def callback():
        s = sh if sh is not None else torch.cuda.current_stream(dev).cuda_stream
        _lib.check(lib.socu_launch_run(h, s), "socu_launch_run")

    callback._socu_arrays = keep
    callback.kernel_count = int(lib.socu_launch_kernel_count(h))
    callback.uses_cuda_graph = bool(use_cuda_graph)
    handle = _LaunchHandle(lib, h, keep)
    callback._handle = handle
    callback.profile = _profiler(lib, handle, sh, dev)
    callback.settings = dict(settings or {})
    return callback


_OPS = {"factor": _lib.OP_FACTOR, "factor_and_solve": _lib.OP_FACTOR_AND_SOLVE, "solve": _lib.OP_SOLVE,
        "forward": _lib.OP_FORWARD, "backward": _lib.OP_BACKWARD}


def _launch_with_settings(op, L, E, x, dtype, settings, use_cuda_graph=True, mask=None, info=None):
    """Graph-captured launch of `op` (a name of _OPS) with explicit launch
    settings (the autotuner's candidates)."""
    with_x = op != "factor"
    return _create(_OPS[op], L, E, x if with_x else None, mask, dtype, None, None, use_cuda_graph, with_x,
                   settings={k: v for k, v in settings.items() if v}, info=info)


# ---------------------------------------------------------------------------
# public factories (socu/block_tridiag_solver.py:739-1727)
# ---------------------------------------------------------------------------

def create_cholesky_factor_launch(L, E, mask=None, block_dim=None, block_size=None,
                                  dtype=torch.float64, device=None, stream=None,
                                  use_cuda_graph=False, *, keep_inverse=False, info=None):
    """In-place ND Cholesky factor of (L, E); returns a zero-argument callable.

    keep_inverse (extension, n <= 64): also store W_i^T = C_i^{-T} in the strict
    upper triangle of every L_i, for the ``factor_has_inverse`` sweeps.
    info (extension): int32 tensor (batch_dim,) on the device, rewritten by every
    call: 0 where the factorisation succeeded, else 1 + the first failing node
    (lowest separator level, then lowest block index) whose pivot was not
    positive (the reference has no numerical status)."""
    op = _lib.OP_FACTOR_INV if keep_inverse else _lib.OP_FACTOR
    return _create(op, L, E, None, mask, dtype, device, stream, use_cuda_graph, False,
                   _settings(block_dim, block_size), info)


def create_cholesky_factor_and_solve_launch(L, E, x, mask=None, block_dim=None, block_size=None,
                                            dtype=torch.float64, device=None, stream=None,
                                            use_cuda_graph=False, *, info=None):
    """Factor fused with the forward sweep, then the backward sweep; x: b in, solution out.

    info (extension): per-instance factor status, as for create_cholesky_factor_launch."""
    return _create(_lib.OP_FACTOR_AND_SOLVE, L, E, x, mask, dtype, device, stream, use_cuda_graph, True,
                   _settings(block_dim, block_size), info)


def create_cholesky_forward_substitution_launch(L, E, x, mask=None, block_dim=None, block_size=None,
                                                dtype=torch.float64, device=None, stream=None,
                                                use_cuda_graph=False, *, factor_has_inverse=False):
    """Forward sweep on a stored factor; x: b in, y out.

    factor_has_inverse (extension, n <= 64): the factor carries W_i^T in its
    upper triangles (factor_and_solve, or factor with keep_inverse=True); the
    sweep then multiplies by W_i instead of solving with C_i."""
    op = _lib.OP_FORWARD_INV if factor_has_inverse else _lib.OP_FORWARD
    return _create(op, L, E, x, mask, dtype, device, stream, use_cuda_graph, True,
                   _settings(block_dim, block_size))


def create_cholesky_backward_substitution_launch(L, E, x, mask=None, block_dim=None, block_size=None,
                                                 dtype=torch.float64, device=None, stream=None,
                                                 use_cuda_graph=False, *, factor_has_inverse=False):
    """Backward sweep on a stored factor; x: y in, solution out.

    factor_has_inverse (extension, n <= 64): the factor carries W_i^T in its
    upper triangles (factor_and_solve, or factor with keep_inverse=True); the
    sweep then multiplies by W_i instead of solving with C_i."""
    op = _lib.OP_BACKWARD_INV if factor_has_inverse else _lib.OP_BACKWARD
    return _create(op, L, E, x, mask, dtype, device, stream, use_cuda_graph, True,
                   _settings(block_dim, block_size))


def create_cholesky_solve_launch(L, E, x, mask=None, block_dim=None, block_size=None,
                                 dtype=torch.float64, device=None, stream=None,
                                 use_cuda_graph=False, *, factor_has_inverse=False):
    """Forward then backward sweep on a stored factor; x: b in, solution out.

    factor_has_inverse (extension, n <= 64): the factor carries W_i^T in its
    upper triangles (factor_and_solve, or factor with keep_inverse=True); the
    sweep then multiplies by W_i instead of solving with C_i."""
    op = _lib.OP_SOLVE_INV if factor_has_inverse else _lib.OP_SOLVE
    return _create(op, L, E, x, mask, dtype, device, stream, use_cuda_graph, True,
                   _settings(block_dim, block_size))


# ---------------------------------------------------------------------------
# extension: moving L to the device
# ---------------------------------------------------------------------------

def copy_lower_blocks(dst, src, stream=None):
    """Copy the lower triangles of the n x n blocks of ``src`` into ``dst``
    (same shape (..., n, n), contiguous, same dtype; pinned host or device
    memory on either side), in 16-row bands, asynchronously on ``stream``
    (default: the current stream of the device side).  Every factor and the
    FP64 residual read only lower(L_i), so a caller that streams L from host
    memory for each solve moves (n + 16) / 2n of its bytes (62.5 % at n = 64).
    Elements of ``dst`` above the bands are left unchanged.  Returns the bytes
    moved.  No counterpart in the reference."""
    if dst.shape != src.shape or dst.dtype != src.dtype:
        raise ValueError("dst and src must have the same shape and dtype")
    if dst.dim() < 2 or dst.shape[-1] != dst.shape[-2]:
        raise ValueError("blocks must be square: shape (..., n, n)")
    if not (dst.is_contiguous() and src.is_contiguous()):
        raise ValueError("dst and src must be contiguous")
    n = int(dst.shape[-1])
    count = dst.numel() // (n * n) if n else 0
    dev = dst.device if dst.is_cuda else src.device
    if dev.type != "cuda":
        raise ValueError("one side must be CUDA memory")
    sh = _stream_handle(stream if stream is not None else torch.cuda.current_stream(dev), dev)
    lib = _lib.load()
    _lib.check(lib.socu_copy_lower_blocks_async(ctypes.c_void_p(dst.data_ptr()), ctypes.c_void_p(src.data_ptr()),
                                                count, n, dst.element_size(), sh), "socu_copy_lower_blocks_async")
    return int(lib.socu_lower_blocks_bytes(count, n, dst.element_size()))
