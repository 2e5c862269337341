"""JAX entry points with the names and semantics of socu.jax (socu/jax.py:270-337).

    cholesky_factor(L, E, pad_problem=True)             -> (L, E)      E of storage length S
    cholesky_solve(L, E, b, pad_problem=True)           -> x
    cholesky_factor_and_solve(L, E, b, pad_problem=True)-> (L, E, x)
    forward_substitution(L, E, b, pad_problem=True)     -> y
    backward_substitution(L, E, y, pad_problem=True)    -> x

Inputs are (N, n, n) / (N-1 or S, n, n) / (N, n, m) arrays, or the same with a
leading batch axis; E is zero-padded to the storage length S as in
socu/jax.py:72-82 and the factor is returned with S slots.  ``vmap`` over any
argument is routed to one batched call (socu/jax.py:223-263).

``pad_problem`` is accepted for compatibility.  The reference pads n to its
Warp tile multiple with identity blocks (socu/jax.py:85-129) and slices the
result back, which leaves the results unchanged; the CUDA kernels here take
any n, so no padding is done.

Arrays cross into the library through DLPack on the array's own device
(no host copy); the JAX inputs are not modified (JAX arrays are immutable, the
library works on copies).  This eager path runs outside ``jax.jit``; inside
jit the same C-ABI functions would be registered as an XLA FFI custom call
(every plain entry point takes a stream and allocates nothing), which needs
XLA's FFI headers.

JAX is imported lazily: this module imports without JAX (its shape helpers
are plain array code) and the entry points raise ImportError when JAX is
missing.
"""
from __future__ import annotations

__all__ = ["cholesky_factor", "cholesky_solve", "cholesky_factor_and_solve", "forward_substitution",
           "backward_substitution"]


def _storage_len(N):
    from .block_tridiag_solver import calculate_off_diag_storage_len
    return calculate_off_diag_storage_len(N)


# ---------------------------------------------------------------------------
# shape logic (array-library agnostic; socu/jax.py:25-82)
# ---------------------------------------------------------------------------
def _validate_problem_shapes(L, E, b=None):
    if L.ndim not in (3, 4):
        raise ValueError(f"L must be 3- or 4-dimensional, got shape {L.shape}")
    if E.ndim != L.ndim:
        raise ValueError(f"E must have the same rank as L, got L: {L.shape}, E: {E.shape}")
    h = L.ndim - 3
    N, n = L.shape[h], L.shape[h + 1]
    if L.shape[-1] != n:
        raise ValueError(f"L must be square in last two dimensions, got shape {L.shape}")
    if tuple(E.shape[h + 1:]) != tuple(L.shape[h + 1:]):
        raise ValueError(f"E block dimensions must match L's n={n}, got E shape {E.shape}")
    if L.ndim == 4 and E.shape[0] != L.shape[0]:
        raise ValueError(f"L and E must have the same batch size, got L: {L.shape}, E: {E.shape}")
    if b is not None:
        if b.ndim != L.ndim:
            raise ValueError(f"b must have the same rank as L, got L: {L.shape}, b: {b.shape}")
        if b.shape[h] != N:
            raise ValueError(f"b horizon dimension must be {N}, got b shape {b.shape}")
        if b.shape[h + 1] != n:
            raise ValueError(f"b block dimension must be {n}, got b shape {b.shape}")
        if L.ndim == 4 and b.shape[0] != L.shape[0]:
            raise ValueError(f"L and b must have the same batch size, got L: {L.shape}, b: {b.shape}")
        if L.dtype != b.dtype:
            raise ValueError(f"L and b must have same dtype, got L: {L.dtype}, b: {b.dtype}")
    if L.dtype != E.dtype:
        raise ValueError(f"L and E must have same dtype, got L: {L.dtype}, E: {E.dtype}")


def _to_batched(L, E, b=None):
    was_unbatched = L.ndim == 3
    if was_unbatched:
        L, E = L[None, ...], E[None, ...]
        if b is not None:
            b = b[None, ...]
    return L, E, b, was_unbatched


def _ensure_E_size(horizon, E, xp):
    """Zero-pad E (B, k, n, n) to the storage length of `horizon`."""
    S = _storage_len(horizon)
    if E.shape[1] < S:
        return xp.pad(E, ((0, 0), (0, S - E.shape[1]), (0, 0), (0, 0)))
    return E


# ---------------------------------------------------------------------------
# JAX side
# ---------------------------------------------------------------------------
def _jax():
    try:
        import jax
        import jax.numpy as jnp
    except ImportError as e:  # pragma: no cover - depends on the environment
        raise ImportError("socu_b200.jax needs JAX (jax, jaxlib with CUDA); it is not installed") from e
    return jax, jnp


def _impl(L, E, b, mode):
    """Batched (B, ...) JAX arrays in, JAX arrays out; one library call."""
    import torch

    from . import block_tridiag_solver as bts

    jax, jnp = _jax()
    E = _ensure_E_size(L.shape[1], E, jnp)

    def to_torch(a):
        return torch.utils.dlpack.from_dlpack(a).clone()

    def to_jax(t):
        return jax.dlpack.from_dlpack(t)

    Lt, Et = to_torch(L), to_torch(E)
    if Lt.device.type != "cuda":
        raise ValueError("socu_b200 runs on CUDA devices only; the JAX arrays are not on a GPU")
    if mode == "factor":
        bts.create_cholesky_factor_launch(Lt, Et, use_cuda_graph=False)()
        torch.cuda.current_stream(Lt.device).synchronize()
        return to_jax(Lt), to_jax(Et)
    xt = to_torch(b)
    create = {"solve": bts.create_cholesky_solve_launch,
              "forward": bts.create_cholesky_forward_substitution_launch,
              "backward": bts.create_cholesky_backward_substitution_launch,
              "factor_and_solve": bts.create_cholesky_factor_and_solve_launch}[mode]
    create(Lt, Et, xt, use_cuda_graph=False)()
    torch.cuda.current_stream(Lt.device).synchronize()
    if mode == "factor_and_solve":
        return to_jax(Lt), to_jax(Et), to_jax(xt)
    return to_jax(xt)


def _call(L, E, b, mode, impl=None):
    """Validate, add the batch axis, run one batched call, drop the axis again
    (socu/jax.py:198-220)."""
    _validate_problem_shapes(L, E, b)
    L, E, b, was_unbatched = _to_batched(L, E, b)
    out = (impl or _impl)(L, E, b, mode)
    if not was_unbatched:
        return out
    if mode in ("solve", "forward", "backward"):
        return out[0]
    return tuple(o[0] for o in out)


_OPS = {}


def _op(mode, has_b):
    """custom_vmap-wrapped op (vmap routed to one batched call), built once."""
    key = (mode, has_b)
    if key in _OPS:
        return _OPS[key]
    jax, jnp = _jax()

    if has_b:
        @jax.custom_batching.custom_vmap
        def op(L, E, b):
            return _call(L, E, b, mode)

        @op.def_vmap
        def op_vmap(axis_size, in_batched, L, E, b):
            L = L if in_batched[0] else jnp.broadcast_to(L, (axis_size,) + L.shape)
            E = E if in_batched[1] else jnp.broadcast_to(E, (axis_size,) + E.shape)
            b = b if in_batched[2] else jnp.broadcast_to(b, (axis_size,) + b.shape)
            out = _impl(L, E, b, mode)
            return out, (True, True, True) if mode == "factor_and_solve" else True
    else:
        @jax.custom_batching.custom_vmap
        def op(L, E):
            return _call(L, E, None, mode)

        @op.def_vmap
        def op_vmap(axis_size, in_batched, L, E):
            L = L if in_batched[0] else jnp.broadcast_to(L, (axis_size,) + L.shape)
            E = E if in_batched[1] else jnp.broadcast_to(E, (axis_size,) + E.shape)
            return _impl(L, E, None, mode), (True, True)

    _OPS[key] = op
    return op


def cholesky_factor(L, E, pad_problem: bool = True):
    return _op("factor", False)(L, E)


def cholesky_solve(L, E, b, pad_problem: bool = True):
    return _op("solve", True)(L, E, b)


def cholesky_factor_and_solve(L, E, b, pad_problem: bool = True):
    return _op("factor_and_solve", True)(L, E, b)


def forward_substitution(L, E, b, pad_problem: bool = True):
    return _op("forward", True)(L, E, b)


def backward_substitution(L, E, y, pad_problem: bool = True):
    return _op("backward", True)(L, E, y)
