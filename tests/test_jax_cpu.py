"""socu_b200.jax: the JAX entry points' shape logic (JAX itself is not
installed in the test image; the helpers are plain array code)."""
import importlib.util

import numpy as np
import pytest

from oracle.nd_cholesky import off_diag_storage_len
from socu_b200 import jax as sj

HAVE_JAX = importlib.util.find_spec("jax") is not None


def _fake_impl(calls):
    def impl(L, E, b, mode):
        E = sj._ensure_E_size(L.shape[1], E, np)
        calls.append((mode, L.shape, E.shape, None if b is None else b.shape))
        if mode == "factor":
            return L, E
        if mode == "factor_and_solve":
            return L, E, b
        return b
    return impl


@pytest.mark.parametrize("batched", [False, True])
def test_batching_and_storage_padding(batched):
    N, n, m = 10, 4, 2
    L = np.zeros((N, n, n)); E = np.zeros((N - 1, n, n)); b = np.zeros((N, n, m))
    if batched:
        L, E, b = L[None].repeat(3, 0), E[None].repeat(3, 0), b[None].repeat(3, 0)
    calls = []
    Lo, Eo, xo = sj._call(L, E, b, "factor_and_solve", impl=_fake_impl(calls))
    B = 3 if batched else 1
    assert calls == [("factor_and_solve", (B, N, n, n), (B, off_diag_storage_len(N), n, n), (B, N, n, m))]
    lead = (3,) if batched else ()
    assert Lo.shape == lead + (N, n, n) and Eo.shape == lead + (off_diag_storage_len(N), n, n)
    assert xo.shape == lead + (N, n, m)
    x = sj._call(L, E, b, "solve", impl=_fake_impl(calls))
    assert x.shape == lead + (N, n, m)
    Lf, Ef = sj._call(L, E, None, "factor", impl=_fake_impl(calls))
    assert Ef.shape == lead + (off_diag_storage_len(N), n, n)


@pytest.mark.parametrize("args,msg", [
    ((np.zeros((2, 2)), np.zeros((2, 2)), None), "L must be 3- or 4-dimensional"),
    ((np.zeros((4, 3, 3)), np.zeros((1, 3, 3, 3)), None), "E must have the same rank as L"),
    ((np.zeros((4, 3, 2)), np.zeros((3, 3, 2)), None), "L must be square"),
    ((np.zeros((4, 3, 3)), np.zeros((3, 2, 2)), None), "E block dimensions must match"),
    ((np.zeros((2, 4, 3, 3)), np.zeros((3, 3, 3, 3)), None), "same batch size"),
    ((np.zeros((4, 3, 3)), np.zeros((3, 3, 3)), np.zeros((5, 3, 1))), "b horizon dimension must be 4"),
    ((np.zeros((4, 3, 3)), np.zeros((3, 3, 3)), np.zeros((4, 2, 1))), "b block dimension must be 3"),
    ((np.zeros((4, 3, 3)), np.zeros((3, 3, 3)), np.zeros((4, 3, 1), dtype=np.float32)), "same dtype"),
    ((np.zeros((4, 3, 3)), np.zeros((3, 3, 3), dtype=np.float32), None), "L and E must have same dtype"),
])
def test_validation_messages_match_the_reference(args, msg):
    with pytest.raises(ValueError, match=msg):
        sj._validate_problem_shapes(*args)


def test_entry_points_need_jax():
    if HAVE_JAX:
        pytest.skip("JAX present")
    with pytest.raises(ImportError, match="JAX"):
        sj.cholesky_factor(np.zeros((2, 1, 1)), np.zeros((1, 1, 1)))
