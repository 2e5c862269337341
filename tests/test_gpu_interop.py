"""Arrays from other CUDA libraries (needs a B200).

The reference factories take Warp arrays; a Warp user switching over keeps
passing them (socu README.md:214-235: L, E, x as wp.array, the batch mask as a
wp.bool array whose contents may change between calls, also under a CUDA
graph).  Any object exposing __cuda_array_interface__ is accepted and used
in place, without a copy.  Here plain wrapper objects stand in for Warp arrays
(Warp is not installed): they expose only __cuda_array_interface__ (and, for
the mask, a dtype named "bool", typestr "|b1" as a wp.bool array reports).
"""
import numpy as np
import pytest
import torch

from oracle import generators
from socu_b200.block_tridiag_solver import (create_cholesky_backward_substitution_launch,
                                            create_cholesky_factor_and_solve_launch, create_cholesky_factor_launch,
                                            create_cholesky_forward_substitution_launch, create_cholesky_solve_launch)

pytestmark = pytest.mark.gpu


class CudaArray:
    """Minimal foreign CUDA array: memory owned elsewhere, described by the
    __cuda_array_interface__ protocol (version 3) only."""

    def __init__(self, t: torch.Tensor, dtype_name=None):
        self._t = t
        self.dtype = dtype_name or str(t.dtype).replace("torch.", "")
        self.shape = tuple(t.shape)
        self.ndim = t.ndim

    @property
    def __cuda_array_interface__(self):
        return self._t.__cuda_array_interface__


class WarpBoolMask(CudaArray):
    """A uint8 buffer described as booleans, as a wp.bool array is."""

    @property
    def __cuda_array_interface__(self):
        cai = dict(self._t.__cuda_array_interface__)
        cai["typestr"] = "|b1"
        return cai


def _inputs(B, N, n, m, seed=0):
    Ls, Es, bs = [], [], []
    for k in range(B):
        L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=seed + k)
        Ls.append(L); Es.append(E); bs.append(b)
    dev = "cuda"
    return (torch.tensor(np.stack(Ls), device=dev), torch.tensor(np.stack(Es), device=dev),
            torch.tensor(np.stack(bs), device=dev))


@pytest.mark.parametrize("use_cuda_graph", [False, True])
def test_all_five_factories_accept_cuda_array_interface(use_cuda_graph):
    B, N, n, m = 2, 20, 12, 3
    L0, E0, b0 = _inputs(B, N, n, m)
    # torch tensors: the expected results
    L, E, x = L0.clone(), E0.clone(), b0.clone()
    create_cholesky_factor_and_solve_launch(L, E, x)()
    xs = b0.clone()
    create_cholesky_solve_launch(L, E, xs)()
    torch.cuda.synchronize()
    # the same through wrapper objects, memory shared with the wrapped tensors
    Lw, Ew, xw = L0.clone(), E0.clone(), b0.clone()
    kw = dict(use_cuda_graph=use_cuda_graph)
    A, Ea, Xa = CudaArray(Lw), CudaArray(Ew), CudaArray(xw)
    create_cholesky_factor_launch(A, Ea, **kw)()
    for fn in (create_cholesky_forward_substitution_launch, create_cholesky_backward_substitution_launch):
        fn(A, Ea, Xa, **kw)()
    torch.cuda.synchronize()
    assert torch.equal(torch.tril(Lw), torch.tril(L)) and torch.equal(Ew, E)
    assert float((xw - xs).abs().max()) <= 1e-12 * float(xs.abs().max())
    xw.copy_(b0)
    create_cholesky_solve_launch(A, Ea, Xa, **kw)()
    torch.cuda.synchronize()
    assert torch.equal(xw, xs)
    Lw.copy_(L0); Ew.copy_(E0); xw.copy_(b0)
    create_cholesky_factor_and_solve_launch(A, Ea, Xa, **kw)()
    torch.cuda.synchronize()
    assert torch.equal(xw, x)


@pytest.mark.parametrize("use_cuda_graph", [False, True])
def test_bool_mask_from_foreign_array_updated_in_place(use_cuda_graph):
    B, N, n, m = 3, 9, 10, 2
    L0, E0, b0 = _inputs(B, N, n, m, seed=7)
    mbuf = torch.tensor([1, 0, 1], dtype=torch.uint8, device="cuda")
    mask = WarpBoolMask(mbuf, dtype_name="bool")
    L, E, x = L0.clone(), E0.clone(), b0.clone()
    run = create_cholesky_factor_and_solve_launch(CudaArray(L), CudaArray(E), CudaArray(x), mask=mask,
                                                  use_cuda_graph=use_cuda_graph)
    run()
    torch.cuda.synchronize()
    assert torch.equal(L[1], L0[1]) and torch.equal(E[1], E0[1]) and torch.equal(x[1], b0[1])
    assert not torch.equal(x[0], b0[0]) and not torch.equal(x[2], b0[2])
    ref = x.clone()
    # flip the mask in place: the bound launch (and its graph) must read it anew
    L.copy_(L0); E.copy_(E0); x.copy_(b0)
    mbuf.copy_(torch.tensor([0, 1, 0], dtype=torch.uint8))
    run()
    torch.cuda.synchronize()
    assert torch.equal(x[0], b0[0]) and torch.equal(x[2], b0[2])
    assert not torch.equal(x[1], b0[1])
    mbuf.fill_(1)
    L.copy_(L0); E.copy_(E0); x.copy_(b0)
    run()
    torch.cuda.synchronize()
    assert torch.equal(x[0], ref[0]) and torch.equal(x[2], ref[2])


def test_non_bool_mask_rejected_like_the_reference():
    L0, E0, b0 = _inputs(2, 5, 4, 1)
    bad = CudaArray(torch.ones(2, dtype=torch.int32, device="cuda"))
    with pytest.raises(AssertionError, match="wp.bool"):
        create_cholesky_factor_and_solve_launch(CudaArray(L0), CudaArray(E0), CudaArray(b0), mask=bad)
