"""Per-instance factor status (needs a B200).

The reference has no numerical status: its potrf takes the square root of
whatever pivot it meets (socu/blas/potrf.py:97-117), so a non-SPD instance
silently yields NaN.  The `info` extension reports, per batch entry, 0 or
1 + the first failing node in elimination order (lowest separator level, then
lowest block index).  Cases: an SPD instance (0); two level-0 nodes made
negative definite (the lower index is reported); a level-1 node whose Schur
complement is indefinite while every level-0 node is fine (failures it causes
at higher levels are not reported); a masked-out instance (0).  The SPD
instances' results must not change when info is requested.
"""
import numpy as np
import pytest
import torch

from oracle import generators
from socu_b200 import _lib
from socu_b200.block_tridiag_solver import create_cholesky_factor_and_solve_launch, create_cholesky_factor_launch

pytestmark = pytest.mark.gpu
N, n, m = 20, 8, 2


def _batch(dtype):
    Ls, Es, bs = [], [], []
    for k in range(5):
        L, E, b = generators.readme_problem(N, n, m, shift=10.0, seed=40 + k)
        Ls.append(L); Es.append(E); bs.append(b)
    Ls[1][4] = -Ls[1][4]          # level-0 nodes 4 and 10 fail: report node 4
    Ls[1][10] = -Ls[1][10]
    Ls[3][1] = 1e-6 * np.eye(n)   # level-1 node 1: 1e-6 I - F F^T - G^T G is indefinite
    dev = "cuda"
    return tuple(torch.tensor(np.stack(a), dtype=dtype, device=dev) for a in (Ls, Es, bs))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("use_cuda_graph", [False, True])
def test_info_reports_first_failing_node(dtype, use_cuda_graph):
    L0, E0, b0 = _batch(dtype)
    mask = torch.tensor([1, 1, 1, 1, 0], dtype=torch.bool, device="cuda")
    info = torch.full((5,), -7, dtype=torch.int32, device="cuda")
    L, E, x = L0.clone(), E0.clone(), b0.clone()
    run = create_cholesky_factor_and_solve_launch(L, E, x, mask=mask, dtype=dtype, use_cuda_graph=use_cuda_graph,
                                                  info=info)
    run()
    torch.cuda.synchronize()
    assert info.tolist() == [0, 5, 0, 2, 0]
    assert torch.isfinite(x[[0, 2]]).all()
    assert torch.equal(x[4], b0[4])        # masked out: untouched
    # same SPD results without info
    L2, E2, x2 = L0.clone(), E0.clone(), b0.clone()
    create_cholesky_factor_and_solve_launch(L2, E2, x2, mask=mask, dtype=dtype)()
    assert torch.equal(x[[0, 2]], x2[[0, 2]]) and torch.equal(L[[0, 2]], L2[[0, 2]])
    # every run rewrites info
    info.fill_(-7)
    L.copy_(L0); E.copy_(E0); x.copy_(b0)
    L[1] = L0[0]
    E[1] = E0[0]     # instance 1 becomes a copy of the SPD instance 0
    run()
    torch.cuda.synchronize()
    assert info.tolist() == [0, 0, 0, 2, 0]


def test_info_through_the_c_abi_and_factor_only():
    L0, E0, b0 = _batch(torch.float64)
    lib = _lib.load()
    info = torch.full((5,), -1, dtype=torch.int32, device="cuda")
    L, E = L0.clone(), E0.clone()
    st = lib.socu_cholesky_run_info(_lib.OP_FACTOR, _lib.FLOAT64, L.data_ptr(), E.data_ptr(), None, None,
                                    info.data_ptr(), 5, N, n, 0, torch.cuda.current_stream().cuda_stream)
    assert st == 0
    torch.cuda.synchronize()
    assert info.tolist() == [0, 5, 0, 2, 0]
    # info is only defined for the factor ops
    x = b0.clone()
    st = lib.socu_cholesky_run_info(_lib.OP_SOLVE, _lib.FLOAT64, L.data_ptr(), E.data_ptr(), x.data_ptr(), None,
                                    info.data_ptr(), 5, N, n, m, None)
    assert st == -1
    info2 = torch.zeros(5, dtype=torch.int32, device="cuda")
    L, E = L0.clone(), E0.clone()
    create_cholesky_factor_launch(L, E, info=info2, keep_inverse=True)()
    torch.cuda.synchronize()
    assert info2.tolist() == [0, 5, 0, 2, 0]
