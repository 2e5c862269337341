"""GPU parity of the drop-in API against the oracle (needs a B200).

Mirrors socu's tests/test_block_tridiag_solver.py: the same generator, grid
(N x n x dtype x graph), sequences (factor+solve, factor_and_solve,
factor+forward+backward), tolerances (1e-10 f64, 1e-4 f32, absolute 2-norms)
and mask semantics, plus exact factor-layout parity with the oracle and
run-to-run bitwise determinism.
"""
import ctypes
import functools

import numpy as np
import pytest
import torch

from oracle import dense, generators, nd_cholesky as nd
from socu_b200 import _lib
from socu_b200.block_tridiag_solver import (
    calculate_off_diag_storage_len,
    create_cholesky_backward_substitution_launch,
    create_cholesky_factor_and_solve_launch,
    create_cholesky_factor_launch,
    create_cholesky_forward_substitution_launch,
    create_cholesky_solve_launch,
)

pytestmark = pytest.mark.gpu

TOLERANCE = {torch.float32: 1e-4, torch.float64: 1e-10}
DEV = "cuda"


@functools.lru_cache(maxsize=None)
def problem(n, N):
    """Reference test inputs and the oracle's solution/factor (float64 numpy)."""
    _, L, E, b = generators.reference_test_problem(n, N)
    Lf, Ef, x = nd.nd_factor_and_solve(L, E, b.reshape(N, n, 1))
    if n * N <= 1500:  # dense check of the oracle itself on small cases
        A = generators.dense_from_blocks(L, E)
        assert np.linalg.norm(x.ravel() - dense.reference_solution(A, b)) < 1e-10
    return L, E, b, x[0].ravel(), Lf[0], Ef[0]


def residual(L, E, b, x):
    N, n = L.shape[0], L.shape[1]
    return np.linalg.norm(b - nd.block_tridiag_matmul(L, E, x.reshape(N, n, 1)).ravel())


def t(a, dtype):
    return torch.tensor(a, dtype=dtype, device=DEV)


@pytest.mark.parametrize("N", [1, 2, 3, 4, 7, 8, 20, 100])
@pytest.mark.parametrize("use_cuda_graph", [False, True])
@pytest.mark.parametrize("n", [1, 10, 32, 36, 64, 68])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_cholesky_solver(n, N, use_cuda_graph, dtype):
    tol = TOLERANCE[dtype]
    L_np, E_np, b_np, x_ref, _, _ = problem(n, N)
    L, E, x = t(L_np, dtype), t(E_np, dtype), t(b_np.reshape(N, n, 1), dtype)
    kw = dict(use_cuda_graph=use_cuda_graph, dtype=dtype)
    factor = create_cholesky_factor_launch(L, E, **kw)
    solve = create_cholesky_solve_launch(L, E, x, **kw)
    factor_and_solve = create_cholesky_factor_and_solve_launch(L, E, x, **kw)
    forward = create_cholesky_forward_substitution_launch(L, E, x, **kw)
    backward = create_cholesky_backward_substitution_launch(L, E, x, **kw)

    def reset():
        L.copy_(t(L_np, dtype)); E.copy_(t(E_np, dtype)); x.copy_(t(b_np.reshape(N, n, 1), dtype))

    reset()
    factor(); solve()
    xr = x.double().cpu().numpy().ravel()
    assert np.linalg.norm(x_ref - xr) < tol
    assert residual(L_np, E_np, b_np, xr) < tol

    reset()
    factor_and_solve()
    xc = x.double().cpu().numpy().ravel()
    assert np.linalg.norm(x_ref - xc) < tol
    assert residual(L_np, E_np, b_np, xc) < tol
    assert np.linalg.norm(xr - xc) < tol

    # L, E hold the factor from factor_and_solve
    x.copy_(t(b_np.reshape(N, n, 1), dtype))
    forward(); backward()
    xs = x.double().cpu().numpy().ravel()
    assert np.linalg.norm(xr - xs) < tol


@pytest.mark.parametrize("n,N", [(1, 7), (10, 20), (32, 8), (36, 100), (64, 20), (68, 7)])
def test_factor_layout_matches_oracle(n, N):
    """The in-place factor equals the oracle's block by block (lower(L), all of E)."""
    L_np, E_np, _, _, Lf, Ef = problem(n, N)
    L, E = t(L_np, torch.float64), t(E_np, torch.float64)
    create_cholesky_factor_launch(L, E)()
    Lg = np.tril(L.cpu().numpy())
    assert np.abs(Lg - np.tril(Lf)).max() <= 1e-10 * np.abs(Lf).max()
    if Ef.shape[0]:
        assert np.abs(E.cpu().numpy() - Ef).max() <= 1e-10 * max(1.0, np.abs(Ef).max())


def test_oracle_factor_solved_on_gpu():
    """A factor produced elsewhere (the oracle, upper triangles zero) is solved
    correctly: the sweeps read only the lower triangle."""
    n, N = 36, 20
    L_np, E_np, b_np, x_ref, Lf, Ef = problem(n, N)
    L, E, x = t(Lf, torch.float64), t(Ef, torch.float64), t(b_np.reshape(N, n, 1), torch.float64)
    create_cholesky_solve_launch(L, E, x)()
    assert np.linalg.norm(x.cpu().numpy().ravel() - x_ref) < 1e-10


@pytest.mark.parametrize("N", [1, 7, 20])
@pytest.mark.parametrize("use_cuda_graph", [False, True])
@pytest.mark.parametrize("n", [10, 36])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_cholesky_solver_mask(n, N, use_cuda_graph, dtype):
    """Active batch entries are solved, inactive ones are left bit-identical;
    the mask is updated in place between runs (captured graphs must see it)."""
    B = 4
    L1, E1, b1, x_ref, _, _ = problem(n, N)
    L_np = np.tile(L1, (B, 1, 1, 1)); E_np = np.tile(E1, (B, 1, 1, 1))
    b_np = np.tile(b1.reshape(N, n, 1), (B, 1, 1, 1))
    L, E, x = t(L_np, dtype), t(E_np, dtype), t(b_np, dtype)
    mask = torch.zeros(B, dtype=torch.bool, device=DEV)
    kw = dict(use_cuda_graph=use_cuda_graph, dtype=dtype)
    factor = create_cholesky_factor_launch(L, E, mask, **kw)
    solve = create_cholesky_solve_launch(L, E, x, mask, **kw)
    factor_and_solve = create_cholesky_factor_and_solve_launch(L, E, x, mask, **kw)
    forward = create_cholesky_forward_substitution_launch(L, E, x, mask, **kw)
    backward = create_cholesky_backward_substitution_launch(L, E, x, mask, **kw)
    sequences = {
        "factor + solve": [factor, solve],
        "factor_and_solve": [factor_and_solve],
        "factor + forward + backward": [factor, forward, backward],
    }
    for mask_np in ([True, False, True, False], [False, True, False, True]):
        mask.copy_(torch.tensor(mask_np))
        for name, launches in sequences.items():
            for arr, ref in ((L, L_np), (E, E_np), (x, b_np)):
                arr.copy_(t(ref, dtype))
            for launch in launches:
                launch()
            outs = ((L.cpu().numpy(), L_np), (E.cpu().numpy(), E_np), (x.cpu().numpy(), b_np))
            for k, active in enumerate(mask_np):
                if active:
                    err = np.linalg.norm(x_ref - outs[2][0][k].astype(np.float64).ravel())
                    assert err < TOLERANCE[dtype], f"{name}, batch {k}: {err}"
                else:
                    for out, ref in outs:
                        np.testing.assert_array_equal(out[k], ref[k].astype(out.dtype),
                                                      err_msg=f"{name}: inactive entry {k} modified")


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_deterministic_bitwise(dtype):
    """No floating-point atomics: two runs give bit-identical factors and solutions."""
    n, N, B, m = 36, 100, 3, 4
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0, seed=7)
    outs = []
    for _ in range(2):
        L = t(np.tile(L_np, (B, 1, 1, 1)), dtype); E = t(np.tile(E_np, (B, 1, 1, 1)), dtype)
        x = t(np.tile(b_np, (B, 1, 1, 1)), dtype)
        create_cholesky_factor_and_solve_launch(L, E, x, dtype=dtype)()
        outs.append((L.cpu(), E.cpu(), x.cpu()))
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)


def test_c_abi_direct_call():
    """The C ABI used without the Python layer: raw pointers, sizes, stream."""
    lib = _lib.load()
    n, N, m, B = 32, 20, 3, 2
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0, seed=11)
    L = t(np.tile(L_np, (B, 1, 1, 1)), torch.float64)
    E = t(np.tile(E_np, (B, 1, 1, 1)), torch.float64)
    x = t(np.tile(b_np, (B, 1, 1, 1)), torch.float64)
    s = torch.cuda.current_stream().cuda_stream
    assert lib.socu_cholesky_factor(_lib.FLOAT64, L.data_ptr(), E.data_ptr(), None, B, N, n, s) == 0
    assert lib.socu_cholesky_solve(_lib.FLOAT64, L.data_ptr(), E.data_ptr(), x.data_ptr(), None,
                                   B, N, n, m, s) == 0
    torch.cuda.synchronize()
    A = generators.dense_from_blocks(L_np, E_np)
    x_ref = np.linalg.solve(A, b_np.reshape(N * n, m)).reshape(N, n, m)
    for k in range(B):
        assert np.abs(x[k].cpu().numpy() - x_ref).max() < 1e-10


@pytest.mark.parametrize("path", ["readme_N100_n8_m1_s10", "readme_N33_n12_m3_s10", "ref_n36_N7",
                                  "readme_N17_n5_m2_s10"])
def test_golden_fixtures(path):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", path + ".npz"))
    L_np, E_np, b_np, x_ref = g["L"], g["E"], g["b"], g["x_ref"]
    N, n = L_np.shape[:2]
    b3 = b_np.reshape(N, n, -1)
    L, E, x = t(L_np, torch.float64), t(E_np, torch.float64), t(b3, torch.float64)
    create_cholesky_factor_and_solve_launch(L, E, x)()
    assert np.abs(x.cpu().numpy() - x_ref.reshape(b3.shape)).max() <= 1e-10 * max(1, np.abs(x_ref).max())
    assert np.abs(np.tril(L.cpu().numpy()) - g["L_fac"]).max() <= 1e-10 * np.abs(g["L_fac"]).max()
    if g["E_fac"].size:
        assert np.abs(E.cpu().numpy() - g["E_fac"]).max() <= 1e-10 * np.abs(g["E_fac"]).max()


@pytest.mark.parametrize("n,m", [(128, 32), (100, 40), (48, 1)])
def test_large_blocks_and_wide_rhs(n, m):
    """Largest block size of the configs (n=128) and more RHS than one pass."""
    N = 9
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0, seed=5)
    L, E, x = t(L_np, torch.float64), t(E_np, torch.float64), t(b_np, torch.float64)
    create_cholesky_factor_and_solve_launch(L, E, x)()
    _, _, xo = nd.nd_factor_and_solve(L_np, E_np, b_np)
    assert np.abs(x.cpu().numpy() - xo[0]).max() <= 1e-10 * max(1, np.abs(xo).max())


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("n,m", [(100, 3), (128, 32), (128, 40)])
def test_streamed_sweeps_large_blocks(dtype, n, m):
    """Blocks too large to stay resident in shared memory: the sweeps stream the
    coupling blocks in 32-column chunks through DMMA products.  Forward +
    backward on a stored factor and factor_and_solve against the oracle."""
    N = 21
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0 + 2.0 * np.sqrt(n), seed=n + m)
    _, _, xo = nd.nd_factor_and_solve(L_np, E_np, b_np)
    tol = TOLERANCE[dtype]
    scale = max(1.0, np.abs(xo).max())
    L, E, x = t(L_np, dtype), t(E_np, dtype), t(b_np, dtype)
    create_cholesky_factor_launch(L, E, dtype=dtype)()
    create_cholesky_forward_substitution_launch(L, E, x, dtype=dtype)()
    create_cholesky_backward_substitution_launch(L, E, x, dtype=dtype)()
    assert np.abs(x.double().cpu().numpy() - xo[0]).max() <= tol * scale
    L, E, x = t(L_np, dtype), t(E_np, dtype), t(b_np, dtype)
    create_cholesky_factor_and_solve_launch(L, E, x, dtype=dtype, use_cuda_graph=True)()
    assert np.abs(x.double().cpu().numpy() - xo[0]).max() <= tol * scale


@pytest.mark.parametrize("n", [48, 64, 61])
def test_register_chain_matches_shared_chain_bitwise(n):
    """The float inverse-first node keeps its trailing tiles in registers when
    they fit (2 per thread: 256-thread CTAs here); with 64-thread CTAs they do
    not and the shared-memory chain runs.  Same operations in the same order:
    the factors and solutions must agree bit for bit, and with the oracle."""
    from socu_b200.block_tridiag_solver import _launch_with_settings

    N, m = 29, 5
    L0, E0, b0 = generators.readme_problem(N, n, m, shift=10.0 + 2.0 * np.sqrt(n), seed=7 + n)
    outs = []
    for threads in (256, 64):
        L, E, x = (torch.tensor(a, dtype=torch.float32, device=DEV) for a in (L0, E0, b0))
        _launch_with_settings("factor_and_solve", L, E, x, torch.float32, {"node_threads": threads})()
        torch.cuda.synchronize()
        outs.append((L, E, x))
    for a, b in zip(outs[0], outs[1]):
        assert torch.equal(a, b)
    x_ref = nd.nd_factor_and_solve(L0, E0, b0)[2][0]
    assert np.abs(outs[0][2].double().cpu().numpy() - x_ref).max() <= 1e-4 * max(1.0, np.abs(x_ref).max())
