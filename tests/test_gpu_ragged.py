"""GPU: ragged batches of uneven (N, n, m) in one persistent launch."""
import numpy as np
import pytest
import torch

from oracle import generators, nd_cholesky as nd
from socu_b200.block_tridiag_solver import create_cholesky_factor_and_solve_launch
from socu_b200.problems import fill_ragged, ragged_shapes
from socu_b200.ragged import (RaggedBatch, create_ragged_factor_and_solve_launch,
                              create_ragged_refined_solve_launch)

pytestmark = pytest.mark.gpu
DEV = "cuda"

# edge cases: N = 1, 2, odd and power-of-two horizons, n = 1, odd n, n at the
# 32-tile boundary and the 64 limit, m up to 5
SHAPES = [(1, 8, 1), (2, 3, 2), (3, 1, 1), (7, 16, 4), (8, 17, 1), (31, 32, 4), (64, 48, 1), (100, 33, 5),
          (16, 64, 2), (5, 64, 1), (129, 8, 4), (40, 24, 3), (1, 64, 3), (2, 48, 4), (63, 12, 2), (17, 40, 1)]


def _problems(shapes, seed=3, shift=10.0):
    out = []
    for k, (N, n, m) in enumerate(shapes):
        L, E, b = generators.readme_problem(N, n, m, shift=shift, seed=seed + k)
        out.append((L, E, b))
    return out


def _batch(shapes, probs, dtype, refine=False, max_iter=10):
    N, n, m = (np.array([s[j] for s in shapes]) for j in range(3))
    rb = RaggedBatch(N, n, m, dtype=dtype, device=DEV, refine=refine, max_iter=max_iter)
    L, E, x = rb.pack([p[0] for p in probs], [p[1] for p in probs], [p[2] for p in probs])
    return rb, L, E, x


@pytest.mark.parametrize("graph", [False, True])
def test_ragged_fp64_matches_oracle_and_uniform_path(graph):
    probs = _problems(SHAPES)
    rb, L, E, x = _batch(SHAPES, probs, torch.float64)
    run = create_ragged_factor_and_solve_launch(rb, L, E, x, use_cuda_graph=graph)
    run()
    torch.cuda.synchronize()
    assert rb.error_flag() == 0
    for i, (L0, E0, b0) in enumerate(probs):
        Lo, Eo, xo = nd.nd_factor_and_solve(L0, E0, b0)
        xs = rb.x_view(x, i).cpu().numpy()
        scale = max(1.0, np.abs(xo).max())
        assert np.abs(xs - xo[0]).max() <= 1e-10 * scale, SHAPES[i]
        # factor: lower triangles of L and the coupling / fill-in slots
        Ls = rb.L_view(L, i).cpu().numpy()
        assert np.abs(np.tril(Ls) - np.tril(Lo[0])).max() <= 1e-10 * max(1.0, np.abs(Lo).max()), SHAPES[i]
        N = SHAPES[i][0]
        if N > 1:
            Es = rb.E_view(E, i).cpu().numpy()
            assert np.abs(Es - Eo[0]).max() <= 1e-10 * max(1.0, np.abs(Eo).max()), SHAPES[i]
        # uniform launch on the same instance (B = 1): same kernels, same data flow
        Lu, Eu, xu = (torch.tensor(a[None], device=DEV) for a in (L0, E0, b0))
        create_cholesky_factor_and_solve_launch(Lu, Eu, xu, use_cuda_graph=False)()
        torch.cuda.synchronize()
        assert float((rb.x_view(x, i) - xu[0]).abs().max()) <= 1e-12 * scale, SHAPES[i]


def test_ragged_fp32_plain_path():
    probs = _problems(SHAPES, seed=11)
    rb, L, E, x = _batch(SHAPES, probs, torch.float32)
    create_ragged_factor_and_solve_launch(rb, L, E, x)()
    torch.cuda.synchronize()
    assert rb.error_flag() == 0
    for i, (L0, E0, b0) in enumerate(probs):
        xo = nd.nd_factor_and_solve(L0, E0, b0)[2][0]
        xs = rb.x_view(x, i).double().cpu().numpy()
        assert np.abs(xs - xo).max() <= 2e-4 * max(1.0, np.abs(xo).max()), SHAPES[i]


@pytest.mark.parametrize("graph", [False, True])
def test_ragged_refine_reaches_fp64_backward_error(graph):
    probs = _problems(SHAPES, seed=21)
    rb, L, E, b = _batch(SHAPES, probs, torch.float64, refine=True, max_iter=10)
    L0c, E0c, b0c = L.clone(), E.clone(), b.clone()
    x = torch.full_like(b, float("nan"))
    run = create_ragged_refined_solve_launch(rb, L, E, b, x, tol=1e-12, use_cuda_graph=graph)
    run()
    torch.cuda.synchronize()
    assert rb.error_flag() == 0
    eta = run.eta.cpu().numpy()
    it = run.iterations.cpu().numpy()
    assert (eta <= 1e-12).all(), (eta, it)
    assert (it >= 1).all() and (it <= 10).all(), it
    assert torch.equal(L, L0c) and torch.equal(E, E0c) and torch.equal(b, b0c)
    for i, (L0, E0, b0) in enumerate(probs):
        xs = rb.x_view(x, i).cpu().numpy()
        # the kernel's eta against the oracle's backward error of the same x
        assert nd.backward_error(L0, E0, xs, b0)[0] <= 1e-12, SHAPES[i]
        xo = nd.nd_factor_and_solve(L0, E0, b0)[2][0]
        kappa = np.linalg.cond(generators.dense_from_blocks(L0, E0))
        err = np.abs(xs - xo).max() / max(1e-300, np.abs(xo).max())
        assert err <= 20 * kappa * 1e-12 + 1e-14, (SHAPES[i], err, kappa)


def test_ragged_reruns_are_bitwise_identical():
    shapes = SHAPES[:10]
    probs = _problems(shapes, seed=5)
    rb, L, E, x = _batch(shapes, probs, torch.float64)
    L0, E0, x0 = L.clone(), E.clone(), x.clone()
    run = create_ragged_factor_and_solve_launch(rb, L, E, x, use_cuda_graph=True)
    outs = []
    for _ in range(3):
        L.copy_(L0), E.copy_(E0), x.copy_(x0)
        run()
        torch.cuda.synchronize()
        outs.append((L.clone(), E.clone(), x.clone()))
    for o in outs[1:]:
        assert all(torch.equal(a, c) for a, c in zip(o, outs[0]))
    assert rb.error_flag() == 0


def test_ragged_refine_stops_on_breakdown():
    # shift 0.1 makes D_chol nearly singular for n = 64: the float factor of
    # some instances breaks down, which must end those instances with
    # iters < 0 instead of hanging or poisoning the others
    shapes = [(40, 64, 1), (20, 16, 2), (30, 64, 1)]
    probs = [generators.readme_problem(40, 64, 1, shift=0.1, seed=1),
             generators.readme_problem(20, 16, 2, shift=10.0, seed=2),
             generators.readme_problem(30, 64, 1, shift=0.1, seed=3)]
    rb, L, E, b = _batch(shapes, probs, torch.float64, refine=True, max_iter=6)
    x = torch.zeros_like(b)
    run = create_ragged_refined_solve_launch(rb, L, E, b, x, tol=1e-12, use_cuda_graph=False)
    run()
    torch.cuda.synchronize()
    assert rb.error_flag() == 0
    it = run.iterations.cpu().numpy()
    eta = run.eta.cpu().numpy()
    assert 1 <= it[1] <= 6 and eta[1] <= 1e-12
    for k in (0, 2):
        assert it[k] < 0 or (1 <= it[k] <= 6), it


def _torch_backward_error(rb, L, E, x, b):
    """Per-instance normwise backward error with torch block products."""
    out = torch.empty(rb.count, dtype=torch.float64)
    for i in range(rb.count):
        N = int(rb.horizons[i])
        D = rb.L_view(L, i)
        Dl = torch.tril(D)
        Ds = Dl + torch.tril(D, -1).transpose(-1, -2)
        Ei = rb.E_view(E, i)[:N - 1]
        xi, bi = rb.x_view(x, i), rb.x_view(b, i)
        y = Ds @ xi
        if N > 1:
            y[1:] += Ei @ xi[:-1]
            y[:-1] += Ei.transpose(-1, -2) @ xi[1:]
        r = (bi - y).abs().max()
        rows = Ds.abs().sum(-1)
        if N > 1:
            rows[1:] += Ei.abs().sum(-1)
            rows[:-1] += Ei.abs().sum(-2)
        den = rows.max() * xi.abs().max() + bi.abs().max()
        out[i] = float(r / den)
    return out


def test_ragged_mpc_batch_4096_instances():
    """4096 instances, N ~ U{8..256}, n in {8,16,32,48}, m in {1,4}, shift 10:
    FP64 plain and mixed+refine, every instance checked."""
    N, n, m = ragged_shapes(0, 4096)
    plain = RaggedBatch(N, n, m, dtype=torch.float64, device=DEV)
    L, E, b = plain.empty()
    fill_ragged(plain, L, E, b, seed=0)
    mixed = RaggedBatch(N, n, m, dtype=torch.float64, device=DEV, refine=True, max_iter=10)
    x = torch.zeros_like(b)
    run = create_ragged_refined_solve_launch(mixed, L, E, b, x, tol=1e-12)
    run()
    torch.cuda.synchronize()
    assert mixed.error_flag() == 0
    assert float(run.eta.max()) <= 1e-12
    it = run.iterations
    assert int(it.min()) >= 1 and int(it.max()) <= 10
    eta_mixed = _torch_backward_error(plain, L, E, x, b)
    assert float(eta_mixed.max()) <= 1e-12
    Lf, Ef, xf = L.clone(), E.clone(), b.clone()
    create_ragged_factor_and_solve_launch(plain, Lf, Ef, xf)()
    torch.cuda.synchronize()
    assert plain.error_flag() == 0
    eta_plain = _torch_backward_error(plain, L, E, xf, b)
    assert float(eta_plain.max()) <= 1e-13
    # both paths solve the same systems
    scale = float(xf.abs().max())
    assert float((x - xf).abs().max()) <= 1e-6 * scale
