"""The tcgen05 tensor-core building block of the float path (needs a B200).

socu_tc_selftest runs one CTA through the same staging (TF32 hi/lo split into
the K-major core-matrix layout), shared-memory and instruction descriptors,
tcgen05.mma issue, commit-to-mbarrier and tensor-memory loads as the solver's
tensor-core kernels.  D = A B^T must match an FP64 product to FP32 accuracy
(3xTF32: relative error ~1e-6 of |A| |B|), with no wait running out.
"""
import pytest
import torch

from socu_b200 import _lib

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("N,K", [(16, 8), (64, 64), (128, 64), (64, 128), (32, 152)])
def test_tc_gemm_matches_fp64(N, K):
    lib = _lib.load()
    g = torch.Generator(device="cuda").manual_seed(N * 1000 + K)
    A = torch.randn(128, K, device="cuda", generator=g)
    B = torch.randn(N, K, device="cuda", generator=g)
    D = torch.full((128, N), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = lib.socu_tc_selftest(A.data_ptr(), B.data_ptr(), D.data_ptr(), 128, N, K, err.data_ptr(),
                              torch.cuda.current_stream().cuda_stream)
    assert st == 0, lib.socu_status_string(st)
    torch.cuda.synchronize()
    assert int(err) == 0
    ref = A.double() @ B.double().T
    scale = (A.double().abs() @ B.double().abs().T)
    rel = float(((D.double() - ref).abs() / scale).max())
    assert rel <= 2e-5, rel   # FP32 accumulation over K terms; one TF32 pass would give ~1e-3
    # a single TF32 pass would be ~1e-3 off: the split really runs
    assert torch.isfinite(D).all()


def test_tc_m64_accumulator_lanes():
    """An M = 64 accumulator occupies lanes 0-15 of each of the four 32-lane
    sub-partitions of tensor memory: row r sits in lane 32 (r // 16) + r % 16."""
    lib = _lib.load()
    N, K = 32, 16
    g = torch.Generator(device="cuda").manual_seed(7)
    A = torch.randn(64, K, device="cuda", generator=g)
    B = torch.randn(N, K, device="cuda", generator=g)
    D = torch.zeros(128, N, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.socu_tc_selftest(A.data_ptr(), B.data_ptr(), D.data_ptr(), 64, N, K, err.data_ptr(), None) == 0
    torch.cuda.synchronize()
    assert int(err) == 0
    ref = A.double() @ B.double().T
    lanes = torch.tensor([32 * (r // 16) + r % 16 for r in range(64)], device="cuda")
    rel = float(((D[lanes].double() - ref).abs() / (A.double().abs() @ B.double().abs().T)).max())
    assert rel <= 2e-5, rel


@pytest.mark.parametrize("n", [16, 48, 64, 68, 100, 128])
@pytest.mark.parametrize("op", ["factor_and_solve", "factor+solve"])
def test_tc_update_parity(n, op):
    """Float factor with the Schur updates on the tensor cores (update_tensor_cores=1)
    against the oracle at the reference's float tolerance, no wait running out."""
    import numpy as np

    from oracle import generators, nd_cholesky as nd
    from socu_b200.block_tridiag_solver import _launch_with_settings

    N = 21
    L_np, E_np, b_np = generators.readme_problem(N, n, 3, shift=10.0 + 2.0 * np.sqrt(n), seed=n)
    _, _, x_ref = nd.nd_factor_and_solve(L_np, E_np, b_np)
    L, E, x = (torch.tensor(a, dtype=torch.float32, device="cuda") for a in (L_np, E_np, b_np))
    settings = {"update_tensor_cores": 1}
    if op == "factor_and_solve":
        _launch_with_settings("factor_and_solve", L, E, x, torch.float32, settings)()
    else:
        _launch_with_settings("factor", L, E, None, torch.float32, settings)()
        _launch_with_settings("solve", L, E, x, torch.float32, settings)()
    torch.cuda.synchronize()
    lib = _lib.load()
    import ctypes
    flag = ctypes.c_int(0)
    assert lib.socu_tc_error(ctypes.byref(flag), 1) == 0 and flag.value == 0
    rel = np.abs(x.double().cpu().numpy() - x_ref[0]).max() / np.abs(x_ref).max()
    assert rel < 1e-4, rel


@pytest.mark.parametrize("n,m", [(8, 1), (16, 4), (32, 8), (48, 3), (64, 8), (64, 40), (68, 2), (100, 5), (128, 32)])
@pytest.mark.parametrize("op", ["factor_and_solve", "factor+solve"])
def test_tc_node_parity(n, m, op):
    """Float level nodes with their products on the tensor cores (node_tensor_cores=1),
    alone and together with the tensor-core Schur update, against the oracle."""
    import ctypes

    import numpy as np

    from oracle import generators, nd_cholesky as nd
    from socu_b200.block_tridiag_solver import _launch_with_settings

    N = 37
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0 + 2.0 * np.sqrt(n), seed=100 + n)
    _, _, x_ref = nd.nd_factor_and_solve(L_np, E_np, b_np)
    lib = _lib.load()
    for settings in ({"node_tensor_cores": 1}, {"node_tensor_cores": 1, "update_tensor_cores": 1}):
        L, E, x = (torch.tensor(a, dtype=torch.float32, device="cuda") for a in (L_np, E_np, b_np))
        if op == "factor_and_solve":
            _launch_with_settings("factor_and_solve", L, E, x, torch.float32, settings)()
        else:
            _launch_with_settings("factor", L, E, None, torch.float32, settings)()
            _launch_with_settings("solve", L, E, x, torch.float32, settings)()
        torch.cuda.synchronize()
        flag = ctypes.c_int(0)
        assert lib.socu_tc_error(ctypes.byref(flag), 1) == 0 and flag.value == 0
        rel = np.abs(x.double().cpu().numpy() - x_ref[0]).max() / np.abs(x_ref).max()
        assert rel < 1e-4, (settings, rel)


@pytest.mark.parametrize("node_tc", [1, 4])
@pytest.mark.parametrize("n,m", [(32, 4), (64, 8), (128, 8), (96, 32)])
def test_refined_solve_with_tensor_cores(n, m, node_tc):
    """The mixed solve's float factor on the tensor cores (tuned table entry)
    still reaches the FP64 backward-error bound."""
    import numpy as np

    from oracle import generators, nd_cholesky as nd
    from socu_b200 import autotune
    from socu_b200.mixed import create_cholesky_refined_solve_launch

    N = 64
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0 + 2.0 * np.sqrt(n), seed=3)
    L, E, b = (torch.tensor(a, device="cuda") for a in (L_np, E_np, b_np))
    autotune.install(torch.float32, n, m, {"node_tensor_cores": node_tc, "update_tensor_cores": 1})
    try:
        x = torch.zeros_like(b)
        run = create_cholesky_refined_solve_launch(L, E, b, x, tol=1e-12, max_iter=10)
        run()
        torch.cuda.synchronize()
    finally:
        autotune.install(torch.float32, n, m, None)
    assert float(run.eta.max()) <= 1e-12, (float(run.eta.max()), int(run.iterations.max()))
    assert nd.backward_error(L_np, E_np, x.cpu().numpy(), b_np)[0] <= 1e-12


@pytest.mark.parametrize("n,m", [(72, 1), (96, 5), (100, 3), (128, 32), (128, 1), (120, 64)])
@pytest.mark.parametrize("op", ["factor_and_solve", "factor+solve"])
def test_tmem_node_parity(n, m, op):
    """Float level nodes with 64 < n <= 128 resident in tensor memory, trailing
    updates on the tensor cores (node_tensor_cores=4), alone and with the
    tensor-core Schur update: solution and factor layout against the oracle."""
    import ctypes

    import numpy as np

    from oracle import generators, nd_cholesky as nd
    from socu_b200.block_tridiag_solver import _launch_with_settings

    N = 37
    L_np, E_np, b_np = generators.readme_problem(N, n, m, shift=10.0 + 2.0 * np.sqrt(n), seed=200 + n)
    Lf_ref, Ef_ref, x_ref = nd.nd_factor_and_solve(L_np, E_np, b_np)
    lib = _lib.load()
    for settings in ({"node_tensor_cores": 4}, {"node_tensor_cores": 4, "update_tensor_cores": 1}):
        L, E, x = (torch.tensor(a, dtype=torch.float32, device="cuda") for a in (L_np, E_np, b_np))
        if op == "factor_and_solve":
            _launch_with_settings("factor_and_solve", L, E, x, torch.float32, settings)()
        else:
            _launch_with_settings("factor", L, E, None, torch.float32, settings)()
            torch.cuda.synchronize()
            # factor layout: lower(L_i) = C_i with a zero upper triangle, E as the oracle's
            Lh = L.double().cpu().numpy()
            assert np.array_equal(np.triu(Lh, 1), np.zeros_like(Lh))
            assert np.abs(Lh - Lf_ref[0]).max() <= 1e-4 * np.abs(Lf_ref).max()
            assert np.abs(E.double().cpu().numpy() - Ef_ref[0]).max() <= 1e-4 * max(1.0, np.abs(Ef_ref).max())
            _launch_with_settings("solve", L, E, x, torch.float32, settings)()
        torch.cuda.synchronize()
        flag = ctypes.c_int(0)
        assert lib.socu_tc_error(ctypes.byref(flag), 1) == 0 and flag.value == 0
        rel = np.abs(x.double().cpu().numpy() - x_ref[0]).max() / np.abs(x_ref).max()
        assert rel < 1e-4, (settings, rel)


@pytest.mark.parametrize("use_cuda_graph", [False, True])
def test_tmem_node_info_and_mask(use_cuda_graph):
    """node_tensor_cores=4 reports the first failing node (here a negated level-0
    block, node 6) and leaves masked-out instances untouched."""
    import numpy as np

    from oracle import generators
    from socu_b200.block_tridiag_solver import _launch_with_settings

    N, n, m = 20, 96, 3
    P = [generators.readme_problem(N, n, m, shift=30.0, seed=60 + k) for k in range(3)]
    L0, E0, b0 = (np.stack([q[i] for q in P]) for i in range(3))
    L0[1][6] = -L0[1][6]
    L, E, x = (torch.tensor(a, dtype=torch.float32, device="cuda") for a in (L0, E0, b0))
    mask = torch.tensor([1, 1, 0], dtype=torch.bool, device="cuda")
    info = torch.full((3,), -7, dtype=torch.int32, device="cuda")
    _launch_with_settings("factor_and_solve", L, E, x, torch.float32, {"node_tensor_cores": 4}, mask=mask,
                          info=info, use_cuda_graph=use_cuda_graph)()
    torch.cuda.synchronize()
    assert info.tolist() == [0, 7, 0]
    assert torch.isfinite(x[0]).all()
    assert torch.equal(x[2].cpu(), torch.tensor(b0[2], dtype=torch.float32))
