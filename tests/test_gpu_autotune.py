"""Autotuner on the GPU (needs a B200): every candidate launch setting gives
results that pass the reference tolerances against the oracle, a tuning run
installs and caches its winner, and the reference's block_dim / block_size
arguments are honoured without changing results beyond those tolerances."""
import json

import numpy as np
import pytest
import torch

from oracle import generators, nd_cholesky as nd
from socu_b200 import _lib, autotune
from socu_b200.block_tridiag_solver import (_launch_with_settings, create_cholesky_factor_and_solve_launch,
                                            create_cholesky_factor_launch, create_cholesky_solve_launch)

pytestmark = pytest.mark.gpu
TOL = {torch.float32: 1e-4, torch.float64: 1e-10}


@pytest.fixture(autouse=True)
def clean_table():
    _lib.load().socu_tuning_clear()
    yield
    _lib.load().socu_tuning_clear()


def _case(n, N, m):
    _, L, E, b = generators.reference_test_problem(n, N)
    b = np.concatenate([b.reshape(N, n, 1)] * m, axis=-1)
    _, _, x = nd.nd_factor_and_solve(L, E, b)
    return L, E, b, x[0]


def _settings_grid(n, dtype):
    for knob, values in autotune.candidates(n, 4, dtype).items():
        for v in values[1:]:
            yield {knob: v}


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("n,N", [(10, 20), (36, 33), (64, 16), (68, 9)])
@pytest.mark.parametrize("op", ["factor_and_solve", "factor+solve"])
def test_every_candidate_passes_parity(dtype, n, N, op):
    m = 4
    L_np, E_np, b_np, x_ref = _case(n, N, m)
    tol = TOL[dtype]
    for settings in _settings_grid(n, dtype):
        L = torch.tensor(L_np, dtype=dtype, device="cuda")
        E = torch.tensor(E_np, dtype=dtype, device="cuda")
        x = torch.tensor(b_np, dtype=dtype, device="cuda")
        if op == "factor_and_solve":
            _launch_with_settings("factor_and_solve", L, E, x, dtype, settings)()
        else:
            _launch_with_settings("factor", L, E, None, dtype, settings)()
            _launch_with_settings("solve", L, E, x, dtype, settings)()
        torch.cuda.synchronize()
        err = np.linalg.norm(x.double().cpu().numpy() - x_ref) / np.sqrt(m)
        assert err < tol, (settings, err)


def test_tune_installs_and_caches(tmp_path):
    path = tmp_path / "tune.json"
    best, ms, trials = autotune.tune(36, 2, torch.float64, horizon=64, batch=2, reps=3, warmup=1, path=path)
    assert ms > 0 and len(trials) > 5
    assert autotune.current_settings(torch.float64, 36, 2) == {k: best.get(k, 0) for k in _lib.Tuning.FIELDS}
    entries = json.loads(path.read_text())["entries"]
    assert len(entries) == 1 and entries[0]["n"] == 36 and entries[0]["n_rhs"] == 2
    assert entries[0]["device"] == torch.cuda.get_device_name()
    # a launch created now runs with the tuned settings and stays correct
    L_np, E_np, b_np, x_ref = _case(36, 20, 2)
    L, E, x = (torch.tensor(a, device="cuda") for a in (L_np, E_np, b_np))
    create_cholesky_factor_and_solve_launch(L, E, x)()
    assert np.linalg.norm(x.cpu().numpy() - x_ref) < 1e-10


@pytest.mark.parametrize("block_dim,block_size", [(64, 16), (128, 32), (256, None), (None, 16)])
@pytest.mark.parametrize("n", [32, 68])
def test_block_dim_block_size_overrides(block_dim, block_size, n):
    N = 20
    L_np, E_np, b_np, x_ref = _case(n, N, 1)
    L, E, x = (torch.tensor(a, device="cuda") for a in (L_np, E_np, b_np))
    run = create_cholesky_factor_and_solve_launch(L, E, x, block_dim=block_dim, block_size=block_size,
                                                  use_cuda_graph=True)
    run()
    assert np.linalg.norm(x.cpu().numpy() - x_ref) < 1e-10
    if block_dim is not None:
        assert run.settings["node_threads"] in (64, 128, 256)
    L2, E2, x2 = (torch.tensor(a, device="cuda") for a in (L_np, E_np, b_np))
    create_cholesky_factor_launch(L2, E2, block_dim=block_dim, block_size=block_size)()
    create_cholesky_solve_launch(L2, E2, x2, block_dim=block_dim, block_size=block_size)()
    assert np.linalg.norm(x2.cpu().numpy() - x_ref) < 1e-10


def test_profile_reports_kernel_kinds():
    L_np, E_np, b_np, _ = _case(32, 64, 2)
    L, E, x = (torch.tensor(a, device="cuda") for a in (L_np, E_np, b_np))
    run = create_cholesky_factor_and_solve_launch(L, E, x)
    prof = run.profile()
    assert set(prof) == {"node", "update", "pull", "backward"}
    K = 7   # levels of N = 64
    assert prof["node"][1] == K and prof["backward"][1] == K and prof["update"][1] == K - 1
    assert all(ms > 0 for ms, _ in prof.values())
    assert sum(c for _, c in prof.values()) == run.kernel_count
