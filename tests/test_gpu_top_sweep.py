"""GPU: on request (SOCU_TOP_SWEEP=1) the top levels of the sweeps run in one
cluster-resident kernel (k_top: forward levels with at most 16 tasks, then
backward levels with at most 16 nodes, a cluster barrier between levels, the
next item's blocks copied by TMA while the current one computes); by default
(SOCU_TOP_SWEEP=0) every level keeps its own launch.  Both must give the same
bits (same products, chosen by the same per-level settings), against the
oracle as well; the top kernel must actually run (fewer launches) and no TMA
wait may run out.  Shapes cover the bench shape, batches with a mask, several
vector chunks (m = 40), a horizon whose every level fits the cluster (N = 7:
the forward level 0 runs in it), a single-level horizon, float and FP64,
factors with and without their inverses, the forward-only and backward-only
ops, the mixed refined solve, and the cp.async block path (SOCU_TMA=0)."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [  # (B, N, n, m)
    (1, 1024, 64, 8),
    (3, 100, 32, 3),
    (2, 50, 48, 40),
    (1, 7, 8, 2),
    (1, 1, 8, 4),
    (4, 300, 16, 1),
]

SCRIPT = r"""
import ctypes, json, sys
import numpy as np, torch
from oracle import generators
from socu_b200 import _lib
from socu_b200.block_tridiag_solver import (create_cholesky_factor_and_solve_launch,
    create_cholesky_factor_launch, create_cholesky_solve_launch,
    create_cholesky_forward_substitution_launch, create_cholesky_backward_substitution_launch)
from socu_b200.mixed import create_cholesky_refined_solve_launch
out = {}
for (B, N, n, m) in json.loads(sys.argv[1]):
    P = [generators.readme_problem(N, n, m, shift=10.0 + 2.0 * n ** 0.5, seed=N * 5 + n + k) for k in range(B)]
    L0, E0, b0 = (np.stack([q[i] for q in P]) for i in range(3))
    key0 = f"{B}_{N}_{n}_{m}"
    for dt in (torch.float32, torch.float64):
        key = key0 + "_" + str(dt)[-7:]
        L, E, x = (torch.tensor(a, dtype=dt, device="cuda") for a in (L0, E0, b0))
        mask = torch.ones(B, dtype=torch.bool, device="cuda")
        if B > 1:
            mask[1] = False
        run = create_cholesky_factor_and_solve_launch(L, E, x, mask, dtype=dt)
        run()
        out[key + "_fs_k"] = run.kernel_count
        # stored factor (no inverses): solve, then forward and backward apart
        L2, E2, x2 = (torch.tensor(a, dtype=dt, device="cuda") for a in (L0, E0, b0))
        create_cholesky_factor_launch(L2, E2, dtype=dt)()
        x3 = x2.clone()
        run = create_cholesky_solve_launch(L2, E2, x2, dtype=dt, use_cuda_graph=True)
        run()
        out[key + "_s_k"] = run.kernel_count
        create_cholesky_forward_substitution_launch(L2, E2, x3, dtype=dt)()
        torch.cuda.synchronize()
        out[key + "_f"] = x3.double().cpu().numpy().tolist()
        create_cholesky_backward_substitution_launch(L2, E2, x3, dtype=dt)()
        torch.cuda.synchronize()
        out[key + "_fs"] = x.double().cpu().numpy().tolist()
        out[key + "_s"] = x2.double().cpu().numpy().tolist()
        out[key + "_fb"] = x3.double().cpu().numpy().tolist()
    L, E, b = (torch.tensor(a, dtype=torch.float64, device="cuda") for a in (L0, E0, b0))
    xm = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, xm, tol=1e-12, max_iter=10)
    run()
    torch.cuda.synchronize()
    out[key0 + "_mixed"] = xm.cpu().numpy().tolist()
    out[key0 + "_mixed_k"] = run.round_kernel_count
lib = _lib.load()
flag = ctypes.c_int(0)
assert lib.socu_tc_error(ctypes.byref(flag), 1) == 0
out["tc_error"] = flag.value
print(json.dumps(out))
"""


def _run(top, tma="1"):
    env = dict(os.environ, SOCU_TOP_SWEEP=top, SOCU_TMA=tma,
               PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", SCRIPT, json.dumps(CASES)], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


@pytest.fixture(scope="module")
def runs():
    return {"top": _run("1"), "levels": _run("0"), "top_cp_async": _run("1", "0")}


def test_top_sweep_matches_per_level_launches_bitwise(runs):
    top, levels, cpa = runs["top"], runs["levels"], runs["top_cp_async"]
    for r in (top, levels, cpa):
        assert r["tc_error"] == 0
    assert top.keys() == levels.keys() == cpa.keys()
    for k in top:
        if k == "tc_error" or k.endswith("_k"):
            continue
        a, b = np.asarray(top[k]), np.asarray(levels[k])
        assert np.array_equal(a, b), (k, float(np.abs(a - b).max()))
        assert np.array_equal(np.asarray(cpa[k]), b), k


def test_top_sweep_replaces_level_launches(runs):
    top, levels = runs["top"], runs["levels"]
    # the bench shape: 11 levels; forward levels 6-10 and backward levels 5-10 in one launch
    assert levels["1_1024_64_8_float32_s_k"] - top["1_1024_64_8_float32_s_k"] == 10
    assert levels["1_1024_64_8_float32_fs_k"] - top["1_1024_64_8_float32_fs_k"] == 5
    assert levels["1_1024_64_8_mixed_k"] - top["1_1024_64_8_mixed_k"] == 10
    # one level: the backward sweep of factor_and_solve keeps its launch, a solve's
    # forward and backward level share one
    assert levels["1_1_8_4_float64_fs_k"] == top["1_1_8_4_float64_fs_k"]
    assert levels["1_1_8_4_float64_s_k"] - top["1_1_8_4_float64_s_k"] == 1
    # N = 7: all three forward and three backward levels in one kernel
    assert top["1_7_8_2_float64_s_k"] == 1


def test_top_sweep_against_oracle(runs):
    from oracle import generators, nd_cholesky as nd

    top = runs["top"]
    for (B, N, n, m) in CASES:
        P = [generators.readme_problem(N, n, m, shift=10.0 + 2.0 * n ** 0.5, seed=N * 5 + n + k) for k in range(B)]
        L0, E0, b0 = (np.stack([q[i] for q in P]) for i in range(3))
        x_ref = nd.nd_factor_and_solve(L0, E0, b0)[2]
        scale = max(1.0, float(np.abs(x_ref).max()))
        active = [k for k in range(B) if not (B > 1 and k == 1)]
        for dt, tol in (("float32", 1e-4), ("float64", 1e-10)):
            key = f"{B}_{N}_{n}_{m}_{dt}"
            for suffix in ("_s", "_fb"):
                assert np.abs(np.asarray(top[key + suffix]) - x_ref).max() <= tol * scale, (key, suffix)
            xf = np.asarray(top[key + "_fs"])
            assert np.abs(xf[active] - x_ref[active]).max() <= tol * scale, (key, "factor_and_solve")
            if B > 1:   # masked-out entry untouched
                assert np.array_equal(xf[1], b0[1].astype(np.float32 if dt == "float32" else np.float64))
        xm = np.asarray(top[f"{B}_{N}_{n}_{m}_mixed"])
        assert np.abs(xm - x_ref).max() <= 1e-9 * scale
