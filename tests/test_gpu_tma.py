"""GPU: the resident sweeps stage their factor / coupling blocks and vector
chunks with TMA tensor copies (cp.async.bulk.tensor, mbarrier completion) by
default; SOCU_TMA=0 keeps them on per-thread cp.async copies.  Both stagings
must give the same bits (same arithmetic on the same shared layout), against
the oracle as well, with no TMA wait running out.  Shapes cover TMA for blocks
and vectors, blocks only (float m = 1, 2: vector rows under 16 bytes), neither
(float n = 30: block rows of 120 bytes), several vector chunks (m = 40) and
batches with a mask."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [  # (B, N, n, m)
    (1, 33, 16, 8),
    (2, 64, 64, 8),
    (1, 40, 32, 1),
    (1, 17, 24, 2),
    (1, 21, 30, 5),
    (3, 50, 48, 40),
    (1, 1, 8, 4),
]

SCRIPT = r"""
import ctypes, json, sys
import numpy as np, torch
from oracle import generators
from socu_b200 import _lib
from socu_b200.block_tridiag_solver import (create_cholesky_factor_and_solve_launch,
    create_cholesky_factor_launch, create_cholesky_solve_launch)
from socu_b200.mixed import create_cholesky_refined_solve_launch
out = {}
for (B, N, n, m) in json.loads(sys.argv[1]):
    P = [generators.readme_problem(N, n, m, shift=10.0 + 2.0 * n ** 0.5, seed=N * 7 + n + k) for k in range(B)]
    L0, E0, b0 = (np.stack([q[i] for q in P]) for i in range(3))
    for dt in (torch.float32, torch.float64):
        L, E, x = (torch.tensor(a, dtype=dt, device="cuda") for a in (L0, E0, b0))
        mask = torch.ones(B, dtype=torch.bool, device="cuda")
        if B > 1:
            mask[1] = False
        create_cholesky_factor_and_solve_launch(L, E, x, mask, dtype=dt)()
        L2, E2, x2 = (torch.tensor(a, dtype=dt, device="cuda") for a in (L0, E0, b0))
        create_cholesky_factor_launch(L2, E2, dtype=dt)()
        create_cholesky_solve_launch(L2, E2, x2, dtype=dt, use_cuda_graph=True)()
        torch.cuda.synchronize()
        key = f"{B}_{N}_{n}_{m}_{str(dt)[-7:]}"
        out[key + "_fs"] = x.double().cpu().numpy().tolist()
        out[key + "_s"] = x2.double().cpu().numpy().tolist()
    L, E, b = (torch.tensor(a, dtype=torch.float64, device="cuda") for a in (L0, E0, b0))
    xm = torch.zeros_like(b)
    run = create_cholesky_refined_solve_launch(L, E, b, xm, tol=1e-12, max_iter=10)
    run()
    torch.cuda.synchronize()
    out[f"{B}_{N}_{n}_{m}_mixed"] = xm.cpu().numpy().tolist()
lib = _lib.load()
flag = ctypes.c_int(0)
assert lib.socu_tc_error(ctypes.byref(flag), 1) == 0
out["tc_error"] = flag.value
print(json.dumps(out))
"""


def _run(tma):
    env = dict(os.environ, SOCU_TMA=tma, PYTHONPATH=ROOT + os.pathsep + os.environ.get("PYTHONPATH", ""))
    r = subprocess.run([sys.executable, "-c", SCRIPT, json.dumps(CASES)], cwd=ROOT, env=env,
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-3000:]
    return json.loads(r.stdout.strip().splitlines()[-1])


def test_tma_staging_matches_cp_async_bitwise():
    from oracle import generators, nd_cholesky as nd

    with_tma, without = _run("1"), _run("0")
    assert with_tma["tc_error"] == 0 and without["tc_error"] == 0
    assert with_tma.keys() == without.keys()
    for k in with_tma:
        if k == "tc_error":
            continue
        a, b = np.asarray(with_tma[k]), np.asarray(without[k])
        assert np.array_equal(a, b), (k, float(np.abs(a - b).max()))
    # and both against the oracle
    for (B, N, n, m) in CASES:
        P = [generators.readme_problem(N, n, m, shift=10.0 + 2.0 * n ** 0.5, seed=N * 7 + n + k) for k in range(B)]
        L0, E0, b0 = (np.stack([q[i] for q in P]) for i in range(3))
        x_ref = nd.nd_factor_and_solve(L0, E0, b0)[2]
        scale = max(1.0, float(np.abs(x_ref).max()))
        for dt, tol in (("float32", 1e-4), ("float64", 1e-10)):
            key = f"{B}_{N}_{n}_{m}_{dt[-7:]}"
            xs = np.asarray(with_tma[key + "_s"])
            assert np.abs(xs - x_ref).max() <= tol * scale, (key, "solve")
            xf = np.asarray(with_tma[key + "_fs"])
            active = [k for k in range(B) if not (B > 1 and k == 1)]
            assert np.abs(xf[active] - x_ref[active]).max() <= tol * scale, (key, "factor_and_solve")
            if B > 1:   # masked-out entry untouched
                assert np.array_equal(xf[1], b0[1].astype(np.float32 if dt == "float32" else np.float64))
        xm = np.asarray(with_tma[f"{B}_{N}_{n}_{m}_mixed"])
        assert np.abs(xm - x_ref).max() <= 1e-9 * scale
