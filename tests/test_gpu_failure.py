"""Failure detection of the ragged work queue, without any GPU fault (needs a B200).

The persistent ragged kernel's CTAs wait on the device queue for their next
task.  Every wait is bounded: when the queue makes no progress for the wait
limit (%globaltimer), the waiting CTA records error word 1 and returns.  The
failure is made on the host: one instance's first tasks are withheld from the
queue, so that instance never starts and the queue stalls once the others
are done.  The launch must end by itself within about the limit, report the
error, leave the withheld instance untouched, finish the other instances
exactly as a healthy batch does, and leave the CUDA context usable.
"""
import time

import pytest
import torch

from socu_b200.problems import fill_ragged
from socu_b200.ragged import (RaggedBatch, create_ragged_factor_and_solve_launch,
                              create_ragged_refined_solve_launch)

pytestmark = pytest.mark.gpu

SHAPES = ([12, 30, 7, 19], [8, 16, 4, 12], [1, 2, 1, 3])


def _packed(batch, seed=3):
    L, E, b = batch.empty()
    fill_ragged(batch, L, E, b, seed=seed)
    return L, E, b


def test_stalled_queue_ends_with_timeout_and_context_survives():
    healthy = RaggedBatch(*SHAPES, dtype=torch.float64)
    L, E, b = _packed(healthy)
    Lh, Eh, xh = L.clone(), E.clone(), b.clone()
    create_ragged_factor_and_solve_launch(healthy, Lh, Eh, xh, use_cuda_graph=False)()
    assert healthy.error_flag() == 0

    stalled = RaggedBatch(*SHAPES, dtype=torch.float64)
    stalled.set_wait_limit(1e-3)
    stalled.withhold_instance(1)
    Ls, Es, xs = L.clone(), E.clone(), b.clone()
    run = create_ragged_factor_and_solve_launch(stalled, Ls, Es, xs, use_cuda_graph=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    run()
    torch.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    assert stalled.error_flag() == 1
    assert elapsed < 1.0, elapsed          # ended by the 1 ms wait limit, not by a 4 s default
    for name, got, ref, orig in (("L", Ls, Lh, L), ("E", Es, Eh, E), ("x", xs, xh, b)):
        view = getattr(stalled, f"{name}_view")
        assert torch.equal(view(got, 1), view(orig, 1)), f"withheld instance changed its {name}"
        for i in (0, 2, 3):
            assert torch.equal(view(got, i), view(ref, i)), f"instance {i} {name} differs from the healthy run"

    # the context is still usable: the healthy batch runs again, bit for bit
    Lh2, Eh2, xh2 = L.clone(), E.clone(), b.clone()
    create_ragged_factor_and_solve_launch(healthy, Lh2, Eh2, xh2, use_cuda_graph=True)()
    assert healthy.error_flag() == 0
    assert torch.equal(xh2, xh)


def test_stalled_refined_queue_ends_with_timeout():
    batch = RaggedBatch(*SHAPES, dtype=torch.float64, refine=True, max_iter=5)
    batch.set_wait_limit(2e-3)
    batch.withhold_instance(2)
    L, E, b = _packed(batch, seed=5)
    x = torch.zeros_like(b)
    run = create_ragged_refined_solve_launch(batch, L, E, b, x, tol=1e-12, use_cuda_graph=False)
    run()
    torch.cuda.synchronize()
    assert batch.error_flag() == 1
    eta = run.eta.cpu()
    assert all(float(eta[i]) <= 1e-12 for i in (0, 1, 3))
    assert int(run.iterations[2]) == 0       # never started


def test_wait_limit_validated():
    batch = RaggedBatch([4], [4], [1], dtype=torch.float64)
    with pytest.raises(RuntimeError):
        batch.set_wait_limit(0.0)
    with pytest.raises(RuntimeError):
        batch.withhold_instance(1)
