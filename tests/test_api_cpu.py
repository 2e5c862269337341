"""Host-side behaviour of the drop-in API that needs no GPU: validation order,
messages and exception types of socu/block_tridiag_solver.py:749-774, dtype
handling, optimal_problem_settings, and the CPU rejection."""
import pytest
import torch

from socu_b200 import block_tridiag_solver as bts


def arrays(B=2, N=5, n=4, m=1, dtype=torch.float64):
    S = bts.calculate_off_diag_storage_len(N)
    return (torch.zeros(B, N, n, n, dtype=dtype), torch.zeros(B, S, n, n, dtype=dtype),
            torch.zeros(B, N, n, m, dtype=dtype))


def test_helpers():
    assert bts.calculate_recursive_iterations(1) == 1
    assert bts.calculate_off_diag_storage_len(100) == 190
    with pytest.raises(AssertionError):
        bts.calculate_recursive_iterations(0)


def test_optimal_problem_settings_matches_reference_table():
    s = bts.optimal_problem_settings(36, torch.float64)
    assert s["block_size"] == {"factor": 16, "solve": 16}
    assert s["pad_multiple"] == {"factor": 8, "solve": 8}
    s = bts.optimal_problem_settings(10, "float64")
    assert s["block_size"] == {"factor": 16, "solve": 32}
    assert s["pad_multiple"] == {"factor": 2, "solve": 2}
    s = bts.optimal_problem_settings(10, torch.float32)
    assert s["pad_multiple"] == {"factor": 4, "solve": 4}
    s = bts.optimal_problem_settings(64, "float32")
    assert s["block_size"]["factor"] == 32 and s["pad_multiple"]["factor"] == 16
    with pytest.raises(ValueError):
        bts.optimal_problem_settings(8, torch.float16)


def test_mask_shape_check():
    # tests/test_block_tridiag_solver.py:223-229 of socu
    L, E, _ = arrays(B=2)
    with pytest.raises(AssertionError, match=r"mask must have shape \(batch_dim,\)"):
        bts.create_cholesky_factor_launch(L, E, mask=torch.ones(3, dtype=torch.bool))
    with pytest.raises(AssertionError, match="mask must be a wp.bool array"):
        bts.create_cholesky_factor_launch(L, E, mask=torch.ones(2, dtype=torch.int32))


def test_shape_assertions():
    L, E, x = arrays()
    with pytest.raises(AssertionError, match="same number of dimensions"):
        bts.create_cholesky_factor_launch(L, E[0])
    with pytest.raises(ValueError, match="L must have 4 or 3 dimensions"):
        bts.create_cholesky_factor_launch(L[0, 0], E[0, 0])
    with pytest.raises(AssertionError, match="same batch dimension"):
        bts.create_cholesky_factor_launch(L, E[:1])
    with pytest.raises(AssertionError, match="last two dimensions"):
        bts.create_cholesky_factor_launch(L[..., :3], E)
    with pytest.raises(AssertionError, match="same block size"):
        bts.create_cholesky_factor_launch(L, E[..., :3, :3])
    with pytest.raises(AssertionError, match="calculate_off_diag_storage_len"):
        bts.create_cholesky_factor_launch(L, E[:, :-1])
    with pytest.raises(AssertionError, match="x has incorrect dimensions"):
        bts.create_cholesky_solve_launch(L, E, x[:, :-1])
    with pytest.raises(AssertionError, match="L, E, and x must have same batch dimension"):
        bts.create_cholesky_solve_launch(L, E, x[:1])
    with pytest.raises(AssertionError, match="L, E, and x must have the same number of dimensions"):
        bts.create_cholesky_factor_and_solve_launch(L, E, x[0])


def test_cpu_arrays_rejected_loudly():
    L, E, x = arrays()
    with pytest.raises(ValueError, match="CUDA"):
        bts.create_cholesky_factor_launch(L, E)
    with pytest.raises(ValueError, match="use_cuda_graph=True requires a CUDA device"):
        bts.create_cholesky_solve_launch(L, E, x, use_cuda_graph=True)
    with pytest.raises(ValueError, match="dtype must be"):
        bts.create_cholesky_factor_launch(L, E, dtype="float16")


def test_three_dim_inputs_validate():
    L, E, x = arrays(B=1)
    with pytest.raises(ValueError, match="CUDA"):
        bts.create_cholesky_factor_and_solve_launch(L[0], E[0], x[0])
