"""GPU: copy_lower_blocks moves the lower triangles of n x n blocks (16-row
bands) between pinned host and device memory; the mixed solve fed that way
gives the same result as with full copies (every kernel reads only lower(L))."""
import numpy as np
import pytest
import torch

from oracle import generators
from socu_b200.block_tridiag_solver import copy_lower_blocks
from socu_b200.mixed import create_cholesky_refined_solve_launch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [1, 8, 16, 30, 64, 100])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_band_copy_host_to_device_and_back(n, dtype):
    src = torch.randn(3, 5, n, n, dtype=dtype).pin_memory()
    dst = torch.full((3, 5, n, n), 7.0, dtype=dtype, device="cuda")
    moved = copy_lower_blocks(dst, src)
    torch.cuda.synchronize()
    r = torch.arange(n).view(n, 1)
    c = torch.arange(n).view(1, n)
    band = c < torch.clamp((r // 16) * 16 + 16, max=n)      # columns a band carries
    got = dst.cpu()
    assert torch.equal(got[..., band], src[..., band])
    assert torch.all(got[..., ~band] == 7.0)
    assert moved == int(band.sum()) * 15 * src.element_size()
    back = torch.zeros(3, 5, n, n, dtype=dtype).pin_memory()
    copy_lower_blocks(back, dst)
    torch.cuda.synchronize()
    assert torch.equal(back[..., band], src[..., band])


def test_mixed_solve_from_band_copies():
    N, n, m = 64, 64, 4
    L0, E0, b0 = generators.readme_problem(N, n, m, shift=10.0, seed=5)
    Lh = torch.tensor(L0).unsqueeze(0).pin_memory()
    L = torch.zeros_like(Lh, device="cuda")          # the part above the bands is never read
    copy_lower_blocks(L, Lh)
    E, b = (torch.tensor(a, device="cuda").unsqueeze(0) for a in (E0, b0))
    x_band, x_full = torch.zeros_like(b), torch.zeros_like(b)
    create_cholesky_refined_solve_launch(L, E, b, x_band, tol=1e-12, max_iter=10)()
    create_cholesky_refined_solve_launch(Lh.cuda(), E, b, x_full, tol=1e-12, max_iter=10)()
    torch.cuda.synchronize()
    assert torch.equal(x_band, x_full)
