"""Seeded synthetic SPD block-tridiagonal problems, generated on the device.

The construction is the reference README's (README.md:100-121) with the
diagonal shift as a parameter:

    D_chol[i] = tril(randn(n, n)) + shift * I,   E_chol[i] = randn(n, n)
    L[i] = D_chol[i] D_chol[i]^T (+ E_chol[i-1] E_chol[i-1]^T for i > 0)
    E[i] = E_chol[i] D_chol[i]^T   (i < N-1; the storage tail is zero)
    b    = randn(N, n, m)

so Psi = C C^T with C the block-bidiagonal (D_chol, E_chol) factor.  Values
come from a torch generator on the target device seeded per problem; they are
synthetic stand-ins with the reference's shapes and distributions.
"""
from __future__ import annotations

import numpy as np
import torch

from .block_tridiag_solver import calculate_off_diag_storage_len

__all__ = ["readme_blocks", "ragged_shapes", "fill_ragged"]


def _fill(L, E, b, N, n, m, shift, gen):
    dev, dt = L.device, L.dtype
    B = L.shape[0]
    Dc = torch.randn(B, N, n, n, generator=gen, device=dev, dtype=dt).tril_()
    Dc.diagonal(dim1=-2, dim2=-1).add_(shift)
    L.copy_(Dc @ Dc.transpose(-1, -2))
    E.zero_()
    if N > 1:
        Ec = torch.randn(B, N - 1, n, n, generator=gen, device=dev, dtype=dt)
        L[:, 1:] += Ec @ Ec.transpose(-1, -2)
        E[:, :N - 1] = Ec @ Dc[:, :N - 1].transpose(-1, -2)
    b.copy_(torch.randn(B, N, n, m, generator=gen, device=dev, dtype=dt))


def readme_blocks(N, n, m=1, shift=10.0, seed=0, batch=1, device="cuda", dtype=torch.float64):
    """(L (B,N,n,n), E (B,S,n,n), b (B,N,n,m)) in the reference layouts."""
    S = calculate_off_diag_storage_len(N)
    kw = dict(device=device, dtype=dtype)
    L = torch.empty(batch, N, n, n, **kw)
    E = torch.empty(batch, S, n, n, **kw)
    b = torch.empty(batch, N, n, m, **kw)
    gen = torch.Generator(device=device).manual_seed(int(seed))
    _fill(L, E, b, N, n, m, shift, gen)
    return L, E, b


def ragged_shapes(seed, count, n_choices=(8, 16, 32, 48), m_choices=(1, 4), n_min=8, n_max=256):
    """Per-instance (N, n, m) of an uneven MPC-style batch: instance i draws
    N ~ U{n_min..n_max}, n and m uniformly from the choices, from a NumPy
    generator seeded with seed + i."""
    N = np.empty(count, dtype=np.int64)
    n = np.empty(count, dtype=np.int64)
    m = np.empty(count, dtype=np.int64)
    for i in range(count):
        rng = np.random.default_rng(seed + i)
        N[i] = rng.integers(n_min, n_max + 1)
        n[i] = rng.choice(list(n_choices))
        m[i] = rng.choice(list(m_choices))
    return N, n, m


def fill_ragged(batch, L, E, b, seed, shift=10.0):
    """Fill packed ragged arrays (see socu_b200.ragged.RaggedBatch) with one
    README problem per instance, instance i seeded with seed + i."""
    gen = torch.Generator(device=L.device)
    for i in range(batch.count):
        N, n, m = int(batch.horizons[i]), int(batch.block_sizes[i]), int(batch.n_rhs[i])
        gen.manual_seed(int(seed) + i)
        _fill(batch.L_view(L, i).unsqueeze(0), batch.E_view(E, i).unsqueeze(0), batch.x_view(b, i).unsqueeze(0),
              N, n, m, shift, gen)
