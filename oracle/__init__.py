"""CPU oracle for the nested-dissection block-tridiagonal Cholesky.

TEST INFRASTRUCTURE ONLY.  Nothing in the product package (``socu_b200``)
imports this package.  It is used by ``tests/`` (as the checker), by
``__graft_entry__.smoke()`` (as the checker) and by ``bench.py`` (as the timed
CPU baseline, ``cpu_baseline.kind == "port"``).

Contents
--------
``nd_cholesky``  NumPy restatement of the reference's level schedule, storage
                 offsets, per-node factor math and both substitution sweeps
                 (socu/block_tridiag_solver.py, socu/blas/*.py).
``generators``   Seeded input generators: the reference test generator
                 (tests/test_block_tridiag_solver.py:45-80) and the README
                 generator with a diagonal shift (README.md:100-121).
``dense``        Dense SciPy checks: the reference tests' own oracle (dense
                 Cholesky + two triangular solves) and the dense Cholesky of
                 the nested-dissection permuted matrix, which pins the exact
                 (L, E[storage_len]) factor layout block by block.

Parity pinning: the reference itself (Python + NVIDIA Warp) cannot run in
this environment (warp-lang is not installed and there is no network).  The
oracle is pinned instead against (a) the reference tests' own known answer,
SciPy dense Cholesky on the reference test generator at the reference
tolerances, and (b) the dense Cholesky of P Psi P^T, whose blocks are by
uniqueness of the Cholesky factor exactly the blocks the reference stores.
"""
