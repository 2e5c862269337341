"""Generate the golden fixtures under tests/golden/ (run from the repo root):

    python tests/golden/make_golden.py

Each ``ref_n{n}_N{N}.npz`` holds, for the reference test generator
(tests/test_block_tridiag_solver.py:45-80 of socu; seed 42):
  L, E, b         the inputs, bit-identical to the reference tests'
  x_ref           SciPy dense Cholesky + two triangular solves (the reference
                  tests' own oracle, :75-78)
  L_fac, E_fac    the factor blocks in socu's in-place storage layout, read off
                  the dense Cholesky of the nested-dissection permuted matrix
``readme_N{N}_n{n}_m{m}_s{s}.npz`` does the same for the README generator with
a diagonal shift s (README.md:100-121) and a dense FP64 ``numpy.linalg.solve``
as x_ref.
"""
from __future__ import annotations

import pathlib
import sys

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parent.parent))

from oracle import dense, generators  # noqa: E402

REF_CASES = [(1, 1), (1, 7), (10, 1), (10, 2), (10, 3), (10, 8), (10, 20), (32, 4), (36, 7), (36, 5)]
README_CASES = [(100, 8, 1, 10.0), (33, 12, 3, 10.0), (17, 5, 2, 10.0)]


def main():
    for n, N in REF_CASES:
        A, L, E, b = generators.reference_test_problem(n, N)
        x_ref = dense.reference_solution(A, b)
        Lf, Ef = dense.permuted_factor(L, E)
        np.savez_compressed(HERE / f"ref_n{n}_N{N}.npz", L=L, E=E, b=b, x_ref=x_ref, L_fac=Lf, E_fac=Ef)
    for N, n, m, s in README_CASES:
        L, E, b = generators.readme_problem(N, n, m, shift=s, seed=1234)
        A = generators.dense_from_blocks(L, E)
        x_ref = np.linalg.solve(A, b.reshape(N * n, m)).reshape(N, n, m)
        Lf, Ef = dense.permuted_factor(L, E)
        np.savez_compressed(HERE / f"readme_N{N}_n{n}_m{m}_s{int(s)}.npz", L=L, E=E, b=b, x_ref=x_ref,
                            L_fac=Lf, E_fac=Ef)


if __name__ == "__main__":
    main()
