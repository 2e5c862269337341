"""Ragged batches on the host: packed layout, validation, shape draws."""
import numpy as np
import pytest

from oracle import generators
from oracle.nd_cholesky import off_diag_storage_len
from socu_b200 import _lib
from socu_b200.problems import ragged_shapes
from socu_b200.ragged import ragged_layout


def test_layout_packs_instances_back_to_back():
    N = [1, 2, 7, 100, 33]
    n = [3, 64, 8, 32, 1]
    m = [1, 4, 2, 1, 9]
    offL, offE, offx, tot = ragged_layout(N, n, m)
    eL = eE = ex = 0
    for i in range(len(N)):
        assert (offL[i], offE[i], offx[i]) == (eL, eE, ex)
        eL += N[i] * n[i] * n[i]
        eE += off_diag_storage_len(N[i]) * n[i] * n[i]
        ex += N[i] * n[i] * m[i]
    assert list(tot) == [eL, eE, ex]


def test_layout_empty_batch():
    offL, offE, offx, tot = ragged_layout([], [], [])
    assert len(offL) == 0 and list(tot) == [0, 0, 0]


@pytest.mark.parametrize("bad,status", [(([0], [4], [1]), -1), (([4], [0], [1]), -1), (([4], [4], [0]), -1),
                                        (([4], [65], [1]), -3)])
def test_layout_rejects_bad_shapes(bad, status):
    lib = _lib.load()
    N, n, m = (np.asarray(a, dtype=np.int64) for a in bad)
    tot = np.zeros(3, dtype=np.int64)
    ptr = lambda a: a.ctypes.data_as(__import__("ctypes").c_void_p)
    assert lib.socu_ragged_layout(ptr(N), ptr(n), ptr(m), 1, None, None, None, ptr(tot)) == status
    with pytest.raises(RuntimeError):
        ragged_layout(*bad)


def test_shape_draws_match_the_oracle_generator():
    N, n, m = ragged_shapes(7, 12)
    for i in range(12):
        Ni, ni, mi = generators.ragged_instance(7, i)[:3]
        assert (N[i], n[i], m[i]) == (Ni, ni, mi)
    assert N.min() >= 8 and N.max() <= 256
    assert set(n) <= {8, 16, 32, 48} and set(m) <= {1, 4}
