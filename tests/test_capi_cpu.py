"""The C-ABI library loads and exports every symbol include/socu_b200.h declares.

No compute calls: only entry points that return before touching a GPU
(pure helpers, argument validation, empty batches).
"""
import ctypes
import os
import re

import pytest

from socu_b200 import _lib
from socu_b200 import block_tridiag_solver as bts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "socu_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(socu_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def test_every_declared_symbol_is_exported(lib):
    names = header_functions()
    assert len(names) >= 10
    for name in names:
        assert hasattr(lib, name), name
    assert set(names) == set(_lib.exported_symbols())


def test_storage_helpers_match_python(lib):
    for N in [1, 2, 3, 4, 7, 8, 20, 100, 128, 1024, 16384, 12345]:
        assert lib.socu_off_diag_storage_len(N) == bts.calculate_off_diag_storage_len(N)
        assert lib.socu_recursive_iterations(N) == bts.calculate_recursive_iterations(N)
    assert lib.socu_off_diag_storage_len(0) == -1
    assert lib.socu_recursive_iterations(-3) == -1


def test_status_strings(lib):
    assert lib.socu_status_string(0) == b"ok"
    assert lib.socu_status_string(-1) == b"invalid argument"
    assert lib.socu_version().startswith(b"socu_b200")


def test_max_block_size_covers_configs(lib):
    assert lib.socu_max_block_size(_lib.FLOAT64, 32) >= 128
    assert lib.socu_max_block_size(_lib.FLOAT32, 32) >= 128


def test_invalid_arguments_rejected_without_gpu(lib):
    # bad dtype / sizes / null pointers return before any CUDA call
    assert lib.socu_cholesky_factor(7, None, None, None, 1, 4, 4, None) == -1
    assert lib.socu_cholesky_factor(_lib.FLOAT64, None, None, None, 1, 0, 4, None) == -1
    assert lib.socu_cholesky_factor(_lib.FLOAT64, None, None, None, 1, 4, 4, None) == -1
    assert lib.socu_cholesky_solve(_lib.FLOAT64, None, None, None, None, 1, 4, 4, 0, None) == -1
    assert lib.socu_cholesky_factor(_lib.FLOAT64, None, None, None, 1, 4, 100000, None) == -3
    # an empty batch is a no-op
    assert lib.socu_cholesky_factor(_lib.FLOAT64, None, None, None, 0, 4, 4, None) == 0
    h = ctypes.c_void_p()
    assert lib.socu_launch_create(None, 0, 1, None, None, None, None, 1, 4, 4, 1, 0, None) == -1
    assert lib.socu_launch_create(ctypes.byref(h), 0, 1, None, None, None, None, 0, 4, 4, 0, 0, None) == 0
    assert lib.socu_launch_kernel_count(h) == 0
    assert lib.socu_launch_destroy(h) == 0
    assert lib.socu_launch_run(None, None) == -1


def test_launch_kernel_count_without_gpu(lib):
    # counting needs no device: per level node (+ update) for the factor
    h = ctypes.c_void_p()
    fake = 0x1000  # never dereferenced: counting mode does not launch
    st = lib.socu_launch_create(ctypes.byref(h), _lib.OP_FACTOR, _lib.FLOAT64, fake, fake, None, None,
                                1, 100, 32, 0, 0, None)
    assert st == 0
    assert lib.socu_launch_kernel_count(h) == (7 - 1) * 2 + 1  # K = 7 levels: node + update, last one node only
    lib.socu_launch_destroy(h)
