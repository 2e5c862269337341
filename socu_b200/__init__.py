"""socu_b200: B200-native (sm_100a) nested-dissection block-tridiagonal SPD Cholesky.

Drop-in for socu's ``block_tridiag_solver`` API on PyTorch CUDA tensors; the
compute path is the hand-written CUDA in ``libsocu_b200.so`` (C ABI declared
in ``include/socu_b200.h``).
"""
__version__ = "0.1.0"
