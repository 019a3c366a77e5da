"""sparkit_b200: the sparkit preconditioned-Krylov hot path on B200 (sm_100a).

Host mirrors of the reference's storage classes live in ``formats``; the
GPU drop-in (device matrices, multiply, preconditioners, solvers) in
``gpu``; seeded workload generators in ``matgen``.  The compute runs in the
in-tree C-ABI library libsparkit_b200.so (include/sparkit_b200.h); there is
no CPU fallback.
"""
from .formats import (Block_sparse_row_matrix, Compressed_row_matrix, Ellpack_matrix,  # noqa: F401
                      Jagged_diagonal_matrix, to_block_sparse_row, to_ellpack, to_jagged_diagonal)

__version__ = "0.1.0"
