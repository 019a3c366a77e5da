"""The host-side conversions (sparkit_b200/formats.py) against the
reference's own to_ellpack / to_jagged_diagonal / to_block_sparse_row."""
import numpy as np
import pytest

from sparkit_b200 import formats, matgen
from tests.helpers import SPMV_CASES, golden_csr


def _same(a, b, fields):
    for f in fields:
        assert np.array_equal(getattr(a, f)(), getattr(b, f)()), f


@pytest.mark.parametrize("name", SPMV_CASES)
def test_conversions_match_reference(reference, golden, name):
    A = golden_csr(golden, f"spmv/{name}/float64")
    _same(formats.to_ellpack(A), reference.to_ellpack(A), ("col_ind", "values"))
    assert formats.to_ellpack(A).max_nnz_per_row() == reference.to_ellpack(A).max_nnz_per_row()
    _same(formats.to_jagged_diagonal(A), reference.to_jagged_diagonal(A), ("perm", "jdiag", "col_ind", "values"))
    for br, bc in ((2, 2), (3, 3), (2, 3), (1, 4)):
        _same(formats.to_block_sparse_row(A, br, bc), reference.to_block_sparse_row(A, br, bc),
              ("row_ptr", "col_ind", "values"))


def test_empty_layouts():
    A = formats.Compressed_row_matrix((3, 3), np.zeros(4, np.int64), np.zeros(0, np.int64), np.zeros(0))
    E = formats.to_ellpack(A)
    assert E.max_nnz_per_row() == 0 and E.col_ind().size == 0
    J = formats.to_jagged_diagonal(A)
    assert J.jdiag().tolist() == [0] and J.perm().size == 0
    B = formats.to_block_sparse_row(A, 2, 2)
    assert B.row_ptr().tolist() == [0, 0, 0] and B.num_blocks() == 0


def test_from_entries_sorts_and_deduplicates():
    A = formats.Compressed_row_matrix.from_entries((3, 3), [2, 0, 0, 2], [1, 2, 0, 1], [1.0, 2.0, 3.0, 1.0])
    assert A.row_ptr().tolist() == [0, 2, 2, 3]
    assert A.col_ind().tolist() == [0, 2, 1]


def test_workload_generators_shapes():
    A = matgen.laplacian_3d_dirichlet(8)
    assert A.shape() == (512, 512) and A.size() == 7 * 512 - 6 * 64
    assert np.all(np.diff(A.col_ind()[A.row_ptr()[100]:A.row_ptr()[101]]) > 0)
    L = matgen.laplacian_2d_dirichlet(256)
    assert L.size() == 326656  # n = 65,536 5-point Dirichlet grid
    V = matgen.vector_laplacian_3d_bsr_csr(3)
    B = formats.to_block_sparse_row(V, 3, 3)
    assert B.num_blocks() == 7 * 27 - 6 * 9
