"""Host-side mirrors of sparkit's four hot-path storage classes and the
conversions that build them from CSR.

Each class holds exactly the arrays the reference class exposes (int64
indices, as sparkit's size_type is std::ptrdiff_t), so that a
Device_matrix upload receives the same layout the C++ drop-in reads from
the reference objects:

* Compressed_row_matrix  -- Compressed_row_matrix.hpp:20-132
* Ellpack_matrix         -- Ellpack_matrix.hpp:20-122, Ellpack_sparsity_Impl.cpp:10-48
* Jagged_diagonal_matrix -- Jagged_diagonal_matrix.hpp:20-144, Jagged_diagonal_sparsity_Impl.cpp:11-93
* Block_sparse_row_matrix -- Block_sparse_row_matrix.hpp:21-150, Block_sparse_row_sparsity_Impl.cpp:11-51

The conversions restate to_ellpack (conversions.hpp:427), to_jagged_diagonal
(conversions.hpp:641) and to_block_sparse_row (conversions.hpp:524) with
numpy; tests/test_formats.py checks them array for array against the
reference's own conversions.
"""
import numpy as np


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


class Compressed_row_matrix:
    """CSR: row_ptr[nrow+1], col_ind[nnz] sorted and unique per row, values[nnz]."""

    def __init__(self, shape, row_ptr, col_ind, values, dtype=None):
        self._shape = (int(shape[0]), int(shape[1]))
        self._row_ptr = _i64(row_ptr)
        self._col_ind = _i64(col_ind)
        dt = np.dtype(dtype) if dtype is not None else np.asarray(values).dtype
        if dt not in (np.float64, np.float32):
            dt = np.dtype(np.float64)
        self._values = np.ascontiguousarray(np.asarray(values, dtype=dt))
        if self._row_ptr.shape[0] != self._shape[0] + 1:
            raise ValueError("row_ptr must have nrow + 1 entries")
        if self._col_ind.shape[0] != self._row_ptr[-1] or self._values.shape[0] != self._row_ptr[-1]:
            raise ValueError("col_ind and values must have row_ptr[nrow] entries")

    @classmethod
    def from_entries(cls, shape, rows, cols, values, dtype=np.float64):
        """Sorts by (row, column) and keeps one entry per index, as
        Compressed_row_matrix::from_entries (Compressed_row_matrix.hpp:97-127)."""
        rows, cols = _i64(rows), _i64(cols)
        values = np.asarray(values, dtype=dtype)
        nr, nc = int(shape[0]), int(shape[1])
        if nr * max(nc, 1) < (1 << 62):
            # one stable sort of row * ncol + col: the order of the
            # two-key lexsort, several times faster
            order = np.argsort(rows * max(nc, 1) + cols, kind="stable")
        else:
            order = np.lexsort((cols, rows))
        rows, cols, values = rows[order], cols[order], values[order]
        if rows.size:
            keep = np.ones(rows.size, dtype=bool)
            keep[1:] = (rows[1:] != rows[:-1]) | (cols[1:] != cols[:-1])
            rows, cols, values = rows[keep], cols[keep], values[keep]
        counts = np.bincount(rows, minlength=int(shape[0])) if rows.size else np.zeros(int(shape[0]), np.int64)
        rp = np.zeros(int(shape[0]) + 1, dtype=np.int64)
        np.cumsum(counts, out=rp[1:])
        return cls(shape, rp, cols, values)

    def shape(self):
        return self._shape

    def size(self):
        return int(self._row_ptr[-1])

    def row_ptr(self):
        return self._row_ptr

    def col_ind(self):
        return self._col_ind

    def values(self):
        return self._values

    @property
    def dtype(self):
        return self._values.dtype

    def astype(self, dtype):
        return Compressed_row_matrix(self._shape, self._row_ptr, self._col_ind, self._values.astype(dtype))

    def row_lengths(self):
        return np.diff(self._row_ptr)


class Ellpack_matrix:
    """ELLPACK: row-major nrow x width col_ind with -1 padding, values with
    zero padding; width = max_nnz_per_row()."""

    def __init__(self, shape, width, col_ind, values):
        self._shape = (int(shape[0]), int(shape[1]))
        self._width = int(width)
        self._col_ind = _i64(col_ind)
        self._values = np.ascontiguousarray(values)
        if self._col_ind.size != self._shape[0] * self._width:
            raise ValueError("col_ind must hold nrow * width slots")

    def shape(self):
        return self._shape

    def max_nnz_per_row(self):
        return self._width

    def col_ind(self):
        return self._col_ind

    def values(self):
        return self._values

    def size(self):
        return int(np.count_nonzero(self._col_ind != -1))

    @property
    def dtype(self):
        return self._values.dtype


class Jagged_diagonal_matrix:
    """Jagged diagonal: perm (rows by decreasing length, ties by index),
    jdiag[njd+1], col_ind / values in jagged-diagonal order."""

    def __init__(self, shape, perm, jdiag, col_ind, values):
        self._shape = (int(shape[0]), int(shape[1]))
        self._perm = _i64(perm)
        self._jdiag = _i64(jdiag)
        self._col_ind = _i64(col_ind)
        self._values = np.ascontiguousarray(values)

    def shape(self):
        return self._shape

    def perm(self):
        return self._perm

    def jdiag(self):
        return self._jdiag

    def col_ind(self):
        return self._col_ind

    def values(self):
        return self._values

    def num_jdiags(self):
        return int(self._jdiag.size - 1)

    def size(self):
        return int(self._jdiag[-1])

    @property
    def dtype(self):
        return self._values.dtype


class Block_sparse_row_matrix:
    """Block CSR over ceil(nrow / block_rows) block rows with dense row-major
    block_rows x block_cols blocks."""

    def __init__(self, shape, block_rows, block_cols, row_ptr, col_ind, values):
        self._shape = (int(shape[0]), int(shape[1]))
        self._br = int(block_rows)
        self._bc = int(block_cols)
        self._row_ptr = _i64(row_ptr)
        self._col_ind = _i64(col_ind)
        self._values = np.ascontiguousarray(values)

    def shape(self):
        return self._shape

    def block_rows(self):
        return self._br

    def block_cols(self):
        return self._bc

    def num_block_rows(self):
        return (self._shape[0] + self._br - 1) // self._br

    def num_blocks(self):
        return int(self._col_ind.size)

    def row_ptr(self):
        return self._row_ptr

    def col_ind(self):
        return self._col_ind

    def values(self):
        return self._values

    def size(self):
        return int(self._values.size)

    @property
    def dtype(self):
        return self._values.dtype


def to_ellpack(csr):
    """to_ellpack (conversions.hpp:427-467): entry k of row i goes to slot
    i * width + k; width = longest row; -1 / 0 padding."""
    n, m = csr.shape()
    lens = csr.row_lengths()
    width = int(lens.max()) if n and csr.size() else 0
    col = np.full(n * width, -1, dtype=np.int64)
    val = np.zeros(n * width, dtype=csr.dtype)
    if width:
        rows = np.repeat(np.arange(n, dtype=np.int64), lens)
        k = np.arange(csr.size(), dtype=np.int64) - csr.row_ptr()[rows]
        slot = rows * width + k
        col[slot] = csr.col_ind()
        val[slot] = csr.values()
    return Ellpack_matrix((n, m), width, col, val)


def to_jagged_diagonal(csr):
    """to_jagged_diagonal (conversions.hpp:641-691) with the layout of
    Jagged_diagonal_sparsity_Impl.cpp:11-93."""
    n, m = csr.shape()
    nnz = csr.size()
    if nnz == 0:
        return Jagged_diagonal_matrix((n, m), np.zeros(0, np.int64), np.zeros(1, np.int64),
                                      np.zeros(0, np.int64), np.zeros(0, csr.dtype))
    lens = csr.row_lengths()
    perm = np.argsort(-lens, kind="stable").astype(np.int64)
    plen = lens[perm]
    max_nnz = int(plen[0])
    # width of diagonal k = rows with length >= k + 1
    widths = np.searchsorted(-plen, -np.arange(1, max_nnz + 1), side="right").astype(np.int64)
    jdiag = np.zeros(max_nnz + 1, dtype=np.int64)
    np.cumsum(widths, out=jdiag[1:])
    # entry k of permuted row i -> jdiag[k] + i
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    k = np.arange(nnz, dtype=np.int64) - csr.row_ptr()[rows]
    inv = np.empty(n, dtype=np.int64)
    inv[perm] = np.arange(n, dtype=np.int64)
    dest = jdiag[k] + inv[rows]
    col = np.empty(nnz, dtype=np.int64)
    val = np.empty(nnz, dtype=csr.dtype)
    col[dest] = csr.col_ind()
    val[dest] = csr.values()
    return Jagged_diagonal_matrix((n, m), perm, jdiag, col, val)


def to_block_sparse_row(csr, block_rows, block_cols):
    """to_block_sparse_row (conversions.hpp:524-577): the set of touched
    (block row, block column) pairs in sorted order, dense zero-filled
    row-major blocks."""
    n, m = csr.shape()
    br, bc = int(block_rows), int(block_cols)
    nbr = (n + br - 1) // br
    lens = csr.row_lengths()
    rows = np.repeat(np.arange(n, dtype=np.int64), lens)
    cols = csr.col_ind()
    bi, bj = rows // br, cols // bc
    nbc = (m + bc - 1) // bc
    key = bi * max(nbc, 1) + bj
    uniq, inv = np.unique(key, return_inverse=True)
    ub_i, ub_j = uniq // max(nbc, 1), uniq % max(nbc, 1)
    counts = np.bincount(ub_i, minlength=nbr) if uniq.size else np.zeros(nbr, np.int64)
    rp = np.zeros(nbr + 1, dtype=np.int64)
    np.cumsum(counts, out=rp[1:])
    vals = np.zeros(uniq.size * br * bc, dtype=csr.dtype)
    vals[inv * br * bc + (rows % br) * bc + (cols % bc)] = csr.values()
    return Block_sparse_row_matrix((n, m), br, bc, rp, ub_j.astype(np.int64), vals)
