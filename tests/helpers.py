"""Helpers shared by the tests: matrices from golden arrays and entry lists."""
import numpy as np

from sparkit_b200 import formats
from sparkit_b200.formats import Compressed_row_matrix


def csr_from_entries(shape, entries, dtype=np.float64):
    if entries:
        e = np.array(entries, dtype=np.float64)
        return Compressed_row_matrix.from_entries(shape, e[:, 0].astype(np.int64), e[:, 1].astype(np.int64),
                                                  e[:, 2], dtype=dtype)
    return Compressed_row_matrix(shape, np.zeros(shape[0] + 1, np.int64), np.zeros(0, np.int64),
                                 np.zeros(0, dtype))


def golden_csr(g, tag):
    shape = tuple(int(v) for v in g[f"{tag}/shape"])
    return Compressed_row_matrix(shape, g[f"{tag}/row_ptr"], g[f"{tag}/col_ind"], g[f"{tag}/values"])


def golden_problem(g, name):
    rp = g[f"solve/{name}/row_ptr"]
    n = rp.size - 1
    return Compressed_row_matrix((n, n), rp, g[f"solve/{name}/col_ind"], g[f"solve/{name}/values"])


def convert(A, fmt, block=(3, 3)):
    if fmt == "csr":
        return A
    if fmt == "ell":
        return formats.to_ellpack(A)
    if fmt == "jad":
        return formats.to_jagged_diagonal(A)
    if fmt.startswith("bsr"):
        return formats.to_block_sparse_row(A, *block)
    raise ValueError(fmt)


SPMV_CASES = ["lap2d_16", "lap3d_6", "zipf_400", "vec3_4", "rect_37x53", "longrow_3000", "odd_7"]
BSR_BLOCKS = {"bsr22": (2, 2), "bsr33": (3, 3), "bsr23": (2, 3)}
