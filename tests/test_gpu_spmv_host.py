"""The host-buffer product (sk_spmv_host, the drop-in multiply(A, x)) cuts
a CSR product of at least 8 MiB of y into row chunks of about 4 MiB: x
goes up in prefixes on one copy stream, each chunk's product waits for the
prefix its columns reach, and y comes down chunk by chunk on another.
Whatever the pattern (banded, reversed, wide, skewed rows, empty chunks)
the result is the device product's, bit for bit, and the oracle's where
each row is summed by one thread."""
import numpy as np
import pytest

from sparkit_b200 import formats, gpu, matgen

pytestmark = pytest.mark.gpu


def _device_product(Ad, x):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yd = torch.empty(Ad.shape()[0], dtype=xd.dtype, device="cuda")
    Ad.spmv(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


def _reverse_rows(A):
    n = A.shape()[0]
    rp, ci, va = A.row_ptr(), A.col_ind(), A.values()
    lens = np.diff(rp)[::-1]
    rp2 = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp2[1:])
    # entry k of new row i is entry k of old row n-1-i
    order = np.repeat(rp[:-1][::-1] - rp2[:-1], lens) + np.arange(rp2[-1])
    return formats.Compressed_row_matrix(A.shape(), rp2, ci[order], va[order])


def _check(A, x, oracle=None, exact=True):
    Ad = gpu.Device_matrix(A)
    y = gpu.multiply(Ad, x)
    assert np.array_equal(y, _device_product(Ad, x))
    if oracle is not None and exact:
        assert np.array_equal(y, oracle.spmv(A, x))
    # the plan is kept: a second call with another x on the same handle
    x2 = -2.0 * x[::-1].copy()
    assert np.array_equal(gpu.multiply(Ad, x2), _device_product(Ad, x2))
    Ad.close()
    return y


def test_banded_and_reversed(gpu_lib, oracle):
    """The 128^3 7-point Laplacian (2,097,152 rows, SELL path; 4 chunks in
    FP64, 2 in FP32) in natural order (chunk c reads x up to one grid plane
    past its rows) and with its rows reversed (chunk 0 reads the last
    columns, so its piece is all of x)."""
    A = matgen.laplacian_3d_dirichlet(128)
    x = matgen.uniform_vector(A.shape()[1], seed=11)
    for M in (A, _reverse_rows(A)):
        _check(M, x, oracle)
        _check(M.astype(np.float32), x.astype(np.float32), oracle)


def test_wide_and_empty_chunks(gpu_lib, oracle):
    """A wide matrix (1.2M x 3.6M, row r reads columns 3r..3r+2): the last
    piece carries the columns no chunk reads before the end.  A 2.4M-row
    matrix whose first three quarters of rows are empty: those chunks have
    no piece of x."""
    n = 1_200_000
    r = np.repeat(np.arange(n), 3)
    c = 3 * r + np.tile(np.arange(3), n)
    rng = np.random.default_rng(3)
    W = formats.Compressed_row_matrix.from_entries((n, 3 * n), r, c, rng.standard_normal(r.size))
    _check(W, matgen.uniform_vector(3 * n, seed=2), oracle)
    m = 2_400_000
    rows = np.arange(3 * m // 4, m)
    H = formats.Compressed_row_matrix.from_entries((m, m), rows, rows, rng.standard_normal(rows.size))
    y = _check(H, matgen.uniform_vector(m, seed=4), oracle)
    assert not y[: 3 * m // 4].any()


def test_skewed_rows_tiled_path(gpu_lib, oracle):
    """A 1.2M-row Zipf(1.5) matrix (rows up to 2048 entries: the tiled CSR
    kernel, chunks cut at its tile boundaries)."""
    A = matgen.zipf_random(1_200_000, s=1.5, cap=2048, seed=0)
    _check(A, matgen.uniform_vector(A.shape()[1], seed=1), oracle, exact=False)
