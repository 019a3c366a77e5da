"""ELLPACK, jagged-diagonal and BSR handles built on the device from a CSR
handle (sk_ell_from_csr / sk_jad_from_csr / sk_bsr_from_csr), read back
through the export calls and held bit for bit against the reference's own
conversions (golden fixtures), against the host restatement at full size,
and through the product: a converted handle multiplies exactly like the
handle uploaded from the host conversion."""
import numpy as np
import pytest

from sparkit_b200 import formats, gpu, matgen
from sparkit_b200.formats import Compressed_row_matrix
from tests.golden.make_golden import CONVERT_BLOCKS
from tests.helpers import SPMV_CASES, golden_csr

pytestmark = pytest.mark.gpu

CASES = SPMV_CASES + ["empty_5x4"]


def _csr(golden, name, dtype=np.float64):
    if name == "empty_5x4":
        return Compressed_row_matrix((5, 4), np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0, dtype))
    return golden_csr(golden, f"spmv/{name}/float64").astype(dtype)


def _same(got, want):
    assert got.dtype == want.dtype, (got.dtype, want.dtype)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("name", CASES)
def test_conversions_match_reference_fixtures(gpu_lib, golden, name):
    A = _csr(golden, name)
    Ad = gpu.Device_matrix(A)
    tag = f"convert/{name}"
    E = gpu.to_ellpack(Ad).to_host()
    if f"{tag}/ell/width" in golden:
        assert E.max_nnz_per_row() == int(golden[f"{tag}/ell/width"])
        _same(E.col_ind(), golden[f"{tag}/ell/col_ind"])
        _same(E.values(), golden[f"{tag}/ell/values"])
    else:  # the host restatement, pinned to the reference on the CPU
        R = formats.to_ellpack(A)
        assert E.max_nnz_per_row() == R.max_nnz_per_row()
        _same(E.col_ind(), R.col_ind())
        _same(E.values(), R.values())
    J = gpu.to_jagged_diagonal(Ad).to_host()
    for f in ("perm", "jdiag", "col_ind", "values"):
        _same(getattr(J, f)(), golden[f"{tag}/jad/{f}"])
    for br, bc in CONVERT_BLOCKS:
        B = gpu.to_block_sparse_row(Ad, br, bc).to_host()
        for f in ("row_ptr", "col_ind", "values"):
            _same(getattr(B, f)(), golden[f"{tag}/bsr{br}x{bc}/{f}"])


@pytest.mark.parametrize("name", ["lap3d_6", "zipf_400", "rect_37x53", "longrow_3000", "odd_7"])
def test_converted_handles_multiply_like_uploaded_ones(gpu_lib, golden, name):
    """The same layout gives the same product bits, FP64 and FP32."""
    for dt in (np.float64, np.float32):
        A = _csr(golden, name, dt)
        Ad = gpu.Device_matrix(A)
        x = matgen.uniform_vector(A.shape()[1], seed=4, dtype=dt)
        pairs = [(gpu.to_ellpack(Ad), formats.to_ellpack(A)),
                 (gpu.to_jagged_diagonal(Ad), formats.to_jagged_diagonal(A))]
        for br, bc in ((2, 2), (3, 3), (2, 3), (5, 7)):
            pairs.append((gpu.to_block_sparse_row(Ad, br, bc), formats.to_block_sparse_row(A, br, bc)))
        for dev, host in pairs:
            up = gpu.Device_matrix(host)
            assert dev.info()["nnz"] == up.info()["nnz"] and dev.info()["width"] == up.info()["width"]
            assert dev.build_ms() > 0.0 and up.build_ms() == 0.0
            _same(gpu.multiply(dev, x), gpu.multiply(up, x))


def test_export_roundtrip_of_uploaded_handles(gpu_lib, golden):
    """Export reads back exactly what the host upload stored."""
    A = _csr(golden, "rect_37x53")
    for host in (A, formats.to_ellpack(A), formats.to_jagged_diagonal(A), formats.to_block_sparse_row(A, 2, 3)):
        back = gpu.Device_matrix(host).to_host()
        assert type(back) is type(host)
        fields = {"Compressed_row_matrix": ("row_ptr", "col_ind", "values"),
                  "Ellpack_matrix": ("col_ind", "values"),
                  "Jagged_diagonal_matrix": ("perm", "jdiag", "col_ind", "values"),
                  "Block_sparse_row_matrix": ("row_ptr", "col_ind", "values")}[type(host).__name__]
        for f in fields:
            _same(getattr(back, f)(), getattr(host, f)())


def test_jad_ties_and_multipass_sort(gpu_lib):
    """Row lengths up to 700 (three radix passes of 8 bits) with many ties:
    the permutation keeps equal-length rows in row order."""
    rng = np.random.default_rng(12)
    n, m = 50_000, 4096
    lens = np.where(rng.random(n) < 0.002, rng.integers(256, 700, n), rng.integers(0, 12, n))
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lens, out=rp[1:])
    ci = np.concatenate([np.sort(rng.choice(m, k, replace=False)) for k in lens]).astype(np.int64)
    A = Compressed_row_matrix((n, m), rp, ci, rng.standard_normal(rp[-1]))
    J = gpu.to_jagged_diagonal(gpu.Device_matrix(A)).to_host()
    R = formats.to_jagged_diagonal(A)
    for f in ("perm", "jdiag", "col_ind", "values"):
        _same(getattr(J, f)(), getattr(R, f)())


@pytest.mark.parametrize("which", ["lap3d_128", "zipf_1m"])
def test_full_size_against_host_restatement(gpu_lib, which):
    """The matrices of the format sweep: the 128^3 7-point Laplacian
    (CSR -> ELL, JAD) and the 3x3-block vector Laplacian on a 64^3 grid
    (CSR -> BSR, 786k rows), and the 1M-row Zipf matrix (CSR -> JAD; its ELL
    of 2.05e9 slots is checked through the product, against SciPy in FP64:
    two sums of at most 2048 terms in any order differ by at most
    2 * 2048 * 2^-53 of |A| |x|)."""
    if which == "lap3d_128":
        A = matgen.laplacian_3d_dirichlet(128)
        Ad = gpu.Device_matrix(A)
        for dev, host in ((gpu.to_ellpack(Ad), formats.to_ellpack(A)),
                          (gpu.to_jagged_diagonal(Ad), formats.to_jagged_diagonal(A))):
            got = dev.to_host()
            for f in ("col_ind", "values"):
                _same(getattr(got, f)(), getattr(host, f)())
        V = matgen.vector_laplacian_3d_bsr_csr(64, seed=0)
        got = gpu.to_block_sparse_row(gpu.Device_matrix(V), 3, 3).to_host()
        want = formats.to_block_sparse_row(V, 3, 3)
        for f in ("row_ptr", "col_ind", "values"):
            _same(getattr(got, f)(), getattr(want, f)())
    else:
        import scipy.sparse as sp
        A = matgen.zipf_random(1_000_000, s=1.5, cap=2048, seed=0)
        Ad = gpu.Device_matrix(A)
        got = gpu.to_jagged_diagonal(Ad).to_host()
        want = formats.to_jagged_diagonal(A)
        for f in ("perm", "jdiag", "col_ind", "values"):
            _same(getattr(got, f)(), getattr(want, f)())
        E = gpu.to_ellpack(Ad)
        assert E.info()["width"] == int(np.diff(A.row_ptr()).max())
        x = matgen.uniform_vector(A.shape()[1], seed=1)
        y = gpu.multiply(E, x)
        E.close()
        n, m = A.shape()
        S = sp.csr_matrix((A.values(), A.col_ind(), A.row_ptr()), shape=(n, m))
        bound = 2 * 2048 * 2.0 ** -53 * (abs(S) @ np.abs(x)) + 1e-300
        assert np.all(np.abs(y - S @ x) <= bound)


def test_conversion_arguments(gpu_lib, golden):
    from sparkit_b200 import _lib
    A = _csr(golden, "odd_7")
    Ad = gpu.Device_matrix(A)
    with pytest.raises(_lib.SkError):
        gpu.to_block_sparse_row(Ad, 0, 2)
    with pytest.raises(_lib.SkError):
        gpu.to_block_sparse_row(Ad, 257, 1)
    E = gpu.to_ellpack(Ad)
    with pytest.raises(_lib.SkError):
        gpu.to_jagged_diagonal(E)  # the source must be CSR
