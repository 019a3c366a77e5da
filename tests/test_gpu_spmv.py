"""SpMV parity on the GPU, through the C ABI.

Bar: bit-exact against the reference wherever each row is summed by one
thread in storage order (every ELL, JAD and BSR row; CSR row blocks whose
rows hold at most 32 entries).  CSR blocks with longer rows are summed by
several lanes; there the normwise error
||y - y_ref||_inf / || |A| |x| ||_inf must stay below 1e-14 (FP64) or
1e-6 (FP32)."""
import numpy as np
import pytest

from sparkit_b200 import _lib, formats, gpu, matgen
from tests.helpers import BSR_BLOCKS, SPMV_CASES, convert, csr_from_entries, golden_csr

pytestmark = pytest.mark.gpu

TOL = {np.dtype(np.float64): 1e-14, np.dtype(np.float32): 1e-6}


def normwise_err(A, x, y, y_ref):
    absA = formats.Compressed_row_matrix(A.shape(), A.row_ptr(), A.col_ind(), np.abs(A.values()).astype(np.float64))
    rows = np.repeat(np.arange(A.shape()[0]), A.row_lengths())
    scale = np.zeros(A.shape()[0])
    np.add.at(scale, rows, np.abs(A.values()).astype(np.float64) * np.abs(x.astype(np.float64))[A.col_ind()])
    denom = max(scale.max() if scale.size else 0.0, np.finfo(np.float64).tiny)
    del absA
    return np.max(np.abs(y.astype(np.float64) - y_ref.astype(np.float64))) / denom if y.size else 0.0


def test_known_answers(gpu_lib, known):
    for case in known["spmv"]:
        A = csr_from_entries(tuple(case["shape"]), case["entries"])
        M = convert(A, case["format"], tuple(case.get("block", (3, 3))))
        Ad = gpu.Device_matrix(M)
        y = gpu.multiply(Ad, np.array(case["x"]))
        assert y.tolist() == case["y"], case["name"]


@pytest.mark.parametrize("name", SPMV_CASES)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_golden_all_formats(gpu_lib, golden, name, dtype):
    tag = f"spmv/{name}/{dtype}"
    A = golden_csr(golden, tag)
    x = golden[f"{tag}/x"]
    for fmt in ("csr", "ell", "jad"):
        y = gpu.multiply(gpu.Device_matrix(convert(A, fmt)), x)
        y_ref = golden[f"{tag}/y_{fmt}"]
        if fmt == "csr" and A.row_lengths().max(initial=0) > 32:
            assert normwise_err(A, x, y, y_ref) <= TOL[A.dtype], fmt
        else:
            assert np.array_equal(y, y_ref), fmt
    for key, blk in BSR_BLOCKS.items():
        y = gpu.multiply(gpu.Device_matrix(formats.to_block_sparse_row(A, *blk)), x)
        assert np.array_equal(y, golden[f"{tag}/y_bsr{blk[0]}{blk[1]}"]), key


def test_lap3d_128_full_size_bitwise(gpu_lib, oracle):
    """The benchmark matrix (n = 2,097,152, nnz = 14,581,760) in every
    scalar format, bit for bit against the oracle."""
    A = matgen.laplacian_3d_dirichlet(128)
    assert A.size() == 14581760
    x = matgen.uniform_vector(A.shape()[0], seed=1)
    y_ref = oracle.spmv(A, x)
    for fmt in ("csr", "ell", "jad"):
        M = convert(A, fmt)
        Ad = gpu.Device_matrix(M)
        assert np.array_equal(gpu.multiply(Ad, x), y_ref), fmt
        Ad.close()
    A32 = A.astype(np.float32)
    x32 = x.astype(np.float32)
    assert np.array_equal(gpu.multiply(gpu.Device_matrix(A32), x32), oracle.spmv(A32, x32))


def test_vector_laplacian_bsr33_bitwise(gpu_lib, oracle):
    V = matgen.vector_laplacian_3d_bsr_csr(24, seed=3)
    B = formats.to_block_sparse_row(V, 3, 3)
    x = matgen.uniform_vector(V.shape()[0], seed=2)
    assert np.array_equal(gpu.multiply(gpu.Device_matrix(B), x), oracle.spmv(B, x))


def test_zipf_skewed_rows(gpu_lib, oracle):
    """Skewed rows (Zipf(1.5) lengths capped at 2048) exercise the lane and
    long-row paths; checked normwise, and bit-exact for ELL / JAD."""
    A = matgen.zipf_random(60000, s=1.5, cap=2048, seed=5)
    x = matgen.uniform_vector(A.shape()[0], seed=6)
    y_ref = oracle.spmv(A, x)
    y = gpu.multiply(gpu.Device_matrix(A), x)
    assert normwise_err(A, x, y, y_ref) <= 1e-14
    J = formats.to_jagged_diagonal(A)
    assert np.array_equal(gpu.multiply(gpu.Device_matrix(J), x), oracle.spmv(J, x))
    # a row longer than one CTA tile (2048 entries) takes the long-row path
    n = 5000
    rng = np.random.default_rng(9)
    rows = np.concatenate([np.full(4500, 17), rng.integers(0, n, 3000)])
    cols = np.concatenate([rng.permutation(n)[:4500], rng.integers(0, n, 3000)])
    L = formats.Compressed_row_matrix.from_entries((n, n), rows, cols, rng.standard_normal(rows.size))
    xl = matgen.uniform_vector(n, seed=8)
    yl = gpu.multiply(gpu.Device_matrix(L), xl)
    assert normwise_err(L, xl, yl, oracle.spmv(L, xl)) <= 1e-14


def test_device_pointer_path_and_fp32_copy(gpu_lib, oracle):
    import torch
    A = matgen.laplacian_3d_dirichlet(32)
    n = A.shape()[0]
    x = matgen.uniform_vector(n, seed=3)
    Ad = gpu.Device_matrix(A)
    xd = torch.from_numpy(x).cuda()
    yd = torch.empty_like(xd)
    Ad.spmv(xd, yd)
    torch.cuda.synchronize()
    assert np.array_equal(yd.cpu().numpy(), oracle.spmv(A, x))
    Ad.add_f32_values()
    x32 = xd.float()
    y32 = torch.empty_like(x32)
    Ad.spmv_f32(x32, y32)
    torch.cuda.synchronize()
    assert np.array_equal(y32.cpu().numpy(), oracle.spmv(A.astype(np.float32), x.astype(np.float32)))


def test_edge_shapes(gpu_lib):
    # zero rows, zero columns, all-empty rows
    for shape in ((0, 0), (0, 5), (4, 0), (6, 6)):
        A = formats.Compressed_row_matrix(shape, np.zeros(shape[0] + 1, np.int64), np.zeros(0, np.int64),
                                          np.zeros(0))
        for fmt in ("csr", "ell", "jad", "bsr22"):
            M = convert(A, fmt, (2, 2))
            y = gpu.multiply(gpu.Device_matrix(M), np.ones(shape[1]))
            assert y.shape == (shape[0],) and not y.any()


def test_index_validation(gpu_lib):
    A = formats.Compressed_row_matrix((2, 2), [0, 1, 2], [0, 5], [1.0, 2.0])  # column 5 >= ncol
    with pytest.raises(_lib.SkError) as e:
        gpu.Device_matrix(A)
    assert e.value.status == 2  # SK_INDEX_OVERFLOW
    E = formats.Ellpack_matrix((2, 2), 1, [0, 1 << 33], [1.0, 1.0])  # beyond int32
    with pytest.raises(_lib.SkError):
        gpu.Device_matrix(E)
    big = formats.Compressed_row_matrix((1, 1 << 31), [0, 0], np.zeros(0, np.int64), np.zeros(0))
    with pytest.raises(_lib.SkError) as e:
        gpu.Device_matrix(big)
    assert e.value.status == 2


def _poisoned_product(Ad, x):
    """y = A x on the device into a NaN-filled output, so that a row the
    kernel skips shows up as NaN."""
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yd = torch.full((Ad.shape()[0],), float("nan"), dtype=xd.dtype, device="cuda")
    Ad.spmv(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("fmt", ["csr", "ell", "jad", "bsr22", "bsr33"])
def test_small_case_sweep_writes_every_row(gpu_lib, oracle, fmt):
    """Small-case sweep (n = 1..64; empty rows; a single dense row; a row
    longer than 32 among short ones) with NaN-poisoned outputs, against the
    oracle: every row is written, with the oracle's bits where one thread
    sums the row (every non-CSR format and CSR rows of up to 32 entries)."""
    rng = np.random.default_rng(21)
    cases = []
    for n in list(range(1, 17)) + [31, 32, 33, 63, 64]:
        lens = rng.integers(0, min(n, 6) + 1, size=n)
        lens[rng.integers(0, n)] = 0                      # an empty row
        cases.append((n, lens))
    dense = np.zeros(48, dtype=np.int64)
    dense[17] = 48                                         # one dense row
    cases.append((48, dense))
    mixed = rng.integers(0, 4, size=64)
    mixed[5] = 40                                          # a row longer than 32
    cases.append((64, mixed))
    for n, lens in cases:
        rp = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
        ci = np.concatenate([np.sort(rng.choice(n, size=int(k), replace=False)) for k in lens]).astype(np.int64) \
            if lens.sum() else np.zeros(0, np.int64)
        va = rng.standard_normal(int(lens.sum()))
        A = formats.Compressed_row_matrix((n, n), rp, ci, va)
        block = BSR_BLOCKS.get(fmt, (3, 3))
        M = convert(A, fmt, block)
        x = rng.uniform(-1, 1, n)
        y = _poisoned_product(gpu.Device_matrix(M), x)
        y_ref = oracle.spmv(M, x)
        assert not np.isnan(y).any(), (fmt, n)
        if fmt == "csr":
            short = lens <= 32
            assert np.array_equal(y[short], y_ref[short]), (fmt, n)
            assert normwise_err(A, x, y, y_ref) <= 1e-14, (fmt, n)
        else:
            assert np.array_equal(y, y_ref), (fmt, n)


@pytest.mark.parametrize("dtype,n", [(np.float64, 300_000), (np.float32, 600_000)])
def test_panel_product_bit_identical(gpu_lib, oracle, dtype, n):
    """The column-panel copy (sk_matrix_add_panels) of a large skewed matrix
    (Zipf(1.5) row lengths up to 2048, uniform columns over an x of 2.4 MB)
    sums every row in ascending column order from 0, panel after panel: the
    oracle's bits for rows of every length.  x once 16-byte aligned (16-byte staging
    copies) and once at an 8- or 4-byte offset (element copies)."""
    import torch
    Z = matgen.zipf_random(n, s=1.5, cap=2048, seed=5, dtype=dtype)
    Zd = gpu.Device_matrix(Z)
    assert Zd.layout() == "split"
    assert Zd.add_panels() and Zd.layout() == "panels"
    x = matgen.uniform_vector(n, seed=6, dtype=dtype)
    yr = oracle.spmv(Z, x)
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    for shift in (0, 1):
        buf = torch.empty(n + 1, dtype=tdt, device="cuda")
        xd = buf[shift:shift + n]
        xd.copy_(torch.from_numpy(x))
        yd = torch.full((n,), float("nan"), dtype=tdt, device="cuda")
        Zd.spmv(xd, yd)
        torch.cuda.synchronize()
        assert np.array_equal(yd.cpu().numpy(), yr), shift


def test_panel_copy_only_where_the_order_is_not_kept(gpu_lib, oracle):
    """A SELL-32 handle already sums each row in storage order, so the panel
    copy is refused; a small skewed handle takes it and then matches the
    oracle bit for bit (one panel, a handful of row blocks)."""
    A = matgen.laplacian_2d_dirichlet(64)
    Ad = gpu.Device_matrix(A)
    assert Ad.layout() == "sell" and not Ad.add_panels() and Ad.layout() == "sell"
    Z = matgen.zipf_random(20_000, s=1.5, cap=2048, seed=1)
    Zd = gpu.Device_matrix(Z)
    assert Zd.layout() in ("split", "native")
    assert Zd.add_panels() and Zd.layout() == "panels"
    x = matgen.uniform_vector(Z.shape()[0], seed=2)
    assert np.array_equal(gpu.multiply(Zd, x), oracle.spmv(Z, x))
