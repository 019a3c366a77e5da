"""The diagonal copy of a CSR handle (sk_matrix_add_diagonals).  It is built
only for patterns on at most 16 diagonals whose rows hold ascending
columns, and every product and solver step on the handle then gives the
bits it gives without the copy: the rows are summed over their stored
entries in CSR order, and the kernels with fused reductions run the SELL
grid, so the same rows meet in the same CTAs.  The persistent FP32 inner
solve over the copy runs its own grid and is held to the iteration band."""
import numpy as np
import pytest

from sparkit_b200 import _lib, formats, gpu, matgen

pytestmark = pytest.mark.gpu


def _pair(A):
    plain = gpu.Device_matrix(A)
    dia = gpu.Device_matrix(A)
    assert dia.add_diagonals()
    return plain, dia


def _device_product(Ad, x):
    import torch
    xd = torch.from_numpy(np.ascontiguousarray(x)).cuda()
    yd = torch.empty(Ad.shape()[0], dtype=xd.dtype, device="cuda")
    Ad.spmv(xd, yd)
    torch.cuda.synchronize()
    return yd.cpu().numpy()


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_products_keep_their_bits(gpu_lib, oracle, dtype):
    """3-D and 2-D Dirichlet Laplacians (boundary rows miss diagonals) and a
    GRF diffusion stencil: the host and device products equal those of the
    handle without the copy and the oracle's, bit for bit; the byte model
    drops the column indices."""
    dt = np.dtype(dtype)
    for A in (matgen.laplacian_3d_dirichlet(24), matgen.laplacian_2d_dirichlet(37),
              matgen.diffusion_3d_grf(16, sigma=2.0, corr_len=4.0, seed=2)):
        M = A.astype(dt)
        plain, dia = _pair(M)
        n = M.shape()[0]
        assert dia.info()["spmv_bytes"] < plain.info()["spmv_bytes"]
        x = matgen.uniform_vector(n, seed=5, dtype=dt)
        y = gpu.multiply(dia, x)
        assert np.array_equal(y, gpu.multiply(plain, x))
        assert np.array_equal(y, oracle.spmv(M, x))
        assert np.array_equal(_device_product(dia, x), _device_product(plain, x))


def test_absent_entries_are_not_read(gpu_lib):
    """Rows that do not store a diagonal never touch x there: an inf or a
    NaN in x reaches exactly the rows whose CSR entries reach it."""
    g = 8
    A = matgen.laplacian_3d_dirichlet(g)
    plain, dia = _pair(A)
    x = matgen.uniform_vector(A.shape()[1], seed=1)
    x[g - 1] = np.inf  # row g (k = 0) stores no entry at column g - 1
    x[3 * g * g] = np.nan
    y = gpu.multiply(dia, x)
    assert np.array_equal(y, gpu.multiply(plain, x), equal_nan=True)
    assert np.isfinite(y[g])


def test_refused_patterns(gpu_lib, oracle):
    """More than 16 diagonals, planes more than half empty, a row whose
    columns do not ascend, or a duplicated column: no copy, and the handle
    multiplies as before.  A non-CSR handle is an error."""
    rng = np.random.default_rng(4)
    n = 3000
    cases = []
    offs = np.arange(-10, 10)  # 20 diagonals
    r = np.repeat(np.arange(n), offs.size)
    c = r + np.tile(offs, n)
    keep = (c >= 0) & (c < n)
    cases.append(formats.Compressed_row_matrix.from_entries((n, n), r[keep], c[keep], rng.standard_normal(keep.sum())))
    r = np.concatenate([np.arange(n), [5, 9], [7]])
    c = np.concatenate([np.arange(n), [5 + 100, 9 + 100], [7 + 300]])  # 3 diagonals, 3 off-diagonal entries
    cases.append(formats.Compressed_row_matrix.from_entries((n, n), r, c, rng.standard_normal(r.size)))
    L = matgen.laplacian_2d_dirichlet(40)
    rp, ci, va = L.row_ptr().copy(), L.col_ind().copy(), L.values().copy()
    ci[rp[100]:rp[101]] = ci[rp[100]:rp[101]][::-1].copy()  # row 100 descending
    va[rp[100]:rp[101]] = va[rp[100]:rp[101]][::-1].copy()
    cases.append(formats.Compressed_row_matrix(L.shape(), rp, ci, va))
    cases.append(matgen.zipf_random(5000, s=1.5, cap=64, seed=3))
    for A in cases:
        Ad = gpu.Device_matrix(A)
        assert not Ad.add_diagonals()
        x = matgen.uniform_vector(A.shape()[1], seed=2)
        y = gpu.multiply(Ad, x)
        assert np.allclose(y, oracle.spmv(A, x), rtol=1e-13, atol=1e-13)
    E = gpu.Device_matrix(formats.to_ellpack(matgen.laplacian_2d_dirichlet(8)))
    with pytest.raises(_lib.SkError):
        E.add_diagonals()


def test_solvers_keep_their_bits(gpu_lib, oracle):
    """Jacobi-CG and BiCGSTAB in FP64, and the mixed solver with its
    per-step inner solve (FP32 products through the diagonal copy), on a
    GRF diffusion problem: the same iteration counts and the same solution
    bits with and without the copy.  The persistent inner solve over the
    copy runs twice the CTAs of the SELL one, so its dot products are summed
    in another order: it reaches the tolerance on the true FP64 residual
    with inner iteration counts within 2% of the SELL solve's and of the
    per-step solve's over the same copy."""
    import torch
    A = matgen.diffusion_3d_grf(24, sigma=2.0, corr_len=8.0, seed=0)
    n = A.shape()[0]
    plain, dia = _pair(A)
    b = torch.from_numpy(matgen.uniform_vector(n, seed=0)).cuda()

    def run(solve):
        out = []
        for Ad in (plain, dia):
            x = torch.zeros_like(b)
            s = solve(Ad, x)
            torch.cuda.synchronize()
            out.append((s, x.cpu().numpy()))
        return out

    (s0, x0), (s1, x1) = run(lambda Ad, x: gpu.conjugate_gradient(
        b, x, gpu.CGConfig(1e-10, 10 ** 6, 20000), gpu.spmv(Ad), gpu.jacobi(Ad)))
    assert s0.converged and s0.computed_iterations == s1.computed_iterations
    assert np.array_equal(x0, x1)
    (s0, x0), (s1, x1) = run(lambda Ad, x: gpu.bicgstab(
        b, x, gpu.Bicgstab_config(1e-10, 20000), gpu.spmv(Ad), gpu.jacobi(Ad)))
    assert s0.converged and s0.computed_iterations == s1.computed_iterations
    assert np.array_equal(x0, x1)
    inner = {}
    for persistent in (True, False):
        cfg = gpu.Mixed_config(1e-10, 1e-5, 50, 100000, persistent=persistent)
        (s0, x0), (s1, x1) = run(lambda Ad, x: gpu.mixed_cg(b, x, cfg, gpu.spmv(Ad)))
        assert s0.converged and s1.converged and s0.persistent == persistent and s1.persistent == persistent
        inner[persistent] = (s0.inner_iterations, s1.inner_iterations)
        if persistent:
            rel = np.linalg.norm(b.cpu().numpy() - oracle.spmv(A, x1)) / np.linalg.norm(b.cpu().numpy())
            assert rel < 1e-10, rel
        else:
            assert (s0.outer_iterations, s0.inner_iterations) == (s1.outer_iterations, s1.inner_iterations)
            assert np.array_equal(x0, x1)
    sell_p, dia_p = inner[True]
    dia_s = inner[False][1]
    assert abs(dia_p - sell_p) <= 0.02 * sell_p + 2, inner
    assert abs(dia_p - dia_s) <= 0.02 * dia_s + 2, inner


def test_host_pipeline_with_diagonals(gpu_lib, oracle):
    """The 128^3 Laplacian through the pipelined host-buffer product (4 row
    chunks, each a launch of the diagonal kernel over its rows)."""
    A = matgen.laplacian_3d_dirichlet(128)
    plain, dia = _pair(A)
    x = matgen.uniform_vector(A.shape()[1], seed=1)
    y = gpu.multiply(dia, x)
    assert np.array_equal(y, gpu.multiply(plain, x))
    assert np.array_equal(y, oracle.spmv(A, x))
