"""Parity at the benchmark configurations' own sizes (or the nearest size
the CPU oracle solves in seconds), through the C ABI.

* Configuration 3's plain solver: FP64 Jacobi-CG on the 3-D variable-
  coefficient diffusion problem (GRF sigma = 2, correlation length 8), at
  64^3: the same decision, iteration counts within +-2%.
* Configuration 3's mixed solver at 64^3: the true FP64 residual below
  1e-10, with inner FP32 work comparable to the plain solver's.
* Configuration 4's plain solver: Jacobi-FGMRES(30) on the 512^2 upwind
  convection-diffusion problem over a budget of 300 iterations: the per-step
  residual estimates |g_{j+1}| follow the oracle's.
* Configuration 2's matrix B: the full 1,000,000-row Zipf(1.5) CSR product
  in FP64, normwise within 1e-14 of the oracle's.
* Configuration 5: a batch that holds systems of n near 64k next to small
  ones; every system reaches 1e-10 on its true FP64 residual.
The oracle is bit-exact with the compiled reference on every routine used
here (test_oracle.py)."""
import numpy as np
import pytest

from sparkit_b200 import gpu, matgen
from sparkit_b200.formats import Compressed_row_matrix

pytestmark = pytest.mark.gpu


def iters_close(a, b):
    return abs(a - b) <= max(2, int(np.ceil(0.02 * b)))


@pytest.fixture(scope="module")
def grf64():
    A = matgen.diffusion_3d_grf(64, sigma=2.0, corr_len=8.0, seed=0)
    b = matgen.uniform_vector(A.shape()[0], seed=0)
    return A, b


def test_config3_plain_jacobi_cg_64cubed(gpu_lib, oracle, grf64):
    A, b = grf64
    n = A.shape()[0]
    xr, sr = oracle.cg(A, b, np.zeros(n), 1e-10, 10 ** 6, 200000, left="jacobi")
    Ad = gpu.Device_matrix(A)
    x = np.zeros(n)
    s = gpu.conjugate_gradient(b, x, gpu.CGConfig(1e-10, 10 ** 6, 200000), gpu.spmv(Ad), gpu.jacobi(Ad))
    assert s.converged and sr["converged"]
    assert iters_close(s.computed_iterations, sr["computed_iterations"]), (s.computed_iterations,
                                                                           sr["computed_iterations"])
    rel = np.linalg.norm(b - oracle.spmv(A, x)) / np.linalg.norm(b)
    rel_ref = np.linalg.norm(b - oracle.spmv(A, xr)) / np.linalg.norm(b)
    assert rel < max(2e-10, 2 * rel_ref), (rel, rel_ref)


@pytest.mark.parametrize("diagonal_copy", [False, True])
def test_config3_mixed_64cubed(gpu_lib, oracle, grf64, diagonal_copy):
    import torch
    A, b = grf64
    n = A.shape()[0]
    Ad = gpu.Device_matrix(A)
    if diagonal_copy:
        assert Ad.add_diagonals()
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    s = gpu.mixed_cg(bd, xd, gpu.Mixed_config(1e-10, 1e-5, 100, 200000), gpu.spmv(Ad))
    torch.cuda.synchronize()
    rel = np.linalg.norm(b - oracle.spmv(A, xd.cpu().numpy())) / np.linalg.norm(b)
    assert s.converged and s.persistent and rel < 1e-10, (s, rel)
    _, sr = oracle.cg(A, b, np.zeros(n), 1e-10, 10 ** 6, 200000, left="jacobi")
    assert s.inner_iterations <= 1.5 * sr["computed_iterations"], (s.inner_iterations, sr["computed_iterations"])


def test_config4_plain_fgmres_512sq_history(gpu_lib, oracle):
    A, _ = matgen.convdiff_2d_grf(512, seed=777)
    n = A.shape()[0]
    b = np.random.default_rng(3).uniform(-1, 1, n)
    Ad = gpu.Device_matrix(A)
    J = gpu.jacobi(Ad)
    x = np.zeros(n)
    s = gpu.fgmres(b, x, gpu.Fgmres_config(1e-8, 30, 300, True), gpu.spmv(Ad), J)
    xr, sr = oracle.fgmres(A, b, np.zeros(n), 1e-8, 30, 300, prec="jacobi", collect=True)
    assert s.computed_iterations == sr["computed_iterations"] == 300
    assert s.converged == sr["converged"]
    h, hr = np.array(s.iteration_residuals), np.array(sr["iteration_residuals"])
    assert h.size == hr.size == 300
    assert np.allclose(h, hr, rtol=1e-8, atol=0), np.max(np.abs(h - hr) / hr)
    assert np.linalg.norm(x - xr) <= 1e-8 * np.linalg.norm(xr)


def test_config2_matrix_b_full_csr_product(gpu_lib, oracle):
    """The full matrix B (1M rows, Zipf(1.5) lengths up to 2048, 68.9M
    entries).  The default split product sums rows of up to 32 entries in
    the reference's order (bit for bit) and longer rows in a fixed tree
    (normwise 1e-14); with the column-panel copy every row is summed in the
    reference's order and the product equals the oracle's bit for bit."""
    Z = matgen.zipf_random(1_000_000, s=1.5, cap=2048, seed=0)
    n = Z.shape()[0]
    x = matgen.uniform_vector(n, seed=1)
    Zd = gpu.Device_matrix(Z)
    assert Zd.layout() == "split"
    y = gpu.multiply(Zd, x)
    yr = oracle.spmv(Z, x)
    rows = np.repeat(np.arange(n), np.diff(np.asarray(Z.row_ptr())))
    scale = np.zeros(n)
    np.add.at(scale, rows, np.abs(np.asarray(Z.values())) * np.abs(x[np.asarray(Z.col_ind())]))
    err = np.max(np.abs(y - yr)) / np.max(scale)
    assert err <= 1e-14, err
    short = np.diff(np.asarray(Z.row_ptr())) <= 32
    assert np.array_equal(y[short], yr[short])
    assert Zd.add_panels() and Zd.layout() == "panels"
    assert np.array_equal(gpu.multiply(Zd, x), yr)


def test_config5_batch_with_64k_systems(gpu_lib, oracle):
    import torch
    big = matgen.batched_spd_systems(6, nmin=50000, nmax=65536, seed=11)
    small = matgen.batched_spd_systems(40, nmin=1000, nmax=8000, seed=12)
    offs = np.concatenate([big[0], big[0][-1] + small[0][1:]])
    rp = np.concatenate([big[1][:-1], big[1][-1] + small[1]])
    ci = np.concatenate([big[2], small[2] + big[0][-1]])
    v = np.concatenate([big[3], small[3]])
    B = gpu.Batch(offs, rp, ci, v)
    n = int(offs[-1])
    b = matgen.uniform_vector(n, seed=13)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    inner, outer, rel, conv = B.solve(bd, xd, gpu.Batch_config())
    x = xd.cpu().numpy()
    assert conv.all() and (rel < 1e-10).all()
    assert np.diff(offs).max() >= 50000
    for s in list(range(6)) + [6, 25, 45]:
        a, e = offs[s], offs[s + 1]
        rows = rp[a:e + 1] - rp[a]
        A = Compressed_row_matrix((e - a, e - a), rows, ci[rp[a]:rp[e]] - a, v[rp[a]:rp[e]].astype(np.float64))
        r = b[a:e] - oracle.spmv(A, x[a:e])
        assert np.linalg.norm(r) / np.linalg.norm(b[a:e]) < 1e-10, s
        if s < 6:
            _, sr = oracle.cg(A, b[a:e], np.zeros(e - a), 1e-10, 10 ** 6, 100000, left="jacobi")
            assert inner[s] <= 1.6 * sr["computed_iterations"] + 20, (s, inner[s], sr["computed_iterations"])
