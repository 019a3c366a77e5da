"""The failure paths, driven by ordinary host input on a healthy GPU.

Breakdowns: BiCGSTAB systems whose exact arithmetic makes rho = 0 after a
step, or <r_hat, v> = 0 in the first step, end with SK_BREAKDOWN and
converged == false.  At rho = 0 the reference's step returns without using
budget, so its loop never ends (bicgstab.hpp:203-204); at <r_hat, v> = 0 it
divides by zero (:211) and spends its budget on NaNs.  An exact initial
guess (r_0 = 0, so rho_0 = 0) is where the reference spins from the start;
here it ends converged after 0 iterations.

Timeouts: every grid-barrier wait of the persistent kernels is bounded.
sk_debug_set_wait shortens the bound to 1 ms and makes each barrier wait for
one arrival more than the grid makes, so the first wait runs out on a
correct solve: the kernel returns, the call reports SK_TIMEOUT, and the
same handles solve normally once the setting is cleared."""
import numpy as np
import pytest

from sparkit_b200 import _lib, gpu, matgen
from sparkit_b200.formats import Compressed_row_matrix

pytestmark = pytest.mark.gpu

SK_BREAKDOWN, SK_TIMEOUT = 4, 6


def dense_csr(a):
    a = np.asarray(a, dtype=np.float64)
    rows, cols = np.nonzero(a)
    rp = np.zeros(a.shape[0] + 1, dtype=np.int64)
    np.add.at(rp, rows + 1, 1)
    return Compressed_row_matrix(a.shape, np.cumsum(rp), cols.astype(np.int64), a[rows, cols])


def test_bicgstab_rho_breakdown(gpu_lib):
    # step 1: r_0 = -e_1, v = (1, 0, 2), alpha = -1, s = (0, 0, 2), t = (0, 4, 2),
    # omega = 0.2, r_1 = (0, -0.8, 1.6): rho_1 = <r_0, r_1> = 0 exactly, r_1 != 0
    A = dense_csr([[-1, 0, 0], [0, 2, 2], [-2, -1, 1]])
    Ad = gpu.Device_matrix(A)
    x = np.zeros(3)
    s = gpu.bicgstab(np.array([-1.0, 0.0, 0.0]), x, gpu.Bicgstab_config(1e-12, 100), gpu.spmv(Ad))
    assert s.status == SK_BREAKDOWN and not s.converged and s.computed_iterations == 2, s


def test_bicgstab_rhat_v_breakdown(gpu_lib):
    A = dense_csr([[0, 1], [1, 0]])
    Ad = gpu.Device_matrix(A)
    s = gpu.bicgstab(np.array([1.0, 0.0]), np.zeros(2), gpu.Bicgstab_config(1e-12, 100), gpu.spmv(Ad))
    assert s.status == SK_BREAKDOWN and not s.converged and s.computed_iterations == 1, s


def test_bicgstab_exact_initial_guess(gpu_lib):
    A = matgen.tridiagonal_matrix(64, -1.0, 4.0, -1.0)
    Ad = gpu.Device_matrix(A)
    x0 = np.arange(64, dtype=np.float64) - 20.0   # integers: A x0 is exact
    b = gpu.multiply(Ad, x0)
    x = x0.copy()
    s = gpu.bicgstab(b, x, gpu.Bicgstab_config(1e-12, 100), gpu.spmv(Ad), gpu.jacobi(Ad))
    assert s.status == 0 and s.converged and s.computed_iterations == 0
    assert np.array_equal(x, x0)


@pytest.fixture
def short_unmeetable_waits(gpu_lib):
    gpu.debug_set_wait(1_000_000, True)
    try:
        yield
    finally:
        gpu.debug_set_wait(0, False)


def test_mixed_inner_barrier_timeout(gpu_lib, oracle):
    import torch
    A = matgen.laplacian_3d_dirichlet(16)
    n = A.shape()[0]
    b = matgen.uniform_vector(n, seed=1)
    Ad = gpu.Device_matrix(A)
    bd = torch.from_numpy(b).cuda()
    cfg = gpu.Mixed_config(1e-10, 1e-5, 20, 10000)
    gpu.debug_set_wait(1_000_000, True)
    try:
        xd = torch.zeros_like(bd)
        with pytest.raises(_lib.SkError) as e:
            gpu.mixed_cg(bd, xd, cfg, gpu.spmv(Ad))
        assert e.value.status == SK_TIMEOUT and "barrier" in str(e.value)
    finally:
        gpu.debug_set_wait(0, False)
    xd = torch.zeros_like(bd)
    s = gpu.mixed_cg(bd, xd, cfg, gpu.spmv(Ad))
    torch.cuda.synchronize()
    rel = np.linalg.norm(b - oracle.spmv(A, xd.cpu().numpy())) / np.linalg.norm(b)
    assert s.persistent and s.converged and rel < 1e-10


@pytest.mark.parametrize("solver", ["gmres", "fgmres"])
def test_arnoldi_barrier_timeout(gpu_lib, oracle, solver):
    A = matgen.convection_diffusion_2d(48, 48, 1.0, 0.9, 0.5)
    n = A.shape()[0]
    b = oracle.spmv(A, matgen.uniform_vector(n, seed=2))
    Ad = gpu.Device_matrix(A)
    J = gpu.jacobi(Ad)
    if solver == "gmres":
        run = lambda x: gpu.gmres(b, x, gpu.Gmres_config(1e-10, 30, 3000), gpu.spmv(Ad), left=J)
    else:
        run = lambda x: gpu.fgmres(b, x, gpu.Fgmres_config(1e-10, 30, 3000), gpu.spmv(Ad), J)
    gpu.debug_set_wait(1_000_000, True)
    try:
        with pytest.raises(_lib.SkError) as e:
            run(np.zeros(n))
        assert e.value.status == SK_TIMEOUT and "Arnoldi" in str(e.value)
    finally:
        gpu.debug_set_wait(0, False)
    x = np.zeros(n)
    s = run(x)
    assert s.converged
    assert np.linalg.norm(b - oracle.spmv(A, x)) <= 1e-8 * np.linalg.norm(b)


def test_debug_set_wait_limits(gpu_lib):
    with pytest.raises(_lib.SkError):
        gpu.debug_set_wait(11_000_000_000, False)
    gpu.debug_set_wait(0, False)


@pytest.mark.parametrize("solver", ["cg", "bicgstab", "cgs", "minres"])
def test_one_launch_solver_barrier_timeout(gpu_lib, oracle, solver):
    """The FP64 solves that run whole in one cooperative launch wait at
    bounded grid barriers: with an unmeetable target and a 1 ms limit the
    kernel gives up, the call reports SK_TIMEOUT, and the same handle then
    solves normally."""
    A = matgen.convection_diffusion_2d(48, 48, 1.0, 0.9, 0.5) if solver in ("bicgstab", "cgs") \
        else matgen.laplacian_2d_dirichlet(48)
    n = A.shape()[0]
    b = oracle.spmv(A, matgen.uniform_vector(n, seed=2))
    Ad = gpu.Device_matrix(A)
    J = gpu.jacobi(Ad)
    run = {"cg": lambda x: gpu.conjugate_gradient(b, x, gpu.CGConfig(1e-10, 3000, 3000), gpu.spmv(Ad), J),
           "bicgstab": lambda x: gpu.bicgstab(b, x, gpu.Bicgstab_config(1e-10, 3000), gpu.spmv(Ad), J),
           "cgs": lambda x: gpu.cgs(b, x, gpu.Cgs_config(1e-10, 3000), gpu.spmv(Ad), J),
           "minres": lambda x: gpu.minres(b, x, gpu.Minres_config(1e-10, 3000), gpu.spmv(Ad), J)}[solver]
    gpu.debug_set_wait(1_000_000, True)
    try:
        with pytest.raises(_lib.SkError) as e:
            run(np.zeros(n))
        assert e.value.status == SK_TIMEOUT and "barrier" in str(e.value)
    finally:
        gpu.debug_set_wait(0, False)
    x = np.zeros(n)
    s = run(x)
    assert s.converged
    assert np.linalg.norm(b - oracle.spmv(A, x)) <= 1e-8 * np.linalg.norm(b)
