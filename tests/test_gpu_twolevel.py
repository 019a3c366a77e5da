"""The two-level grid preconditioner (smoother plus an aggregation coarse-grid
correction) on the GPU, through the C ABI: its apply against a NumPy FP64
restatement, its effect inside FGMRES(30), and argument checks."""
import numpy as np
import pytest

from sparkit_b200 import _lib, gpu, matgen

pytestmark = pytest.mark.gpu


def _dense_parts(A, nx, ny, agg):
    import scipy.sparse as sp
    n = nx * ny
    M = sp.csr_matrix((np.asarray(A.values()), np.asarray(A.col_ind()), np.asarray(A.row_ptr())), shape=(n, n))
    i = np.arange(n)
    cid = ((i // nx) // agg) * (nx // agg) + (i % nx) // agg
    P = sp.csr_matrix((np.ones(n), (i, cid)), shape=(n, (nx // agg) * (ny // agg)))
    Ac = (P.T @ M @ P).toarray()
    return M, P, np.linalg.inv(Ac)


@pytest.mark.parametrize("post", [False, True])
def test_twolevel_apply_matches_numpy(gpu_lib, post):
    """Jacobi smoother: z = D^-1 r; z += P Ac^-1 P^T (r - A z)
    [; z += D^-1 (r - A z)], against the same steps in NumPy (the coarse
    inverse from LAPACK in FP64 there; a banded LU here, its inverse stored
    in FP32 and applied with FP64 products: within 1e-6)."""
    import torch
    from tests.test_gpu_learned import rect_convdiff
    nx, ny, agg = 64, 48, 8
    A = rect_convdiff(nx, ny, 4)  # a rectangular grid
    M, P, Aci = _dense_parts(A, nx, ny, agg)
    Ad = gpu.Device_matrix(A)
    J = gpu.jacobi(Ad)
    T = gpu.twolevel(Ad, J, nx, ny, agg, post_smooth=post)
    r = np.random.default_rng(2).standard_normal(nx * ny)
    rd = torch.from_numpy(r).cuda()
    zd = torch.zeros_like(rd)
    T.apply(rd, zd)
    torch.cuda.synchronize()
    d = M.diagonal()
    z = r / d
    z = z + P @ (Aci @ (P.T @ (r - M @ z)))
    if post:
        z = z + (r - M @ z) / d
    got = zd.cpu().numpy()
    # the coarse inverse is stored in FP32 (products and sums in FP64)
    assert np.linalg.norm(got - z) / np.linalg.norm(z) < 1e-6
    # repeatable bit for bit (fixed-order reductions)
    z2 = torch.zeros_like(rd)
    T.apply(rd, z2)
    torch.cuda.synchronize()
    assert np.array_equal(z2.cpu().numpy(), got)


def test_twolevel_fgmres_converges_where_jacobi_stalls(gpu_lib, oracle):
    """FGMRES(30) on 128 x 128 upwind convection-diffusion (cell Peclet 30):
    Jacobi alone does not reach 1e-8 in 3000 iterations; with the coarse
    correction it does, with the true residual below the tolerance."""
    import torch
    n = 128
    A = matgen.convdiff_2d_grf(n, seed=777, peclet=30.0)[0]
    Ad = gpu.Device_matrix(A)
    b = np.random.default_rng(3).uniform(-1, 1, n * n)
    bd = torch.from_numpy(b).cuda()
    cfg = gpu.Fgmres_config(1e-8, 30, 3000)
    J = gpu.jacobi(Ad)
    res = {}
    for name, M in (("jacobi", J), ("twolevel", gpu.twolevel(Ad, J, n, n, 8))):
        xd = torch.zeros_like(bd)
        s = gpu.fgmres(bd, xd, cfg, gpu.spmv(Ad), M)
        torch.cuda.synchronize()
        rel = np.linalg.norm(b - oracle.spmv(A, xd.cpu().numpy())) / np.linalg.norm(b)
        res[name] = (s.converged, s.computed_iterations, rel)
    conv, its, rel = res["twolevel"]
    assert conv and rel < 1.5e-8, res
    assert (not res["jacobi"][0]) or res["jacobi"][1] >= 3 * its, res


def test_twolevel_rejects_bad_arguments(gpu_lib):
    import torch  # noqa: F401
    A = matgen.laplacian_2d_dirichlet(32)
    Ad = gpu.Device_matrix(A)
    J = gpu.jacobi(Ad)
    with pytest.raises(_lib.SkError):
        gpu.twolevel(Ad, J, 32, 32, 5)  # 5 does not divide 32
    with pytest.raises(_lib.SkError):
        gpu.twolevel(Ad, J, 32, 16, 4)  # 32 x 16 is not the matrix size
    with pytest.raises(_lib.SkError):
        gpu.twolevel(Ad, J, 32, 32, 0)
