"""The mixed-precision solver (FP32 inner CG, FP64 refinement) reaches the
FP64 tolerance on the true residual and needs a comparable number of FP32
iterations to the plain FP64 solver's."""
import numpy as np
import pytest

from sparkit_b200 import gpu, matgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("jacobi", [True, False])
def test_mixed_reaches_fp64_tolerance(gpu_lib, oracle, jacobi):
    import torch
    A = matgen.diffusion_3d_grf(24, sigma=1.0, corr_len=4.0, seed=1)
    n = A.shape()[0]
    b = matgen.uniform_vector(n, seed=3)
    Ad = gpu.Device_matrix(A)
    bd = torch.from_numpy(b).cuda()
    xd = torch.zeros_like(bd)
    s = gpu.mixed_cg(bd, xd, gpu.Mixed_config(1e-10, 1e-5, 50, 100000, True), gpu.spmv(Ad), jacobi_inner=jacobi)
    torch.cuda.synchronize()
    x = xd.cpu().numpy()
    rel = np.linalg.norm(b - oracle.spmv(A, x)) / np.linalg.norm(b)
    assert s.converged and rel < 1e-10, (s, rel)
    assert abs(s.residual_norm / np.linalg.norm(b) - rel) < 1e-12
    assert 2 <= s.outer_iterations <= 6
    # the residual history is the true FP64 residual of each outer step
    assert len(s.residual_history) == s.outer_iterations + 1
    assert all(a > b for a, b in zip(s.residual_history, s.residual_history[1:]))
    # comparable work to the FP64 solver
    _, sr = oracle.cg(A, b, np.zeros(n), 1e-10, 10 ** 6, 100000, left="jacobi" if jacobi else None)
    assert s.inner_iterations <= 2 * sr["computed_iterations"]


def test_mixed_zero_rhs(gpu_lib):
    import torch
    A = matgen.laplacian_3d_dirichlet(8)
    Ad = gpu.Device_matrix(A)
    bd = torch.zeros(A.shape()[0], dtype=torch.float64, device="cuda")
    xd = torch.ones_like(bd)
    s = gpu.mixed_cg(bd, xd, gpu.Mixed_config(), gpu.spmv(Ad))
    torch.cuda.synchronize()
    assert s.converged and not xd.any()
