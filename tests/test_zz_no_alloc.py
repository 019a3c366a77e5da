"""The no-allocation Chebyshev apply (sk_chebyshev_apply_noalloc), called
through the C ABI, against the regular handle-based apply.

It serves callers that cannot allocate device memory when they apply the
preconditioner (a callback inside another solver library's loop, where that
library reserved all device memory up front), so its work vectors live in a
static device array shared by all calls.  Two calls in a row must each give exactly the regular apply's
result, so the second call cannot be affected by what the first one left in
the shared array.  This file is collected last, and passes alone in a fresh
process as well as after the other tests."""
import numpy as np
import pytest

from sparkit_b200 import _lib, formats, gpu, matgen

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_noalloc_chebyshev_matches_regular_apply(gpu_lib, dtype):
    import torch
    A = matgen.poisson_2d(64, 64, 0.5, dtype=dtype)  # n = 4096
    n = A.shape()[0]
    Ad = gpu.Device_matrix(A)
    lmin, lmax, degree = 0.5, 8.5, 8
    M = gpu.chebyshev_preconditioner(Ad, lmin, lmax, degree)
    for seed in (1, 2):  # two calls in a row, different right-hand sides
        r = torch.from_numpy(matgen.uniform_vector(n, seed=seed, dtype=dtype)).cuda()
        z_ref = torch.empty_like(r)
        M.apply(r, z_ref)
        z = torch.full_like(r, float("nan"))
        gpu.chebyshev_apply_noalloc(Ad, lmin, lmax, degree, r, z)
        torch.cuda.synchronize()
        assert torch.equal(z, z_ref), seed


def test_noalloc_chebyshev_degree_zero_and_limits(gpu_lib):
    import torch
    A = matgen.tridiagonal_matrix(100, -1.0, 4.0, -1.0)
    Ad = gpu.Device_matrix(A)
    r = torch.from_numpy(matgen.uniform_vector(100, seed=3)).cuda()
    z_ref = torch.empty_like(r)
    gpu.chebyshev_preconditioner(Ad, 2.0, 6.0, 0).apply(r, z_ref)
    z = torch.empty_like(r)
    gpu.chebyshev_apply_noalloc(Ad, 2.0, 6.0, 0, r, z)
    torch.cuda.synchronize()
    assert torch.equal(z, z_ref)
    with pytest.raises(_lib.SkError) as e:
        gpu.chebyshev_apply_noalloc(Ad, 2.0, 6.0, 65, r, z)
    assert e.value.status == 1
    # one row more than the static array holds is refused, not run
    n = (1 << 20) + 1
    big = formats.Compressed_row_matrix((n, n), np.arange(n + 1, dtype=np.int64), np.arange(n, dtype=np.int64),
                                        np.ones(n))
    Bd = gpu.Device_matrix(big)
    rb = torch.ones(n, dtype=torch.float64, device="cuda")
    zb = torch.empty_like(rb)
    with pytest.raises(_lib.SkError) as e:
        gpu.chebyshev_apply_noalloc(Bd, 0.5, 2.0, 4, rb, zb)
    assert e.value.status == 1 and "1048576" in str(e.value)
