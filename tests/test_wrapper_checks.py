"""The Python wrappers refuse device vectors that the C entry points would
misuse, before anything is launched.

The entry points that take device vectors (sk_precond_apply,
sk_chebyshev_apply_noalloc, sk_spmv, the device forms of the solvers) take
no length and trust the pointers they are given.  A host array, a CPU
tensor, a short vector, a strided view or the other precision would be read
or written out of bounds on the GPU.  These tests run without a GPU: the
wrappers are given a matrix object with no device handle, so a check that
failed to fire would reach the library with a null handle instead of
launching anything."""
import numpy as np
import pytest
import torch

from sparkit_b200 import gpu


def fake_matrix(n=8, dtype=np.float64):
    return gpu.Device_matrix._wrap(None, dtype, (n, n))


BAD = [
    (lambda n: np.zeros(n), TypeError, "CUDA torch tensor"),
    (lambda n: torch.zeros(n, dtype=torch.float32), TypeError, "dtype"),
    (lambda n: torch.zeros(2 * n, dtype=torch.float64)[::2], ValueError, "contiguous"),
    (lambda n: torch.zeros(n - 1, dtype=torch.float64), ValueError, "values"),
    (lambda n: torch.zeros(n, dtype=torch.float64), ValueError, "CUDA device"),
]


@pytest.mark.parametrize("make,exc,msg", BAD)
def test_noalloc_apply_refuses(make, exc, msg):
    Ad = fake_matrix()
    with pytest.raises(exc, match=msg):
        gpu.chebyshev_apply_noalloc(Ad, 0.5, 8.5, 4, make(8), torch.zeros(8, dtype=torch.float64))


@pytest.mark.parametrize("make,exc,msg", BAD)
def test_precond_apply_refuses(make, exc, msg):
    M = gpu._Precond(None, fake_matrix(), 8)
    with pytest.raises(exc, match=msg):
        M.apply(make(8), torch.zeros(8, dtype=torch.float64))


@pytest.mark.parametrize("make,exc,msg", BAD)
def test_spmv_and_device_solve_refuse(make, exc, msg):
    Ad = fake_matrix()
    with pytest.raises(exc, match=msg):
        Ad.spmv(make(8), torch.zeros(8, dtype=torch.float64))
    if not isinstance(make(8), np.ndarray):  # a numpy b selects the host form
        with pytest.raises(exc, match=msg):
            gpu.conjugate_gradient(make(8), torch.zeros(8, dtype=torch.float64), gpu.CGConfig(1e-10, 10, 10),
                                   gpu.spmv(Ad))


def test_fp32_matrix_refuses_fp64_vectors():
    M = gpu._Precond(None, fake_matrix(dtype=np.float32), 8)
    with pytest.raises(TypeError, match="float32"):
        M.apply(torch.zeros(8, dtype=torch.float64), torch.zeros(8, dtype=torch.float64))


def test_host_solve_refuses_wrong_length():
    Ad = fake_matrix()
    with pytest.raises(ValueError, match="8 values"):
        gpu.conjugate_gradient(np.ones(7), np.zeros(7), gpu.CGConfig(1e-10, 10, 10), gpu.spmv(Ad))
