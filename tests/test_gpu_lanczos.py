"""Implicitly restarted Lanczos and the eigenvalue estimates on the GPU
(sk_lanczos, sk_eigenvalue_bounds, sk_spectral_radius,
sk_chebyshev_create_auto) against the reference's own results (golden
fixtures) and the oracle, with the exact spectra of Laplacians as a
size-independent check."""
import numpy as np
import pytest

from sparkit_b200 import _lib, formats, gpu, matgen
from tests.golden.make_golden import LANCZOS_TARGETS, eigen_matrices

pytestmark = pytest.mark.gpu


def _scale(vals):
    return max(1.0, float(np.max(np.abs(vals))))


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_estimates_match_reference_fixtures(gpu_lib, golden, dtype):
    """The same start vectors (the reference's mt19937 sequence), the same
    restarts and host arithmetic; only the dot products are summed in a
    different order and the restart rotations are applied to the basis as
    one product.  FP64: eigenvalues within 1e-8 of the spectral scale,
    restart counts within one, Ritz vectors equal up to sign.  FP32: within
    2e-3 wherever the reference's FP32 value agrees with its FP64 value to
    that tolerance; where it does not (FP32 runs exhaust their restarts, and
    with the Krylov space exhausted the result depends on the summation
    order, test_oracle.py records it) the values lie in the FP64 spectrum."""
    dt = np.dtype(dtype)
    tol = 1e-8 if dtype == "float64" else 2e-3

    def check(got, want, want64, hull, s, what):
        if dtype == "float64" or np.all(np.abs(want - want64) <= tol * s):
            assert np.all(np.abs(got - want) <= tol * s), (what, got, want)
        else:
            assert np.all(got >= hull[0] - tol * s) and np.all(got <= hull[1] + tol * s), (what, got, hull)

    for name, A in eigen_matrices().items():
        Ad = gpu.Device_matrix(A.astype(dt))
        tag = f"eigen/{name}/{dtype}"
        ref_b = golden[f"{tag}/bounds"].astype(np.float64)
        hull = golden[f"eigen/{name}/float64/bounds"]
        s = _scale(hull)
        mag = max(abs(hull[0]), abs(hull[1]))
        lo, hi = gpu.estimate_eigenvalue_bounds(Ad)
        check(np.array([lo, hi]), ref_b, hull, hull, s, (name, "bounds"))
        rho = gpu.estimate_spectral_radius(Ad)
        check(np.array([rho]), np.array([float(golden[f"{tag}/radius"])]),
              np.array([float(golden[f"eigen/{name}/float64/radius"])]), (0.0, mag), s, (name, "radius"))
        for target in LANCZOS_TARGETS:
            r = gpu.lanczos(Ad, nev=3, m=12, tol=1e-8, max_restarts=5, target=target, collect=True, vectors=True)
            key = f"{tag}/lanczos/{target}"
            want = golden[f"{key}/eigenvalues"]
            want64 = golden[f"eigen/{name}/float64/lanczos/{target}/eigenvalues"]
            assert r["eigenvalues"].shape == want.shape, (name, target)
            # magnitude targets return signed Ritz values within -+ max |lambda|
            h = (-mag, mag) if target.endswith("magnitude") else hull
            check(r["eigenvalues"], want, want64, h, s, (name, target))
            restarts, conv_count, conv = golden[f"{key}/scalars"].tolist()
            if dtype == "float64":
                assert abs(r["computed_restarts"] - restarts) <= 1, (name, target)
                if r["computed_restarts"] == restarts:
                    assert r["converged"] == bool(conv), (name, target)
                    assert len(r["restart_residuals"]) == len(golden[f"{key}/restart_residuals"])
                X = r["eigenvectors"].cpu().numpy()
                Xr = golden[f"{key}/eigenvectors"]
                for k in range(len(want)):
                    # well separated Ritz values only: a vector is defined up to sign
                    gaps = np.abs(want - want[k])
                    gaps[k] = np.inf
                    if np.min(gaps) > 1e-4 * _scale(want) and golden[f"{key}/residual_norms"][k] < 1e-6:
                        assert abs(abs(float(X[k] @ Xr[k])) - 1.0) < 1e-6, (name, target, k)


def test_bounds_match_oracle_48cubed(gpu_lib, oracle):
    """The 48^3 Dirichlet Laplacian (110,592 rows): the device bounds equal
    the oracle's (which equals the reference bit for bit) to 1e-9
    relative, and lie inside the exact spectrum 6 -+ 6 cos(pi / 49)."""
    A = matgen.laplacian_3d_dirichlet(48)
    lo_r, hi_r = oracle.eigenvalue_bounds(A)
    lo, hi = gpu.estimate_eigenvalue_bounds(gpu.Device_matrix(A))
    assert abs(lo - lo_r) <= 1e-9 * 12 and abs(hi - hi_r) <= 1e-9 * 12, ((lo, hi), (lo_r, hi_r))
    c = 6 * np.cos(np.pi / 49)
    assert 6 - c - 1e-12 <= lo and hi <= 6 + c + 1e-12


def test_bounds_of_the_128cubed_laplacian(gpu_lib):
    """The format sweep's matrix A (2.1M rows): Ritz values lie inside the
    spectrum [6 - 6 cos(pi/129), 6 + 6 cos(pi/129)], the largest within
    1e-3 of the top (well separated from the start), and the ELL, JAD and
    BSR handles give the same bounds as CSR (their products sum rows in the
    same order)."""
    A = matgen.laplacian_3d_dirichlet(128)
    Ad = gpu.Device_matrix(A)
    lo, hi = gpu.estimate_eigenvalue_bounds(Ad)
    c = 6 * np.cos(np.pi / 129)
    assert 6 - c - 1e-12 <= lo < hi <= 6 + c + 1e-12
    assert (6 + c) - hi < 1e-3, hi
    rho = gpu.estimate_spectral_radius(Ad)
    assert abs(rho - hi) < 1e-2 and rho <= 6 + c + 1e-12
    for M in (gpu.to_ellpack(Ad), gpu.to_jagged_diagonal(Ad)):
        lo2, hi2 = gpu.estimate_eigenvalue_bounds(M)
        assert abs(lo2 - lo) <= 1e-10 and abs(hi2 - hi) <= 1e-10


def test_chebyshev_auto_in_cg(gpu_lib, oracle):
    """chebyshev_preconditioner with automatic bounds: the same bounds as
    sk_eigenvalue_bounds, the same coefficients as the explicit form, and
    a CG solve it preconditions converges with the true residual below the
    tolerance, in fewer iterations than Jacobi.  The matrix is the shifted
    96 x 96 Poisson problem (spectrum about [1, 9]): a degree-8 Chebyshev
    approximation of 1/x over a Dirichlet Laplacian's whole spectrum
    (condition ~7600) is not positive definite, whatever the bounds."""
    A = matgen.poisson_2d(96, 96, 1.0)
    n = A.shape()[0]
    Ad = gpu.Device_matrix(A)
    lo, hi = gpu.estimate_eigenvalue_bounds(Ad)
    M = gpu.chebyshev_preconditioner_auto(Ad, 8)
    assert (M.lambda_min, M.lambda_max) == (lo, hi)
    E = gpu.chebyshev_preconditioner(Ad, lo, hi, 8)
    assert np.array_equal(M.values(), E.values())
    b = oracle.spmv(A, matgen.uniform_vector(n, seed=5))
    x = np.zeros(n)
    s = gpu.conjugate_gradient(b, x, gpu.CGConfig(1e-10, 1000, 2000), gpu.spmv(Ad), M, gpu.identity)
    assert s.converged
    assert np.linalg.norm(b - oracle.spmv(A, x)) <= 1e-9 * np.linalg.norm(b)
    J = gpu.conjugate_gradient(b, np.zeros(n), gpu.CGConfig(1e-10, 1000, 2000), gpu.spmv(Ad), gpu.jacobi(Ad),
                               gpu.identity)
    assert s.computed_iterations < J.computed_iterations


def test_lanczos_arguments(gpu_lib):
    A = matgen.laplacian_2d_dirichlet(8)
    Ad = gpu.Device_matrix(A)
    with pytest.raises(_lib.SkError):
        gpu.lanczos(Ad, nev=1, m=0)
    with pytest.raises(_lib.SkError):
        gpu.lanczos(Ad, nev=0, m=5)
    R = formats.Compressed_row_matrix((3, 4), np.array([0, 1, 2, 3]), np.array([0, 1, 2]), np.ones(3))
    with pytest.raises(_lib.SkError):
        gpu.estimate_eigenvalue_bounds(gpu.Device_matrix(R))
    # nev >= m: the wanted values are all Ritz values, returned at once
    r = gpu.lanczos(Ad, nev=6, m=6, target="smallest_algebraic")
    assert r["converged"] and r["computed_restarts"] == 1 and r["eigenvalues"].size == 6
    # no restarts: no convergence test, the values of the first factorisation
    r = gpu.lanczos(Ad, nev=1, m=10, max_restarts=0)
    assert not r["converged"] and r["computed_restarts"] == 0 and r["residual_norms"].size == 0
