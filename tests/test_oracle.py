"""Pins the CPU oracle (oracle/sk_oracle.c) before it is trusted:
against the known-answer vectors of the reference's Catch2 tests and, bit
for bit, against outputs of the reference itself (tests/golden/, made by
tests/golden/make_golden.py; plus live runs when the compiled reference is
present)."""
import numpy as np
import pytest

from sparkit_b200 import formats, matgen
from tests.helpers import BSR_BLOCKS, SPMV_CASES, convert, csr_from_entries, golden_csr, golden_problem


def test_spmv_known_answers(oracle, known):
    for case in known["spmv"]:
        A = csr_from_entries(tuple(case["shape"]), case["entries"])
        M = convert(A, case["format"], tuple(case.get("block", (3, 3))))
        y = oracle.spmv(M, np.array(case["x"]))
        assert y.tolist() == case["y"], case["name"]


def test_jacobi_known_answers(oracle, known):
    for case in known["jacobi"]:
        A = csr_from_entries(tuple(case["shape"]), case["entries"])
        if case.get("throws"):
            with pytest.raises(ValueError):
                oracle.jacobi(A)
            continue
        inv = oracle.jacobi(A)
        if "inv_d" in case:
            np.testing.assert_allclose(inv, case["inv_d"], rtol=1e-15)
        if "z" in case:
            assert (inv * np.array(case["r"])).tolist() == case["z"]


def test_layout_known_answers(known):
    for case in known["layouts"]:
        A = csr_from_entries(tuple(case["shape"]), case["entries"])
        if "perm" in case:
            J = formats.to_jagged_diagonal(A)
            assert J.perm().tolist() == case["perm"]
            assert J.jdiag().tolist() == case["jdiag"]
        if "width" in case:
            E = formats.to_ellpack(A)
            assert E.max_nnz_per_row() == case["width"]
            assert E.col_ind().tolist() == case["col_ind"]


@pytest.mark.parametrize("name", SPMV_CASES)
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_spmv_matches_reference_bitwise(oracle, golden, name, dtype):
    tag = f"spmv/{name}/{dtype}"
    A = golden_csr(golden, tag)
    x = golden[f"{tag}/x"]
    for fmt in ("csr", "ell", "jad"):
        y = oracle.spmv(convert(A, fmt), x)
        assert np.array_equal(y, golden[f"{tag}/y_{fmt}"]), fmt
    for key, blk in BSR_BLOCKS.items():
        y = oracle.spmv(formats.to_block_sparse_row(A, *blk), x)
        assert np.array_equal(y, golden[f"{tag}/y_bsr{blk[0]}{blk[1]}"]), key


def test_preconditioners_match_reference_bitwise(oracle, golden):
    P = matgen.poisson_2d(8, 8, 0.5)
    assert np.array_equal(oracle.jacobi(P), golden["jacobi/poisson8/inv_d"])
    for lmin, lmax, deg in ((0.5, 8.5, 8), (3.0, 13.0, 4), (1.0, 1.0, 5), (2.0, 6.0, 0)):
        key = f"cheb/{lmin}_{lmax}_{deg}"
        assert np.array_equal(oracle.chebyshev_coeffs(lmin, lmax, deg), golden[f"{key}/coeffs_f64"])
        assert np.array_equal(oracle.chebyshev_coeffs(lmin, lmax, deg, np.float32), golden[f"{key}/coeffs_f32"])
        z = oracle.chebyshev_apply(P, lmin, lmax, deg, golden[f"{key}/r"])
        assert np.array_equal(z, golden[f"{key}/z"]), key


PROBLEMS = ["grid16", "tridiag4", "convdiff", "nonsym", "lap2d_24", "upwind_20"]
SPD = {"grid16", "tridiag4", "lap2d_24"}
PRECS = {"none": None, "jacobi": "jacobi", "cheb": ("chebyshev", 0.5, 9.0, 6)}


@pytest.mark.parametrize("name", PROBLEMS)
@pytest.mark.parametrize("pname", list(PRECS))
def test_solvers_match_reference_bitwise(oracle, golden, name, pname):
    A = golden_problem(golden, name)
    n = A.shape()[0]
    b = golden[f"solve/{name}/b"]
    spec = PRECS[pname]
    runs = {"bicgstab": lambda: oracle.bicgstab(A, b, np.zeros(n), 1e-12, 500, left=spec, collect=True),
            "fgmres": lambda: oracle.fgmres(A, b, np.zeros(n), 1e-12, 5, 500, prec=spec, collect=True),
            "gmres_left": lambda: oracle.gmres(A, b, np.zeros(n), 1e-12, 5, 500, left=spec, collect=True),
            "gmres_right": lambda: oracle.gmres(A, b, np.zeros(n), 1e-12, 6, 500, right=spec, collect=True),
            "cgs": lambda: oracle.cgs(A, b, np.zeros(n), 1e-12, 500, left=spec, collect=True)}
    if name in SPD:
        runs["minres"] = lambda: oracle.minres(A, b, np.zeros(n), 1e-12, 500, left=spec, collect=True)
        runs["cg_left"] = lambda: oracle.cg(A, b, np.zeros(n), 1e-12, 50, 500, left=spec, collect=True)
        runs["cg_right"] = lambda: oracle.cg(A, b, np.zeros(n), 1e-12, 7, 500, right=spec, collect=True)
    for rname, fn in runs.items():
        key = f"solve/{name}/{pname}/{rname}"
        x, s = fn()
        # a run that diverges (CGS with the Chebyshev bounds on some of these
        # problems) ends in NaN in the reference too: NaN matches NaN here
        assert np.array_equal(x, golden[f"{key}/x"], equal_nan=True), key
        assert s["computed_iterations"] == int(golden[f"{key}/iters"]), key
        assert int(s["converged"]) == int(golden[f"{key}/converged"]), key
        assert np.array_equal(s["residual_norm"], float(golden[f"{key}/residual_norm"]), equal_nan=True), key
        assert np.array_equal(np.array(s["iteration_residuals"]), golden[f"{key}/history"], equal_nan=True), key


def test_cg_edge_cases_match_reference(oracle, reference):
    A = matgen.poisson_2d(4, 4, 5.0)
    n = 16
    b = oracle.spmv(A, np.arange(1, n + 1, dtype=np.float64))
    # zero right-hand side: x = 0, converged, no iterations
    x, s = oracle.cg(A, np.zeros(n), np.ones(n), 1e-12, 50, 100)
    xr, sr = reference.cg(A, np.zeros(n), np.ones(n), 1e-12, 50, 100)
    assert np.array_equal(x, xr) and not x.any() and s["converged"] and s["computed_iterations"] == 0
    assert s == sr
    # max_iterations = 1: not converged after exactly one iteration
    x, s = oracle.cg(A, b, np.zeros(n), 1e-14, 50, 1)
    xr, sr = reference.cg(A, b, np.zeros(n), 1e-14, 50, 1)
    assert s["computed_iterations"] == 1 and not s["converged"] and s == sr and np.array_equal(x, xr)


def test_float_solvers_match_reference(oracle, reference):
    A = matgen.laplacian_2d_dirichlet(20, dtype=np.float32)
    n = A.shape()[0]
    b = matgen.uniform_vector(n, seed=4, dtype=np.float32)
    for spec in (None, "jacobi"):
        x, s = oracle.cg(A, b, np.zeros(n, np.float32), 1e-5, 1000, 1000, left=spec, collect=True)
        xr, sr = reference.cg(A, b, np.zeros(n, np.float32), 1e-5, 1000, 1000, left=spec, collect=True)
        assert np.array_equal(x, xr) and s == sr
        x, s = oracle.bicgstab(A, b, np.zeros(n, np.float32), 1e-5, 1000, left=spec, collect=True)
        xr, sr = reference.bicgstab(A, b, np.zeros(n, np.float32), 1e-5, 1000, left=spec, collect=True)
        assert np.array_equal(x, xr) and s == sr
        x, s = oracle.fgmres(A, b, np.zeros(n, np.float32), 1e-5, 10, 1000, prec=spec, collect=True)
        xr, sr = reference.fgmres(A, b, np.zeros(n, np.float32), 1e-5, 10, 1000, prec=spec, collect=True)
        assert np.array_equal(x, xr) and s == sr
        x, s = oracle.gmres(A, b, np.zeros(n, np.float32), 1e-5, 10, 1000, left=spec, right=spec, collect=True)
        xr, sr = reference.gmres(A, b, np.zeros(n, np.float32), 1e-5, 10, 1000, left=spec, right=spec,
                                 collect=True)
        assert np.array_equal(x, xr) and s == sr


def test_gmres_edge_cases_match_reference(oracle, reference):
    """gmres.hpp:164-176 and :186-187: zero right-hand side, a budget that
    ends inside a restart cycle, and both preconditioners at once."""
    A = matgen.convdiff_2d_grf(12, seed=3)[0]
    n = A.shape()[0]
    b = matgen.uniform_vector(n, seed=2)
    x, s = oracle.gmres(A, np.zeros(n), np.ones(n), 1e-10, 5, 50, left="jacobi")
    xr, sr = reference.gmres(A, np.zeros(n), np.ones(n), 1e-10, 5, 50, left="jacobi")
    assert not x.any() and s["converged"] and s["computed_iterations"] == 0 and s == sr
    for spec in ("jacobi", ("chebyshev", 0.2, 9.0, 4)):
        x, s = oracle.gmres(A, b, np.zeros(n), 1e-14, 7, 23, left=spec, right=spec, collect=True)
        xr, sr = reference.gmres(A, b, np.zeros(n), 1e-14, 7, 23, left=spec, right=spec, collect=True)
        assert s["computed_iterations"] == 23 and not s["converged"]
        assert np.array_equal(x, xr) and s == sr


def test_cgs_minres_match_reference(oracle, reference):
    """cgs.hpp and minres.hpp beyond the fixtures: right and two-sided
    preconditioning, FP32, a zero right-hand side, and budgets that end the
    solve (CGS spends two products per step, so an odd budget ends after
    the step that reaches it)."""
    A = matgen.laplacian_2d_dirichlet(14)
    n = A.shape()[0]
    b = matgen.uniform_vector(n, seed=7)
    C = matgen.convdiff_2d_grf(12, seed=4)[0]
    bc = matgen.uniform_vector(C.shape()[0], seed=8)
    cheb = ("chebyshev", 0.3, 8.5, 5)
    for spec_l, spec_r in ((None, "jacobi"), ("jacobi", "jacobi"), (cheb, None), (None, cheb)):
        for fn in ("cgs", "minres"):
            M, rhs = (A, b) if fn == "minres" else (C, bc)
            m = M.shape()[0]
            x, s = getattr(oracle, fn)(M, rhs, np.zeros(m), 1e-11, 400, left=spec_l, right=spec_r, collect=True)
            xr, sr = getattr(reference, fn)(M, rhs, np.zeros(m), 1e-11, 400, left=spec_l, right=spec_r,
                                            collect=True)
            assert np.array_equal(x, xr) and s == sr, (fn, spec_l, spec_r)
    A32 = matgen.laplacian_2d_dirichlet(12, dtype=np.float32)
    b32 = matgen.uniform_vector(A32.shape()[0], seed=9, dtype=np.float32)
    for fn in ("cgs", "minres"):
        x, s = getattr(oracle, fn)(A32, b32, np.zeros(144, np.float32), 1e-5, 300, left="jacobi", collect=True)
        xr, sr = getattr(reference, fn)(A32, b32, np.zeros(144, np.float32), 1e-5, 300, left="jacobi", collect=True)
        assert np.array_equal(x, xr) and s == sr, fn
        x, s = getattr(oracle, fn)(A32, np.zeros(144, np.float32), np.ones(144, np.float32), 1e-5, 300)
        assert s["converged"] and s["computed_iterations"] == 0 and not x.any()
        x, s = getattr(oracle, fn)(A, b, np.zeros(n), 1e-15, 7, collect=True)
        xr, sr = getattr(reference, fn)(A, b, np.zeros(n), 1e-15, 7, collect=True)
        assert np.array_equal(x, xr) and s == sr and not s["converged"], fn
        assert s["computed_iterations"] == (8 if fn == "cgs" else 7)


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_eigen_estimates_match_reference_fixtures(oracle, golden, dtype):
    """lanczos / estimate_eigenvalue_bounds / estimate_spectral_radius
    (lanczos.hpp:495, conditioning.hpp:112, :132): the oracle reproduces the
    reference's eigenvalues, residual norms, restart residuals, Ritz vectors
    and counts bit for bit, for every target, FP64 and FP32 (the start
    vectors come from the reference's own mt19937 sequence)."""
    from tests.golden.make_golden import LANCZOS_TARGETS, eigen_matrices
    dt = np.dtype(dtype)
    for name, A in eigen_matrices().items():
        Ad = A.astype(dt)
        tag = f"eigen/{name}/{dtype}"
        assert np.array_equal(np.array(oracle.eigenvalue_bounds(Ad), dtype=dt), golden[f"{tag}/bounds"]), name
        assert np.array_equal(np.array(oracle.spectral_radius(Ad), dtype=dt), golden[f"{tag}/radius"]), name
        for target in LANCZOS_TARGETS:
            r = oracle.lanczos(Ad, nev=3, m=12, tol=1e-8, max_restarts=5, target=target, collect=True,
                               vectors=True)
            key = f"{tag}/lanczos/{target}"
            for k in ("eigenvalues", "residual_norms", "restart_residuals", "eigenvectors"):
                assert np.array_equal(r[k], golden[f"{key}/{k}"]), (name, target, k)
            assert [r["computed_restarts"], r["converged_count"], int(r["converged"])] == \
                golden[f"{key}/scalars"].tolist(), (name, target)


def test_eigen_estimates_match_reference(oracle, reference):
    """Beyond the fixtures, against the compiled reference: other Krylov
    dimensions and restart budgets (0 restarts: no convergence check), the
    remaining targets, and the bounds of the 3D Laplacian against the
    exact extreme eigenvalues 6 -+ 6 cos(pi / 9)."""
    A = matgen.laplacian_3d_dirichlet(8)
    for kw in (dict(nev=1, m=31, tol=1e-10, max_restarts=10, target="largest_real"),
               dict(nev=2, m=8, tol=1e-12, max_restarts=0, target="smallest_real"),
               dict(nev=4, m=20, tol=1e-6, max_restarts=3, target="smallest_magnitude")):
        r = oracle.lanczos(A, collect=True, vectors=True, **kw)
        rr = reference.lanczos(A, collect=True, vectors=True, **kw)
        for k in ("eigenvalues", "residual_norms", "restart_residuals", "eigenvectors"):
            assert np.array_equal(r[k], rr[k]), (kw, k)
        assert (r["computed_restarts"], r["converged_count"], r["converged"]) == \
            (rr["computed_restarts"], rr["converged_count"], rr["converged"])
    lo, hi = oracle.eigenvalue_bounds(A)
    assert (lo, hi) == reference.eigenvalue_bounds(A)
    exact = 6 * np.cos(np.pi / 9)
    assert abs(hi - (6 + exact)) < 1e-8 and abs(lo - (6 - exact)) < 1e-6


def test_fp32_lanczos_depends_on_summation_order(oracle):
    """The reference's Lanczos convergence test is fixed at 1e-10 |theta|
    (conditioning.hpp:141), below FP32 resolution, so every FP32 estimate
    runs all its restarts.  On the 16-point grid (n = 16, Krylov dimension
    min(n, 31) = n) the space is exhausted and each restart feeds on
    rounding noise: reversing the dot products' summation order moves the
    FP32 bounds by more than 0.1, while the FP64 ones stay put.  The GPU's
    FP32 parity is therefore stated where the reference's FP32 value is
    stable (test_gpu_lanczos.py)."""
    A = matgen.poisson_2d(4, 4, 5.0)
    try:
        out = {}
        for mode in (0, 2):
            oracle.set_dot_order(mode)
            out[mode] = (oracle.eigenvalue_bounds(A), oracle.eigenvalue_bounds(A.astype(np.float32)))
    finally:
        oracle.set_dot_order(0)
    (d0, f0), (d2, f2) = out[0], out[2]
    assert max(abs(d0[0] - d2[0]), abs(d0[1] - d2[1])) < 1e-12
    assert max(abs(f0[0] - f2[0]), abs(f0[1] - f2[1])) > 0.1


def _dense(shape, entries):
    D = np.zeros(shape)
    for r, c, v in entries:
        D[int(r), int(c)] = v
    return D


def _csr_dense(A):
    D = np.zeros(A.shape())
    rp, ci, va = A.row_ptr(), A.col_ind(), A.values()
    for r in range(A.shape()[0]):
        D[r, ci[rp[r]:rp[r + 1]]] = va[rp[r]:rp[r + 1]]
    return D


def test_matrix_market_known_answers(oracle, known):
    """The reference's own Catch2 cases for read_matrix_market,
    parse_banner and write_matrix_market (matrix_market_test.cpp)."""
    from oracle.binding import MatrixMarketError
    from tests.helpers import csr_from_entries
    mm = known["matrix_market"]
    for case in mm["read"]:
        A = oracle.mm_read(case["text"].encode())
        assert A.shape() == tuple(case["shape"]), case["source"]
        assert np.array_equal(_csr_dense(A), _dense(case["shape"], case["entries"])), case["source"]
    for case in mm["rejected"]:
        with pytest.raises(MatrixMarketError):
            oracle.mm_read(case["text"].encode())
    for case in mm["write"]:
        A = csr_from_entries(tuple(case["shape"]), case["entries"])
        assert oracle.mm_write(A) == case["text"].encode(), case["source"]


def _same_bits(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_matrix_market_matches_reference_fixtures(oracle, golden, dtype):
    """read_matrix_market + to_compressed_row on seeded texts (duplicates,
    symmetric, skew, pattern, signed integers, CRLF, out-of-range reals)
    and write_matrix_market of the result, against the compiled
    reference's outputs, bit for bit (the sign of zero included)."""
    from tests.golden.make_golden import mm_texts
    for name in mm_texts():
        tag = f"mm/{name}/{dtype}"
        A = oracle.mm_read(bytes(golden[f"mm/{name}/text"]), np.dtype(dtype))
        assert A.shape() == tuple(golden[f"{tag}/shape"]), name
        for f in ("row_ptr", "col_ind", "values"):
            assert _same_bits(getattr(A, f)(), golden[f"{tag}/{f}"]), (name, f)
        assert oracle.mm_write(A) == bytes(golden[f"{tag}/written"]), name


def test_matrix_market_matches_reference_live(oracle, reference):
    """Beyond the fixtures, against the compiled reference itself: seeded
    random files of every symmetry and field, FP64 and FP32."""
    rng = np.random.default_rng(5)
    for trial in range(12):
        n, m = int(rng.integers(2, 40)), int(rng.integers(2, 40))
        sym = ["general", "symmetric", "skew-symmetric", "hermitian"][trial % 4]
        field = ["real", "integer", "pattern"][trial % 3]
        if sym != "general":
            m = n
        k = int(rng.integers(0, 3 * n))
        r, c = rng.integers(1, n + 1, k), rng.integers(1, m + 1, k)
        if sym != "general":
            r, c = np.maximum(r, c), np.minimum(r, c)
        vals = rng.standard_normal(k) * 10.0 ** rng.integers(-5, 5, k)
        lines = [f"%%MatrixMarket matrix coordinate {field} {sym}", f"{n} {m} {k}"]
        for a, b, v in zip(r, c, vals):
            lines.append(f"{a} {b}" if field == "pattern" else
                         f"{a} {b} {int(v * 100)}" if field == "integer" else f"{a} {b} {v:.17g}")
        text = ("\n".join(lines) + "\n").encode()
        for dt in (np.float64, np.float32):
            A, B = oracle.mm_read(text, dt), reference.mm_read(text, dt)
            for f in ("row_ptr", "col_ind", "values"):
                assert _same_bits(getattr(A, f)(), getattr(B, f)()), (trial, sym, field, f)
            assert oracle.mm_write(A) == reference.mm_write(B)


def test_generators_match_reference(reference):
    pairs = [(matgen.poisson_2d(4, 4, 5.0), reference.poisson_2d(4, 4, 5.0)),
             (matgen.poisson_2d(5, 3), reference.poisson_2d(5, 3)),
             (matgen.convdiff_centered_2d(4, 4, 1.0, 0.3, 0.3, 5.0),
              reference.convdiff_centered_2d(4, 4, 1.0, 0.3, 0.3, 5.0)),
             (matgen.convection_diffusion_2d(6, 5, 1.0, 0.7, 0.2),
              reference.convection_diffusion_2d(6, 5, 1.0, 0.7, 0.2)),
             (matgen.tridiagonal_matrix(6, -1.0, 4.0, -1.0), reference.tridiagonal(6, -1.0, 4.0, -1.0)),
             (matgen.nonsymmetric_sample(), reference.nonsymmetric_sample())]
    for a, b in pairs:
        for f in ("row_ptr", "col_ind", "values"):
            assert np.array_equal(getattr(a, f)(), getattr(b, f)())


def test_krylov_iteration_counts_depend_on_summation_order(oracle):
    """Evidence for the BiCGSTAB / CGS parity band of the GPU tests in the
    default tree order: the reference algorithm itself (bit-exact with the
    compiled reference in the sequential order 0), with its dot products
    summed in 256-entry chunks (order 1), from the last element down (order
    2) or accurately, in double-double rounded once (order 3), needs a
    different number of matrix-vector products on the upwind
    convection-diffusion problems: BiCGSTAB and CGS move by up to about 9%,
    even under the accurate sum, while FGMRES(30) stays within 1%.  Only the
    reference's own sequential order reproduces its counts
    (test_gpu_sequential.py runs the GPU solvers in that order)."""
    shift = {"bicgstab": 0.0, "cgs": 0.0, "fgmres": 0.0}
    try:
        for g in (48, 96):
            A = matgen.convection_diffusion_2d(g, g, 1.0, 0.9, 0.5)
            n = A.shape()[0]
            b = oracle.spmv(A, matgen.uniform_vector(n, seed=2))
            for prec in (None, "jacobi"):
                base = None
                for mode in (0, 1, 2, 3):
                    oracle.set_dot_order(mode)
                    _, s = oracle.bicgstab(A, b, np.zeros(n), 1e-10, 20000, left=prec)
                    _, c = oracle.cgs(A, b, np.zeros(n), 1e-10, 20000, left=prec)
                    _, f = oracle.fgmres(A, b, np.zeros(n), 1e-10, 30, 20000, prec=prec)
                    its = {"bicgstab": s["computed_iterations"], "cgs": c["computed_iterations"],
                           "fgmres": f["computed_iterations"]}
                    assert s["converged"] and c["converged"] and f["converged"]
                    if base is None:
                        base = its
                    for k in its:
                        shift[k] = max(shift[k], abs(its[k] - base[k]) / base[k])
    finally:
        oracle.set_dot_order(0)
    assert shift["bicgstab"] > 0.05 and shift["cgs"] > 0.05, shift
    assert shift["fgmres"] <= 0.01, shift
