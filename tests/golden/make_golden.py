"""Generates the golden fixtures in tests/golden/ by running the sparkit
reference itself (compiled from its sources into oracle/_ref by
oracle/build_ref.sh).  Run from the repository root:

    python -m tests.golden.make_golden

Outputs
  reference_outputs.npz  -- inputs and reference outputs, keyed by case:
      SpMV of every format (reference conversions + multiply) on seeded
      matrices, the conversions' own arrays, Matrix Market texts read and
      written, Jacobi inverse diagonals, Chebyshev coefficients and applies,
      and CG / BiCGSTAB / FGMRES solutions, summaries and residual histories
      on the matrices of the reference's solver tests.
known_answers.json (hand-written, not generated) holds the known-answer
vectors of the reference's Catch2 tests.
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.binding import Reference  # noqa: E402
from sparkit_b200 import matgen  # noqa: E402
from sparkit_b200.formats import Compressed_row_matrix  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_outputs.npz")

# block shapes of the conversion fixtures: square, rectangular, blocks that
# do not divide the matrix, and block rows taller than a warp
CONVERT_BLOCKS = ((1, 1), (2, 2), (3, 3), (2, 3), (1, 4), (4, 4), (5, 7), (33, 2), (64, 1))


def spmv_matrices():
    """Seeded small matrices covering the layouts' edge cases."""
    rng = np.random.default_rng(7)
    mats = {
        "lap2d_16": matgen.laplacian_2d_dirichlet(16),
        "lap3d_6": matgen.laplacian_3d_dirichlet(6),
        "zipf_400": matgen.zipf_random(400, s=1.5, cap=96, seed=3),
        "vec3_4": matgen.vector_laplacian_3d_bsr_csr(4, seed=1),
    }
    # rectangular with empty rows
    n, m = 37, 53
    rows = rng.integers(0, n, 160)
    cols = rng.integers(0, m, 160)
    keep = rows % 5 != 2  # rows 2, 7, 12, ... stay empty
    mats["rect_37x53"] = Compressed_row_matrix.from_entries((n, m), rows[keep], cols[keep],
                                                            rng.standard_normal(keep.sum()))
    # one long row among short ones (exercises the long-row CSR path)
    n = 3000
    rows = np.concatenate([np.full(2600, 5), rng.integers(0, n, 4000)])
    cols = np.concatenate([rng.permutation(n)[:2600], rng.integers(0, n, 4000)])
    mats["longrow_3000"] = Compressed_row_matrix.from_entries((n, n), rows, cols,
                                                              rng.standard_normal(rows.size))
    # nrow not a multiple of the BSR block size (the reference truncates)
    mats["odd_7"] = matgen.tridiagonal_matrix(7, -1.0, 4.0, -2.0)
    return mats


LANCZOS_TARGETS = ("largest_magnitude", "smallest_magnitude", "largest_algebraic", "smallest_algebraic")


def eigen_matrices():
    """Symmetric matrices for the eigenvalue estimates: definite, an
    indefinite shifted Laplacian, n below the Krylov dimension, and 2 I,
    whose first Lanczos residual is exactly zero (the reference rejects
    shapes below 2 x 2, Shape.cpp:8-10)."""
    from sparkit_b200.formats import Compressed_row_matrix as C
    L = matgen.laplacian_2d_dirichlet(10)
    n = L.shape()[0]
    lens = np.diff(L.row_ptr())
    rows = np.repeat(np.arange(n), lens)
    vals = L.values() - 3.0 * (rows == L.col_ind())  # spectrum in (-3, 5)
    return {
        "lap2d_24": matgen.laplacian_2d_dirichlet(24),
        "grid16": matgen.poisson_2d(4, 4, 5.0),
        "tridiag50": matgen.tridiagonal_matrix(50, -1.0, 4.0, -1.0),
        "lap3d_6": matgen.laplacian_3d_dirichlet(6),
        "indef_100": C((n, n), L.row_ptr(), L.col_ind(), vals),
        "tridiag5": matgen.tridiagonal_matrix(5, -1.0, 2.0, -1.0),
        "twoI_4x4": C((4, 4), np.arange(5), np.arange(4), np.full(4, 2.0)),
    }


def mm_texts():
    """Seeded Matrix Market texts for the reader's fixtures: comments and a
    blank line before the size line, duplicate entries (the last one wins),
    symmetric files with diagonals and duplicates, skew-symmetric (read as
    stored), pattern, signed integers, CRLF line ends, extreme and
    oddly written reals, and 17-digit values."""
    rng = np.random.default_rng(21)
    out = {}

    def body(entries, fmt):
        return "".join(fmt(*e) for e in entries)

    n, m, k = 200, 150, 3000
    r, c = rng.integers(1, n + 1, k), rng.integers(1, m + 1, k)
    r[-40:], c[-40:] = r[:40], c[:40]  # duplicates of earlier entries
    v = rng.standard_normal(k) * 10.0 ** rng.integers(-8, 8, k)
    out["general_dup"] = ("%%MatrixMarket matrix coordinate real general\n% seeded\n\n%\n"
                          f"{n} {m} {k}\n" + body(zip(r, c, v), lambda a, b, x: f"{a} {b} {x:.17g}\n"))
    n, k = 120, 900
    r, c = rng.integers(1, n + 1, k), rng.integers(1, n + 1, k)
    r, c = np.maximum(r, c), np.minimum(r, c)  # lower triangle
    r[:60] = c[:60]  # diagonal entries
    r[-30:], c[-30:] = r[60:90], c[60:90]
    v = rng.uniform(-1, 1, k)
    out["symmetric_dup"] = (f"%%MatrixMarket matrix coordinate real symmetric\n{n} {n} {k}\n" +
                            body(zip(r, c, v), lambda a, b, x: f"{a} {b} {x:.17g}\n"))
    out["skew"] = ("%%MatrixMarket matrix coordinate real skew-symmetric\n5 5 4\n2 1 1.5\n3 1 -2\n"
                   "4 2 3.25\n5 4 0.5\n")
    out["pattern_sym"] = "%%MatrixMarket matrix coordinate pattern symmetric\n4 4 5\n1 1\n2 1\n3 2\n4 4\n4 1\n"
    out["integer_signed"] = ("%%MatrixMarket matrix coordinate integer general\n4 3 5\n1 1 -7\n2 3 +12\n"
                             "4 2 0\n3 1 123456789\n1 1 9\n")
    out["crlf"] = "%%MatrixMarket matrix coordinate real general\r\n3 3 3\r\n1 1 1.5\r\n2 3 -2.25\r\n3 2 1e3\r\n"
    out["odd_reals"] = ("%%MatrixMarket matrix coordinate real general\n3 4 11\n1 1 1e-300\n1 2 5e-324\n"
                        "1 3 1.7976931348623157e308\n1 4 -0.0\n2 1 1.\n2 2 .5\n2 3 +3\n3 1 1E5\n"
                        "3 4 0.1000000000000000055511151231257827\n3 3 -1e400\n3 2 1e-400\n")
    out["tabs_and_spaces"] = "%%MatrixMarket matrix coordinate real general\n  3\t3  2\n\t1   1\t2.5  \n 3 3 -1\n"
    return out


def main():
    R = Reference()
    out = {}
    for name, A in spmv_matrices().items():
        for dt in (np.float64, np.float32):
            Ad = A.astype(dt)
            tag = f"spmv/{name}/{np.dtype(dt).name}"
            x = matgen.uniform_vector(Ad.shape()[1], seed=11, dtype=dt)
            out[f"{tag}/row_ptr"] = Ad.row_ptr()
            out[f"{tag}/col_ind"] = Ad.col_ind()
            out[f"{tag}/values"] = Ad.values()
            out[f"{tag}/shape"] = np.array(Ad.shape())
            out[f"{tag}/x"] = x
            out[f"{tag}/y_csr"] = R.spmv(Ad, x, "csr")
            out[f"{tag}/y_ell"] = R.spmv(Ad, x, "ell")
            out[f"{tag}/y_jad"] = R.spmv(Ad, x, "jad")
            for br, bc in ((2, 2), (3, 3), (2, 3)):
                out[f"{tag}/y_bsr{br}{bc}"] = R.spmv(Ad, x, "bsr", (br, bc))
    # the reference's own conversions (FP64), the input of the device-side
    # construction tests; the ELL of longrow_3000 (7.8M padded slots) is
    # left out, its layout is the CSR padded to the longest row
    convs = dict(spmv_matrices())
    convs["empty_5x4"] = Compressed_row_matrix((5, 4), np.zeros(6, np.int64), np.zeros(0, np.int64), np.zeros(0))
    for name, A in convs.items():
        tag = f"convert/{name}"
        lens = np.diff(A.row_ptr())
        if A.shape()[0] * int(lens.max()) <= 200000:
            E = R.to_ellpack(A)
            out[f"{tag}/ell/width"] = np.array(E.max_nnz_per_row())
            out[f"{tag}/ell/col_ind"] = E.col_ind()
            out[f"{tag}/ell/values"] = E.values()
        J = R.to_jagged_diagonal(A)
        for f in ("perm", "jdiag", "col_ind", "values"):
            out[f"{tag}/jad/{f}"] = getattr(J, f)()
        for br, bc in CONVERT_BLOCKS:
            B = R.to_block_sparse_row(A, br, bc)
            for f in ("row_ptr", "col_ind", "values"):
                out[f"{tag}/bsr{br}x{bc}/{f}"] = getattr(B, f)()
    # Lanczos and the eigenvalue estimates (conditioning.hpp:112, :132;
    # lanczos.hpp:495) on symmetric matrices, FP64 and FP32; "twoI_4x4" (2 I)
    # takes the zero-beta random restart (lanczos.hpp:184-186)
    for name, A in eigen_matrices().items():
        for dt in (np.float64, np.float32):
            Ad = A.astype(dt)
            tag = f"eigen/{name}/{np.dtype(dt).name}"
            out[f"{tag}/bounds"] = np.array(R.eigenvalue_bounds(Ad), dtype=dt)
            out[f"{tag}/radius"] = np.array(R.spectral_radius(Ad), dtype=dt)
            for target in LANCZOS_TARGETS:
                r = R.lanczos(Ad, nev=3, m=12, tol=1e-8, max_restarts=5, target=target, collect=True,
                              vectors=True)
                key = f"{tag}/lanczos/{target}"
                for k in ("eigenvalues", "residual_norms", "restart_residuals", "eigenvectors"):
                    out[f"{key}/{k}"] = r[k]
                out[f"{key}/scalars"] = np.array([r["computed_restarts"], r["converged_count"],
                                                  int(r["converged"])])
    # Matrix Market: the reference's read_matrix_market + to_compressed_row
    # on seeded texts (both value types), and its write_matrix_market of the
    # results
    for name, text in mm_texts().items():
        raw = text.encode()
        out[f"mm/{name}/text"] = np.frombuffer(raw, dtype=np.uint8)
        for dt in (np.float64, np.float32):
            M = R.mm_read(raw, dt)
            tag = f"mm/{name}/{np.dtype(dt).name}"
            out[f"{tag}/shape"] = np.array(M.shape())
            out[f"{tag}/row_ptr"] = M.row_ptr()
            out[f"{tag}/col_ind"] = M.col_ind()
            out[f"{tag}/values"] = M.values()
            out[f"{tag}/written"] = np.frombuffer(R.mm_write(M), dtype=np.uint8)
    # preconditioners
    P = matgen.poisson_2d(8, 8, 0.5)
    out["jacobi/poisson8/inv_d"] = R.jacobi(P)
    for lmin, lmax, deg in ((0.5, 8.5, 8), (3.0, 13.0, 4), (1.0, 1.0, 5), (2.0, 6.0, 0)):
        key = f"cheb/{lmin}_{lmax}_{deg}"
        out[f"{key}/coeffs_f64"] = R.chebyshev_coeffs(P, lmin, lmax, deg)
        out[f"{key}/coeffs_f32"] = R.chebyshev_coeffs(P.astype(np.float32), lmin, lmax, deg)
        r = matgen.uniform_vector(P.shape()[0], seed=5)
        out[f"{key}/r"] = r
        out[f"{key}/z"] = R.chebyshev_apply(P, lmin, lmax, deg, r)
    # solvers on the reference tests' matrices (and a Dirichlet grid)
    problems = {
        "grid16": matgen.poisson_2d(4, 4, 5.0),
        "tridiag4": matgen.tridiagonal_matrix(4, -1.0, 4.0, -1.0),
        "convdiff": matgen.convdiff_centered_2d(4, 4, 1.0, 0.3, 0.3, 5.0),
        "nonsym": matgen.nonsymmetric_sample(),
        "lap2d_24": matgen.laplacian_2d_dirichlet(24),
        "upwind_20": matgen.convection_diffusion_2d(20, 20, 1.0, 0.8, 0.4),
    }
    spd = {"grid16", "tridiag4", "lap2d_24"}
    for name, A in problems.items():
        n = A.shape()[0]
        xt = np.arange(1, n + 1, dtype=np.float64) if n <= 16 else matgen.uniform_vector(n, seed=0)
        b = R.spmv(A, xt, "csr")
        base = f"solve/{name}"
        out[f"{base}/row_ptr"] = A.row_ptr()
        out[f"{base}/col_ind"] = A.col_ind()
        out[f"{base}/values"] = A.values()
        out[f"{base}/b"] = b
        precs = {"none": None, "jacobi": "jacobi", "cheb": ("chebyshev", 0.5, 9.0, 6)}
        for pname, spec in precs.items():
            runs = []
            if name in spd:
                runs.append(("cg_left", lambda: R.cg(A, b, np.zeros(n), 1e-12, 50, 500, left=spec, collect=True)))
                runs.append(("cg_right", lambda: R.cg(A, b, np.zeros(n), 1e-12, 7, 500, right=spec, collect=True)))
            runs.append(("bicgstab", lambda: R.bicgstab(A, b, np.zeros(n), 1e-12, 500, left=spec, collect=True)))
            runs.append(("fgmres", lambda: R.fgmres(A, b, np.zeros(n), 1e-12, 5, 500, prec=spec, collect=True)))
            runs.append(("gmres_left", lambda: R.gmres(A, b, np.zeros(n), 1e-12, 5, 500, left=spec, collect=True)))
            runs.append(("gmres_right", lambda: R.gmres(A, b, np.zeros(n), 1e-12, 6, 500, right=spec, collect=True)))
            runs.append(("cgs", lambda: R.cgs(A, b, np.zeros(n), 1e-12, 500, left=spec, collect=True)))
            if name in spd:
                runs.append(("minres", lambda: R.minres(A, b, np.zeros(n), 1e-12, 500, left=spec, collect=True)))
            for rname, fn in runs:
                x, s = fn()
                key = f"{base}/{pname}/{rname}"
                out[f"{key}/x"] = x
                out[f"{key}/iters"] = np.array(s["computed_iterations"])
                out[f"{key}/converged"] = np.array(int(s["converged"]))
                out[f"{key}/residual_norm"] = np.array(s["residual_norm"])
                out[f"{key}/history"] = np.array(s["iteration_residuals"])
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT}: {len(out)} arrays, {os.path.getsize(OUT)} bytes")


if __name__ == "__main__":
    main()
