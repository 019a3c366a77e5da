"""ctypes access to the CPU oracle (liboracle.so, the C restatement) and to
the compiled reference (_ref/libsparkit_ref.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py, never by the sparkit_b200 package.

Preconditioners are given as specs: None / "identity", "jacobi", or
("chebyshev", lambda_min, lambda_max, degree).
"""
import ctypes
import os

import numpy as np

from sparkit_b200.formats import (Block_sparse_row_matrix, Compressed_row_matrix, Ellpack_matrix,
                                  Jagged_diagonal_matrix)

from .build import ORACLE_SO, REF_SO, build_oracle

c_i64 = ctypes.c_int64
c_vp = ctypes.c_void_p


class Operator(ctypes.Structure):
    _fields_ = [("format", ctypes.c_int32), ("nrow", c_i64), ("ncol", c_i64), ("width", c_i64),
                ("block_rows", c_i64), ("block_cols", c_i64), ("row_ptr", c_vp), ("col_ind", c_vp),
                ("perm", c_vp), ("vals", c_vp)]


class Precond(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int32), ("inv_diag", c_vp), ("coeffs", c_vp), ("lambda_min", ctypes.c_double),
                ("lambda_max", ctypes.c_double), ("degree", c_i64), ("op", c_vp)]


class CgCfg(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("restart_iterations", c_i64), ("max_iterations", c_i64),
                ("collect_residuals", ctypes.c_int32)]


class KrylovCfg(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("max_iterations", c_i64), ("collect_residuals", ctypes.c_int32)]


class FgmresCfg(ctypes.Structure):
    _fields_ = [("tolerance", ctypes.c_double), ("restart_dimension", c_i64), ("max_iterations", c_i64),
                ("collect_residuals", ctypes.c_int32)]


class Summary(ctypes.Structure):
    _fields_ = [("residual_norm", ctypes.c_double), ("computed_iterations", c_i64), ("converged", ctypes.c_int32),
                ("status", ctypes.c_int32), ("history_length", c_i64)]

    def as_dict(self, hist=None):
        d = dict(residual_norm=self.residual_norm, computed_iterations=self.computed_iterations,
                 converged=bool(self.converged), status=self.status)
        if hist is not None:
            d["iteration_residuals"] = hist[: self.history_length].tolist()
        return d



class LanczosCfg(ctypes.Structure):
    _fields_ = [("num_eigenvalues", c_i64), ("krylov_dimension", c_i64), ("tolerance", ctypes.c_double),
                ("max_restarts", c_i64), ("target", ctypes.c_int32), ("collect_residuals", ctypes.c_int32)]


class LanczosOut(ctypes.Structure):
    _fields_ = [("count", c_i64), ("computed_restarts", c_i64), ("converged_count", c_i64),
                ("residual_count", c_i64), ("restart_residuals_count", c_i64), ("converged", ctypes.c_int32)]

    def as_dict(self, ev, vecs, res, rr):
        d = dict(eigenvalues=ev[: self.count].copy(), residual_norms=res[: self.residual_count].copy(),
                 computed_restarts=self.computed_restarts, converged_count=self.converged_count,
                 converged=bool(self.converged), restart_residuals=rr[: self.restart_residuals_count].copy())
        if vecs is not None:
            d["eigenvectors"] = vecs[: self.count].copy()
        return d


# Eigen_target (eigen_target.hpp:13-20)
EIGEN_TARGETS = ("largest_magnitude", "smallest_magnitude", "largest_algebraic", "smallest_algebraic",
                 "largest_real", "smallest_real")


class MmCsr(ctypes.Structure):
    _fields_ = [("nrow", c_i64), ("ncol", c_i64), ("nnz", c_i64), ("row_ptr", c_vp), ("col_ind", c_vp),
                ("values", c_vp), ("err", ctypes.c_char * 256)]


class MatrixMarketError(ValueError):
    """The reason a Matrix Market text was rejected."""


def _pad_to_blocks(x, bc):
    """x followed by zeros up to a whole number of bc-wide block columns."""
    m = -(-x.size // int(bc)) * int(bc)
    if m == x.size:
        return x
    xp = np.zeros(m, dtype=x.dtype)
    xp[:x.size] = x
    return xp

def _p(a):
    return None if a is None else a.ctypes.data_as(c_vp)


def _sfx(dtype):
    return "f64" if np.dtype(dtype) == np.float64 else "f32"


class Oracle:
    """The plain-C restatement (sk_oracle.c)."""

    def __init__(self):
        build_oracle()
        self.L = ctypes.CDLL(ORACLE_SO)
        self._keep = []

    def _operator(self, A):
        keep = []

        def k(a):
            a = np.ascontiguousarray(a)
            keep.append(a)
            return _p(a)

        n, m = A.shape()
        if isinstance(A, Compressed_row_matrix):
            op = Operator(0, n, m, 0, 0, 0, k(A.row_ptr()), k(A.col_ind()), None, k(A.values()))
        elif isinstance(A, Ellpack_matrix):
            op = Operator(1, n, m, A.max_nnz_per_row(), 0, 0, None, k(A.col_ind()), None, k(A.values()))
        elif isinstance(A, Jagged_diagonal_matrix):
            perm = A.perm() if A.perm().size else np.arange(n, dtype=np.int64)
            op = Operator(2, n, m, A.num_jdiags(), 0, 0, k(A.jdiag()), k(A.col_ind()), k(perm), k(A.values()))
        elif isinstance(A, Block_sparse_row_matrix):
            op = Operator(3, n, m, 0, A.block_rows(), A.block_cols(), k(A.row_ptr()), k(A.col_ind()), None,
                          k(A.values()))
        else:
            raise TypeError(type(A))
        return op, keep

    def set_dot_order(self, mode):
        """0: the reference's sequential dot products; 1: chunked order;
        2: reversed order."""
        self.L.sko_set_dot_order(int(mode))

    def spmv(self, A, x):
        x = np.ascontiguousarray(x, dtype=A.dtype)
        y = np.zeros(A.shape()[0], dtype=A.dtype)
        s = _sfx(A.dtype)
        n = A.shape()[0]
        if isinstance(A, Compressed_row_matrix):
            getattr(self.L, f"sko_csr_spmv_{s}")(c_i64(n), _p(A.row_ptr()), _p(A.col_ind()), _p(A.values()),
                                                  _p(x), _p(y))
        elif isinstance(A, Ellpack_matrix):
            getattr(self.L, f"sko_ell_spmv_{s}")(c_i64(n), c_i64(A.max_nnz_per_row()), _p(A.col_ind()),
                                                  _p(A.values()), _p(x), _p(y))
        elif isinstance(A, Jagged_diagonal_matrix):
            perm = A.perm() if A.perm().size else np.arange(n, dtype=np.int64)
            getattr(self.L, f"sko_jad_spmv_{s}")(c_i64(n), c_i64(A.num_jdiags()), _p(perm), _p(A.jdiag()),
                                                  _p(A.col_ind()), _p(A.values()), _p(x), _p(y))
        elif isinstance(A, Block_sparse_row_matrix):
            # a partial last block column reads past x (spmv.hpp:148-174 has
            # no bound there): those reads see zeros, as on the device
            xp = _pad_to_blocks(x, A.block_cols())
            getattr(self.L, f"sko_bsr_spmv_{s}")(c_i64(n), c_i64(A.block_rows()), c_i64(A.block_cols()),
                                                  _p(A.row_ptr()), _p(A.col_ind()), _p(A.values()), _p(xp), _p(y))
        else:
            raise TypeError(type(A))
        return y

    def jacobi(self, A):
        n, m = A.shape()
        out = np.zeros(min(n, m), dtype=A.dtype)
        rc = getattr(self.L, f"sko_jacobi_{_sfx(A.dtype)}")(c_i64(n), c_i64(m), _p(A.row_ptr()), _p(A.col_ind()),
                                                            _p(A.values()), _p(out))
        if rc != 0:
            raise ValueError("jacobi: zero diagonal entry")
        return out

    def chebyshev_coeffs(self, lmin, lmax, degree, dtype=np.float64):
        out = np.zeros(degree + 1, dtype=dtype)
        f = getattr(self.L, f"sko_chebyshev_coeffs_{_sfx(dtype)}")
        if np.dtype(dtype) == np.float64:
            f(ctypes.c_double(lmin), ctypes.c_double(lmax), c_i64(degree), _p(out))
        else:
            f(ctypes.c_float(lmin), ctypes.c_float(lmax), c_i64(degree), _p(out))
        return out

    def _precond(self, spec, A, keep):
        if spec is None or spec == "identity":
            return None
        if spec == "jacobi":
            inv = self.jacobi(A)
            keep.append(inv)
            return Precond(1, _p(inv), None, 0.0, 0.0, 0, None)
        kind, lmin, lmax, deg = spec
        assert kind == "chebyshev"
        co = self.chebyshev_coeffs(lmin, lmax, deg, A.dtype)
        keep.append(co)
        return Precond(2, None, _p(co), float(lmin), float(lmax), int(deg), None)

    def chebyshev_apply(self, A, lmin, lmax, degree, r):
        op, keep = self._operator(A)
        co = self.chebyshev_coeffs(lmin, lmax, degree, A.dtype)
        r = np.ascontiguousarray(r, dtype=A.dtype)
        z = np.zeros_like(r)
        f = getattr(self.L, f"sko_chebyshev_apply_{_sfx(A.dtype)}")
        if A.dtype == np.float64:
            f(ctypes.byref(op), _p(co), ctypes.c_double(lmin), ctypes.c_double(lmax), c_i64(degree), _p(r), _p(z))
        else:
            f(ctypes.byref(op), _p(co), ctypes.c_float(lmin), ctypes.c_float(lmax), c_i64(degree), _p(r), _p(z))
        return z

    def _solve(self, name, A, precs, b, x0, cfg_struct, max_hist, prec_matrix=None):
        op, keep = self._operator(A)
        pm = prec_matrix if prec_matrix is not None else A
        ps = [self._precond(s, pm, keep) for s in precs]
        b = np.ascontiguousarray(b, dtype=A.dtype)
        x = np.array(x0, dtype=A.dtype, copy=True)
        hist = np.zeros(max(int(max_hist), 1) + 4)
        s = Summary()
        args = [ctypes.byref(op)] + [ctypes.byref(p) if p is not None else None for p in ps]
        getattr(self.L, f"sko_{name}_{_sfx(A.dtype)}")(*args, _p(b), _p(x), ctypes.byref(cfg_struct),
                                                        ctypes.byref(s), _p(hist))
        if name == "cg":
            s.history_length = s.computed_iterations if cfg_struct.collect_residuals else 0
        return x, s.as_dict(hist)

    def cg(self, A, b, x0, tol, restart, max_it, left=None, right=None, collect=False, prec_matrix=None):
        return self._solve("cg", A, [left, right], b, x0, CgCfg(tol, restart, max_it, int(collect)), max_it,
                           prec_matrix)

    def bicgstab(self, A, b, x0, tol, max_it, left=None, right=None, collect=False, prec_matrix=None):
        return self._solve("bicgstab", A, [left, right], b, x0, KrylovCfg(tol, max_it, int(collect)), max_it + 2,
                           prec_matrix)

    def fgmres(self, A, b, x0, tol, restart, max_it, prec=None, collect=False, prec_matrix=None):
        return self._solve("fgmres", A, [prec], b, x0, FgmresCfg(tol, restart, max_it, int(collect)), max_it,
                           prec_matrix)

    def gmres(self, A, b, x0, tol, restart, max_it, left=None, right=None, collect=False, prec_matrix=None):
        return self._solve("gmres", A, [left, right], b, x0, FgmresCfg(tol, restart, max_it, int(collect)), max_it,
                           prec_matrix)

    def cgs(self, A, b, x0, tol, max_it, left=None, right=None, collect=False, prec_matrix=None):
        return self._solve("cgs", A, [left, right], b, x0, KrylovCfg(tol, max_it, int(collect)), max_it + 2,
                           prec_matrix)

    def minres(self, A, b, x0, tol, max_it, left=None, right=None, collect=False, prec_matrix=None):
        return self._solve("minres", A, [left, right], b, x0, KrylovCfg(tol, max_it, int(collect)), max_it + 2,
                           prec_matrix)

    # -------------------------------------------------------------- #
    # Matrix Market (sk_oracle_mm.c)                                   #
    # -------------------------------------------------------------- #

    def mm_read(self, text, dtype=np.float64):
        """read_matrix_market<T> + to_compressed_row on the text (bytes)."""
        dt = np.dtype(dtype)
        text = bytes(text)
        m = MmCsr()
        rc = getattr(self.L, f"sko_mm_read_{_sfx(dt)}")(text, c_i64(len(text)), ctypes.byref(m))
        if rc:
            raise MatrixMarketError(m.err.decode())
        try:
            rp = np.ctypeslib.as_array(ctypes.cast(m.row_ptr, ctypes.POINTER(c_i64)), (m.nrow + 1,)).copy()
            ci = (np.ctypeslib.as_array(ctypes.cast(m.col_ind, ctypes.POINTER(c_i64)), (m.nnz,)).copy()
                  if m.nnz else np.zeros(0, np.int64))
            ct = ctypes.c_double if dt == np.float64 else ctypes.c_float
            va = (np.ctypeslib.as_array(ctypes.cast(m.values, ctypes.POINTER(ct)), (m.nnz,)).copy()
                  if m.nnz else np.zeros(0, dt))
        finally:
            self.L.sko_mm_free(ctypes.byref(m))
        return Compressed_row_matrix((m.nrow, m.ncol), rp, ci, va)

    def mm_write(self, A):
        """write_matrix_market of a CSR matrix, as bytes."""
        n, mcol = A.shape()
        f = getattr(self.L, f"sko_mm_write_{_sfx(A.dtype)}")
        f.restype = c_vp
        ln = c_i64()
        rp = np.ascontiguousarray(A.row_ptr(), np.int64)
        ci = np.ascontiguousarray(A.col_ind(), np.int64)
        va = np.ascontiguousarray(A.values())
        ptr = f(c_i64(n), c_i64(mcol), _p(rp), _p(ci), _p(va), ctypes.byref(ln))
        try:
            return ctypes.string_at(ptr, ln.value)
        finally:
            self.L.sko_free(c_vp(ptr))

    # -------------------------------------------------------------- #
    # Lanczos and the eigenvalue estimates (sk_oracle_lanczos.h)       #
    # -------------------------------------------------------------- #

    def tridiagonal_eigen(self, d, e, tol=1e-15, max_iterations=None, vectors=True):
        """tridiagonal_eigen (dense_tridiagonal_eigen.hpp:58): unsorted
        eigenvalues and, per eigenvalue, its eigenvector (rows)."""
        d = np.array(d, dtype=np.float64)
        e = np.array(e, dtype=np.float64)
        n = d.size
        Q = np.zeros((n, n)) if vectors else None
        maxit = 30 * n if max_iterations is None else max_iterations
        self.L.sko_tridiagonal_eigen_f64(c_i64(n), _p(d), _p(e), ctypes.c_double(tol), c_i64(maxit), _p(Q))
        return d, Q

    def lanczos(self, A, nev=1, m=20, tol=1e-10, max_restarts=10, target="largest_algebraic", collect=False,
                vectors=False):
        """lanczos(n, cfg, multiply(A)) (lanczos.hpp:495)."""
        op, keep = self._operator(A)
        n = A.shape()[0]
        ev = np.zeros(max(nev, 1), A.dtype)
        res = np.zeros(max(nev, 1), A.dtype)
        vecs = np.zeros((max(nev, 1), n), A.dtype) if vectors else None
        rr = np.zeros(max_restarts + 2)
        cfg = LanczosCfg(nev, m, tol, max_restarts, EIGEN_TARGETS.index(target), int(collect))
        out = LanczosOut()
        getattr(self.L, f"sko_lanczos_{_sfx(A.dtype)}")(ctypes.byref(op), ctypes.byref(cfg), _p(ev), _p(vecs),
                                                       _p(res), _p(rr), ctypes.byref(out))
        return out.as_dict(ev, vecs, res, rr)

    def eigenvalue_bounds(self, A, num_iter=30):
        """estimate_eigenvalue_bounds (conditioning.hpp:132): (lmin, lmax)."""
        op, keep = self._operator(A)
        out = np.zeros(2, A.dtype)
        getattr(self.L, f"sko_eigenvalue_bounds_{_sfx(A.dtype)}")(ctypes.byref(op), c_i64(num_iter), _p(out))
        return out[0], out[1]

    def spectral_radius(self, A, num_iter=20):
        """estimate_spectral_radius (conditioning.hpp:112)."""
        op, keep = self._operator(A)
        f = getattr(self.L, f"sko_spectral_radius_{_sfx(A.dtype)}")
        f.restype = ctypes.c_double if A.dtype == np.float64 else ctypes.c_float
        return f(ctypes.byref(op), c_i64(num_iter))

    # -------------------------------------------------------------- #
    # Learned preconditioner network (sk_oracle_net.c)                #
    # -------------------------------------------------------------- #

    def net_param_count(self):
        self.L.skon_param_count.restype = c_i64
        return int(self.L.skon_param_count())

    def net_apply(self, params, v, coef, H, W, round_bf16=True):
        """z = s * net(features(v)); coef = grid_planes(A, H, W)."""
        params = np.ascontiguousarray(params, dtype=np.float32)
        v = np.ascontiguousarray(v, dtype=np.float64)
        coef = np.ascontiguousarray(coef, dtype=np.float32)
        z = np.zeros(H * W)
        y = np.zeros(H * W)
        self.L.skon_apply(ctypes.c_int(H), ctypes.c_int(W), _p(params), _p(v), _p(coef), ctypes.c_int(int(round_bf16)),
                          _p(z), _p(y))
        return z, y

    def net_features(self, r, coef, B, H, W, round_bf16=True):
        r = np.ascontiguousarray(r, dtype=np.float64)
        coef = np.ascontiguousarray(coef, dtype=np.float32)
        x = np.zeros(B * H * W * 8)
        s = np.zeros(B)
        self.L.skon_features(ctypes.c_int(B), ctypes.c_int(H), ctypes.c_int(W), _p(r), _p(coef),
                             ctypes.c_int(int(round_bf16)), _p(x), _p(s))
        return x.reshape(B, H, W, 8), s

    def net_loss_grad(self, params, r, e, coef, B, H, W, mu=0.0, round_bf16=True, grad=True):
        """Loss of a batch (r, e: B*H*W each; coef: B stacked grid_planes)
        and its gradient with respect to the flat parameters."""
        self.L.skon_loss_grad.restype = ctypes.c_double
        params = np.ascontiguousarray(params, dtype=np.float32)
        r = np.ascontiguousarray(r, dtype=np.float64)
        e = np.ascontiguousarray(e, dtype=np.float64)
        coef = np.ascontiguousarray(coef, dtype=np.float32)
        g = np.zeros(self.net_param_count()) if grad else None
        y = np.zeros(B * H * W)
        loss = self.L.skon_loss_grad(ctypes.c_int(B), ctypes.c_int(H), ctypes.c_int(W), _p(params), _p(r), _p(e),
                                     _p(coef), ctypes.c_double(mu), ctypes.c_int(int(round_bf16)), _p(g), _p(y))
        return float(loss), g, y

    def adam(self, p, m, v, g, lr, b1, b2, eps, t):
        """In place on float32 arrays."""
        self.L.skon_adam(c_i64(p.size), _p(p), _p(m), _p(v), _p(np.ascontiguousarray(g, dtype=np.float32)),
                         ctypes.c_float(lr), ctypes.c_float(b1), ctypes.c_float(b2), ctypes.c_float(eps), c_i64(t))


def grid_planes(A, H, W):
    """The six coefficient planes of a 5-point matrix on an H x W grid (row
    index y * W + x): diagonal, west, east, south, north (float32 of the
    entries, 0 where the neighbour is missing) and float32(1 / diagonal)."""
    n = H * W
    rp, ci, va = A.row_ptr(), A.col_ind(), A.values().astype(np.float64)
    rows = np.repeat(np.arange(n, dtype=np.int64), np.diff(rp))
    off = ci - rows
    planes = np.zeros((6, n), dtype=np.float32)
    d64 = np.zeros(n)
    for k, o in enumerate((0, -1, 1, -W, W)):
        sel = off == o
        if k == 1:
            sel &= (rows % W) > 0
        if k == 2:
            sel &= (rows % W) < W - 1
        planes[k, rows[sel]] = va[sel].astype(np.float32)
        if k == 0:
            d64[rows[sel]] = va[sel]
    planes[5] = (1.0 / d64).astype(np.float32)
    return planes


class Reference:
    """The sparkit reference itself, compiled from its sources
    (oracle/build_ref.sh).  Raises OSError when it was not built."""

    KINDS = {None: 0, "identity": 0, "jacobi": 1}

    def __init__(self):
        if not os.path.exists(REF_SO):
            raise OSError(f"{REF_SO} not built (needs the reference sources; see oracle/build_ref.sh)")
        self.L = ctypes.CDLL(REF_SO)
        for name in dir(self.L):
            pass
        for s in ("f64", "f32"):
            for fn in ("ref_csr_create", "ref_to_ellpack", "ref_to_jagged_diagonal", "ref_to_block_sparse_row",
                       "ref_poisson_2d", "ref_tridiagonal", "ref_convdiff_centered_2d",
                       "ref_convection_diffusion_2d", "ref_nonsymmetric_sample"):
                getattr(self.L, f"{fn}_{s}").restype = c_vp
            getattr(self.L, f"ref_multiply_threads_{s}").restype = ctypes.c_double

    # handles -------------------------------------------------------
    def csr_handle(self, A):
        f = getattr(self.L, f"ref_csr_create_{_sfx(A.dtype)}")
        n, m = A.shape()
        return f(c_i64(n), c_i64(m), _p(A.row_ptr()), _p(A.col_ind()), _p(A.values()))

    def destroy(self, h, dtype):
        getattr(self.L, f"ref_destroy_{_sfx(dtype)}")(c_vp(h))

    def info(self, h, dtype):
        out = np.zeros(5, dtype=np.int64)
        getattr(self.L, f"ref_info_{_sfx(dtype)}")(c_vp(h), _p(out))
        return out

    def export_csr(self, h, dtype):
        n, m, nnz, _, _ = self.info(h, dtype)
        rp = np.zeros(n + 1, np.int64)
        ci = np.zeros(nnz, np.int64)
        va = np.zeros(nnz, dtype)
        getattr(self.L, f"ref_export_{_sfx(dtype)}")(c_vp(h), _p(rp), _p(ci), None, _p(va))
        return Compressed_row_matrix((n, m), rp, ci, va)

    def to_ellpack(self, A):
        s = _sfx(A.dtype)
        h = self.csr_handle(A)
        e = getattr(self.L, f"ref_to_ellpack_{s}")(c_vp(h))
        n, m, nnz, w, _ = self.info(e, A.dtype)
        ci = np.zeros(n * w, np.int64)
        va = np.zeros(n * w, A.dtype)
        getattr(self.L, f"ref_export_{s}")(c_vp(e), None, _p(ci), None, _p(va))
        self.destroy(h, A.dtype)
        self.destroy(e, A.dtype)
        return Ellpack_matrix((n, m), w, ci, va)

    def to_jagged_diagonal(self, A):
        s = _sfx(A.dtype)
        h = self.csr_handle(A)
        e = getattr(self.L, f"ref_to_jagged_diagonal_{s}")(c_vp(h))
        n, m, nnz, njd, _ = self.info(e, A.dtype)
        jd = np.zeros(njd + 1, np.int64)
        ci = np.zeros(nnz, np.int64)
        pm = np.zeros(n if nnz else 0, np.int64)
        va = np.zeros(nnz, A.dtype)
        getattr(self.L, f"ref_export_{s}")(c_vp(e), _p(jd), _p(ci), _p(pm) if pm.size else None, _p(va))
        self.destroy(h, A.dtype)
        self.destroy(e, A.dtype)
        return Jagged_diagonal_matrix((n, m), pm, jd, ci, va)

    def to_block_sparse_row(self, A, br, bc):
        s = _sfx(A.dtype)
        h = self.csr_handle(A)
        e = getattr(self.L, f"ref_to_block_sparse_row_{s}")(c_vp(h), c_i64(br), c_i64(bc))
        n, m, nvals, nblocks, nbr = self.info(e, A.dtype)
        rp = np.zeros(nbr + 1, np.int64)
        ci = np.zeros(nblocks, np.int64)
        va = np.zeros(nblocks * br * bc, A.dtype)
        getattr(self.L, f"ref_export_{s}")(c_vp(e), _p(rp), _p(ci), None, _p(va))
        self.destroy(h, A.dtype)
        self.destroy(e, A.dtype)
        return Block_sparse_row_matrix((n, m), br, bc, rp, ci, va)

    def convert_seconds(self, A, fmt, block=(3, 3)):
        """Wall time of the reference's own conversion of A (CSR) to fmt:
        the CSR handle is built before and the result destroyed after the
        timed call."""
        import time
        s = _sfx(A.dtype)
        h = self.csr_handle(A)
        t0 = time.perf_counter()
        if fmt == "ell":
            e = getattr(self.L, f"ref_to_ellpack_{s}")(c_vp(h))
        elif fmt == "jad":
            e = getattr(self.L, f"ref_to_jagged_diagonal_{s}")(c_vp(h))
        else:
            e = getattr(self.L, f"ref_to_block_sparse_row_{s}")(c_vp(h), c_i64(block[0]), c_i64(block[1]))
        secs = time.perf_counter() - t0
        self.destroy(e, A.dtype)
        self.destroy(h, A.dtype)
        return secs

    def mm_read(self, text, dtype=np.float64):
        """The reference's read_matrix_market<T> + to_compressed_row."""
        dt = np.dtype(dtype)
        text = bytes(text)
        f = getattr(self.L, f"ref_mm_read_{_sfx(dt)}")
        f.restype = c_vp
        err = ctypes.create_string_buffer(512)
        h = f(text, c_i64(len(text)), err, c_i64(512))
        if not h:
            raise MatrixMarketError(err.value.decode())
        A = self.export_csr(h, dt)
        self.destroy(h, dt)
        return A

    def mm_read_seconds(self, text, dtype=np.float64):
        """Wall time of the reference's read_matrix_market + to_compressed_row
        on the text (the arrays are not copied out)."""
        import time
        dt = np.dtype(dtype)
        text = bytes(text)
        f = getattr(self.L, f"ref_mm_read_{_sfx(dt)}")
        f.restype = c_vp
        err = ctypes.create_string_buffer(512)
        t0 = time.perf_counter()
        h = f(text, c_i64(len(text)), err, c_i64(512))
        secs = time.perf_counter() - t0
        if not h:
            raise MatrixMarketError(err.value.decode())
        self.destroy(h, dt)
        return secs

    def mm_write(self, A):
        """The reference's write_matrix_market of a CSR matrix, as bytes."""
        h = self.csr_handle(A)
        f = getattr(self.L, f"ref_mm_write_{_sfx(A.dtype)}")
        f.restype = c_i64
        n = f(c_vp(h), None, c_i64(0))
        buf = ctypes.create_string_buffer(int(n) + 1)
        f(c_vp(h), buf, c_i64(n))
        self.destroy(h, A.dtype)
        return buf.raw[:n]

    def lanczos(self, A, nev=1, m=20, tol=1e-10, max_restarts=10, target="largest_algebraic", collect=False,
                vectors=False):
        h = self.csr_handle(A)
        n = A.shape()[0]
        ev = np.zeros(max(nev, 1), A.dtype)
        res = np.zeros(max(nev, 1), A.dtype)
        vecs = np.zeros((max(nev, 1), n), A.dtype) if vectors else None
        rr = np.zeros(max_restarts + 2)
        out = LanczosOut()
        getattr(self.L, f"ref_lanczos_{_sfx(A.dtype)}")(c_vp(h), c_i64(nev), c_i64(m), ctypes.c_double(tol),
                                                       c_i64(max_restarts), EIGEN_TARGETS.index(target),
                                                       int(collect), _p(ev), _p(vecs), _p(res), _p(rr),
                                                       ctypes.byref(out))
        self.destroy(h, A.dtype)
        return out.as_dict(ev, vecs, res, rr)

    def eigenvalue_bounds(self, A, num_iter=30):
        h = self.csr_handle(A)
        out = np.zeros(2, A.dtype)
        getattr(self.L, f"ref_eigenvalue_bounds_{_sfx(A.dtype)}")(c_vp(h), c_i64(num_iter), _p(out))
        self.destroy(h, A.dtype)
        return out[0], out[1]

    def spectral_radius(self, A, num_iter=20):
        h = self.csr_handle(A)
        f = getattr(self.L, f"ref_spectral_radius_{_sfx(A.dtype)}")
        f.restype = ctypes.c_double
        v = f(c_vp(h), c_i64(num_iter))
        self.destroy(h, A.dtype)
        return A.dtype.type(v)

    def _handle_any(self, A):
        """Reference handle of A in its own format (built through the
        reference's conversion from CSR, which the format tests pin)."""
        s = _sfx(A.dtype)
        if isinstance(A, Compressed_row_matrix):
            return self.csr_handle(A), []
        raise TypeError("reference handles are built from CSR; convert with the reference's to_*")

    def spmv(self, A, x, fmt="csr", block=(3, 3)):
        """multiply() of the reference on A (CSR) converted to fmt."""
        s = _sfx(A.dtype)
        h = self.csr_handle(A)
        if fmt == "ell":
            h2 = getattr(self.L, f"ref_to_ellpack_{s}")(c_vp(h))
        elif fmt == "jad":
            h2 = getattr(self.L, f"ref_to_jagged_diagonal_{s}")(c_vp(h))
        elif fmt == "bsr":
            h2 = getattr(self.L, f"ref_to_block_sparse_row_{s}")(c_vp(h), c_i64(block[0]), c_i64(block[1]))
        else:
            h2 = None
        x = np.ascontiguousarray(x, dtype=A.dtype)
        if fmt == "bsr":  # see Oracle.spmv: the partial last block column reads zeros
            x = _pad_to_blocks(x, block[1])
        y = np.zeros(A.shape()[0], A.dtype)
        getattr(self.L, f"ref_multiply_{s}")(c_vp(h2 or h), _p(x), c_i64(x.size), _p(y))
        if h2:
            self.destroy(h2, A.dtype)
        self.destroy(h, A.dtype)
        return y

    def jacobi(self, A):
        h = self.csr_handle(A)
        out = np.zeros(min(A.shape()), A.dtype)
        rc = getattr(self.L, f"ref_jacobi_{_sfx(A.dtype)}")(c_vp(h), _p(out))
        self.destroy(h, A.dtype)
        if rc != 0:
            raise ValueError("jacobi: zero diagonal entry")
        return out

    def chebyshev_coeffs(self, A, lmin, lmax, degree):
        h = self.csr_handle(A)
        out = np.zeros(degree + 1, A.dtype)
        getattr(self.L, f"ref_chebyshev_coeffs_{_sfx(A.dtype)}")(c_vp(h), ctypes.c_double(lmin),
                                                                   ctypes.c_double(lmax), c_i64(degree), _p(out))
        self.destroy(h, A.dtype)
        return out

    def chebyshev_apply(self, A, lmin, lmax, degree, r):
        h = self.csr_handle(A)
        r = np.ascontiguousarray(r, dtype=A.dtype)
        z = np.zeros_like(r)
        getattr(self.L, f"ref_chebyshev_apply_{_sfx(A.dtype)}")(c_vp(h), ctypes.c_double(lmin),
                                                                  ctypes.c_double(lmax), c_i64(degree), _p(r), _p(z))
        self.destroy(h, A.dtype)
        return z

    @staticmethod
    def _pk(spec):
        if spec is None or spec == "identity":
            return 0, 0.0, 0.0, 0
        if spec == "jacobi":
            return 1, 0.0, 0.0, 0
        _, lmin, lmax, deg = spec
        return 2, float(lmin), float(lmax), int(deg)

    def cg(self, A, b, x0, tol, restart, max_it, left=None, right=None, collect=False):
        h = self.csr_handle(A)
        lk, lmin, lmax, deg = self._pk(left)
        rk, rmin, rmax, rdeg = self._pk(right)
        if lk == 2 and rk == 2:
            assert (lmin, lmax, deg) == (rmin, rmax, rdeg)
        if rk == 2:
            lmin, lmax, deg = rmin, rmax, rdeg
        b = np.ascontiguousarray(b, dtype=A.dtype)
        x = np.array(x0, dtype=A.dtype, copy=True)
        hist = np.zeros(max_it + 4)
        s = Summary()
        rc = getattr(self.L, f"ref_cg_{_sfx(A.dtype)}")(c_vp(h), _p(b), _p(x), ctypes.c_double(tol), c_i64(restart),
                                                        c_i64(max_it), int(collect), lk, rk, ctypes.c_double(lmin),
                                                        ctypes.c_double(lmax), c_i64(deg), ctypes.byref(s), _p(hist))
        self.destroy(h, A.dtype)
        if rc == -1:
            raise ValueError("jacobi: zero diagonal entry")
        return x, s.as_dict(hist)

    def bicgstab(self, A, b, x0, tol, max_it, left=None, right=None, collect=False):
        h = self.csr_handle(A)
        lk, lmin, lmax, deg = self._pk(left)
        rk, rmin, rmax, rdeg = self._pk(right)
        if rk == 2:
            lmin, lmax, deg = rmin, rmax, rdeg
        b = np.ascontiguousarray(b, dtype=A.dtype)
        x = np.array(x0, dtype=A.dtype, copy=True)
        hist = np.zeros(max_it + 4)
        s = Summary()
        rc = getattr(self.L, f"ref_bicgstab_{_sfx(A.dtype)}")(c_vp(h), _p(b), _p(x), ctypes.c_double(tol),
                                                              c_i64(max_it), int(collect), lk, rk,
                                                              ctypes.c_double(lmin), ctypes.c_double(lmax), c_i64(deg),
                                                              ctypes.byref(s), _p(hist))
        self.destroy(h, A.dtype)
        if rc == -1:
            raise ValueError("jacobi: zero diagonal entry")
        return x, s.as_dict(hist)

    def fgmres(self, A, b, x0, tol, restart, max_it, prec=None, collect=False):
        h = self.csr_handle(A)
        pk, lmin, lmax, deg = self._pk(prec)
        b = np.ascontiguousarray(b, dtype=A.dtype)
        x = np.array(x0, dtype=A.dtype, copy=True)
        hist = np.zeros(max_it + 4)
        s = Summary()
        rc = getattr(self.L, f"ref_fgmres_{_sfx(A.dtype)}")(c_vp(h), _p(b), _p(x), ctypes.c_double(tol),
                                                            c_i64(restart), c_i64(max_it), int(collect), pk,
                                                            ctypes.c_double(lmin), ctypes.c_double(lmax), c_i64(deg),
                                                            ctypes.byref(s), _p(hist))
        self.destroy(h, A.dtype)
        if rc == -1:
            raise ValueError("jacobi: zero diagonal entry")
        return x, s.as_dict(hist)

    def gmres(self, A, b, x0, tol, restart, max_it, left=None, right=None, collect=False):
        h = self.csr_handle(A)
        lk, lmin, lmax, deg = self._pk(left)
        rk, rmin, rmax, rdeg = self._pk(right)
        if rk == 2:
            lmin, lmax, deg = rmin, rmax, rdeg
        b = np.ascontiguousarray(b, dtype=A.dtype)
        x = np.array(x0, dtype=A.dtype, copy=True)
        hist = np.zeros(max_it + 4)
        s = Summary()
        rc = getattr(self.L, f"ref_gmres_{_sfx(A.dtype)}")(c_vp(h), _p(b), _p(x), ctypes.c_double(tol),
                                                           c_i64(restart), c_i64(max_it), int(collect), lk, rk,
                                                           ctypes.c_double(lmin), ctypes.c_double(lmax), c_i64(deg),
                                                           ctypes.byref(s), _p(hist))
        self.destroy(h, A.dtype)
        if rc == -1:
            raise ValueError("jacobi: zero diagonal entry")
        return x, s.as_dict(hist)

    def _krylov2(self, name, A, b, x0, tol, max_it, left, right, collect):
        h = self.csr_handle(A)
        lk, lmin, lmax, deg = self._pk(left)
        rk, rmin, rmax, rdeg = self._pk(right)
        if rk == 2:
            lmin, lmax, deg = rmin, rmax, rdeg
        b = np.ascontiguousarray(b, dtype=A.dtype)
        x = np.array(x0, dtype=A.dtype, copy=True)
        hist = np.zeros(max_it + 4)
        s = Summary()
        rc = getattr(self.L, f"ref_{name}_{_sfx(A.dtype)}")(c_vp(h), _p(b), _p(x), ctypes.c_double(tol),
                                                           c_i64(max_it), int(collect), lk, rk,
                                                           ctypes.c_double(lmin), ctypes.c_double(lmax), c_i64(deg),
                                                           ctypes.byref(s), _p(hist))
        self.destroy(h, A.dtype)
        if rc == -1:
            raise ValueError("jacobi: zero diagonal entry")
        return x, s.as_dict(hist)

    def cgs(self, A, b, x0, tol, max_it, left=None, right=None, collect=False):
        return self._krylov2("cgs", A, b, x0, tol, max_it, left, right, collect)

    def minres(self, A, b, x0, tol, max_it, left=None, right=None, collect=False):
        return self._krylov2("minres", A, b, x0, tol, max_it, left, right, collect)

    # generators of the reference's tests ----------------------------
    def _gen(self, name, dtype, *args):
        h = getattr(self.L, f"ref_{name}_{_sfx(dtype)}")(*args)
        A = self.export_csr(h, dtype)
        self.destroy(h, dtype)
        return A

    def poisson_2d(self, nx, ny, shift=0.0, dtype=np.float64):
        return self._gen("poisson_2d", dtype, c_i64(nx), c_i64(ny), ctypes.c_double(shift))

    def tridiagonal(self, n, sub, diag, sup, dtype=np.float64):
        return self._gen("tridiagonal", dtype, c_i64(n), ctypes.c_double(sub), ctypes.c_double(diag),
                         ctypes.c_double(sup))

    def convdiff_centered_2d(self, nx, ny, d, cx, cy, shift=0.0, dtype=np.float64):
        return self._gen("convdiff_centered_2d", dtype, c_i64(nx), c_i64(ny), ctypes.c_double(d),
                         ctypes.c_double(cx), ctypes.c_double(cy), ctypes.c_double(shift))

    def convection_diffusion_2d(self, nx, ny, d, cx, cy, dtype=np.float64):
        return self._gen("convection_diffusion_2d", dtype, c_i64(nx), c_i64(ny), ctypes.c_double(d),
                         ctypes.c_double(cx), ctypes.c_double(cy))

    def nonsymmetric_sample(self, dtype=np.float64):
        return self._gen("nonsymmetric_sample", dtype)

    # timing of the reference's multiply on several host threads ---------
    def multiply_threads_seconds(self, A, x, nthreads, reps, fmt="csr"):
        s = _sfx(A.dtype)
        h = self.csr_handle(A)
        h2 = None
        if fmt == "ell":
            h2 = getattr(self.L, f"ref_to_ellpack_{s}")(c_vp(h))
        elif fmt == "jad":
            h2 = getattr(self.L, f"ref_to_jagged_diagonal_{s}")(c_vp(h))
        x = np.ascontiguousarray(x, dtype=A.dtype)
        t = getattr(self.L, f"ref_multiply_threads_{s}")(c_vp(h2 or h), _p(x), c_i64(x.size), int(nthreads),
                                                         int(reps))
        if h2:
            self.destroy(h2, A.dtype)
        self.destroy(h, A.dtype)
        return t


def reference_available():
    return os.path.exists(REF_SO)
