"""Python mirror of the drop-in GPU path; every call goes through the C ABI
of include/sparkit_b200.h.

Names and argument meaning follow the reference:

* ``Device_matrix(A)`` uploads a Compressed_row_matrix / Ellpack_matrix /
  Jagged_diagonal_matrix / Block_sparse_row_matrix once.
* ``multiply(Ad, x)`` is multiply(A, span<T const>) -> vector<T>
  (sparse_blas.hpp:19, spmv.hpp:119/148/182): host array in, host array out.
* ``jacobi(Ad)``, ``chebyshev_preconditioner(Ad, lmin, lmax, degree)`` are
  the set-up calls of jacobi.hpp:27 and chebyshev_preconditioner.hpp:46;
  ``identity`` (None) is the copy callable of the reference tests.
* ``conjugate_gradient(b, x, cfg, spmv(Ad), left, right)``,
  ``bicgstab(b, x, cfg, spmv(Ad), left, right)`` and
  ``fgmres(b, x, cfg, spmv(Ad), preconditioner)`` mirror
  conjugate_gradient.hpp:347, bicgstab.hpp:391 and fgmres.hpp:459; b and x
  are numpy arrays (x in/out, copied once each way) or CUDA torch tensors
  (device resident, no copies).
"""
import ctypes
from dataclasses import dataclass, field
from typing import List

import numpy as np

from . import _lib
from ._lib import check, lib
from .formats import (Block_sparse_row_matrix, Compressed_row_matrix, Ellpack_matrix,
                      Jagged_diagonal_matrix)

identity = None


def _dtype_code(dt):
    dt = np.dtype(dt)
    if dt == np.float64:
        return _lib.SK_F64
    if dt == np.float32:
        return _lib.SK_F32
    raise TypeError(f"unsupported value type {dt}")


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(ctypes.c_void_p) if a.size else ctypes.c_void_p(a.ctypes.data)
    return ctypes.c_void_p(int(a.data_ptr()))


def _is_device(a):
    return not isinstance(a, np.ndarray) and hasattr(a, "data_ptr")


def _check_vec(a, n, dtype, device, name):
    """Raises unless `a` is a contiguous CUDA torch tensor of `n` values of
    `dtype` on CUDA device `device` (None: any).  The C entry points that
    take device vectors take no length, so a host array, a CPU tensor, a
    short vector or the other precision would otherwise be read or written
    out of bounds by the kernels; this check runs before anything is
    launched."""
    import torch
    if not isinstance(a, torch.Tensor):
        raise TypeError(f"{name} must be a CUDA torch tensor, not {type(a).__name__}")
    want = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
    if a.dtype != want:
        raise TypeError(f"{name} has dtype {a.dtype}; the matrix holds {np.dtype(dtype).name} values")
    if not a.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    if a.numel() != n:
        raise ValueError(f"{name} holds {a.numel()} values; {n} are needed")
    if not a.is_cuda:
        raise ValueError(f"{name} is on {a.device}, not on a CUDA device")
    if device is not None and a.device.index != device:
        raise ValueError(f"{name} is on cuda:{a.device.index}; the matrix is on cuda:{device}")


def _current_device():
    try:
        import torch
        return torch.cuda.current_device() if torch.cuda.is_available() else None
    except Exception:
        return None


CUDA_STREAM_LEGACY = 1  # cudaStreamLegacy


def torch_stream(s=None):
    """The sk_stream of a torch stream (default: the current one).  torch's
    default stream has handle 0, which the C ABI would read as "the
    handle's own stream", so it is passed as cudaStreamLegacy instead."""
    import torch
    s = torch.cuda.current_stream() if s is None else s
    return ctypes.c_void_p(s.cuda_stream if s.cuda_stream else CUDA_STREAM_LEGACY)


def _stream_of(a):
    if _is_device(a):
        import torch
        return torch_stream(torch.cuda.current_stream(a.device))
    return None


class Device_matrix:
    """A device-resident copy of one reference matrix object."""

    def __init__(self, A, dtype=None):
        values = A.values()
        dt = np.dtype(dtype) if dtype is not None else values.dtype
        values = np.ascontiguousarray(values, dtype=dt)
        code = _dtype_code(dt)
        h = ctypes.c_void_p()
        n, m = A.shape()
        if isinstance(A, Compressed_row_matrix):
            check(lib().sk_csr_create(ctypes.byref(h), n, m, _ptr(A.row_ptr()), _ptr(A.col_ind()),
                                      _ptr(values), code))
        elif isinstance(A, Ellpack_matrix):
            check(lib().sk_ell_create(ctypes.byref(h), n, m, A.max_nnz_per_row(), _ptr(A.col_ind()),
                                      _ptr(values), code))
        elif isinstance(A, Jagged_diagonal_matrix):
            perm = A.perm() if A.perm().size else None
            check(lib().sk_jad_create(ctypes.byref(h), n, m, A.num_jdiags(), _ptr(perm), _ptr(A.jdiag()),
                                      _ptr(A.col_ind()), _ptr(values), code))
        elif isinstance(A, Block_sparse_row_matrix):
            check(lib().sk_bsr_create(ctypes.byref(h), n, m, A.block_rows(), A.block_cols(),
                                      _ptr(A.row_ptr()), _ptr(A.col_ind()), _ptr(values), code))
        else:
            raise TypeError(f"no device form for {type(A).__name__}")
        self.handle = h
        self.dtype = dt
        self._shape = (n, m)
        self._block = (A.block_rows(), A.block_cols()) if isinstance(A, Block_sparse_row_matrix) else None
        self.device = _current_device()

    @classmethod
    def _wrap(cls, h, dtype, shape, block=None):
        self = cls.__new__(cls)
        self.handle = h
        self.dtype = np.dtype(dtype)
        self._shape = tuple(shape)
        self._block = block
        self.device = _current_device()
        return self

    def shape(self):
        return self._shape

    def to_host(self):
        """The handle as the reference's host object, read back from the
        device (sk_csr_export / sk_ell_export / sk_jad_export /
        sk_bsr_export)."""
        inf = self.info()
        n, m = self._shape
        fmt, nnz, w = inf["format"], inf["nnz"], inf["width"]
        z = lambda k, dt=np.int64: np.zeros(k, dtype=dt)
        if fmt == 0:
            rp, ci, va = z(n + 1), z(nnz), z(nnz, self.dtype)
            check(lib().sk_csr_export(self.handle, _ptr(rp), _ptr(ci), _ptr(va)))
            return Compressed_row_matrix((n, m), rp, ci, va)
        if fmt == 1:
            ci, va = z(n * w), z(n * w, self.dtype)
            check(lib().sk_ell_export(self.handle, _ptr(ci), _ptr(va)))
            return Ellpack_matrix((n, m), w, ci, va)
        if fmt == 2:
            pm, jd, ci, va = z(n if w else 0), z(w + 1), z(nnz), z(nnz, self.dtype)
            check(lib().sk_jad_export(self.handle, _ptr(pm), _ptr(jd), _ptr(ci), _ptr(va)))
            return Jagged_diagonal_matrix((n, m), pm, jd, ci, va)
        br, bc = self._block
        nbr = (n + br - 1) // br
        rp, ci, va = z(nbr + 1), z(w), z(w * br * bc, self.dtype)
        check(lib().sk_bsr_export(self.handle, _ptr(rp), _ptr(ci), _ptr(va)))
        return Block_sparse_row_matrix((n, m), br, bc, rp, ci, va)

    def info(self):
        """dict of sk_matrix_info: format, dtype, nrow, ncol, nnz, width,
        device_bytes, spmv_bytes (algorithmic bytes of one product)."""
        arr = (ctypes.c_int64 * 8)()
        check(lib().sk_matrix_info(self.handle, arr))
        keys = ("format", "dtype", "nrow", "ncol", "nnz", "width", "device_bytes", "spmv_bytes")
        return dict(zip(keys, list(arr)))

    LAYOUTS = ("native", "sell", "diagonals", "split", "panels")

    def layout(self):
        """The device layout the product runs on (sk_matrix_layout): one of
        LAYOUTS."""
        v = ctypes.c_int32(0)
        check(lib().sk_matrix_layout(self.handle, ctypes.byref(v)))
        return self.LAYOUTS[v.value]

    def build_ms(self):
        """Device time of the kernels that built this handle on the device
        (sk_matrix_build_ms); 0.0 for a handle uploaded from the host."""
        v = ctypes.c_double()
        check(lib().sk_matrix_build_ms(self.handle, ctypes.byref(v)))
        return v.value

    def add_f32_values(self):
        check(lib().sk_matrix_add_f32_values(self.handle))

    def add_panels(self):
        """Adds the column-panel copy of a CSR handle whose rows are too long
        for SELL-32, so that every product sums each row in the reference's
        order (sk_matrix_add_panels); False when the handle does not qualify
        (the handle is then unchanged)."""
        built = ctypes.c_int(0)
        check(lib().sk_matrix_add_panels(self.handle, ctypes.byref(built)))
        return bool(built.value)

    def add_diagonals(self):
        """Adds the diagonal copy of a stencil-pattern CSR handle; False when
        the pattern does not qualify (the handle is then unchanged)."""
        built = ctypes.c_int(0)
        check(lib().sk_matrix_add_diagonals(self.handle, ctypes.byref(built)))
        return bool(built.value)

    def spmv(self, x, y, stream=None):
        """y = A x on device tensors (or raw device pointers, which the
        caller vouches for)."""
        n, m = self._shape
        if not isinstance(x, int):
            _check_vec(x, m, self.dtype, self.device, "x")
        if not isinstance(y, int):
            _check_vec(y, n, self.dtype, self.device, "y")
        xs = _ptr(x) if not isinstance(x, int) else ctypes.c_void_p(x)
        ys = _ptr(y) if not isinstance(y, int) else ctypes.c_void_p(y)
        st = stream if stream is not None else _stream_of(x)
        check(lib().sk_spmv(self.handle, xs, ys, st))

    def spmv_f32(self, x, y, stream=None):
        n, m = self._shape
        _check_vec(x, m, np.float32, self.device, "x")
        _check_vec(y, n, np.float32, self.device, "y")
        st = stream if stream is not None else _stream_of(x)
        check(lib().sk_spmv_f32(self.handle, _ptr(x), _ptr(y), st))

    def close(self):
        if getattr(self, "handle", None) and not _lib.shutting_down():
            lib().sk_matrix_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _convert(fn, Ad, *args, block=None):
    h = ctypes.c_void_p()
    check(fn(ctypes.byref(h), Ad.handle, *args))
    return Device_matrix._wrap(h, Ad.dtype, Ad.shape(), block)


def to_ellpack(Ad):
    """to_ellpack(Compressed_row_matrix) (conversions.hpp:427-467), built on
    the device from a CSR handle: sk_ell_from_csr."""
    return _convert(lib().sk_ell_from_csr, Ad)


def to_jagged_diagonal(Ad):
    """to_jagged_diagonal(Compressed_row_matrix) (conversions.hpp:641-691)
    on the device: sk_jad_from_csr."""
    return _convert(lib().sk_jad_from_csr, Ad)


def to_block_sparse_row(Ad, block_rows, block_cols):
    """to_block_sparse_row(csr, block_rows, block_cols)
    (conversions.hpp:524-577) on the device: sk_bsr_from_csr."""
    return _convert(lib().sk_bsr_from_csr, Ad, int(block_rows), int(block_cols),
                    block=(int(block_rows), int(block_cols)))


def read_matrix_market(source, dtype=np.float64, threads=0):
    """read_matrix_market<T>(path) followed by to_compressed_row
    (matrix_market.hpp:45-115) into a device CSR handle.  `source` is a path,
    or bytes holding the file's text.  Errors raise SkError with the reason."""
    dt = np.dtype(dtype)
    h = ctypes.c_void_p()
    if isinstance(source, (bytes, bytearray)):
        buf = bytes(source)
        check(lib().sk_matrix_market_read_buffer(ctypes.byref(h), buf, len(buf), _dtype_code(dt), int(threads)))
    else:
        check(lib().sk_matrix_market_read(ctypes.byref(h), str(source).encode(), _dtype_code(dt), int(threads)))
    arr = (ctypes.c_int64 * 8)()
    check(lib().sk_matrix_info(h, arr))
    return Device_matrix._wrap(h, dt, (arr[2], arr[3]))


def write_matrix_market(Ad, path, precision=0, threads=0):
    """write_matrix_market(path, A) (matrix_market.hpp:119-150) of a CSR
    handle; precision 0 prints 6 significant digits as the reference does."""
    check(lib().sk_matrix_market_write(Ad.handle, str(path).encode(), int(precision), int(threads)))


def multiply(Ad, x):
    """multiply(A, span<T const>) -> vector<T>, host in / host out."""
    x = np.ascontiguousarray(x, dtype=Ad.dtype)
    if x.shape[0] != Ad.shape()[1]:
        raise ValueError("x length must equal the column count")
    y = np.empty(Ad.shape()[0], dtype=Ad.dtype)
    check(lib().sk_spmv_host(Ad.handle, _ptr(x), _ptr(y)))
    return y


class spmv:
    """The linear-operator argument of the solvers: y = A x on the device."""

    def __init__(self, Ad):
        self.A = Ad


class _Precond:
    def __init__(self, handle, Ad, n):
        self.handle = handle
        self.A = Ad
        self.n = n

    def apply(self, r, z, stream=None):
        """z = M^{-1} r on device tensors."""
        _check_vec(r, self.n, self.A.dtype, self.A.device, "r")
        _check_vec(z, self.n, self.A.dtype, self.A.device, "z")
        st = stream if stream is not None else _stream_of(r)
        check(lib().sk_precond_apply(self.handle, self.n, _ptr(r), _ptr(z), st))

    def values(self):
        cnt = ctypes.c_int64()
        check(lib().sk_precond_values(self.handle, None, 0, ctypes.byref(cnt)))
        out = np.empty(cnt.value, dtype=self.A.dtype)
        check(lib().sk_precond_values(self.handle, _ptr(out), cnt.value, ctypes.byref(cnt)))
        return out

    def close(self):
        if getattr(self, "handle", None) and not _lib.shutting_down():
            lib().sk_precond_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class jacobi(_Precond):
    """jacobi(A) (jacobi.hpp:27-35).  A zero diagonal raises ValueError,
    the Python form of the reference's std::invalid_argument."""

    def __init__(self, Ad):
        h = ctypes.c_void_p()
        st = lib().sk_jacobi_create(ctypes.byref(h), Ad.handle)
        if st == 8:  # SK_ZERO_DIAGONAL
            raise ValueError("jacobi: zero diagonal entry")
        check(st)
        super().__init__(h, Ad, min(Ad.shape()))


class chebyshev_preconditioner(_Precond):
    """chebyshev_preconditioner(A, lambda_min, lambda_max, degree)
    (chebyshev_preconditioner.hpp:46-84)."""

    def __init__(self, Ad, lambda_min, lambda_max, degree):
        h = ctypes.c_void_p()
        check(lib().sk_chebyshev_create(ctypes.byref(h), Ad.handle, float(lambda_min), float(lambda_max),
                                        int(degree)))
        super().__init__(h, Ad, Ad.shape()[0])
        self.lambda_min, self.lambda_max, self.degree = lambda_min, lambda_max, degree


class chebyshev_preconditioner_auto(chebyshev_preconditioner):
    """chebyshev_preconditioner(A, lambda_min, lambda_max, degree) with the
    bounds from estimate_eigenvalue_bounds(A, num_iter) (conditioning.hpp:132),
    computed on the device (sk_chebyshev_create_auto)."""

    def __init__(self, Ad, degree, num_iter=30):
        h = ctypes.c_void_p()
        b = np.zeros(2)
        check(lib().sk_chebyshev_create_auto(ctypes.byref(h), Ad.handle, int(degree), int(num_iter), _ptr(b)))
        _Precond.__init__(self, h, Ad, Ad.shape()[0])
        self.lambda_min, self.lambda_max, self.degree = float(b[0]), float(b[1]), degree


# Eigen_target (eigen_target.hpp:13-20)
EIGEN_TARGETS = ("largest_magnitude", "smallest_magnitude", "largest_algebraic", "smallest_algebraic",
                 "largest_real", "smallest_real")


def lanczos(Ad, nev=1, m=20, tol=1e-10, max_restarts=10, target="largest_algebraic", collect=False,
            vectors=False):
    """lanczos(n, Lanczos_config, multiply(A)) (lanczos.hpp:495-503) on the
    device: a dict of the Lanczos_result fields (eigenvectors as a device
    tensor of shape (count, n) when vectors=True)."""
    import torch
    n = Ad.shape()[0]
    cfg = _lib.LanczosConfig(int(nev), int(m), float(tol), int(max_restarts), EIGEN_TARGETS.index(target),
                             int(collect))
    ev = np.zeros(max(int(nev), 1))
    res = np.zeros(max(int(nev), 1))
    rr = np.zeros(int(max_restarts) + 2)
    vecs = torch.zeros((max(int(nev), 1), n), dtype=torch.float64 if Ad.dtype == np.float64 else torch.float32,
                       device="cuda") if vectors else None
    out = _lib.LanczosSummary()
    st = _stream_of(vecs) if vecs is not None else None
    check(lib().sk_lanczos(Ad.handle, ctypes.byref(cfg), _ptr(ev), _ptr(res), _ptr(rr),
                           _ptr(vecs) if vecs is not None else None, ctypes.byref(out), st))
    d = dict(eigenvalues=ev[: out.count].astype(Ad.dtype), residual_norms=res[: out.residual_count].astype(Ad.dtype),
             restart_residuals=rr[: out.restart_residuals_count], computed_restarts=out.computed_restarts,
             converged_count=out.converged_count, converged=bool(out.converged))
    if vecs is not None:
        d["eigenvectors"] = vecs[: out.count]
    return d


def estimate_spectral_radius(Ad, num_iter=20):
    """estimate_spectral_radius(n, multiply(A), num_iter) (conditioning.hpp:112)."""
    v = ctypes.c_double()
    check(lib().sk_spectral_radius(Ad.handle, int(num_iter), ctypes.byref(v)))
    return v.value


def estimate_eigenvalue_bounds(Ad, num_iter=30):
    """estimate_eigenvalue_bounds(n, multiply(A), num_iter)
    (conditioning.hpp:132): (lambda_min, lambda_max)."""
    lo, hi = ctypes.c_double(), ctypes.c_double()
    check(lib().sk_eigenvalue_bounds(Ad.handle, int(num_iter), ctypes.byref(lo), ctypes.byref(hi)))
    return lo.value, hi.value


SUM_TREE, SUM_SEQUENTIAL = 0, 1


def set_summation_order(order):
    """sk_set_summation_order: SUM_TREE (default, fast, deterministic) or
    SUM_SEQUENTIAL (the reference's element-order sums, for validation)."""
    check(lib().sk_set_summation_order(int(order)))


def summation_order():
    v = ctypes.c_int32()
    check(lib().sk_get_summation_order(ctypes.byref(v)))
    return v.value


def debug_set_wait(limit_ns=0, unmeetable=False):
    """sk_debug_set_wait: the time bound of the persistent kernels'
    grid-barrier waits (0 restores 2 s) and, for tests of the timeout path,
    barriers that wait for one arrival more than the grid makes."""
    check(lib().sk_debug_set_wait(int(limit_ns), int(bool(unmeetable))))


def chebyshev_apply_noalloc(Ad, lambda_min, lambda_max, degree, r, z, stream=None):
    """z = p(A) r like chebyshev_preconditioner(Ad, ...).apply(r, z), for
    callers that cannot allocate device memory at apply time: no handle is
    created and the work vectors live in the library's static device array
    (square CSR, at most 1,048,576 rows, degree <= 64; overlapping calls on
    the GPU race; the first call on a device should precede any stream
    capture).  r and z must be contiguous CUDA tensors of n values of the
    matrix's value type on its device; anything else raises before a launch."""
    n = Ad.shape()[0]
    _check_vec(r, n, Ad.dtype, Ad.device, "r")
    _check_vec(z, n, Ad.dtype, Ad.device, "z")
    st = stream if stream is not None else _stream_of(r)
    check(lib().sk_chebyshev_apply_noalloc(Ad.handle, float(lambda_min), float(lambda_max), int(degree),
                                           _ptr(r), _ptr(z), st))


@dataclass
class CGConfig:
    """CGConfig<T> (conjugate_gradient.hpp:48-74)."""
    tolerance: float = 0.0
    restart_iterations: int = 0
    max_iterations: int = 0
    collect_residuals: bool = False


@dataclass
class Bicgstab_config:
    """Bicgstab_config<T> (bicgstab.hpp:25-42)."""
    tolerance: float = 0.0
    max_iterations: int = 0
    collect_residuals: bool = False


@dataclass
class Fgmres_config:
    """Fgmres_config<T> (fgmres.hpp:25-47)."""
    tolerance: float = 0.0
    restart_dimension: int = 0
    max_iterations: int = 0
    collect_residuals: bool = False


@dataclass
class Summary:
    """CGSummary / Bicgstab_summary / Fgmres_summary, plus the device
    status (0, or 4 = SK_BREAKDOWN)."""
    residual_norm: float = 0.0
    computed_iterations: int = 0
    converged: bool = False
    iteration_residuals: List[float] = field(default_factory=list)
    status: int = 0


CGSummary = Bicgstab_summary = Fgmres_summary = Summary


def _handle(M):
    return None if M is None else M.handle


def _run(fn_dev, fn_host, b, x, Ad, cfg_struct, max_hist, collect):
    s = _lib.Summary()
    hist = np.zeros(max(int(max_hist), 1) + 4, dtype=np.float64) if collect else None
    if _is_device(b):
        n = Ad.shape()[0]
        _check_vec(b, n, Ad.dtype, Ad.device, "b")
        _check_vec(x, n, Ad.dtype, Ad.device, "x")
        st = _stream_of(b)
        check(fn_dev(_ptr(b), _ptr(x), ctypes.byref(cfg_struct), ctypes.byref(s), _ptr(hist), st))
    else:
        if not (isinstance(x, np.ndarray) and x.flags.c_contiguous and x.dtype == Ad.dtype):
            raise TypeError("x must be a contiguous numpy array of the matrix's value type")
        bb = np.ascontiguousarray(b, dtype=Ad.dtype)
        n = Ad.shape()[0]
        if bb.shape != (n,) or x.shape != (n,):
            raise ValueError(f"b and x must hold {n} values (got {bb.shape} and {x.shape})")
        check(fn_host(_ptr(bb), _ptr(x), ctypes.byref(cfg_struct), ctypes.byref(s), _ptr(hist)))
    out = Summary(s.residual_norm, s.computed_iterations, bool(s.converged), [], s.status)
    if collect:
        out.iteration_residuals = hist[: s.history_length].tolist()
    return out


def _op_matrix(op):
    if not isinstance(op, spmv):
        raise TypeError("the linear operator must be sparkit_b200.gpu.spmv(Device_matrix): "
                        "arbitrary host callables are not accelerated")
    return op.A


def conjugate_gradient(b, x, cfg, op, left=identity, right=identity):
    """conjugate_gradient(bfirst, blast, xfirst, xlast, cfg, op, left, right)."""
    Ad = _op_matrix(op)
    c = _lib.CgConfig(cfg.tolerance, cfg.restart_iterations, cfg.max_iterations, int(cfg.collect_residuals))
    L = lib()
    return _run(lambda bp, xp, cp, sp, hp, st: L.sk_cg_solve(Ad.handle, _handle(left), _handle(right), bp, xp,
                                                             cp, sp, hp, st),
                lambda bp, xp, cp, sp, hp: L.sk_cg_solve_host(Ad.handle, _handle(left), _handle(right), bp, xp,
                                                              cp, sp, hp),
                b, x, Ad, c, cfg.max_iterations, cfg.collect_residuals)


def bicgstab(b, x, cfg, op, left=identity, right=identity):
    """bicgstab(bfirst, blast, xfirst, xlast, cfg, op, left, right)."""
    Ad = _op_matrix(op)
    c = _lib.BicgstabConfig(cfg.tolerance, cfg.max_iterations, int(cfg.collect_residuals))
    L = lib()
    return _run(lambda bp, xp, cp, sp, hp, st: L.sk_bicgstab_solve(Ad.handle, _handle(left), _handle(right), bp,
                                                                   xp, cp, sp, hp, st),
                lambda bp, xp, cp, sp, hp: L.sk_bicgstab_solve_host(Ad.handle, _handle(left), _handle(right),
                                                                    bp, xp, cp, sp, hp),
                b, x, Ad, c, cfg.max_iterations + 2, cfg.collect_residuals)


@dataclass
class Cgs_config:
    """Cgs_config<T> (cgs.hpp:25-42)."""
    tolerance: float = 0.0
    max_iterations: int = 0
    collect_residuals: bool = False


@dataclass
class Minres_config:
    """Minres_config<T> (minres.hpp:25-45)."""
    tolerance: float = 0.0
    max_iterations: int = 0
    collect_residuals: bool = False


def _krylov2(name, b, x, cfg, op, left, right, max_hist):
    Ad = _op_matrix(op)
    c = _lib.BicgstabConfig(cfg.tolerance, cfg.max_iterations, int(cfg.collect_residuals))
    L = lib()
    dev, host = getattr(L, f"sk_{name}_solve"), getattr(L, f"sk_{name}_solve_host")
    return _run(lambda bp, xp, cp, sp, hp, st: dev(Ad.handle, _handle(left), _handle(right), bp, xp, cp, sp, hp, st),
                lambda bp, xp, cp, sp, hp: host(Ad.handle, _handle(left), _handle(right), bp, xp, cp, sp, hp),
                b, x, Ad, c, max_hist, cfg.collect_residuals)


def cgs(b, x, cfg, op, left=identity, right=identity):
    """cgs(bfirst, blast, xfirst, xlast, cfg, op, left, right)."""
    return _krylov2("cgs", b, x, cfg, op, left, right, cfg.max_iterations // 2 + 4)


def minres(b, x, cfg, op, left=identity, right=identity):
    """minres(bfirst, blast, xfirst, xlast, cfg, op, left, right)."""
    return _krylov2("minres", b, x, cfg, op, left, right, cfg.max_iterations + 2)


def fgmres(b, x, cfg, op, preconditioner=identity):
    """fgmres(bfirst, blast, xfirst, xlast, cfg, op, preconditioner)."""
    Ad = _op_matrix(op)
    c = _lib.FgmresConfig(cfg.tolerance, cfg.restart_dimension, cfg.max_iterations, int(cfg.collect_residuals))
    L = lib()
    return _run(lambda bp, xp, cp, sp, hp, st: L.sk_fgmres_solve(Ad.handle, _handle(preconditioner), bp, xp, cp,
                                                                 sp, hp, st),
                lambda bp, xp, cp, sp, hp: L.sk_fgmres_solve_host(Ad.handle, _handle(preconditioner), bp, xp,
                                                                  cp, sp, hp),
                b, x, Ad, c, cfg.max_iterations, cfg.collect_residuals)


@dataclass
class Gmres_config:
    """Gmres_config<T> (gmres.hpp:25-47)."""
    tolerance: float = 0.0
    restart_dimension: int = 0
    max_iterations: int = 0
    collect_residuals: bool = False


def gmres(b, x, cfg, op, left=identity, right=identity):
    """gmres(bfirst, blast, xfirst, xlast, cfg, op, left, right)."""
    Ad = _op_matrix(op)
    c = _lib.FgmresConfig(cfg.tolerance, cfg.restart_dimension, cfg.max_iterations, int(cfg.collect_residuals))
    L = lib()
    return _run(lambda bp, xp, cp, sp, hp, st: L.sk_gmres_solve(Ad.handle, _handle(left), _handle(right), bp, xp,
                                                                cp, sp, hp, st),
                lambda bp, xp, cp, sp, hp: L.sk_gmres_solve_host(Ad.handle, _handle(left), _handle(right), bp, xp,
                                                                 cp, sp, hp),
                b, x, Ad, c, cfg.max_iterations, cfg.collect_residuals)


@dataclass
class Mixed_config:
    """FP32-inner / FP64-outer iterative refinement (sk_mixed_cg_solve)."""
    tolerance: float = 1e-10
    inner_tolerance: float = 1e-5
    max_outer: int = 100
    max_inner: int = 100000
    collect_residuals: bool = False
    adaptive_last_step: bool = True
    l2_window: bool = True
    persistent: bool = True      # one cooperative launch per inner solve


@dataclass
class Mixed_summary:
    residual_norm: float = 0.0
    outer_iterations: int = 0
    inner_iterations: int = 0
    converged: bool = False
    status: int = 0
    residual_history: List[float] = field(default_factory=list)
    setup_ms: float = 0.0
    inner_ms: float = 0.0
    outer_ms: float = 0.0
    persistent: bool = False


def mixed_cg(b, x, cfg, op, jacobi_inner=True):
    """Solves A x = b to cfg.tolerance on the true FP64 residual with FP32
    CG inner solves (Jacobi-preconditioned unless jacobi_inner is False).
    b and x are FP64 CUDA tensors (x holds the initial guess)."""
    Ad = _op_matrix(op)
    c = _lib.MixedConfig(cfg.tolerance, cfg.inner_tolerance, cfg.max_outer, cfg.max_inner,
                         int(cfg.collect_residuals), int(cfg.adaptive_last_step), int(cfg.l2_window),
                         0 if cfg.persistent else 1)
    s = _lib.MixedSummary()
    hist = np.zeros(cfg.max_outer + 2) if cfg.collect_residuals else None
    n = Ad.shape()[0]
    _check_vec(b, n, np.float64, Ad.device, "b")
    _check_vec(x, n, np.float64, Ad.device, "x")
    check(lib().sk_mixed_cg_solve(Ad.handle, int(jacobi_inner), _ptr(b), _ptr(x), ctypes.byref(c), ctypes.byref(s),
                                  _ptr(hist), _stream_of(b)))
    out = Mixed_summary(s.residual_norm, s.outer_iterations, s.inner_iterations, bool(s.converged), s.status,
                        [], s.setup_ms, s.inner_ms, s.outer_ms, s.inner_kernel == 0)
    if hist is not None:
        out.residual_history = hist[: s.outer_iterations + 1].tolist()
    return out


@dataclass
class Mixed_fgmres_config:
    """FP32-inner FGMRES(m) / FP64-outer iterative refinement
    (sk_mixed_fgmres_solve)."""
    tolerance: float = 1e-10
    inner_tolerance: float = 1e-4
    restart_dimension: int = 30
    max_outer: int = 50
    max_inner: int = 3000
    collect_residuals: bool = False
    adaptive_last_step: bool = True


def mixed_fgmres(b, x, cfg, op, preconditioner=identity):
    """Solves A x = b to cfg.tolerance on the true FP64 residual with FP32
    FGMRES(m) inner solves whose Hessenberg least-squares problem runs in
    FP64.  b and x are FP64 CUDA tensors (x holds the initial guess)."""
    Ad = _op_matrix(op)
    n = Ad.shape()[0]
    _check_vec(b, n, np.float64, Ad.device, "b")
    _check_vec(x, n, np.float64, Ad.device, "x")
    c = _lib.MixedFgmresConfig(cfg.tolerance, cfg.inner_tolerance, cfg.restart_dimension, cfg.max_outer,
                               cfg.max_inner, int(cfg.collect_residuals), int(cfg.adaptive_last_step))
    s = _lib.MixedSummary()
    hist = np.zeros(cfg.max_outer + 2) if cfg.collect_residuals else None
    check(lib().sk_mixed_fgmres_solve(Ad.handle, _handle(preconditioner), _ptr(b), _ptr(x), ctypes.byref(c),
                                      ctypes.byref(s), _ptr(hist), _stream_of(b)))
    out = Mixed_summary(s.residual_norm, s.outer_iterations, s.inner_iterations, bool(s.converged), s.status,
                        [], s.setup_ms, s.inner_ms, s.outer_ms, False)
    if hist is not None:
        out.residual_history = hist[: s.outer_iterations + 1].tolist()
    return out


# ------------------------------------------------------------------
# Learned variable preconditioner of FGMRES (no reference counterpart:
# fgmres.hpp:452-470 takes any callable as its variable preconditioner)
# ------------------------------------------------------------------

class Net:
    """The convolutional encoder-decoder of the learned preconditioner
    (sk_net_create): seeded He initialisation, FP32 master weights, BF16
    copies for the tensor-core convolutions."""

    def __init__(self, seed=0):
        h = ctypes.c_void_p()
        check(lib().sk_net_create(ctypes.byref(h), int(seed)))
        self.handle = h

    @staticmethod
    def param_count():
        return int(lib().sk_net_param_count())

    def params(self):
        out = np.empty(self.param_count(), dtype=np.float32)
        check(lib().sk_net_get_params(self.handle, _ptr(out), out.size))
        return out

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().sk_net_set_params(self.handle, _ptr(p), p.size))

    def set_legacy_mma(self, on):
        """Test hook: the convolutions on mma.sync instead of tcgen05."""
        check(lib().sk_net_set_legacy_mma(self.handle, int(bool(on))))

    def loss_grad(self, pairs, idx, mu=0.0):
        """Loss of the batch of pair indices `idx` and its FP32 gradient."""
        idx = np.ascontiguousarray(idx, dtype=np.int32)
        loss = ctypes.c_double()
        g = np.empty(self.param_count(), dtype=np.float32)
        check(lib().sk_net_loss_grad(self.handle, pairs.handle, _ptr(idx), idx.size, float(mu), ctypes.byref(loss),
                                     _ptr(g), g.size))
        return loss.value, g

    def train(self, pairs, cfg):
        c = _lib.TrainConfig(cfg.steps, cfg.batch, cfg.lr, cfg.lr_final_ratio, cfg.beta1, cfg.beta2, cfg.eps,
                             cfg.mu, cfg.seed)
        s = _lib.TrainSummary()
        hist = np.zeros(max(cfg.steps, 1))
        check(lib().sk_net_train(self.handle, pairs.handle, ctypes.byref(c), ctypes.byref(s), _ptr(hist)))
        return Train_summary(s.first_loss, s.last_loss, s.ms, s.steps, hist[: s.steps].tolist())

    def close(self):
        if getattr(self, "handle", None) and not _lib.shutting_down():
            lib().sk_net_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Pairs:
    """(residual, error) training pairs on an nx x ny grid (sk_pairs_*)."""

    def __init__(self, nx, ny, capacity, max_instances):
        h = ctypes.c_void_p()
        check(lib().sk_pairs_create(ctypes.byref(h), int(nx), int(ny), int(capacity), int(max_instances)))
        self.handle, self.nx, self.ny = h, nx, ny

    def add_instance(self, Ad):
        i = ctypes.c_int32()
        check(lib().sk_pairs_add_instance(self.handle, Ad.handle, ctypes.byref(i)))
        return i.value

    def add(self, instance, r, e):
        check(lib().sk_pairs_add(self.handle, int(instance), _ptr(r), _ptr(e), _stream_of(r)))

    def harvest(self, instance, Ad, b, xstar, restart=30, cycles=100):
        """Pairs from the plain Jacobi-FGMRES(restart) run on Ad x = b from
        x = 0, one per restart cycle (b, xstar: FP64 CUDA tensors)."""
        n = ctypes.c_int64()
        check(lib().sk_learned_harvest(self.handle, int(instance), Ad.handle, _ptr(b), _ptr(xstar), int(restart),
                                       int(cycles), ctypes.byref(n)))
        return n.value

    def __len__(self):
        n = ctypes.c_int64()
        check(lib().sk_pairs_count(self.handle, ctypes.byref(n)))
        return n.value

    def close(self):
        if getattr(self, "handle", None) and not _lib.shutting_down():
            lib().sk_pairs_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def train_coarse_corrected_smoother(m, instances=200, held=10, cycles=40, steps=8000, agg=8, seed=1):
    """A network for the smoother of the two-level form (twolevel(...,
    coarse_first=True)), which only sees coarse-corrected residuals.  Pairs:
    on `instances` + `held` seeded m^2 convection-diffusion instances
    (matgen.convdiff_2d_grf), FGMRES(30) restart cycles from x = 0 (Jacobi,
    or on every third instance the coarse correction alone), after each
    cycle r = b - A x and e = x* - x moved past the coarse correction
    c = P Ac^-1 P^T r (aggregates of agg x agg cells): (r - A c, e - c).
    Returns the trained Net and a summary with the held-out loss (the last
    `held` instances' pairs) before and after training."""
    import time

    import numpy as np
    import torch

    from . import matgen
    pairs = Pairs(m, m, (instances + held) * cycles, instances + held)
    t0 = time.perf_counter()
    held_idx = []
    for k in range(instances + held):
        Am = matgen.convdiff_2d_grf(m, seed=100 + k)[0]
        Amd = Device_matrix(Am)
        inst = pairs.add_instance(Amd)
        xs = np.random.default_rng(k).uniform(-1, 1, m * m) if k % 2 == 0 else \
            matgen.gaussian_random_field((m, m), 1.0, m / 16, seed=k).ravel()
        xsd = torch.from_numpy(xs).cuda()
        b = torch.empty_like(xsd)
        Amd.spmv(xsd, b)
        J = jacobi(Amd)
        C = twolevel(Amd, None, m, m, agg)
        x = torch.zeros_like(b)
        r = torch.empty_like(b)
        z = torch.empty_like(b)
        az = torch.empty_like(b)
        for _ in range(cycles):
            fgmres(b, x, Fgmres_config(1e-14, 30, 30), spmv(Amd), C if k % 3 == 0 else J)
            Amd.spmv(x, r)
            r = b - r
            C.apply(r, z)
            Amd.spmv(z, az)
            if k >= instances:
                held_idx.append(len(pairs))
            pairs.add(inst, (r - az).contiguous(), (xsd - x - z).contiguous())
        Amd.close()
    torch.cuda.synchronize()
    harvest_s = time.perf_counter() - t0
    net = Net(seed=seed)
    idx = np.array(held_idx, dtype=np.int32)

    def held_loss():
        return float(np.mean([net.loss_grad(pairs, idx[i:i + 8], mu=1.0)[0] for i in range(0, len(idx), 8)]))

    before = held_loss()
    ts = net.train(pairs, Train_config(steps=steps, batch=8, lr=2e-3, mu=1.0, seed=3))
    h = np.array(ts.loss_history)
    info = {"pairs": len(pairs), "held_out_pairs": len(held_idx), "grid": m, "aggregates": agg,
            "harvest_s": harvest_s, "steps": steps, "batch": 8, "train_ms": ts.ms,
            "loss_first20": float(h[:20].mean()), "loss_last50": float(h[-50:].mean()),
            "held_out_loss_before": before, "held_out_loss_after": held_loss()}
    pairs.close()
    return net, info


@dataclass
class Train_config:
    steps: int = 1000
    batch: int = 4
    lr: float = 1e-3
    lr_final_ratio: float = 0.1
    beta1: float = 0.9
    beta2: float = 0.999
    eps: float = 1e-8
    mu: float = 0.0
    seed: int = 0


@dataclass
class Train_summary:
    first_loss: float
    last_loss: float
    ms: float
    steps: int
    loss_history: List[float] = field(default_factory=list)


class learned_preconditioner(_Precond):
    """The trained network as the variable preconditioner of the FP64 CSR
    5-point matrix Ad on an nx x ny grid (row y * nx + x)."""

    def __init__(self, Ad, net, nx, ny):
        h = ctypes.c_void_p()
        check(lib().sk_learned_create(ctypes.byref(h), Ad.handle, net.handle, int(nx), int(ny)))
        super().__init__(h, Ad, Ad.shape()[0])
        self.net = net  # keeps the network alive

    def planes(self):
        out = np.empty(6 * self.n, dtype=np.float32)
        check(lib().sk_learned_planes(self.handle, _ptr(out), out.size))
        return out.reshape(6, self.n)


class twolevel(_Precond):
    """Smoother plus an exact coarse-grid correction (sk_twolevel_create),
    P piecewise constant over agg x agg aggregates of the nx x ny grid and
    Ac = P^T A P:
      default:           z = S(r); z += P Ac^-1 P^T (r - A z)
                         [post_smooth: z += S(r - A z)]
      coarse_first:      z = P Ac^-1 P^T r; z += S(r - A z)
    `smoother` is a jacobi, chebyshev_preconditioner or
    learned_preconditioner of the same matrix, or None (coarse only)."""

    def __init__(self, Ad, smoother, nx, ny, agg, post_smooth=False, coarse_first=False):
        h = ctypes.c_void_p()
        flags = (1 if post_smooth else 0) | (2 if coarse_first else 0)
        check(lib().sk_twolevel_create(ctypes.byref(h), Ad.handle, smoother.handle if smoother else None, int(nx),
                                       int(ny), int(agg), flags))
        super().__init__(h, Ad, Ad.shape()[0])
        self.smoother = smoother  # keeps the smoother alive


def fgmres_fallback(b, x, cfg, op, preconditioner, fallback, stall_ratio=0.9):
    """fgmres with a variable preconditioner and an automatic fallback:
    after a restart cycle whose residual estimate stays above stall_ratio
    times its start, the rest of the solve uses `fallback`.  b, x: FP64
    CUDA tensors.  Returns (Summary, first cycle on the fallback or -1)."""
    Ad = _op_matrix(op)
    c = _lib.FgmresConfig(cfg.tolerance, cfg.restart_dimension, cfg.max_iterations, int(cfg.collect_residuals))
    s = _lib.Summary()
    sw = ctypes.c_int64()
    hist = np.zeros(max(cfg.max_iterations, 1)) if cfg.collect_residuals else None
    check(lib().sk_fgmres_fallback_solve(Ad.handle, _handle(preconditioner), _handle(fallback), _ptr(b), _ptr(x),
                                         ctypes.byref(c), float(stall_ratio), ctypes.byref(s), _ptr(hist),
                                         ctypes.byref(sw), _stream_of(b)))
    out = Summary(s.residual_norm, s.computed_iterations, bool(s.converged), [], s.status)
    if hist is not None:
        out.iteration_residuals = hist[: s.history_length].tolist()
    return out, sw.value


@dataclass
class Batch_config:
    """Settings of sk_batched_cg_solve."""
    tolerance: float = 1e-10
    inner_tolerance: float = 1e-5
    max_outer: int = 30
    max_inner: int = 20000
    adaptive_last_step: bool = True
    lanes_per_row: int = 1
    threads_per_cta: int = 512


class Batch:
    """Many independent SPD systems (the diagonal blocks of one FP32 CSR
    matrix) solved together on the device: one persistent launch, one CTA
    per system, FP32 Jacobi-CG inside FP64 iterative refinement."""

    def __init__(self, sys_offsets, row_ptr, col_ind, values):
        sys_offsets = np.ascontiguousarray(sys_offsets, dtype=np.int64)
        row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int64)
        col_ind = np.ascontiguousarray(col_ind, dtype=np.int64)
        values = np.ascontiguousarray(values, dtype=np.float32)
        h = ctypes.c_void_p()
        check(lib().sk_batch_create(ctypes.byref(h), sys_offsets.size - 1, _ptr(sys_offsets), _ptr(row_ptr),
                                    _ptr(col_ind), _ptr(values)))
        self.handle = h
        self.nsys = sys_offsets.size - 1
        self.nrow = int(sys_offsets[-1])
        self._res = None

    def _results(self):
        import torch
        if self._res is None:
            n = self.nsys
            self._res = (torch.zeros(n, dtype=torch.int32, device="cuda"), torch.zeros(n, dtype=torch.int32, device="cuda"),
                         torch.zeros(n, dtype=torch.float64, device="cuda"), torch.zeros(n, dtype=torch.int32, device="cuda"))
        t = self._res
        return _lib.BatchResults(_ptr(t[0]), _ptr(t[1]), _ptr(t[2]), _ptr(t[3])), t

    @staticmethod
    def _cfg(c):
        return _lib.BatchConfig(c.tolerance, c.inner_tolerance, c.max_outer, c.max_inner, int(c.adaptive_last_step),
                                c.lanes_per_row, c.threads_per_cta)

    def autotune(self, b, x, cfg=None, sample=512):
        """Times every (lanes_per_row, threads_per_cta) variant on the
        `sample` largest systems; returns (lanes, threads, timings_ms)."""
        cfg = cfg or Batch_config()
        res, _ = self._results()
        g, t = ctypes.c_int32(), ctypes.c_int32()
        nvar = lib().sk_batched_variant_count()
        ms = np.zeros(nvar)
        check(lib().sk_batched_autotune(self.handle, _ptr(b), _ptr(x), ctypes.byref(self._cfg(cfg)), ctypes.byref(res),
                                        int(sample), ctypes.byref(g), ctypes.byref(t), _ptr(ms)))
        return g.value, t.value, ms

    def solve(self, b, x, cfg=None):
        """Solves all systems; returns per-system numpy arrays
        (inner_iterations, outer_iterations, relative_residual, converged)."""
        cfg = cfg or Batch_config()
        res, t = self._results()
        check(lib().sk_batched_cg_solve(self.handle, _ptr(b), _ptr(x), ctypes.byref(self._cfg(cfg)),
                                        ctypes.byref(res), _stream_of(b)))
        return tuple(a.cpu().numpy() for a in t)

    def close(self):
        if getattr(self, "handle", None) and not _lib.shutting_down():
            lib().sk_batch_destroy(self.handle)
        self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def device_count():
    n = ctypes.c_int()
    check(lib().sk_device_count(ctypes.byref(n)))
    return n.value
