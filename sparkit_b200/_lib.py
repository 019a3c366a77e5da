"""ctypes binding of the C ABI in include/sparkit_b200.h.

Loads the in-tree ``libsparkit_b200.so``.  There is no fallback: if the
library is missing or cannot load, every entry point raises.
"""
import atexit
import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libsparkit_b200.so")

c_i64 = ctypes.c_int64
c_i32 = ctypes.c_int32
c_dbl = ctypes.c_double
c_vp = ctypes.c_void_p
P_i64 = ctypes.POINTER(ctypes.c_int64)

SK_OK = 0
STATUS_NAMES = {
    0: "SK_OK", 1: "SK_INVALID_ARG", 2: "SK_INDEX_OVERFLOW", 3: "SK_OUT_OF_MEMORY",
    4: "SK_BREAKDOWN", 5: "SK_NOT_CONVERGED", 6: "SK_TIMEOUT", 7: "SK_CUDA_ERROR",
    8: "SK_ZERO_DIAGONAL", 9: "SK_NOT_SUPPORTED", 10: "SK_NO_DEVICE",
}
SK_F64, SK_F32 = 0, 1
SK_CSR, SK_ELL, SK_JAD, SK_BSR = 0, 1, 2, 3


class SkError(RuntimeError):
    """A failed C-ABI call: .status holds the sk_status code."""

    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class CgConfig(ctypes.Structure):
    _fields_ = [("tolerance", c_dbl), ("restart_iterations", c_i64),
                ("max_iterations", c_i64), ("collect_residuals", c_i32)]


class BicgstabConfig(ctypes.Structure):
    _fields_ = [("tolerance", c_dbl), ("max_iterations", c_i64), ("collect_residuals", c_i32)]


class FgmresConfig(ctypes.Structure):
    _fields_ = [("tolerance", c_dbl), ("restart_dimension", c_i64),
                ("max_iterations", c_i64), ("collect_residuals", c_i32)]


class MixedConfig(ctypes.Structure):
    _fields_ = [("tolerance", c_dbl), ("inner_tolerance", c_dbl), ("max_outer", c_i64),
                ("max_inner", c_i64), ("collect_residuals", c_i32), ("adaptive_last_step", c_i32),
                ("l2_window", c_i32), ("inner_kernel", c_i32)]


class MixedFgmresConfig(ctypes.Structure):
    _fields_ = [("tolerance", c_dbl), ("inner_tolerance", c_dbl), ("restart_dimension", c_i64),
                ("max_outer", c_i64), ("max_inner", c_i64), ("collect_residuals", c_i32),
                ("adaptive_last_step", c_i32)]


class MixedSummary(ctypes.Structure):
    _fields_ = [("residual_norm", c_dbl), ("outer_iterations", c_i64), ("inner_iterations", c_i64),
                ("converged", c_i32), ("status", c_i32), ("setup_ms", c_dbl), ("inner_ms", c_dbl),
                ("outer_ms", c_dbl), ("inner_kernel", c_i32)]


class TrainConfig(ctypes.Structure):
    _fields_ = [("steps", c_i64), ("batch", c_i32), ("lr", ctypes.c_float), ("lr_final_ratio", ctypes.c_float),
                ("beta1", ctypes.c_float), ("beta2", ctypes.c_float), ("eps", ctypes.c_float), ("mu", c_dbl),
                ("seed", ctypes.c_uint64)]


class TrainSummary(ctypes.Structure):
    _fields_ = [("first_loss", c_dbl), ("last_loss", c_dbl), ("ms", c_dbl), ("steps", c_i64)]


class BatchConfig(ctypes.Structure):
    _fields_ = [("tolerance", c_dbl), ("inner_tolerance", c_dbl), ("max_outer", c_i64), ("max_inner", c_i64),
                ("adaptive_last_step", c_i32), ("lanes_per_row", c_i32), ("threads_per_cta", c_i32)]


class BatchResults(ctypes.Structure):
    _fields_ = [("inner_iterations", c_vp), ("outer_iterations", c_vp), ("relative_residual", c_vp),
                ("converged", c_vp)]


class Summary(ctypes.Structure):
    _fields_ = [("residual_norm", c_dbl), ("computed_iterations", c_i64),
                ("converged", c_i32), ("status", c_i32), ("history_length", c_i64)]


class LanczosConfig(ctypes.Structure):
    _fields_ = [("num_eigenvalues", c_i64), ("krylov_dimension", c_i64), ("tolerance", c_dbl),
                ("max_restarts", c_i64), ("target", c_i32), ("collect_residuals", c_i32)]


class LanczosSummary(ctypes.Structure):
    _fields_ = [("count", c_i64), ("computed_restarts", c_i64), ("converged_count", c_i64),
                ("residual_count", c_i64), ("restart_residuals_count", c_i64), ("converged", c_i32),
                ("status", c_i32)]


# (name, argtypes) of every exported function, in header order.
SIGNATURES = [
    ("sk_version", []),
    ("sk_last_error", []),
    ("sk_device_count", [ctypes.POINTER(ctypes.c_int)]),
    ("sk_launch_count", [P_i64]),
    ("sk_debug_set_wait", [ctypes.c_uint64, ctypes.c_int32]),
    ("sk_set_summation_order", [ctypes.c_int32]),
    ("sk_get_summation_order", [ctypes.POINTER(ctypes.c_int32)]),
    ("sk_device_alloc", [ctypes.POINTER(c_vp), ctypes.c_size_t]),
    ("sk_device_free", [c_vp]),
    ("sk_memcpy_h2d", [c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("sk_memcpy_d2h", [c_vp, c_vp, ctypes.c_size_t, c_vp]),
    ("sk_stream_synchronize", [c_vp]),
    ("sk_csr_create", [ctypes.POINTER(c_vp), c_i64, c_i64, c_vp, c_vp, c_vp, ctypes.c_int]),
    ("sk_ell_create", [ctypes.POINTER(c_vp), c_i64, c_i64, c_i64, c_vp, c_vp, ctypes.c_int]),
    ("sk_jad_create", [ctypes.POINTER(c_vp), c_i64, c_i64, c_i64, c_vp, c_vp, c_vp, c_vp, ctypes.c_int]),
    ("sk_bsr_create", [ctypes.POINTER(c_vp), c_i64, c_i64, c_i64, c_i64, c_vp, c_vp, c_vp, ctypes.c_int]),
    ("sk_ell_from_csr", [ctypes.POINTER(c_vp), c_vp]),
    ("sk_jad_from_csr", [ctypes.POINTER(c_vp), c_vp]),
    ("sk_bsr_from_csr", [ctypes.POINTER(c_vp), c_vp, c_i64, c_i64]),
    ("sk_matrix_build_ms", [c_vp, ctypes.POINTER(c_dbl)]),
    ("sk_csr_export", [c_vp, c_vp, c_vp, c_vp]),
    ("sk_ell_export", [c_vp, c_vp, c_vp]),
    ("sk_jad_export", [c_vp, c_vp, c_vp, c_vp, c_vp]),
    ("sk_bsr_export", [c_vp, c_vp, c_vp, c_vp]),
    ("sk_matrix_market_read", [ctypes.POINTER(c_vp), ctypes.c_char_p, ctypes.c_int, c_i32]),
    ("sk_matrix_market_read_buffer", [ctypes.POINTER(c_vp), ctypes.c_char_p, c_i64, ctypes.c_int, c_i32]),
    ("sk_matrix_market_write", [c_vp, ctypes.c_char_p, c_i32, c_i32]),
    ("sk_matrix_destroy", [c_vp]),
    ("sk_matrix_info", [c_vp, P_i64]),
    ("sk_matrix_layout", [c_vp, ctypes.POINTER(ctypes.c_int32)]),
    ("sk_matrix_add_f32_values", [c_vp]),
    ("sk_matrix_add_diagonals", [c_vp, ctypes.POINTER(ctypes.c_int)]),
    ("sk_matrix_add_panels", [c_vp, ctypes.POINTER(ctypes.c_int)]),
    ("sk_spmv", [c_vp, c_vp, c_vp, c_vp]),
    ("sk_spmv_f32", [c_vp, c_vp, c_vp, c_vp]),
    ("sk_spmv_host", [c_vp, c_vp, c_vp]),
    ("sk_dot", [ctypes.c_int, c_i64, c_vp, c_vp, ctypes.POINTER(c_dbl), c_vp]),
    ("sk_nrm2", [ctypes.c_int, c_i64, c_vp, ctypes.POINTER(c_dbl), c_vp]),
    ("sk_axpy", [ctypes.c_int, c_i64, c_dbl, c_vp, c_vp, c_vp]),
    ("sk_xpay", [ctypes.c_int, c_i64, c_vp, c_dbl, c_vp, c_vp]),
    ("sk_jacobi_create", [ctypes.POINTER(c_vp), c_vp]),
    ("sk_chebyshev_create", [ctypes.POINTER(c_vp), c_vp, c_dbl, c_dbl, c_i64]),
    ("sk_lanczos", [c_vp, ctypes.POINTER(LanczosConfig), c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(LanczosSummary),
                    c_vp]),
    ("sk_spectral_radius", [c_vp, c_i64, ctypes.POINTER(c_dbl)]),
    ("sk_eigenvalue_bounds", [c_vp, c_i64, ctypes.POINTER(c_dbl), ctypes.POINTER(c_dbl)]),
    ("sk_chebyshev_create_auto", [ctypes.POINTER(c_vp), c_vp, c_i64, c_i64, c_vp]),
    ("sk_precond_apply", [c_vp, c_i64, c_vp, c_vp, c_vp]),
    ("sk_precond_values", [c_vp, c_vp, c_i64, P_i64]),
    ("sk_precond_destroy", [c_vp]),
    ("sk_chebyshev_apply_noalloc", [c_vp, c_dbl, c_dbl, c_i64, c_vp, c_vp, c_vp]),
    ("sk_cg_solve", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(CgConfig), ctypes.POINTER(Summary),
                     c_vp, c_vp]),
    ("sk_bicgstab_solve", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(BicgstabConfig),
                           ctypes.POINTER(Summary), c_vp, c_vp]),
    ("sk_fgmres_solve", [c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(FgmresConfig), ctypes.POINTER(Summary),
                         c_vp, c_vp]),
    ("sk_gmres_solve", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(FgmresConfig), ctypes.POINTER(Summary),
                        c_vp, c_vp]),
    ("sk_cgs_solve", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(BicgstabConfig), ctypes.POINTER(Summary),
                      c_vp, c_vp]),
    ("sk_minres_solve", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(BicgstabConfig), ctypes.POINTER(Summary),
                         c_vp, c_vp]),
    ("sk_mixed_cg_solve", [c_vp, c_i32, c_vp, c_vp, ctypes.POINTER(MixedConfig), ctypes.POINTER(MixedSummary),
                           c_vp, c_vp]),
    ("sk_mixed_fgmres_solve", [c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(MixedFgmresConfig),
                               ctypes.POINTER(MixedSummary), c_vp, c_vp]),
    ("sk_batch_create", [ctypes.POINTER(c_vp), c_i64, c_vp, c_vp, c_vp, c_vp]),
    ("sk_batch_destroy", [c_vp]),
    ("sk_batched_cg_solve", [c_vp, c_vp, c_vp, ctypes.POINTER(BatchConfig), ctypes.POINTER(BatchResults), c_vp]),
    ("sk_batched_autotune", [c_vp, c_vp, c_vp, ctypes.POINTER(BatchConfig), ctypes.POINTER(BatchResults), c_i64,
                             ctypes.POINTER(c_i32), ctypes.POINTER(c_i32), c_vp]),
    ("sk_batched_variant_count", []),
    ("sk_net_create", [ctypes.POINTER(c_vp), ctypes.c_uint64]),
    ("sk_net_destroy", [c_vp]),
    ("sk_net_param_count", []),
    ("sk_net_get_params", [c_vp, c_vp, c_i64]),
    ("sk_net_set_params", [c_vp, c_vp, c_i64]),
    ("sk_net_set_legacy_mma", [c_vp, c_i32]),
    ("sk_net_status", [c_vp]),
    ("sk_pairs_create", [ctypes.POINTER(c_vp), c_i64, c_i64, c_i64, c_i32]),
    ("sk_pairs_destroy", [c_vp]),
    ("sk_pairs_count", [c_vp, P_i64]),
    ("sk_pairs_add_instance", [c_vp, c_vp, ctypes.POINTER(c_i32)]),
    ("sk_pairs_add", [c_vp, c_i32, c_vp, c_vp, c_vp]),
    ("sk_learned_harvest", [c_vp, c_i32, c_vp, c_vp, c_vp, c_i64, c_i64, P_i64]),
    ("sk_net_train", [c_vp, c_vp, ctypes.POINTER(TrainConfig), ctypes.POINTER(TrainSummary), c_vp]),
    ("sk_net_loss_grad", [c_vp, c_vp, c_vp, c_i32, c_dbl, ctypes.POINTER(c_dbl), c_vp, c_i64]),
    ("sk_learned_create", [ctypes.POINTER(c_vp), c_vp, c_vp, c_i64, c_i64]),
    ("sk_learned_planes", [c_vp, c_vp, c_i64]),
    ("sk_twolevel_create", [ctypes.POINTER(c_vp), c_vp, c_vp, c_i64, c_i64, c_i64, c_i32]),
    ("sk_fgmres_fallback_solve", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(FgmresConfig), c_dbl,
                                  ctypes.POINTER(Summary), c_vp, P_i64, c_vp]),
    ("sk_cg_solve_host", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(CgConfig), ctypes.POINTER(Summary),
                          c_vp]),
    ("sk_bicgstab_solve_host", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(BicgstabConfig),
                                ctypes.POINTER(Summary), c_vp]),
    ("sk_fgmres_solve_host", [c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(FgmresConfig), ctypes.POINTER(Summary),
                              c_vp]),
    ("sk_gmres_solve_host", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(FgmresConfig), ctypes.POINTER(Summary),
                             c_vp]),
    ("sk_cgs_solve_host", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(BicgstabConfig), ctypes.POINTER(Summary),
                           c_vp]),
    ("sk_minres_solve_host", [c_vp, c_vp, c_vp, c_vp, c_vp, ctypes.POINTER(BicgstabConfig),
                              ctypes.POINTER(Summary), c_vp]),
]

_lock = threading.Lock()
_lib = None
_shutting_down = False


def _mark_shutdown():
    global _shutting_down
    _shutting_down = True


atexit.register(_mark_shutdown)


def shutting_down():
    """True once the interpreter exits: handles are then left to the
    process teardown instead of being destroyed in arbitrary GC order."""
    return _shutting_down


def lib():
    """The loaded library; raises OSError when the .so is absent."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise OSError(
                    f"{LIB_PATH} is missing: build it with `python -m sparkit_b200.build` "
                    "(there is no CPU fallback)")
            L = ctypes.CDLL(LIB_PATH)
            for name, args in SIGNATURES:
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = (ctypes.c_char_p if name in ("sk_version", "sk_last_error")
                              else c_i64 if name == "sk_net_param_count" else ctypes.c_int)
            _lib = L
    return _lib


def check(status):
    """Raises SkError for a non-zero sk_status."""
    if status != SK_OK:
        msg = lib().sk_last_error()
        raise SkError(status, msg.decode() if msg else "")
    return status


def launch_count():
    n = c_i64(0)
    check(lib().sk_launch_count(ctypes.byref(n)))
    return n.value
