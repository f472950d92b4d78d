"""ctypes binding of libsil_b200.so (the sm_100a C ABI in include/sil_b200.h).

The library is built in-tree by similie_b200/build.py.  Loading fails loudly
when it is missing: there is no CPU implementation behind this API.
"""
import ctypes
import os

SIL_MAX_DIMS = 6
SIL_OK = 0
SIL_F64 = 0
SIL_F32 = 1

STATUS_NAMES = {
    0: "SIL_OK", 1: "SIL_ERR_INVALID", 2: "SIL_ERR_UNSUPPORTED", 3: "SIL_ERR_CUDA",
    4: "SIL_ERR_ALLOC", 5: "SIL_ERR_NONFINITE", 6: "SIL_ERR_STALLED", 7: "SIL_ERR_BUDGET",
}

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libsil_b200.so")


class SilField(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.c_void_p),
        ("dtype", ctypes.c_int32),
        ("ndims", ctypes.c_int32),
        ("ncomp", ctypes.c_int32),
        ("reserved", ctypes.c_int32),
        ("front", ctypes.c_int64 * SIL_MAX_DIMS),
        ("extent", ctypes.c_int64 * SIL_MAX_DIMS),
        ("stride", ctypes.c_int64 * SIL_MAX_DIMS),
        ("comp_stride", ctypes.c_int64),
    ]


class SilMag2dProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("node_mu", ctypes.c_void_p),
        ("rhs", ctypes.c_void_p),
        ("solution", ctypes.c_void_p),
    ]


class SilBHCurve(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_int32),
        ("b", ctypes.c_void_p),
        ("h", ctypes.c_void_p),
    ]


class SilMag2dNlProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("node_mu", ctypes.c_void_p),
        ("node_ferro", ctypes.c_void_p),
        ("curve", SilBHCurve),
        ("rhs", ctypes.c_void_p),
        ("solution", ctypes.c_void_p),
    ]


class SilMag3dProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("x", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("node_mu", ctypes.c_void_p),
        ("rhs", ctypes.c_void_p),
        ("solution", ctypes.c_void_p),
        ("gauge_penalty", ctypes.c_double),
        ("gauge", ctypes.c_int32),
    ]


class SilMag3dNlProblem(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int64),
        ("ny", ctypes.c_int64),
        ("nz", ctypes.c_int64),
        ("x", ctypes.c_void_p),
        ("y", ctypes.c_void_p),
        ("z", ctypes.c_void_p),
        ("node_mu", ctypes.c_void_p),
        ("node_ferro", ctypes.c_void_p),
        ("curve", SilBHCurve),
        ("rhs", ctypes.c_void_p),
        ("solution", ctypes.c_void_p),
        ("gauge_penalty", ctypes.c_double),
        ("gauge", ctypes.c_int32),
    ]


class SilMenuSettings(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("sor_relaxation_factor", ctypes.c_double),
        ("chebyshev_iterations", ctypes.c_int32),
        ("chebyshev_lower_bound", ctypes.c_double),
        ("chebyshev_upper_bound", ctypes.c_double),
        ("ir_iterations", ctypes.c_int32),
        ("ir_relaxation_factor", ctypes.c_double),
    ]


class SilPrecondSample(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32),
        ("ny", ctypes.c_int32),
        ("offset", ctypes.c_int64),
    ]


class SilSolveSettings(ctypes.Structure):
    _fields_ = [
        ("solver", ctypes.c_int32),
        ("max_iterations", ctypes.c_int32),
        ("relative_tolerance", ctypes.c_double),
        ("inner_iterations", ctypes.c_int32),
        ("inner_tolerance", ctypes.c_double),
        ("preconditioner", ctypes.c_void_p),
        ("stall_window", ctypes.c_int32),
        ("flexible_directions", ctypes.c_int32),
        ("jacobian_preconditioner", ctypes.c_void_p),
    ]


class SilSolveDiagnostics(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("refinements", ctypes.c_int32),
        ("status", ctypes.c_int32),
        ("initial_residual_l2", ctypes.c_double),
        ("final_residual_l2", ctypes.c_double),
        ("final_relative_residual", ctypes.c_double),
        ("learned_iterations", ctypes.c_int32),
        ("fallback", ctypes.c_int32),
    ]


class SilError(RuntimeError):
    def __init__(self, status, message):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


_lib = None

# (name, restype, argtypes) for every symbol include/sil_b200.h declares.
_P = ctypes.c_void_p
_F = ctypes.POINTER(SilField)
SIGNATURES = [
    ("sil_status_string", ctypes.c_char_p, [ctypes.c_int]),
    ("sil_last_error", ctypes.c_char_p, []),
    ("sil_deriv", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_int, _F, _F]),
    ("sil_transposed_coboundary", ctypes.c_int, [_P, ctypes.c_uint32, ctypes.c_int, _F, _F]),
    ("sil_geometry_create", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                           ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64)]),
    ("sil_geometry_destroy", ctypes.c_int, [_P]),
    ("sil_hodge_star", ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_int, _F, _F]),
    ("sil_fill_discrete_hodge_star", ctypes.c_int, [_P, _P, ctypes.c_int, _F]),
    ("sil_codifferential", ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_int, _F, _F]),
    ("sil_laplacian_plan_create", ctypes.c_int, [ctypes.POINTER(_P), _P, ctypes.c_uint32, ctypes.c_int, _F, _F,
                                                 ctypes.c_int]),
    ("sil_laplacian_plan_create_metric", ctypes.c_int, [ctypes.POINTER(_P), _P, ctypes.c_int, ctypes.c_int, _F, _F,
                                                        _F, _F]),
    ("sil_codifferential_plan_create", ctypes.c_int, [ctypes.POINTER(_P), _P, ctypes.c_int, ctypes.c_int, _F, _F]),
    ("sil_codifferential_run", ctypes.c_int, [_P, _P, _F, _F]),
    ("sil_codifferential_plan_destroy", ctypes.c_int, [_P]),
    ("sil_laplacian_run", ctypes.c_int, [_P, _P, _F, _F]),
    ("sil_laplacian_plan_destroy", ctypes.c_int, [_P]),
    ("sil_laplacian_plan_scratch_bytes", ctypes.c_size_t, [_P]),
    ("sil_laplacian_plan_kernel", ctypes.c_int, [_P]),
    ("sil_laplacian_plan_variant", ctypes.c_int, [_P]),
    ("sil_laplacian_plan_status", ctypes.c_int, [_P]),
    ("sil_laplacian_plan_set_wait_bound", ctypes.c_int, [_P, ctypes.c_int32]),
    ("sil_laplacian", ctypes.c_int, [_P, _P, ctypes.c_uint32, ctypes.c_int, _F, _F]),
    ("sil_mag2d_apply", ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int64, _P, _P, _P]),
    ("sil_mag2d_apply_noalloc", ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int64, _P, _P, _P]),
    ("sil_mag2d_nl_apply", ctypes.c_int, [_P, ctypes.POINTER(SilMag2dNlProblem), _P, _P]),
    ("sil_mag2d_nl_apply_jacobian", ctypes.c_int, [_P, ctypes.POINTER(SilMag2dNlProblem), _P, _P, _P]),
    ("sil_mag2d_nl_solve_batch", ctypes.c_int, [ctypes.POINTER(SilMag2dNlProblem), ctypes.c_int,
                                                ctypes.POINTER(SilSolveSettings),
                                                ctypes.POINTER(SilSolveDiagnostics), _P]),
    ("sil_mag2d_solve_batch", ctypes.c_int, [ctypes.POINTER(SilMag2dProblem), ctypes.c_int,
                                             ctypes.POINTER(SilSolveSettings),
                                             ctypes.POINTER(SilSolveDiagnostics), _P]),
    ("sil_fill_discrete_hodge_star_metric", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _F, _F, _F]),
    ("sil_hodge_star_stored", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _F, _F, _F]),
    ("sil_precond_num_params", ctypes.c_int64, []),
    ("sil_precond_create", ctypes.c_int, [ctypes.POINTER(_P), ctypes.c_uint64, _P]),
    ("sil_precond_destroy", None, [_P]),
    ("sil_precond_get_params", ctypes.c_int, [_P, _P]),
    ("sil_precond_set_params", ctypes.c_int, [_P, _P, _P]),
    ("sil_precond_get_optimizer_state", ctypes.c_int, [_P, _P, _P, ctypes.POINTER(ctypes.c_int64)]),
    ("sil_precond_set_optimizer_state", ctypes.c_int, [_P, _P, _P, ctypes.c_int64, _P]),
    ("sil_precond_apply", ctypes.c_int, [_P, _P, ctypes.POINTER(SilPrecondSample), ctypes.c_int, _P, _P, _P]),
    ("sil_precond_apply_active", ctypes.c_int,
     [_P, _P, ctypes.POINTER(SilPrecondSample), ctypes.c_int, _P, _P, _P, _P]),
    ("sil_precond_loss_grad", ctypes.c_int, [_P, _P, ctypes.POINTER(SilPrecondSample), ctypes.c_int, _P, _P, _P,
                                             ctypes.POINTER(ctypes.c_double), _P, _P]),
    ("sil_precond_train_step", ctypes.c_int, [_P, _P, ctypes.POINTER(SilPrecondSample), ctypes.c_int, _P, _P, _P,
                                              ctypes.c_float, ctypes.POINTER(ctypes.c_double)]),
    ("sil_precond_debug_fetch", ctypes.c_int, [_P, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int64]),
    ("sil_mag3d_apply", ctypes.c_int, [_P, ctypes.POINTER(SilMag3dProblem), _P, _P]),
    ("sil_mag3d_operator_create", ctypes.c_int, [ctypes.POINTER(_P), _P, ctypes.POINTER(SilMag3dProblem)]),
    ("sil_mag3d_operator_apply", ctypes.c_int, [_P, _P, _P, _P]),
    ("sil_mag3d_operator_destroy", ctypes.c_int, [_P]),
    ("sil_mag3d_solve_batch", ctypes.c_int, [ctypes.POINTER(SilMag3dProblem), ctypes.c_int,
                                             ctypes.POINTER(SilSolveSettings),
                                             ctypes.POINTER(SilSolveDiagnostics), _P]),
    ("sil_mag2d_assemble", ctypes.c_int, [_P, ctypes.c_int64, ctypes.c_int64, _P, ctypes.POINTER(_P)]),
    ("sil_mag3d_assemble", ctypes.c_int, [_P, ctypes.POINTER(SilMag3dProblem), ctypes.POINTER(_P)]),
    ("sil_mag2d_nl_assemble_jacobian", ctypes.c_int, [_P, ctypes.POINTER(SilMag2dNlProblem), _P, ctypes.POINTER(_P)]),
    ("sil_mag3d_nl_assemble_jacobian", ctypes.c_int, [_P, ctypes.POINTER(SilMag3dNlProblem), _P, ctypes.POINTER(_P)]),
    ("sil_csr_get", ctypes.c_int, [_P, ctypes.POINTER(ctypes.c_int64), ctypes.POINTER(ctypes.c_int64),
                                   ctypes.POINTER(_P), ctypes.POINTER(_P), ctypes.POINTER(_P)]),
    ("sil_csr_copy", ctypes.c_int, [_P, _P, _P, _P, _P]),
    ("sil_csr_spmv", ctypes.c_int, [_P, _P, _P, _P]),
    ("sil_csr_destroy", None, [_P]),
    ("sil_csr_precond_create", ctypes.c_int, [_P, _P, ctypes.POINTER(SilMenuSettings), ctypes.POINTER(_P)]),
    ("sil_csr_precond_apply", ctypes.c_int, [_P, _P, _P, _P]),
    ("sil_csr_precond_destroy", None, [_P]),
    ("sil_csr_solve", ctypes.c_int, [_P, _P, _P, _P, _P, ctypes.POINTER(SilSolveSettings),
                                     ctypes.POINTER(SilSolveDiagnostics)]),
    ("sil_csr_krylov_solve", ctypes.c_int, [_P, _P, _P, ctypes.c_int32, ctypes.c_int32, _P, _P,
                                            ctypes.POINTER(SilSolveSettings), ctypes.POINTER(SilSolveDiagnostics)]),
    ("sil_mag3d_nl_apply", ctypes.c_int, [_P, ctypes.POINTER(SilMag3dNlProblem), _P, _P]),
    ("sil_mag3d_nl_apply_jacobian", ctypes.c_int, [_P, ctypes.POINTER(SilMag3dNlProblem), _P, _P, _P]),
    ("sil_mag3d_nl_solve_batch", ctypes.c_int, [ctypes.POINTER(SilMag3dNlProblem), ctypes.c_int,
                                                ctypes.POINTER(SilSolveSettings),
                                                ctypes.POINTER(SilSolveDiagnostics), _P]),
]


def lib():
    """Load the CUDA library (building it first if sources are newer)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from . import build as _build
            _build.build()
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"similie_b200: CUDA library {LIB_PATH} is missing; run similie_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(status, what=""):
    if status != SIL_OK:
        msg = lib().sil_last_error().decode(errors="replace")
        raise SilError(status, f"{what}: {msg}" if what else msg)
