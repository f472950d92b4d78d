"""Assembled (CSR) magnetostatics operators, the reference's preconditioner
menu on them, and a preconditioned CG on the GPU.

Mirrors the reference's ``use_matrix_free = false`` path and its
``PreconditionerType`` menu (src/similie/solvers/
minimize_strong_formulation_residual.hpp:53-75, 921-1304;
onelab_interface/magnetostatics_onelab.hpp:3120-3737 for the assembly): the
operator of ``magnetostatics.apply`` / ``magnetostatics3d.apply`` becomes a
device CSR matrix, a preconditioner is built on it by name (the reference's
``SIMILIE_PRECONDITIONER`` spellings), and ``solve`` runs CG from x = 0 to
the relative tolerance.
"""
import ctypes

import numpy as np

from . import _native
from ._native import check, lib
from .magnetostatics import Diagnostics

# names as the reference's parse_preconditioner accepts them
# (minimize_strong_formulation_residual.hpp:87-115)
_KINDS = {
    "identity": 0, "jacobi": 1,
    "spdisai": 2, "spd-isai": 2, "spd_isai": 2,
    "symmetricgaussseidel": 3, "symmetric-gauss-seidel": 3, "symmetric_gauss_seidel": 3,
    "ssor": 4,
    "chebyshevjacobi": 5, "chebyshev-jacobi": 5, "chebyshev_jacobi": 5,
    "irjacobi": 6, "ir-jacobi": 6, "ir_jacobi": 6,
    "generalisai": 7, "general-isai": 7, "general_isai": 7, "isai": 7,
}
KINDS = ("identity", "jacobi", "spd-isai", "symmetric-gauss-seidel", "ssor", "chebyshev-jacobi", "ir-jacobi",
         "general-isai")


def kind_of(name):
    """The menu index of a preconditioner name (case-insensitive, as the reference's spellings)."""
    key = str(name).lower()
    if key not in _KINDS:
        raise ValueError(f"unknown strong-formulation preconditioner: {name}")
    return _KINDS[key]


def _stream(stream):
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)


class CsrMatrix:
    """A device CSR matrix owned by the library (int32 row pointers and columns, FP64 values)."""

    def __init__(self, handle):
        self._h = ctypes.c_void_p(handle)

    @classmethod
    def mag2d(cls, nx, ny, node_mu_dev, stream=None):
        h = ctypes.c_void_p()
        check(lib().sil_mag2d_assemble(_stream(stream), nx, ny, ctypes.c_void_p(node_mu_dev.data_ptr()),
                                       ctypes.byref(h)), "mag2d_assemble")
        return cls(h.value)

    @classmethod
    def mag3d(cls, x, y, z, node_mu_dev, gamma=20.0, gauge="penalty", stream=None):
        from .magnetostatics3d import _f64, _problem_struct
        x, y, z = _f64(x), _f64(y), _f64(z)
        p = _problem_struct(x, y, z, node_mu_dev, gamma, gauge=gauge)
        h = ctypes.c_void_p()
        check(lib().sil_mag3d_assemble(_stream(stream), ctypes.byref(p), ctypes.byref(h)), "mag3d_assemble")
        return cls(h.value)

    def _info(self):
        n, nnz = ctypes.c_int64(), ctypes.c_int64()
        ptr, col, val = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        check(lib().sil_csr_get(self._h, ctypes.byref(n), ctypes.byref(nnz), ctypes.byref(ptr), ctypes.byref(col),
                                ctypes.byref(val)), "csr_get")
        return n.value, nnz.value, ptr.value, col.value, val.value

    @property
    def shape(self):
        n = self._info()[0]
        return n, n

    @property
    def nnz(self):
        return self._info()[1]

    def to_scipy(self):
        """A host copy as scipy.sparse.csr_matrix."""
        import scipy.sparse as sp
        n, nnz = self._info()[:2]
        hp = np.zeros(n + 1, dtype=np.int32)
        hc = np.zeros(max(nnz, 1), dtype=np.int32)
        hv = np.zeros(max(nnz, 1), dtype=np.float64)
        check(lib().sil_csr_copy(_stream(None), self._h, ctypes.c_void_p(hp.ctypes.data),
                                 ctypes.c_void_p(hc.ctypes.data), ctypes.c_void_p(hv.ctypes.data)), "csr_copy")
        return sp.csr_matrix((hv[:nnz], hc[:nnz], hp), shape=(n, n))

    def spmv(self, x_dev, y_dev, stream=None):
        check(lib().sil_csr_spmv(_stream(stream), self._h, ctypes.c_void_p(x_dev.data_ptr()),
                                 ctypes.c_void_p(y_dev.data_ptr())), "csr_spmv")
        return y_dev

    def close(self):
        if self._h is not None and self._h.value:
            lib().sil_csr_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def menu_settings(kind="jacobi", sor_relaxation_factor=0.0, chebyshev_iterations=0, chebyshev_lower_bound=0.0,
                  chebyshev_upper_bound=0.0, ir_iterations=0, ir_relaxation_factor=0.0):
    """A sil_menu_settings for one menu entry (0 keeps the reference's default of a field)."""
    cfg = _native.SilMenuSettings()
    cfg.kind = kind_of(kind)
    cfg.sor_relaxation_factor = sor_relaxation_factor
    cfg.chebyshev_iterations = chebyshev_iterations
    cfg.chebyshev_lower_bound = chebyshev_lower_bound
    cfg.chebyshev_upper_bound = chebyshev_upper_bound
    cfg.ir_iterations = ir_iterations
    cfg.ir_relaxation_factor = ir_relaxation_factor
    return cfg


def jacobian2d(problem_struct, state_dev, stream=None):
    """The Jacobian of a 2D nonlinear problem (a SilMag2dNlProblem) at `state` as a CsrMatrix."""
    h = ctypes.c_void_p()
    check(lib().sil_mag2d_nl_assemble_jacobian(_stream(stream), ctypes.byref(problem_struct),
                                               ctypes.c_void_p(state_dev.data_ptr()), ctypes.byref(h)),
          "mag2d_nl_assemble_jacobian")
    return CsrMatrix(h.value)


def jacobian3d(problem_struct, state_dev, stream=None):
    """The Jacobian of a 3D nonlinear problem (a SilMag3dNlProblem) at `state` as a CsrMatrix."""
    h = ctypes.c_void_p()
    check(lib().sil_mag3d_nl_assemble_jacobian(_stream(stream), ctypes.byref(problem_struct),
                                               ctypes.c_void_p(state_dev.data_ptr()), ctypes.byref(h)),
          "mag3d_nl_assemble_jacobian")
    return CsrMatrix(h.value)


class Preconditioner:
    """One entry of the reference's preconditioner menu, built on a CsrMatrix (which it keeps alive)."""

    def __init__(self, matrix, kind="jacobi", sor_relaxation_factor=0.0, chebyshev_iterations=0,
                 chebyshev_lower_bound=0.0, chebyshev_upper_bound=0.0, ir_iterations=0, ir_relaxation_factor=0.0,
                 stream=None):
        self.matrix = matrix
        cfg = menu_settings(kind, sor_relaxation_factor, chebyshev_iterations, chebyshev_lower_bound,
                            chebyshev_upper_bound, ir_iterations, ir_relaxation_factor)
        h = ctypes.c_void_p()
        check(lib().sil_csr_precond_create(_stream(stream), matrix._h, ctypes.byref(cfg), ctypes.byref(h)),
              "csr_precond_create")
        self._h = h

    def apply(self, r_dev, z_dev, stream=None):
        check(lib().sil_csr_precond_apply(_stream(stream), self._h, ctypes.c_void_p(r_dev.data_ptr()),
                                          ctypes.c_void_p(z_dev.data_ptr())), "csr_precond_apply")
        return z_dev

    def close(self):
        if self._h is not None and self._h.value:
            lib().sil_csr_precond_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# the reference's SIMILIE_SOLVER values (minimize_strong_formulation_residual.hpp:1069-1130)
SOLVERS = {"cg": 0, "minres": 1, "fcg": 2, "gmres": 3, "bicgstab": 4, "gcr": 5, "idr": 6}


def solve(matrix, preconditioner, rhs_dev, x_dev, tol=1e-10, max_iterations=100000, stream=None, solver="cg",
          dim=0):
    """The assembled-matrix solve from x = 0 with a Krylov method of the reference's menu (CG by
    default; dim: GMRES / GCR Krylov dimension or IDR subspace, 0 for the reference's 100 / 8);
    returns Diagnostics."""
    st = _native.SilSolveSettings()
    st.max_iterations = max_iterations
    st.relative_tolerance = tol
    d = _native.SilSolveDiagnostics()
    if solver not in SOLVERS:
        raise ValueError(f"unknown solver: {solver}")
    check(lib().sil_csr_krylov_solve(_stream(stream), matrix._h, preconditioner._h, SOLVERS[solver], dim,
                                     ctypes.c_void_p(rhs_dev.data_ptr()), ctypes.c_void_p(x_dev.data_ptr()),
                                     ctypes.byref(st), ctypes.byref(d)), "csr_krylov_solve")
    return Diagnostics(d.iterations, bool(d.converged), d.refinements, d.status, d.initial_residual_l2,
                       d.final_residual_l2, d.final_relative_residual)
