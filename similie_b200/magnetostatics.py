"""2D linear magnetostatics on structured rectilinear grids (host set-up + GPU solve).

Mirrors SimiLie's run_on_quadrilateral_grid / MagnetostaticsOperator2D /
minimize_strong_formulation_residual for the linear case
(onelab_interface/magnetostatics_onelab.hpp:4354-4565;
src/similie/solvers/minimize_strong_formulation_residual.hpp:1308-1382):

  * cell inputs: permeability mu and current density J_z per cell;
  * node permeability = mean over the (up to 4) adjacent cells (4491-4519);
  * right-hand side b_i = sum over adjacent cells of 1/4 * area * J_z, zero on
    the boundary (4414-4451);
  * operator y = d^T (nu d A) with identity rows on the Dirichlet boundary;
  * Jacobi-preconditioned CG from 0 to ||b - A x|| <= tol ||b||.

Arrays are flat, x fastest (row = i + nx * j), like the reference's solver
views.  The set-up runs on the host as in the reference; the operator and
the solve run on the GPU through the C ABI.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native
from ._native import check, lib

SOLVERS = {"cg": 0, "mixed": 1, "learned": 2}


def node_mu(nx, ny, cell_mu, mu0=1.0):
    """Mean permeability of the cells adjacent to each node."""
    cm = np.asarray(cell_mu, dtype=np.float64).reshape(ny - 1, nx - 1)
    acc = np.zeros((ny, nx))
    cnt = np.zeros((ny, nx))
    for dj in (0, 1):
        for di in (0, 1):
            acc[dj:dj + ny - 1, di:di + nx - 1] += cm
            cnt[dj:dj + ny - 1, di:di + nx - 1] += 1
    out = np.where(cnt > 0, acc / np.maximum(cnt, 1), mu0)
    return out.ravel()


def rhs(x, y, cell_j):
    """b_i = sum over adjacent cells of 1/4 * cell area * J, zero on the boundary."""
    x = np.asarray(x, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    nx, ny = len(x), len(y)
    cj = np.asarray(cell_j, dtype=np.float64).reshape(ny - 1, nx - 1)
    area = np.outer(np.diff(y), np.diff(x))
    contrib = 0.25 * area * cj
    b = np.zeros((ny, nx))
    for dj in (0, 1):
        for di in (0, 1):
            b[dj:dj + ny - 1, di:di + nx - 1] += contrib
    b[0, :] = b[-1, :] = 0.0
    b[:, 0] = b[:, -1] = 0.0
    return b.ravel()


@dataclass
class Problem:
    """One structured 2D problem: node coordinates and cell inputs."""
    x: np.ndarray
    y: np.ndarray
    cell_mu: np.ndarray
    cell_j: np.ndarray
    meta: dict = field(default_factory=dict)

    @property
    def nx(self):
        return len(self.x)

    @property
    def ny(self):
        return len(self.y)

    def node_mu(self):
        return node_mu(self.nx, self.ny, self.cell_mu)

    def rhs(self):
        return rhs(self.x, self.y, self.cell_j)


def synthetic_problem(rng, n, coils=None, cores=None, mu_core=1000.0):
    """Unit square, n x n nodes, 1-8 rectangular coils with J ~ U[-1, 1] and
    0-3 rectangles of relative permeability `mu_core` (corners U[0.1, 0.9])."""
    x = np.linspace(0.0, 1.0, n)
    y = np.linspace(0.0, 1.0, n)
    ncell = n - 1
    xc = 0.5 * (x[1:] + x[:-1])
    yc = 0.5 * (y[1:] + y[:-1])
    XC, YC = np.meshgrid(xc, yc)  # shape (ny-1, nx-1), x fastest
    cell_j = np.zeros((ncell, ncell))
    cell_mu = np.ones((ncell, ncell))
    nco = int(rng.integers(1, 9)) if coils is None else coils
    nmu = int(rng.integers(0, 4)) if cores is None else cores
    for _ in range(nco):
        a, b = np.sort(rng.uniform(0.1, 0.9, 2))
        c, d = np.sort(rng.uniform(0.1, 0.9, 2))
        cell_j[(XC >= a) & (XC <= b) & (YC >= c) & (YC <= d)] += rng.uniform(-1, 1)
    for _ in range(nmu):
        a, b = np.sort(rng.uniform(0.1, 0.9, 2))
        c, d = np.sort(rng.uniform(0.1, 0.9, 2))
        cell_mu[(XC >= a) & (XC <= b) & (YC >= c) & (YC <= d)] = mu_core
    if not np.any(cell_j):
        cell_j[ncell // 2, ncell // 2] = 1.0
    return Problem(x, y, cell_mu.ravel(), cell_j.ravel(), {"coils": nco, "cores": nmu})


def synthetic_batch(seed, count=64, sizes=(128, 256, 384, 512, 768, 1024)):
    rng = np.random.default_rng(seed)
    return [synthetic_problem(rng, int(rng.choice(sizes))) for _ in range(count)]


def apply(node_mu_dev, a_dev, y_dev, nx, ny, stream=None):
    """y = K a on the GPU (torch CUDA float64 tensors, flat nx*ny)."""
    import torch
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    check(lib().sil_mag2d_apply(s, nx, ny, ctypes.c_void_p(node_mu_dev.data_ptr()), ctypes.c_void_p(a_dev.data_ptr()),
                                ctypes.c_void_p(y_dev.data_ptr())), "mag2d_apply")
    return y_dev


@dataclass
class Diagnostics:
    iterations: int
    converged: bool
    refinements: int
    status: int
    initial_residual_l2: float
    final_residual_l2: float
    final_relative_residual: float
    learned_iterations: int = 0
    fallback: bool = False


def solve_batch(mus, rhss, sols, shapes, solver="cg", tol=1e-10, max_iterations=200000, inner_iterations=4000,
                inner_tolerance=1e-4, stream=None, preconditioner=None, stall_window=200, flexible_directions=8):
    """minimize_strong_formulation_residual for a batch of linear problems.

    mus, rhss, sols: lists of torch CUDA float64 tensors (flat nx*ny);
    shapes: list of (nx, ny).  solver: "cg" (FP64), "mixed" (FP32 inner CG
    inside FP64 refinement) or "learned" (flexible CG with `preconditioner`, a
    similie_b200.precond.LearnedPreconditioner, at most 64 problems, keeping
    `flexible_directions` (1..16) A-orthogonal directions, then the mixed
    solver for problems whose preconditioned residual stalls).
    Returns one Diagnostics per problem."""
    import torch
    n = len(shapes)
    probs = (_native.SilMag2dProblem * n)()
    for p, (nx, ny) in enumerate(shapes):
        probs[p].nx, probs[p].ny = nx, ny
        probs[p].node_mu = mus[p].data_ptr()
        probs[p].rhs = rhss[p].data_ptr()
        probs[p].solution = sols[p].data_ptr()
    st = _native.SilSolveSettings()
    st.solver = SOLVERS[solver]
    st.max_iterations = max_iterations
    st.relative_tolerance = tol
    st.inner_iterations = inner_iterations
    st.inner_tolerance = inner_tolerance
    st.stall_window = stall_window
    st.flexible_directions = flexible_directions
    if preconditioner is not None:
        st.preconditioner = preconditioner._h.value
    diag = (_native.SilSolveDiagnostics * n)()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    rc = lib().sil_mag2d_solve_batch(probs, n, ctypes.byref(st), diag, s)
    out = [Diagnostics(d.iterations, bool(d.converged), d.refinements, d.status, d.initial_residual_l2,
                       d.final_residual_l2, d.final_relative_residual, d.learned_iterations, bool(d.fallback))
           for d in diag]
    check(rc, "mag2d_solve_batch")
    return out


# ----------------------------------------------------------------- nonlinear (saturating) material

def node_ferro(nx, ny, cell_nonlinear):
    """Share of the adjacent cells made of the nonlinear material, per node; a
    node follows the B-H curve when it is above 1/2
    (onelab_interface/magnetostatics_onelab.hpp:4491-4517)."""
    return node_mu(nx, ny, np.asarray(cell_nonlinear, dtype=np.float64), mu0=0.0)


def synthetic_bh_curve(b_knee, mu_r=1000.0, samples=64, b_max=4.0):
    """Samples (b, h) of a saturating curve h = (b / mu_r) (1 + (b / b_knee)^4)
    on b in [0, b_max * b_knee]: permeability mu_r below the knee, falling
    beyond it.  A synthetic stand-in for a measured B-H table.

    The field of the reference's material law is the derivative of
    b h(b) / 2, which involves dh/db: with h interpolated linearly between
    samples it jumps at every sample, so Newton converges when the solution's
    moments stay off those kinks (mild saturation) and can stall otherwise."""
    b = np.linspace(0.0, b_max * b_knee, samples)
    h = (b / mu_r) * (1.0 + (b / b_knee) ** 4)
    return b, h


def nonlinear_knee(n):
    """Knee of the synthetic curve for an n x n unit-square problem of the
    batched distribution: the moments are potential differences, so they
    scale with the spacing 1/(n-1); at this knee the strongest moments in the
    cores saturate."""
    return 80.0 / (n - 1)


def nonlinear_problem(n, seed):
    """(Problem, node_mu, node_ferro, curve b, curve h) of a seeded nonlinear
    problem: the batched distribution's permeability-1000 rectangles made of
    the saturating material."""
    rng = np.random.default_rng(seed)
    p = synthetic_problem(rng, n, cores=int(rng.integers(1, 4)))
    b, h = synthetic_bh_curve(nonlinear_knee(n))
    return p, p.node_mu(), node_ferro(n, n, p.cell_mu > 1.0), b, h


class _Curve:
    def __init__(self, b, h):
        self.b = np.ascontiguousarray(b, dtype=np.float64)
        self.h = np.ascontiguousarray(h, dtype=np.float64)

    def struct(self):
        return _native.SilBHCurve(len(self.b), self.b.ctypes.data, self.h.ctypes.data)


def _nl_problem(nx, ny, mu, ferro, curve, rhs=None, sol=None):
    p = _native.SilMag2dNlProblem()
    p.nx, p.ny = nx, ny
    p.node_mu = mu.data_ptr()
    p.node_ferro = ferro.data_ptr()
    p.curve = curve.struct()
    p.rhs = rhs.data_ptr() if rhs is not None else None
    p.solution = sol.data_ptr() if sol is not None else None
    return p


def nl_apply(node_mu_dev, node_ferro_dev, curve_b, curve_h, a_dev, y_dev, nx, ny, stream=None):
    """y = F(a), the nonlinear residual operator (torch CUDA float64 tensors)."""
    import torch
    c = _Curve(curve_b, curve_h)
    p = _nl_problem(nx, ny, node_mu_dev, node_ferro_dev, c)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    check(lib().sil_mag2d_nl_apply(s, ctypes.byref(p), ctypes.c_void_p(a_dev.data_ptr()),
                                   ctypes.c_void_p(y_dev.data_ptr())), "mag2d_nl_apply")
    return y_dev


def nl_apply_jacobian(node_mu_dev, node_ferro_dev, curve_b, curve_h, state_dev, x_dev, y_dev, nx, ny, stream=None):
    """y = J(state) x."""
    import torch
    c = _Curve(curve_b, curve_h)
    p = _nl_problem(nx, ny, node_mu_dev, node_ferro_dev, c)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    check(lib().sil_mag2d_nl_apply_jacobian(s, ctypes.byref(p), ctypes.c_void_p(state_dev.data_ptr()),
                                            ctypes.c_void_p(x_dev.data_ptr()), ctypes.c_void_p(y_dev.data_ptr())),
          "mag2d_nl_apply_jacobian")
    return y_dev


def _menu_pointer(st, jacobian_preconditioner):
    """Points st.jacobian_preconditioner at a menu entry (a name or a dict of
    sil_menu_settings fields); returns the structure to keep alive."""
    if jacobian_preconditioner is None:
        return None
    from .assembled import menu_settings
    cfg = (menu_settings(jacobian_preconditioner) if isinstance(jacobian_preconditioner, str)
           else menu_settings(**jacobian_preconditioner))
    st.jacobian_preconditioner = ctypes.addressof(cfg)
    return cfg


def nl_solve_batch(mus, ferros, curves, rhss, sols, shapes, tol=1e-10, max_iterations=100000, stream=None,
                   jacobian_preconditioner=None):
    """Newton + line search for a batch of nonlinear problems (minimize_strong_formulation_residual,
    nonlinear branch).  curves: list of (b, h) sample arrays; sols hold the initial guesses and
    receive the solutions.  jacobian_preconditioner: None for the matrix-free Jacobi-CG, or a menu
    entry ("ssor", or a dict of sil_menu_settings fields) for CG on the assembled Jacobian.
    Returns one Diagnostics per problem (refinements = Newton steps)."""
    import torch
    n = len(shapes)
    keep = [_Curve(b, h) for b, h in curves]
    probs = (_native.SilMag2dNlProblem * n)()
    for k, (nx, ny) in enumerate(shapes):
        probs[k] = _nl_problem(nx, ny, mus[k], ferros[k], keep[k], rhss[k], sols[k])
    st = _native.SilSolveSettings()
    st.max_iterations = max_iterations
    st.relative_tolerance = tol
    menu = _menu_pointer(st, jacobian_preconditioner)
    diag = (_native.SilSolveDiagnostics * n)()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    rc = lib().sil_mag2d_nl_solve_batch(probs, n, ctypes.byref(st), diag, s)
    out = [Diagnostics(d.iterations, bool(d.converged), d.refinements, d.status, d.initial_residual_l2,
                       d.final_residual_l2, d.final_relative_residual) for d in diag]
    check(rc, "mag2d_nl_solve_batch")
    return out
