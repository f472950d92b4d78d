"""3D linear magnetostatics on stretched rectilinear grids (host set-up + GPU solve).

Mirrors SimiLie's MagnetostaticsOperator3D (curl-curl residual operator with
the Coulomb-gauge penalty, precomputed-stencil apply) and
minimize_strong_formulation_residual for the linear case
(onelab_interface/magnetostatics_onelab.hpp:1525-2396, 4919-4975, 5030-5067;
src/similie/solvers/minimize_strong_formulation_residual.hpp:127, 1308-1382):

  * cell inputs: permeability mu and the current density J (3 components)
    per cell, cell = ci + (nx-1) * (cj + (ny-1) * ck);
  * node permeability = mean over the (up to 8) adjacent cells;
  * right-hand side b[3*node + c] = sum over adjacent cells of
    1/8 * (cell face normal to c) * J_c, zero on the boundary;
  * operator y = curl^T (W curl A) + gamma H_A A with identity rows on the
    Dirichlet boundary, W = (d_m / (d_a d_b)) / mu at the sampled node,
    H_A = d_a d_b / d_c, d = central local node spacing; gamma defaults to 20
    like the reference's vector_potential_gauge_penalty.

Node arrays are flat, x fastest (node = i + nx * (j + ny * k)), unknowns
interleaved by component (row = 3 * node + c), like the reference's solver
views.  The set-up runs on the host as in the reference; the operator and
the solve run on the GPU through the C ABI.
"""
import ctypes
from dataclasses import dataclass, field

import numpy as np

from . import _native
from ._native import check, lib
from .magnetostatics import SOLVERS, Diagnostics

DEFAULT_GAUGE_PENALTY = 20.0


def stretched_coords(n, ratio=1.01, length=1.0):
    """n node coordinates on [0, length] whose spacings grow geometrically by `ratio`."""
    h = ratio ** np.arange(n - 1, dtype=np.float64)
    c = np.concatenate([[0.0], np.cumsum(h)])
    return c * (length / c[-1])


def _cells(a, nx, ny, nz, ncomp=1):
    shape = (nz - 1, ny - 1, nx - 1) if ncomp == 1 else (nz - 1, ny - 1, nx - 1, ncomp)
    return np.asarray(a, dtype=np.float64).reshape(shape)


def node_mu(nx, ny, nz, cell_mu, mu0=1.0):
    """Mean permeability of the cells adjacent to each node."""
    cm = _cells(cell_mu, nx, ny, nz)
    acc = np.zeros((nz, ny, nx))
    cnt = np.zeros((nz, ny, nx))
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                acc[dk:dk + nz - 1, dj:dj + ny - 1, di:di + nx - 1] += cm
                cnt[dk:dk + nz - 1, dj:dj + ny - 1, di:di + nx - 1] += 1
    return np.where(cnt > 0, acc / np.maximum(cnt, 1), mu0).ravel()


def rhs(x, y, z, cell_j):
    """b[3*node + c] = sum over adjacent cells of 1/8 * face_c * J_c, zero on the boundary."""
    x, y, z = (np.asarray(v, dtype=np.float64) for v in (x, y, z))
    nx, ny, nz = len(x), len(y), len(z)
    cj = _cells(cell_j, nx, ny, nz, 3)
    wx, wy, wz = np.diff(x), np.diff(y), np.diff(z)
    faces = (
        (wz[:, None, None] * wy[None, :, None]) * np.ones((1, 1, nx - 1)),
        (wz[:, None, None] * np.ones((1, ny - 1, 1))) * wx[None, None, :],
        np.ones((nz - 1, 1, 1)) * (wy[:, None] * wx[None, :])[None],
    )
    b = np.zeros((nz, ny, nx, 3))
    for c in range(3):
        contrib = 0.125 * faces[c] * cj[..., c]
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    b[dk:dk + nz - 1, dj:dj + ny - 1, di:di + nx - 1, c] += contrib
    b[0] = b[-1] = 0.0
    b[:, 0] = b[:, -1] = 0.0
    b[:, :, 0] = b[:, :, -1] = 0.0
    return b.ravel()


@dataclass
class Problem:
    """One structured 3D problem: node coordinates and cell inputs."""
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    cell_mu: np.ndarray
    cell_j: np.ndarray
    gamma: float = DEFAULT_GAUGE_PENALTY
    meta: dict = field(default_factory=dict)

    @property
    def shape(self):
        return len(self.x), len(self.y), len(self.z)

    def node_mu(self):
        return node_mu(*self.shape, self.cell_mu)

    def rhs(self):
        return rhs(self.x, self.y, self.z, self.cell_j)


def synthetic_problem(rng, n, loops=None, ratio=1.01, gamma=DEFAULT_GAUGE_PENALTY, tube=None):
    """Unit cube, n^3 nodes with geometric spacing `ratio` per axis, mu = 1,
    2-6 toroidal current loops (radius U[0.1, 0.3], random centre and axis,
    current U[-1, 1] along the loop inside a tube around the ring)."""
    x = stretched_coords(n, ratio)
    xc = 0.5 * (x[1:] + x[:-1])
    ZC, YC, XC = np.meshgrid(xc, xc, xc, indexing="ij")  # (nz-1, ny-1, nx-1), x fastest
    ncell = (n - 1) ** 3
    cell_j = np.zeros((n - 1, n - 1, n - 1, 3))
    nloops = int(rng.integers(2, 7)) if loops is None else loops
    hmax = float(np.max(np.diff(x)))
    rt = max(0.03, 2.5 * hmax) if tube is None else tube
    for _ in range(nloops):
        radius = rng.uniform(0.1, 0.3)
        centre = rng.uniform(radius + rt, 1.0 - radius - rt, 3)
        axis = rng.normal(size=3)
        axis /= np.linalg.norm(axis)
        current = rng.uniform(-1.0, 1.0)
        dx, dy, dz = XC - centre[0], YC - centre[1], ZC - centre[2]
        dn = dx * axis[0] + dy * axis[1] + dz * axis[2]
        px, py, pz = dx - dn * axis[0], dy - dn * axis[1], dz - dn * axis[2]
        rho = np.sqrt(px * px + py * py + pz * pz)
        inside = (rho - radius) ** 2 + dn * dn < rt * rt
        inv = np.where(inside, 1.0 / np.maximum(rho, 1e-300), 0.0) * current
        # tangent = axis x (p / rho)
        cell_j[..., 0] += (axis[1] * pz - axis[2] * py) * inv
        cell_j[..., 1] += (axis[2] * px - axis[0] * pz) * inv
        cell_j[..., 2] += (axis[0] * py - axis[1] * px) * inv
    return Problem(x, x.copy(), x.copy(), np.ones(ncell), cell_j.ravel(), gamma,
                   {"loops": nloops, "ratio": ratio, "tube": rt})


def synthetic_batch(seed, count=8, n=256, **kw):
    rng = np.random.default_rng(seed)
    return [synthetic_problem(rng, n, **kw) for _ in range(count)]


GAUGES = {"penalty": 0, "divergence": 1}


def _problem_struct(x, y, z, mu, gamma, rhs_dev=None, sol_dev=None, gauge="penalty"):
    p = _native.SilMag3dProblem()
    p.nx, p.ny, p.nz = len(x), len(y), len(z)
    p.x, p.y, p.z = (v.ctypes.data for v in (x, y, z))
    p.node_mu = mu.data_ptr()
    p.rhs = 0 if rhs_dev is None else rhs_dev.data_ptr()
    p.solution = 0 if sol_dev is None else sol_dev.data_ptr()
    p.gauge_penalty = gamma
    p.gauge = GAUGES[gauge]
    return p


def _f64(v):
    return np.ascontiguousarray(v, dtype=np.float64)


def apply(x, y, z, node_mu_dev, a_dev, y_dev, gamma=DEFAULT_GAUGE_PENALTY, stream=None, gauge="penalty"):
    """y = K a on the GPU (torch CUDA float64 tensors; node_mu flat nodes, a/y flat 3*nodes).
    gauge: "penalty" (gamma * star A) or "divergence" (gamma times the
    codifferential gauge term, the reference's SIMILIE_DIVERGENCE_GAUGE_3D)."""
    import torch
    x, y, z = _f64(x), _f64(y), _f64(z)
    p = _problem_struct(x, y, z, node_mu_dev, gamma, gauge=gauge)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    check(lib().sil_mag3d_apply(s, ctypes.byref(p), ctypes.c_void_p(a_dev.data_ptr()),
                                ctypes.c_void_p(y_dev.data_ptr())), "mag3d_apply")
    return y_dev


class Operator:
    """y = K a with the set-up done once (spacing tables, 1/mu, the divergence
    gauge's table), as the reference's MagnetostaticsOperator3D precomputes
    its stencils; apply() is one kernel on the stream and can be captured in
    a CUDA graph.  node_mu_dev is read at construction."""

    def __init__(self, x, y, z, node_mu_dev, gamma=DEFAULT_GAUGE_PENALTY, stream=None, gauge="penalty"):
        import torch
        self._coords = tuple(_f64(v) for v in (x, y, z))
        self.nodes = len(self._coords[0]) * len(self._coords[1]) * len(self._coords[2])
        p = _problem_struct(*self._coords, node_mu_dev, gamma, gauge=gauge)
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
        h = ctypes.c_void_p()
        check(lib().sil_mag3d_operator_create(ctypes.byref(h), s, ctypes.byref(p)), "mag3d_operator_create")
        self._h = h

    def apply(self, a_dev, y_dev, stream=None):
        import torch
        s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
        check(lib().sil_mag3d_operator_apply(self._h, s, ctypes.c_void_p(a_dev.data_ptr()),
                                             ctypes.c_void_p(y_dev.data_ptr())), "mag3d_operator_apply")
        return y_dev

    def __del__(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            lib().sil_mag3d_operator_destroy(h)
            self._h = None


def solve_batch(coords, mus, rhss, sols, gammas=None, solver="cg", tol=1e-10, max_iterations=200000,
                inner_iterations=4000, inner_tolerance=1e-4, stream=None, gauge="penalty"):
    """minimize_strong_formulation_residual for a batch of 3D linear problems.

    coords: list of (x, y, z) host coordinate arrays; mus: torch CUDA float64
    node permeabilities; rhss, sols: torch CUDA float64 (3*nodes).  Returns
    one Diagnostics per problem."""
    import torch
    n = len(coords)
    gammas = [DEFAULT_GAUGE_PENALTY] * n if gammas is None else list(gammas)
    keep = [tuple(_f64(v) for v in c) for c in coords]
    probs = (_native.SilMag3dProblem * n)()
    for p in range(n):
        probs[p] = _problem_struct(*keep[p], mus[p], gammas[p], rhss[p], sols[p], gauge=gauge)
    st = _native.SilSolveSettings()
    st.solver = SOLVERS[solver]
    st.max_iterations = max_iterations
    st.relative_tolerance = tol
    st.inner_iterations = inner_iterations
    st.inner_tolerance = inner_tolerance
    diag = (_native.SilSolveDiagnostics * n)()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    rc = lib().sil_mag3d_solve_batch(probs, n, ctypes.byref(st), diag, s)
    out = [Diagnostics(d.iterations, bool(d.converged), d.refinements, d.status, d.initial_residual_l2,
                       d.final_residual_l2, d.final_relative_residual, d.learned_iterations, bool(d.fallback))
           for d in diag]
    check(rc, "mag3d_solve_batch")
    return out


# ----------------------------------------------------------------- nonlinear material

def node_ferro(nx, ny, nz, cell_nonlinear):
    """Share of the adjacent cells made of the nonlinear material, per node (0 where a
    node has no cell); a node follows the B-H curve when it is above 1/2
    (onelab_interface/magnetostatics_onelab.hpp:5030-5066)."""
    return node_mu(nx, ny, nz, np.asarray(cell_nonlinear, dtype=np.float64), mu0=0.0)


def nonlinear_knee(n):
    """Knee of the synthetic B-H curve for an n^3 unit-cube problem of the
    loop-current distribution: the 3D curl moments are circulations of A
    around a cell face and scale with the spacing 1/(n-1); at this knee the
    strongest moments in the core saturate mildly."""
    return 0.08 / (n - 1)


def nonlinear_problem(n, seed, tube=0.12):
    """(Problem, node_mu, node_ferro, curve b, curve h) of a seeded 3D
    nonlinear problem: the loop-current distribution with a random box core
    of permeability 1000 made of the saturating material."""
    from .magnetostatics import synthetic_bh_curve
    rng = np.random.default_rng(seed)
    p = synthetic_problem(rng, n, tube=tube)
    nc = n - 1
    lo = rng.integers(nc // 4, nc // 2, 3)
    hi = lo + rng.integers(nc // 6 + 1, nc // 3 + 1, 3)
    core = np.zeros((nc, nc, nc), dtype=bool)
    core[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] = True
    p.cell_mu = np.where(core, 1000.0, 1.0).ravel()
    p.meta["core"] = (lo.tolist(), hi.tolist())
    b, h = synthetic_bh_curve(nonlinear_knee(n))
    return p, p.node_mu(), node_ferro(n, n, n, core.ravel()), b, h


def _nl_problem_struct(x, y, z, mu, ferro, curve, gamma, rhs_dev=None, sol_dev=None, gauge="penalty"):
    p = _native.SilMag3dNlProblem()
    p.nx, p.ny, p.nz = len(x), len(y), len(z)
    p.x, p.y, p.z = (v.ctypes.data for v in (x, y, z))
    p.node_mu = mu.data_ptr()
    p.node_ferro = ferro.data_ptr()
    p.curve = curve.struct()
    p.rhs = 0 if rhs_dev is None else rhs_dev.data_ptr()
    p.solution = 0 if sol_dev is None else sol_dev.data_ptr()
    p.gauge_penalty = gamma
    p.gauge = GAUGES[gauge]
    return p


def nl_apply(x, y, z, node_mu_dev, node_ferro_dev, curve_b, curve_h, a_dev, y_dev, gamma=DEFAULT_GAUGE_PENALTY,
             stream=None, gauge="penalty"):
    """y = F(a), the 3D nonlinear operator (torch CUDA float64 tensors, a/y flat 3*nodes)."""
    import torch
    from .magnetostatics import _Curve
    x, y, z = _f64(x), _f64(y), _f64(z)
    c = _Curve(curve_b, curve_h)
    p = _nl_problem_struct(x, y, z, node_mu_dev, node_ferro_dev, c, gamma, gauge=gauge)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    check(lib().sil_mag3d_nl_apply(s, ctypes.byref(p), ctypes.c_void_p(a_dev.data_ptr()),
                                   ctypes.c_void_p(y_dev.data_ptr())), "mag3d_nl_apply")
    return y_dev


def nl_apply_jacobian(x, y, z, node_mu_dev, node_ferro_dev, curve_b, curve_h, state_dev, v_dev, y_dev,
                      gamma=DEFAULT_GAUGE_PENALTY, stream=None, gauge="penalty"):
    """y = J(state) v for the 3D nonlinear operator."""
    import torch
    from .magnetostatics import _Curve
    x, y, z = _f64(x), _f64(y), _f64(z)
    c = _Curve(curve_b, curve_h)
    p = _nl_problem_struct(x, y, z, node_mu_dev, node_ferro_dev, c, gamma, gauge=gauge)
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    check(lib().sil_mag3d_nl_apply_jacobian(s, ctypes.byref(p), ctypes.c_void_p(state_dev.data_ptr()),
                                            ctypes.c_void_p(v_dev.data_ptr()), ctypes.c_void_p(y_dev.data_ptr())),
          "mag3d_nl_apply_jacobian")
    return y_dev


def nl_solve_batch(coords, mus, ferros, curves, rhss, sols, gammas=None, tol=1e-10, max_iterations=100000,
                   stream=None, jacobian_preconditioner=None, gauge="penalty"):
    """Newton + line search for a batch of 3D nonlinear problems.  coords: (x, y, z) host arrays;
    curves: (b, h) sample arrays; sols hold the initial guesses and receive the solutions.
    jacobian_preconditioner as in magnetostatics.nl_solve_batch.
    Returns one Diagnostics per problem (refinements = Newton steps)."""
    import torch
    from .magnetostatics import _Curve, _menu_pointer
    n = len(coords)
    gammas = [DEFAULT_GAUGE_PENALTY] * n if gammas is None else list(gammas)
    keep = [tuple(_f64(v) for v in c) for c in coords]
    kc = [_Curve(b, h) for b, h in curves]
    probs = (_native.SilMag3dNlProblem * n)()
    for k in range(n):
        probs[k] = _nl_problem_struct(*keep[k], mus[k], ferros[k], kc[k], gammas[k], rhss[k], sols[k], gauge=gauge)
    st = _native.SilSolveSettings()
    st.max_iterations = max_iterations
    st.relative_tolerance = tol
    menu = _menu_pointer(st, jacobian_preconditioner)
    diag = (_native.SilSolveDiagnostics * n)()
    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream if stream is None else stream)
    rc = lib().sil_mag3d_nl_solve_batch(probs, n, ctypes.byref(st), diag, s)
    del menu
    out = [Diagnostics(d.iterations, bool(d.converged), d.refinements, d.status, d.initial_residual_l2,
                       d.final_residual_l2, d.final_relative_residual) for d in diag]
    check(rc, "mag3d_nl_solve_batch")
    return out
