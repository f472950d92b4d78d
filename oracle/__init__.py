"""CPU oracle for SimiLie's DEC operators -- TEST INFRASTRUCTURE ONLY.

A C++/OpenMP restatement of the reference algorithms (see sil_oracle.cpp for
the file:line each routine follows).  Only the test-suite, the smoke check
and the CPU-baseline leg of bench.py may use it, and only as the checker.

Arrays are numpy float64.  A field array has its lattice axes first and the
form-component axis last unless `comp_axis` says otherwise; any strides are
accepted (component-first and component-last layouts both work).
"""
import ctypes

import numpy as np

from . import build as _build

SILO_MAX_DIMS = 6


class _Field(ctypes.Structure):
    _fields_ = [
        ("data", ctypes.POINTER(ctypes.c_double)),
        ("ndims", ctypes.c_int32),
        ("ncomp", ctypes.c_int32),
        ("front", ctypes.c_int64 * SILO_MAX_DIMS),
        ("extent", ctypes.c_int64 * SILO_MAX_DIMS),
        ("stride", ctypes.c_int64 * SILO_MAX_DIMS),
        ("comp_stride", ctypes.c_int64),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        _lib = ctypes.CDLL(path)
        P = ctypes.POINTER(_Field)
        dp = ctypes.POINTER(ctypes.c_double)
        i64 = ctypes.c_int64
        _lib.silo_coboundary.argtypes = [ctypes.c_uint32, ctypes.c_int, P, P]
        _lib.silo_transposed_coboundary.argtypes = [ctypes.c_uint32, ctypes.c_int, P, P]
        _lib.silo_fill_hodge_star.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P]
        _lib.silo_apply_hodge_star.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P]
        _lib.silo_hodge_matrix.argtypes = [ctypes.c_int, ctypes.c_int, P, P, ctypes.POINTER(i64), dp]
        _lib.silo_codifferential.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P]
        _lib.silo_laplacian.argtypes = [ctypes.c_int, ctypes.c_int, P, P, P, P]
        _lib.silo_laplacian_prefilled.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.POINTER(P), P, P]
        _lib.silo_laplacian_hodge_ncomp.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.silo_laplacian_hodge_kin.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.silo_mag2d_node_mu.argtypes = [i64, i64, dp, ctypes.c_double, dp]
        _lib.silo_mag2d_rhs.argtypes = [i64, i64, dp, dp, dp, dp]
        _lib.silo_mag2d_apply.argtypes = [i64, i64, dp, dp, dp]
        _lib.silo_mag2d_diagonal.argtypes = [i64, i64, dp, dp]
        _lib.silo_mag2d_cg.argtypes = [i64, i64, dp, dp, dp, ctypes.c_double, ctypes.c_int, dp]
        _lib.silo_num_threads.argtypes = []
        ci = ctypes.c_int
        _lib.silo_bh_eval.argtypes = [ci, dp, dp, ci, dp, dp, dp, dp]
        _lib.silo_mag2d_nl_apply.argtypes = [i64, i64, dp, dp, ci, dp, dp, dp, dp]
        _lib.silo_mag2d_nl_jacobian_apply.argtypes = [i64, i64, dp, dp, ci, dp, dp, dp, dp, dp]
        _lib.silo_mag2d_nl_jacobian_diagonal.argtypes = [i64, i64, dp, dp, ci, dp, dp, dp, dp]
        _lib.silo_mag2d_nl_solve.argtypes = [i64, i64, dp, dp, ci, dp, dp, dp, dp, ctypes.c_double, ci,
                                             ctypes.POINTER(ci), dp]
        _lib.silo_mag3d_node_mu.argtypes = [i64, i64, i64, dp, ctypes.c_double, dp]
        _lib.silo_mag3d_rhs.argtypes = [i64, i64, i64, dp, dp, dp, dp, dp]
        _lib.silo_mag3d_apply.argtypes = [i64, i64, i64, dp, dp, dp, dp, ctypes.c_double, dp, dp]
        _lib.silo_mag3d_diagonal.argtypes = [i64, i64, i64, dp, dp, dp, dp, ctypes.c_double, dp]
        _lib.silo_mag3d_cg.argtypes = [i64, i64, i64, dp, dp, dp, dp, ctypes.c_double, dp, dp, ctypes.c_double,
                                       ctypes.c_int, dp]
        d = ctypes.c_double
        ip = ctypes.POINTER(ctypes.c_int64)
        i32p = ctypes.POINTER(ctypes.c_int32)
        _lib.silo_csr_precond_apply.argtypes = [i64, ip, i32p, dp, ci, dp, dp, dp]
        _lib.silo_csr_isai_values.argtypes = [i64, ip, i32p, dp, ci, dp]
        _lib.silo_csr_pcg.argtypes = [i64, ip, i32p, dp, ci, dp, dp, dp, d, ci, dp]
        _lib.silo_reduce_primal.argtypes = [ci, ci, ctypes.POINTER(_Field), ip, dp, dp]
        _lib.silo_reconstruct_primal.argtypes = [ci, ci, ctypes.POINTER(_Field), ip, dp, dp]
        _lib.silo_csr_krylov.argtypes = [i64, ip, i32p, dp, ci, ci, ci, dp, dp, dp, d, ci, dp]
        _lib.silo_mag2d_nl_solve_menu.argtypes = [i64, i64, dp, dp, ci, dp, dp, ci, dp, dp, dp, d, ci,
                                                  ctypes.POINTER(ci), dp]
        _lib.silo_mag3d_nl_solve_menu.argtypes = [i64, i64, i64, dp, dp, dp, dp, dp, d, ci, dp, dp, ci, dp, dp, dp,
                                                  d, ci, ctypes.POINTER(ci), dp]
        _lib.silo_mag3d_nl_apply.argtypes = [i64, i64, i64, dp, dp, dp, dp, dp, d, ci, dp, dp, dp, dp]
        _lib.silo_mag3d_nl_jacobian_apply.argtypes = [i64, i64, i64, dp, dp, dp, dp, dp, d, ci, dp, dp, dp, dp, dp]
        _lib.silo_mag3d_nl_jacobian_diagonal.argtypes = [i64, i64, i64, dp, dp, dp, dp, dp, d, ci, dp, dp, dp, dp]
        _lib.silo_mag3d_nl_solve.argtypes = [i64, i64, i64, dp, dp, dp, dp, dp, d, ci, dp, dp, dp, dp, d, ci,
                                             ctypes.POINTER(ci), dp]
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def field(arr, comp_axis=-1, front=None):
    """Describe a float64 numpy array as a strided oracle field."""
    if arr.dtype != np.float64:
        raise TypeError("oracle fields are float64")
    nd = arr.ndim
    comp_axis = comp_axis % nd
    axes = [a for a in range(nd) if a != comp_axis]
    f = _Field()
    f.data = _ptr(arr)
    f.ndims = len(axes)
    f.ncomp = arr.shape[comp_axis]
    for i, a in enumerate(axes):
        f.front[i] = 0 if front is None else int(front[i])
        f.extent[i] = arr.shape[a]
        f.stride[i] = arr.strides[a] // 8
    f.comp_stride = arr.strides[comp_axis] // 8
    f._keep = arr
    return f


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} rejected its arguments (rc={rc})")


def binom(n, k):
    from math import comb
    return comb(n, k) if 0 <= k <= n else 0


def coboundary(inp, out, k, form_mask=None, comp_axis=-1, in_front=None, out_front=None):
    """d on a k-form (clamped sampling); fills `out` in place."""
    fi = field(inp, comp_axis, in_front)
    fo = field(out, comp_axis, out_front)
    mask = form_mask if form_mask is not None else (1 << fi.ndims) - 1
    _check(lib().silo_coboundary(mask, k, ctypes.byref(fi), ctypes.byref(fo)), "coboundary")
    return out


def transposed_coboundary(inp, out, k, form_mask=None, comp_axis=-1, in_front=None, out_front=None):
    fi = field(inp, comp_axis, in_front)
    fo = field(out, comp_axis, out_front)
    mask = form_mask if form_mask is not None else (1 << fi.ndims) - 1
    _check(lib().silo_transposed_coboundary(mask, k, ctypes.byref(fi), ctypes.byref(fo)),
           "transposed coboundary")
    return out


def position_from_coords(coords):
    """Tensor-product position field (n comps per node) from 1D coordinates."""
    grids = np.meshgrid(*[np.asarray(c, dtype=np.float64) for c in coords], indexing="ij")
    return np.ascontiguousarray(np.stack(grids, axis=-1))


def identity_metric(shape, n):
    m = np.zeros(tuple(shape) + (n * n,), dtype=np.float64)
    for i in range(n):
        m[..., i * n + i] = 1.0
    return m


def hodge_ncomp(n, k_in):
    return n ** k_in * binom(n, n - k_in)


def fill_hodge_star(n, k_in, position, metric=None):
    shape = position.shape[:-1]
    hs = np.zeros(tuple(shape) + (hodge_ncomp(n, k_in),), dtype=np.float64)
    fp = field(position)
    fm = field(metric) if metric is not None else None
    fh = field(hs)
    _check(lib().silo_fill_hodge_star(n, k_in, ctypes.byref(fp),
                                      ctypes.byref(fm) if fm is not None else None,
                                      ctypes.byref(fh)), "fill_hodge_star")
    return hs


def apply_hodge_star(n, k_in, hodge, inp):
    out = np.zeros(inp.shape[:-1] + (binom(n, n - k_in),), dtype=np.float64)
    _check(lib().silo_apply_hodge_star(n, k_in, ctypes.byref(field(hodge)), ctypes.byref(field(inp)),
                                       ctypes.byref(field(out))), "apply_hodge_star")
    return out


def hodge_matrix(n, k_in, position, node, metric=None):
    m = np.zeros((binom(n, n - k_in), binom(n, k_in)), dtype=np.float64)
    nd = (ctypes.c_int64 * n)(*node)
    fm = field(metric) if metric is not None else None
    _check(lib().silo_hodge_matrix(n, k_in, ctypes.byref(field(position)),
                                   ctypes.byref(fm) if fm is not None else None, nd, _ptr(m)),
           "hodge_matrix")
    return m


def codifferential(n, k, position, inp, metric=None, out_shape=None):
    shape = out_shape if out_shape is not None else inp.shape[:-1]
    out = np.zeros(tuple(shape) + (binom(n, k - 1),), dtype=np.float64)
    fm = field(metric) if metric is not None else None
    _check(lib().silo_codifferential(n, k, ctypes.byref(field(position)),
                                     ctypes.byref(fm) if fm is not None else None,
                                     ctypes.byref(field(inp)), ctypes.byref(field(out))),
           "codifferential")
    return out


def laplacian(n, k, position, inp, metric=None, out_shape=None):
    """Staged Hodge Laplacian; default output lattice is the input minus its last node per axis."""
    shape = out_shape if out_shape is not None else tuple(s - 1 for s in inp.shape[:-1])
    out = np.zeros(tuple(shape) + (binom(n, k),), dtype=np.float64)
    fm = field(metric) if metric is not None else None
    _check(lib().silo_laplacian(n, k, ctypes.byref(field(position)),
                                ctypes.byref(fm) if fm is not None else None,
                                ctypes.byref(field(inp)), ctypes.byref(field(out))), "laplacian")
    return out


class StagedLaplacian:
    """Reference-structured staged Laplacian: stored Hodge tensors filled once,
    then run() chains the separate d/Hodge/transposed-d passes."""

    def __init__(self, n, k, position, metric=None):
        self.n, self.k = n, k
        self.hodges = []
        for which in range(4):
            nc = lib().silo_laplacian_hodge_ncomp(n, k, which)
            if nc == 0:
                self.hodges.append(None)
                continue
            kin = lib().silo_laplacian_hodge_kin(n, k, which)
            self.hodges.append(fill_hodge_star(n, kin, position, metric))

    def run(self, inp, out):
        fields = [field(h) if h is not None else None for h in self.hodges]
        P = ctypes.POINTER(_Field)
        arr = (P * 4)(*[ctypes.pointer(f) if f is not None else P() for f in fields])
        _check(lib().silo_laplacian_prefilled(self.n, self.k, arr, ctypes.byref(field(inp)),
                                              ctypes.byref(field(out))), "laplacian")
        return out


# ----------------------------------------------------------------- magnetostatics 2D

def mag2d_node_mu(nx, ny, cell_mu, mu0=1.0):
    out = np.zeros(nx * ny)
    c = np.ascontiguousarray(cell_mu, dtype=np.float64)
    lib().silo_mag2d_node_mu(nx, ny, _ptr(c), mu0, _ptr(out))
    return out


def mag2d_rhs(x, y, cell_j):
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    c = np.ascontiguousarray(cell_j, dtype=np.float64)
    out = np.zeros(len(x) * len(y))
    lib().silo_mag2d_rhs(len(x), len(y), _ptr(x), _ptr(y), _ptr(c), _ptr(out))
    return out


def mag2d_apply(nx, ny, node_mu, a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    mu = np.ascontiguousarray(node_mu, dtype=np.float64)
    out = np.zeros(nx * ny)
    lib().silo_mag2d_apply(nx, ny, _ptr(mu), _ptr(a), _ptr(out))
    return out


def mag2d_diagonal(nx, ny, node_mu):
    mu = np.ascontiguousarray(node_mu, dtype=np.float64)
    out = np.zeros(nx * ny)
    lib().silo_mag2d_diagonal(nx, ny, _ptr(mu), _ptr(out))
    return out


def mag2d_cg(nx, ny, node_mu, rhs, tol=1e-10, max_iter=100000):
    mu = np.ascontiguousarray(node_mu, dtype=np.float64)
    b = np.ascontiguousarray(rhs, dtype=np.float64)
    x = np.zeros(nx * ny)
    rel = ctypes.c_double(0.0)
    it = lib().silo_mag2d_cg(nx, ny, _ptr(mu), _ptr(b), _ptr(x), tol, max_iter, ctypes.byref(rel))
    return x, it, rel.value


def num_threads():
    return lib().silo_num_threads()


# ----------------------------------------------------------------- magnetostatics 2D, nonlinear material

def bh_eval(curve_b, curve_h, q):
    """F(q) = h/b at b = sqrt(q) of the interpolated B-H curve and its first two q-derivatives."""
    b, h, q = _f64(curve_b), _f64(curve_h), _f64(q)
    f, df, d2f = np.zeros(len(q)), np.zeros(len(q)), np.zeros(len(q))
    lib().silo_bh_eval(len(b), _ptr(b), _ptr(h), len(q), _ptr(q), _ptr(f), _ptr(df), _ptr(d2f))
    return f, df, d2f


def mag2d_nl_apply(nx, ny, node_mu, node_ferro, curve_b, curve_h, a):
    mu, fe, b, h, a = _f64(node_mu), _f64(node_ferro), _f64(curve_b), _f64(curve_h), _f64(a)
    out = np.zeros(nx * ny)
    lib().silo_mag2d_nl_apply(nx, ny, _ptr(mu), _ptr(fe), len(b), _ptr(b), _ptr(h), _ptr(a), _ptr(out))
    return out


def mag2d_nl_jacobian_apply(nx, ny, node_mu, node_ferro, curve_b, curve_h, state, x):
    mu, fe, b, h = _f64(node_mu), _f64(node_ferro), _f64(curve_b), _f64(curve_h)
    st, x = _f64(state), _f64(x)
    out = np.zeros(nx * ny)
    lib().silo_mag2d_nl_jacobian_apply(nx, ny, _ptr(mu), _ptr(fe), len(b), _ptr(b), _ptr(h), _ptr(st), _ptr(x),
                                       _ptr(out))
    return out


def mag2d_nl_jacobian_diagonal(nx, ny, node_mu, node_ferro, curve_b, curve_h, state):
    mu, fe, b, h, st = _f64(node_mu), _f64(node_ferro), _f64(curve_b), _f64(curve_h), _f64(state)
    out = np.zeros(nx * ny)
    lib().silo_mag2d_nl_jacobian_diagonal(nx, ny, _ptr(mu), _ptr(fe), len(b), _ptr(b), _ptr(h), _ptr(st), _ptr(out))
    return out


def mag2d_nl_solve(nx, ny, node_mu, node_ferro, curve_b, curve_h, rhs, x0=None, tol=1e-10, max_iter=100000):
    """Newton + line search; returns (x, cg_iterations, newton_steps, final relative residual)."""
    mu, fe, b, h, rhs = _f64(node_mu), _f64(node_ferro), _f64(curve_b), _f64(curve_h), _f64(rhs)
    x = np.zeros(nx * ny) if x0 is None else np.array(x0, dtype=np.float64)
    steps = ctypes.c_int(0)
    rel = ctypes.c_double(0.0)
    it = lib().silo_mag2d_nl_solve(nx, ny, _ptr(mu), _ptr(fe), len(b), _ptr(b), _ptr(h), _ptr(rhs), _ptr(x), tol,
                                   max_iter, ctypes.byref(steps), ctypes.byref(rel))
    return x, it, steps.value, rel.value


# ----------------------------------------------------------------- magnetostatics 3D

def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def mag3d_node_mu(nx, ny, nz, cell_mu, mu0=1.0):
    out = np.zeros(nx * ny * nz)
    c = _f64(cell_mu)
    lib().silo_mag3d_node_mu(nx, ny, nz, _ptr(c), mu0, _ptr(out))
    return out


def mag3d_rhs(x, y, z, cell_j):
    x, y, z, cj = _f64(x), _f64(y), _f64(z), _f64(cell_j)
    out = np.zeros(3 * len(x) * len(y) * len(z))
    lib().silo_mag3d_rhs(len(x), len(y), len(z), _ptr(x), _ptr(y), _ptr(z), _ptr(cj), _ptr(out))
    return out


def mag3d_apply(x, y, z, node_mu, gamma, a):
    x, y, z, mu, a = _f64(x), _f64(y), _f64(z), _f64(node_mu), _f64(a)
    out = np.zeros_like(a)
    lib().silo_mag3d_apply(len(x), len(y), len(z), _ptr(x), _ptr(y), _ptr(z), _ptr(mu), gamma, _ptr(a), _ptr(out))
    return out


def mag3d_diagonal(x, y, z, node_mu, gamma):
    x, y, z, mu = _f64(x), _f64(y), _f64(z), _f64(node_mu)
    out = np.zeros(3 * len(x) * len(y) * len(z))
    lib().silo_mag3d_diagonal(len(x), len(y), len(z), _ptr(x), _ptr(y), _ptr(z), _ptr(mu), gamma, _ptr(out))
    return out


def mag3d_cg(x, y, z, node_mu, gamma, rhs, tol=1e-10, max_iter=100000):
    x, y, z, mu, b = _f64(x), _f64(y), _f64(z), _f64(node_mu), _f64(rhs)
    sol = np.zeros_like(b)
    rel = ctypes.c_double(0.0)
    it = lib().silo_mag3d_cg(len(x), len(y), len(z), _ptr(x), _ptr(y), _ptr(z), _ptr(mu), gamma, _ptr(b), _ptr(sol),
                             tol, max_iter, ctypes.byref(rel))
    return sol, it, rel.value


# ----------------------------------------------------------------- magnetostatics 3D, nonlinear material

def _nl3_args(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h):
    x, y, z, mu, fe, b, h = (_f64(v) for v in (x, y, z, node_mu, node_ferro, curve_b, curve_h))
    keep = (x, y, z, mu, fe, b, h)
    args = [len(x), len(y), len(z), _ptr(x), _ptr(y), _ptr(z), _ptr(mu), _ptr(fe), float(gamma), len(b), _ptr(b),
            _ptr(h)]
    return keep, args


def mag3d_nl_apply(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h, a):
    keep, args = _nl3_args(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h)
    a = _f64(a)
    out = np.zeros_like(a)
    lib().silo_mag3d_nl_apply(*args, _ptr(a), _ptr(out))
    return out


def mag3d_nl_jacobian_apply(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h, state, v):
    keep, args = _nl3_args(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h)
    st, v = _f64(state), _f64(v)
    out = np.zeros_like(v)
    lib().silo_mag3d_nl_jacobian_apply(*args, _ptr(st), _ptr(v), _ptr(out))
    return out


def mag3d_nl_jacobian_diagonal(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h, state):
    keep, args = _nl3_args(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h)
    st = _f64(state)
    out = np.zeros_like(st)
    lib().silo_mag3d_nl_jacobian_diagonal(*args, _ptr(st), _ptr(out))
    return out


def mag3d_nl_solve(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h, rhs, x0=None, tol=1e-10,
                   max_iter=100000):
    """Newton + line search on the 3D operator; returns (x, cg_iterations, newton_steps, final relative residual)."""
    keep, args = _nl3_args(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h)
    rhs = _f64(rhs)
    sol = np.zeros_like(rhs) if x0 is None else np.array(x0, dtype=np.float64)
    steps = ctypes.c_int(0)
    rel = ctypes.c_double(0.0)
    it = lib().silo_mag3d_nl_solve(*args, _ptr(rhs), _ptr(sol), tol, max_iter, ctypes.byref(steps),
                                   ctypes.byref(rel))
    return sol, it, steps.value, rel.value


# ----------------------------------------------------------------- assembled operators, preconditioner menu

PRECONDITIONERS = {"identity": 0, "jacobi": 1, "spd-isai": 2, "symmetric-gauss-seidel": 3, "ssor": 4,
                   "chebyshev-jacobi": 5, "ir-jacobi": 6, "general-isai": 7}
MENU_DEFAULTS = {"sor_relaxation_factor": 1.2, "chebyshev_iterations": 8, "chebyshev_lower_bound": 0.05,
                 "chebyshev_upper_bound": 1.5, "ir_iterations": 8, "ir_relaxation_factor": 1.0}


def _offset3(target, at):
    """The offset d in {-1, 0, 1} with (at + d) mod 3 == target."""
    d = (target - at % 3) % 3
    return np.where(d == 2, -1, d)


def _probe_assemble(dims, apply):
    """CSR of a linear operator whose row touches only columns in the 3x3
    (2D nodes) or 3x3x3 (3D nodes x 3 components) neighbourhood, by one apply
    per column colour (node coordinates mod 3, and component): columns of one
    colour never share a row.  Exact zeros are dropped, columns ascending."""
    import scipy.sparse as sp
    if len(dims) == 2:
        nx, ny = dims
        n = nx * ny
        r = np.arange(n)
        i, j, k = r % nx, r // nx, np.zeros(n, dtype=np.int64)
        colors = [(cx, cy, 0, None) for cy in range(3) for cx in range(3)]
        col_color = (r % nx) % 3 + 3 * ((r // nx) % 3)
    else:
        nx, ny, nz = dims
        n = 3 * nx * ny * nz
        r = np.arange(n)
        node = r // 3
        i, j, k = node % nx, (node // nx) % ny, node // (nx * ny)
        colors = [(cx, cy, cz, c) for cz in range(3) for cy in range(3) for cx in range(3) for c in range(3)]
        col_color = (r % 3) + 3 * (i % 3 + 3 * (j % 3) + 9 * (k % 3))
    rows, cols, vals = [], [], []
    for cx, cy, cz, c in colors:
        color = cx + 3 * cy if len(dims) == 2 else c + 3 * (cx + 3 * cy + 9 * cz)
        y = apply((col_color == color).astype(np.float64))
        di, dj = _offset3(cx, i), _offset3(cy, j)
        ok = (i + di >= 0) & (i + di < nx) & (j + dj >= 0) & (j + dj < ny)
        if len(dims) == 2:
            col = (i + di) + nx * (j + dj)
        else:
            dk = _offset3(cz, k)
            ok &= (k + dk >= 0) & (k + dk < nz)
            col = 3 * ((i + di) + nx * ((j + dj) + ny * (k + dk))) + c
        ok &= y != 0.0
        rows.append(r[ok])
        cols.append(col[ok])
        vals.append(y[ok])
    A = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    A.sort_indices()
    return A


def assemble2d(nx, ny, node_mu):
    """The 2D operator as a CSR matrix (the reference's assemble_matrix_data,
    onelab_interface/magnetostatics_onelab.hpp:3554-3737), probed through
    mag2d_apply with nine colours (i mod 3, j mod 3)."""
    return _probe_assemble((nx, ny), lambda v: mag2d_apply(nx, ny, node_mu, v))


def assemble3d(x, y, z, node_mu, gamma):
    """The 3D operator as a CSR matrix (magnetostatics_onelab.hpp:3120-3534),
    probed through mag3d_apply with 27 node colours times 3 components."""
    return _probe_assemble((len(x), len(y), len(z)), lambda v: mag3d_apply(x, y, z, node_mu, gamma, v))


def _csr_args(A):
    ptr = np.ascontiguousarray(A.indptr, dtype=np.int64)
    col = np.ascontiguousarray(A.indices, dtype=np.int32)
    val = np.ascontiguousarray(A.data, dtype=np.float64)
    keep = (ptr, col, val)
    args = [A.shape[0], ptr.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
            col.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _ptr(val)]
    return keep, args


def _menu_params(**kw):
    p = dict(MENU_DEFAULTS)
    p.update(kw)
    return np.array([p["sor_relaxation_factor"], p["chebyshev_iterations"], p["chebyshev_lower_bound"],
                     p["chebyshev_upper_bound"], p["ir_iterations"], p["ir_relaxation_factor"]], dtype=np.float64)


def csr_precond_apply(A, kind, r, **params):
    keep, args = _csr_args(A)
    pv = _menu_params(**params)
    r = _f64(r)
    z = np.zeros_like(r)
    rc = lib().silo_csr_precond_apply(*args, PRECONDITIONERS[kind], _ptr(pv), _ptr(r), _ptr(z))
    if rc != 0:
        raise ValueError("singular ISAI system")
    return z


def csr_isai_values(A, kind):
    """Values of the ISAI factor: Z on the pattern of tril(A) (spd-isai) or M on that of A (general-isai)."""
    import scipy.sparse as sp
    keep, args = _csr_args(A)
    pat = sp.tril(A, format="csr") if kind == "spd-isai" else A.copy()
    pat.sort_indices()
    out = np.zeros(pat.nnz)
    rc = lib().silo_csr_isai_values(*args, PRECONDITIONERS[kind], _ptr(out))
    if rc != 0:
        raise ValueError("singular ISAI system")
    pat.data = out
    return pat


def csr_pcg(A, b, kind="jacobi", tol=1e-10, max_iter=100000, **params):
    """Preconditioned CG from x = 0; returns (x, iterations, final relative residual)."""
    keep, args = _csr_args(A)
    pv = _menu_params(**params)
    b = _f64(b)
    x = np.zeros_like(b)
    rel = ctypes.c_double(0.0)
    it = lib().silo_csr_pcg(*args, PRECONDITIONERS[kind], _ptr(pv), _ptr(b), _ptr(x), tol, max_iter,
                            ctypes.byref(rel))
    if it < 0:
        raise ValueError("singular ISAI system")
    return x, it, rel.value


def jacobian2d_csr(nx, ny, node_mu, node_ferro, curve_b, curve_h, state):
    """The 2D nonlinear operator's Jacobian at `state` as a CSR matrix (probed)."""
    return _probe_assemble((nx, ny), lambda v: mag2d_nl_jacobian_apply(nx, ny, node_mu, node_ferro, curve_b, curve_h,
                                                                       state, v))


def mag2d_nl_solve_menu(nx, ny, node_mu, node_ferro, curve_b, curve_h, rhs, kind, x0=None, tol=1e-10,
                        max_iter=100000, **params):
    """Newton + line search, each linear solve a CG with the menu preconditioner on the assembled
    Jacobian; returns (x, cg_iterations, newton_steps, final relative residual)."""
    mu, fe, b, h, rhs = _f64(node_mu), _f64(node_ferro), _f64(curve_b), _f64(curve_h), _f64(rhs)
    pv = _menu_params(**params)
    x = np.zeros(nx * ny) if x0 is None else np.array(x0, dtype=np.float64)
    steps = ctypes.c_int(0)
    rel = ctypes.c_double(0.0)
    it = lib().silo_mag2d_nl_solve_menu(nx, ny, _ptr(mu), _ptr(fe), len(b), _ptr(b), _ptr(h), PRECONDITIONERS[kind],
                                        _ptr(pv), _ptr(rhs), _ptr(x), tol, max_iter, ctypes.byref(steps),
                                        ctypes.byref(rel))
    if it < 0:
        raise ValueError("singular ISAI system")
    return x, it, steps.value, rel.value


def mag3d_nl_solve_menu(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h, rhs, kind, x0=None, tol=1e-10,
                        max_iter=100000, **params):
    keep, args = _nl3_args(x, y, z, node_mu, node_ferro, gamma, curve_b, curve_h)
    pv = _menu_params(**params)
    rhs = _f64(rhs)
    sol = np.zeros_like(rhs) if x0 is None else np.array(x0, dtype=np.float64)
    steps = ctypes.c_int(0)
    rel = ctypes.c_double(0.0)
    it = lib().silo_mag3d_nl_solve_menu(*args, PRECONDITIONERS[kind], _ptr(pv), _ptr(rhs), _ptr(sol), tol, max_iter,
                                        ctypes.byref(steps), ctypes.byref(rel))
    if it < 0:
        raise ValueError("singular ISAI system")
    return sol, it, steps.value, rel.value


KRYLOV = {"cg": 0, "minres": 1, "fcg": 2, "gmres": 3, "bicgstab": 4, "gcr": 5, "idr": 6}
KRYLOV_DIMS = {"gmres": 100, "gcr": 100, "idr": 8}


def csr_krylov(A, b, solver="cg", kind="jacobi", tol=1e-10, max_iter=100000, dim=None, **params):
    """The reference's SIMILIE_SOLVER menu with a menu preconditioner, x from 0;
    returns (x, iterations, final relative residual)."""
    keep, args = _csr_args(A)
    pv = _menu_params(**params)
    b = _f64(b)
    x = np.zeros_like(b)
    rel = ctypes.c_double(0.0)
    d = KRYLOV_DIMS.get(solver, 0) if dim is None else dim
    it = lib().silo_csr_krylov(*args, KRYLOV[solver], d, PRECONDITIONERS[kind], _ptr(pv), _ptr(b), _ptr(x), tol,
                               max_iter, ctypes.byref(rel))
    if it < 0:
        raise ValueError("unknown solver or singular ISAI system")
    return x, it, rel.value


# ----------------------------------------------------------------- primal reduction / reconstruction

def reduce_primal(n, k, position, node, form):
    """Reduction<Primal>::run at one node of a position field ([...][n])."""
    fp = field(np.ascontiguousarray(position, dtype=np.float64))
    nd = np.ascontiguousarray(node, dtype=np.int64)
    f = _f64(form)
    out = np.zeros(binom(n, k))
    _check(lib().silo_reduce_primal(n, k, ctypes.byref(fp), nd.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                    _ptr(f), _ptr(out)), "reduce_primal")
    return out


def reconstruct_primal(n, k, position, node, cochain):
    """Reconstruction<Primal>::run at one node."""
    fp = field(np.ascontiguousarray(position, dtype=np.float64))
    nd = np.ascontiguousarray(node, dtype=np.int64)
    c = _f64(cochain)
    out = np.zeros(binom(n, k))
    _check(lib().silo_reconstruct_primal(n, k, ctypes.byref(fp), nd.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                         _ptr(c), _ptr(out)), "reconstruct_primal")
    return out
