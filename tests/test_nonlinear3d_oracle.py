"""CPU oracle of the nonlinear (saturating-material) 3D magnetostatics: the
operator's reduction to the linear 3D operator (no ferromagnetic node, or a
straight curve), the Jacobian against a finite-difference directional
derivative, its symmetry and diagonal, and the Newton solve with line
search."""
import numpy as np
import pytest

import oracle as O
import similie_b200.magnetostatics as mag
import similie_b200.magnetostatics3d as m3


def _grid(rng, nx, ny, nz):
    return [np.cumsum(rng.uniform(0.5, 1.5, n)) / n for n in (nx, ny, nz)]


def _random_case(shape, seed):
    rng = np.random.default_rng(seed)
    x, y, z = _grid(rng, *shape)
    nodes = int(np.prod(shape))
    mu = rng.choice([1.0, 1000.0, 500.5], nodes)
    ferro = rng.choice([0.0, 0.5, 0.75, 1.0], nodes)
    return rng, x, y, z, mu, ferro


def test_without_ferromagnetic_nodes_it_is_the_linear_operator():
    rng, x, y, z, mu, _ = _random_case((9, 8, 7), 1)
    b, h = mag.synthetic_bh_curve(0.3)
    a = rng.standard_normal(3 * 9 * 8 * 7)
    y0 = O.mag3d_nl_apply(x, y, z, mu, np.zeros(mu.size), 20.0, b, h, a)
    np.testing.assert_array_equal(y0, O.mag3d_apply(x, y, z, mu, 20.0, a))


def test_straight_curve_gives_the_linear_operator():
    rng, x, y, z, mu, _ = _random_case((8, 9, 10), 2)
    a = rng.standard_normal(3 * mu.size)
    b = np.linspace(0.0, 2.0, 5)
    h = b / 1000.0
    y_nl = O.mag3d_nl_apply(x, y, z, mu, np.ones(mu.size), 7.5, b, h, a)
    y_lin = O.mag3d_apply(x, y, z, np.full(mu.size, 1000.0), 7.5, a)
    np.testing.assert_allclose(y_nl, y_lin, rtol=1e-12, atol=1e-14 * np.abs(y_lin).max())


@pytest.mark.parametrize("seed", [3, 4])
def test_jacobian_is_the_derivative_of_the_operator(seed):
    shape = (9, 10, 8)
    rng, x, y, z, mu, ferro = _random_case(shape, seed)
    b, h = mag.synthetic_bh_curve(0.3)
    n = 3 * mu.size
    st = rng.standard_normal(n) * 1.5          # moments well past the knee and the last sample
    v = rng.standard_normal(n)
    jv = O.mag3d_nl_jacobian_apply(x, y, z, mu, ferro, 20.0, b, h, st, v)
    eps = 1e-7
    fd = (O.mag3d_nl_apply(x, y, z, mu, ferro, 20.0, b, h, st + eps * v)
          - O.mag3d_nl_apply(x, y, z, mu, ferro, 20.0, b, h, st - eps * v)) / (2 * eps)
    assert np.linalg.norm(jv - fd) <= 1e-5 * np.linalg.norm(jv)
    inner = np.zeros(shape[::-1] + (3,), dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.ravel()
    # diagonal = J e_row at interior rows of every component
    dg = O.mag3d_nl_jacobian_diagonal(x, y, z, mu, ferro, 20.0, b, h, st)
    rows = np.flatnonzero(inner)
    for row in rng.choice(rows, 24, replace=False):
        e = np.zeros(n)
        e[row] = 1.0
        assert dg[row] == pytest.approx(O.mag3d_nl_jacobian_apply(x, y, z, mu, ferro, 20.0, b, h, st, e)[row],
                                        rel=1e-13)
    assert np.all(dg[~inner] == 1.0)


def test_jacobian_symmetry_follows_the_hodge_weights():
    """Row m of a ferromagnetic node's Hessian is weighted by hodge_m, so the
    Jacobian is symmetric where the three weights agree (uniform spacing) and
    not on an anisotropic grid, as in the reference (which runs CG on it)."""
    shape = (8, 8, 8)
    rng = np.random.default_rng(11)
    nodes = int(np.prod(shape))
    mu = rng.choice([1.0, 1000.0], nodes)
    ferro = rng.choice([0.0, 1.0], nodes)
    b, h = mag.synthetic_bh_curve(0.3)
    n = 3 * nodes
    st = rng.standard_normal(n) * 1.5
    inner = np.zeros(shape[::-1] + (3,), dtype=bool)
    inner[1:-1, 1:-1, 1:-1] = True
    inner = inner.ravel()
    v = np.where(inner, rng.standard_normal(n), 0.0)
    w = np.where(inner, rng.standard_normal(n), 0.0)

    def asym(x, y, z):
        a1 = w @ O.mag3d_nl_jacobian_apply(x, y, z, mu, ferro, 20.0, b, h, st, v)
        a2 = v @ O.mag3d_nl_jacobian_apply(x, y, z, mu, ferro, 20.0, b, h, st, w)
        return abs(a1 - a2) / abs(a1)

    uniform = np.linspace(0.0, 1.0, 8)
    assert asym(uniform, uniform, uniform) <= 1e-12
    assert asym(*_grid(rng, *shape)) > 1e-6


@pytest.mark.parametrize("n,seed", [(17, 3), (13, 6)])
def test_newton_solve_converges(n, seed):
    p, mu, ferro, b, h = m3.nonlinear_problem(n, seed)
    rhs = p.rhs()
    x, it, steps, rel = O.mag3d_nl_solve(p.x, p.y, p.z, mu, ferro, p.gamma, b, h, rhs, tol=1e-10)
    assert rel <= 1e-10
    assert steps >= 2, "the material should make the problem nonlinear"
    r = rhs - O.mag3d_nl_apply(p.x, p.y, p.z, mu, ferro, p.gamma, b, h, x)
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(rhs)
    xl, _, _ = O.mag3d_cg(p.x, p.y, p.z, mu, p.gamma, rhs, tol=1e-12)
    assert np.linalg.norm(x - xl) > 1e-5 * np.linalg.norm(xl)


def test_straight_curve_solves_in_one_step():
    n = 11
    p, mu, ferro, _, _ = m3.nonlinear_problem(n, 8)
    b = np.linspace(0.0, 1.0, 4)
    h = b / 1000.0
    mu_eff = np.where(ferro > 0.5, 1000.0, mu)
    x, it, steps, rel = O.mag3d_nl_solve(p.x, p.y, p.z, mu, ferro, p.gamma, b, h, p.rhs(), tol=1e-10)
    assert rel <= 1e-10 and steps == 1
    xl, _, _ = O.mag3d_cg(p.x, p.y, p.z, mu_eff, p.gamma, p.rhs(), tol=1e-12)
    assert np.linalg.norm(x - xl) <= 1e-8 * np.linalg.norm(xl)
