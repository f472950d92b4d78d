"""CPU oracle of the nonlinear (saturating-material) 2D magnetostatics: the
interpolated B-H curve and its derivatives, the operator's reduction to the
linear operator for a straight curve, the Jacobian against a finite-difference
directional derivative, its diagonal and symmetry, and the Newton solve with
line search."""
import numpy as np
import pytest

import oracle as O
import similie_b200.magnetostatics as mag


def _problem(n, seed, cores=2):
    rng = np.random.default_rng(seed)
    p = mag.synthetic_problem(rng, n, cores=cores)
    mu = p.node_mu()
    ferro = mag.node_ferro(n, n, p.cell_mu > 1.0)
    b, h = mag.synthetic_bh_curve(mag.nonlinear_knee(n))
    return p, mu, ferro, b, h


def test_curve_values_and_derivatives():
    b, h = mag.synthetic_bh_curve(0.5, samples=16)
    # F at the samples is h/b
    q = b[1:] ** 2
    f, df, d2f = O.bh_eval(b, h, q)
    np.testing.assert_allclose(f, h[1:] / b[1:], rtol=1e-14)
    # derivatives against central differences inside the intervals
    mid = 0.5 * (b[1:-1] + b[2:])
    qm = mid ** 2
    eps = 1e-6 * qm
    fp, _, _ = O.bh_eval(b, h, qm + eps)
    fm, _, _ = O.bh_eval(b, h, qm - eps)
    _, df_m, d2f_m = O.bh_eval(b, h, qm)
    np.testing.assert_allclose(df_m, (fp - fm) / (2 * eps), rtol=1e-5)
    _, dfp, _ = O.bh_eval(b, h, qm + eps)
    _, dfm, _ = O.bh_eval(b, h, qm - eps)
    np.testing.assert_allclose(d2f_m, (dfp - dfm) / (2 * eps), rtol=1e-4)
    # q = 0: the first slope, no derivatives
    f0, df0, d2f0 = O.bh_eval(b, h, np.array([0.0]))
    assert f0[0] == (h[1] - h[0]) / (b[1] - b[0]) and df0[0] == 0.0 and d2f0[0] == 0.0


def test_straight_curve_gives_the_linear_operator():
    n = 33
    p, mu, _, _, _ = _problem(n, 1)
    rng = np.random.default_rng(2)
    a = rng.standard_normal(n * n)
    b = np.linspace(0.0, 2.0, 5)
    h = b / 1000.0
    ferro = np.ones(n * n)
    y_nl = O.mag2d_nl_apply(n, n, mu, ferro, b, h, a)
    y_lin = O.mag2d_apply(n, n, np.full(n * n, 1000.0), a)
    np.testing.assert_allclose(y_nl, y_lin, rtol=1e-12, atol=1e-15 * np.abs(y_lin).max())
    # no ferromagnetic node: the linear operator with the node permeability
    y0 = O.mag2d_nl_apply(n, n, mu, np.zeros(n * n), b, h, a)
    np.testing.assert_array_equal(y0, O.mag2d_apply(n, n, mu, a))


@pytest.mark.parametrize("seed", [3, 4])
def test_jacobian_is_the_derivative_of_the_operator(seed):
    n = 33
    p, mu, ferro, b, h = _problem(n, seed)
    rng = np.random.default_rng(seed + 10)
    # a state whose moments reach the saturated part of the curve
    st = rng.standard_normal(n * n) * 3 * b[-1]
    x = rng.standard_normal(n * n)
    jx = O.mag2d_nl_jacobian_apply(n, n, mu, ferro, b, h, st, x)
    eps = 1e-7
    fd = (O.mag2d_nl_apply(n, n, mu, ferro, b, h, st + eps * x)
          - O.mag2d_nl_apply(n, n, mu, ferro, b, h, st - eps * x)) / (2 * eps)
    assert np.linalg.norm(jx - fd) <= 1e-5 * np.linalg.norm(jx)
    # symmetric
    y = rng.standard_normal(n * n)
    y2 = y.reshape(n, n).copy()
    x2 = x.reshape(n, n).copy()
    for v in (y2, x2):  # interior-only vectors: boundary rows are identity, not part of the symmetric block
        v[0] = v[-1] = 0
        v[:, 0] = v[:, -1] = 0
    xi, yi = x2.ravel(), y2.ravel()
    a1 = yi @ O.mag2d_nl_jacobian_apply(n, n, mu, ferro, b, h, st, xi)
    a2 = xi @ O.mag2d_nl_jacobian_apply(n, n, mu, ferro, b, h, st, yi)
    assert abs(a1 - a2) <= 1e-10 * max(abs(a1), 1e-300)
    # diagonal
    dg = O.mag2d_nl_jacobian_diagonal(n, n, mu, ferro, b, h, st)
    for row in (n + 1, 5 * n + 7, (n // 2) * n + n // 2, n * n - n - 2):
        e = np.zeros(n * n)
        e[row] = 1.0
        assert dg[row] == pytest.approx(O.mag2d_nl_jacobian_apply(n, n, mu, ferro, b, h, st, e)[row], rel=1e-13)


@pytest.mark.parametrize("n", [49, 65])
def test_newton_solve_converges(n):
    p, mu, ferro, b, h = mag.nonlinear_problem(n, 3)
    rhs = p.rhs()
    x, it, steps, rel = O.mag2d_nl_solve(n, n, mu, ferro, b, h, rhs, tol=1e-10)
    assert rel <= 1e-10
    assert steps >= 3, "the material should make the problem nonlinear"
    r = rhs - O.mag2d_nl_apply(n, n, mu, ferro, b, h, x)
    assert np.linalg.norm(r) <= 1e-10 * np.linalg.norm(rhs)
    # the saturated solution differs from the linear one
    xl, _, _ = O.mag2d_cg(n, n, mu, rhs, tol=1e-12)
    assert np.linalg.norm(x - xl) > 1e-3 * np.linalg.norm(xl)


def test_straight_curve_solves_in_one_step():
    n = 33
    p, mu, _, _, _ = _problem(n, 8)
    b = np.linspace(0.0, 1.0, 4)
    h = b / 1000.0
    ferro = mag.node_ferro(n, n, p.cell_mu > 1.0)
    mu_eff = np.where(ferro > 0.5, 1000.0, mu)
    x, it, steps, rel = O.mag2d_nl_solve(n, n, mu, ferro, b, h, p.rhs(), tol=1e-10)
    assert rel <= 1e-10 and steps == 1
    xl, _, _ = O.mag2d_cg(n, n, mu_eff, p.rhs(), tol=1e-12)
    assert np.linalg.norm(x - xl) <= 1e-8 * np.linalg.norm(xl)
