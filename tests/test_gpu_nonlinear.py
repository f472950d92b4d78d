"""GPU nonlinear (saturating-material) 2D magnetostatics against the CPU
oracle: the residual operator and its Jacobian on saturated states, the
Newton solve with line search (same Newton steps, solution and 1e-10
residual as the oracle), the straight-curve limit against the linear solver,
and argument checks."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def mag():
    import similie_b200.magnetostatics as m
    return m


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("shape", [(49, 49), (64, 37), (130, 96)])
def test_operator_and_jacobian_match_the_oracle(torch, mag, shape):
    nx, ny = shape
    rng = np.random.default_rng(nx * 7 + ny)
    mu = rng.choice([1.0, 1000.0, 500.5], nx * ny)
    ferro = rng.choice([0.0, 0.5, 0.75, 1.0], nx * ny)
    b, h = mag.synthetic_bh_curve(0.3)
    st = rng.standard_normal(nx * ny) * 1.5       # moments well past the knee and the last sample
    x = rng.standard_normal(nx * ny)
    y = torch.zeros(nx * ny, dtype=torch.float64, device="cuda")
    mag.nl_apply(_dev(torch, mu), _dev(torch, ferro), b, h, _dev(torch, st), y, nx, ny)
    ref = O.mag2d_nl_apply(nx, ny, mu, ferro, b, h, st)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    mag.nl_apply_jacobian(_dev(torch, mu), _dev(torch, ferro), b, h, _dev(torch, st), _dev(torch, x), y, nx, ny)
    ref = O.mag2d_nl_jacobian_apply(nx, ny, mu, ferro, b, h, st, x)
    np.testing.assert_allclose(y.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


def test_newton_solve_matches_the_oracle(torch, mag):
    cases = [mag.nonlinear_problem(n, 3) + (n,) for n in (49, 65)]
    mus = [_dev(torch, c[1]) for c in cases]
    ferros = [_dev(torch, c[2]) for c in cases]
    rhss = [_dev(torch, c[0].rhs()) for c in cases]
    sols = [torch.zeros_like(r) for r in rhss]
    shapes = [(c[5], c[5]) for c in cases]
    d = mag.nl_solve_batch(mus, ferros, [(c[3], c[4]) for c in cases], rhss, sols, shapes, tol=1e-10)
    for (p, mu, ferro, b, h, n), x, dg in zip(cases, sols, d):
        assert dg.converged and dg.status == 0, dg
        xo, it, steps, rel = O.mag2d_nl_solve(n, n, mu, ferro, b, h, p.rhs(), tol=1e-10)
        assert dg.refinements == steps
        xg = x.cpu().numpy()
        rhs = p.rhs()
        r = rhs - O.mag2d_nl_apply(n, n, mu, ferro, b, h, xg)
        assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(rhs)
        assert np.linalg.norm(xg - xo) <= 1e-8 * np.linalg.norm(xo)


def test_straight_curve_matches_the_linear_solver(torch, mag):
    n = 96
    rng = np.random.default_rng(21)
    p = mag.synthetic_problem(rng, n, cores=2)
    mu = p.node_mu()
    ferro = mag.node_ferro(n, n, p.cell_mu > 1.0)
    b = np.linspace(0.0, 1.0, 4)
    h = b / 1000.0
    mu_eff = np.where(ferro > 0.5, 1000.0, mu)
    rhs = _dev(torch, p.rhs())
    x = torch.zeros_like(rhs)
    d = mag.nl_solve_batch([_dev(torch, mu)], [_dev(torch, ferro)], [(b, h)], [rhs], [x], [(n, n)], tol=1e-10)
    assert d[0].converged and d[0].refinements == 1
    xl = torch.zeros_like(rhs)
    mag.solve_batch([_dev(torch, mu_eff)], [rhs], [xl], [(n, n)], solver="cg", tol=1e-12)
    assert float(torch.linalg.norm(x - xl) / torch.linalg.norm(xl)) <= 1e-8


def test_bad_curves_are_rejected(torch, mag):
    from similie_b200._native import SilError
    n = 16
    z = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    for b, h in (([0.0, 1.0, 1.0], [0.0, 1.0, 2.0]),      # b not strictly increasing
                 ([0.0], [0.0]),                          # fewer than 2 samples
                 (np.linspace(0, 1, 65), np.linspace(0, 1, 65))):  # more than 64
        with pytest.raises(SilError):
            mag.nl_apply(z, z, np.asarray(b), np.asarray(h), z, z.clone(), n, n)
