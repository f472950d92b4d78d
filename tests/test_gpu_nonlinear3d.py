"""GPU nonlinear (saturating-material) 3D magnetostatics against the CPU
oracle: the operator and its Jacobian on saturated states over anisotropic
grids, the Newton solve with line search (same Newton steps, solution and
1e-10 residual as the oracle), the straight-curve limit against the linear
3D solver, and a zero right-hand side."""
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
def m3():
    import similie_b200.magnetostatics3d as m
    return m


@pytest.fixture(scope="module")
def mag():
    import similie_b200.magnetostatics as m
    return m


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.mark.parametrize("shape", [(9, 10, 8), (17, 13, 11), (33, 20, 24)])
def test_operator_and_jacobian_match_the_oracle(torch, m3, mag, shape):
    rng = np.random.default_rng(sum(shape))
    x, y, z = [np.cumsum(rng.uniform(0.5, 1.5, n)) / n for n in shape]
    nodes = int(np.prod(shape))
    mu = rng.choice([1.0, 1000.0, 500.5], nodes)
    ferro = rng.choice([0.0, 0.5, 0.75, 1.0], nodes)
    b, h = mag.synthetic_bh_curve(0.3)
    st = rng.standard_normal(3 * nodes) * 1.5      # moments well past the knee and the last sample
    v = rng.standard_normal(3 * nodes)
    gamma = 12.5
    out = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    m3.nl_apply(x, y, z, _dev(torch, mu), _dev(torch, ferro), b, h, _dev(torch, st), out, gamma=gamma)
    ref = O.mag3d_nl_apply(x, y, z, mu, ferro, gamma, b, h, st)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    m3.nl_apply_jacobian(x, y, z, _dev(torch, mu), _dev(torch, ferro), b, h, _dev(torch, st), _dev(torch, v), out,
                         gamma=gamma)
    ref = O.mag3d_nl_jacobian_apply(x, y, z, mu, ferro, gamma, b, h, st, v)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-12, atol=1e-13 * np.abs(ref).max())


def test_newton_solve_matches_the_oracle(torch, m3):
    cases = [m3.nonlinear_problem(n, seed) + (n,) for n, seed in ((17, 3), (17, 4), (13, 6))]
    coords = [(c[0].x, c[0].y, c[0].z) for c in cases]
    mus = [_dev(torch, c[1]) for c in cases]
    ferros = [_dev(torch, c[2]) for c in cases]
    rhss = [_dev(torch, c[0].rhs()) for c in cases]
    sols = [torch.zeros_like(r) for r in rhss]
    d = m3.nl_solve_batch(coords, mus, ferros, [(c[3], c[4]) for c in cases], rhss, sols, tol=1e-10)
    for (p, mu, ferro, b, h, n), xs, dg in zip(cases, sols, d):
        assert dg.converged and dg.status == 0, dg
        xo, it, steps, rel = O.mag3d_nl_solve(p.x, p.y, p.z, mu, ferro, p.gamma, b, h, p.rhs(), tol=1e-10)
        assert dg.refinements == steps
        xg = xs.cpu().numpy()
        rhs = p.rhs()
        r = rhs - O.mag3d_nl_apply(p.x, p.y, p.z, mu, ferro, p.gamma, b, h, xg)
        assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(rhs)
        assert np.linalg.norm(xg - xo) <= 1e-8 * np.linalg.norm(xo)


def test_straight_curve_matches_the_linear_solver(torch, m3):
    n = 24
    p, mu, ferro, _, _ = m3.nonlinear_problem(n, 21)
    b = np.linspace(0.0, 1.0, 4)
    h = b / 1000.0
    mu_eff = np.where(ferro > 0.5, 1000.0, mu)
    rhs = _dev(torch, p.rhs())
    xs = torch.zeros_like(rhs)
    coords = [(p.x, p.y, p.z)]
    d = m3.nl_solve_batch(coords, [_dev(torch, mu)], [_dev(torch, ferro)], [(b, h)], [rhs], [xs], tol=1e-10)
    # one step solves the linear problem; the CG's recursive residual may leave the true one just above
    # the tolerance, and a second step then finishes
    assert d[0].converged and d[0].refinements <= 2
    xl = torch.zeros_like(rhs)
    m3.solve_batch(coords, [_dev(torch, mu_eff)], [rhs], [xl], solver="cg", tol=1e-12)
    assert float(torch.linalg.norm(xs - xl) / torch.linalg.norm(xl)) <= 1e-8


def test_zero_rhs_needs_no_step(torch, m3):
    p, mu, ferro, b, h = m3.nonlinear_problem(9, 2, tube=0.2)
    rhs = torch.zeros(3 * 9 ** 3, dtype=torch.float64, device="cuda")
    xs = torch.zeros_like(rhs)
    d = m3.nl_solve_batch([(p.x, p.y, p.z)], [_dev(torch, mu)], [_dev(torch, ferro)], [(b, h)], [rhs], [xs])
    assert d[0].converged and d[0].refinements == 0 and d[0].iterations == 0
    assert float(torch.abs(xs).max()) == 0.0
