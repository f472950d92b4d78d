"""The 3D nonlinear operator with the divergence gauge on the GPU: the
operator and its Jacobian against the oracle's nonlinear curl-curl (penalty
off) plus the divergence-gauge term of the reference restated in
tests/test_divergence_gauge.py, and the straight-curve solve against the
linear divergence-gauge solve."""
import numpy as np
import pytest

import oracle as O
from test_divergence_gauge import gauge_term, probe_coefficients

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def _gauge(x, y, z, gamma, v):
    E0, E1, w = probe_coefficients(x, y, z)
    n = (len(x), len(y), len(z))
    A = v.reshape(n[2], n[1], n[0], 3).transpose(2, 1, 0, 3)       # [x][y][z][3]
    G = gauge_term(E0, E1, w, A).transpose(2, 1, 0, 3).ravel()       # back to the solver layout
    interior = np.zeros((n[2], n[1], n[0], 3), dtype=bool)
    interior[1:-1, 1:-1, 1:-1] = True
    return gamma * np.where(interior.ravel(), G, 0.0)


def test_gauged_operator_and_jacobian_match_the_oracle(torch):
    import similie_b200.magnetostatics as mag
    import similie_b200.magnetostatics3d as m3
    rng = np.random.default_rng(31)
    shape = (9, 8, 10)
    x, y, z = [np.cumsum(rng.uniform(0.5, 1.5, k)) / k for k in shape]
    nodes = int(np.prod(shape))
    mu = rng.choice([1.0, 1000.0], nodes)
    ferro = rng.choice([0.0, 1.0], nodes)
    b, h = mag.synthetic_bh_curve(0.3)
    st = rng.standard_normal(3 * nodes) * 1.5
    v = rng.standard_normal(3 * nodes)
    gamma = -4.0
    out = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    m3.nl_apply(x, y, z, _dev(torch, mu), _dev(torch, ferro), b, h, _dev(torch, st), out, gamma=gamma,
                gauge="divergence")
    ref = O.mag3d_nl_apply(x, y, z, mu, ferro, 0.0, b, h, st) + _gauge(x, y, z, gamma, st)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())
    m3.nl_apply_jacobian(x, y, z, _dev(torch, mu), _dev(torch, ferro), b, h, _dev(torch, st), _dev(torch, v), out,
                         gamma=gamma, gauge="divergence")
    ref = O.mag3d_nl_jacobian_apply(x, y, z, mu, ferro, 0.0, b, h, st, v) + _gauge(x, y, z, gamma, v)
    np.testing.assert_allclose(out.cpu().numpy(), ref, rtol=1e-11, atol=1e-11 * np.abs(ref).max())


def test_straight_curve_matches_the_linear_divergence_gauge_solve(torch):
    import similie_b200.magnetostatics3d as m3
    p, mu, ferro, _, _ = m3.nonlinear_problem(13, 6)
    b = np.linspace(0.0, 1.0, 4)
    h = b / 1000.0
    mu_eff = np.where(ferro > 0.5, 1000.0, mu)
    rhs = _dev(torch, p.rhs())
    coords = [(p.x, p.y, p.z)]
    x = torch.zeros_like(rhs)
    d = m3.nl_solve_batch(coords, [_dev(torch, mu)], [_dev(torch, ferro)], [(b, h)], [rhs], [x], tol=1e-10,
                          gammas=[p.gamma], gauge="divergence")
    assert d[0].converged and d[0].refinements <= 2
    xl = torch.zeros_like(rhs)
    m3.solve_batch(coords, [_dev(torch, mu_eff)], [rhs], [xl], gammas=[p.gamma], solver="cg", tol=1e-12,
                   gauge="divergence")
    assert float(torch.linalg.norm(x - xl) / torch.linalg.norm(xl)) <= 1e-8
