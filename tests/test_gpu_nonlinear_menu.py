"""GPU nonlinear solves with the reference's preconditioner menu: the
Jacobian assembled at the state against the oracle's, and Newton whose
linear solves run CG with SSOR / SpdIsai on the assembled Jacobian against
the oracle's same scheme (Newton steps, CG iterations, solution)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


def test_assembled_jacobian_2d_matches_the_oracle(torch):
    import similie_b200.assembled as asm
    import similie_b200.magnetostatics as mag
    n = 33
    p, mu, fe, b, h = mag.nonlinear_problem(n, 4)
    rng = np.random.default_rng(7)
    st = rng.standard_normal(n * n) * 3 * b[-1]
    c = mag._Curve(b, h)
    mu_d, fe_d = _dev(torch, mu), _dev(torch, fe)
    prob = mag._nl_problem(n, n, mu_d, fe_d, c)
    J = asm.jacobian2d(prob, _dev(torch, st)).to_scipy()
    R = O.jacobian2d_csr(n, n, mu, fe, b, h, st)
    assert abs(J - R).max() <= 1e-12 * np.abs(R.data).max()


@pytest.mark.parametrize("kind", ["ssor", "spd-isai"])
def test_menu_newton_2d_matches_the_oracle(torch, kind):
    import similie_b200.magnetostatics as mag
    n = 49
    p, mu, fe, b, h = mag.nonlinear_problem(n, 3)
    rhs = p.rhs()
    x = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    d = mag.nl_solve_batch([_dev(torch, mu)], [_dev(torch, fe)], [(b, h)], [_dev(torch, rhs)], [x], [(n, n)],
                           tol=1e-10, jacobian_preconditioner=kind)[0]
    xo, it, steps, rel = O.mag2d_nl_solve_menu(n, n, mu, fe, b, h, rhs, kind, tol=1e-10)
    assert d.converged and d.status == 0 and d.refinements == steps
    assert abs(d.iterations - it) <= max(3, it // 20)
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-8 * np.linalg.norm(xo)


def test_menu_newton_3d_matches_the_oracle(torch):
    import similie_b200.magnetostatics3d as m3
    p, mu, fe, b, h = m3.nonlinear_problem(13, 6)
    rhs = p.rhs()
    x = torch.zeros(rhs.size, dtype=torch.float64, device="cuda")
    d = m3.nl_solve_batch([(p.x, p.y, p.z)], [_dev(torch, mu)], [_dev(torch, fe)], [(b, h)], [_dev(torch, rhs)], [x],
                          tol=1e-10, jacobian_preconditioner="ssor")[0]
    xo, it, steps, rel = O.mag3d_nl_solve_menu(p.x, p.y, p.z, mu, fe, p.gamma, b, h, rhs, "ssor", tol=1e-10)
    assert d.converged and d.refinements == steps
    assert abs(d.iterations - it) <= max(3, it // 20)
    assert np.linalg.norm(x.cpu().numpy() - xo) <= 1e-8 * np.linalg.norm(xo)
