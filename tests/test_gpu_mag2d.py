"""GPU magnetostatics: operator parity with the oracle and batched solves that
reach the FP64 1e-10 relative residual measured by the oracle's operator."""
import numpy as np
import pytest

import oracle as O
from helpers import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def mag():
    import similie_b200.magnetostatics as m
    import similie_b200
    similie_b200.lib()
    return m


def test_host_setup_matches_oracle(mag):
    rng = np.random.default_rng(0)
    p = mag.synthetic_problem(rng, 33)
    np.testing.assert_allclose(p.node_mu(), O.mag2d_node_mu(p.nx, p.ny, p.cell_mu), rtol=1e-15)
    np.testing.assert_allclose(p.rhs(), O.mag2d_rhs(p.x, p.y, p.cell_j), rtol=1e-14, atol=1e-18)


@pytest.mark.parametrize("n", [5, 33, 130])
def test_apply_matches_oracle(torch, mag, n):
    rng = np.random.default_rng(n)
    p = mag.synthetic_problem(rng, n)
    mu = p.node_mu()
    a = rng.standard_normal(n * n)
    ref = O.mag2d_apply(n, n, mu, a)
    tm = torch.from_numpy(mu).cuda()
    ta = torch.from_numpy(a).cuda()
    ty = torch.zeros_like(ta)
    mag.apply(tm, ta, ty, n, n)
    assert rel_err(ty.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("solver", ["cg", "mixed"])
def test_batched_solve_reaches_tolerance(torch, mag, solver):
    rng = np.random.default_rng(11)
    probs = [mag.synthetic_problem(rng, n) for n in (17, 64, 128, 33, 96)]
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    sols = [torch.zeros_like(r) for r in rhss]
    diags = mag.solve_batch(mus, rhss, sols, [(p.nx, p.ny) for p in probs], solver=solver, tol=1e-10)
    for p, d, x in zip(probs, diags, sols):
        assert d.converged, d
        xb = x.cpu().numpy()
        b = p.rhs()
        r = b - O.mag2d_apply(p.nx, p.ny, p.node_mu(), xb)
        rel = np.linalg.norm(r) / np.linalg.norm(b)
        assert rel <= 1e-10, (p.nx, rel, d)
        assert abs(rel - d.final_relative_residual) <= 1e-12 + 1e-3 * rel
        # same solution as the oracle's CG (both converged to 1e-10)
        xo, _, _ = O.mag2d_cg(p.nx, p.ny, p.node_mu(), b, tol=1e-12)
        assert rel_err(xb, xo) < 1e-6
