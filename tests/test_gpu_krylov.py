"""GPU Krylov menu (the reference's SIMILIE_SOLVER choices) on the assembled
operators against the CPU restatement: every method with two menu
preconditioners reaches the tolerance with the restatement's iteration count
(up to reduction-order drift), the true residual and the direct solution."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla

import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def case2d(torch):
    import similie_b200.assembled as asm
    import similie_b200.magnetostatics as mag
    rng = np.random.default_rng(11)
    p = mag.synthetic_problem(rng, 33, cores=2)
    mu = p.node_mu()
    A = asm.CsrMatrix.mag2d(33, 33, torch.from_numpy(mu).cuda())
    G = A.to_scipy()
    b = p.rhs()
    return A, G, b, spla.spsolve(G.tocsc(), b)


@pytest.mark.parametrize("solver", ["minres", "fcg", "gmres", "bicgstab", "gcr", "idr"])
@pytest.mark.parametrize("kind", ["jacobi", "ssor"])
def test_krylov_matches_the_restatement(torch, case2d, solver, kind):
    import similie_b200.assembled as asm
    A, G, b, xd = case2d
    P = asm.Preconditioner(A, kind)
    x = torch.zeros(G.shape[0], dtype=torch.float64, device="cuda")
    d = asm.solve(A, P, torch.from_numpy(b).cuda(), x, tol=1e-10, max_iterations=20000, solver=solver)
    xo, it, rel = O.csr_krylov(G, b, solver, kind, tol=1e-10, max_iter=20000)
    assert d.converged and d.status == 0
    assert abs(d.iterations - it) <= max(3, it // 10)
    xg = x.cpu().numpy()
    assert np.linalg.norm(b - G @ xg) <= 2e-10 * np.linalg.norm(b)
    assert np.linalg.norm(xg - xd) <= 1e-8 * np.linalg.norm(xd)


def test_krylov_on_the_3d_operator(torch):
    import similie_b200.assembled as asm
    import similie_b200.magnetostatics3d as m3
    rng = np.random.default_rng(6)
    pr = m3.synthetic_problem(rng, 9, tube=0.2)
    A = asm.CsrMatrix.mag3d(pr.x, pr.y, pr.z, torch.from_numpy(pr.node_mu()).cuda(), gamma=pr.gamma)
    G = A.to_scipy()
    b = pr.rhs()
    P = asm.Preconditioner(A, "jacobi")
    for solver in ("gmres", "bicgstab", "idr"):
        x = torch.zeros(G.shape[0], dtype=torch.float64, device="cuda")
        d = asm.solve(A, P, torch.from_numpy(b).cuda(), x, tol=1e-10, max_iterations=20000, solver=solver)
        assert d.converged, solver
        assert np.linalg.norm(b - G @ x.cpu().numpy()) <= 2e-10 * np.linalg.norm(b)
