"""CPU restatement of the reference's SIMILIE_SOLVER menu (CG, MINRES, FCG,
GMRES, BiCGSTAB, GCR, IDR) on the assembled operators: every solver with two
menu preconditioners reaches the tolerance with a matching true residual and
the direct solution, and the identities between methods hold (FCG = CG for a
fixed preconditioner, GMRES(m) = GCR(m), MINRES ~ CG on an SPD problem)."""
import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

import oracle as O
import similie_b200.magnetostatics as mag
import similie_b200.magnetostatics3d as m3


@pytest.fixture(scope="module")
def case2d():
    rng = np.random.default_rng(11)
    p = mag.synthetic_problem(rng, 33, cores=2)
    A = O.assemble2d(33, 33, p.node_mu())
    b = p.rhs()
    return A, b, spla.spsolve(A.tocsc(), b)


@pytest.mark.parametrize("solver", list(O.KRYLOV))
@pytest.mark.parametrize("kind", ["jacobi", "ssor"])
def test_every_solver_reaches_the_tolerance(case2d, solver, kind):
    A, b, xd = case2d
    x, it, rel = O.csr_krylov(A, b, solver, kind, tol=1e-10, max_iter=20000)
    true = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert 0 < it < 20000 and rel <= 1e-10 and true <= 2e-10
    assert np.linalg.norm(x - xd) <= 1e-8 * np.linalg.norm(xd)


def test_identities_between_methods(case2d):
    A, b, _ = case2d
    its = {s: O.csr_krylov(A, b, s, "jacobi", tol=1e-10)[1] for s in O.KRYLOV}
    assert its["fcg"] == its["cg"]
    assert its["gmres"] == its["gcr"]
    # restarting after 5 directions costs iterations but still converges
    _, it5, rel5 = O.csr_krylov(A, b, "gmres", "jacobi", tol=1e-10, dim=5, max_iter=50000)
    assert rel5 <= 1e-10 and it5 > its["gmres"]
    # on a symmetric positive definite matrix MINRES and CG take about the same steps
    S = (A + A.T) * 0.5 + sp.identity(A.shape[0], format="csr") * 1e-3
    i_cg = O.csr_krylov(S, b, "cg", "jacobi", tol=1e-10)[1]
    i_mr = O.csr_krylov(S, b, "minres", "jacobi", tol=1e-10)[1]
    assert abs(i_cg - i_mr) <= max(3, i_cg // 10)


@pytest.mark.parametrize("solver", ["gmres", "bicgstab", "idr", "minres"])
def test_solvers_on_the_3d_operator(solver):
    rng = np.random.default_rng(6)
    pr = m3.synthetic_problem(rng, 9, tube=0.2)
    A = O.assemble3d(pr.x, pr.y, pr.z, pr.node_mu(), pr.gamma)
    b = pr.rhs()
    x, it, rel = O.csr_krylov(A, b, solver, "jacobi", tol=1e-10, max_iter=20000)
    assert rel <= 1e-10
    assert np.linalg.norm(b - A @ x) <= 2e-10 * np.linalg.norm(b)
