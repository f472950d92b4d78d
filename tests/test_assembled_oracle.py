"""CPU oracle of the assembled-operator path: the probed CSR matrices against
the matrix-free operators, and the reference's preconditioner menu against
the defining property of each algorithm (FSAI's unit diagonal, ISAI's
interpolation, the SSOR factorisation, Chebyshev and Richardson convergence
on a known spectrum), then preconditioned CG with every menu entry."""
import numpy as np
import pytest
import scipy.sparse as sp

import oracle as O
import similie_b200.magnetostatics as mag
import similie_b200.magnetostatics3d as m3


def _problem2d(n=17, seed=1):
    rng = np.random.default_rng(seed)
    p = mag.synthetic_problem(rng, n, cores=2)
    return p, p.node_mu()


def test_assembled_2d_matches_the_operator():
    rng = np.random.default_rng(4)
    nx, ny = 13, 9
    mu = rng.choice([1.0, 1000.0, 500.5], nx * ny)
    A = O.assemble2d(nx, ny, mu)
    for _ in range(3):
        v = rng.standard_normal(nx * ny)
        np.testing.assert_allclose(A @ v, O.mag2d_apply(nx, ny, mu, v), rtol=1e-13, atol=1e-12)
    assert np.all(np.diff(A.indptr) <= 9) and A.has_sorted_indices
    assert np.all(A.data != 0.0)


def test_assembled_3d_matches_the_operator():
    rng = np.random.default_rng(5)
    x, y, z = [np.cumsum(rng.uniform(0.5, 1.5, n)) / n for n in (6, 5, 7)]
    mu = rng.choice([1.0, 1000.0], 6 * 5 * 7)
    A = O.assemble3d(x, y, z, mu, 20.0)
    v = rng.standard_normal(A.shape[0])
    ref = O.mag3d_apply(x, y, z, mu, 20.0, v)
    np.testing.assert_allclose(A @ v, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    assert np.diff(A.indptr).max() <= 81 and A.has_sorted_indices


def _laplacian_1d(n):
    main = np.full(n, 2.0)
    off = np.full(n - 1, -1.0)
    return sp.diags([off, main, off], [-1, 0, 1], format="csr")


def test_jacobi_and_identity():
    p, mu = _problem2d()
    A = O.assemble2d(17, 17, mu)
    r = np.random.default_rng(0).standard_normal(A.shape[0])
    np.testing.assert_array_equal(O.csr_precond_apply(A, "identity", r), r)
    np.testing.assert_allclose(O.csr_precond_apply(A, "jacobi", r), r / A.diagonal(), rtol=1e-15)


def test_spd_isai_is_the_factorized_approximate_inverse():
    p, mu = _problem2d()
    A = O.assemble2d(17, 17, mu)
    A = (A + A.T) * 0.5            # an SPD matrix with the operator's pattern
    Z = O.csr_isai_values(A, "spd-isai")
    assert (sp.triu(Z, 1)).nnz == 0
    # FSAI: Z A Z^T has a unit diagonal, and M = Z^T Z is what the apply uses
    np.testing.assert_allclose((Z @ A @ Z.T).diagonal(), 1.0, rtol=1e-12)
    r = np.random.default_rng(1).standard_normal(A.shape[0])
    np.testing.assert_allclose(O.csr_precond_apply(A, "spd-isai", r), Z.T @ (Z @ r), rtol=1e-12, atol=1e-14)
    # exact when the inverse factor lies in the pattern (a diagonal matrix)
    D = sp.diags(np.linspace(1.0, 3.0, 20), format="csr")
    np.testing.assert_allclose(O.csr_precond_apply(D, "spd-isai", r[:20]), r[:20] / D.diagonal(), rtol=1e-14)


def test_general_isai_interpolates_the_identity_on_its_pattern():
    rng = np.random.default_rng(2)
    x, y, z = [np.cumsum(rng.uniform(0.5, 1.5, n)) / n for n in (5, 5, 6)]
    A = O.assemble3d(x, y, z, rng.choice([1.0, 1000.0], 150), 20.0)
    M = O.csr_isai_values(A, "general-isai")
    MA = (M @ A).tocsr()
    for i in range(0, A.shape[0], 7):
        cols = A.indices[A.indptr[i]:A.indptr[i + 1]]
        row = MA[i].toarray().ravel()[cols]
        expect = (cols == i).astype(float)
        np.testing.assert_allclose(row, expect, atol=1e-10)


@pytest.mark.parametrize("kind,omega", [("ssor", 1.2), ("symmetric-gauss-seidel", 1.0)])
def test_ssor_is_the_symmetric_sor_factorisation(kind, omega):
    p, mu = _problem2d(n=9)
    A = O.assemble2d(9, 9, mu).toarray()
    D = np.diag(np.diag(A))
    E = -np.tril(A, -1)
    F = -np.triu(A, 1)
    M = (D - omega * E) @ np.linalg.inv(D) @ (D - omega * F) / (omega * (2.0 - omega))
    r = np.random.default_rng(3).standard_normal(81)
    z = O.csr_precond_apply(sp.csr_matrix(A), kind, r, sor_relaxation_factor=omega)
    np.testing.assert_allclose(z, np.linalg.solve(M, r), rtol=1e-10, atol=1e-12)


def test_chebyshev_and_richardson_converge_on_a_known_spectrum():
    n = 40
    A = _laplacian_1d(n)
    lam = 2.0 - 2.0 * np.cos(np.arange(1, n + 1) * np.pi / (n + 1))   # eigenvalues of A; D = 2I
    lo, hi = lam.min() / 2.0, lam.max() / 2.0
    b = np.random.default_rng(4).standard_normal(n)
    x = np.linalg.solve(A.toarray(), b)
    # condition number hi / lo = 665: the error falls by about (sqrt(665) - 1) / (sqrt(665) + 1) per step
    z = O.csr_precond_apply(A, "chebyshev-jacobi", b, chebyshev_iterations=400, chebyshev_lower_bound=lo,
                            chebyshev_upper_bound=hi)
    assert np.linalg.norm(z - x) <= 1e-11 * np.linalg.norm(x)
    z80 = O.csr_precond_apply(A, "chebyshev-jacobi", b, chebyshev_iterations=80, chebyshev_lower_bound=lo,
                              chebyshev_upper_bound=hi)
    assert 1e-4 < np.linalg.norm(z80 - x) / np.linalg.norm(x) < 1e-2
    # a few steps are a fixed linear operator: linear in b
    f = lambda v: O.csr_precond_apply(A, "chebyshev-jacobi", v)
    np.testing.assert_allclose(f(2.0 * b + b[::-1]), 2.0 * f(b) + f(b[::-1]), rtol=1e-12, atol=1e-12)
    # damped Jacobi on a diagonally dominant matrix
    B = A + sp.identity(n, format="csr") * 2.0
    xb = np.linalg.solve(B.toarray(), b)
    zb = O.csr_precond_apply(B, "ir-jacobi", b, ir_iterations=200, ir_relaxation_factor=0.9)
    assert np.linalg.norm(zb - xb) <= 1e-10 * np.linalg.norm(xb)
    z1 = O.csr_precond_apply(B, "ir-jacobi", b, ir_iterations=1, ir_relaxation_factor=0.9)
    np.testing.assert_allclose(z1, 0.9 * (b / B.diagonal()), rtol=1e-15)


@pytest.mark.parametrize("kind", ["identity", "jacobi", "spd-isai", "symmetric-gauss-seidel", "ssor",
                                  "chebyshev-jacobi", "ir-jacobi", "general-isai"])
def test_every_menu_entry_solves_the_2d_problem(kind):
    p, mu = _problem2d(n=33)
    A = O.assemble2d(33, 33, mu)
    b = p.rhs()
    x, it, rel = O.csr_pcg(A, b, kind, tol=1e-10)
    assert rel <= 1e-10
    assert np.linalg.norm(b - A @ x) <= 2e-10 * np.linalg.norm(b)
    xm, _, _ = O.mag2d_cg(33, 33, mu, b, tol=1e-12)
    assert np.linalg.norm(x - xm) <= 1e-7 * np.linalg.norm(xm)


def test_stronger_preconditioners_take_fewer_iterations_in_3d():
    rng = np.random.default_rng(6)
    pr = m3.synthetic_problem(rng, 9, tube=0.2)
    A = O.assemble3d(pr.x, pr.y, pr.z, pr.node_mu(), pr.gamma)
    b = pr.rhs()
    its = {k: O.csr_pcg(A, b, k, tol=1e-10)[1] for k in ("jacobi", "spd-isai", "symmetric-gauss-seidel", "ssor")}
    assert its["symmetric-gauss-seidel"] < its["jacobi"] and its["spd-isai"] < its["jacobi"]
    assert its["ssor"] < its["jacobi"]


def test_menu_newton_matches_the_matrix_free_newton():
    """The nonlinear branch with an assembled Jacobian: Jacobi on the assembled
    matrix is the matrix-free Jacobi-CG; SSOR and SpdIsai take the same Newton
    steps with fewer CG iterations."""
    p, mu, fe, b, h = mag.nonlinear_problem(49, 3)
    rhs = p.rhs()
    x0, it0, s0, r0 = O.mag2d_nl_solve(49, 49, mu, fe, b, h, rhs)
    xj, itj, sj, rj = O.mag2d_nl_solve_menu(49, 49, mu, fe, b, h, rhs, "jacobi")
    assert (itj, sj) == (it0, s0) and np.linalg.norm(xj - x0) <= 1e-14 * np.linalg.norm(x0)
    for kind in ("ssor", "spd-isai"):
        x, it, st, rel = O.mag2d_nl_solve_menu(49, 49, mu, fe, b, h, rhs, kind)
        assert st == s0 and rel <= 1e-10 and it < it0
        assert np.linalg.norm(x - x0) <= 1e-12 * np.linalg.norm(x0)
    p3, mu3, fe3, b3, h3 = m3.nonlinear_problem(13, 6)
    rhs3 = p3.rhs()
    y0, jt0, t0, _ = O.mag3d_nl_solve(p3.x, p3.y, p3.z, mu3, fe3, p3.gamma, b3, h3, rhs3)
    y1, jt1, t1, rel = O.mag3d_nl_solve_menu(p3.x, p3.y, p3.z, mu3, fe3, p3.gamma, b3, h3, rhs3, "ssor")
    assert t1 == t0 and rel <= 1e-10 and jt1 < jt0
    assert np.linalg.norm(y1 - y0) <= 1e-9 * np.linalg.norm(y0)


def test_assembled_jacobian_matches_the_jacobian_apply():
    p, mu, fe, b, h = mag.nonlinear_problem(33, 4)
    rng = np.random.default_rng(7)
    st = rng.standard_normal(33 * 33) * 3 * b[-1]
    J = O.jacobian2d_csr(33, 33, mu, fe, b, h, st)
    v = rng.standard_normal(33 * 33)
    ref = O.mag2d_nl_jacobian_apply(33, 33, mu, fe, b, h, st, v)
    np.testing.assert_allclose(J @ v, ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
