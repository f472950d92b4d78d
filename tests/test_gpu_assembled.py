"""GPU assembled-operator path against the CPU oracle: the probed CSR
matrices (2D, 3D with either gauge), every preconditioner of the reference's
menu applied on the GPU-assembled matrix against the oracle on the same
matrix, and the preconditioned CG (iterations, residual, solution)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

MENU = ["identity", "jacobi", "spd-isai", "symmetric-gauss-seidel", "ssor", "chebyshev-jacobi", "ir-jacobi",
        "general-isai"]


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def asm():
    import similie_b200.assembled as a
    return a


def _dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()


@pytest.fixture(scope="module")
def case2d(torch, asm):
    import similie_b200.magnetostatics as mag
    rng = np.random.default_rng(11)
    n = 33
    p = mag.synthetic_problem(rng, n, cores=2)
    mu = p.node_mu()
    A = asm.CsrMatrix.mag2d(n, n, _dev(torch, mu))
    return n, p, mu, A


@pytest.fixture(scope="module")
def case3d(torch, asm):
    import similie_b200.magnetostatics3d as m3
    rng = np.random.default_rng(12)
    pr = m3.synthetic_problem(rng, 9, tube=0.2)
    mu = pr.node_mu()
    A = asm.CsrMatrix.mag3d(pr.x, pr.y, pr.z, _dev(torch, mu), gamma=pr.gamma)
    return pr, mu, A


def test_assembled_2d_matches_the_oracle(torch, case2d):
    n, p, mu, A = case2d
    G = A.to_scipy()
    R = O.assemble2d(n, n, mu)
    # same entries up to rounding (an entry that cancels to exactly zero in
    # one arithmetic and not the other may be present in only one)
    assert G.has_sorted_indices and abs(G.nnz - R.nnz) <= R.nnz // 100
    assert abs(G - R).max() <= 1e-13 * np.abs(R.data).max()
    v = np.random.default_rng(0).standard_normal(n * n)
    y = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    A.spmv(_dev(torch, v), y)
    np.testing.assert_allclose(y.cpu().numpy(), G @ v, rtol=1e-14, atol=1e-14 * np.abs(G @ v).max())


def test_assembled_3d_matches_the_oracle(torch, asm, case3d):
    pr, mu, A = case3d
    G = A.to_scipy()
    R = O.assemble3d(pr.x, pr.y, pr.z, mu, pr.gamma)
    assert G.has_sorted_indices and abs(G.nnz - R.nnz) <= R.nnz // 100
    assert abs(G - R).max() <= 1e-12 * np.abs(R.data).max()


def test_assembled_divergence_gauge_matches_the_gpu_operator(torch, asm):
    import similie_b200.magnetostatics3d as m3
    rng = np.random.default_rng(13)
    x, y, z = [np.cumsum(rng.uniform(0.5, 1.5, n)) / n for n in (7, 6, 8)]
    mu = _dev(torch, rng.choice([1.0, 1000.0], 7 * 6 * 8))
    A = asm.CsrMatrix.mag3d(x, y, z, mu, gamma=-3.0, gauge="divergence")
    v = _dev(torch, rng.standard_normal(3 * 7 * 6 * 8))
    out = torch.zeros_like(v)
    ref = torch.zeros_like(v)
    A.spmv(v, out)
    m3.apply(x, y, z, mu, v, ref, gamma=-3.0, gauge="divergence")
    torch.cuda.synchronize()
    scale = float(torch.abs(ref).max())
    assert float(torch.abs(out - ref).max()) <= 1e-12 * scale


@pytest.mark.parametrize("kind", MENU)
def test_preconditioners_match_the_oracle(torch, asm, case2d, case3d, kind):
    for A in (case2d[3], case3d[2]):
        G = A.to_scipy()
        P = asm.Preconditioner(A, kind)
        r = np.random.default_rng(1).standard_normal(G.shape[0])
        z = torch.zeros(G.shape[0], dtype=torch.float64, device="cuda")
        P.apply(_dev(torch, r), z)
        ref = O.csr_precond_apply(G, kind, r)
        np.testing.assert_allclose(z.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())


@pytest.mark.parametrize("kind", ["symmetric-gauss-seidel", "ssor"])
def test_single_launch_sweeps_repeat_exactly(torch, asm, kind):
    """SSOR and symmetric Gauss-Seidel run each triangular sweep as one
    launch (one CTA walking the levels): applied again and again,
    stream-ordered and replayed from a CUDA graph, on a 2D matrix of 96^2
    rows (191 levels per sweep), every result is the first one bit for bit
    and matches the oracle."""
    import similie_b200.magnetostatics as mag
    rng = np.random.default_rng(23)
    n = 96
    p = mag.synthetic_problem(rng, n, cores=2)
    mu = p.node_mu()
    A = asm.CsrMatrix.mag2d(n, n, _dev(torch, mu))
    G = A.to_scipy()
    P = asm.Preconditioner(A, kind)
    r = _dev(torch, rng.standard_normal(G.shape[0]))
    first = torch.zeros_like(r)
    P.apply(r, first)
    torch.cuda.synchronize()
    ref = O.csr_precond_apply(G, kind, r.cpu().numpy())
    np.testing.assert_allclose(first.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.abs(ref).max())
    for _ in range(20):
        z = torch.full_like(r, float("nan"))
        P.apply(r, z)
        assert torch.equal(z, first)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    outs = [torch.full_like(r, float("nan")) for _ in range(4)]
    with torch.cuda.stream(s):
        P.apply(r, outs[0])
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for o in outs:
            P.apply(r, o)
    for _ in range(3):
        for o in outs:
            o.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        for o in outs:
            assert torch.equal(o, first)


@pytest.mark.parametrize("kind", MENU)
def test_cg_matches_the_oracle_2d(torch, asm, case2d, kind):
    n, p, mu, A = case2d
    G = A.to_scipy()
    b = p.rhs()
    P = asm.Preconditioner(A, kind)
    x = torch.zeros(n * n, dtype=torch.float64, device="cuda")
    d = asm.solve(A, P, _dev(torch, b), x, tol=1e-10)
    xo, it, rel = O.csr_pcg(G, b, kind, tol=1e-10)
    assert d.converged and d.status == 0
    # dot products summed in another order: the Krylov paths drift apart
    # slowly.  With the reference's default bounds [0.05, 1.5] the Chebyshev
    # polynomial is indefinite on this spectrum (up to 2), and the oracle's own
    # count moves by 8 % under 1e-15 perturbations of b.
    slack = it // 8 if kind == "chebyshev-jacobi" else it // 20
    assert abs(d.iterations - it) <= max(3, slack)
    xg = x.cpu().numpy()
    assert np.linalg.norm(b - G @ xg) <= 2e-10 * np.linalg.norm(b)
    assert np.linalg.norm(xg - xo) <= 1e-8 * np.linalg.norm(xo)


@pytest.mark.parametrize("kind", ["jacobi", "spd-isai", "ssor"])
def test_cg_solves_the_3d_problem(torch, asm, case3d, kind):
    pr, mu, A = case3d
    G = A.to_scipy()
    b = pr.rhs()
    P = asm.Preconditioner(A, kind)
    x = torch.zeros(G.shape[0], dtype=torch.float64, device="cuda")
    d = asm.solve(A, P, _dev(torch, b), x, tol=1e-10)
    xo, it, rel = O.csr_pcg(G, b, kind, tol=1e-10)
    assert d.converged and abs(d.iterations - it) <= max(3, it // 20)
    xg = x.cpu().numpy()
    assert np.linalg.norm(b - G @ xg) <= 2e-10 * np.linalg.norm(b)


def test_zero_rhs_and_bad_settings(torch, asm, case2d):
    from similie_b200._native import SilError
    n, p, mu, A = case2d
    P = asm.Preconditioner(A, "jacobi")
    x = torch.ones(n * n, dtype=torch.float64, device="cuda")
    d = asm.solve(A, P, torch.zeros(n * n, dtype=torch.float64, device="cuda"), x)
    assert d.converged and d.iterations == 0 and float(torch.abs(x).max()) == 0.0
    with pytest.raises(SilError):
        asm.Preconditioner(A, "chebyshev-jacobi", chebyshev_lower_bound=2.0, chebyshev_upper_bound=1.0)
    with pytest.raises(ValueError):
        asm.kind_of("no-such-preconditioner")
