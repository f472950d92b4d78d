"""GPU 3D magnetostatics (curl-curl + gauge penalty): operator parity with the
oracle on stretched grids and batched solves of uneven sizes that reach the
FP64 1e-10 relative residual measured by the oracle's operator."""
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
def m3():
    import similie_b200.magnetostatics3d as m
    import similie_b200
    similie_b200.lib()
    return m


def _grid(m3, rng, nx, ny, nz, ratio):
    x = m3.stretched_coords(nx, ratio)
    y = m3.stretched_coords(ny, 1.0 / ratio, 0.7)
    z = m3.stretched_coords(nz, ratio, 1.3) + 0.25
    cell_mu = np.where(rng.random((nx - 1) * (ny - 1) * (nz - 1)) < 0.2, 1000.0, 1.0)
    return x, y, z, cell_mu


@pytest.mark.parametrize("shape,ratio,gamma", [((3, 3, 3), 1.0, 20.0), ((9, 11, 7), 1.01, 20.0),
                                                ((24, 17, 20), 1.05, 3.5)])
def test_apply_matches_oracle(torch, m3, shape, ratio, gamma):
    rng = np.random.default_rng(sum(shape))
    nx, ny, nz = shape
    x, y, z, cell_mu = _grid(m3, rng, nx, ny, nz, ratio)
    mu = m3.node_mu(nx, ny, nz, cell_mu)
    a = rng.standard_normal(3 * nx * ny * nz)
    ref = O.mag3d_apply(x, y, z, mu, gamma, a)
    ty = torch.zeros(a.size, dtype=torch.float64, device="cuda")
    m3.apply(x, y, z, torch.from_numpy(mu).cuda(), torch.from_numpy(a).cuda(), ty, gamma)
    assert rel_err(ty.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("shape", [(13, 10, 9), (40, 17, 70), (3, 3, 3), (33, 9, 33)])
@pytest.mark.parametrize("gauge", ["penalty", "divergence"])
def test_operator_object_matches_the_per_call_apply(torch, m3, gauge, shape):
    """The operator object (set-up once, one kernel per apply, replayable from
    a CUDA graph) gives the per-call apply's result bit for bit, and the
    oracle's to 1e-12 (penalty gauge), on grids with and without
    deep-interior nodes."""
    rng = np.random.default_rng(31)
    nx, ny, nz = shape
    x, y, z, cell_mu = _grid(m3, rng, nx, ny, nz, 1.03)
    mu_h = m3.node_mu(nx, ny, nz, cell_mu)
    mu = torch.from_numpy(mu_h).cuda()
    a = torch.from_numpy(rng.standard_normal(3 * nx * ny * nz)).cuda()
    ref = torch.zeros_like(a)
    m3.apply(x, y, z, mu, a, ref, 20.0, gauge=gauge)
    op = m3.Operator(x, y, z, mu, 20.0, gauge=gauge)
    got = torch.full_like(a, float("nan"))
    op.apply(a, got)
    torch.cuda.synchronize()
    assert torch.equal(got, ref)
    if gauge == "penalty":
        assert rel_err(got.cpu().numpy(), O.mag3d_apply(x, y, z, mu_h, 20.0, a.cpu().numpy())) <= 1e-12
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        op.apply(a, got)
    torch.cuda.current_stream().wait_stream(s)
    g = torch.cuda.CUDAGraph()
    out2 = torch.full_like(a, float("nan"))
    with torch.cuda.graph(g):
        op.apply(a, out2)
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(out2, ref)


def test_apply_is_symmetric(torch, m3):
    rng = np.random.default_rng(5)
    x, y, z, cell_mu = _grid(m3, rng, 10, 9, 8, 1.02)
    mu = torch.from_numpy(m3.node_mu(10, 9, 8, cell_mu)).cuda()
    u = torch.randn(3 * 720, dtype=torch.float64, device="cuda")
    v = torch.randn(3 * 720, dtype=torch.float64, device="cuda")
    # restrict to interior rows: boundary rows are the identity
    au, av = torch.zeros_like(u), torch.zeros_like(v)
    m3.apply(x, y, z, mu, u, au)
    m3.apply(x, y, z, mu, v, av)
    b = np.zeros((8, 9, 10, 3), dtype=bool)
    b[0] = b[-1] = True
    b[:, 0] = b[:, -1] = True
    b[:, :, 0] = b[:, :, -1] = True
    interior = torch.from_numpy(~b.ravel()).cuda()
    u, v = u * interior, v * interior
    m3.apply(x, y, z, mu, u, au)
    m3.apply(x, y, z, mu, v, av)
    lhs = float(torch.dot(v, au * interior))
    rhs = float(torch.dot(u, av * interior))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)


@pytest.mark.parametrize("solver", ["cg", "mixed"])
def test_batched_solve_reaches_tolerance(torch, m3, solver):
    rng = np.random.default_rng(21)
    probs = [m3.synthetic_problem(rng, n, tube=0.12) for n in (10, 17, 24)]
    # one anisotropic grid in the same batch
    x, y, z, _ = _grid(m3, rng, 13, 9, 15, 1.03)
    cj = rng.uniform(-1, 1, 12 * 8 * 14 * 3)
    probs.append(m3.Problem(x, y, z, np.ones(12 * 8 * 14), cj, 7.0))
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    sols = [torch.zeros_like(r) for r in rhss]
    diags = m3.solve_batch([(p.x, p.y, p.z) for p in probs], mus, rhss, sols, [p.gamma for p in probs],
                           solver=solver, tol=1e-10)
    for p, d, xs in zip(probs, diags, sols):
        assert d.converged, d
        xb = xs.cpu().numpy()
        b = p.rhs()
        r = b - O.mag3d_apply(p.x, p.y, p.z, p.node_mu(), p.gamma, xb)
        rel = np.linalg.norm(r) / np.linalg.norm(b)
        assert rel <= 1e-10, (p.shape, rel, d)
        assert abs(rel - d.final_relative_residual) <= 1e-12 + 1e-3 * rel
        xo, _, _ = O.mag3d_cg(p.x, p.y, p.z, p.node_mu(), p.gamma, b, tol=1e-12)
        assert rel_err(xb, xo) < 1e-6
