"""Batched solves on the distributions of the benchmark workloads, checked
problem by problem against the oracle.

* 2D: sixteen problems drawn exactly as the 64-problem benchmark batch draws
  them (grid sizes uniform over {128, 256, 384, 512, 768, 1024}^2, 1-8 coils,
  0-3 permeability-1000 rectangles), solved by the plain FP64 solver, the
  FP32-inner / FP64-refinement solver and the learned preconditioner; every
  solution's relative residual, measured by the oracle's FP64 operator, is at
  most 1e-10.
* 2D inclusions: problems with two or three permeability-1000 rectangles (the
  ones that set the learned batch's time), where the preconditioned solve
  must still take far fewer iterations than the plain solver.
* 3D: grids of 48^3-64^3 nodes stretched by 1.01 per axis with toroidal
  loop currents and gauge penalty 20 (the 256^3 benchmark batch's shape at a
  size the oracle solves in seconds); each solution is checked by the
  oracle's operator and against the oracle's own CG solution.
"""
import os

import numpy as np
import pytest

import oracle as O
from helpers import rel_err

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "similie_b200", "data",
                       "precond_2d.npy")


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def batch2d(torch):
    import similie_b200.magnetostatics as mag
    probs = mag.synthetic_batch(seed=20, count=16)
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    return probs, mus, rhss


def _oracle_residuals(probs, sols):
    out = []
    for p, x in zip(probs, sols):
        b = p.rhs()
        r = b - O.mag2d_apply(p.nx, p.ny, p.node_mu(), x.cpu().numpy())
        out.append(float(np.linalg.norm(r) / np.linalg.norm(b)))
    return out


@pytest.mark.parametrize("solver", ["cg", "mixed", "learned"])
def test_benchmark_distribution_reaches_1e10(torch, batch2d, solver):
    import similie_b200.magnetostatics as mag
    from similie_b200.precond import LearnedPreconditioner
    probs, mus, rhss = batch2d
    assert {p.nx for p in probs} >= {128, 1024}
    net = None
    if solver == "learned":
        if not os.path.exists(WEIGHTS):
            pytest.skip("trained weights not present")
        net = LearnedPreconditioner(seed=0)
        net.load(WEIGHTS)
    sols = [torch.zeros_like(r) for r in rhss]
    diags = mag.solve_batch(mus, rhss, sols, [(p.nx, p.ny) for p in probs], solver=solver, tol=1e-10,
                            preconditioner=net)
    rels = _oracle_residuals(probs, sols)
    for p, d, rel in zip(probs, diags, rels):
        assert d.converged, (p.nx, d)
        assert rel <= 1e-10, (p.nx, p.meta, rel, d)
        # the solver's own FP64 true residual is the oracle's
        assert abs(rel - d.final_relative_residual) <= 1e-12 + 1e-3 * rel


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="trained weights not present")
def test_learned_gain_on_inclusion_problems(torch):
    import similie_b200.magnetostatics as mag
    from similie_b200.precond import LearnedPreconditioner
    rng = np.random.default_rng(23)
    probs = [mag.synthetic_problem(rng, n, cores=c) for n, c in ((384, 2), (512, 3), (512, 2), (768, 3))]
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    shapes = [(p.nx, p.ny) for p in probs]
    net = LearnedPreconditioner(seed=0)
    net.load(WEIGHTS)
    sl = [torch.zeros_like(r) for r in rhss]
    dl = mag.solve_batch(mus, rhss, sl, shapes, solver="learned", preconditioner=net, stall_window=100000)
    sp = [torch.zeros_like(r) for r in rhss]
    dp = mag.solve_batch(mus, rhss, sp, shapes, solver="cg")
    for p, a, b, rel in zip(probs, dl, dp, _oracle_residuals(probs, sl)):
        assert a.converged and b.converged and rel <= 1e-10, (p.nx, a, b, rel)
        assert not a.fallback
        assert 3 * a.iterations < b.iterations, (p.nx, p.meta, a, b)


@pytest.mark.parametrize("solver", ["cg", "mixed"])
def test_stretched_3d_batch_matches_oracle(torch, solver):
    import similie_b200.magnetostatics3d as m3
    rng = np.random.default_rng(29)
    probs = [m3.synthetic_problem(rng, n, ratio=1.01, gamma=20.0) for n in (48, 56, 64)]
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    sols = [torch.zeros_like(r) for r in rhss]
    diags = m3.solve_batch([(p.x, p.y, p.z) for p in probs], mus, rhss, sols, [p.gamma for p in probs],
                           solver=solver, tol=1e-10)
    for p, d, xs in zip(probs, diags, sols):
        assert d.converged, (p.shape, d)
        xb = xs.cpu().numpy()
        b = p.rhs()
        mu = p.node_mu()
        rel = np.linalg.norm(b - O.mag3d_apply(p.x, p.y, p.z, mu, p.gamma, xb)) / np.linalg.norm(b)
        assert rel <= 1e-10, (p.shape, rel, d)
        assert abs(rel - d.final_relative_residual) <= 1e-12 + 1e-3 * rel
        xo, _, _ = O.mag3d_cg(p.x, p.y, p.z, mu, p.gamma, b, tol=1e-12)
        assert rel_err(xb, xo) < 1e-6
