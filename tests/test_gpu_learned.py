"""GPU learned-preconditioner solves: the flexible CG with the trained network
reaches the FP64 1e-10 residual (checked by the oracle's operator) in far fewer
iterations than the same loop without the network and than the plain solver,
and a stalling preconditioner hands its problems to the plain solver."""
import os

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

WEIGHTS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "similie_b200", "data",
                       "precond_2d.npy")


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def mods():
    import similie_b200.magnetostatics as mag
    import similie_b200.precond as pc
    return mag, pc


def _batch(mag, torch, seed, sizes, cores):
    rng = np.random.default_rng(seed)
    probs = [mag.synthetic_problem(rng, n, cores=cores) for n in sizes]
    mus = [torch.from_numpy(p.node_mu()).cuda() for p in probs]
    rhss = [torch.from_numpy(p.rhs()).cuda() for p in probs]
    return probs, mus, rhss


def _check(probs, sols, diags):
    for p, x, d in zip(probs, sols, diags):
        assert d.converged, d
        b = p.rhs()
        r = b - O.mag2d_apply(p.nx, p.ny, p.node_mu(), x.cpu().numpy())
        assert np.linalg.norm(r) / np.linalg.norm(b) <= 1e-10


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="trained weights not present")
def test_trained_network_beats_the_loop_without_it(torch, mods):
    mag, pc = mods
    probs, mus, rhss = _batch(mag, torch, 31, (256, 384, 512), cores=0)
    shapes = [(p.nx, p.ny) for p in probs]
    net = pc.LearnedPreconditioner(seed=0)
    net.load(WEIGHTS)
    sols = [torch.zeros_like(r) for r in rhss]
    d_net = mag.solve_batch(mus, rhss, sols, shapes, solver="learned", preconditioner=net, stall_window=100000)
    _check(probs, sols, d_net)
    # the same flexible CG without the network: output convolution zeroed, M = two Jacobi steps
    params = net.get_params()
    params[-(9 * 32 + 1):] = 0.0
    bare = pc.LearnedPreconditioner(seed=0)
    bare.set_params(params)
    sols0 = [torch.zeros_like(r) for r in rhss]
    d_bare = mag.solve_batch(mus, rhss, sols0, shapes, solver="learned", preconditioner=bare, stall_window=100000,
                             inner_iterations=20000)
    _check(probs, sols0, d_bare)
    sols1 = [torch.zeros_like(r) for r in rhss]
    d_plain = mag.solve_batch(mus, rhss, sols1, shapes, solver="cg")
    for a, b, c in zip(d_net, d_bare, d_plain):
        assert not a.fallback
        assert 4 * a.learned_iterations < b.learned_iterations, (a, b)
        assert 4 * a.learned_iterations < c.iterations, (a, c)


def test_stall_hands_problems_to_the_plain_solver(torch, mods):
    mag, pc = mods
    probs, mus, rhss = _batch(mag, torch, 32, (96, 130), cores=2)
    shapes = [(p.nx, p.ny) for p in probs]
    net = pc.LearnedPreconditioner(seed=0)   # untrained: a poor preconditioner
    sols = [torch.zeros_like(r) for r in rhss]
    d = mag.solve_batch(mus, rhss, sols, shapes, solver="learned", preconditioner=net, stall_window=20)
    _check(probs, sols, d)
    assert any(x.fallback for x in d)
    assert all(x.iterations > x.learned_iterations for x in d if x.fallback)


@pytest.mark.skipif(not os.path.exists(WEIGHTS), reason="trained weights not present")
def test_more_flexible_directions_cut_iterations_on_inclusions(torch, mods):
    """FCG(m): keeping 8 A-orthogonal directions instead of one takes the
    preconditioned solve of inclusion problems (where the network's correction
    varies most from step to step) to 1e-10 in markedly fewer iterations."""
    mag, pc = mods
    probs, mus, rhss = _batch(mag, torch, 33, (256, 384), cores=2)
    shapes = [(p.nx, p.ny) for p in probs]
    net = pc.LearnedPreconditioner(seed=0)
    net.load(WEIGHTS)
    its = {}
    for m in (1, 4, 8, 16):
        sols = [torch.zeros_like(r) for r in rhss]
        d = mag.solve_batch(mus, rhss, sols, shapes, solver="learned", preconditioner=net, stall_window=100000,
                            inner_iterations=20000, flexible_directions=m)
        _check(probs, sols, d)
        assert not any(x.fallback for x in d)
        its[m] = sum(x.learned_iterations for x in d)
    assert 3 * its[8] < 2 * its[1], its
    assert its[16] <= its[4], its


def test_flexible_directions_above_the_ring_size_are_rejected(torch, mods):
    mag, pc = mods
    probs, mus, rhss = _batch(mag, torch, 34, (64,), cores=0)
    net = pc.LearnedPreconditioner(seed=0)
    sols = [torch.zeros_like(r) for r in rhss]
    from similie_b200._native import SilError
    with pytest.raises(SilError, match="flexible_directions"):
        mag.solve_batch(mus, rhss, sols, [(64, 64)], solver="learned", preconditioner=net, flexible_directions=17)
