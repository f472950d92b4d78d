"""Staged codifferential and Hodge Laplacian built from a (metric, position)
pair -- the reference's StagedCodifferential(exec, tensor, metric, position)
and StagedLaplacian(exec, out, in, metric, position) -- on perturbed
(non-orthogonal) lattices with a dense symmetric positive definite metric per
node, every rank in 1D, 2D and 3D, against the oracle's staged chain over
the same stored Hodge tensors (1e-12 relative, max-norm)."""
from math import comb

import numpy as np
import pytest

import oracle as O
from helpers import rel_err

pytestmark = pytest.mark.gpu

TOL = 1e-12
SHAPES = {1: (29,), 2: (21, 17), 3: (9, 8, 7)}


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


@pytest.fixture(scope="module")
def sil():
    import similie_b200
    similie_b200.lib()
    return similie_b200


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=torch.float64)


def _lattice(n, seed):
    rng = np.random.default_rng(seed)
    shape = SHAPES[n]
    coords = [np.cumsum(rng.uniform(0.3, 1.7, s)) for s in shape]
    pos = O.position_from_coords(coords) + 0.02 * rng.standard_normal(shape + (n,))
    a = rng.standard_normal(shape + (n, n)) * 0.3
    met = np.einsum("...ij,...kj->...ik", a, a) + np.eye(n)
    return rng, shape, pos, np.ascontiguousarray(met.reshape(shape + (n * n,)))


@pytest.mark.parametrize("n,k", [(n, k) for n in (1, 2, 3) for k in range(n + 1)])
def test_metric_laplacian_matches_oracle(torch, sil, n, k):
    rng, shape, pos, met = _lattice(n, 300 + 10 * n + k)
    w = rng.standard_normal(shape + (comb(n, k),))
    ref = O.laplacian(n, k, pos, w, metric=met)
    geo = sil.MetricGeometry(dev(torch, pos), dev(torch, met))
    inp = dev(torch, w)
    out = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
    plan = sil.make_staged_laplacian(geo, out, inp, k)
    assert plan.kernel == 4
    plan.run(out, inp)
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), ref) <= TOL, (n, k)
    # a second run on other data through the same stored tensors
    w2 = rng.standard_normal(w.shape)
    plan.run(out, dev(torch, w2))
    assert rel_err(out.cpu().numpy(), O.laplacian(n, k, pos, w2, metric=met)) <= TOL, (n, k)


@pytest.mark.parametrize("n,k", [(n, k) for n in (1, 2, 3) for k in range(1, n + 1)])
def test_metric_codifferential_matches_oracle(torch, sil, n, k):
    rng, shape, pos, met = _lattice(n, 400 + 10 * n + k)
    w = rng.standard_normal(shape + (comb(n, k),))
    ref = O.codifferential(n, k, pos, w, metric=met)
    geo = sil.MetricGeometry(dev(torch, pos), dev(torch, met))
    st = sil.make_staged_codifferential(geo, k)
    out = torch.full(ref.shape, float("nan"), dtype=torch.float64, device="cuda")
    st.run(out, dev(torch, w))
    torch.cuda.synchronize()
    assert rel_err(out.cpu().numpy(), ref) <= TOL, (n, k)


@pytest.mark.parametrize("n,k", [(2, 1), (3, 1), (3, 2)])
def test_identity_metric_agrees_with_the_rectilinear_plan(torch, sil, n, k):
    """On a rectilinear grid with the identity metric (metric None) the
    stored-tensor plan and the coordinate-driven plan compute the same
    Laplacian."""
    rng = np.random.default_rng(500 + n + k)
    shape = SHAPES[n]
    coords = [np.cumsum(rng.uniform(0.5, 1.5, s)) for s in shape]
    pos = O.position_from_coords(coords)
    w = dev(torch, rng.standard_normal(shape + (comb(n, k),)))
    out_shape = tuple(s - 1 for s in shape) + (comb(n, k),)
    a = torch.zeros(out_shape, dtype=torch.float64, device="cuda")
    b = torch.zeros_like(a)
    sil.make_staged_laplacian(sil.MetricGeometry(dev(torch, pos)), a, w, k).run(a, w)
    sil.make_staged_laplacian(sil.Geometry(coords), b, w, k).run(b, w)
    torch.cuda.synchronize()
    assert rel_err(a.cpu().numpy(), b.cpu().numpy()) <= TOL


def test_metric_plan_rejects_fields_outside_the_position_lattice(torch, sil):
    _, shape, pos, met = _lattice(2, 7)
    geo = sil.MetricGeometry(dev(torch, pos), dev(torch, met))
    inp = torch.zeros(shape[0] + 1, shape[1], 2, dtype=torch.float64, device="cuda")
    out = torch.zeros(shape[0], shape[1] - 1, 2, dtype=torch.float64, device="cuda")
    with pytest.raises(sil.SilError):
        sil.make_staged_laplacian(geo, out, inp, 1).run(out, inp)
