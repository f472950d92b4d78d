"""The reference examples' correctness checks through the GPU Laplacian
(examples/2d_laplacian.cpp:240-251, 2d_vector_laplacian.cpp:241-267): on
the 1003^2 Greville grid of [-5, 5]^2 the Laplacian is 1 near (5/8 Lx, 0)
and 0 near (7/8 Lx, 0) within 5e-2, and equals the oracle's to 1e-12."""
import numpy as np
import pytest

import oracle as O
from test_oracle import _example_index, _greville_cubic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch as t
    assert t.cuda.is_available()
    return t


def _fields():
    x = _greville_cubic(-5.0, 5.0, 1000)
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    R, alpha = 2.0, 0.25
    inside = r <= R
    rs = np.where(inside, 1.0, r)
    phi = np.where(inside, -alpha * r * r, alpha * R * R * (2.0 * np.log(R / rs) - 1.0))
    w = np.zeros(X.shape + (2,))
    w[..., 0] = np.where(inside, Y * (r / 3.0 - R / 2.0), -Y * R ** 3 / (6.0 * rs * rs))
    w[..., 1] = np.where(inside, -X * (r / 3.0 - R / 2.0), X * R ** 3 / (6.0 * rs * rs))
    return x, phi[..., None], w


@pytest.mark.parametrize("k", [0, 1])
def test_example_checks_on_the_gpu(torch, k):
    import similie_b200 as sil
    x, phi, w = _fields()
    field = phi if k == 0 else w
    n = len(x)
    geo = sil.Geometry([x, x])
    inp = torch.from_numpy(np.ascontiguousarray(field)).cuda()
    out = torch.zeros((n - 1, n - 1, field.shape[-1]), dtype=torch.float64, device="cuda")
    sil.laplacian(geo, out, inp, k)
    lap = out.cpu().numpy()
    ref = O.laplacian(2, k, O.position_from_coords([x, x]), field)
    assert np.max(np.abs(lap - ref)) <= 1e-12 * np.max(np.abs(ref))
    iy = _example_index(0.5, n - 1)
    for frac, expected in ((5 / 8, 1.0), (7 / 8, 0.0)):
        v = lap[_example_index(frac, n - 1), iy]
        assert abs(np.linalg.norm(v) - expected) <= 5e-2
