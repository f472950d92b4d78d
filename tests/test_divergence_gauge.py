"""3D divergence gauge (the reference's SIMILIE_DIVERGENCE_GAUGE_3D): the
codifferential's per-node coefficients read off six parity probes reproduce
the oracle codifferential (CPU); on the GPU the gauged 3D operator matches
the oracle curl-curl plus the codifferential gauge term, and the gauged
solve converges to 1e-10 under that operator."""
import numpy as np
import pytest

import oracle as O
import similie_b200.magnetostatics3d as m3


def _grid(n):
    return (m3.stretched_coords(n, 1.1), m3.stretched_coords(n, 1.05) * 1.3, m3.stretched_coords(n, 1.2))


def probe_coefficients(x, y, z):
    """E0, E1 ([x][y][z][3]) and w ([x][y][z]) of the gauge from the oracle codifferential."""
    n = (len(x), len(y), len(z))
    pos = O.position_from_coords([x, y, z])
    interior = np.zeros(n, bool)
    interior[1:-1, 1:-1, 1:-1] = True
    idx = np.indices(n)
    E0, E1 = np.zeros(n + (3,)), np.zeros(n + (3,))
    for a in range(3):
        for p in (0, 1):
            P = np.zeros(n + (3,))
            P[..., a] = ((idx[a] % 2 == p) & interior).astype(float)
            Q = O.codifferential(3, 1, pos, P)[..., 0]
            same = idx[a] % 2 == p
            E0[..., a][same] = Q[same]
            E1[..., a][~same] = Q[~same]
    ls = lambda c: np.r_[c[1] - c[0], 0.5 * (c[2:] - c[:-2]), c[-1] - c[-2]]
    w = ls(x)[:, None, None] * ls(y)[None, :, None] * ls(z)[None, None, :]
    return E0, E1, w


def _shift(v, a):
    """v(m - e_a), zero where m - e_a is outside."""
    out = np.zeros_like(v)
    src = [slice(None)] * 3
    dst = [slice(None)] * 3
    src[a], dst[a] = slice(0, -1), slice(1, None)
    out[tuple(dst)] = v[tuple(src)]
    return out


def gauge_term(E0, E1, w, A):
    """Gauge term per DOF ([x][y][z][3]) of A ([x][y][z][3], boundary values ignored)."""
    DA = sum(E0[..., a] * A[..., a] + E1[..., a] * _shift(A[..., a], a) for a in range(3))
    out = np.zeros_like(A)
    for c in range(3):
        nxt = [slice(None)] * 3
        cur = [slice(None)] * 3
        nxt[c], cur[c] = slice(1, None), slice(0, -1)
        out[..., c] = w * E0[..., c] * DA
        out[..., c][tuple(cur)] += (w * E1[..., c] * DA)[tuple(nxt)]
    return out


def oracle_apply(x, y, z, mu, gamma, a_flat):
    n = (len(x), len(y), len(z))
    y0 = O.mag3d_apply(x, y, z, mu, 0.0, a_flat)          # curl-curl part
    A = a_flat.reshape(n[2], n[1], n[0], 3).transpose(2, 1, 0, 3)
    g = gauge_term(*probe_coefficients(x, y, z), A)
    out = y0.reshape(n[2], n[1], n[0], 3).transpose(2, 1, 0, 3).copy()
    inner = (slice(1, -1),) * 3
    out[inner] += gamma * g[inner]
    return out.transpose(2, 1, 0, 3).ravel()


def test_probes_reproduce_the_codifferential():
    x, y, z = _grid(7)
    E0, E1, w = probe_coefficients(x, y, z)
    rng = np.random.default_rng(1)
    A = rng.standard_normal((7, 7, 7, 3))
    A[0], A[-1] = 0, 0
    A[:, 0], A[:, -1] = 0, 0
    A[:, :, 0], A[:, :, -1] = 0, 0
    ref = O.codifferential(3, 1, O.position_from_coords([x, y, z]), A)[..., 0]
    DA = sum(E0[..., a] * A[..., a] + E1[..., a] * _shift(A[..., a], a) for a in range(3))
    assert np.abs(ref - DA).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.gpu
def test_gauged_operator_and_solve_match_the_oracle():
    import torch
    x, y, z = _grid(11)
    n = (11, 11, 11)
    nodes = 11 ** 3
    rng = np.random.default_rng(3)
    mu = rng.choice([1.0, 1000.0], nodes)
    a = rng.standard_normal(3 * nodes)
    gamma = 20.0
    yg = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    mu_d = torch.from_numpy(mu).cuda()
    m3.apply(x, y, z, mu_d, torch.from_numpy(a).cuda(), yg, gamma=gamma, gauge="divergence")
    ref = oracle_apply(x, y, z, mu, gamma, a)
    np.testing.assert_allclose(yg.cpu().numpy(), ref, rtol=1e-11, atol=1e-12 * np.abs(ref).max())
    # the penalty gauge is unchanged
    m3.apply(x, y, z, mu_d, torch.from_numpy(a).cuda(), yg, gamma=gamma)
    np.testing.assert_allclose(yg.cpu().numpy(), O.mag3d_apply(x, y, z, mu, gamma, a), rtol=1e-12,
                               atol=1e-13 * np.abs(ref).max())
    # gauged solve (FP64 CG), residual under the restated operator
    b = np.zeros((n[2], n[1], n[0], 3))
    b[3:6, 4:7, 3:8, 2] = 1e-3
    b[1:-1, 1:-1, 1:-1, 0] += 1e-4 * rng.standard_normal((9, 9, 9))
    b = b.ravel()
    sol = torch.zeros(3 * nodes, dtype=torch.float64, device="cuda")
    d = m3.solve_batch([(x, y, z)], [mu_d], [torch.from_numpy(b).cuda()], [sol], gammas=[gamma], tol=1e-10,
                       gauge="divergence")
    assert d[0].converged, d[0]
    r = b - oracle_apply(x, y, z, mu, gamma, sol.cpu().numpy())
    assert np.linalg.norm(r) <= 2e-10 * np.linalg.norm(b)
