"""The CPU oracle, pinned against SimiLie's own known-answer tests.

Fixtures come from tests/golden/*.json (extracted from the reference's test
files by tests/golden/make_golden.py) and from the analytic gate functions of
tests/exterior/laplacian.cpp, restated here with their tolerances."""
import numpy as np
import pytest

import oracle as O
from helpers import combos, comp_index, kat_field, load_golden

DER = load_golden("derivative_kat.json")
EXT = load_golden("exterior_kat.json")


def _kat_case_ids():
    return [f"{t['name']}-{t['variant']}" for t in DER["tests"]]


@pytest.mark.parametrize("case", DER["tests"], ids=_kat_case_ids())
def test_derivative_kat(case):
    """tests/exterior/derivative.cpp: EXPECT_EQ (bit-exact) values of d."""
    N, ndim, k_in, k_out = case["N"], len(case["dims"]), case["k_in"], case["k_out"]
    if "spectators" in case:
        pytest.skip("covered by test_derivative_kat_spectators")
    f = kat_field(N, ndim, k_in)
    out_n = N if k_out == 1 else N - 1
    if case["component_first"]:
        inp = np.ascontiguousarray(np.moveaxis(f, -1, 0))
        out = np.full((len(combos(ndim, k_out)),) + (out_n,) * ndim, np.nan)
        O.coboundary(inp, out, k_in, comp_axis=0)
        out = np.moveaxis(out, 0, -1)
    else:
        out = np.full((out_n,) * ndim + (len(combos(ndim, k_out)),), np.nan)
        O.coboundary(f, out, k_in)
    assert not np.isnan(out).any()
    for chk in case["checks"]:
        c = comp_index(ndim, chk["comp_dims"])
        assert out[tuple(chk["node"]) + (c,)] == chk["value"], chk


def test_derivative_kat_spectators():
    """derivative.cpp 2DRotationalWithSpects: a spectator lattice dim and a
    spectator tensor index between the form dims; layout (comp, S, X, I, Y)."""
    case = [t for t in DER["tests"] if t["name"] == "2DRotationalWithSpects"][0]
    inp = np.zeros((2, 3, 3, 10, 3))
    for c in range(2):
        inp[c] = c + 1.0
        inp[c, :, 1, :, 1] = c + 2.0
    out = np.full((1, 3, 2, 10, 2), np.nan)
    # lattice dims after removing the component axis: S=0, X=1, I=2, Y=3; form dims X and Y
    O.coboundary(inp, out, 1, form_mask=(1 << 1) | (1 << 3), comp_axis=0)
    for chk in case["checks"]:
        i, j = chk["node"]
        assert np.all(out[0, :, i, :, j] == chk["value"]), chk


def test_codifferential_kat():
    """codifferential.cpp:38-118 -- delta of (x dx_s, y dy_s) is constant."""
    kat = EXT["codifferential_2d_1form"]
    n = kat["points"]
    x = np.linspace(kat["lower"], kat["upper"], n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    w = np.stack([X * kat["cochain_scale"], Y * kat["cochain_scale"]], -1)
    c = O.codifferential(2, 1, O.position_from_coords([x, x]), w, metric=O.identity_metric((n, n), 2))
    assert np.max(np.abs(c[1:-1, 1:-1, 0] - kat["expected"])) <= kat["tolerance"]


def test_hodge_star_kat():
    """hodge_star.cpp:66-181 -- dense metric: star(3 dx^dy)_z = 1.5 sqrt(6/19), then back to 3."""
    kat = EXT["hodge_star_3d_metric"]
    m = kat["metric"]
    g = np.array([[m["XX"], m["XY"], m["XZ"]], [m["XY"], m["YY"], m["YZ"]], [m["XZ"], m["YZ"], m["ZZ"]]])
    xs = np.linspace(kat["lower"], kat["upper"], kat["points"])
    pos = O.position_from_coords([xs, xs, xs])
    met = np.ascontiguousarray(np.broadcast_to(g.reshape(9), pos.shape[:-1] + (9,)))
    form = np.zeros(pos.shape[:-1] + (3,))
    form[..., 0] = kat["form_xy"]
    hs = O.fill_hodge_star(3, 2, pos, met)
    dual = O.apply_hodge_star(3, 2, hs, form)
    ulp = np.spacing(kat["expected_dual_z"])
    assert np.all(np.abs(dual[..., 2] - kat["expected_dual_z"]) <= kat["tolerance_ulps"] * ulp)
    back = O.apply_hodge_star(3, 1, O.fill_hodge_star(3, 1, pos, met), dual)
    assert np.all(np.abs(back[..., 0] - kat["expected_round_trip_xy"]) <= kat["tolerance_ulps"] * np.spacing(3.0))


def test_hodge_star_orthogonal_closed_form():
    """On an orthogonal grid with the identity metric the reference's
    reconstruction/continuous/reduction chain is the signed spacing ratio."""
    x = np.array([0.0, 0.3, 0.7, 1.6])
    y = np.array([-1.0, -0.5, 0.25])
    pos = O.position_from_coords([x, y])
    hx = np.array([0.3, 0.4, 0.9, 0.9])
    hy = np.array([0.5, 0.75, 0.75])
    for i in range(4):
        for j in range(3):
            m1 = O.hodge_matrix(2, 1, pos, (i, j))
            np.testing.assert_allclose(m1, [[0, -hx[i] / hy[j]], [hy[j] / hx[i], 0]], rtol=1e-14, atol=1e-15)
            m0 = O.hodge_matrix(2, 0, pos, (i, j))
            np.testing.assert_allclose(m0, [[hx[i] * hy[j]]], rtol=1e-14)
            m2 = O.hodge_matrix(2, 2, pos, (i, j))
            np.testing.assert_allclose(m2, [[1 / (hx[i] * hy[j])]], rtol=1e-14)


def _gate(name):
    return [g for g in EXT["laplacian_gates"] if g["name"] == name][0]


def _check_gate(values, coords, bands, tol):
    n_checked = 0
    for v, c in zip(values, coords):
        for lo, hi, expect in bands:
            if lo < c < hi:
                assert abs(v - expect) <= tol, (c, v, expect)
                n_checked += 1
    assert n_checked > 0


def test_laplacian_gate_1d():
    """laplacian.cpp 1D0Form / 1D1Form: Laplacian of -a r^2 (|r| <= R) is +1 (positive Laplacian)."""
    for name, k in (("1D0Form", 0), ("1D1Form", 1)):
        g = _gate(name)
        n, R, a = g["points"], g["R"], g["alpha"]
        x = np.linspace(-5, 5, n)
        r = np.abs(x)
        pot = np.where(r <= R, -a * r * r, -a * R * (2 * r - R))[:, None].copy()
        lap = O.laplacian(1, k, O.position_from_coords([x]), pot)
        xs = x[: n - 1]
        _check_gate(lap[1:-1, 0], xs[1:-1], [(-10, -1.2 * R, 0.0), (1.2 * R, 10, 0.0), (-0.8 * R, 0.8 * R, 1.0)],
                    g["tolerance"])


def test_laplacian_gate_2d():
    g = _gate("2D0Form")
    n, R, a = g["points"], g["R"], g["alpha"]
    x = np.linspace(-5, 5, n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    with np.errstate(divide="ignore"):
        pot = np.where(r <= R, -a * r * r, a * R * R * (2 * np.log(R / np.maximum(r, 1e-300)) - 1))[..., None].copy()
    lap = O.laplacian(2, 0, O.position_from_coords([x, x]), pot)
    _check_gate(lap[1:-1, n // 2, 0], x[1:n - 2], [(-10, -1.2 * R, 0.0), (1.2 * R, 10, 0.0), (-0.8 * R, 0.8 * R, 1.0)],
                g["tolerance"])
    g = _gate("2D1Form")
    fac = np.where(r <= R, r / 3 - R / 2, -R ** 3 / (6 * np.maximum(r, 1e-300) ** 2))
    pot = np.stack([Y * fac, -X * fac], -1)
    lap = O.laplacian(2, 1, O.position_from_coords([x, x]), pot)
    _check_gate(lap[1:-1, n // 2, 1], x[1:n - 2],
                [(-10, -1.2 * R, 0.0), (1.2 * R, 10, 0.0), (-0.8 * R, -0.2 * R, -1.0), (0.2 * R, 0.8 * R, 1.0)],
                g["tolerance"])


def test_laplacian_gate_3d():
    n = _gate("3D1Form")["points"]
    x = np.linspace(-5, 5, n)
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y + Z * Z)
    th = np.arctan2(Y, X)
    for name, k in (("3D1Form", 1), ("3D2Form", 2)):
        g = _gate(name)
        R, a = g["R"], g["alpha"]
        mag = np.where(r <= R, a * r * r, a * R ** 4 / np.maximum(r, 1e-300) ** 2)
        pos = O.position_from_coords([x, x, x])
        if k == 1:
            pot = np.stack([mag * np.sin(th), -mag * np.cos(th), np.zeros_like(r)], -1)
            comp, sign = 1, 1.0            # Y component
        else:
            pot = np.stack([np.zeros_like(r), mag * np.cos(th), mag * np.sin(th)], -1)  # (XY, XZ, YZ)
            comp, sign = 1, -1.0           # XZ component, opposite sign pattern
        lap = O.laplacian(3, k, pos, np.ascontiguousarray(pot))
        _check_gate(lap[1:-1, n // 2, n // 2, comp], x[1:n - 2],
                    [(-10, -1.3 * R, 0.0), (1.3 * R, 10, 0.0), (-0.7 * R, -0.3 * R, -sign), (0.3 * R, 0.7 * R, sign)],
                    g["tolerance"])


def test_staged_matches_oneshot():
    """Prefilled staged chain == one-shot chain (same reference structure)."""
    rng = np.random.default_rng(3)
    x = np.cumsum(rng.uniform(0.5, 1.5, 9))
    y = np.cumsum(rng.uniform(0.5, 1.5, 7))
    pos = O.position_from_coords([x, y])
    for k in range(3):
        inp = rng.standard_normal((9, 7, len(combos(2, k))))
        a = O.laplacian(2, k, pos, inp)
        st = O.StagedLaplacian(2, k, pos)
        b = np.zeros_like(a)
        st.run(inp, b)
        assert np.array_equal(a, b)


def test_mag2d_operator_symmetric_on_interior():
    rng = np.random.default_rng(0)
    nx, ny = 9, 7
    mu = rng.uniform(1.0, 5.0, nx * ny)
    interior = np.zeros((ny, nx), bool)
    interior[1:-1, 1:-1] = True
    interior = interior.ravel()
    cols = []
    for c in np.flatnonzero(interior):
        e = np.zeros(nx * ny)
        e[c] = 1.0
        cols.append(O.mag2d_apply(nx, ny, mu, e)[interior])
    K = np.array(cols).T
    np.testing.assert_allclose(K, K.T, rtol=1e-14, atol=1e-14)
    assert np.all(np.linalg.eigvalsh(K) > 0)
    np.testing.assert_allclose(np.diag(K), O.mag2d_diagonal(nx, ny, mu)[interior], rtol=1e-14)


def test_mag2d_cg_converges():
    nx, ny = 33, 29
    x = np.linspace(0, 1, nx)
    y = np.linspace(0, 1, ny)
    cj = np.zeros((ny - 1) * (nx - 1))
    cj.reshape(ny - 1, nx - 1)[10:18, 8:20] = 1.0
    cm = np.ones_like(cj)
    cm.reshape(ny - 1, nx - 1)[3:9, 3:25] = 1000.0
    mu = O.mag2d_node_mu(nx, ny, cm)
    b = O.mag2d_rhs(x, y, cj)
    sol, it, rel = O.mag2d_cg(nx, ny, mu, b, tol=1e-10)
    r = b - O.mag2d_apply(nx, ny, mu, sol)
    assert np.linalg.norm(r) <= 1.1e-10 * np.linalg.norm(b)
    assert it > 10


def test_mag3d_host_setup_matches_oracle():
    from similie_b200 import magnetostatics3d as m3
    rng = np.random.default_rng(3)
    p = m3.synthetic_problem(rng, 14, tube=0.15)
    nx, ny, nz = p.shape
    np.testing.assert_allclose(p.node_mu(), O.mag3d_node_mu(nx, ny, nz, p.cell_mu), rtol=1e-15)
    np.testing.assert_allclose(p.rhs(), O.mag3d_rhs(p.x, p.y, p.z, p.cell_j), rtol=1e-13, atol=1e-18)
    assert np.count_nonzero(p.cell_j) > 0


def test_mag3d_stretched_coords():
    from similie_b200 import magnetostatics3d as m3
    x = m3.stretched_coords(256, 1.01)
    h = np.diff(x)
    assert x[0] == 0.0 and abs(x[-1] - 1.0) < 1e-15
    np.testing.assert_allclose(h[1:] / h[:-1], 1.01, rtol=1e-12)


def test_mag3d_oracle_operator_properties():
    """Interior block symmetric positive definite, diagonal consistent, CG converges."""
    from similie_b200 import magnetostatics3d as m3
    rng = np.random.default_rng(9)
    nx, ny, nz = 5, 6, 5
    x, y, z = m3.stretched_coords(nx, 1.1), m3.stretched_coords(ny, 0.9), m3.stretched_coords(nz, 1.05)
    mu = rng.uniform(1.0, 10.0, nx * ny * nz)
    n = 3 * nx * ny * nz
    A = np.stack([O.mag3d_apply(x, y, z, mu, 20.0, e) for e in np.eye(n)], axis=1)
    b = np.zeros((nz, ny, nx, 3), dtype=bool)
    b[0] = b[-1] = True
    b[:, 0] = b[:, -1] = True
    b[:, :, 0] = b[:, :, -1] = True
    inner = np.flatnonzero(~b.ravel())
    K = A[np.ix_(inner, inner)]
    assert np.abs(K - K.T).max() <= 1e-13 * np.abs(K).max()
    assert np.linalg.eigvalsh(K).min() > 0
    np.testing.assert_allclose(O.mag3d_diagonal(x, y, z, mu, 20.0), np.diag(A), rtol=1e-13)
    rhs = np.zeros(n)
    rhs[inner] = rng.standard_normal(inner.size)
    sol, it, rel = O.mag3d_cg(x, y, z, mu, 20.0, rhs, tol=1e-11)
    assert rel <= 1e-11 and np.linalg.norm(A @ sol - rhs) <= 1e-10 * np.linalg.norm(rhs)


def _greville_cubic(lo, hi, ncells):
    """Greville points of uniform cubic B-splines with clamped knots on
    [lo, hi] (the reference examples' Mesher<3>, ncells + 3 points): the knot
    averages, uniform inside and lo + h/3, hi - h/3 next to the ends."""
    h = (hi - lo) / ncells
    inner = lo + h * np.arange(1, ncells)
    return np.concatenate([[lo, lo + h / 3.0], inner, [hi - h / 3.0, hi]])


def _example_index(frac, extent):
    return int(np.floor(frac * (extent - 1) + 0.5))      # std::llround on a positive value


def test_examples_2d_laplacian_correctness_checks():
    """examples/2d_laplacian.cpp:97-113, 240-251: potential -alpha r^2 inside
    R = 2 and alpha R^2 (2 log(R/r) - 1) outside on the 1003^2 Greville grid
    of [-5, 5]^2; the Laplacian (a positive operator) is 1 near (5/8 Lx, 0)
    and 0 near (7/8 Lx, 0), within 5e-2."""
    x = _greville_cubic(-5.0, 5.0, 1000)
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    R, alpha = 2.0, 0.25
    rs = np.where(r <= R, 1.0, r)          # the outside branch is only taken away from the origin
    phi = np.where(r <= R, -alpha * r * r, alpha * R * R * (2.0 * np.log(R / rs) - 1.0))
    lap = O.laplacian(2, 0, O.position_from_coords([x, x]), phi[..., None])
    ext = lap.shape[0]
    iy = _example_index(0.5, ext)
    assert abs(lap[_example_index(5 / 8, ext), iy, 0] - 1.0) <= 5e-2
    assert abs(lap[_example_index(7 / 8, ext), iy, 0] - 0.0) <= 5e-2


def test_examples_2d_vector_laplacian_correctness_checks():
    """examples/2d_vector_laplacian.cpp:189-215, 241-267: the rotational
    1-form field of the example; the Laplacian's magnitude is 1 near
    (5/8 Lx, 0) and 0 near (7/8 Lx, 0), within 5e-2."""
    x = _greville_cubic(-5.0, 5.0, 1000)
    X, Y = np.meshgrid(x, x, indexing="ij")
    r = np.sqrt(X * X + Y * Y)
    R = 2.0
    inside = r <= R
    rs = np.where(inside, 1.0, r)          # the outside branch is only taken away from the origin
    w = np.zeros(X.shape + (2,))
    w[..., 0] = np.where(inside, Y * (r / 3.0 - R / 2.0), -Y * R ** 3 / (6.0 * rs * rs))
    w[..., 1] = np.where(inside, -X * (r / 3.0 - R / 2.0), X * R ** 3 / (6.0 * rs * rs))
    lap = O.laplacian(2, 1, O.position_from_coords([x, x]), w)
    ext = lap.shape[0]
    iy = _example_index(0.5, ext)
    for frac, expected in ((5 / 8, 1.0), (7 / 8, 0.0)):
        v = lap[_example_index(frac, ext), iy]
        assert abs(np.hypot(v[0], v[1]) - expected) <= 5e-2


def _kat_position(fn):
    """Positions of the reference's 2 x 2 test lattice: UniformPointSampling
    on [0, 2] with 2 points, so xi, eta in {0, 2}."""
    c = np.array([0.0, 2.0])
    xi, eta = np.meshgrid(c, c, indexing="ij")
    px, py = fn(xi, eta)
    return np.ascontiguousarray(np.stack([px, py], axis=-1))


@pytest.mark.parametrize("k,form,reduced", [(0, [3.5], [3.5]), (1, [3.0, -1.0], [6.0, 2.0]), (2, [4.0], [32.0])])
def test_reduction_kat(k, form, reduced):
    """tests/exterior/reduction_and_reconstruction.cpp:231-283: primal
    reduction of constant forms on the sheared lattice (xi + eta, 2 eta)."""
    pos = _kat_position(lambda xi, eta: (xi + eta, 2.0 * eta))
    assert list(O.reduce_primal(2, k, pos, [0, 0], form)) == reduced


@pytest.mark.parametrize("k,form", [(0, [3.5]), (1, [3.0, -1.0]), (2, [4.0])])
def test_reconstruction_kat(k, form):
    """tests/exterior/reduction_and_reconstruction.cpp:285-329: reduce, then
    reconstruct, on the lattice (2 xi, 3 eta): the form comes back."""
    pos = _kat_position(lambda xi, eta: (2.0 * xi, 3.0 * eta))
    red = O.reduce_primal(2, k, pos, [0, 0], form)
    assert list(O.reconstruct_primal(2, k, pos, [0, 0], red)) == form
