"""GPU parity of the DEC operators against the CPU oracle.

Bar: the coboundary and its transpose are bit-exact in FP64; the Hodge star,
codifferential and Laplacian agree with the oracle to 1e-12 relative
(max-norm over the field); FP32 variants state their error against the FP64
oracle (bound 1e-5 relative here)."""
from math import comb

import numpy as np
import pytest

import oracle as O
from helpers import (comp_index, gaussian_random_field, kat_field, load_golden, rel_err, sinusoid_field,
                     stretched_coords)

pytestmark = pytest.mark.gpu

TOL = 1e-12


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


def dev(torch, a, dtype=None):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype or torch.float64)


def host(t):
    return t.detach().cpu().double().numpy()


# ----------------------------------------------------------------- coboundary

DER = load_golden("derivative_kat.json")
EXT = load_golden("exterior_kat.json")


@pytest.mark.parametrize("case", [t for t in DER["tests"] if "spectators" not in t],
                         ids=lambda t: f"{t['name']}-{t['variant']}")
def test_deriv_kat_gpu(torch, sil, case):
    N, ndim, k_in, k_out = case["N"], len(case["dims"]), case["k_in"], case["k_out"]
    f = kat_field(N, ndim, k_in)
    out_n = N if k_out == 1 else N - 1
    nco = comb(ndim, k_out)
    if case["component_first"]:
        inp = dev(torch, np.moveaxis(f, -1, 0))
        out = torch.full((nco,) + (out_n,) * ndim, float("nan"), device="cuda", dtype=torch.float64)
        sil.deriv(out, inp, k_in, comp_axis=0)
        res = np.moveaxis(host(out), 0, -1)
    else:
        inp = dev(torch, f)
        out = torch.full((out_n,) * ndim + (nco,), float("nan"), device="cuda", dtype=torch.float64)
        sil.deriv(out, inp, k_in)
        res = host(out)
    for chk in case["checks"]:
        assert res[tuple(chk["node"]) + (comp_index(ndim, chk["comp_dims"]),)] == chk["value"]
    ref = np.full_like(res, np.nan)
    O.coboundary(f, ref, k_in)
    assert np.array_equal(res, ref)


def test_deriv_kat_spectators_gpu(torch, sil):
    inp = np.zeros((2, 3, 3, 10, 3))
    for c in range(2):
        inp[c] = c + 1.0
        inp[c, :, 1, :, 1] = c + 2.0
    out = torch.full((1, 3, 2, 10, 2), float("nan"), device="cuda", dtype=torch.float64)
    sil.deriv(out, dev(torch, inp), 1, form_dims=(1, 3), comp_axis=0)
    res = host(out)
    case = [t for t in DER["tests"] if t["name"] == "2DRotationalWithSpects"][0]
    for chk in case["checks"]:
        i, j = chk["node"]
        assert np.all(res[0, :, i, :, j] == chk["value"])


def _random_case(rng, n, k, transposed):
    shape = tuple(int(s) for s in rng.integers(3, 9, size=n))
    inp = rng.standard_normal(shape + (comb(n, k),))
    # output box: arbitrary front/extent overlapping the input (clamped or zero-outside sampling)
    front = tuple(int(v) for v in rng.integers(-1, 2, size=n))
    oshape = tuple(int(max(1, s + int(rng.integers(-2, 2)))) for s in shape)
    return inp, front, oshape


@pytest.mark.parametrize("n", [1, 2, 3, 4])
@pytest.mark.parametrize("transposed", [False, True])
def test_coboundary_random_bit_exact(torch, sil, n, transposed):
    rng = np.random.default_rng(100 + n + 10 * transposed)
    for k in range(n):
        for comp_first in (False, True):
            inp, front, oshape = _random_case(rng, n, k, transposed)
            nco = comb(n, k + 1)
            ref = np.full(oshape + (nco,), np.nan)
            fn = O.transposed_coboundary if transposed else O.coboundary
            fn(inp, ref, k, out_front=front)
            if comp_first:
                ti = dev(torch, np.moveaxis(inp, -1, 0))
                to = torch.full((nco,) + oshape, float("nan"), device="cuda", dtype=torch.float64)
                g = sil.transposed_coboundary if transposed else sil.deriv
                g(to, ti, k, comp_axis=0, out_front=front)
                res = np.moveaxis(host(to), 0, -1)
            else:
                ti = dev(torch, inp)
                to = torch.full(oshape + (nco,), float("nan"), device="cuda", dtype=torch.float64)
                g = sil.transposed_coboundary if transposed else sil.deriv
                g(to, ti, k, out_front=front)
                res = host(to)
            assert np.array_equal(res, ref), (n, k, comp_first)


def test_coboundary_fp32(torch, sil):
    rng = np.random.default_rng(7)
    inp = rng.standard_normal((33, 17, 2)).astype(np.float32)
    ref = np.zeros((32, 16, 1))
    O.coboundary(inp.astype(np.float64), ref, 1)
    out = torch.zeros((32, 16, 1), device="cuda", dtype=torch.float32)
    sil.deriv(out, dev(torch, inp, torch.float32), 1)
    assert rel_err(host(out), ref) < 1e-6


# ----------------------------------------------------------------- Hodge star

def _geometry(sil, coords):
    return sil.Geometry(coords)


def _coords(rng, shape):
    return [np.cumsum(rng.uniform(0.3, 1.7, s)) for s in shape]


@pytest.mark.parametrize("n", [1, 2, 3])
def test_hodge_star_vs_oracle(torch, sil, n):
    rng = np.random.default_rng(20 + n)
    shape = tuple(int(s) for s in rng.integers(3, 7, size=n))
    coords = _coords(rng, shape)
    geo = _geometry(sil, coords)
    pos = O.position_from_coords(coords)
    for k in range(n + 1):
        inp = rng.standard_normal(shape + (comb(n, k),))
        ref = O.apply_hodge_star(n, k, O.fill_hodge_star(n, k, pos), inp)
        out = torch.zeros(shape + (comb(n, n - k),), device="cuda", dtype=torch.float64)
        sil.hodge_star(geo, out, dev(torch, inp), k)
        assert rel_err(host(out), ref) <= TOL, (n, k)


@pytest.mark.parametrize("shape", [(9, 7, 300), (5, 3, 6), (3, 4, 2), (4, 5, 7)])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
def test_hodge_star_dense_3d_path_matches_table_driven(torch, sil, dtype, shape):
    """Dense [x][y][z][c] fields take the row kernel (FP64 1- and 2-forms with
    an even z extent: the node-pair kernel over one flat range of pairs); a
    strided view of the same data takes the table-driven kernel; both must
    agree bit for bit."""
    rng = np.random.default_rng(77)
    coords = _coords(rng, shape)
    geo = _geometry(sil, coords)
    dt = getattr(torch, dtype)
    for k in range(4):
        inp = torch.from_numpy(rng.standard_normal(shape + (comb(3, k),))).to(dt).cuda()
        dense = torch.zeros(shape + (comb(3, 3 - k),), device="cuda", dtype=dt)
        sil.hodge_star(geo, dense, inp, k)
        big = torch.zeros(shape + (comb(3, 3 - k) + 1,), device="cuda", dtype=dt)
        strided = big[..., : comb(3, 3 - k)]            # comp stride 1, node stride ncomp + 1: not dense
        sil.hodge_star(geo, strided, inp, k)
        assert torch.equal(dense, strided), k


@pytest.mark.parametrize("n", [1, 2, 3])
def test_fill_hodge_star_general_metric_vs_oracle(torch, sil, n):
    """Dense per-node SPD metric on a perturbed (non-orthogonal) lattice: the GPU
    restatement of fill_discrete_hodge_star matches the oracle for every rank,
    and the stored tensor applied on the GPU matches the oracle's tensor_prod."""
    rng = np.random.default_rng(90 + n)
    shape = tuple(int(s) for s in rng.integers(3, 6, size=n))
    coords = _coords(rng, shape)
    pos = O.position_from_coords(coords) + 0.02 * rng.standard_normal(shape + (n,))
    a = rng.standard_normal(shape + (n, n)) * 0.3
    met = np.einsum("...ij,...kj->...ik", a, a) + np.eye(n)
    met = np.ascontiguousarray(met.reshape(shape + (n * n,)))
    for k in range(n + 1):
        ref = O.fill_hodge_star(n, k, pos, met)
        out = torch.full(ref.shape, float("nan"), device="cuda", dtype=torch.float64)
        sil.fill_discrete_hodge_star_metric(out, dev(torch, pos), k, metric=dev(torch, met))
        assert rel_err(host(out), ref) <= TOL, (n, k)
        form = rng.standard_normal(shape + (comb(n, k),))
        dref = O.apply_hodge_star(n, k, ref, form)
        dgpu = torch.zeros(shape + (comb(n, n - k),), device="cuda", dtype=torch.float64)
        sil.hodge_star_stored(out, dgpu, dev(torch, form), n, k)
        assert rel_err(host(dgpu), dref) <= TOL, (n, k)


def test_hodge_star_dense_metric_kat_gpu(torch, sil):
    """hodge_star.cpp:66-181 on the GPU: star(3 dx^dy)_z = 1.5 sqrt(6/19) with the
    test's dense metric, and back to 3, within the reference's 4 ULP."""
    kat = EXT["hodge_star_3d_metric"]
    m = kat["metric"]
    g = np.array([[m["XX"], m["XY"], m["XZ"]], [m["XY"], m["YY"], m["YZ"]], [m["XZ"], m["YZ"], m["ZZ"]]])
    xs = np.linspace(kat["lower"], kat["upper"], kat["points"])
    pos = O.position_from_coords([xs, xs, xs])
    met = np.ascontiguousarray(np.broadcast_to(g.reshape(9), pos.shape[:-1] + (9,)))
    form = np.zeros(pos.shape[:-1] + (3,))
    form[..., 0] = kat["form_xy"]
    shape = pos.shape[:-1]
    h2 = torch.zeros(shape + (9 * 3,), device="cuda", dtype=torch.float64)
    sil.fill_discrete_hodge_star_metric(h2, dev(torch, pos), 2, metric=dev(torch, met))
    dual = torch.zeros(shape + (3,), device="cuda", dtype=torch.float64)
    sil.hodge_star_stored(h2, dual, dev(torch, form), 3, 2)
    d = host(dual)
    ulp = np.spacing(kat["expected_dual_z"])
    assert np.all(np.abs(d[..., 2] - kat["expected_dual_z"]) <= kat["tolerance_ulps"] * ulp)
    h1 = torch.zeros(shape + (3 * 3,), device="cuda", dtype=torch.float64)
    sil.fill_discrete_hodge_star_metric(h1, dev(torch, pos), 1, metric=dev(torch, met))
    back = torch.zeros(shape + (3,), device="cuda", dtype=torch.float64)
    sil.hodge_star_stored(h1, back, dual, 3, 1)
    assert np.all(np.abs(host(back)[..., 0] - kat["expected_round_trip_xy"]) <= kat["tolerance_ulps"] * np.spacing(3.0))


@pytest.mark.parametrize("n", [1, 2, 3])
def test_fill_discrete_hodge_star_vs_oracle(torch, sil, n):
    rng = np.random.default_rng(30 + n)
    shape = tuple(int(s) for s in rng.integers(3, 6, size=n))
    coords = _coords(rng, shape)
    geo = _geometry(sil, coords)
    pos = O.position_from_coords(coords)
    for k in range(n + 1):
        ref = O.fill_hodge_star(n, k, pos)
        out = torch.full(ref.shape, float("nan"), device="cuda", dtype=torch.float64)
        sil.fill_discrete_hodge_star(geo, out, k)
        assert rel_err(host(out), ref) <= TOL, (n, k)


# ----------------------------------------------------------------- codifferential / Laplacian

@pytest.mark.parametrize("n", [1, 2, 3])
def test_codifferential_vs_oracle(torch, sil, n):
    rng = np.random.default_rng(40 + n)
    shape = tuple(int(s) for s in rng.integers(4, 9, size=n))
    coords = _coords(rng, shape)
    geo = _geometry(sil, coords)
    pos = O.position_from_coords(coords)
    for k in range(1, n + 1):
        inp = rng.standard_normal(shape + (comb(n, k),))
        ref = O.codifferential(n, k, pos, inp)
        out = torch.zeros(shape + (comb(n, k - 1),), device="cuda", dtype=torch.float64)
        sil.codifferential(geo, out, dev(torch, inp), k)
        assert rel_err(host(out), ref) <= TOL, (n, k)


def test_codifferential_kat_gpu(torch, sil):
    kat = load_golden("exterior_kat.json")["codifferential_2d_1form"]
    n = kat["points"]
    x = np.linspace(kat["lower"], kat["upper"], n)
    X, Y = np.meshgrid(x, x, indexing="ij")
    w = np.stack([X * kat["cochain_scale"], Y * kat["cochain_scale"]], -1)
    out = torch.zeros((n, n, 1), device="cuda", dtype=torch.float64)
    sil.codifferential(sil.Geometry([x, x]), out, dev(torch, w), 1)
    assert np.max(np.abs(host(out)[1:-1, 1:-1, 0] - kat["expected"])) <= kat["tolerance"]


@pytest.mark.parametrize("n", [1, 2, 3])
@pytest.mark.parametrize("mode", ["fused", "unfused"])
def test_laplacian_vs_oracle(torch, sil, n, mode):
    rng = np.random.default_rng(50 + n)
    shape = tuple(int(s) for s in rng.integers(5, 10, size=n))
    coords = _coords(rng, shape)
    geo = _geometry(sil, coords)
    pos = O.position_from_coords(coords)
    for k in range(n + 1):
        inp = rng.standard_normal(shape + (comb(n, k),))
        for oshape in (tuple(s - 1 for s in shape), shape):
            ref = O.laplacian(n, k, pos, inp, out_shape=oshape)
            out = torch.zeros(oshape + (comb(n, k),), device="cuda", dtype=torch.float64)
            ti = dev(torch, inp)
            st = sil.make_staged_laplacian(geo, out, ti, k, mode=mode)
            st.run(out, ti)
            st.status()
            assert rel_err(host(out), ref) <= TOL, (n, k, oshape, mode, st.kernel)


def test_laplacian_free_function(torch, sil):
    rng = np.random.default_rng(61)
    coords = _coords(rng, (12, 9))
    pos = O.position_from_coords(coords)
    geo = _geometry(sil, coords)
    for k in range(3):
        inp = rng.standard_normal((12, 9, comb(2, k)))
        ref = O.laplacian(2, k, pos, inp)
        out = torch.zeros((11, 8, comb(2, k)), device="cuda", dtype=torch.float64)
        sil.laplacian(geo, out, dev(torch, inp), k)
        assert rel_err(host(out), ref) <= TOL


def _two_d_case(rng, nx, ny, stretched=True):
    if stretched:
        coords = [stretched_coords(nx, 1.003), stretched_coords(ny, 0.998, start=-0.5)]
    else:
        coords = [np.arange(nx) / nx, np.arange(ny) / ny]
    return coords


@pytest.mark.parametrize("shape", [(67, 300), (130, 257), (9, 129), (300, 128)])
def test_tma_1form_kernel_matches_generic_and_oracle(torch, sil, shape):
    """The TMA-staged 1-form kernel agrees bit for bit with the table-driven
    fused kernel and to 1e-12 with the oracle; odd sizes exercise partial
    strips and segment boundaries."""
    nx, ny = shape
    rng = np.random.default_rng(nx * 1000 + ny)
    coords = _two_d_case(rng, nx, ny)
    geo = _geometry(sil, coords)
    inp = rng.standard_normal((nx, ny, 2))
    ti = dev(torch, inp)
    out = torch.full((nx - 1, ny - 1, 2), float("nan"), device="cuda", dtype=torch.float64)
    st = sil.make_staged_laplacian(geo, out, ti, 1)
    assert st.kernel == 2
    st.run(out, ti)
    st.status()
    gen = torch.full_like(out, float("nan"))
    sil.laplacian(geo, gen, ti, 1)
    a, b = host(out), host(gen)
    assert np.array_equal(a, b)
    ref = O.laplacian(2, 1, O.position_from_coords(coords), inp)
    assert rel_err(a, ref) <= TOL


@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("shape", [(67, 300), (45, 1100), (130, 513), (900, 260)])
def test_every_tma_pipeline_shape_is_bit_exact(torch, sil, shape, dtype, monkeypatch):
    """Every pipeline shape the autotuner may pick -- the single-column
    shapes 0-5 and the FP64 column-pair shapes 6-8 (512-column strips; FP32
    runs shape 0 there) -- agrees bit for bit with the table-driven kernel;
    the widths exercise partial 512-column strips and the quarter-box and
    halo neighbours, the heights bands of one row up to bands of many."""
    nx, ny = shape
    if dtype == "float32" and ny % 2:
        pytest.skip("the FP32 TMA kernel takes even y extents")
    dt = getattr(torch, dtype)
    rng = np.random.default_rng(nx + 7 * ny)
    coords = _two_d_case(rng, nx, ny)
    geo = _geometry(sil, coords)
    inp = rng.standard_normal((nx, ny, 2))
    ti = dev(torch, inp, dt)
    gen = torch.full((nx - 1, ny - 1, 2), float("nan"), device="cuda", dtype=dt)
    sil.laplacian(geo, gen, ti, 1)
    ref = host(gen)
    for v in range(9):
        monkeypatch.setenv("SIMILIE_B200_LAP1_VARIANT", str(v))
        out = torch.full_like(gen, float("nan"))
        st = sil.make_staged_laplacian(geo, out, ti, 1)
        assert st.kernel == 2
        st.run(out, ti)
        st.status()
        assert st.variant == v
        assert np.array_equal(host(out), ref), v


def test_tma_1form_kernel_output_offset(torch, sil):
    """Output box starting inside the input (nonzero front offset)."""
    rng = np.random.default_rng(5)
    nx, ny = 70, 200
    coords = _two_d_case(rng, nx, ny)
    geo = _geometry(sil, coords)
    inp = rng.standard_normal((nx, ny, 2))
    ti = dev(torch, inp)
    out = torch.zeros((50, 150, 2), device="cuda", dtype=torch.float64)
    st = sil.make_staged_laplacian(geo, out, ti, 1, out_front=(5, 7))
    assert st.kernel == 2
    st.run(out, ti)
    ref = O.laplacian(2, 1, O.position_from_coords(coords), inp, out_shape=(nx - 1, ny - 1))
    assert rel_err(host(out), ref[5:55, 7:157]) <= TOL


def test_tma_1form_kernel_fp32(torch, sil):
    rng = np.random.default_rng(6)
    nx, ny = 130, 516
    coords = _two_d_case(rng, nx, ny)
    geo = _geometry(sil, coords)
    inp = gaussian_random_field(max(nx, ny), 9)[:nx, :ny]
    ti = dev(torch, inp, torch.float32)
    out = torch.zeros((nx - 1, ny - 1, 2), device="cuda", dtype=torch.float32)
    st = sil.make_staged_laplacian(geo, out, ti, 1)
    assert st.kernel == 2
    st.run(out, ti)
    gen = torch.zeros_like(out)
    sil.laplacian(geo, gen, ti, 1)
    assert np.array_equal(host(out), host(gen))
    ref = O.laplacian(2, 1, O.position_from_coords(coords), inp.astype(np.float32).astype(np.float64))
    assert rel_err(host(out), ref) < 1e-5


def test_scalar_laplacian_512(torch, sil):
    """512^2 0-form workload: uniform spacing 1/512, sinusoidal modes + noise."""
    n = 512
    phi = sinusoid_field(n, seed=1)
    coords = [np.arange(n) / n, np.arange(n) / n]
    geo = _geometry(sil, coords)
    ti = dev(torch, phi[..., None])
    out = torch.zeros((n - 1, n - 1, 1), device="cuda", dtype=torch.float64)
    st = sil.make_staged_laplacian(geo, out, ti, 0)
    assert st.kernel == 1
    st.run(out, ti)
    ref = O.laplacian(2, 0, O.position_from_coords(coords), phi[..., None])
    assert rel_err(host(out), ref) <= TOL
    d = torch.zeros((n, n, 2), device="cuda", dtype=torch.float64)
    sil.deriv(d, ti, 0)
    dref = np.zeros((n, n, 2))
    O.coboundary(phi[..., None].copy(), dref, 0)
    assert np.array_equal(host(d), dref)


def test_vector_laplacian_4096_windows(torch, sil):
    """Full 4096^2 1-form workload (k^-2 Gaussian random field) through the
    TMA kernel, compared with the oracle on windows covering the corners, the
    edges and the interior (operators are local: each window carries a 3-node
    margin that is excluded from the comparison unless it is a true edge)."""
    n = 4096
    w = gaussian_random_field(n, seed=2)
    coords = [np.arange(n) / n, np.arange(n) / n]
    geo = _geometry(sil, coords)
    ti = dev(torch, w)
    out = torch.zeros((n - 1, n - 1, 2), device="cuda", dtype=torch.float64)
    st = sil.make_staged_laplacian(geo, out, ti, 1)
    assert st.kernel == 2
    st.run(out, ti)
    st.status()
    res = host(out)
    m = 3
    for (i0, j0) in [(0, 0), (0, n - 64), (n - 64, 0), (n - 64, n - 64), (2000, 1500), (0, 2048), (1024, 0)]:
        i1, j1 = min(i0 + 64, n), min(j0 + 64, n)
        a0, b0 = max(i0 - m, 0), max(j0 - m, 0)
        a1, b1 = min(i1 + m, n), min(j1 + m, n)
        sub = np.ascontiguousarray(w[a0:a1, b0:b1])
        subc = [coords[0][a0:a1], coords[1][b0:b1]]
        ref = O.laplacian(2, 1, O.position_from_coords(subc), sub, out_shape=sub.shape[:2])
        # valid region: away from artificial window edges
        vi0 = 0 if a0 == 0 else m
        vj0 = 0 if b0 == 0 else m
        vi1 = (a1 - a0) - (1 if a1 == n else m)
        vj1 = (b1 - b0) - (1 if b1 == n else m)
        got = res[a0 + vi0:a0 + vi1, b0 + vj0:b0 + vj1]
        assert rel_err(got, ref[vi0:vi1, vj0:vj1]) <= TOL, (i0, j0)


@pytest.mark.parametrize("k,n", [(1, 700), (0, 600)])
def test_chained_runs_read_the_previous_runs_output(torch, sil, k, n):
    """Back-to-back runs where each run reads the previous run's output, with
    no synchronisation between them and again replayed from a CUDA graph: the
    kernels may start early (programmatic dependent launch) but read their
    input only once the previous run has finished, so the chain equals the
    one run step by step with a synchronisation after each, bit for bit."""
    rng = np.random.default_rng(40 + k)
    coords = _two_d_case(rng, n, n)
    geo = _geometry(sil, coords)
    nc = 2 if k == 1 else 1
    fields = [dev(torch, rng.standard_normal((n, n, nc)))]
    for s in range(1, 4):
        fields.append(torch.full((n - s, n - s, nc), float("nan"), device="cuda", dtype=torch.float64))
    plans = [sil.make_staged_laplacian(geo, fields[s + 1], fields[s], k) for s in range(3)]
    for s, p in enumerate(plans):
        assert p.kernel == (2 if k == 1 else 1)
        p.run(fields[s + 1], fields[s])
        torch.cuda.synchronize()
        p.status()
    ref = fields[3].clone()
    for _ in range(3):
        for f in fields[1:]:
            f.fill_(float("nan"))
        for s, p in enumerate(plans):
            p.run(fields[s + 1], fields[s])
        torch.cuda.synchronize()
        assert torch.equal(fields[3], ref)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for s, p in enumerate(plans):
            p.run(fields[s + 1], fields[s])
    torch.cuda.current_stream().wait_stream(side)
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for s, p in enumerate(plans):
            p.run(fields[s + 1], fields[s])
    for _ in range(3):
        for f in fields[1:]:
            f.fill_(float("nan"))
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(fields[3], ref)
