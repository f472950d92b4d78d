"""Structured-grid ingestion from msh2 meshes: the C++ reader
(include/sil/gmsh_structured_grid.hpp, through tests/cpp/gmsh_reader.cpp) and
the Python one recover the grid coordinates and the per-cell physical tags of
shuffled 2D and 3D meshes, reject what the reference rejects, and the result
feeds the magnetostatics inputs."""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
import similie_b200.gmsh_grid as G
import similie_b200.magnetostatics as mag

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def reader(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("no g++")
    exe = str(tmp_path_factory.mktemp("gmsh") / "gmsh_reader")
    subprocess.check_call([gxx, "-std=c++17", "-O1", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "cpp", "gmsh_reader.cpp"), "-o", exe])

    def run(path):
        out = subprocess.run([exe, str(path)], check=True, capture_output=True, text=True).stdout.split("\n")
        if out[0].startswith("error"):
            return out[0]
        dim = int(out[0].split()[1])
        coords = [np.array([float(v) for v in out[1 + a].split()[2:]]) for a in range(dim)]
        tags = np.array([int(v) for v in out[1 + dim].split()[1:]])
        return dim, coords, tags
    return run


def _grids():
    rng = np.random.default_rng(4)
    x = np.cumsum(np.r_[0.0, rng.uniform(0.05, 0.2, 8)])
    y = np.cumsum(np.r_[-0.3, rng.uniform(0.05, 0.2, 6)])
    z = np.cumsum(np.r_[1.0, rng.uniform(0.1, 0.3, 2)])
    t2 = rng.integers(1, 4, (len(x) - 1) * (len(y) - 1))
    t3 = rng.integers(1, 4, (len(x) - 1) * (len(y) - 1) * (len(z) - 1))
    return [([x, y], t2), ([x, y, z], t3)]


@pytest.mark.parametrize("case", [0, 1])
def test_both_readers_recover_the_grid(tmp_path, reader, case):
    coords, tags = _grids()[case]
    path = tmp_path / "mesh.msh"
    G.write_msh2(str(path), coords, tags, seed=11)
    dim, got, gt, _ = G.read_structured_grid(str(path))
    assert dim == len(coords)
    for a in range(dim):
        np.testing.assert_array_equal(got[a], coords[a])
    np.testing.assert_array_equal(gt, tags)
    cdim, cgot, ctags = reader(path)
    assert cdim == dim
    for a in range(dim):
        np.testing.assert_array_equal(cgot[a], coords[a])
    np.testing.assert_array_equal(ctags, tags)


def _edit(path, drop_element=None, replace=None):
    lines = open(path).read().split("\n")
    if replace:
        lines = [replace.get(l, l) for l in lines]
    if drop_element is not None:
        i = lines.index("$Elements")
        n = int(lines[i + 1])
        body = lines[i + 2:i + 2 + n]
        quads = [l for l in body if l.split()[1] in ("3", "5")]
        body.remove(quads[drop_element])
        lines = lines[:i + 1] + [str(n - 1)] + body + lines[i + 2 + n:]
    open(path, "w").write("\n".join(lines))


def test_rejections(tmp_path, reader):
    coords, tags = _grids()[0]
    p = tmp_path / "m.msh"
    # a missing cell
    G.write_msh2(str(p), coords, tags, seed=3)
    _edit(p, drop_element=0)
    with pytest.raises(ValueError, match="cover"):
        G.read_structured_grid(str(p))
    assert "cover" in reader(p)
    # msh4
    G.write_msh2(str(p), coords, tags)
    _edit(p, replace={"2.2 0 8": "4.1 0 8"})
    with pytest.raises(ValueError, match="msh2"):
        G.read_structured_grid(str(p))
    assert "msh2" in reader(p)
    # a triangle in the mesh
    G.write_msh2(str(p), coords, tags)
    txt = open(p).read().replace("$EndElements", "")
    lines = txt.rstrip("\n").split("\n")
    i = lines.index("$Elements")
    lines[i + 1] = str(int(lines[i + 1]) + 1)
    lines.append(f"{int(lines[i + 1])} 2 2 7 7 1 2 3")
    open(p, "w").write("\n".join(lines) + "\n$EndElements\n")
    with pytest.raises(ValueError, match="topology"):
        G.read_structured_grid(str(p))
    assert "topology" in reader(p)


def test_ingested_grid_feeds_the_solver(tmp_path):
    # a 17 x 17 unit-square grid: tag 2 = permeability-1000 core, tag 3 = coil
    n = 17
    x = np.linspace(0.0, 1.0, n)
    tags = np.ones((n - 1, n - 1), dtype=np.int64)
    tags[6:10, 6:10] = 2
    tags[2:4, 2:5] = 3
    path = tmp_path / "core.msh"
    G.write_msh2(str(path), [x, x], tags.ravel(), seed=5)
    dim, coords, ctags, _ = G.read_structured_grid(str(path))
    p = G.problem_from_grid(coords, ctags, {2: 1000.0}, {3: 1.0})
    direct = mag.Problem(x, x, np.where(tags.ravel() == 2, 1000.0, 1.0), np.where(tags.ravel() == 3, 1.0, 0.0))
    np.testing.assert_array_equal(p.node_mu(), direct.node_mu())
    np.testing.assert_array_equal(p.rhs(), direct.rhs())
    sol, it, rel = O.mag2d_cg(n, n, p.node_mu(), p.rhs(), tol=1e-10)
    assert rel <= 1e-10 and np.abs(sol).max() > 0


def test_xdmf_export_round_trip(tmp_path):
    import xml.etree.ElementTree as ET
    import similie_b200.xdmf as X
    rng = np.random.default_rng(2)
    x, y, z = np.linspace(0, 1, 5), np.linspace(0, 2, 4), np.linspace(1, 3, 3)
    a = rng.standard_normal(5 * 4 * 3)
    b = rng.standard_normal(5 * 4 * 3 * 3)
    files = X.write_xdmf(str(tmp_path / "out.xmf"), [x, y, z], {"A": a, "B": b})
    assert all(os.path.exists(f) for f in files)
    root = ET.parse(str(tmp_path / "out.xmf")).getroot()
    assert root.find("Domain/Grid/Topology").get("Dimensions") == "3 4 5"
    coords, fields = X.read_xdmf(str(tmp_path / "out.xmf"))
    for c, r in zip(coords, (x, y, z)):
        np.testing.assert_array_equal(c, r)
    np.testing.assert_array_equal(fields["A"], a)
    np.testing.assert_array_equal(fields["B"], b)


def test_tag_rule_precedence_and_counts():
    import similie_b200.gmsh_grid as gg
    tags = np.array([1, 2, 3, 4, 5, 6, 7, 1])
    rules = dict(magnetic_material_tags=(1, 4), positive_conductor_tags=(2, 4), negative_conductor_tags=(3,),
                 positive_conductor_x_tags=(5,), negative_conductor_x_tags=(6, 2), mu0=1.0, core_mu=500.0,
                 current_density_z=2.0, current_density_x=3.0, nonlinear=True)
    mu, j, nl, counts = gg.cell_inputs_from_tags(tags, 3, **rules)
    j = j.reshape(-1, 3)
    # 4 is both material and conductor: the material comes first
    np.testing.assert_array_equal(mu, [500, 1, 1, 500, 1, 1, 1, 500])
    np.testing.assert_array_equal(nl, [1, 0, 0, 1, 0, 0, 0, 1])
    # 2 is a -x conductor and a +z conductor: x groups come first in 3D
    np.testing.assert_array_equal(j[:, 0], [0, -3, 0, 0, 3, -3, 0, 0])
    np.testing.assert_array_equal(j[:, 2], [0, 0, -2, 0, 0, 0, 0, 0])
    assert counts == {"core": 3, "coil": 4, "air": 1}
    # 2D: no x groups, J_z only
    mu2, j2, nl2, c2 = gg.cell_inputs_from_tags(tags, 2, **rules)
    np.testing.assert_array_equal(j2, [0, 2, -2, 0, 0, 0, 0, 0])
    assert c2 == {"core": 3, "coil": 2, "air": 3}


def test_hexahedral_mesh_to_3d_problem(tmp_path):
    import similie_b200.gmsh_grid as gg
    import similie_b200.magnetostatics3d as m3
    rng = np.random.default_rng(5)
    coords = [np.cumsum(rng.uniform(0.5, 1.5, n)) for n in (5, 4, 6)]
    tags = rng.choice([10, 20, 30], size=(5, 3, 4))   # (ncz, ncy, ncx), x fastest
    path = str(tmp_path / "box.msh")
    gg.write_msh2(path, coords, tags.ravel(), seed=3)
    dim, got_coords, got_tags, _ = gg.read_structured_grid(path)
    assert dim == 3
    prob, nl, counts = gg.problem3d_from_grid(got_coords, got_tags, magnetic_material_tags=(10,),
                                              positive_conductor_tags=(20,), core_mu=1000.0,
                                              current_density_z=1.5, nonlinear=True)
    flat = tags.ravel()
    np.testing.assert_array_equal(prob.cell_mu, np.where(flat == 10, 1000.0, 1.0))
    np.testing.assert_array_equal(prob.cell_j.reshape(-1, 3)[:, 2], np.where(flat == 20, 1.5, 0.0))
    assert counts["air"] == int((flat == 30).sum())
    ferro = m3.node_ferro(5, 4, 6, nl)
    assert ferro.shape == (5 * 4 * 6,) and ferro.max() <= 1.0
    assert prob.rhs().shape == (3 * 5 * 4 * 6,)
