"""Structured-grid ingestion from Gmsh msh2 ASCII meshes (the Python side of
include/sil/gmsh_structured_grid.hpp): the rectilinear grid a quadrilateral
or hexahedral mesh forms and each cell's physical tag, turned into the cell
inputs (permeability, current density) of the magnetostatics solves.
Restates onelab_interface/gmsh_structured_grid.hpp:239-553."""
import numpy as np

from . import magnetostatics as mag

COORD_TOL = 1e-12
_NODES = {15: 1, 1: 2, 2: 3, 3: 4, 4: 4, 5: 8, 6: 6, 7: 5}


def _unique(values):
    v = np.sort(np.asarray(values, dtype=np.float64))
    keep = [0] + [i for i in range(1, len(v)) if v[i] - v[i - 1] >= COORD_TOL]
    return v[keep]


def _nearest(c, x):
    i = int(np.searchsorted(c, x))
    if i == len(c):
        return len(c) - 1
    if i > 0 and abs(c[i - 1] - x) <= abs(c[i] - x):
        return i - 1
    return i


def read_structured_grid(path):
    """(dim, [coords per axis], cell_tags flat x-fastest, plane z or None)."""
    toks = open(path).read().split()
    pos, nodes, cells, dim, saw = 0, [], [], 0, False
    while pos < len(toks):
        t = toks[pos]
        pos += 1
        if t == "$MeshFormat":
            version, ftype = float(toks[pos]), int(toks[pos + 1])
            pos += 3
            if version < 2.0 or version >= 3.0 or ftype != 0:
                raise ValueError("only Gmsh msh2 ASCII meshes are supported")
        elif t == "$Nodes":
            n = int(toks[pos])
            pos += 1
            for _ in range(n):
                nodes.append((int(toks[pos]), float(toks[pos + 1]), float(toks[pos + 2]), float(toks[pos + 3])))
                pos += 4
        elif t == "$Elements":
            saw = True
            n = int(toks[pos])
            pos += 1
            for _ in range(n):
                etype, ntags = int(toks[pos + 1]), int(toks[pos + 2])
                tags = [int(v) for v in toks[pos + 3:pos + 3 + ntags]]
                pos += 3 + ntags
                nn = _NODES.get(etype)
                if nn is None:
                    raise ValueError(f"unsupported Gmsh element type {etype} found in mesh")
                en = [int(v) for v in toks[pos:pos + nn]]
                pos += nn
                if etype in (3, 5):
                    d = 2 if etype == 3 else 3
                    if dim not in (0, d):
                        raise ValueError("unsupported mesh topology: the whole mesh must be quadrilaterals or hexahedra")
                    dim = d
                    cells.append((tags[0] if tags else 0, en))
                elif etype not in (15, 1):
                    raise ValueError("unsupported mesh topology: the whole mesh must be quadrilaterals or hexahedra")
    if not nodes:
        raise ValueError("the provided mesh does not contain any node")
    if not saw or not cells:
        raise ValueError("unsupported mesh topology: the whole mesh must be quadrilaterals or hexahedra")
    coords = [_unique([n[1 + a] for n in nodes]) for a in range(3)]
    plane = None
    if dim == 2:
        if len(coords[2]) != 1:
            raise ValueError("the quadrilateral mesh nodes do not lie on a single plane")
        plane = float(coords[2][0])
        coords = coords[:2]
    shape = [len(c) for c in coords]
    seen = {}
    index_of = {}
    for tag, *x in nodes:
        ix = tuple(_nearest(coords[a], x[a]) for a in range(dim))
        if ix in seen and any(abs(seen[ix][a] - x[a]) >= COORD_TOL for a in range(3)):
            raise ValueError("duplicated nodes on the detected rectilinear grid")
        seen.setdefault(ix, x)
        index_of[tag] = ix
    if len(seen) != int(np.prod(shape)):
        raise ValueError("the mesh nodes do not form a full rectilinear grid")
    ncell = [s - 1 for s in shape]
    if len(cells) != int(np.prod(ncell)):
        raise ValueError("the cells do not cover a full rectilinear grid")
    tags = np.zeros(int(np.prod(ncell)), dtype=np.int64)
    taken = np.zeros(len(tags), dtype=bool)
    for ptag, en in cells:
        if any(t not in index_of for t in en):
            raise ValueError("a cell references an unknown node")
        ix = np.array([index_of[t] for t in en])
        lo, hi = ix.min(axis=0), ix.max(axis=0)
        if np.any(hi != lo + 1):
            raise ValueError("a cell does not match a single rectilinear grid cell")
        lin = int(lo[0] + ncell[0] * (lo[1] + (ncell[1] * lo[2] if dim == 3 else 0)))
        if taken[lin]:
            raise ValueError("duplicated cell on the detected rectilinear grid")
        taken[lin] = True
        tags[lin] = ptag
    return dim, coords, tags, plane


def write_msh2(path, coords, cell_tags, seed=None):
    """Write a rectilinear grid as a msh2 ASCII mesh of quadrilaterals (2
    axes) or hexahedra (3 axes) with one physical tag per cell; `seed`
    shuffles the node tags and the element order."""
    rng = np.random.default_rng(seed)
    dim = len(coords)
    shape = [len(c) for c in coords]
    nnode = int(np.prod(shape))
    perm = rng.permutation(nnode) + 1 if seed is not None else np.arange(1, nnode + 1)

    def nid(*ix):
        lin = ix[0] + shape[0] * (ix[1] + (shape[1] * ix[2] if dim == 3 else 0))
        return int(perm[lin])

    lines = ["$MeshFormat", "2.2 0 8", "$EndMeshFormat", "$Nodes", str(nnode)]
    node_lines = []
    for lin in range(nnode):
        i = lin % shape[0]
        j = (lin // shape[0]) % shape[1]
        k = lin // (shape[0] * shape[1]) if dim == 3 else 0
        z = coords[2][k] if dim == 3 else 0.0
        node_lines.append(f"{int(perm[lin])} {float(coords[0][i])!r} {float(coords[1][j])!r} {float(z)!r}")
    if seed is not None:
        node_lines = [node_lines[q] for q in rng.permutation(nnode)]
    lines += node_lines + ["$EndNodes"]
    ncell = [s - 1 for s in shape]
    elems = []
    tags = np.asarray(cell_tags).ravel()
    for lin in range(int(np.prod(ncell))):
        i = lin % ncell[0]
        j = (lin // ncell[0]) % ncell[1]
        if dim == 2:
            conn = [nid(i, j), nid(i + 1, j), nid(i + 1, j + 1), nid(i, j + 1)]
            elems.append((3, int(tags[lin]), conn))
        else:
            k = lin // (ncell[0] * ncell[1])
            conn = [nid(i, j, k), nid(i + 1, j, k), nid(i + 1, j + 1, k), nid(i, j + 1, k),
                    nid(i, j, k + 1), nid(i + 1, j, k + 1), nid(i + 1, j + 1, k + 1), nid(i, j + 1, k + 1)]
            elems.append((5, int(tags[lin]), conn))
    # a boundary line element, read and ignored
    elems.append((1, 99, [nid(0, 0, *([0] if dim == 3 else [])), nid(1, 0, *([0] if dim == 3 else []))]))
    if seed is not None:
        elems = [elems[q] for q in rng.permutation(len(elems))]
    lines += ["$Elements", str(len(elems))]
    for e, (etype, tag, conn) in enumerate(elems, start=1):
        lines.append(f"{e} {etype} 2 {tag} {tag} " + " ".join(map(str, conn)))
    lines += ["$EndElements"]
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")


def problem_from_grid(coords, cell_tags, mu_by_tag, j_by_tag, mu_default=1.0):
    """A 2D magnetostatics Problem from a structured grid: per-cell relative
    permeability and current density looked up by physical tag."""
    x, y = (np.asarray(c, dtype=np.float64) for c in coords)
    tags = np.asarray(cell_tags).ravel()
    cell_mu = np.array([mu_by_tag.get(int(t), mu_default) for t in tags], dtype=np.float64)
    cell_j = np.array([j_by_tag.get(int(t), 0.0) for t in tags], dtype=np.float64)
    return mag.Problem(x, y, cell_mu, cell_j, {"source": "gmsh"})


def cell_inputs_from_tags(cell_tags, dim, magnetic_material_tags=(), positive_conductor_tags=(),
                          negative_conductor_tags=(), positive_conductor_x_tags=(), negative_conductor_x_tags=(),
                          mu0=1.0, core_mu=1000.0, current_density_z=0.0, current_density_x=0.0, nonlinear=False):
    """The reference's tag-to-cell-input rule (onelab_interface/
    magnetostatics_onelab.hpp:4376-4397 in 2D, 4870-4897 in 3D): the first
    group a cell's physical tag belongs to decides, in the order magnetic
    material (permeability core_mu, and the nonlinear flag when the run uses
    the nonlinear material), conductors along +x / -x (3D only), conductors
    along +z / -z; any other cell is air (permeability mu0, no current).

    Returns (cell_mu, cell_j, cell_nonlinear, counts): cell_j has one
    component in 2D (J_z) and three in 3D, counts the core, coil and air
    cells."""
    tags = np.asarray(cell_tags).ravel().astype(np.int64)
    n = tags.size
    cell_mu = np.full(n, float(mu0))
    cell_j = np.zeros((n, 3))
    cell_nl = np.zeros(n, dtype=bool)
    counts = {"core": 0, "coil": 0, "air": 0}
    groups = [("core", magnetic_material_tags, None, 0.0)]
    if dim == 3:
        groups += [("coil", positive_conductor_x_tags, 0, current_density_x),
                   ("coil", negative_conductor_x_tags, 0, -current_density_x)]
    groups += [("coil", positive_conductor_tags, 2, current_density_z),
               ("coil", negative_conductor_tags, 2, -current_density_z)]
    decided = np.zeros(n, dtype=bool)
    for kind, group, comp, value in groups:
        hit = np.isin(tags, np.asarray(list(group), dtype=np.int64)) & ~decided
        if kind == "core":
            cell_mu[hit] = core_mu
            cell_nl[hit] = bool(nonlinear)
        else:
            cell_j[hit, comp] = value
        counts[kind] += int(hit.sum())
        decided |= hit
    counts["air"] = int((~decided).sum())
    return cell_mu, (cell_j[:, 2].copy() if dim == 2 else cell_j.ravel()), cell_nl, counts


def problem3d_from_grid(coords, cell_tags, gamma=None, **rules):
    """A 3D magnetostatics Problem from a structured hexahedral grid by the
    reference's tag rule (cell_inputs_from_tags); returns (problem,
    cell_nonlinear, counts).  With the nonlinear material, the node
    ferromagnetic share is magnetostatics3d.node_ferro(nx, ny, nz,
    cell_nonlinear)."""
    from . import magnetostatics3d as m3
    x, y, z = (np.asarray(c, dtype=np.float64) for c in coords)
    cell_mu, cell_j, cell_nl, counts = cell_inputs_from_tags(cell_tags, 3, **rules)
    g = m3.DEFAULT_GAUGE_PENALTY if gamma is None else gamma
    return m3.Problem(x, y, z, cell_mu, cell_j, g, {"source": "gmsh"}), cell_nl, counts
