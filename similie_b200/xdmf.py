"""XDMF export of structured-grid fields (nodal scalars and vectors on a
rectilinear 2D or 3D grid) for visualisation, with the heavy data as raw
little-endian binary files beside the .xmf (no HDF5 library is needed).
The grid is written as XDMF's VXVY / VXVYVZ rectilinear topology, so x is
the fastest axis of every array, as in the solvers' flat layouts."""
import os
import xml.etree.ElementTree as ET

import numpy as np


def write_xdmf(path, coords, fields):
    """coords: node coordinates per axis (2 or 3 arrays); fields: {name:
    array} with nx*ny[*nz] values (scalar) or nx*ny[*nz]*c values (c
    components, component fastest).  Writes path (.xmf) and one
    <path stem>.<name>.bin per array; returns the list of files written."""
    coords = [np.asarray(c, dtype=np.float64) for c in coords]
    dim = len(coords)
    if dim not in (2, 3):
        raise ValueError("2 or 3 axes")
    shape = [len(c) for c in coords]
    nnode = int(np.prod(shape))
    stem = os.path.splitext(path)[0]
    base = os.path.basename(stem)
    written = [path]

    def item(parent, name, arr, dims):
        fn = f"{stem}.{name}.bin"
        np.ascontiguousarray(arr, dtype="<f8").tofile(fn)
        written.append(fn)
        d = ET.SubElement(parent, "DataItem", Dimensions=" ".join(map(str, dims)), NumberType="Float",
                          Precision="8", Format="Binary", Endian="Little")
        d.text = os.path.basename(fn)

    root = ET.Element("Xdmf", Version="3.0")
    grid = ET.SubElement(ET.SubElement(root, "Domain"), "Grid", Name=base, GridType="Uniform")
    # XDMF lists topology dimensions slowest axis first
    ET.SubElement(grid, "Topology", TopologyType="3DRectMesh" if dim == 3 else "2DRectMesh",
                  Dimensions=" ".join(map(str, shape[::-1])))
    geo = ET.SubElement(grid, "Geometry", GeometryType="VXVYVZ" if dim == 3 else "VXVY")
    for a, name in zip(range(dim), "xyz"):
        item(geo, f"coord_{name}", coords[a], [shape[a]])
    for name, arr in fields.items():
        a = np.asarray(arr, dtype=np.float64).ravel()
        if a.size % nnode:
            raise ValueError(f"field {name}: size {a.size} is not a multiple of {nnode} nodes")
        c = a.size // nnode
        at = ET.SubElement(grid, "Attribute", Name=name, AttributeType="Scalar" if c == 1 else "Vector",
                           Center="Node")
        item(at, name, a, shape[::-1] + ([c] if c > 1 else []))
    ET.ElementTree(root).write(path, xml_declaration=True, encoding="utf-8")
    return written


def read_xdmf(path):
    """(coords, {name: flat array}) back from a file of write_xdmf."""
    root = ET.parse(path).getroot()
    grid = root.find("Domain/Grid")
    d = os.path.dirname(path)
    load = lambda it: np.fromfile(os.path.join(d, it.text), dtype="<f8")
    coords = [load(it) for it in grid.find("Geometry").findall("DataItem")]
    fields = {at.get("Name"): load(at.find("DataItem")) for at in grid.findall("Attribute")}
    return coords, fields
