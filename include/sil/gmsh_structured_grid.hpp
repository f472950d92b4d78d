// gmsh_structured_grid.hpp -- structured-grid ingestion from Gmsh msh2 ASCII
// meshes: the node coordinates of the rectilinear grid a quadrilateral (2D)
// or hexahedral (3D) mesh forms, and the physical tag of every cell in the
// grid's flat order (cell = i + ncx * (j + ncy * k), x fastest), ready to be
// turned into per-cell permeability / current inputs of the magnetostatics
// solves.  Restates onelab_interface/gmsh_structured_grid.hpp:239-553
// (parse_supported_msh2_mesh, build_structured_grid): same accepted element
// types, same checks and the same error messages' meaning.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace sil {
namespace compat {
namespace gmsh {

struct StructuredGrid
{
    int dim = 0;                      // 2 (quadrilaterals) or 3 (hexahedra)
    std::vector<double> coords[3];    // node coordinates per axis, increasing
    double plane_z = 0.0;             // 2D: the z of the mesh plane
    std::vector<int> cell_tags;       // physical tag per cell, flat x-fastest order
    std::int64_t nodes(int a) const { return static_cast<std::int64_t>(coords[a].size()); }
    std::int64_t cells(int a) const { return nodes(a) - 1; }
};

namespace detail {

constexpr double kCoordTol = 1.0e-12;

// Nodes of a Gmsh element type; -1 for types outside the supported set
// (points, lines, triangles, quadrilaterals, tetrahedra, hexahedra, prisms,
// pyramids of order 1).
inline int nodes_of(int type)
{
    switch (type) {
    case 15: return 1;  // point
    case 1: return 2;   // line
    case 2: return 3;   // triangle
    case 3: return 4;   // quadrilateral
    case 4: return 4;   // tetrahedron
    case 5: return 8;   // hexahedron
    case 6: return 6;   // prism
    case 7: return 5;   // pyramid
    default: return -1;
    }
}

// Elements of lower dimension (boundary groups) are read and ignored.
inline bool is_boundary_element(int type) { return type == 15 || type == 1; }

inline std::vector<double> unique_sorted(std::vector<double> v)
{
    std::sort(v.begin(), v.end());
    std::vector<double> out;
    for (double x : v)
        if (out.empty() || std::abs(x - out.back()) >= kCoordTol) out.push_back(x);
    return out;
}

inline std::size_t nearest(std::vector<double> const& c, double x)
{
    auto const it = std::lower_bound(c.begin(), c.end(), x);
    std::size_t i = static_cast<std::size_t>(it - c.begin());
    if (i == c.size()) return c.size() - 1;
    if (i > 0 && std::abs(c[i - 1] - x) <= std::abs(c[i] - x)) return i - 1;
    return i;
}

struct Node
{
    std::size_t tag;
    double x[3];
};

struct Cell
{
    int tag;
    std::vector<std::size_t> nodes;
};

}  // namespace detail

// Read a msh2 ASCII mesh made wholly of quadrilaterals or of hexahedra whose
// nodes form a full rectilinear grid.  Throws std::runtime_error otherwise.
inline StructuredGrid read_structured_grid(std::string const& path)
{
    std::ifstream in(path);
    if (!in.is_open()) throw std::runtime_error("failed to open mesh file: " + path);
    std::vector<detail::Node> nodes;
    std::vector<detail::Cell> cells;
    int dim = 0;
    bool saw_elements = false;
    std::string token;
    while (in >> token) {
        if (token == "$MeshFormat") {
            double version = 0.0;
            int file_type = 0, data_size = 0;
            in >> version >> file_type >> data_size;
            if (version < 2.0 || version >= 3.0 || file_type != 0)
                throw std::runtime_error("only Gmsh msh2 ASCII meshes are supported");
        } else if (token == "$Nodes") {
            std::size_t count = 0;
            in >> count;
            nodes.resize(count);
            for (auto& n : nodes) in >> n.tag >> n.x[0] >> n.x[1] >> n.x[2];
        } else if (token == "$Elements") {
            saw_elements = true;
            std::size_t count = 0;
            in >> count;
            for (std::size_t e = 0; e < count; ++e) {
                std::size_t etag = 0, ntags = 0;
                int type = 0;
                in >> etag >> type >> ntags;
                std::vector<int> tags(ntags);
                for (auto& t : tags) in >> t;
                int const nn = detail::nodes_of(type);
                if (nn < 0) throw std::runtime_error("unsupported Gmsh element type " + std::to_string(type) + " found in mesh");
                std::vector<std::size_t> en(static_cast<std::size_t>(nn));
                for (auto& v : en) in >> v;
                if (type == 3 || type == 5) {
                    int const d = type == 3 ? 2 : 3;
                    if (dim != 0 && dim != d)
                        throw std::runtime_error("unsupported mesh topology: the whole mesh must be quadrilaterals or hexahedra");
                    dim = d;
                    cells.push_back({tags.empty() ? 0 : tags[0], std::move(en)});
                } else if (!detail::is_boundary_element(type)) {
                    throw std::runtime_error("unsupported mesh topology: the whole mesh must be quadrilaterals or hexahedra");
                }
            }
        }
    }
    if (nodes.empty()) throw std::runtime_error("the provided mesh does not contain any node");
    if (!saw_elements || cells.empty())
        throw std::runtime_error("unsupported mesh topology: the whole mesh must be quadrilaterals or hexahedra");

    StructuredGrid g;
    g.dim = dim;
    for (int a = 0; a < 3; ++a) {
        std::vector<double> v;
        v.reserve(nodes.size());
        for (auto const& n : nodes) v.push_back(n.x[a]);
        g.coords[a] = detail::unique_sorted(std::move(v));
    }
    if (dim == 2) {
        if (g.coords[2].size() != 1) throw std::runtime_error("the quadrilateral mesh nodes do not lie on a single plane");
        g.plane_z = g.coords[2][0];
        g.coords[2].clear();
    }
    // node tag -> grid index; every grid node must be present exactly once
    std::int64_t const nx = g.nodes(0), ny = g.nodes(1), nz = dim == 3 ? g.nodes(2) : 1;
    std::vector<char> seen(static_cast<std::size_t>(nx * ny * nz), 0);
    std::vector<double> first(static_cast<std::size_t>(3 * nx * ny * nz), 0.0);
    std::map<std::size_t, std::array<std::int64_t, 3>> index_of;
    for (auto const& n : nodes) {
        std::array<std::int64_t, 3> ix {static_cast<std::int64_t>(detail::nearest(g.coords[0], n.x[0])),
                                        static_cast<std::int64_t>(detail::nearest(g.coords[1], n.x[1])),
                                        dim == 3 ? static_cast<std::int64_t>(detail::nearest(g.coords[2], n.x[2])) : 0};
        std::size_t const lin = static_cast<std::size_t>(ix[0] + nx * (ix[1] + ny * ix[2]));
        if (seen[lin]) {
            for (int a = 0; a < 3; ++a)
                if (std::abs(first[3 * lin + a] - n.x[a]) >= detail::kCoordTol)
                    throw std::runtime_error("duplicated nodes on the detected rectilinear grid");
        } else {
            seen[lin] = 1;
            for (int a = 0; a < 3; ++a) first[3 * lin + a] = n.x[a];
        }
        index_of[n.tag] = ix;
    }
    for (char s : seen)
        if (!s) throw std::runtime_error("the mesh nodes do not form a full rectilinear grid");
    std::int64_t const ncx = nx - 1, ncy = ny - 1, ncz = dim == 3 ? nz - 1 : 1;
    if (static_cast<std::int64_t>(cells.size()) != ncx * ncy * ncz)
        throw std::runtime_error("the cells do not cover a full rectilinear grid");
    g.cell_tags.assign(static_cast<std::size_t>(ncx * ncy * ncz), 0);
    std::vector<char> taken(g.cell_tags.size(), 0);
    for (auto const& c : cells) {
        std::array<std::int64_t, 3> lo {INT64_MAX, INT64_MAX, INT64_MAX}, hi {0, 0, 0};
        for (std::size_t t : c.nodes) {
            auto const it = index_of.find(t);
            if (it == index_of.end()) throw std::runtime_error("a cell references an unknown node");
            for (int a = 0; a < 3; ++a) {
                lo[a] = std::min(lo[a], it->second[a]);
                hi[a] = std::max(hi[a], it->second[a]);
            }
        }
        for (int a = 0; a < dim; ++a)
            if (hi[a] != lo[a] + 1) throw std::runtime_error("a cell does not match a single rectilinear grid cell");
        std::size_t const lin = static_cast<std::size_t>(lo[0] + ncx * (lo[1] + ncy * (dim == 3 ? lo[2] : 0)));
        if (taken[lin]) throw std::runtime_error("duplicated cell on the detected rectilinear grid");
        taken[lin] = 1;
        g.cell_tags[lin] = c.tag;
    }
    return g;
}

}  // namespace gmsh
}  // namespace compat
}  // namespace sil
