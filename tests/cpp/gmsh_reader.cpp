// Reads a msh2 mesh with include/sil/gmsh_structured_grid.hpp and prints the
// grid (dim, node counts, coordinates, cell tags) or the error message.
#include <cstdio>
#include <stdexcept>

#include "sil/gmsh_structured_grid.hpp"

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    try {
        auto const g = sil::compat::gmsh::read_structured_grid(argv[1]);
        std::printf("dim %d\n", g.dim);
        for (int a = 0; a < g.dim; ++a) {
            std::printf("axis %d", a);
            for (double x : g.coords[a]) std::printf(" %.17g", x);
            std::printf("\n");
        }
        std::printf("tags");
        for (int t : g.cell_tags) std::printf(" %d", t);
        std::printf("\n");
    } catch (std::runtime_error const& e) {
        std::printf("error %s\n", e.what());
    }
    return 0;
}
