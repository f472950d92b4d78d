// mag_ops.cuh -- the 2D magnetostatics residual operator at one row, shared
// by the solver and the learned preconditioner.
//
// Operator (onelab_interface/magnetostatics_onelab.hpp:1271-1426 with the
// moment stencils of magnetostatics_quantities.hpp:100-123 built at
// 1095-1258): for an interior node (i,j), over the interior sampled nodes s
// whose moment stencil touches the row, y = sum_s c(s->row) * moment(s) / mu(s);
// flat layout row = i + nx*j, identity rows on the Dirichlet boundary.
#pragma once

#include <cstdint>

namespace sil {

// `a(idx)` loads the operand at flat index idx (a pointer read, or a value
// formed on the fly, e.g. a search direction z + beta p); (i, j) are the
// row's node coordinates, row = i + nx * j.
template <class T, class A>
__device__ __forceinline__ T mag_apply_node_ij(A const& a, T const* nu, int nx, int ny, int row, int i, int j)
{
    if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) return a(row);
    T const a0 = a(row);
    T residual = T(0);
    if (j >= 2) {
        int const s = row - nx;
        T m0 = T(0);
        m0 = m0 - a(s);
        m0 = m0 + a0;
        residual = residual + m0 * nu[s];  // c = +1
    }
    {
        T m0 = T(0);
        m0 = m0 - a0;
        m0 = m0 + a(row + nx);
        residual = residual - m0 * nu[row];  // c = -1
    }
    if (i >= 2) {
        int const s = row - 1;
        T m1 = T(0);
        m1 = m1 + a(s);
        m1 = m1 - a0;
        residual = residual - m1 * nu[s];  // c = -1
    }
    {
        T m1 = T(0);
        m1 = m1 + a0;
        m1 = m1 - a(row + 1);
        residual = residual + m1 * nu[row];  // c = +1
    }
    return residual;
}

template <class T, class A>
__device__ __forceinline__ T mag_apply_node_ld(A const& a, T const* nu, int64_t nx64, int64_t ny64, int64_t row64)
{
    // problems hold fewer than 2^31 nodes (checked by the entry points): 32-bit index arithmetic
    int const nx = static_cast<int>(nx64), ny = static_cast<int>(ny64), row = static_cast<int>(row64);
    int const j = row / nx, i = row - j * nx;
    return mag_apply_node_ij<T>(a, nu, nx, ny, row, i, j);
}

template <class T>
__device__ __forceinline__ T mag_apply_node(T const* a, T const* nu, int64_t nx64, int64_t ny64, int64_t row64)
{
    return mag_apply_node_ld<T>([a](int idx) { return a[idx]; }, nu, nx64, ny64, row64);
}

} // namespace sil
