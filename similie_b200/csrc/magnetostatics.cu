// magnetostatics.cu -- 2D and 3D linear magnetostatics on the GPU: the matrix-free residual
// operator d^T (nu d A) with identity rows on the Dirichlet boundary, and a
// batched Jacobi-preconditioned conjugate-gradient solve (FP64, or FP32
// inner sweeps inside FP64 iterative refinement).
//
// Operator (onelab_interface/magnetostatics_onelab.hpp:1271-1426 with the
// moment stencils of magnetostatics_quantities.hpp:100-123 built at
// 1095-1258): for an interior node (i,j), over the interior sampled nodes s
// whose moment stencil touches the row,
//   y = sum_s c(s->row) * moment(s) / mu(s)
// with moment0(s) = A(s+ey) - A(s) (c = +1 at s+ey, -1 at s) and
// moment1(s) = A(s) - A(s+ex) (c = -1 at s+ex, +1 at s); X moments first,
// sampled nodes in ascending flat order.  Boundary rows are the identity.
// Sampled nodes on the first row/column are excluded, as in the reference.
//
// Solver (minimize_strong_formulation_residual.hpp:1028-1304): CG from
// x = 0 with the inverse diagonal as preconditioner, stopped when
// ||r|| <= tol ||b||; the final residual is re-evaluated in FP64.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <mutex>
#include <vector>

#include "mag_ops.cuh"
#include "precond_net.cuh"
#include "sil_internal.cuh"

namespace sil {

namespace {

constexpr int kThreads = 256;
constexpr int kNodesPerThread = 16;
constexpr int kItemNodes = kThreads * kNodesPerThread;  // nodes per work item (one CTA)

// ------------------------------------------------------------------ operator

__global__ void mag_apply_kernel(double const* nu, double const* a, double* y, int64_t nx, int64_t ny)
{
    int64_t const row = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (row >= nx * ny) return;
    y[row] = mag_apply_node(a, nu, nx, ny, row);
}

__global__ void reciprocal_kernel(double const* mu, double* nu, int64_t n)
{
    int64_t const i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (i < n) nu[i] = 1.0 / mu[i];
}

// ------------------------------------------------------------------ batched CG

// Directions the flexible CG keeps at most.
constexpr int kMaxDirs = 16;

struct Item
{
    int prob;
    int index;  // item index within its problem
    int64_t begin;
    int64_t end;
};

template <class T>
struct Vecs
{
    T* x;
    T* r;
    T* z;
    T* p;
    T* q;
    T* dinv;
    T* nu;
    T* ph;  // flexible CG: m stored directions p_j at ph + j * hstride
    T* qh;  // and their images q_j = A p_j
    T* p2;  // persistent CG: the direction's second buffer (p and p2 alternate)
};

struct ProbInfo
{
    int dim;                  // 2: scalar A_z on an nx x ny grid; 3: vector A on nx x ny x nz
    int64_t nx, ny, nz;
    int64_t nodes;            // grid nodes
    int64_t n;                // unknowns: nodes (2D) or 3 * nodes (3D)
    double gamma;             // 3D gauge penalty
    int nitems;
    int first_item;
    double const* ls64[3];    // 3D: reference local spacing per axis and its inverse
    double const* ils64[3];
    float const* ls32[3];
    float const* ils32[3];
    int gauge;                // 3D: 0 penalty, 1 divergence gauge
    double const* gd64;       // divergence gauge, 8 per node: E0[3], E1[3], w, 0
    float const* gd32;
    int max_iters;            // iteration budget: the problem stops once it has done this many
};

template <class T>
__device__ __forceinline__ T const* spacing(ProbInfo const& pi, int axis)
{
    if constexpr (sizeof(T) == 8) return pi.ls64[axis];
    else return pi.ls32[axis];
}

template <class T>
__device__ __forceinline__ T const* inv_spacing(ProbInfo const& pi, int axis)
{
    if constexpr (sizeof(T) == 8) return pi.ils64[axis];
    else return pi.ils32[axis];
}

// 3D curl-curl + gauge penalty at DOF row = 3*node + c (onelab_interface/
// magnetostatics_onelab.hpp:2242-2396).  The moments are the curl
// components at the interior sampled nodes s whose stencil holds the DOF,
//   B_x(s) = A_y(s) - A_z(s) - A_y(s+z) + A_z(s+y)
//   B_y(s) = -A_x(s) + A_z(s) + A_x(s+z) - A_z(s+x)
//   B_z(s) = A_x(s) - A_y(s) - A_x(s+y) + A_y(s+x)
// (boundary DOFs dropped from the stencils), weighted by the Hodge factor of
// B (d_m / (d_a d_b), central local spacings) and 1/mu(s); the gauge term is
// gamma * (d_a d_b / d_c) * A.  Boundary rows are the identity.
template <class T>
__device__ __forceinline__ T const* gauge_table(ProbInfo const& pi)
{
    if constexpr (sizeof(T) == 8) return pi.gd64;
    else return pi.gd32;
}

// Divergence gauge.  The codifferential of the 1-form A at node m is
// (D A)(m) = sum_a E0(m, a) A_a(m) + E1(m, a) A_a(m - e_a), with the
// coefficients of boundary columns zero (they are dropped from the
// reference's stencils, magnetostatics_onelab.hpp:1894-1945).  The gauge
// term of row (n, c) is sum over the codifferential rows holding the column,
// m = n and m = n + e_c, of w(m) D(m, (n, c)) (D A)(m).
template <class T, class A>
__device__ __forceinline__ T gauge_div_ld(A const& a, T const* gd, int m, int i, int j, int k, int nx, int ny)
{
    T const* e = gd + 8 * m;
    T s = T(0);
    s = s + e[0] * a(3 * m);
    if (i > 0) s = s + e[3] * a(3 * (m - 1));
    s = s + e[1] * a(3 * m + 1);
    if (j > 0) s = s + e[4] * a(3 * (m - nx) + 1);
    s = s + e[2] * a(3 * m + 2);
    if (k > 0) s = s + e[5] * a(3 * (m - nx * ny) + 2);
    return s;
}

template <class T>
__device__ __forceinline__ T gauge_div(T const* a, T const* gd, int m, int i, int j, int k, int nx, int ny)
{
    return gauge_div_ld<T>([a](int idx) { return a[idx]; }, gd, m, i, j, k, nx, ny);
}

// Gauge term of component c at interior node n = (i, j, k), given (D A)(n).
template <class T, class A>
__device__ __forceinline__ T gauge_term_ld(A const& a, T const* gd, int n, int i, int j, int k, int nx, int ny, int c,
                                           T div_n)
{
    int const step = c == 0 ? 1 : (c == 1 ? nx : nx * ny);
    int const m = n + step;
    T const div_m = gauge_div_ld<T>(a, gd, m, i + (c == 0), j + (c == 1), k + (c == 2), nx, ny);
    T t = T(0);
    t = t + gd[8 * n + 6] * gd[8 * n + c] * div_n;
    t = t + gd[8 * m + 6] * gd[8 * m + 3 + c] * div_m;
    return t;
}

template <class T>
__device__ __forceinline__ T gauge_term(T const* a, T const* gd, int n, int i, int j, int k, int nx, int ny, int c,
                                        T div_n)
{
    int const step = c == 0 ? 1 : (c == 1 ? nx : nx * ny);
    int const m = n + step;
    T const div_m = gauge_div(a, gd, m, i + (c == 0), j + (c == 1), k + (c == 2), nx, ny);
    T t = T(0);
    t = t + gd[8 * n + 6] * gd[8 * n + c] * div_n;
    t = t + gd[8 * m + 6] * gd[8 * m + 3 + c] * div_m;
    return t;
}

// G: the divergence-gauge code is compiled in (kernels of batches that hold
// a divergence-gauge problem); without it the kernels keep the register
// budget of the penalty operator.
template <class T, bool G = false>
__device__ T mag3d_apply_row(T const* a, T const* nu, ProbInfo const& pi, int64_t row64)
{
    // fewer than 2^31 unknowns per problem (checked by the entry points)
    int const row = static_cast<int>(row64);
    int const node = row / 3;
    int const c = row - 3 * node;
    int const nx = static_cast<int>(pi.nx), ny = static_cast<int>(pi.ny), nz = static_cast<int>(pi.nz);
    int const t = node / nx, i = node - t * nx, k = t / ny, j = t - k * ny;
    auto interior = [&](int ii, int jj, int kk) {
        return ii > 0 && jj > 0 && kk > 0 && ii + 1 < nx && jj + 1 < ny && kk + 1 < nz;
    };
    if (!interior(i, j, k)) return a[row];
    int const sy = 3 * nx, sz = 3 * nx * ny;
    // A at node (i, j, k) + offset, component cc; zero on the Dirichlet boundary
    auto A = [&](int di, int dj, int dk, int cc) -> T {
        return interior(i + di, j + dj, k + dk) ? a[row - c + 3 * di + sy * dj + sz * dk + cc] : T(0);
    };
    // curl moments at the sampled node (i, j, k) + (oi, oj, ok)
    auto bx = [&](int oi, int oj, int ok) {
        T m = T(0);
        m = m + A(oi, oj, ok, 1);
        m = m - A(oi, oj, ok, 2);
        m = m - A(oi, oj, ok + 1, 1);
        m = m + A(oi, oj + 1, ok, 2);
        return m;
    };
    auto by = [&](int oi, int oj, int ok) {
        T m = T(0);
        m = m - A(oi, oj, ok, 0);
        m = m + A(oi, oj, ok, 2);
        m = m + A(oi, oj, ok + 1, 0);
        m = m - A(oi + 1, oj, ok, 2);
        return m;
    };
    auto bz = [&](int oi, int oj, int ok) {
        T m = T(0);
        m = m + A(oi, oj, ok, 0);
        m = m - A(oi, oj, ok, 1);
        m = m - A(oi, oj + 1, ok, 0);
        m = m + A(oi + 1, oj, ok, 1);
        return m;
    };
    T const* lx = spacing<T>(pi, 0);
    T const* ly = spacing<T>(pi, 1);
    T const* lz = spacing<T>(pi, 2);
    T const* ilx = inv_spacing<T>(pi, 0);
    T const* ily = inv_spacing<T>(pi, 1);
    T const* ilz = inv_spacing<T>(pi, 2);
    int const nd = node;
    auto w = [&](int oi, int oj, int ok, int m) -> T {
        T const nuv = nu[nd + oi + nx * oj + nx * ny * ok];
        if (m == 0) return lx[i + oi] * ily[j + oj] * ilz[k + ok] * nuv;
        if (m == 1) return ly[j + oj] * ilx[i + oi] * ilz[k + ok] * nuv;
        return lz[k + ok] * ilx[i + oi] * ily[j + oj] * nuv;
    };
    T res = T(0);
    T ha;
    if (c == 0) {
        res = res - w(0, 0, 0, 1) * by(0, 0, 0);
        if (interior(i, j, k - 1)) res = res + w(0, 0, -1, 1) * by(0, 0, -1);
        res = res + w(0, 0, 0, 2) * bz(0, 0, 0);
        if (interior(i, j - 1, k)) res = res - w(0, -1, 0, 2) * bz(0, -1, 0);
        ha = ly[j] * lz[k] * ilx[i];
    } else if (c == 1) {
        res = res + w(0, 0, 0, 0) * bx(0, 0, 0);
        if (interior(i, j, k - 1)) res = res - w(0, 0, -1, 0) * bx(0, 0, -1);
        res = res - w(0, 0, 0, 2) * bz(0, 0, 0);
        if (interior(i - 1, j, k)) res = res + w(-1, 0, 0, 2) * bz(-1, 0, 0);
        ha = lx[i] * lz[k] * ily[j];
    } else {
        res = res - w(0, 0, 0, 0) * bx(0, 0, 0);
        if (interior(i, j - 1, k)) res = res + w(0, -1, 0, 0) * bx(0, -1, 0);
        res = res + w(0, 0, 0, 1) * by(0, 0, 0);
        if (interior(i - 1, j, k)) res = res - w(-1, 0, 0, 1) * by(-1, 0, 0);
        ha = lx[i] * ly[j] * ilz[k];
    }
    if constexpr (G) {
        if (pi.gauge) {
            T const* gd = gauge_table<T>(pi);
            T const dn = gauge_div(a, gd, node, i, j, k, nx, ny);
            return res + static_cast<T>(pi.gamma) * gauge_term(a, gd, node, i, j, k, nx, ny, c, dn);
        }
    }
    return res + static_cast<T>(pi.gamma) * ha * a[row];
}

// The curl-curl part of the three rows of an interior node (i, j, k), from
// accessors: A(di, dj, dk, c) the 1-form at node (i, j, k) + (di, dj, dk),
// component c, zero at boundary nodes; NU(oi, oj, ok) the reluctivity at
// the sampled node (i, j, k) + (oi, oj, ok).  The curl moments shared
// between the components are formed once; each component sums its terms in
// the order of mag3d_apply_row, so the values are the same whatever the
// accessors read from.
template <class T, class AF, class NF>
__device__ __forceinline__ void mag3d_curl_rows(AF const& A, NF const& NU, ProbInfo const& pi, int i, int j, int k,
                                                T* res)
{
    int const nx = static_cast<int>(pi.nx), ny = static_cast<int>(pi.ny), nz = static_cast<int>(pi.nz);
    auto interior = [&](int ii, int jj, int kk) {
        return ii > 0 && jj > 0 && kk > 0 && ii + 1 < nx && jj + 1 < ny && kk + 1 < nz;
    };
    auto bx = [&](int oi, int oj, int ok) {
        T m = T(0);
        m = m + A(oi, oj, ok, 1);
        m = m - A(oi, oj, ok, 2);
        m = m - A(oi, oj, ok + 1, 1);
        m = m + A(oi, oj + 1, ok, 2);
        return m;
    };
    auto by = [&](int oi, int oj, int ok) {
        T m = T(0);
        m = m - A(oi, oj, ok, 0);
        m = m + A(oi, oj, ok, 2);
        m = m + A(oi, oj, ok + 1, 0);
        m = m - A(oi + 1, oj, ok, 2);
        return m;
    };
    auto bz = [&](int oi, int oj, int ok) {
        T m = T(0);
        m = m + A(oi, oj, ok, 0);
        m = m - A(oi, oj, ok, 1);
        m = m - A(oi, oj + 1, ok, 0);
        m = m + A(oi + 1, oj, ok, 1);
        return m;
    };
    T const* lx = spacing<T>(pi, 0);
    T const* ly = spacing<T>(pi, 1);
    T const* lz = spacing<T>(pi, 2);
    T const* ilx = inv_spacing<T>(pi, 0);
    T const* ily = inv_spacing<T>(pi, 1);
    T const* ilz = inv_spacing<T>(pi, 2);
    auto w = [&](int oi, int oj, int ok, int m) -> T {
        T const nuv = NU(oi, oj, ok);
        if (m == 0) return lx[i + oi] * ily[j + oj] * ilz[k + ok] * nuv;
        if (m == 1) return ly[j + oj] * ilx[i + oi] * ilz[k + ok] * nuv;
        return lz[k + ok] * ilx[i + oi] * ily[j + oj] * nuv;
    };
    bool const in_k = interior(i, j, k - 1), in_j = interior(i, j - 1, k), in_i = interior(i - 1, j, k);
    T const Bx = bx(0, 0, 0), By = by(0, 0, 0), Bz = bz(0, 0, 0);
    T const Wx = w(0, 0, 0, 0), Wy = w(0, 0, 0, 1), Wz = w(0, 0, 0, 2);
    {
        T r = T(0);
        r = r - Wy * By;
        if (in_k) r = r + w(0, 0, -1, 1) * by(0, 0, -1);
        r = r + Wz * Bz;
        if (in_j) r = r - w(0, -1, 0, 2) * bz(0, -1, 0);
        res[0] = r;
    }
    {
        T r = T(0);
        r = r + Wx * Bx;
        if (in_k) r = r - w(0, 0, -1, 0) * bx(0, 0, -1);
        r = r - Wz * Bz;
        if (in_i) r = r + w(-1, 0, 0, 2) * bz(-1, 0, 0);
        res[1] = r;
    }
    {
        T r = T(0);
        r = r - Wx * Bx;
        if (in_j) r = r + w(0, -1, 0, 0) * bx(0, -1, 0);
        r = r + Wy * By;
        if (in_i) r = r - w(-1, 0, 0, 1) * by(-1, 0, 0);
        res[2] = r;
    }
}

// Penalty gauge term of component c at node (i, j, k): gamma (d_a d_b / d_c) A_c.
template <class T>
__device__ __forceinline__ T mag3d_penalty(ProbInfo const& pi, int i, int j, int k, int c, T ac)
{
    T const g = static_cast<T>(pi.gamma);
    if (c == 0) return g * (spacing<T>(pi, 1)[j] * spacing<T>(pi, 2)[k] * inv_spacing<T>(pi, 0)[i]) * ac;
    if (c == 1) return g * (spacing<T>(pi, 0)[i] * spacing<T>(pi, 2)[k] * inv_spacing<T>(pi, 1)[j]) * ac;
    return g * (spacing<T>(pi, 0)[i] * spacing<T>(pi, 1)[j] * inv_spacing<T>(pi, 2)[k]) * ac;
}

// All three rows of an interior node at once, reading a through a loader by
// row index.  DEEP: every node of the stencil (offsets -1..1 per axis) is
// interior, so no neighbour needs the boundary test (the same values, fewer
// instructions).
template <class T, bool G, bool DEEP, class LD>
__device__ __forceinline__ void mag3d_interior_node(LD const& a, T const* nu, ProbInfo const& pi, int node, int i,
                                                    int j, int k, T* out)
{
    int const nx = static_cast<int>(pi.nx), ny = static_cast<int>(pi.ny), nz = static_cast<int>(pi.nz);
    int const row0 = 3 * node;
    auto interior = [&](int ii, int jj, int kk) {
        return DEEP || (ii > 0 && jj > 0 && kk > 0 && ii + 1 < nx && jj + 1 < ny && kk + 1 < nz);
    };
    int const sy = 3 * nx, sz = 3 * nx * ny;
    auto A = [&](int di, int dj, int dk, int cc) -> T {
        return interior(i + di, j + dj, k + dk) ? a(row0 + 3 * di + sy * dj + sz * dk + cc) : T(0);
    };
    auto NU = [&](int oi, int oj, int ok) -> T { return nu[node + oi + nx * oj + nx * ny * ok]; };
    T res[3];
    mag3d_curl_rows<T>(A, NU, pi, i, j, k, res);
    T const g = static_cast<T>(pi.gamma);
    // gauge term per component: penalty g (d_a d_b / d_c) A_c, or the divergence gauge
    T gt[3];
    bool gauge_done = false;
    if constexpr (G) {
        if (pi.gauge) {
            T const* gd = gauge_table<T>(pi);
            T const dn = gauge_div_ld<T>(a, gd, node, i, j, k, nx, ny);
            for (int c = 0; c < 3; ++c) gt[c] = g * gauge_term_ld<T>(a, gd, node, i, j, k, nx, ny, c, dn);
            gauge_done = true;
        }
    }
    if (!gauge_done)
        for (int c = 0; c < 3; ++c) gt[c] = mag3d_penalty<T>(pi, i, j, k, c, a(row0 + c));
    for (int c = 0; c < 3; ++c) out[c] = res[c] + gt[c];
}

// All three rows of a node: identity on the Dirichlet boundary, else the
// interior stencil (without boundary tests where the whole stencil is
// interior).
template <class T, bool G, class LD>
__device__ void mag3d_apply_node_ld(LD const& a, T const* nu, ProbInfo const& pi, int node, T* out)
{
    int const nx = static_cast<int>(pi.nx), ny = static_cast<int>(pi.ny), nz = static_cast<int>(pi.nz);
    int const t = node / nx, i = node - t * nx, k = t / ny, j = t - k * ny;
    if (!(i > 0 && j > 0 && k > 0 && i + 1 < nx && j + 1 < ny && k + 1 < nz)) {
        int const row0 = 3 * node;
        out[0] = a(row0);
        out[1] = a(row0 + 1);
        out[2] = a(row0 + 2);
        return;
    }
    if (i > 1 && j > 1 && k > 1 && i + 2 < nx && j + 2 < ny && k + 2 < nz)
        mag3d_interior_node<T, G, true>(a, nu, pi, node, i, j, k, out);
    else
        mag3d_interior_node<T, G, false>(a, nu, pi, node, i, j, k, out);
}

template <class T, bool G = false>
__device__ __forceinline__ void mag3d_apply_node(T const* a, T const* nu, ProbInfo const& pi, int node, T* out)
{
    mag3d_apply_node_ld<T, G>([a](int idx) { return a[idx]; }, nu, pi, node, out);
}

template <class T, bool G = false>
__device__ __forceinline__ T mag_apply_row(T const* a, T const* nu, ProbInfo const& pi, int64_t row)
{
    if (pi.dim == 2) return mag_apply_node(a, nu, pi.nx, pi.ny, row);
    return mag3d_apply_row<T, G>(a, nu, pi, row);
}

// Diagonal of the operator at a row (Jacobi preconditioner), from mu directly.
__device__ double mag_diag_row(double const* mu, ProbInfo const& pi, int64_t row)
{
    if (pi.dim == 2) {
        int64_t const i = row % pi.nx, j = row / pi.nx;
        if (i == 0 || j == 0 || i + 1 == pi.nx || j + 1 == pi.ny) return 1.0;
        double d = 0.0;
        if (j >= 2) d += 1.0 / mu[row - pi.nx];
        d += 1.0 / mu[row];
        if (i >= 2) d += 1.0 / mu[row - 1];
        d += 1.0 / mu[row];
        return d;
    }
    int64_t const node = row / 3;
    int const c = static_cast<int>(row - 3 * node);
    int64_t const nx = pi.nx, ny = pi.ny, nz = pi.nz;
    int64_t const i = node % nx, t = node / nx, j = t % ny, k = t / ny;
    auto interior = [&](int64_t ii, int64_t jj, int64_t kk) {
        return ii > 0 && jj > 0 && kk > 0 && ii + 1 < nx && jj + 1 < ny && kk + 1 < nz;
    };
    if (!interior(i, j, k)) return 1.0;
    double const* lx = pi.ls64[0];
    double const* ly = pi.ls64[1];
    double const* lz = pi.ls64[2];
    double const* ilx = pi.ils64[0];
    double const* ily = pi.ils64[1];
    double const* ilz = pi.ils64[2];
    auto w = [&](int64_t ii, int64_t jj, int64_t kk, int m) -> double {
        double const nuv = 1.0 / mu[ii + nx * (jj + ny * kk)];
        if (m == 0) return lx[ii] * ily[jj] * ilz[kk] * nuv;
        if (m == 1) return ly[jj] * ilx[ii] * ilz[kk] * nuv;
        return lz[kk] * ilx[ii] * ily[jj] * nuv;
    };
    double d = 0.0;
    if (pi.gauge) {
        // divergence gauge: sum over the codifferential rows m of w(m) D(m, row)^2
        int64_t const step = c == 0 ? 1 : (c == 1 ? nx : nx * ny);
        double const* gd = pi.gd64;
        double const e0 = gd[8 * node + c], e1 = gd[8 * (node + step) + 3 + c];
        double const gdiv = gd[8 * node + 6] * e0 * e0 + gd[8 * (node + step) + 6] * e1 * e1;
        if (c == 0) {
            d += w(i, j, k, 1) + w(i, j, k, 2);
            if (interior(i, j, k - 1)) d += w(i, j, k - 1, 1);
            if (interior(i, j - 1, k)) d += w(i, j - 1, k, 2);
        } else if (c == 1) {
            d += w(i, j, k, 0) + w(i, j, k, 2);
            if (interior(i, j, k - 1)) d += w(i, j, k - 1, 0);
            if (interior(i - 1, j, k)) d += w(i - 1, j, k, 2);
        } else {
            d += w(i, j, k, 0) + w(i, j, k, 1);
            if (interior(i, j - 1, k)) d += w(i, j - 1, k, 0);
            if (interior(i - 1, j, k)) d += w(i - 1, j, k, 1);
        }
        return d + pi.gamma * gdiv;
    }
    if (c == 0) {
        d += w(i, j, k, 1) + w(i, j, k, 2);
        if (interior(i, j, k - 1)) d += w(i, j, k - 1, 1);
        if (interior(i, j - 1, k)) d += w(i, j - 1, k, 2);
        d += pi.gamma * (ly[j] * lz[k] * ilx[i]);
    } else if (c == 1) {
        d += w(i, j, k, 0) + w(i, j, k, 2);
        if (interior(i, j, k - 1)) d += w(i, j, k - 1, 0);
        if (interior(i - 1, j, k)) d += w(i - 1, j, k, 2);
        d += pi.gamma * (lx[i] * lz[k] * ily[j]);
    } else {
        d += w(i, j, k, 0) + w(i, j, k, 1);
        if (interior(i, j - 1, k)) d += w(i, j - 1, k, 0);
        if (interior(i - 1, j, k)) d += w(i - 1, j, k, 1);
        d += pi.gamma * (lx[i] * ly[j] * ilz[k]);
    }
    return d;
}

struct Scalars
{
    double rz;        // r . z of the current iterate
    double rr;        // r . r
    double rr0;       // r . r at the start of the (inner) solve
    double inner_tol2;  // squared relative reduction the inner solve stops at
    double bb;        // b . b (outer right-hand side)
    double alpha, beta;
    double scale;     // outer residual norm used to scale the inner right-hand side
    int done;         // inner / plain solve finished
    int outer_done;   // refinement finished
    int iters;        // iterations of the current solve
    int total_iters;  // all inner iterations
    int nonfinite;
    int counter_a, counter_b, counter_c;
    // flexible CG with the learned preconditioner
    double win_rr;    // r . r at the start of the stall window
    int win_iters;    // iterations into the stall window
    int fallback;     // 1: the plain solver takes over this problem
    int learned_iters;
    double pq_hist[kMaxDirs];  // p_j . q_j of the stored directions
    double coef[kMaxDirs];     // (z . q_j) / (p_j . q_j) of the current z
    // persistent CG
    int pbuf;                  // buffer (0: p, 1: p2) holding the latest direction
    double scale_prev;         // outer residual norm of the previous refinement pass
};

// Deterministic block sum of one double per thread.
__device__ __forceinline__ double block_sum(double v, double* smem)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int const warp = threadIdx.x / 32, lane = threadIdx.x % 32;
    __syncthreads();
    if (lane == 0) smem[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0) {
        for (int w = 0; w < kThreads / 32; ++w) t += smem[w];
    }
    return t;  // valid in thread 0
}

// Last-CTA-of-the-problem reduction of K sums: every CTA publishes its
// partials (thread 0's vals) and counts in; the last CTA of the problem sums
// all partials with the whole block, in a fixed order (deterministic), and
// returns true in its thread 0 with `out` holding the K totals.
template <int K>
__device__ bool finish_reduction_k(double const* vals, double* const* parts, int item_index, int first_item, int nitems,
                                   int* counter, double* out)
{
    __shared__ int is_last;
    __shared__ double red[kThreads / 32];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k) parts[k][first_item + item_index] = vals[k];
        __threadfence();
        is_last = atomicAdd(counter, 1) == nitems - 1;
    }
    __syncthreads();
    if (!is_last) return false;
    __threadfence();
    for (int k = 0; k < K; ++k) {
        double v = 0.0;
        for (int j = threadIdx.x; j < nitems; j += kThreads) v += __ldcg(parts[k] + first_item + j);
        out[k] = block_sum(v, red);
    }
    if (threadIdx.x == 0) {
        *counter = 0;
        return true;
    }
    return false;
}

__device__ bool finish_reduction(double partial, double* partials, int item_index, int first_item, int nitems,
                                 int* counter, double* out)
{
    double* parts[1] = {partials};
    return finish_reduction_k<1>(&partial, parts, item_index, first_item, nitems, counter, out);
}

template <class T>
__global__ void __launch_bounds__(kThreads) cg_init_kernel(Item const* items, ProbInfo const* info, Vecs<T> const* vecs,
                                                           double const* const* rhs64, double const* const* r64,
                                                           Scalars* sc, double* part_a, double* part_b, bool from_r64)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[blockIdx.x];
    Scalars* s = sc + it.prob;
    if (s->outer_done) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    double const scale = from_r64 ? s->scale : 1.0;
    double rz = 0.0, bb = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        double const b = from_r64 ? r64[it.prob][row] / scale : rhs64[it.prob][row];
        T const r = static_cast<T>(b);
        T const z = v.dinv[row] * r;
        v.x[row] = T(0);
        v.r[row] = r;
        v.z[row] = z;
        v.p[row] = z;
        rz += static_cast<double>(r) * static_cast<double>(z);
        bb += static_cast<double>(r) * static_cast<double>(r);
    }
    double const rz_b = block_sum(rz, red);
    double const bb_b = block_sum(bb, red);
    double const vals[2] = {rz_b, bb_b};
    double* parts[2] = {part_a, part_b};
    double tot[2];
    if (finish_reduction_k<2>(vals, parts, it.index, pi.first_item, pi.nitems, &s->counter_a, tot)) {
        double const trz = tot[0], tot_bb = tot[1];
        s->rz = trz;
        s->rr = tot_bb;
        s->rr0 = tot_bb;
        if (!from_r64) s->bb = tot_bb;
        s->iters = 0;
        s->done = (tot_bb == 0.0 || s->total_iters >= pi.max_iters) ? 1 : 0;
        s->nonfinite = 0;
    }
}

// ------------------------------------------------------------------ CG iteration
//
// One Jacobi-CG iteration is two kernels over the items of the problems that
// still iterate (`act`, one CTA per item, so converged problems launch
// nothing):
//   cg_dir_apply  p = z + beta p_old (formed on the fly at the row and at its
//                 stencil neighbours; p double-buffered), q = A p, partial
//                 p.q; the problem's last CTA forms alpha
//   cg_update     x += alpha p, r -= alpha q, z = D^-1 r, partials r.z and
//                 r.r; the last CTA forms beta, counts the iteration, flips
//                 the direction buffer and decides convergence
// Chunks of iterations are captured as a CUDA graph, captured again when the
// set of iterating problems changes.

template <class T, bool G = false>
__global__ void __launch_bounds__(kThreads) cg_dir_apply_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                                Vecs<T> const* vecs, Scalars* sc, double* part)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act[blockIdx.x]];
    Scalars* s = sc + it.prob;
    if (s->done || s->outer_done) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    int const pb = s->pbuf;
    T const* pold = pb == 0 ? v.p : v.p2;
    T* pnew = pb == 0 ? v.p2 : v.p;
    T const beta = static_cast<T>(s->beta);
    T const* z = v.z;
    auto dir = [&](int idx) -> T { return z[idx] + beta * pold[idx]; };
    double pq = 0.0;
    if (pi.dim == 3) {
        // 3D: the direction was formed by cg_direction3_kernel (the curl-curl
        // stencil reads each operand many times, so forming it on the fly
        // would double those loads)
        for (int64_t node = it.begin / 3 + threadIdx.x; node < it.end / 3; node += kThreads) {
            T q[3];
            mag3d_apply_node<T, G>(pnew, v.nu, pi, static_cast<int>(node), q);
            for (int cc = 0; cc < 3; ++cc) {
                int const row = static_cast<int>(3 * node + cc);
                v.q[row] = q[cc];
                pq += static_cast<double>(pnew[row]) * static_cast<double>(q[cc]);
            }
        }
    } else {
        // (i, j) of the thread's rows advance by adding: no division per row
        int const nx = static_cast<int>(pi.nx);
        int row = static_cast<int>(it.begin) + threadIdx.x;
        int j = row / nx, i = row - j * nx;
        for (; row < it.end; row += kThreads) {
            T const q = mag_apply_node_ij<T>(dir, v.nu, nx, static_cast<int>(pi.ny), row, i, j);
            T const pr = dir(row);
            pnew[row] = pr;
            v.q[row] = q;
            pq += static_cast<double>(pr) * static_cast<double>(q);
            i += kThreads;
            while (i >= nx) {
                i -= nx;
                ++j;
            }
        }
    }
    double const pq_b = block_sum(pq, red);
    double tot = 0.0;
    if (finish_reduction(pq_b, part, it.index, pi.first_item, pi.nitems, &s->counter_a, &tot)) {
        s->alpha = s->rz / tot;
        if (!isfinite(s->alpha)) s->nonfinite = 1;
    }
}

// The apply of a batch whose problems are all 3D (the direction formed by
// cg_direction3_kernel): the 3D rows of cg_dir_apply_kernel in a kernel of
// their own, so the register budget is the 3D stencil's and three CTAs fit
// on a multiprocessor (two for the combined kernel).
template <class T, bool G = false>
__global__ void __launch_bounds__(kThreads, 3) cg_apply3_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                                Vecs<T> const* vecs, Scalars* sc, double* part)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act[blockIdx.x]];
    Scalars* s = sc + it.prob;
    if (s->done || s->outer_done) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    T const* pnew = s->pbuf == 0 ? v.p2 : v.p;
    double pq = 0.0;
    for (int64_t node = it.begin / 3 + threadIdx.x; node < it.end / 3; node += kThreads) {
        T q[3];
        mag3d_apply_node<T, G>(pnew, v.nu, pi, static_cast<int>(node), q);
        for (int cc = 0; cc < 3; ++cc) {
            int const row = static_cast<int>(3 * node + cc);
            v.q[row] = q[cc];
            pq += static_cast<double>(pnew[row]) * static_cast<double>(q[cc]);
        }
    }
    double const pq_b = block_sum(pq, red);
    double tot = 0.0;
    if (finish_reduction(pq_b, part, it.index, pi.first_item, pi.nitems, &s->counter_a, &tot)) {
        s->alpha = s->rz / tot;
        if (!isfinite(s->alpha)) s->nonfinite = 1;
    }
}

// p = z + beta p_old into the other direction buffer, for the 3D problems of
// the batch (2D problems form it inside cg_dir_apply_kernel).
template <class T>
__global__ void __launch_bounds__(kThreads) cg_direction3_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                                 Vecs<T> const* vecs, Scalars const* sc)
{
    Item const it = items[act[blockIdx.x]];
    Scalars const* s = sc + it.prob;
    if (s->done || s->outer_done || info[it.prob].dim != 3) return;
    Vecs<T> const v = vecs[it.prob];
    T const* pold = s->pbuf == 0 ? v.p : v.p2;
    T* pnew = s->pbuf == 0 ? v.p2 : v.p;
    T const beta = static_cast<T>(s->beta);
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) pnew[row] = v.z[row] + beta * pold[row];
}

template <class T>
__global__ void __launch_bounds__(kThreads) cg_update_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                             Vecs<T> const* vecs, Scalars* sc, double* part_a,
                                                             double* part_b)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act[blockIdx.x]];
    Scalars* s = sc + it.prob;
    if (s->done || s->outer_done) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    T const* pcur = s->pbuf == 0 ? v.p2 : v.p;
    T const alpha = static_cast<T>(s->alpha);
    double rz = 0.0, rr = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        T const x = v.x[row] + alpha * pcur[row];
        T const r = v.r[row] - alpha * v.q[row];
        T const z = v.dinv[row] * r;
        v.x[row] = x;
        v.r[row] = r;
        v.z[row] = z;
        rz += static_cast<double>(r) * static_cast<double>(z);
        rr += static_cast<double>(r) * static_cast<double>(r);
    }
    double const rz_b = block_sum(rz, red);
    double const rr_b = block_sum(rr, red);
    double const vals[2] = {rz_b, rr_b};
    double* parts[2] = {part_a, part_b};
    double tot[2];
    if (finish_reduction_k<2>(vals, parts, it.index, pi.first_item, pi.nitems, &s->counter_b, tot)) {
        double const trz = tot[0], tot_rr = tot[1];
        s->beta = trz / s->rz;
        s->rz = trz;
        s->rr = tot_rr;
        s->iters += 1;
        s->total_iters += 1;
        s->pbuf ^= 1;
        if (!isfinite(tot_rr) || !isfinite(trz)) s->nonfinite = 1;
        if (tot_rr <= s->inner_tol2 * s->rr0 || s->nonfinite || s->total_iters >= pi.max_iters) s->done = 1;
    }
}

// Start or continue the CG of a refinement pass on the new outer residual:
// r = r64 / scale, z = D^-1 r, x = 0 (the correction restarts; x64 holds the
// previous ones), r.z and r.r.  fresh: p_old = z and beta = 0, so the first
// direction is z.  Otherwise the direction of the previous pass is kept (the
// Krylov space survives the residual replacement).  The pass ended at
// iterate k with (r.z)_k and beta_old = (r.z)_k / (r.z)_{k-1}; the replaced
// residual continues iterate k, so its direction is z + beta' p_{k-1} with
// beta' = (r.z)~ / (r.z)_{k-1}, all in the units of the new scale: p_{k-1}
// is rho p_old there and (r.z)_{k-1} is rho^2 (r.z)_k / beta_old, rho =
// scale_prev / scale, so beta = beta_old (r.z)~ / (rho (r.z)_k) applied to
// the stored p_old.
template <class T>
__global__ void __launch_bounds__(kThreads) cg_replace_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                              Vecs<T> const* vecs, double const* const* r64,
                                                              Scalars* sc, double* part_a, double* part_b, int fresh)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act[blockIdx.x]];
    Scalars* s = sc + it.prob;
    if (s->outer_done) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    double const scale = s->scale;
    T* pold = s->pbuf == 0 ? v.p : v.p2;
    double rz = 0.0, rr = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        T const r = static_cast<T>(r64[it.prob][row] / scale);
        T const z = v.dinv[row] * r;
        v.x[row] = T(0);
        v.r[row] = r;
        v.z[row] = z;
        if (fresh) pold[row] = z;
        rz += static_cast<double>(r) * static_cast<double>(z);
        rr += static_cast<double>(r) * static_cast<double>(r);
    }
    double const rz_b = block_sum(rz, red);
    double const rr_b = block_sum(rr, red);
    double const vals[2] = {rz_b, rr_b};
    double* parts[2] = {part_a, part_b};
    double tot[2];
    if (finish_reduction_k<2>(vals, parts, it.index, pi.first_item, pi.nitems, &s->counter_a, tot)) {
        double const trz = tot[0], tot_rr = tot[1];
        // beta = 0 (the direction restarts from z) on a fresh pass, and when
        // no iterate has run since the last replacement
        bool const keep = !fresh && s->iters > 0 && s->rz > 0.0 && s->scale_prev > 0.0;
        s->beta = keep ? s->beta * trz / ((s->scale_prev / scale) * s->rz) : 0.0;
        if (fresh) s->pbuf = 0;
        s->rz = trz;
        s->rr = tot_rr;
        s->rr0 = tot_rr;
        s->iters = 0;
        s->done = (tot_rr == 0.0 || s->total_iters >= pi.max_iters) ? 1 : 0;
        s->nonfinite = 0;
    }
}

// ------------------------------------------------------------------ flexible CG (learned preconditioner)
//
// Notay's truncated flexible CG, FCG(m): z = M(r) from the learned
// preconditioner, which is not a fixed linear operator, is made A-orthogonal
// to the last m directions, p = z - sum_j (z.q_j)/(p_j.q_j) p_j with
// q_j = A p_j, then alpha = (p.r)/(p.q).  Directions live in a ring of m
// slots; iteration k writes slot k mod m.  m = 1 is the one-step truncation
// p = z + beta p.  A problem whose residual has not dropped 10x over `window`
// iterations is marked for the plain solver.

template <class T>
__device__ __forceinline__ T* fcg_slot(T* base, int64_t hstride, int slot)
{
    return base + static_cast<int64_t>(slot) * hstride;
}

// x = 0, r = r64 / scale (precision T), rr0 = r.r; stall window reset.
// Problems already handed to the plain solver get a zero correction.  After
// the first pass (fresh = 0) the stored directions are kept: the projections
// (z.q_j)/(p_j.q_j) p_j and alpha = (p.r)/(p.q) do not depend on the units
// the directions were formed in, so the flexible CG continues on the
// replaced residual instead of restarting.
template <class T>
__global__ void __launch_bounds__(kThreads) fcg_init_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                            Vecs<T> const* vecs, double const* const* r64,
                                                            Scalars* sc, double* part, int fresh)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars* s = sc + it.prob;
    if (s->outer_done) return;
    Vecs<T> const v = vecs[it.prob];
    if (s->fallback) {
        for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) v.x[row] = T(0);
        return;
    }
    ProbInfo const pi = info[it.prob];
    double const scale = s->scale;
    double rr = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        T const r = static_cast<T>(r64[it.prob][row] / scale);
        v.x[row] = T(0);
        v.r[row] = r;
        rr += static_cast<double>(r) * static_cast<double>(r);
    }
    double const rr_b = block_sum(rr, red);
    double tot = 0.0;
    if (finish_reduction(rr_b, part, it.index, pi.first_item, pi.nitems, &s->counter_a, &tot)) {
        s->rr = tot;
        s->rr0 = tot;
        s->win_rr = tot;
        s->win_iters = 0;
        if (fresh) s->iters = 0;
        s->done = (tot == 0.0 || s->total_iters >= pi.max_iters) ? 1 : 0;
        s->nonfinite = 0;
    }
}

// Partials z.q_j over the stored directions (the first min(iters, m)); the
// last CTA forms coef_j = (z.q_j)/(p_j.q_j).  M >= m is the compile-time bound.
template <class T, int M>
__global__ void __launch_bounds__(kThreads) fcg_orth_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                            Vecs<T> const* vecs, Scalars* sc, double* parts_base,
                                                            int64_t hstride, int m, int nitems_all)
{
    __shared__ double red[kThreads / 32];
    __shared__ double vals[M];
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars* s = sc + it.prob;
    if (s->done || s->outer_done || s->fallback) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    int const nvalid = min(s->iters, m);
    if (nvalid == 0) return;
    double acc[M];
#pragma unroll
    for (int j = 0; j < M; ++j) acc[j] = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        double const z = static_cast<double>(v.z[row]);
#pragma unroll
        for (int j = 0; j < M; ++j)
            if (j < nvalid) acc[j] += z * static_cast<double>(fcg_slot(v.qh, hstride, j)[row]);
    }
#pragma unroll
    for (int j = 0; j < M; ++j) {
        double const t = block_sum(acc[j], red);
        if (threadIdx.x == 0) vals[j] = t;
    }
    __syncthreads();
    double* parts[M];
#pragma unroll
    for (int j = 0; j < M; ++j) parts[j] = parts_base + static_cast<int64_t>(j) * nitems_all;  // one slot per item of the batch
    double tot[M];
    if (finish_reduction_k<M>(vals, parts, it.index, pi.first_item, pi.nitems, &s->counter_a, tot)) {
        for (int j = 0; j < nvalid; ++j) {
            s->coef[j] = tot[j] / s->pq_hist[j];
            if (!isfinite(s->coef[j])) s->nonfinite = 1;
        }
    }
}

// p_slot = z - sum_j coef_j p_j, slot = iters mod m.  When the ring is full
// the slot being written is also the oldest term of the sum; each thread
// reads its element of every p_j before writing.
template <class T, int M>
__global__ void __launch_bounds__(kThreads) fcg_direction_kernel(Item const* items, int const* act, Vecs<T> const* vecs,
                                                                 Scalars const* sc, int64_t hstride, int m)
{
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars const* s = sc + it.prob;
    if (s->done || s->outer_done || s->fallback) return;
    Vecs<T> const v = vecs[it.prob];
    int const nvalid = min(s->iters, m);
    int const slot = s->iters % m;
    T c[M];
#pragma unroll
    for (int j = 0; j < M; ++j) c[j] = j < nvalid ? static_cast<T>(s->coef[j]) : T(0);
    T* const out = fcg_slot(v.ph, hstride, slot);
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        T p = v.z[row];
#pragma unroll
        for (int j = 0; j < M; ++j)
            if (j < nvalid) p -= c[j] * fcg_slot(v.ph, hstride, j)[row];
        out[row] = p;
    }
}

// q_slot = A p_slot, partials p.q and p.r; the last CTA stores p.q for the
// slot and forms alpha.
template <class T>
__global__ void __launch_bounds__(kThreads) fcg_apply_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                             Vecs<T> const* vecs, Scalars* sc, double* part_a,
                                                             double* part_b, int64_t hstride, int m)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars* s = sc + it.prob;
    if (s->done || s->outer_done || s->fallback) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    int const slot = s->iters % m;
    T const* const p = fcg_slot(v.ph, hstride, slot);
    T* const qo = fcg_slot(v.qh, hstride, slot);
    double pq = 0.0, pr = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        T const q = mag_apply_row(p, v.nu, pi, row);
        qo[row] = q;
        double const pv = static_cast<double>(p[row]);
        pq += pv * static_cast<double>(q);
        pr += pv * static_cast<double>(v.r[row]);
    }
    double const pq_b = block_sum(pq, red);
    double const pr_b = block_sum(pr, red);
    double const vals[2] = {pq_b, pr_b};
    double* parts[2] = {part_a, part_b};
    double tot[2];
    if (finish_reduction_k<2>(vals, parts, it.index, pi.first_item, pi.nitems, &s->counter_a, tot)) {
        double const tpq = tot[0], tot_pr = tot[1];
        s->pq_hist[slot] = tpq;
        s->alpha = tot_pr / tpq;
        if (!isfinite(s->alpha)) s->nonfinite = 1;
    }
}

// x += alpha p_slot, r -= alpha q_slot, partial r.r; the last CTA advances
// the iteration (and so the slot) and checks convergence and the stall window.
template <class T>
__global__ void __launch_bounds__(kThreads) fcg_update_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                              Vecs<T> const* vecs, Scalars* sc, double* part,
                                                              int window, int64_t hstride, int m)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars* s = sc + it.prob;
    if (s->done || s->outer_done || s->fallback) return;
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    int const slot = s->iters % m;
    T const* const p = fcg_slot(v.ph, hstride, slot);
    T const* const q = fcg_slot(v.qh, hstride, slot);
    T const alpha = static_cast<T>(s->alpha);
    double rr = 0.0;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        T const r = v.r[row] - alpha * q[row];
        v.x[row] = v.x[row] + alpha * p[row];
        v.r[row] = r;
        rr += static_cast<double>(r) * static_cast<double>(r);
    }
    double const rr_b = block_sum(rr, red);
    double tot = 0.0;
    if (finish_reduction(rr_b, part, it.index, pi.first_item, pi.nitems, &s->counter_c, &tot)) {
        s->rr = tot;
        s->iters += 1;
        s->total_iters += 1;
        s->learned_iters += 1;
        if (!isfinite(tot)) s->nonfinite = 1;
        if (tot <= s->inner_tol2 * s->rr0 || s->nonfinite || s->total_iters >= pi.max_iters) s->done = 1;
        if (++s->win_iters >= window) {
            if (!(tot <= 0.01 * s->win_rr)) {
                s->fallback = 1;
                s->done = 1;
            }
            s->win_rr = tot;
            s->win_iters = 0;
        }
    }
}

// active[p] = 1 while problem p's flexible CG still iterates; the network
// skips the others.
__global__ void fcg_active_kernel(Scalars const* sc, int np, int* active)
{
    int const p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= np) return;
    Scalars const& s = sc[p];
    active[p] = (s.done || s.outer_done || s.fallback) ? 0 : 1;
}

// r64 = b - A x64 and its norm (outer residual, FP64); marks outer convergence.
// act: the items to visit (NULL: every item, one CTA each).
template <bool G = false>
__global__ void __launch_bounds__(kThreads) residual64_kernel(Item const* items, int const* act, ProbInfo const* info,
                                                              double const* const* nu64, double const* const* rhs,
                                                              double* const* x64, double* const* r64, Scalars* sc,
                                                              double* part, double tol2, double floor2, int mark)
{
    __shared__ double red[kThreads / 32];
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars* s = sc + it.prob;
    if (s->outer_done) return;
    ProbInfo const pi = info[it.prob];
    double rr = 0.0;
    if (pi.dim == 3) {
        for (int64_t node = it.begin / 3 + threadIdx.x; node < it.end / 3; node += kThreads) {
            double ax[3];
            mag3d_apply_node<double, G>(x64[it.prob], nu64[it.prob], pi, static_cast<int>(node), ax);
            for (int c = 0; c < 3; ++c) {
                double const r = rhs[it.prob][3 * node + c] - ax[c];
                r64[it.prob][3 * node + c] = r;
                rr += r * r;
            }
        }
    } else {
        for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
            double const ax = mag_apply_row<double, G>(x64[it.prob], nu64[it.prob], pi, row);
            double const r = rhs[it.prob][row] - ax;
            r64[it.prob][row] = r;
            rr += r * r;
        }
    }
    double const rr_b = block_sum(rr, red);
    double tot = 0.0;
    if (finish_reduction(rr_b, part, it.index, pi.first_item, pi.nitems, &s->counter_a, &tot)) {
        s->rr = tot;
        s->scale_prev = s->scale;
        s->scale = sqrt(tot);
        if (mark && (tot <= tol2 * s->bb || !isfinite(tot))) s->outer_done = 1;
        // Next inner solve: reduce the (unit-scaled) residual until the outer
        // residual would be half the tolerance, but never below the floor the
        // inner precision can reach.
        s->inner_tol2 = fmax(floor2, 0.25 * tol2 * s->bb / fmax(tot, 1e-300));
        if (!isfinite(tot)) s->nonfinite = 1;
    }
}

// x64 += scale * e (inner correction, promoted to FP64).
template <class T>
__global__ void __launch_bounds__(kThreads) refine_kernel(Item const* items, int const* act, Vecs<T> const* vecs,
                                                          double* const* x64, Scalars const* sc)
{
    Item const it = items[act != nullptr ? act[blockIdx.x] : blockIdx.x];
    Scalars const* s = sc + it.prob;
    if (s->outer_done) return;
    T const* e = vecs[it.prob].x;
    double const scale = s->scale;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads)
        x64[it.prob][row] += scale * static_cast<double>(e[row]);
}

// nu = 1/mu per node (FP64 and, for the inner solve, the precision T) and
// the inverse diagonal of the operator per unknown.
template <class T>
__global__ void setup_kernel(Item const* items, ProbInfo const* info, double const* const* mu, double* const* nu64,
                             Vecs<T> const* vecs)
{
    Item const it = items[blockIdx.x];
    ProbInfo const pi = info[it.prob];
    Vecs<T> const v = vecs[it.prob];
    double const* m = mu[it.prob];
    int const per_node = pi.dim == 2 ? 1 : 3;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) {
        if (row % per_node == 0) {
            int64_t const node = row / per_node;
            double const nu = 1.0 / m[node];
            nu64[it.prob][node] = nu;
            v.nu[node] = static_cast<T>(nu);
        }
        v.dinv[row] = static_cast<T>(1.0 / mag_diag_row(m, pi, row));
    }
}

__global__ void copy_kernel(Item const* items, double const* const* src, double* const* dst, Scalars const* sc)
{
    Item const it = items[blockIdx.x];
    (void)sc;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) dst[it.prob][row] = src[it.prob][row];
}

template <class T>
__global__ void copy_from_vec_kernel(Item const* items, Vecs<T> const* vecs, double* const* dst)
{
    Item const it = items[blockIdx.x];
    T const* x = vecs[it.prob].x;
    for (int64_t row = it.begin + threadIdx.x; row < it.end; row += kThreads) dst[it.prob][row] = static_cast<double>(x[row]);
}

// ------------------------------------------------------------------ host driver

struct DeviceBuffer
{
    void* ptr = nullptr;
    ~DeviceBuffer() { cudaFree(ptr); }
};

// One problem of a batch, 2D or 3D, as the solver driver sees it.
struct ProblemDesc
{
    int dim;
    int64_t nx, ny, nz;
    double gamma;
    double const* node_mu;
    double const* rhs;
    double* solution;
    double const* coords[3];  // 3D: host node coordinates per axis
    int gauge = 0;            // 3D: 0 penalty, 1 divergence gauge
};

// Central local spacing of a node along one axis (one-sided at the ends),
// the length SimiLie's magnetostatics operator uses for its Hodge factors
// (onelab_interface/magnetostatics_onelab.hpp:856-870).
double local_spacing(double const* c, int64_t n, int64_t i)
{
    if (n < 2) return 1.0;
    if (i == 0) return c[1] - c[0];
    if (i + 1 == n) return c[n - 1] - c[n - 2];
    return 0.5 * (c[i + 1] - c[i - 1]);
}

// ---- divergence gauge: the codifferential's coefficients, read off the
// library's own codifferential (the reference's SimiLie Codifferential::value
// at every node, identity metric, node positions) applied to six probes.
// Probe (a, parity) is 1 on component a at the interior nodes whose index
// along a has that parity; at a node of the same parity the output is the
// coefficient of A_a(m), at the others that of A_a(m - e_a), each already
// zero where the column is a boundary DOF.

__global__ void gauge_probe_kernel(double* p, int nx, int ny, int nz, int a, int parity)
{
    int64_t const node = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (node >= static_cast<int64_t>(nx) * ny * nz) return;
    int const i = static_cast<int>(node % nx);
    int64_t const t = node / nx;
    int const j = static_cast<int>(t % ny), k = static_cast<int>(t / ny);
    int const idx = a == 0 ? i : (a == 1 ? j : k);
    bool const in = i > 0 && j > 0 && k > 0 && i + 1 < nx && j + 1 < ny && k + 1 < nz;
    for (int c = 0; c < 3; ++c) p[3 * node + c] = (c == a && in && idx % 2 == parity) ? 1.0 : 0.0;
}

__global__ void gauge_extract_kernel(double const* q, double* gd, int nx, int ny, int nz, int a, int parity)
{
    int64_t const node = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (node >= static_cast<int64_t>(nx) * ny * nz) return;
    int const i = static_cast<int>(node % nx);
    int64_t const t = node / nx;
    int const j = static_cast<int>(t % ny), k = static_cast<int>(t / ny);
    int const idx = a == 0 ? i : (a == 1 ? j : k);
    if (idx % 2 == parity) gd[8 * node + a] = q[node];
    else gd[8 * node + 3 + a] = q[node];
}

// w(m) = product of the local spacings (the reference's codifferential
// weights, magnetostatics_onelab.hpp:1896-1898); FP32 copy of the table.
__global__ void gauge_weight_kernel(ProbInfo pi, double* gd, float* gd32)
{
    int64_t const node = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (node >= pi.nodes) return;
    int64_t const i = node % pi.nx, t = node / pi.nx, j = t % pi.ny, k = t / pi.ny;
    gd[8 * node + 6] = pi.ls64[0][i] * pi.ls64[1][j] * pi.ls64[2][k];
    gd[8 * node + 7] = 0.0;
    if (gd32 != nullptr)
        for (int q = 0; q < 8; ++q) gd32[8 * node + q] = static_cast<float>(gd[8 * node + q]);
}

// gd (8 doubles per node), gd32 (8 floats per node, may be NULL); probe (3
// doubles per node) and out (1 per node) are scratch.  pi carries the
// device spacing tables.
sil_status build_divergence_gauge(ProblemDesc const& q, ProbInfo const& pi, double* gd, float* gd32, double* probe,
                                  double* out, cudaStream_t st)
{
    int64_t const len[3] = {q.nx, q.ny, q.nz};
    sil_geometry geo = nullptr;
    if (sil_status s = sil_geometry_create(&geo, 3, q.coords, len, nullptr); s != SIL_OK) return s;
    struct GeoGuard
    {
        sil_geometry g;
        ~GeoGuard() { sil_geometry_destroy(g); }
    } guard {geo};
    sil_field in {}, o {};
    in.data = probe;
    in.dtype = SIL_F64;
    in.ndims = 3;
    in.ncomp = 3;
    o.data = out;
    o.dtype = SIL_F64;
    o.ndims = 3;
    o.ncomp = 1;
    int64_t stride = 1;
    for (int a = 0; a < 3; ++a) {
        in.extent[a] = o.extent[a] = len[a];
        in.stride[a] = 3 * stride;  // solver layout: 3 * (i + nx (j + ny k)) + c
        o.stride[a] = stride;
        stride *= len[a];
    }
    in.comp_stride = 1;
    o.comp_stride = 1;
    int const nodes_blocks = static_cast<int>((pi.nodes + 255) / 256);
    int const nx = static_cast<int>(q.nx), ny = static_cast<int>(q.ny), nz = static_cast<int>(q.nz);
    SIL_CUDA_CHECK(cudaMemsetAsync(gd, 0, sizeof(double) * 8 * pi.nodes, st));
    for (int a = 0; a < 3; ++a)
        for (int parity = 0; parity < 2; ++parity) {
            gauge_probe_kernel<<<nodes_blocks, 256, 0, st>>>(probe, nx, ny, nz, a, parity);
            if (sil_status s = sil_codifferential(geo, st, 7u, 1, &in, &o); s != SIL_OK) return s;
            gauge_extract_kernel<<<nodes_blocks, 256, 0, st>>>(out, gd, nx, ny, nz, a, parity);
        }
    gauge_weight_kernel<<<nodes_blocks, 256, 0, st>>>(pi, gd, gd32);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

template <class T>
sil_status solve_batch_rows(std::vector<ProblemDesc> const& probs, sil_solve_settings const& set,
                            sil_solve_diagnostics* diag, cudaStream_t stream, nn::Net* learned, int item_rows)
{
    int const np = static_cast<int>(probs.size());
    // Work items: contiguous row ranges of item_rows rows per problem (3D:
    // whole nodes, four thirds of that), one CTA each.
    std::vector<Item> items;
    std::vector<ProbInfo> info(np);
    int64_t total_rows = 0;
    // 3D spacing tables, per problem [ls_x ls_y ls_z ils_x ils_y ils_z].
    std::vector<double> sp64;
    std::vector<int64_t> sp_off(np, -1);
    for (int p = 0; p < np; ++p) {
        ProblemDesc const& q = probs[p];
        ProbInfo& pi = info[p];
        pi = ProbInfo {};
        pi.dim = q.dim;
        pi.nx = q.nx;
        pi.ny = q.ny;
        pi.nz = q.dim == 3 ? q.nz : 1;
        pi.nodes = pi.nx * pi.ny * pi.nz;
        pi.n = q.dim == 3 ? 3 * pi.nodes : pi.nodes;
        pi.gamma = q.gamma;
        pi.max_iters = set.max_iterations > 0 ? set.max_iterations : 100000;
        pi.first_item = static_cast<int>(items.size());
        int idx = 0;
        // 3D items: whole nodes (3 rows each), four times the 2D item, so
        // the per-CTA prologue is amortised over more of the costlier 3D rows
        int64_t const step = q.dim == 3 ? (4 * item_rows / 3) * 3 : item_rows;
        for (int64_t b = 0; b < pi.n; b += step, ++idx) items.push_back({p, idx, b, std::min(pi.n, b + step)});
        pi.nitems = idx;
        total_rows += pi.n;
        if (q.dim == 3) {
            sp_off[p] = static_cast<int64_t>(sp64.size());
            int64_t const len[3] = {q.nx, q.ny, q.nz};
            for (int a = 0; a < 3; ++a)
                for (int64_t i = 0; i < len[a]; ++i) sp64.push_back(local_spacing(q.coords[a], len[a], i));
            for (int a = 0; a < 3; ++a)
                for (int64_t i = 0; i < len[a]; ++i) sp64.push_back(1.0 / local_spacing(q.coords[a], len[a], i));
        }
    }
    std::vector<float> sp32(sp64.begin(), sp64.end());
    int const nitems = static_cast<int>(items.size());
    int const nvec = 8;  // x r z p q dinv nu p2 in precision T
    size_t const vec_bytes = ((total_rows * sizeof(T) + 255) / 256) * 256;
    size_t const d_bytes = ((total_rows * sizeof(double) + 255) / 256) * 256;
    size_t const ndouble_vecs = 3;  // nu64, r64, x64
    // Flexible CG ring: m stored directions and their images; m = 1 reuses p and q.
    int const fdirs = learned != nullptr ? (set.flexible_directions > 0 ? set.flexible_directions : 8) : 1;
    if (fdirs > kMaxDirs) return fail(SIL_ERR_INVALID, "flexible_directions exceeds 16");
    int const nhist = fdirs > 1 ? 2 * fdirs : 0;
    size_t bytes = (nvec + nhist) * vec_bytes + ndouble_vecs * d_bytes;
    // divergence-gauge coefficient tables (8 doubles + 8 floats per node)
    std::vector<size_t> gauge_off(np, 0);
    bool const any_gauge = std::any_of(probs.begin(), probs.end(), [](ProblemDesc const& q) {
        return q.dim == 3 && q.gauge != 0;
    });
    // the divergence-gauge variants only where a problem needs them
    auto const residual64 = any_gauge ? residual64_kernel<true> : residual64_kernel<false>;
    size_t gauge_bytes = 0;
    for (int p = 0; p < np; ++p) {
        if (probs[p].dim != 3 || probs[p].gauge == 0) continue;
        gauge_off[p] = gauge_bytes;
        gauge_bytes += ((static_cast<size_t>(info[p].nodes) * 8 * (sizeof(double) + sizeof(float)) + 255) / 256) * 256;
    }
    bytes += gauge_bytes + 256;
    bytes += sizeof(Item) * nitems + sizeof(ProbInfo) * np + sizeof(Vecs<T>) * np + sizeof(Scalars) * np
             + (3 + kMaxDirs) * sizeof(double) * nitems + 7 * sizeof(void*) * np
             + sp64.size() * (sizeof(double) + sizeof(float)) + sizeof(int) * np + sizeof(int) * nitems
             + 23 * 256;
    DeviceBuffer buf;
    SIL_CUDA_CHECK(cudaMalloc(&buf.ptr, bytes));
    char* base = static_cast<char*>(buf.ptr);
    auto take = [&](size_t b) {
        char* r = base;
        base += (b + 255) / 256 * 256;
        return r;
    };
    T* vec_base[nvec];
    for (int k = 0; k < nvec; ++k) vec_base[k] = reinterpret_cast<T*>(take(vec_bytes));
    T* hist_base = nhist > 0 ? reinterpret_cast<T*>(take(nhist * vec_bytes)) : nullptr;
    int64_t const hstride = static_cast<int64_t>(vec_bytes / sizeof(T));
    double* nu64_base = reinterpret_cast<double*>(take(d_bytes));
    double* r64_base = reinterpret_cast<double*>(take(d_bytes));
    double* x64_base = reinterpret_cast<double*>(take(d_bytes));
    Item* d_items = reinterpret_cast<Item*>(take(sizeof(Item) * nitems));
    ProbInfo* d_info = reinterpret_cast<ProbInfo*>(take(sizeof(ProbInfo) * np));
    Vecs<T>* d_vecs = reinterpret_cast<Vecs<T>*>(take(sizeof(Vecs<T>) * np));
    Scalars* d_sc = reinterpret_cast<Scalars*>(take(sizeof(Scalars) * np));
    double* part_a = reinterpret_cast<double*>(take(sizeof(double) * nitems));
    double* part_b = reinterpret_cast<double*>(take(sizeof(double) * nitems));
    double* part_c = reinterpret_cast<double*>(take(sizeof(double) * nitems));
    double* part_h = reinterpret_cast<double*>(take(sizeof(double) * kMaxDirs * nitems));
    int* d_active = reinterpret_cast<int*>(take(sizeof(int) * np));
    int* d_act = reinterpret_cast<int*>(take(sizeof(int) * nitems));
    char* gauge_base = gauge_bytes > 0 ? take(gauge_bytes) : nullptr;
    double const** d_mu = reinterpret_cast<double const**>(take(sizeof(void*) * np));
    double const** d_rhs = reinterpret_cast<double const**>(take(sizeof(void*) * np));
    double** d_nu64 = reinterpret_cast<double**>(take(sizeof(void*) * np));
    double** d_x64 = reinterpret_cast<double**>(take(sizeof(void*) * np));
    double** d_r64 = reinterpret_cast<double**>(take(sizeof(void*) * np));
    double** d_sol = reinterpret_cast<double**>(take(sizeof(void*) * np));
    double** d_scratch = reinterpret_cast<double**>(take(sizeof(void*) * np));
    double* d_sp64 = reinterpret_cast<double*>(take(sizeof(double) * sp64.size()));
    float* d_sp32 = reinterpret_cast<float*>(take(sizeof(float) * sp32.size()));
    for (int p = 0; p < np; ++p) {
        if (sp_off[p] < 0) continue;
        int64_t const len[3] = {info[p].nx, info[p].ny, info[p].nz};
        int64_t o = sp_off[p];
        for (int a = 0; a < 3; ++a) {
            info[p].ls64[a] = d_sp64 + o;
            info[p].ls32[a] = d_sp32 + o;
            o += len[a];
        }
        for (int a = 0; a < 3; ++a) {
            info[p].ils64[a] = d_sp64 + o;
            info[p].ils32[a] = d_sp32 + o;
            o += len[a];
        }
    }
    if (!sp64.empty()) {
        SIL_CUDA_CHECK(cudaMemcpyAsync(d_sp64, sp64.data(), sizeof(double) * sp64.size(), cudaMemcpyHostToDevice, stream));
        SIL_CUDA_CHECK(cudaMemcpyAsync(d_sp32, sp32.data(), sizeof(float) * sp32.size(), cudaMemcpyHostToDevice, stream));
    }
    // Divergence gauge tables, with the problem's slices of r64 / x64 as
    // probe scratch (both are rewritten before the solve reads them).
    {
        int64_t goff = 0;
        for (int p = 0; p < np; ++p) {
            if (probs[p].dim == 3 && probs[p].gauge != 0) {
                double* gd = reinterpret_cast<double*>(gauge_base + gauge_off[p]);
                float* g32 = reinterpret_cast<float*>(gd + 8 * info[p].nodes);
                info[p].gauge = 1;
                info[p].gd64 = gd;
                info[p].gd32 = g32;
                sil_status const gs = build_divergence_gauge(probs[p], info[p], gd, g32, r64_base + goff,
                                                             x64_base + goff, stream);
                if (gs != SIL_OK) return gs;
            }
            goff += info[p].n;
        }
    }

    std::vector<Vecs<T>> vecs(np);
    std::vector<double const*> mu(np), rhs(np);
    std::vector<double*> nu64(np), x64(np), r64(np);
    int64_t off = 0;
    for (int p = 0; p < np; ++p) {
        vecs[p] = {vec_base[0] + off, vec_base[1] + off, vec_base[2] + off, vec_base[3] + off,
                   vec_base[4] + off, vec_base[5] + off, vec_base[6] + off,
                   nhist > 0 ? hist_base + off : vec_base[3] + off,
                   nhist > 0 ? hist_base + fdirs * hstride + off : vec_base[4] + off, vec_base[7] + off};
        mu[p] = probs[p].node_mu;
        rhs[p] = probs[p].rhs;
        nu64[p] = nu64_base + off;
        x64[p] = x64_base + off;
        r64[p] = r64_base + off;
        off += info[p].n;
    }
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_items, items.data(), sizeof(Item) * nitems, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_info, info.data(), sizeof(ProbInfo) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_vecs, vecs.data(), sizeof(Vecs<T>) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_mu, mu.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_rhs, rhs.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_nu64, nu64.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_x64, x64.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_r64, r64.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    std::vector<double*> sol(np), scratch(np);
    for (int p = 0; p < np; ++p) {
        sol[p] = probs[p].solution;
        scratch[p] = r64[p];  // FP64 scratch for the final true residual
    }
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_sol, sol.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_scratch, scratch.data(), sizeof(void*) * np, cudaMemcpyHostToDevice, stream));
    SIL_CUDA_CHECK(cudaMemsetAsync(d_sc, 0, sizeof(Scalars) * np, stream));

    setup_kernel<T><<<nitems, kThreads, 0, stream>>>(d_items, d_info, d_mu, d_nu64, d_vecs);
    SIL_CUDA_CHECK(cudaGetLastError());

    double const tol = set.relative_tolerance > 0 ? set.relative_tolerance : 1e-10;
    int const max_iter = set.max_iterations > 0 ? set.max_iterations : 100000;
    int const chunk = 32;
    std::vector<Scalars> hs(np);

    // Items of the problems not yet converged (the CG kernels skip problems
    // whose inner solve has stopped); a chunk of iterations over them is
    // captured as a CUDA graph, captured again once the list has shrunk by a
    // tenth (a longer list is still correct: its finished problems return at
    // once).
    std::vector<int> open_host;
    open_host.reserve(nitems);
    int captured_n = -1;
    bool const any3d = std::any_of(probs.begin(), probs.end(), [](ProblemDesc const& q) { return q.dim == 3; });
    bool const all3d = std::all_of(probs.begin(), probs.end(), [](ProblemDesc const& q) { return q.dim == 3; });
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    auto build_open = [&]() {
        open_host.clear();
        for (int i = 0; i < nitems; ++i)
            if (!hs[items[i].prob].outer_done) open_host.push_back(i);
    };
    auto capture_chunk = [&]() -> sil_status {
        if (exec != nullptr) cudaGraphExecDestroy(exec);
        if (graph != nullptr) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        int const n = static_cast<int>(open_host.size());
        SIL_CUDA_CHECK(cudaMemcpyAsync(d_act, open_host.data(), sizeof(int) * n, cudaMemcpyHostToDevice, stream));
        cudaStream_t cs;
        SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        for (int c = 0; c < chunk && err == cudaSuccess; ++c) {
            if (any3d) cg_direction3_kernel<T><<<n, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc);
            if (all3d && !any_gauge) cg_apply3_kernel<T, false><<<n, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_a);
            else if (any_gauge) cg_dir_apply_kernel<T, true><<<n, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_a);
            else cg_dir_apply_kernel<T, false><<<n, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_a);
            cg_update_kernel<T><<<n, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_b, part_c);
        }
        cudaError_t const err2 = cudaStreamEndCapture(cs, &graph);
        if (err == cudaSuccess) err = err2;
        if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
        cudaStreamDestroy(cs);
        if (err != cudaSuccess) return cuda_fail(err, "solver graph capture");
        captured_n = n;
        return SIL_OK;
    };
    auto read_scalars = [&]() -> sil_status {
        SIL_CUDA_CHECK(cudaMemcpyAsync(hs.data(), d_sc, sizeof(Scalars) * np, cudaMemcpyDeviceToHost, stream));
        SIL_CUDA_CHECK(cudaStreamSynchronize(stream));
        return SIL_OK;
    };

    // Iterative refinement on the FP64 residual with reliable updates: after
    // every chunk of CG iterations in precision T, x64 += ||r|| x, the FP64
    // true residual r = b - A x64 replaces the recurrence's residual, and CG
    // continues with its previous search direction (residual replacement,
    // not a restart), so the Krylov space survives and the recurrence never
    // drifts far from the true residual.  A problem stops iterating once its
    // recurrence reaches half the outer tolerance and converges once the
    // FP64 residual does.  With T = float the chunks run at half the bytes
    // of FP64 and converge at nearly the FP64 rate.
    sil_status st = SIL_OK;
    int refinements = 0;
    SIL_CUDA_CHECK(cudaMemsetAsync(x64_base, 0, d_bytes, stream));

    // Refinement passes whose inner solve is the flexible CG preconditioned by
    // the learned network, until every problem has converged or been handed to
    // the plain solver (stall or budget).
    auto learned_stage = [&](nn::Net* net, int* total_out, int* refinements_out) -> sil_status {
        if constexpr (!std::is_same_v<T, float>) {
            return fail(SIL_ERR_UNSUPPORTED, "learned solve runs in FP32");
        } else {
            std::vector<nn::Sample> samples(np);
            int64_t o = 0;
            for (int p = 0; p < np; ++p) {
                if (info[p].dim != 2) return fail(SIL_ERR_UNSUPPORTED, "learned solve: 2D problems only");
                samples[p] = {static_cast<int32_t>(info[p].nx), static_cast<int32_t>(info[p].ny), o};
                o += info[p].n;
            }
            nn::Workspace* ws = nullptr;
            sil_status lst = net->prepare(samples, stream, &ws);
            if (lst != SIL_OK) return lst;
            // nu is fixed for the whole solve: the network's log(nu) input is formed once
            lst = net->set_static_nu(ws, vec_base[6], stream);
            if (lst != SIL_OK) return lst;
            float const* nuf = vec_base[6];
            float const* dv = vec_base[5];
            float* rv = vec_base[1];
            float* zv = vec_base[2];
            int const window = set.stall_window > 0 ? set.stall_window : 200;
            double const ltol = set.inner_tolerance > 0 ? set.inner_tolerance : 1e-5;
            int const lmax = set.inner_iterations > 0 ? set.inner_iterations : 4000;
            int const lchunk = 8;
            int ln = 0;  // items the flexible CG's kernels visit (listed in d_act)
            // z -> A-orthogonal direction in the next ring slot.
            auto new_direction = [&](cudaStream_t cs) {
                if (fdirs <= 1) {
                    fcg_orth_kernel<T, 1><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_h, hstride, fdirs,
                                                                    nitems);
                    fcg_direction_kernel<T, 1><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_vecs, d_sc, hstride, fdirs);
                } else if (fdirs <= 4) {
                    fcg_orth_kernel<T, 4><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_h, hstride, fdirs,
                                                                    nitems);
                    fcg_direction_kernel<T, 4><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_vecs, d_sc, hstride, fdirs);
                } else if (fdirs <= 8) {
                    fcg_orth_kernel<T, 8><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_h, hstride, fdirs,
                                                                    nitems);
                    fcg_direction_kernel<T, 8><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_vecs, d_sc, hstride, fdirs);
                } else {
                    fcg_orth_kernel<T, 16><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_h, hstride, fdirs,
                                                                    nitems);
                    fcg_direction_kernel<T, 16><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_vecs, d_sc, hstride, fdirs);
                }
            };
            // The flexible CG's kernels visit the items of the problems still
            // iterating (`ln` of them, listed in d_act); the chunk graph is
            // captured again once that list has shrunk by a tenth.
            cudaGraph_t lgraph = nullptr;
            cudaGraphExec_t lexec = nullptr;
            std::vector<int> lopen;
            lopen.reserve(nitems);
            auto build_lopen = [&]() {
                lopen.clear();
                for (int i = 0; i < nitems; ++i) {
                    Scalars const& q = hs[items[i].prob];
                    if (!q.outer_done && !q.fallback && !q.done) lopen.push_back(i);
                }
            };
            auto capture_learned = [&]() -> sil_status {
                if (lexec != nullptr) cudaGraphExecDestroy(lexec);
                if (lgraph != nullptr) cudaGraphDestroy(lgraph);
                lexec = nullptr;
                lgraph = nullptr;
                ln = static_cast<int>(lopen.size());
                SIL_CUDA_CHECK(cudaMemcpyAsync(d_act, lopen.data(), sizeof(int) * ln, cudaMemcpyHostToDevice, stream));
                cudaStream_t cs;
                SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
                sil_status cst = SIL_OK;
                cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
                for (int c = 0; c < lchunk && err == cudaSuccess && cst == SIL_OK; ++c) {
                    fcg_apply_kernel<T><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_a, part_b,
                                                                 hstride, fdirs);
                    fcg_update_kernel<T><<<ln, kThreads, 0, cs>>>(d_items, d_act, d_info, d_vecs, d_sc, part_c, window,
                                                                  hstride, fdirs);
                    fcg_active_kernel<<<(np + 63) / 64, 64, 0, cs>>>(d_sc, np, d_active);
                    cst = net->forward(ws, nuf, dv, rv, zv, cs, d_active);
                    new_direction(cs);
                }
                cudaError_t const err2 = cudaStreamEndCapture(cs, &lgraph);
                if (err == cudaSuccess) err = err2;
                if (err == cudaSuccess && cst == SIL_OK) err = cudaGraphInstantiate(&lexec, lgraph, 0);
                cudaStreamDestroy(cs);
                if (cst != SIL_OK) return cst;
                if (err != cudaSuccess) return cuda_fail(err, "learned solver graph capture");
                return SIL_OK;
            };
            int tot = 0;
            while (lst == SIL_OK && tot < max_iter) {
                residual64<<<nitems, kThreads, 0, stream>>>(d_items, nullptr, d_info, d_nu64, d_rhs, d_x64, d_r64,
                                                                   d_sc, part_a, tol * tol, ltol * ltol, 1);
                SIL_CUDA_CHECK(cudaMemcpyAsync(hs.data(), d_sc, sizeof(Scalars) * np, cudaMemcpyDeviceToHost, stream));
                SIL_CUDA_CHECK(cudaStreamSynchronize(stream));
                bool active = false;
                for (int p = 0; p < np; ++p) active = active || (!hs[p].outer_done && !hs[p].fallback);
                if (!active) break;
                fcg_init_kernel<T><<<nitems, kThreads, 0, stream>>>(d_items, nullptr, d_info, d_vecs, d_r64, d_sc, part_a,
                                                                    *refinements_out == 0 ? 1 : 0);
                // every problem not converged and not handed over iterates after the init
                for (int p = 0; p < np; ++p) hs[p].done = 0;
                build_lopen();
                lst = capture_learned();
                if (lst != SIL_OK) break;
                fcg_active_kernel<<<(np + 63) / 64, 64, 0, stream>>>(d_sc, np, d_active);
                lst = net->forward(ws, nuf, dv, rv, zv, stream, d_active);
                if (lst != SIL_OK) break;
                new_direction(stream);
                SIL_CUDA_CHECK(cudaGetLastError());
                int const budget = std::min(lmax, max_iter - tot);
                int spent = 0;
                while (spent < budget) {
                    SIL_CUDA_CHECK(cudaGraphLaunch(lexec, stream));
                    spent += lchunk;
                    SIL_CUDA_CHECK(cudaMemcpyAsync(hs.data(), d_sc, sizeof(Scalars) * np, cudaMemcpyDeviceToHost, stream));
                    SIL_CUDA_CHECK(cudaStreamSynchronize(stream));
                    build_lopen();
                    if (lopen.empty()) break;
                    if (10 * static_cast<int>(lopen.size()) < 9 * ln) {
                        lst = capture_learned();
                        if (lst != SIL_OK) break;
                    }
                }
                if (lst != SIL_OK) break;
                tot += spent;
                // A problem still unconverged after a full inner budget goes to the plain solver.
                bool flagged = false;
                for (int p = 0; p < np; ++p) {
                    if (!hs[p].outer_done && !hs[p].fallback && !hs[p].done) {
                        hs[p].fallback = 1;
                        flagged = true;
                    }
                }
                refine_kernel<T><<<nitems, kThreads, 0, stream>>>(d_items, nullptr, d_vecs, d_x64, d_sc);
                if (flagged) {
                    SIL_CUDA_CHECK(cudaMemcpyAsync(d_sc, hs.data(), sizeof(Scalars) * np, cudaMemcpyHostToDevice, stream));
                }
                ++*refinements_out;
            }
            if (lexec != nullptr) cudaGraphExecDestroy(lexec);
            if (lgraph != nullptr) cudaGraphDestroy(lgraph);
            net->set_static_nu(ws, nullptr, stream);
            *total_out = tot;
            return lst;
        }
    };
    // bb = ||b||^2 via an init pass from the right-hand side.
    cg_init_kernel<T><<<nitems, kThreads, 0, stream>>>(d_items, d_info, d_vecs, d_rhs, nullptr, d_sc, part_a, part_b,
                                                       false);
    int total = 0;
    if constexpr (std::is_same_v<T, float>) {
        if (learned != nullptr && st == SIL_OK) st = learned_stage(learned, &total, &refinements);
    }
    // Cycle: FP64 residual (outer check) -> residual replacement -> a chunk
    // of iterations -> x64 += ||r|| x; the host reads the problems' state
    // once per cycle.
    auto const residual_open = any_gauge ? residual64_kernel<true> : residual64_kernel<false>;
    build_open();
    if (!open_host.empty()) st = capture_chunk();
    bool fresh = true;
    while (st == SIL_OK && !open_host.empty()) {
        int const n = captured_n;
        residual_open<<<n, kThreads, 0, stream>>>(d_items, d_act, d_info, d_nu64, d_rhs, d_x64, d_r64, d_sc, part_a,
                                                  tol * tol, 0.0, 1);
        st = read_scalars();
        if (st != SIL_OK) break;
        build_open();
        if (open_host.empty() || total >= max_iter) break;
        if (10 * static_cast<int>(open_host.size()) < 9 * captured_n) {
            st = capture_chunk();
            if (st != SIL_OK) break;
        }
        cg_replace_kernel<T><<<captured_n, kThreads, 0, stream>>>(d_items, d_act, d_info, d_vecs, d_r64, d_sc,
                                                                  part_a, part_b, fresh ? 1 : 0);
        SIL_CUDA_CHECK(cudaGetLastError());
        fresh = false;
        SIL_CUDA_CHECK(cudaGraphLaunch(exec, stream));
        total += chunk;
        refine_kernel<T><<<captured_n, kThreads, 0, stream>>>(d_items, d_act, d_vecs, d_x64, d_sc);
        ++refinements;
    }
    if (exec != nullptr) cudaGraphExecDestroy(exec);
    if (graph != nullptr) cudaGraphDestroy(graph);
    if (st == SIL_OK) copy_kernel<<<nitems, kThreads, 0, stream>>>(d_items, d_x64, d_sol, d_sc);
    if (st != SIL_OK) return st;

    // FP64 true residual ||b - A x|| of the returned solution for every problem.
    std::vector<Scalars> hs2(np);
    SIL_CUDA_CHECK(cudaMemcpyAsync(hs2.data(), d_sc, sizeof(Scalars) * np, cudaMemcpyDeviceToHost, stream));
    SIL_CUDA_CHECK(cudaStreamSynchronize(stream));
    for (int p = 0; p < np; ++p) {
        hs2[p].outer_done = 0;
        hs2[p].counter_a = hs2[p].counter_b = hs2[p].counter_c = 0;
    }
    SIL_CUDA_CHECK(cudaMemcpyAsync(d_sc, hs2.data(), sizeof(Scalars) * np, cudaMemcpyHostToDevice, stream));
    residual64<<<nitems, kThreads, 0, stream>>>(d_items, nullptr, d_info, d_nu64, d_rhs, d_sol, d_scratch, d_sc,
                                                       part_a, tol * tol, 0.0, 0);
    SIL_CUDA_CHECK(cudaGetLastError());
    SIL_CUDA_CHECK(cudaMemcpyAsync(hs.data(), d_sc, sizeof(Scalars) * np, cudaMemcpyDeviceToHost, stream));
    SIL_CUDA_CHECK(cudaStreamSynchronize(stream));
    sil_status overall = SIL_OK;
    for (int p = 0; p < np; ++p) {
        sil_solve_diagnostics& d = diag[p];
        d.iterations = hs[p].total_iters;
        d.refinements = refinements;
        d.initial_residual_l2 = std::sqrt(hs[p].bb);
        d.final_residual_l2 = std::sqrt(hs[p].rr);
        d.final_relative_residual = hs[p].bb > 0 ? std::sqrt(hs[p].rr / hs[p].bb) : 0.0;
        d.converged = d.final_relative_residual <= tol && !hs[p].nonfinite;
        d.status = hs[p].nonfinite ? SIL_ERR_NONFINITE : SIL_OK;
        d.learned_iterations = hs[p].learned_iters;
        d.fallback = hs[p].fallback;
        if (hs[p].nonfinite) overall = SIL_ERR_NONFINITE;
    }
    if (overall != SIL_OK) set_error("a problem of the batch met a non-finite value");
    return overall;
}

// Work-item size of the batched CG kernels, picked by timing.  The first
// batch of at least 4 M rows solved in a precision (2D and 3D batches apart)
// runs a 96-iteration solve with items of 2,048, 4,096 and 8,192 rows and
// keeps the fastest for the rest of the process (the tuning solves write the
// caller's solution buffers, which the real solve overwrites).  Smaller
// batches use 4,096 rows until a large one has been tuned.
// SIMILIE_B200_ITEM_ROWS=<rows> forces a size; SIMILIE_B200_AUTOTUNE=0 keeps
// the default.
constexpr int kItemCandidates[3] = {2048, 4096, 8192};
std::mutex g_item_mutex;
int g_item_rows_tuned[4] = {0, 0, 0, 0};  // [precision FP64 / FP32][first problem 2D / 3D]

template <class T>
sil_status choose_item_rows(std::vector<ProblemDesc> const& probs, sil_solve_settings const& set, cudaStream_t stream,
                            int* rows)
{
    *rows = kItemNodes;
    if (char const* e = std::getenv("SIMILIE_B200_ITEM_ROWS")) {
        int const v = std::atoi(e);
        if (v >= kThreads && v % kThreads == 0 && v <= 64 * kThreads) {
            *rows = v;
            return SIL_OK;
        }
    }
    int const key = (sizeof(T) == 8 ? 0 : 2) + (probs.front().dim == 3 ? 1 : 0);
    {
        std::lock_guard<std::mutex> lock(g_item_mutex);
        if (g_item_rows_tuned[key] > 0) {
            *rows = g_item_rows_tuned[key];
            return SIL_OK;
        }
    }
    char const* at = std::getenv("SIMILIE_B200_AUTOTUNE");
    if (at != nullptr && at[0] == '0') return SIL_OK;
    int64_t total = 0;
    for (ProblemDesc const& q : probs) total += (q.dim == 3 ? 3 : 1) * q.nx * q.ny * (q.dim == 3 ? q.nz : 1);
    if (total < (int64_t(1) << 22)) return SIL_OK;
    sil_solve_settings probe = set;
    probe.max_iterations = 96;
    std::vector<sil_solve_diagnostics> scratch(probs.size());
    double best = 1e300;
    int best_rows = kItemNodes;
    for (int c : kItemCandidates) {
        auto const t0 = std::chrono::steady_clock::now();
        sil_status const st = solve_batch_rows<T>(probs, probe, scratch.data(), stream, nullptr, c);
        if (st != SIL_OK) return st;
        double const sec = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (sec < best) {
            best = sec;
            best_rows = c;
        }
    }
    std::lock_guard<std::mutex> lock(g_item_mutex);
    g_item_rows_tuned[key] = best_rows;
    *rows = best_rows;
    return SIL_OK;
}

template <class T>
sil_status solve_batch(std::vector<ProblemDesc> const& probs, sil_solve_settings const& set, sil_solve_diagnostics* diag,
                       cudaStream_t stream, nn::Net* learned = nullptr)
{
    int rows = kItemNodes;
    sil_status const st = choose_item_rows<T>(probs, set, stream, &rows);
    if (st != SIL_OK) return st;
    return solve_batch_rows<T>(probs, set, diag, stream, learned, rows);
}

} // namespace

} // namespace sil

using namespace sil;

extern "C" {

sil_status sil_mag2d_apply(sil_stream stream, int64_t nx, int64_t ny, const double* node_mu, const double* a, double* y)
{
    if (nx < 3 || ny < 3) return fail(SIL_ERR_INVALID, "sil_mag2d_apply: need at least 3x3 nodes");
    if (nx * ny >= (int64_t(1) << 31)) return fail(SIL_ERR_INVALID, "sil_mag2d_apply: fewer than 2^31 nodes supported");
    if (node_mu == nullptr || a == nullptr || y == nullptr) return fail(SIL_ERR_INVALID, "sil_mag2d_apply: NULL pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t const n = nx * ny;
    DeviceBuffer nu;
    SIL_CUDA_CHECK(cudaMallocAsync(&nu.ptr, n * sizeof(double), s));
    int const blocks = static_cast<int>((n + 255) / 256);
    reciprocal_kernel<<<blocks, 256, 0, s>>>(node_mu, static_cast<double*>(nu.ptr), n);
    mag_apply_kernel<<<blocks, 256, 0, s>>>(static_cast<double*>(nu.ptr), a, y, nx, ny);
    SIL_CUDA_CHECK(cudaGetLastError());
    SIL_CUDA_CHECK(cudaFreeAsync(nu.ptr, s));
    nu.ptr = nullptr;
    return SIL_OK;
}

} // extern "C"

// ------------------------------------------------------------------ allocation-free apply

namespace sil {
namespace {

// Scratch of sil_mag2d_apply_noalloc: the reciprocal permeability 1/mu of
// every node.  A fixed array in the library's device image (16 MiB of
// doubles), so the entry point never allocates; every GPU that loads the
// library holds it until the process exits.
constexpr int64_t kNoAllocMaxNodes = int64_t(1) << 21;
static __device__ __align__(256) double g_noalloc_nu[kNoAllocMaxNodes];

constexpr int kNoAllocMaxDevices = 128;
std::mutex g_noalloc_mutex;
double* g_noalloc_ptr[kNoAllocMaxDevices] = {};

// Device address of the scratch array on the current device.  The host-side
// name g_noalloc_nu is only a stand-in for the symbol; its device address is
// looked up once per device, with that device current.
sil_status noalloc_scratch(double** out)
{
    int dev = 0;
    SIL_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(SIL_ERR_UNSUPPORTED, "sil_mag2d_apply_noalloc: device index too large");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (g_noalloc_ptr[dev] == nullptr) {
        void* p = nullptr;
        cudaError_t const err = cudaGetSymbolAddress(&p, g_noalloc_nu);
        if (err != cudaSuccess) return cuda_fail(err, "sil_mag2d_apply_noalloc: cudaGetSymbolAddress");
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    *out = g_noalloc_ptr[dev];
    return SIL_OK;
}

} // namespace
} // namespace sil

extern "C" {

sil_status sil_mag2d_apply_noalloc(sil_stream stream, int64_t nx, int64_t ny, const double* node_mu, const double* a,
                                   double* y)
{
    if (nx < 3 || ny < 3) return fail(SIL_ERR_INVALID, "sil_mag2d_apply_noalloc: need at least 3x3 nodes");
    if (node_mu == nullptr || a == nullptr || y == nullptr)
        return fail(SIL_ERR_INVALID, "sil_mag2d_apply_noalloc: NULL pointer");
    if (nx > kNoAllocMaxNodes || ny > kNoAllocMaxNodes || nx * ny > kNoAllocMaxNodes)
        return fail(SIL_ERR_INVALID, "sil_mag2d_apply_noalloc: nx*ny = " + std::to_string(nx * ny)
                                             + " exceeds the fixed scratch of " + std::to_string(kNoAllocMaxNodes)
                                             + " nodes; use sil_mag2d_apply");
    double* nu = nullptr;
    sil_status const st = noalloc_scratch(&nu);
    if (st != SIL_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t const n = nx * ny;
    int const blocks = static_cast<int>((n + 255) / 256);
    // Every scratch entry the apply reads is written first, so nothing from a
    // previous call needs clearing.
    reciprocal_kernel<<<blocks, 256, 0, s>>>(node_mu, nu, n);
    mag_apply_kernel<<<blocks, 256, 0, s>>>(nu, a, y, nx, ny);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status sil_mag2d_solve_batch(const sil_mag2d_problem* problems, int nproblems, const sil_solve_settings* settings,
                                 sil_solve_diagnostics* diag, sil_stream stream)
{
    if (problems == nullptr || settings == nullptr || diag == nullptr || nproblems < 1)
        return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: NULL argument or empty batch");
    std::vector<ProblemDesc> descs(nproblems);
    for (int p = 0; p < nproblems; ++p) {
        sil_mag2d_problem const& q = problems[p];
        if (q.nx < 3 || q.ny < 3) return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: each problem needs >= 3x3 nodes");
        if (q.nx * q.ny >= (int64_t(1) << 31))
            return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: a problem must have fewer than 2^31 nodes");
        if (q.node_mu == nullptr || q.rhs == nullptr || q.solution == nullptr)
            return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: NULL field pointer");
        descs[p] = {2, q.nx, q.ny, 1, 0.0, q.node_mu, q.rhs, q.solution, {nullptr, nullptr, nullptr}};
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::memset(diag, 0, sizeof(sil_solve_diagnostics) * nproblems);
    if (settings->solver == SIL_SOLVER_CG_F64) return solve_batch<double>(descs, *settings, diag, s);
    if (settings->solver == SIL_SOLVER_MIXED_IR) return solve_batch<float>(descs, *settings, diag, s);
    if (settings->solver == SIL_SOLVER_LEARNED) {
        if (settings->preconditioner == nullptr)
            return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: the learned solver needs a preconditioner");
        if (nproblems > nn::kMaxImages)
            return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: the learned solver takes at most 64 problems per call");
        return solve_batch<float>(descs, *settings, diag, s, &settings->preconditioner->net);
    }
    return fail(SIL_ERR_INVALID, "sil_mag2d_solve_batch: unknown solver kind");
}

} // extern "C"

// ------------------------------------------------------------------ 3D

namespace sil {
namespace {

sil_status check_mag3d(sil_mag3d_problem const& q, char const* who, bool need_fields)
{
    if (q.nx < 3 || q.ny < 3 || q.nz < 3) return fail(SIL_ERR_INVALID, std::string(who) + ": need at least 3x3x3 nodes");
    if (3 * q.nx * q.ny * q.nz >= (int64_t(1) << 31))
        return fail(SIL_ERR_INVALID, std::string(who) + ": fewer than 2^31 unknowns per problem supported");
    if (q.x == nullptr || q.y == nullptr || q.z == nullptr)
        return fail(SIL_ERR_INVALID, std::string(who) + ": NULL coordinate array");
    if (q.node_mu == nullptr) return fail(SIL_ERR_INVALID, std::string(who) + ": NULL node_mu");
    if (need_fields && (q.rhs == nullptr || q.solution == nullptr))
        return fail(SIL_ERR_INVALID, std::string(who) + ": NULL field pointer");
    if (q.gauge != 0 && q.gauge != 1) return fail(SIL_ERR_INVALID, std::string(who) + ": gauge must be 0 or 1");
    if (!std::isfinite(q.gauge_penalty) || (q.gauge == 0 ? !(q.gauge_penalty > 0.0) : q.gauge_penalty == 0.0))
        return fail(SIL_ERR_INVALID, std::string(who) + ": gauge_penalty must be finite and positive "
                                                        "(nonzero for the divergence gauge)");
    double const* c[3] = {q.x, q.y, q.z};
    int64_t const len[3] = {q.nx, q.ny, q.nz};
    for (int a = 0; a < 3; ++a)
        for (int64_t i = 0; i + 1 < len[a]; ++i)
            if (!(c[a][i + 1] > c[a][i]))
                return fail(SIL_ERR_INVALID, std::string(who) + ": node coordinates must increase strictly");
    return SIL_OK;
}

// G: the divergence-gauge variant (the penalty variant keeps fewer registers).
template <bool G>
__global__ void __launch_bounds__(256, 4) mag3d_apply_kernel(ProbInfo pi, double const* nu, double const* a, double* y)
{
    int64_t const node = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (node >= pi.nodes) return;
    double out[3];
    mag3d_apply_node<double, G>(a, nu, pi, static_cast<int>(node), out);
    for (int c = 0; c < 3; ++c) y[3 * node + c] = out[c];
}

} // namespace

sil_status divergence_gauge_table(int64_t nx, int64_t ny, int64_t nz, double const* const coords[3], double const* ls,
                                  double* gd, double* probe, double* out, cudaStream_t st)
{
    ProblemDesc q {};
    q.dim = 3;
    q.nx = nx;
    q.ny = ny;
    q.nz = nz;
    for (int a = 0; a < 3; ++a) q.coords[a] = coords[a];
    q.gauge = 1;
    ProbInfo pi {};
    pi.dim = 3;
    pi.nx = nx;
    pi.ny = ny;
    pi.nz = nz;
    pi.nodes = nx * ny * nz;
    pi.n = 3 * pi.nodes;
    pi.ls64[0] = ls;
    pi.ls64[1] = ls + nx;
    pi.ls64[2] = ls + nx + ny;
    return build_divergence_gauge(q, pi, gd, nullptr, probe, out, st);
}

} // namespace sil

extern "C" {

sil_status sil_mag3d_apply(sil_stream stream, const sil_mag3d_problem* problem, const double* a, double* y)
{
    if (problem == nullptr || a == nullptr || y == nullptr) return fail(SIL_ERR_INVALID, "sil_mag3d_apply: NULL pointer");
    sil_mag3d_problem const& q = *problem;
    sil_status const st = check_mag3d(q, "sil_mag3d_apply", false);
    if (st != SIL_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t const nodes = q.nx * q.ny * q.nz;
    int64_t const len[3] = {q.nx, q.ny, q.nz};
    double const* c[3] = {q.x, q.y, q.z};
    std::vector<double> sp;
    for (int a2 = 0; a2 < 3; ++a2)
        for (int64_t i = 0; i < len[a2]; ++i) sp.push_back(local_spacing(c[a2], len[a2], i));
    for (int a2 = 0; a2 < 3; ++a2)
        for (int64_t i = 0; i < len[a2]; ++i) sp.push_back(1.0 / local_spacing(c[a2], len[a2], i));
    size_t const nu_bytes = (nodes * sizeof(double) + 255) / 256 * 256;
    // divergence gauge: coefficient table (8 per node) and probe scratch (3 + 1 per node)
    size_t const gauge_bytes = q.gauge ? static_cast<size_t>(nodes) * 12 * sizeof(double) : 0;
    DeviceBuffer buf;
    SIL_CUDA_CHECK(cudaMallocAsync(&buf.ptr, nu_bytes + gauge_bytes + sp.size() * sizeof(double), s));
    double* nu = static_cast<double*>(buf.ptr);
    double* gd = reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + nu_bytes);
    double* dsp = reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + nu_bytes + gauge_bytes);
    SIL_CUDA_CHECK(cudaMemcpyAsync(dsp, sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    ProbInfo pi {};
    pi.dim = 3;
    pi.nx = q.nx;
    pi.ny = q.ny;
    pi.nz = q.nz;
    pi.nodes = nodes;
    pi.n = 3 * nodes;
    pi.gamma = q.gauge_penalty;
    int64_t o = 0;
    for (int a2 = 0; a2 < 3; ++a2) {
        pi.ls64[a2] = dsp + o;
        o += len[a2];
    }
    for (int a2 = 0; a2 < 3; ++a2) {
        pi.ils64[a2] = dsp + o;
        o += len[a2];
    }
    if (q.gauge) {
        ProblemDesc desc {3, q.nx, q.ny, q.nz, q.gauge_penalty, q.node_mu, nullptr, nullptr, {q.x, q.y, q.z}, 1};
        sil_status const gs = build_divergence_gauge(desc, pi, gd, nullptr, gd + 8 * nodes, gd + 11 * nodes, s);
        if (gs != SIL_OK) return gs;
        pi.gauge = 1;
        pi.gd64 = gd;
    }
    reciprocal_kernel<<<static_cast<int>((nodes + 255) / 256), 256, 0, s>>>(q.node_mu, nu, nodes);
    auto const kern = pi.gauge ? mag3d_apply_kernel<true> : mag3d_apply_kernel<false>;
    kern<<<static_cast<int>((nodes + 255) / 256), 256, 0, s>>>(pi, nu, a, y);
    SIL_CUDA_CHECK(cudaGetLastError());
    // A copy from pageable memory has left the host table once it returns;
    // the device buffer is freed in stream order after the apply.
    SIL_CUDA_CHECK(cudaFreeAsync(buf.ptr, s));
    buf.ptr = nullptr;
    return SIL_OK;
}

// A 3D operator with its set-up done once: the device spacing tables, the
// node reluctivity 1/mu and (divergence gauge) the codifferential
// coefficient table, so that an apply is one kernel.
} // extern "C"

struct sil_mag3d_operator_s
{
    sil::ProbInfo pi {};
    double const* nu = nullptr;
    void* mem = nullptr;
};

extern "C" {

sil_status sil_mag3d_operator_create(sil_mag3d_operator* out, sil_stream stream, const sil_mag3d_problem* problem)
{
    if (out == nullptr || problem == nullptr) return fail(SIL_ERR_INVALID, "sil_mag3d_operator_create: NULL pointer");
    *out = nullptr;
    sil_mag3d_problem const& q = *problem;
    sil_status const st = check_mag3d(q, "sil_mag3d_operator_create", false);
    if (st != SIL_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    int64_t const nodes = q.nx * q.ny * q.nz;
    int64_t const len[3] = {q.nx, q.ny, q.nz};
    double const* c[3] = {q.x, q.y, q.z};
    std::vector<double> sp;
    for (int a2 = 0; a2 < 3; ++a2)
        for (int64_t i = 0; i < len[a2]; ++i) sp.push_back(local_spacing(c[a2], len[a2], i));
    for (int a2 = 0; a2 < 3; ++a2)
        for (int64_t i = 0; i < len[a2]; ++i) sp.push_back(1.0 / local_spacing(c[a2], len[a2], i));
    size_t const nu_bytes = (nodes * sizeof(double) + 255) / 256 * 256;
    size_t const gauge_bytes = q.gauge ? static_cast<size_t>(nodes) * 12 * sizeof(double) : 0;
    auto* op = new sil_mag3d_operator_s;
    if (cudaMalloc(&op->mem, nu_bytes + gauge_bytes + sp.size() * sizeof(double)) != cudaSuccess) {
        delete op;
        return fail(SIL_ERR_CUDA, "sil_mag3d_operator_create: device allocation failed");
    }
    auto bail = [&](sil_status e) {
        cudaFree(op->mem);
        delete op;
        return e;
    };
    double* nu = static_cast<double*>(op->mem);
    double* gd = reinterpret_cast<double*>(static_cast<char*>(op->mem) + nu_bytes);
    double* dsp = reinterpret_cast<double*>(static_cast<char*>(op->mem) + nu_bytes + gauge_bytes);
    if (cudaMemcpyAsync(dsp, sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, s) != cudaSuccess)
        return bail(fail(SIL_ERR_CUDA, "sil_mag3d_operator_create: table upload failed"));
    ProbInfo& pi = op->pi;
    pi.dim = 3;
    pi.nx = q.nx;
    pi.ny = q.ny;
    pi.nz = q.nz;
    pi.nodes = nodes;
    pi.n = 3 * nodes;
    pi.gamma = q.gauge_penalty;
    int64_t o = 0;
    for (int a2 = 0; a2 < 3; ++a2) {
        pi.ls64[a2] = dsp + o;
        o += len[a2];
    }
    for (int a2 = 0; a2 < 3; ++a2) {
        pi.ils64[a2] = dsp + o;
        o += len[a2];
    }
    if (q.gauge) {
        ProblemDesc desc {3, q.nx, q.ny, q.nz, q.gauge_penalty, q.node_mu, nullptr, nullptr, {q.x, q.y, q.z}, 1};
        sil_status const gs = build_divergence_gauge(desc, pi, gd, nullptr, gd + 8 * nodes, gd + 11 * nodes, s);
        if (gs != SIL_OK) return bail(gs);
        pi.gauge = 1;
        pi.gd64 = gd;
    }
    reciprocal_kernel<<<static_cast<int>((nodes + 255) / 256), 256, 0, s>>>(q.node_mu, nu, nodes);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess)
        return bail(fail(SIL_ERR_CUDA, "sil_mag3d_operator_create: set-up kernels failed"));
    op->nu = nu;
    *out = op;
    return SIL_OK;
}

sil_status sil_mag3d_operator_apply(sil_mag3d_operator op, sil_stream stream, const double* a, double* y)
{
    if (op == nullptr || a == nullptr || y == nullptr) return fail(SIL_ERR_INVALID, "sil_mag3d_operator_apply: NULL pointer");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    auto const kern = op->pi.gauge ? mag3d_apply_kernel<true> : mag3d_apply_kernel<false>;
    kern<<<static_cast<int>((op->pi.nodes + 255) / 256), 256, 0, s>>>(op->pi, op->nu, a, y);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status sil_mag3d_operator_destroy(sil_mag3d_operator op)
{
    if (op == nullptr) return SIL_OK;
    cudaFree(op->mem);
    delete op;
    return SIL_OK;
}

sil_status sil_mag3d_solve_batch(const sil_mag3d_problem* problems, int nproblems, const sil_solve_settings* settings,
                                 sil_solve_diagnostics* diag, sil_stream stream)
{
    if (problems == nullptr || settings == nullptr || diag == nullptr || nproblems < 1)
        return fail(SIL_ERR_INVALID, "sil_mag3d_solve_batch: NULL argument or empty batch");
    std::vector<ProblemDesc> descs(nproblems);
    for (int p = 0; p < nproblems; ++p) {
        sil_mag3d_problem const& q = problems[p];
        sil_status const st = check_mag3d(q, "sil_mag3d_solve_batch", true);
        if (st != SIL_OK) return st;
        descs[p] = {3, q.nx, q.ny, q.nz, q.gauge_penalty, q.node_mu, q.rhs, q.solution, {q.x, q.y, q.z}, q.gauge};
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    std::memset(diag, 0, sizeof(sil_solve_diagnostics) * nproblems);
    if (settings->solver == SIL_SOLVER_CG_F64) return solve_batch<double>(descs, *settings, diag, s);
    if (settings->solver == SIL_SOLVER_MIXED_IR) return solve_batch<float>(descs, *settings, diag, s);
    return fail(SIL_ERR_INVALID, "sil_mag3d_solve_batch: unknown solver kind (the learned solver is 2D only)");
}

} // extern "C"
