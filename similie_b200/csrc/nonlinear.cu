// nonlinear.cu -- 2D and 3D magnetostatics with a saturating ferromagnetic
// material: the nonlinear residual operators, their Jacobians, and the
// Newton solve with a line search whose linear systems are solved by
// Jacobi-CG on the Jacobian (FP64).  The 2D operator is described here; the
// 3D one above its kernels.
//
// Operator (moments criterion, onelab_interface/magnetostatics_onelab.hpp:
// 1271-1426): at an interior row, over the sampled nodes s whose moment
// stencils touch it (the node below, the node itself, the node to the left),
// y = -sum_s c(s -> row) H_comp(B(s), s) with the moments
// B(s) = (a(s + nx) - a(s), a(s) - a(s + 1)); identity rows on the boundary.
// H = B / mu at a linear node; at a ferromagnetic node H_c = B_c (F + q F')
// with F(q) = h(b)/b, b = sqrt(q), q = |B|^2 (the derivative of the
// Hamiltonian q F(q) / 2, src/similie/physics/magnetostatics/
// nonlinear_magnetostatics.py:331-369 through generate_cpp_hamiltonian.py:
// 280-400).  The Jacobian applies each sampled node's 2x2 Hessian of the
// Hamiltonian to the moments of the input (magnetostatics_onelab.hpp:
// 2799-2915): a symmetric 7-point stencil.  Every expression keeps the
// summation order of the reference loops.
#include <algorithm>
#include <cmath>
#include <limits>
#include <string>
#include <thread>
#include <vector>

#include "sil_internal.cuh"

namespace sil {
namespace {

constexpr int kMaxCurve = 64;
constexpr int kBlock = 256;

// Interpolated B-H curve: h piecewise linear in b, intervals bracketed by
// q = b^2, linear extension past the last sample.
// Ref: src/similie/physics/magnetostatics/nonlinear_magnetostatics.py:14-181
struct DevCurve
{
    int n;
    double b[kMaxCurve];
    double h[kMaxCurve];
    double q[kMaxCurve];
    double dh_db[kMaxCurve];
};

struct Geo
{
    int nx, ny;
};

// First interval i with qv <= q[i+1] (0 below the first sample, n-2 past
// the last): the reference's linear scan, as a binary search over the
// strictly increasing q.
__device__ __forceinline__ int bracket_q(DevCurve const& c, double qv)
{
    if (qv <= c.q[0]) return 0;
    int lo = 0, hi = c.n - 2;
    if (!(qv <= c.q[hi + 1])) return c.n - 2;
    while (lo < hi) {
        int const mid = (lo + hi) / 2;
        if (qv <= c.q[mid + 1]) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ double h_from_b(DevCurve const& c, double bv)
{
    if (bv <= c.b[0]) return c.h[0];
    if (bv >= c.b[c.n - 1]) {
        int const k = c.n - 2;
        return c.h[k] + c.dh_db[k] * (bv - c.b[k]);
    }
    int const k = bracket_q(c, bv * bv);
    return c.h[k] + c.dh_db[k] * (bv - c.b[k]);
}

__device__ __forceinline__ double dh_db_from_b(DevCurve const& c, double bv)
{
    if (bv <= c.b[0]) return c.dh_db[0];
    if (bv >= c.b[c.n - 1]) return c.dh_db[c.n - 2];
    return c.dh_db[bracket_q(c, bv * bv)];
}

// F(q), F'(q), F''(q) of F = h/b at b = sqrt(q).
__device__ __forceinline__ void curve_f(DevCurve const& c, double qv, double* f, double* df, double* d2f)
{
    double const bv = sqrt(qv);
    if (bv == 0.0) {
        *f = dh_db_from_b(c, 0.0);
        *df = 0.0;
        *d2f = 0.0;
        return;
    }
    double const hb = h_from_b(c, bv), slope = dh_db_from_b(c, bv);
    *f = hb / bv;
    double const d1 = (slope * bv - hb) / (bv * bv);
    double const intercept = hb - slope * bv;
    double const d2 = 2.0 * intercept / (bv * bv * bv);
    *df = d1 / (2.0 * bv);
    *d2f = d2 / (4.0 * qv) - d1 / (4.0 * qv * bv);
}

__device__ __forceinline__ void node_field(DevCurve const& c, double mu, double ferro, double b0, double b1,
                                           double* h0, double* h1)
{
    if (ferro > 0.5) {
        double const q = b0 * b0 + b1 * b1;
        double F, dF, d2F;
        curve_f(c, q, &F, &dF, &d2F);
        *h0 = b0 * F + q * b0 * dF;
        *h1 = b1 * F + q * b1 * dF;
    } else {
        *h0 = b0 / mu;
        *h1 = b1 / mu;
    }
}

__device__ __forceinline__ void node_jacobian(DevCurve const& c, double mu, double ferro, double b0, double b1,
                                              double* j00, double* j01, double* j11)
{
    if (ferro > 0.5) {
        double const q = b0 * b0 + b1 * b1;
        double F, dF, d2F;
        curve_f(c, q, &F, &dF, &d2F);
        double const base = F + q * dF;
        *j00 = base + 4.0 * b0 * b0 * dF + 2.0 * q * b0 * b0 * d2F;
        *j11 = base + 4.0 * b1 * b1 * dF + 2.0 * q * b1 * b1 * d2F;
        *j01 = 4.0 * b0 * b1 * dF + 2.0 * q * b0 * b1 * d2F;
    } else {
        *j00 = 1.0 / mu;
        *j11 = 1.0 / mu;
        *j01 = 0.0;
    }
}

// Moments at sampled node s of a field v (the reference stencils'
// coefficient order: -1, +1 and +1, -1).
__device__ __forceinline__ double mom0(double const* v, int s, int nx) { return -1.0 * v[s] + 1.0 * v[s + nx]; }
__device__ __forceinline__ double mom1(double const* v, int s) { return 1.0 * v[s] + -1.0 * v[s + 1]; }

__device__ __forceinline__ void stage_curve(DevCurve const& src, DevCurve& dst)
{
    if (threadIdx.x == 0) dst.n = src.n;
    for (int i = threadIdx.x; i < kMaxCurve; i += blockDim.x) {
        dst.b[i] = src.b[i];
        dst.h[i] = src.h[i];
        dst.q[i] = src.q[i];
        dst.dh_db[i] = src.dh_db[i];
    }
    __syncthreads();
}

// Deterministic block sum (fixed tree); valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double* red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
    return t;
}

// Nonlinear operator at one row (the row's own field is evaluated once and
// used for both of its moments).
__device__ __forceinline__ double apply_row(DevCurve const& c, Geo g, double const* a, double const* mu,
                                            double const* ferro, int row)
{
    int const j = row / g.nx, i = row - j * g.nx;
    if (i == 0 || j == 0 || i + 1 == g.nx || j + 1 == g.ny) return a[row];
    double hr0, hr1, h0, h1;
    node_field(c, mu[row], ferro[row], mom0(a, row, g.nx), mom1(a, row), &hr0, &hr1);
    double residual = 0.0;
    if (j - 1 >= 1) {
        int const s = row - g.nx;
        node_field(c, mu[s], ferro[s], mom0(a, s, g.nx), mom1(a, s), &h0, &h1);
        residual -= -1. * h0;
    }
    residual -= 1. * hr0;
    if (i - 1 >= 1) {
        int const s = row - 1;
        node_field(c, mu[s], ferro[s], mom0(a, s, g.nx), mom1(a, s), &h0, &h1);
        residual -= 1. * h1;
    }
    residual -= -1. * hr1;
    return residual;
}

// Jacobian at one row from per-node coefficients (c00, c01, c11) of the
// state: (-outer coefficient) x the X or Y row of each sampled node's 2x2
// block times the input's moments there.
__device__ __forceinline__ double jac_row(Geo g, double const* c00, double const* c01, double const* c11,
                                          double const* x, int row)
{
    int const j = row / g.nx, i = row - j * g.nx;
    if (i == 0 || j == 0 || i + 1 == g.nx || j + 1 == g.ny) return x[row];
    double residual = 0.0;
    double const r0 = mom0(x, row, g.nx), r1 = mom1(x, row);
    if (j - 1 >= 1) {
        int const s = row - g.nx;
        residual += 1.0 * (c00[s] * mom0(x, s, g.nx) + c01[s] * mom1(x, s));
    }
    residual += -1.0 * (c00[row] * r0 + c01[row] * r1);
    if (i - 1 >= 1) {
        int const s = row - 1;
        residual += -1.0 * (c01[s] * mom0(x, s, g.nx) + c11[s] * mom1(x, s));
    }
    residual += 1.0 * (c01[row] * r0 + c11[row] * r1);
    return residual;
}

// out = F(a), or out = rhs - F(a) with per-block partial sums of out^2
// (grid-stride over the rows, fixed grid: deterministic).
__global__ void __launch_bounds__(kBlock) nl_apply_kernel(const __grid_constant__ DevCurve curve, Geo g,
                                                          double const* a, double const* mu, double const* ferro,
                                                          double const* rhs, double* out, double* part)
{
    __shared__ DevCurve c;
    __shared__ double red[kBlock / 32];
    stage_curve(curve, c);
    int const n = g.nx * g.ny;
    double acc = 0.0;
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < n; row += gridDim.x * kBlock) {
        double const f = apply_row(c, g, a, mu, ferro, row);
        if (rhs != nullptr) {
            double const r = rhs[row] - f;
            out[row] = r;
            acc += r * r;
        } else {
            out[row] = f;
        }
    }
    if (part != nullptr) {
        double const t = block_sum(acc, red);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}

// Per interior node: the 2x2 Jacobian block (c00, c01, c11) at the state.
__global__ void __launch_bounds__(kBlock) nl_coef_kernel(const __grid_constant__ DevCurve curve, Geo g,
                                                         double const* x, double const* mu, double const* ferro,
                                                         double* c00, double* c01, double* c11)
{
    __shared__ DevCurve c;
    stage_curve(curve, c);
    int const n = g.nx * g.ny;
    for (int s = blockIdx.x * kBlock + threadIdx.x; s < n; s += gridDim.x * kBlock) {
        int const j = s / g.nx, i = s - j * g.nx;
        if (i == 0 || j == 0 || i + 1 == g.nx || j + 1 == g.ny) {
            c00[s] = 0.0;
            c01[s] = 0.0;
            c11[s] = 0.0;
            continue;
        }
        node_jacobian(c, mu[s], ferro[s], mom0(x, s, g.nx), mom1(x, s), &c00[s], &c01[s], &c11[s]);
    }
}

// Inverse Jacobian diagonal (1 on the boundary), the reference's Jacobi.
__global__ void __launch_bounds__(kBlock) nl_dinv_kernel(Geo g, double const* c00, double const* c01,
                                                         double const* c11, double* dinv)
{
    int const n = g.nx * g.ny;
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < n; row += gridDim.x * kBlock) {
        int const j = row / g.nx, i = row - j * g.nx;
        if (i == 0 || j == 0 || i + 1 == g.nx || j + 1 == g.ny) {
            dinv[row] = 1.0;
            continue;
        }
        double d = 0.0;
        if (j - 1 >= 1) d += c00[row - g.nx];
        d += c00[row] - c01[row];
        if (i - 1 >= 1) d += c11[row - 1];
        d += c11[row] - c01[row];
        dinv[row] = 1.0 / d;
    }
}

// Jacobian apply on the fly (coefficients recomputed from the state).
__global__ void __launch_bounds__(kBlock) nl_jacobian_kernel(const __grid_constant__ DevCurve curve, Geo g,
                                                             double const* st, double const* mu,
                                                             double const* ferro, double const* x, double* y)
{
    __shared__ DevCurve c;
    stage_curve(curve, c);
    int const n = g.nx * g.ny;
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < n; row += gridDim.x * kBlock) {
        int const j = row / g.nx, i = row - j * g.nx;
        if (i == 0 || j == 0 || i + 1 == g.nx || j + 1 == g.ny) {
            y[row] = x[row];
            continue;
        }
        double j00, j01, j11, residual = 0.0;
        double const r0 = mom0(x, row, g.nx), r1 = mom1(x, row);
        if (j - 1 >= 1) {
            int const s = row - g.nx;
            node_jacobian(c, mu[s], ferro[s], mom0(st, s, g.nx), mom1(st, s), &j00, &j01, &j11);
            residual += 1.0 * (j00 * mom0(x, s, g.nx) + j01 * mom1(x, s));
        }
        node_jacobian(c, mu[row], ferro[row], mom0(st, row, g.nx), mom1(st, row), &j00, &j01, &j11);
        residual += -1.0 * (j00 * r0 + j01 * r1);
        double const k01 = j01, k11 = j11;
        if (i - 1 >= 1) {
            int const s = row - 1;
            node_jacobian(c, mu[s], ferro[s], mom0(st, s, g.nx), mom1(st, s), &j00, &j01, &j11);
            residual += -1.0 * (j01 * mom0(x, s, g.nx) + j11 * mom1(x, s));
        }
        residual += 1.0 * (k01 * r0 + k11 * r1);
        y[row] = residual;
    }
}

// ---------------------------------------------------------------- Jacobi-CG on the Jacobian

struct CgState
{
    double rz, pq, alpha, beta, bn, rn;
    int done, iters;
};

// Sum of K interleaved per-block partials (part[k * nparts + b]) in a fixed
// order; one block.
template <int K>
__device__ __forceinline__ void sum_parts(double const* part, int nparts, double* out)
{
    __shared__ double red[kBlock / 32];
    for (int k = 0; k < K; ++k) {
        double v = 0.0;
        for (int b = threadIdx.x; b < nparts; b += kBlock) v += part[k * nparts + b];
        double const t = block_sum(v, red);
        if (threadIdx.x == 0) out[k] = t;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kBlock) norm_finish_kernel(double const* part, int nparts, double* out)
{
    __shared__ double s[1];
    sum_parts<1>(part, nparts, s);
    if (threadIdx.x == 0) *out = sqrt(s[0]);
}

// d = 0, cr = r, z = dinv r, p = z; partials r.z and r.r.
__global__ void __launch_bounds__(kBlock) cg_start_kernel(int n, double const* r, double const* dinv, double* d,
                                                          double* cr, double* z, double* p, double* part)
{
    __shared__ double red[kBlock / 32];
    double rz = 0.0, rr = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        double const rv = r[i], zv = dinv[i] * rv;
        d[i] = 0.0;
        cr[i] = rv;
        z[i] = zv;
        p[i] = zv;
        rz += rv * zv;
        rr += rv * rv;
    }
    double const t0 = block_sum(rz, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t0;
    double const t1 = block_sum(rr, red);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = t1;
}

__global__ void __launch_bounds__(kBlock) cg_init_kernel(double const* part, int nparts, CgState* st, double tol,
                                                         int max_iter)
{
    __shared__ double s[2];
    sum_parts<2>(part, nparts, s);
    if (threadIdx.x == 0) {
        st->rz = s[0];
        st->bn = sqrt(s[1]);
        st->rn = st->bn;
        st->iters = 0;
        st->done = (max_iter <= 0 || !(st->rn > tol * st->bn)) ? 1 : 0;
    }
}

// q = J p and partial p.q.
__global__ void __launch_bounds__(kBlock) cg_jac_kernel(Geo g, double const* c00, double const* c01,
                                                        double const* c11, double const* p, double* q,
                                                        double* part, CgState const* st)
{
    __shared__ double red[kBlock / 32];
    if (st->done) return;
    int const n = g.nx * g.ny;
    double pq = 0.0;
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < n; row += gridDim.x * kBlock) {
        double const qv = jac_row(g, c00, c01, c11, p, row);
        q[row] = qv;
        pq += p[row] * qv;
    }
    double const t = block_sum(pq, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t;
}

__global__ void __launch_bounds__(kBlock) cg_alpha_kernel(double const* part, int nparts, CgState* st)
{
    __shared__ double s[1];
    if (st->done) return;
    sum_parts<1>(part, nparts, s);
    if (threadIdx.x == 0) {
        st->pq = s[0];
        st->alpha = st->rz / s[0];
    }
}

// d += alpha p, cr -= alpha q, z = dinv cr; partials cr.cr and cr.z.
__global__ void __launch_bounds__(kBlock) cg_update_kernel(int n, double* d, double* cr, double const* p,
                                                           double const* q, double const* dinv, double* z,
                                                           double* part, CgState const* st)
{
    __shared__ double red[kBlock / 32];
    if (st->done) return;
    double const alpha = st->alpha;
    double rr = 0.0, rz = 0.0;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) {
        d[i] += alpha * p[i];
        double const rv = cr[i] - alpha * q[i];
        cr[i] = rv;
        double const zv = dinv[i] * rv;
        z[i] = zv;
        rr += rv * rv;
        rz += rv * zv;
    }
    double const t0 = block_sum(rr, red);
    if (threadIdx.x == 0) part[blockIdx.x] = t0;
    double const t1 = block_sum(rz, red);
    if (threadIdx.x == 0) part[gridDim.x + blockIdx.x] = t1;
}

// Convergence test ||cr|| <= tol ||r||, else beta = (r.z)_new / (r.z)_old.
__global__ void __launch_bounds__(kBlock) cg_beta_kernel(double const* part, int nparts, CgState* st, double tol,
                                                         int max_iter)
{
    __shared__ double s[2];
    if (st->done) return;
    sum_parts<2>(part, nparts, s);
    if (threadIdx.x == 0) {
        st->iters += 1;
        st->rn = sqrt(s[0]);
        if (st->rn <= tol * st->bn || st->iters >= max_iter || !isfinite(st->rn)) {
            st->done = 1;
        } else {
            st->beta = s[1] / st->rz;
            st->rz = s[1];
        }
    }
}

__global__ void __launch_bounds__(kBlock) cg_direction_kernel(int n, double* p, double const* z, CgState const* st)
{
    if (st->done) return;
    double const beta = st->beta;
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) p[i] = z[i] + beta * p[i];
}

// cand = x + alpha d.
__global__ void __launch_bounds__(kBlock) axpy_kernel(int n, double const* x, double alpha, double const* d,
                                                      double* out)
{
    for (int i = blockIdx.x * kBlock + threadIdx.x; i < n; i += gridDim.x * kBlock) out[i] = x[i] + alpha * d[i];
}

// ---------------------------------------------------------------- 3D operator
//
// Rows 3 * node + c of the vector potential A (x fastest); interior rows sum,
// over the sampled nodes s whose curl moments hold the row (s = node and its
// neighbours at -e_a for the two other axes), +-hodge_m(s) H_m(B(s)), with
// hodge_m = d_m / (d_a d_b) from the reference's local spacings, then add
// the penalty gauge gamma (d_a d_b / d_c) A_c; boundary rows are the
// identity.  Two passes: the hodge-weighted field per sampled node, then the
// per-row gather in the order of the reference's transposed stencils (by
// sampled node, then moment component).
// Ref: onelab_interface/magnetostatics_onelab.hpp:2241-2396 (operator),
//      2924-3110 (apply_jacobian), 856-910 (Hodge factors).

struct Geo3
{
    int nx, ny, nz;
    double gamma;
    double const* ls[3];  // local spacing per axis
    int gauge;            // 0 penalty, 1 divergence gauge
    double const* gd;     // divergence gauge: 8 per node, E0[3], E1[3], w, 0
};

__device__ __forceinline__ bool interior3(Geo3 const& g, int i, int j, int k)
{
    return i > 0 && j > 0 && k > 0 && i + 1 < g.nx && j + 1 < g.ny && k + 1 < g.nz;
}

__device__ __forceinline__ void node_coords(Geo3 const& g, int s, int* i, int* j, int* k)
{
    int const t = s / g.nx;
    *i = s - t * g.nx;
    *k = t / g.ny;
    *j = t - *k * g.ny;
}

// Divergence gauge, the terms of the linear 3D operator: (D A)(m) =
// sum_a E0(m, a) A_a(m) + E1(m, a) A_a(m - e_a) (boundary columns carry zero
// coefficients), and the term of row (n, c), w(n) E0(n, c) (D A)(n) +
// w(n + e_c) E1(n + e_c, c) (D A)(n + e_c)
// (magnetostatics_onelab.hpp:1890-1945, 2355-2392).
__device__ __forceinline__ double gauge_div3(double const* a, double const* gd, int m, int i, int j, int k, int nx,
                                             int ny)
{
    double const* e = gd + 8 * m;
    double s = 0.0;
    s = s + e[0] * a[3 * m];
    if (i > 0) s = s + e[3] * a[3 * (m - 1)];
    s = s + e[1] * a[3 * m + 1];
    if (j > 0) s = s + e[4] * a[3 * (m - nx) + 1];
    s = s + e[2] * a[3 * m + 2];
    if (k > 0) s = s + e[5] * a[3 * (m - nx * ny) + 2];
    return s;
}

__device__ __forceinline__ double gauge_term3(double const* a, double const* gd, int n, int i, int j, int k, int nx,
                                              int ny, int c)
{
    int const step = c == 0 ? 1 : (c == 1 ? nx : nx * ny);
    int const m = n + step;
    double const div_n = gauge_div3(a, gd, n, i, j, k, nx, ny);
    double const div_m = gauge_div3(a, gd, m, i + (c == 0), j + (c == 1), k + (c == 2), nx, ny);
    double t = 0.0;
    t = t + gd[8 * n + 6] * gd[8 * n + c] * div_n;
    t = t + gd[8 * m + 6] * gd[8 * m + 3 + c] * div_m;
    return t;
}

// Curl moments of v at the interior sampled node s = (i, j, k), columns on
// the boundary dropped, in the stencils' order:
//   B_x = A_y(s) - A_z(s) - A_y(s+z) + A_z(s+y)
//   B_y = -A_x(s) + A_z(s) + A_x(s+z) - A_z(s+x)
//   B_z = A_x(s) - A_y(s) - A_x(s+y) + A_y(s+x)
__device__ __forceinline__ void moments3(Geo3 const& g, double const* v, int s, int i, int j, int k, double* B)
{
    int const b = 3 * s, oy = 3 * g.nx, oz = 3 * g.nx * g.ny;
    bool const ix = interior3(g, i + 1, j, k), iy = interior3(g, i, j + 1, k), iz = interior3(g, i, j, k + 1);
    double const ax = v[b], ay = v[b + 1], az = v[b + 2];
    double m = 0.0;
    m += ay;
    m -= az;
    if (iz) m -= v[b + oz + 1];
    if (iy) m += v[b + oy + 2];
    B[0] = m;
    m = 0.0;
    m -= ax;
    m += az;
    if (iz) m += v[b + oz];
    if (ix) m -= v[b + 3 + 2];
    B[1] = m;
    m = 0.0;
    m += ax;
    m -= ay;
    if (iy) m -= v[b + oy];
    if (ix) m += v[b + 3 + 1];
    B[2] = m;
}

__device__ __forceinline__ void hodge_b3(Geo3 const& g, int i, int j, int k, double* h)
{
    double const dx = g.ls[0][i], dy = g.ls[1][j], dz = g.ls[2][k];
    h[0] = dx / (dy * dz);
    h[1] = dy / (dx * dz);
    h[2] = dz / (dx * dy);
}

__device__ __forceinline__ void node_field3(DevCurve const& c, double mu, double ferro, double const* B, double* H)
{
    if (ferro > 0.5) {
        double const q = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
        double F, dF, d2F;
        curve_f(c, q, &F, &dF, &d2F);
        for (int m = 0; m < 3; ++m) H[m] = B[m] * F + q * B[m] * dF;
    } else {
        for (int m = 0; m < 3; ++m) H[m] = B[m] / mu;
    }
}

// J[3 r + c] = d2H / dB_r dB_c at a sampled node.
__device__ __forceinline__ void node_jacobian3(DevCurve const& c, double mu, double ferro, double const* B, double* J)
{
    if (ferro > 0.5) {
        double const q = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
        double F, dF, d2F;
        curve_f(c, q, &F, &dF, &d2F);
        double const base = F + q * dF;
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc)
                J[3 * r + cc] = (r == cc ? base : 0.0) + 4.0 * B[r] * B[cc] * dF + 2.0 * q * B[r] * B[cc] * d2F;
    } else {
        for (int r = 0; r < 3; ++r)
            for (int cc = 0; cc < 3; ++cc) J[3 * r + cc] = r == cc ? 1.0 / mu : 0.0;
    }
}

// hh[3 s + m] = hodge_m(s) H_m(B(s)) at interior sampled nodes, 0 elsewhere.
__global__ void __launch_bounds__(kBlock) nl3_field_kernel(const __grid_constant__ DevCurve curve, Geo3 g,
                                                           double const* a, double const* mu, double const* ferro,
                                                           double* hh)
{
    __shared__ DevCurve c;
    stage_curve(curve, c);
    int const nodes = g.nx * g.ny * g.nz;
    for (int s = blockIdx.x * kBlock + threadIdx.x; s < nodes; s += gridDim.x * kBlock) {
        int i, j, k;
        node_coords(g, s, &i, &j, &k);
        double* out = hh + 3 * s;
        if (!interior3(g, i, j, k)) {
            out[0] = 0.0;
            out[1] = 0.0;
            out[2] = 0.0;
            continue;
        }
        double B[3], H[3], h[3];
        moments3(g, a, s, i, j, k, B);
        node_field3(c, mu[s], ferro[s], B, H);
        hodge_b3(g, i, j, k, h);
        out[0] = h[0] * H[0];
        out[1] = h[1] * H[1];
        out[2] = h[2] * H[2];
    }
}

// kh[9 s + 3 m + c] = hodge_m(s) J_mc(B(s)) of the state at interior sampled
// nodes, 0 elsewhere.
__global__ void __launch_bounds__(kBlock) nl3_coef_kernel(const __grid_constant__ DevCurve curve, Geo3 g,
                                                          double const* st, double const* mu, double const* ferro,
                                                          double* kh)
{
    __shared__ DevCurve c;
    stage_curve(curve, c);
    int const nodes = g.nx * g.ny * g.nz;
    for (int s = blockIdx.x * kBlock + threadIdx.x; s < nodes; s += gridDim.x * kBlock) {
        int i, j, k;
        node_coords(g, s, &i, &j, &k);
        double* out = kh + 9 * s;
        if (!interior3(g, i, j, k)) {
            for (int e = 0; e < 9; ++e) out[e] = 0.0;
            continue;
        }
        double B[3], J[9], h[3];
        moments3(g, st, s, i, j, k, B);
        node_jacobian3(c, mu[s], ferro[s], B, J);
        hodge_b3(g, i, j, k, h);
        for (int m = 0; m < 3; ++m)
            for (int cc = 0; cc < 3; ++cc) out[3 * m + cc] = h[m] * J[3 * m + cc];
    }
}

// gv[3 s + m] = sum_c kh[9 s + 3 m + c] B_c(x)(s) at interior sampled nodes.
__global__ void __launch_bounds__(kBlock) nl3_jfield_kernel(Geo3 g, double const* kh, double const* x, double* gv,
                                                            CgState const* st)
{
    if (st != nullptr && st->done) return;
    int const nodes = g.nx * g.ny * g.nz;
    for (int s = blockIdx.x * kBlock + threadIdx.x; s < nodes; s += gridDim.x * kBlock) {
        int i, j, k;
        node_coords(g, s, &i, &j, &k);
        double* out = gv + 3 * s;
        if (!interior3(g, i, j, k)) {
            out[0] = 0.0;
            out[1] = 0.0;
            out[2] = 0.0;
            continue;
        }
        double D[3];
        moments3(g, x, s, i, j, k, D);
        double const* K = kh + 9 * s;
        for (int m = 0; m < 3; ++m) out[m] = K[3 * m] * D[0] + K[3 * m + 1] * D[1] + K[3 * m + 2] * D[2];
    }
}

// Per row: the gather of the per-node values hv (+- by the moment
// stencils' coefficients) plus the penalty gauge on v; v[row] on the
// boundary.  MODE 0: out = f.  MODE 1: out = rhs - f, partial sums of
// out^2.  MODE 2 (CG step): out = f, partial sums of v . out; skipped once
// the CG state is done.
template <int MODE>
__global__ void __launch_bounds__(kBlock) nl3_gather_kernel(Geo3 g, double const* hv, double const* v,
                                                            double const* rhs, double* out, double* part,
                                                            CgState const* st)
{
    __shared__ double red[kBlock / 32];
    if (MODE == 2 && st->done) return;
    int const nodes = g.nx * g.ny * g.nz;
    int const nrows = 3 * nodes;
    int const oy = 3 * g.nx, oz = 3 * g.nx * g.ny;
    double acc = 0.0;
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < nrows; row += gridDim.x * kBlock) {
        int const s = row / 3, c = row - 3 * s;
        int i, j, k;
        node_coords(g, s, &i, &j, &k);
        double f;
        if (!interior3(g, i, j, k)) {
            f = v[row];
        } else {
            int const b = 3 * s;
            double const dx = g.ls[0][i], dy = g.ls[1][j], dz = g.ls[2][k];
            double r = 0.0, ha;
            if (c == 0) {
                if (k > 1) r += hv[b - oz + 1];
                if (j > 1) r -= hv[b - oy + 2];
                r -= hv[b + 1];
                r += hv[b + 2];
                ha = dy * dz / dx;
            } else if (c == 1) {
                if (k > 1) r -= hv[b - oz];
                if (i > 1) r += hv[b - 3 + 2];
                r += hv[b];
                r -= hv[b + 2];
                ha = dx * dz / dy;
            } else {
                if (j > 1) r += hv[b - oy];
                if (i > 1) r -= hv[b - 3 + 1];
                r -= hv[b];
                r += hv[b + 1];
                ha = dx * dy / dz;
            }
            if (g.gauge) f = r + g.gamma * gauge_term3(v, g.gd, s, i, j, k, g.nx, g.ny, c);
            else f = __dadd_rn(r, __dmul_rn(__dmul_rn(g.gamma, ha), v[row]));
        }
        if (MODE == 1) {
            double const rv = rhs[row] - f;
            out[row] = rv;
            acc += rv * rv;
        } else {
            out[row] = f;
            if (MODE == 2) acc += v[row] * f;
        }
    }
    if (MODE != 0) {
        double const t = block_sum(acc, red);
        if (threadIdx.x == 0) part[blockIdx.x] = t;
    }
}

// Inverse Jacobian diagonal from the weighted coefficients: for each entry
// of the row, the row's own coefficient in the sampled node's moments times
// that node's weighted Jacobian row; plus the gauge; 1 on the boundary.
__global__ void __launch_bounds__(kBlock) nl3_dinv_kernel(Geo3 g, double const* kh, double* dinv)
{
    int const nodes = g.nx * g.ny * g.nz;
    int const nrows = 3 * nodes;
    int const oy = 9 * g.nx, oz = 9 * g.nx * g.ny;
    for (int row = blockIdx.x * kBlock + threadIdx.x; row < nrows; row += gridDim.x * kBlock) {
        int const s = row / 3, c = row - 3 * s;
        int i, j, k;
        node_coords(g, s, &i, &j, &k);
        if (!interior3(g, i, j, k)) {
            dinv[row] = 1.0;
            continue;
        }
        double const* K = kh + 9 * s;
        double const dx = g.ls[0][i], dy = g.ls[1][j], dz = g.ls[2][k];
        double d = 0.0, ha;
        if (c == 0) {
            if (k > 1) d += K[-oz + 4];
            if (j > 1) d += K[-oy + 8];
            d += K[4] - K[5] - K[7] + K[8];
            ha = dy * dz / dx;
        } else if (c == 1) {
            if (k > 1) d += K[-oz + 0];
            if (i > 1) d += K[-9 + 8];
            d += K[0] - K[2] - K[6] + K[8];
            ha = dx * dz / dy;
        } else {
            if (j > 1) d += K[-oy + 0];
            if (i > 1) d += K[-9 + 4];
            d += K[0] - K[1] - K[3] + K[4];
            ha = dx * dy / dz;
        }
        if (g.gauge) {
            int const step = c == 0 ? 1 : (c == 1 ? g.nx : g.nx * g.ny);
            double const e0 = g.gd[8 * s + c], e1 = g.gd[8 * (s + step) + 3 + c];
            double const gdiv = g.gd[8 * s + 6] * e0 * e0 + g.gd[8 * (s + step) + 6] * e1 * e1;
            dinv[row] = 1.0 / (d + g.gamma * gdiv);
        } else {
            dinv[row] = 1.0 / (d + g.gamma * ha);
        }
    }
}

// ---------------------------------------------------------------- host side

sil_status make_curve(sil_bh_curve const& in, DevCurve* out)
{
    if (in.n < 2 || in.n > kMaxCurve) return fail(SIL_ERR_INVALID, "B-H curve: 2 to 64 samples");
    if (in.b == nullptr || in.h == nullptr) return fail(SIL_ERR_INVALID, "B-H curve: NULL sample array");
    *out = DevCurve {};
    out->n = in.n;
    for (int i = 0; i < in.n; ++i) {
        if (!std::isfinite(in.b[i]) || !std::isfinite(in.h[i])) return fail(SIL_ERR_INVALID, "B-H curve: non-finite sample");
        if (i > 0 && !(in.b[i] > in.b[i - 1])) return fail(SIL_ERR_INVALID, "B-H curve: b must increase strictly");
        out->b[i] = in.b[i];
        out->h[i] = in.h[i];
        out->q[i] = in.b[i] * in.b[i];
    }
    if (in.b[0] < 0.0) return fail(SIL_ERR_INVALID, "B-H curve: b[0] must be >= 0");
    for (int i = 0; i + 1 < in.n; ++i) out->dh_db[i] = (in.h[i + 1] - in.h[i]) / (in.b[i + 1] - in.b[i]);
    return SIL_OK;
}

sil_status check_problem(sil_mag2d_nl_problem const& p, char const* who)
{
    if (p.nx < 3 || p.ny < 3) return fail(SIL_ERR_INVALID, std::string(who) + ": need at least 3x3 nodes");
    if (p.nx * p.ny >= (int64_t(1) << 31)) return fail(SIL_ERR_INVALID, std::string(who) + ": fewer than 2^31 nodes supported");
    if (p.node_mu == nullptr || p.node_ferro == nullptr) return fail(SIL_ERR_INVALID, std::string(who) + ": NULL material array");
    return SIL_OK;
}

unsigned grid_for(int64_t n)
{
    // initialised once, thread-safely (the nonlinear batches call this from
    // several host threads)
    static int const sms = [] {
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev);
        return count > 0 ? count : 148;
    }();
    int64_t const blocks = (n + kBlock - 1) / kBlock;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, 4 * sms)));
}

sil_status check_problem3(sil_mag3d_nl_problem const& p, char const* who, bool need_fields)
{
    std::string const w(who);
    if (p.nx < 3 || p.ny < 3 || p.nz < 3) return fail(SIL_ERR_INVALID, w + ": need at least 3x3x3 nodes");
    // the kernels index the 9 Jacobian coefficients of a node with int
    if (9 * p.nx * p.ny * p.nz >= (int64_t(1) << 31))
        return fail(SIL_ERR_INVALID, w + ": fewer than 2^31 / 9 nodes per problem supported");
    if (p.x == nullptr || p.y == nullptr || p.z == nullptr) return fail(SIL_ERR_INVALID, w + ": NULL coordinate array");
    if (p.node_mu == nullptr || p.node_ferro == nullptr) return fail(SIL_ERR_INVALID, w + ": NULL material array");
    if (need_fields && (p.rhs == nullptr || p.solution == nullptr)) return fail(SIL_ERR_INVALID, w + ": NULL field pointer");
    if (p.gauge != 0 && p.gauge != 1) return fail(SIL_ERR_INVALID, w + ": gauge must be 0 or 1");
    if (!std::isfinite(p.gauge_penalty) || (p.gauge == 0 ? !(p.gauge_penalty > 0.0) : p.gauge_penalty == 0.0))
        return fail(SIL_ERR_INVALID, w + ": gauge_penalty must be finite and positive (nonzero for the divergence gauge)");
    double const* c[3] = {p.x, p.y, p.z};
    int64_t const len[3] = {p.nx, p.ny, p.nz};
    for (int a = 0; a < 3; ++a)
        for (int64_t i = 0; i + 1 < len[a]; ++i)
            if (!(c[a][i + 1] > c[a][i])) return fail(SIL_ERR_INVALID, w + ": node coordinates must increase strictly");
    return SIL_OK;
}

// The reference's local spacing per axis (one-sided at the ends, central
// average inside; magnetostatics_onelab.hpp:856-870), axes concatenated.
std::vector<double> local_spacings(sil_mag3d_nl_problem const& p)
{
    double const* c[3] = {p.x, p.y, p.z};
    int64_t const len[3] = {p.nx, p.ny, p.nz};
    std::vector<double> out;
    for (int a = 0; a < 3; ++a)
        for (int64_t i = 0; i < len[a]; ++i) {
            int64_t const n = len[a];
            double v;
            if (i == 0) v = c[a][1] - c[a][0];
            else if (i + 1 == n) v = c[a][n - 1] - c[a][n - 2];
            else v = 0.5 * (c[a][i + 1] - c[a][i - 1]);
            out.push_back(v);
        }
    return out;
}

Geo3 make_geo3(sil_mag3d_nl_problem const& p, double const* dls, double const* gd = nullptr)
{
    Geo3 g {};
    g.gauge = p.gauge;
    g.gd = gd;
    g.nx = static_cast<int>(p.nx);
    g.ny = static_cast<int>(p.ny);
    g.nz = static_cast<int>(p.nz);
    g.gamma = p.gauge_penalty;
    g.ls[0] = dls;
    g.ls[1] = dls + p.nx;
    g.ls[2] = dls + p.nx + p.ny;
    return g;
}

// The divergence-gauge table of a problem into gd (8 per node); scratch: 4
// doubles per node.
sil_status gauge_table3(sil_mag3d_nl_problem const& p, double const* dls, double* gd, double* scratch,
                        cudaStream_t st)
{
    int64_t const nodes = p.nx * p.ny * p.nz;
    double const* coords[3] = {p.x, p.y, p.z};
    return divergence_gauge_table(p.nx, p.ny, p.nz, coords, dls, gd, scratch, scratch + 3 * nodes, st);
}

// Stream-ordered device allocation, freed in stream order.
struct AsyncBuffer
{
    void* ptr = nullptr;
    cudaStream_t s = nullptr;
    bool sync = false;  // wait for the free (a stream the buffer's owner destroys next)
    ~AsyncBuffer()
    {
        if (ptr != nullptr) {
            cudaFreeAsync(ptr, s);
            if (sync) cudaStreamSynchronize(s);
        }
    }
};

// Up to kConcurrent problems at a time, each on a host thread with its own
// stream (one problem's CG kernels are small and launch bound, so several
// problems together fill the GPU).
template <class Solve>
sil_status run_concurrent(int nproblems, Solve const& solve)
{
    (void)grid_for(1);  // device attributes read on the calling thread's device
    int dev = 0;
    SIL_CUDA_CHECK(cudaGetDevice(&dev));
    constexpr int kConcurrent = 8;
    std::vector<sil_status> status(nproblems, SIL_OK);
    std::vector<std::string> message(nproblems);
    for (int first = 0; first < nproblems; first += kConcurrent) {
        int const last = std::min(nproblems, first + kConcurrent);
        std::vector<std::thread> workers;
        for (int p = first; p < last; ++p) {
            workers.emplace_back([&, p] {
                cudaSetDevice(dev);
                status[p] = solve(p);
                if (status[p] != SIL_OK) message[p] = sil_last_error();
            });
        }
        for (auto& w : workers) w.join();
    }
    for (int p = 0; p < nproblems; ++p)
        if (status[p] != SIL_OK) return fail(status[p], message[p]);
    return SIL_OK;
}

}  // namespace
}  // namespace sil

using namespace sil;

sil_status sil_mag2d_nl_apply(sil_stream stream, const sil_mag2d_nl_problem* problem, const double* a, double* y)
{
    if (problem == nullptr || a == nullptr || y == nullptr) return fail(SIL_ERR_INVALID, "sil_mag2d_nl_apply: NULL argument");
    if (sil_status s = check_problem(*problem, "sil_mag2d_nl_apply"); s != SIL_OK) return s;
    DevCurve c;
    if (sil_status s = make_curve(problem->curve, &c); s != SIL_OK) return s;
    Geo const g {static_cast<int>(problem->nx), static_cast<int>(problem->ny)};
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    nl_apply_kernel<<<grid_for(problem->nx * problem->ny), kBlock, 0, st>>>(c, g, a, problem->node_mu,
                                                                              problem->node_ferro, nullptr, y, nullptr);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status sil_mag2d_nl_apply_jacobian(sil_stream stream, const sil_mag2d_nl_problem* problem, const double* state,
                                       const double* x, double* y)
{
    if (problem == nullptr || state == nullptr || x == nullptr || y == nullptr)
        return fail(SIL_ERR_INVALID, "sil_mag2d_nl_apply_jacobian: NULL argument");
    if (sil_status s = check_problem(*problem, "sil_mag2d_nl_apply_jacobian"); s != SIL_OK) return s;
    DevCurve c;
    if (sil_status s = make_curve(problem->curve, &c); s != SIL_OK) return s;
    Geo const g {static_cast<int>(problem->nx), static_cast<int>(problem->ny)};
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    nl_jacobian_kernel<<<grid_for(problem->nx * problem->ny), kBlock, 0, st>>>(c, g, state, problem->node_mu,
                                                                                 problem->node_ferro, x, y);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

namespace sil {
namespace {

// One linear solve of a Newton step with a menu preconditioner: the Jacobian
// assembled at x, the preconditioner built on it, CG for d from 0.
template <class Ops>
sil_status menu_step(Ops const& ops, sil_menu_settings const& menu, cudaStream_t st, double const* x,
                     double const* r, double* d, double tol, int max_iter, int* iterations)
{
    sil_csr J = nullptr;
    if (sil_status s = ops.assemble_jacobian(st, x, &J); s != SIL_OK) return s;
    sil_csr_precond pc = nullptr;
    sil_status s = sil_csr_precond_create(st, J, &menu, &pc);
    if (s == SIL_OK) {
        sil_solve_settings ls {};
        ls.max_iterations = max_iter;
        ls.relative_tolerance = tol;
        sil_solve_diagnostics ld {};
        s = sil_csr_solve(st, J, pc, r, d, &ls, &ld);
        *iterations = ld.iterations;
        sil_csr_precond_destroy(pc);
    }
    sil_csr_destroy(J);
    return s;
}

// Newton with the line search for one problem on stream st.  v: nine
// vectors of ops.n doubles (r, cand_r, cand, d, cr, z, p, q, dinv); part:
// 2 * ops.G doubles.  Ops supplies
//   residual(s, val, out, part):   out = rhs - F(val), ops.G partials of out^2
//   jacobian_setup(s, x, dinv):    Jacobian coefficients at x, inverse diagonal
//   cg_product(s, p, q, part, cg): q = J p, ops.G partials of p.q, no work once
//                                  the CG state is done
template <class Ops>
sil_status newton(Ops const& ops, double* x, double* const* v, double* part, double* d_norm, CgState* d_cg,
                  cudaStream_t st, double tol, int max_iter, sil_solve_diagnostics& D,
                  sil_menu_settings const* menu = nullptr)
{
    double *r = v[0], *cand_r = v[1], *cand = v[2], *dvec = v[3], *cr = v[4], *z = v[5], *pv = v[6], *qv = v[7],
           *dinv = v[8];
    D = sil_solve_diagnostics {};
    int const n = static_cast<int>(ops.n);
    unsigned const G = ops.G;
    // residual norm of rhs - F(val) into out (returned on the host)
    auto residual = [&](double const* val, double* out, double* norm) -> sil_status {
        ops.residual(st, val, out, part);
        norm_finish_kernel<<<1, kBlock, 0, st>>>(part, static_cast<int>(G), d_norm);
        SIL_CUDA_CHECK(cudaGetLastError());
        SIL_CUDA_CHECK(cudaMemcpyAsync(norm, d_norm, sizeof(double), cudaMemcpyDeviceToHost, st));
        SIL_CUDA_CHECK(cudaStreamSynchronize(st));
        return SIL_OK;
    };
    double res = 0.0;
    if (sil_status s = residual(x, r, &res); s != SIL_OK) return s;
    double const r0 = res;
    D.initial_residual_l2 = r0;
    D.status = SIL_OK;
    if (!std::isfinite(r0)) {
        D.status = SIL_ERR_NONFINITE;
        D.final_residual_l2 = r0;
        D.final_relative_residual = r0;
        return SIL_OK;
    }
    if (r0 == 0.0) {
        D.converged = 1;
        return SIL_OK;
    }
    // 16 CG iterations captured once per problem (the kernels stop doing
    // work once the state is marked done) and replayed until convergence;
    // not needed when a menu preconditioner runs the linear solves.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    if (menu == nullptr) {
        cudaStream_t cs;
        SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
        for (int c = 0; c < 16 && err == cudaSuccess; ++c) {
            ops.cg_product(cs, pv, qv, part, d_cg);
            cg_alpha_kernel<<<1, kBlock, 0, cs>>>(part, static_cast<int>(G), d_cg);
            cg_update_kernel<<<G, kBlock, 0, cs>>>(n, dvec, cr, pv, qv, dinv, z, part, d_cg);
            cg_beta_kernel<<<1, kBlock, 0, cs>>>(part, static_cast<int>(G), d_cg, tol, max_iter);
            cg_direction_kernel<<<G, kBlock, 0, cs>>>(n, pv, z, d_cg);
        }
        cudaError_t const err2 = cudaStreamEndCapture(cs, &graph);
        if (err == cudaSuccess) err = err2;
        if (err == cudaSuccess) err = cudaGraphInstantiate(&exec, graph, 0);
        cudaStreamDestroy(cs);
        if (err != cudaSuccess) {
            if (graph != nullptr) cudaGraphDestroy(graph);
            return cuda_fail(err, "nonlinear CG graph capture");
        }
    }
    struct GraphGuard
    {
        cudaGraph_t g;
        cudaGraphExec_t e;
        ~GraphGuard()
        {
            if (e != nullptr) cudaGraphExecDestroy(e);
            if (g != nullptr) cudaGraphDestroy(g);
        }
    } guard {graph, exec};
    int cg_total = 0, steps = 0;
    for (int it = 0; it < 30; ++it) {
        if (res / r0 <= tol) break;
        ++steps;
        if (menu != nullptr) {
            int its = 0;
            if (sil_status s = menu_step(ops, *menu, st, x, r, dvec, tol, max_iter, &its); s != SIL_OK) return s;
            cg_total += its;
        } else {
            ops.jacobian_setup(st, x, dinv);
            cg_start_kernel<<<G, kBlock, 0, st>>>(n, r, dinv, dvec, cr, z, pv, part);
            cg_init_kernel<<<1, kBlock, 0, st>>>(part, static_cast<int>(G), d_cg, tol, max_iter);
            SIL_CUDA_CHECK(cudaGetLastError());
            CgState hs {};
            for (;;) {
                SIL_CUDA_CHECK(cudaGraphLaunch(exec, st));
                SIL_CUDA_CHECK(cudaMemcpyAsync(&hs, d_cg, sizeof(CgState), cudaMemcpyDeviceToHost, st));
                SIL_CUDA_CHECK(cudaStreamSynchronize(st));
                if (hs.done) break;
            }
            cg_total += hs.iters;
        }
        // line search
        double const cur = res;
        double alpha = 1.0, best_alpha = 0.0, best = std::numeric_limits<double>::infinity(), nr = 0.0;
        for (int ls = 0; ls < 8; ++ls) {
            axpy_kernel<<<G, kBlock, 0, st>>>(n, x, alpha, dvec, cand);
            if (sil_status s = residual(cand, cand_r, &nr); s != SIL_OK) return s;
            if (nr < best) {
                best = nr;
                best_alpha = alpha;
            }
            if (nr < cur) break;
            alpha *= 0.5;
        }
        if (best_alpha != alpha) {
            alpha = best_alpha;
            axpy_kernel<<<G, kBlock, 0, st>>>(n, x, alpha, dvec, cand);
            if (sil_status s = residual(cand, cand_r, &nr); s != SIL_OK) return s;
        }
        SIL_CUDA_CHECK(cudaMemcpyAsync(x, cand, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        std::swap(r, cand_r);
        res = nr;
        if (!std::isfinite(res)) break;
    }
    D.iterations = cg_total;
    D.refinements = steps;
    D.final_residual_l2 = res;
    D.final_relative_residual = res / r0;
    D.converged = (res / r0 <= tol) ? 1 : 0;
    if (!std::isfinite(res)) D.status = SIL_ERR_NONFINITE;
    return SIL_OK;
}

struct Ops2
{
    DevCurve const& C;
    Geo g;
    sil_mag2d_nl_problem const& P;
    double *c00, *c01, *c11;
    int64_t n;
    unsigned G;
    void residual(cudaStream_t s, double const* val, double* out, double* part) const
    {
        nl_apply_kernel<<<G, kBlock, 0, s>>>(C, g, val, P.node_mu, P.node_ferro, P.rhs, out, part);
    }
    void jacobian_setup(cudaStream_t s, double const* x, double* dinv) const
    {
        nl_coef_kernel<<<G, kBlock, 0, s>>>(C, g, x, P.node_mu, P.node_ferro, c00, c01, c11);
        nl_dinv_kernel<<<G, kBlock, 0, s>>>(g, c00, c01, c11, dinv);
    }
    void cg_product(cudaStream_t s, double const* p, double* q, double* part, CgState const* cg) const
    {
        cg_jac_kernel<<<G, kBlock, 0, s>>>(g, c00, c01, c11, p, q, part, cg);
    }
    sil_status assemble_jacobian(cudaStream_t s, double const* x, sil_csr* out) const
    {
        return sil_mag2d_nl_assemble_jacobian(s, &P, x, out);
    }
};

struct Ops3
{
    DevCurve const& C;
    Geo3 g;
    sil_mag3d_nl_problem const& P;
    double* hv;  // 3 per node: the weighted field, or the Jacobian's image in CG
    double* kh;  // 9 per node: weighted Jacobian coefficients
    int64_t n;   // rows: 3 per node
    unsigned G;  // grid of the row and vector kernels
    unsigned Gn; // grid of the node kernels
    void residual(cudaStream_t s, double const* val, double* out, double* part) const
    {
        nl3_field_kernel<<<Gn, kBlock, 0, s>>>(C, g, val, P.node_mu, P.node_ferro, hv);
        nl3_gather_kernel<1><<<G, kBlock, 0, s>>>(g, hv, val, P.rhs, out, part, nullptr);
    }
    void jacobian_setup(cudaStream_t s, double const* x, double* dinv) const
    {
        nl3_coef_kernel<<<Gn, kBlock, 0, s>>>(C, g, x, P.node_mu, P.node_ferro, kh);
        nl3_dinv_kernel<<<G, kBlock, 0, s>>>(g, kh, dinv);
    }
    void cg_product(cudaStream_t s, double const* p, double* q, double* part, CgState const* cg) const
    {
        nl3_jfield_kernel<<<Gn, kBlock, 0, s>>>(g, kh, p, hv, cg);
        nl3_gather_kernel<2><<<G, kBlock, 0, s>>>(g, hv, p, nullptr, q, part, cg);
    }
    sil_status assemble_jacobian(cudaStream_t s, double const* x, sil_csr* out) const
    {
        return sil_mag3d_nl_assemble_jacobian(s, &P, x, out);
    }
};

size_t round256(size_t b) { return (b + 255) / 256 * 256; }

// One problem's Newton solve on its own stream and buffers (the problems of
// a batch run on concurrent host threads).  extra: doubles of the problem's
// own work arrays after the nine Newton vectors.
struct Workspace
{
    struct StreamGuard
    {
        cudaStream_t s = nullptr;
        ~StreamGuard()
        {
            if (s != nullptr) cudaStreamDestroy(s);
        }
    } sg;
    AsyncBuffer buf;
    double* v[9];
    double* part;
    double* d_norm;
    CgState* d_cg;
    double* extra;

    sil_status init(int64_t n, unsigned G, size_t extra_doubles)
    {
        SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking));
        buf.s = sg.s;
        buf.sync = true;
        size_t const vbytes = round256(static_cast<size_t>(n) * sizeof(double));
        size_t const pbytes = round256(2 * static_cast<size_t>(G) * sizeof(double));
        size_t const ebytes = round256(extra_doubles * sizeof(double));
        SIL_CUDA_CHECK(cudaMallocAsync(&buf.ptr, 9 * vbytes + pbytes + 2 * 256 + ebytes, sg.s));
        char* base = static_cast<char*>(buf.ptr);
        for (int k = 0; k < 9; ++k) v[k] = reinterpret_cast<double*>(base + k * vbytes);
        part = reinterpret_cast<double*>(base + 9 * vbytes);
        d_norm = reinterpret_cast<double*>(base + 9 * vbytes + pbytes);
        d_cg = reinterpret_cast<CgState*>(base + 9 * vbytes + pbytes + 256);
        extra = reinterpret_cast<double*>(base + 9 * vbytes + pbytes + 2 * 256);
        return SIL_OK;
    }
};

sil_status solve_one(sil_mag2d_nl_problem const& P, DevCurve const& C, double tol, int max_iter,
                     sil_solve_diagnostics& D, sil_menu_settings const* menu)
{
    int64_t const n = P.nx * P.ny;
    unsigned const G = grid_for(n);
    size_t const vb = round256(static_cast<size_t>(n) * sizeof(double)) / sizeof(double);
    Workspace w;
    if (sil_status s = w.init(n, G, 3 * vb); s != SIL_OK) return s;
    Ops2 const ops {C, Geo {static_cast<int>(P.nx), static_cast<int>(P.ny)}, P, w.extra, w.extra + vb,
                    w.extra + 2 * vb, n, G};
    if (sil_status s = newton(ops, P.solution, w.v, w.part, w.d_norm, w.d_cg, w.sg.s, tol, max_iter, D, menu);
        s != SIL_OK)
        return s;
    SIL_CUDA_CHECK(cudaStreamSynchronize(w.sg.s));
    return SIL_OK;
}

sil_status solve_one3(sil_mag3d_nl_problem const& P, DevCurve const& C, double tol, int max_iter,
                      sil_solve_diagnostics& D, sil_menu_settings const* menu)
{
    int64_t const nodes = P.nx * P.ny * P.nz;
    int64_t const n = 3 * nodes;
    unsigned const G = grid_for(n);
    std::vector<double> const sp = local_spacings(P);
    size_t const hb = round256(static_cast<size_t>(3 * nodes) * sizeof(double)) / sizeof(double);
    size_t const kb = round256(static_cast<size_t>(9 * nodes) * sizeof(double)) / sizeof(double);
    // divergence gauge: its table (8 per node) and the builder's scratch (4 per node)
    size_t const gb = P.gauge ? round256(static_cast<size_t>(12 * nodes) * sizeof(double)) / sizeof(double) : 0;
    Workspace w;
    if (sil_status s = w.init(n, G, hb + kb + gb + sp.size()); s != SIL_OK) return s;
    double* gd = P.gauge ? w.extra + hb + kb : nullptr;
    double* dls = w.extra + hb + kb + gb;
    SIL_CUDA_CHECK(cudaMemcpyAsync(dls, sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, w.sg.s));
    if (P.gauge)
        if (sil_status s = gauge_table3(P, dls, gd, gd + 8 * nodes, w.sg.s); s != SIL_OK) return s;
    Ops3 const ops {C, make_geo3(P, dls, gd), P, w.extra, w.extra + hb, n, G, grid_for(nodes)};
    if (sil_status s = newton(ops, P.solution, w.v, w.part, w.d_norm, w.d_cg, w.sg.s, tol, max_iter, D, menu);
        s != SIL_OK)
        return s;
    SIL_CUDA_CHECK(cudaStreamSynchronize(w.sg.s));
    return SIL_OK;
}

}  // namespace
}  // namespace sil

using namespace sil;

sil_status sil_mag2d_nl_solve_batch(const sil_mag2d_nl_problem* problems, int nproblems,
                                    const sil_solve_settings* settings, sil_solve_diagnostics* diag,
                                    sil_stream stream)
{
    if (problems == nullptr || settings == nullptr || diag == nullptr || nproblems <= 0)
        return fail(SIL_ERR_INVALID, "sil_mag2d_nl_solve_batch: NULL argument or empty batch");
    std::vector<DevCurve> curves(nproblems);
    for (int p = 0; p < nproblems; ++p) {
        sil_mag2d_nl_problem const& q = problems[p];
        if (sil_status s = check_problem(q, "sil_mag2d_nl_solve_batch"); s != SIL_OK) return s;
        if (q.rhs == nullptr || q.solution == nullptr) return fail(SIL_ERR_INVALID, "sil_mag2d_nl_solve_batch: NULL field pointer");
        if (sil_status s = make_curve(q.curve, &curves[p]); s != SIL_OK) return s;
    }
    double const tol = settings->relative_tolerance > 0 ? settings->relative_tolerance : 1e-10;
    int const max_iter = settings->max_iterations > 0 ? settings->max_iterations : 100000;
    // the inputs come from the caller's stream
    SIL_CUDA_CHECK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    sil_menu_settings const* menu = settings->jacobian_preconditioner;
    return run_concurrent(nproblems,
                          [&](int p) { return solve_one(problems[p], curves[p], tol, max_iter, diag[p], menu); });
}

namespace {

sil_status nl3_prepare(sil_mag3d_nl_problem const* problem, char const* who, DevCurve* c)
{
    if (sil_status s = check_problem3(*problem, who, false); s != SIL_OK) return s;
    return make_curve(problem->curve, c);
}

}  // namespace

sil_status sil_mag3d_nl_apply(sil_stream stream, const sil_mag3d_nl_problem* problem, const double* a, double* y)
{
    if (problem == nullptr || a == nullptr || y == nullptr) return fail(SIL_ERR_INVALID, "sil_mag3d_nl_apply: NULL argument");
    DevCurve c;
    if (sil_status s = nl3_prepare(problem, "sil_mag3d_nl_apply", &c); s != SIL_OK) return s;
    sil_mag3d_nl_problem const& P = *problem;
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    int64_t const nodes = P.nx * P.ny * P.nz;
    std::vector<double> const sp = local_spacings(P);
    size_t const hb = round256(static_cast<size_t>(3 * nodes) * sizeof(double));
    size_t const gb = P.gauge ? round256(static_cast<size_t>(12 * nodes) * sizeof(double)) : 0;
    AsyncBuffer buf {nullptr, st, false};
    SIL_CUDA_CHECK(cudaMallocAsync(&buf.ptr, hb + gb + sp.size() * sizeof(double), st));
    double* hv = static_cast<double*>(buf.ptr);
    double* gd = P.gauge ? reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + hb) : nullptr;
    double* dls = reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + hb + gb);
    // a copy from pageable memory has left the host table once it returns
    SIL_CUDA_CHECK(cudaMemcpyAsync(dls, sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    if (P.gauge)
        if (sil_status s = gauge_table3(P, dls, gd, gd + 8 * nodes, st); s != SIL_OK) return s;
    Geo3 const g = make_geo3(P, dls, gd);
    nl3_field_kernel<<<grid_for(nodes), kBlock, 0, st>>>(c, g, a, P.node_mu, P.node_ferro, hv);
    nl3_gather_kernel<0><<<grid_for(3 * nodes), kBlock, 0, st>>>(g, hv, a, nullptr, y, nullptr, nullptr);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status sil_mag3d_nl_apply_jacobian(sil_stream stream, const sil_mag3d_nl_problem* problem, const double* state,
                                       const double* x, double* y)
{
    if (problem == nullptr || state == nullptr || x == nullptr || y == nullptr)
        return fail(SIL_ERR_INVALID, "sil_mag3d_nl_apply_jacobian: NULL argument");
    DevCurve c;
    if (sil_status s = nl3_prepare(problem, "sil_mag3d_nl_apply_jacobian", &c); s != SIL_OK) return s;
    sil_mag3d_nl_problem const& P = *problem;
    cudaStream_t const st = static_cast<cudaStream_t>(stream);
    int64_t const nodes = P.nx * P.ny * P.nz;
    std::vector<double> const sp = local_spacings(P);
    size_t const hb = round256(static_cast<size_t>(3 * nodes) * sizeof(double));
    size_t const kb = round256(static_cast<size_t>(9 * nodes) * sizeof(double));
    size_t const gb = P.gauge ? round256(static_cast<size_t>(12 * nodes) * sizeof(double)) : 0;
    AsyncBuffer buf {nullptr, st, false};
    SIL_CUDA_CHECK(cudaMallocAsync(&buf.ptr, hb + kb + gb + sp.size() * sizeof(double), st));
    double* hv = static_cast<double*>(buf.ptr);
    double* kh = reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + hb);
    double* gd = P.gauge ? reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + hb + kb) : nullptr;
    double* dls = reinterpret_cast<double*>(static_cast<char*>(buf.ptr) + hb + kb + gb);
    SIL_CUDA_CHECK(cudaMemcpyAsync(dls, sp.data(), sp.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    if (P.gauge)
        if (sil_status s = gauge_table3(P, dls, gd, gd + 8 * nodes, st); s != SIL_OK) return s;
    Geo3 const g = make_geo3(P, dls, gd);
    unsigned const gn = grid_for(nodes);
    nl3_coef_kernel<<<gn, kBlock, 0, st>>>(c, g, state, P.node_mu, P.node_ferro, kh);
    nl3_jfield_kernel<<<gn, kBlock, 0, st>>>(g, kh, x, hv, nullptr);
    nl3_gather_kernel<0><<<grid_for(3 * nodes), kBlock, 0, st>>>(g, hv, x, nullptr, y, nullptr, nullptr);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status sil_mag3d_nl_solve_batch(const sil_mag3d_nl_problem* problems, int nproblems,
                                    const sil_solve_settings* settings, sil_solve_diagnostics* diag,
                                    sil_stream stream)
{
    if (problems == nullptr || settings == nullptr || diag == nullptr || nproblems <= 0)
        return fail(SIL_ERR_INVALID, "sil_mag3d_nl_solve_batch: NULL argument or empty batch");
    std::vector<DevCurve> curves(nproblems);
    for (int p = 0; p < nproblems; ++p) {
        if (sil_status s = check_problem3(problems[p], "sil_mag3d_nl_solve_batch", true); s != SIL_OK) return s;
        if (sil_status s = make_curve(problems[p].curve, &curves[p]); s != SIL_OK) return s;
    }
    double const tol = settings->relative_tolerance > 0 ? settings->relative_tolerance : 1e-10;
    int const max_iter = settings->max_iterations > 0 ? settings->max_iterations : 100000;
    // the inputs come from the caller's stream
    SIL_CUDA_CHECK(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    sil_menu_settings const* menu = settings->jacobian_preconditioner;
    return run_concurrent(nproblems,
                          [&](int p) { return solve_one3(problems[p], curves[p], tol, max_iter, diag[p], menu); });
}
