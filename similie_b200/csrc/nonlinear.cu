// nonlinear.cu -- 2D magnetostatics with a saturating ferromagnetic
// material: the nonlinear residual operator, its Jacobian, and the Newton
// solve with a line search whose linear systems are solved by Jacobi-CG on
// the Jacobian (FP64).
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
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    int64_t const blocks = (n + kBlock - 1) / kBlock;
    return static_cast<unsigned>(std::max<int64_t>(1, std::min<int64_t>(blocks, 4 * sms)));
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

// One problem's Newton solve on its own stream and buffers (the problems of
// a batch run on concurrent host threads).
sil_status solve_one(sil_mag2d_nl_problem const& P, DevCurve const& C, double tol, int max_iter,
                     sil_solve_diagnostics& D)
{
    int64_t const maxn = P.nx * P.ny;
    // r, cand_r, cand, d, cr, z, p, q, dinv, c00, c01, c11 + partials + scalars
    int const nvec = 12;
    size_t const vbytes = ((static_cast<size_t>(maxn) * sizeof(double) + 255) / 256) * 256;
    unsigned const gmax = grid_for(maxn);
    size_t const pbytes = ((2 * static_cast<size_t>(gmax) * sizeof(double) + 255) / 256) * 256;
    struct StreamGuard
    {
        cudaStream_t s = nullptr;
        ~StreamGuard()
        {
            if (s != nullptr) cudaStreamDestroy(s);
        }
    } sg;
    SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&sg.s, cudaStreamNonBlocking));
    cudaStream_t const st = sg.s;
    // stream-ordered allocation: freeing does not synchronise the other
    // problems' streams
    struct AsyncBuffer
    {
        void* ptr = nullptr;
        cudaStream_t s;
        ~AsyncBuffer()
        {
            if (ptr != nullptr) {
                cudaFreeAsync(ptr, s);
                cudaStreamSynchronize(s);
            }
        }
    } buf {nullptr, st};
    SIL_CUDA_CHECK(cudaMallocAsync(&buf.ptr, nvec * vbytes + pbytes + 2 * 256, st));
    char* base = static_cast<char*>(buf.ptr);
    double* v[nvec];
    for (int k = 0; k < nvec; ++k) v[k] = reinterpret_cast<double*>(base + k * vbytes);
    double* part = reinterpret_cast<double*>(base + nvec * vbytes);
    double* d_norm = reinterpret_cast<double*>(base + nvec * vbytes + pbytes);
    CgState* d_cg = reinterpret_cast<CgState*>(base + nvec * vbytes + pbytes + 256);
    double *r = v[0], *cand_r = v[1], *cand = v[2], *dvec = v[3], *cr = v[4], *z = v[5], *pv = v[6], *qv = v[7],
           *dinv = v[8], *c00 = v[9], *c01 = v[10], *c11 = v[11];
    do {
        D = sil_solve_diagnostics {};
        Geo const g {static_cast<int>(P.nx), static_cast<int>(P.ny)};
        int const n = g.nx * g.ny;
        unsigned const G = grid_for(n);
        double* x = P.solution;
        // residual norm of rhs - F(v) into out (returned on the host)
        auto residual = [&](double const* val, double* out, double* norm) -> sil_status {
            nl_apply_kernel<<<G, kBlock, 0, st>>>(C, g, val, P.node_mu, P.node_ferro, P.rhs, out, part);
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
            break;
        }
        if (r0 == 0.0) {
            D.converged = 1;
            break;
        }
        // 16 CG iterations captured once per problem (the kernels stop doing
        // work once the state is marked done) and replayed until convergence.
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        {
            cudaStream_t cs;
            SIL_CUDA_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            cudaError_t err = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
            for (int c = 0; c < 16 && err == cudaSuccess; ++c) {
                cg_jac_kernel<<<G, kBlock, 0, cs>>>(g, c00, c01, c11, pv, qv, part, d_cg);
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
                cudaGraphExecDestroy(e);
                cudaGraphDestroy(g);
            }
        } guard {graph, exec};
        int cg_total = 0, steps = 0;
        for (int it = 0; it < 30; ++it) {
            if (res / r0 <= tol) break;
            ++steps;
            nl_coef_kernel<<<G, kBlock, 0, st>>>(C, g, x, P.node_mu, P.node_ferro, c00, c01, c11);
            nl_dinv_kernel<<<G, kBlock, 0, st>>>(g, c00, c01, c11, dinv);
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
    } while (false);
    SIL_CUDA_CHECK(cudaStreamSynchronize(st));
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
    (void)grid_for(1);  // device attributes read once, before the threads start
    int dev = 0;
    SIL_CUDA_CHECK(cudaGetDevice(&dev));
    // Up to kConcurrent problems at a time, each on a host thread with its
    // own stream: one problem's CG kernels are small and launch bound, so
    // several problems together fill the GPU.
    constexpr int kConcurrent = 8;
    std::vector<sil_status> status(nproblems, SIL_OK);
    std::vector<std::string> message(nproblems);
    for (int first = 0; first < nproblems; first += kConcurrent) {
        int const last = std::min(nproblems, first + kConcurrent);
        std::vector<std::thread> workers;
        for (int p = first; p < last; ++p) {
            workers.emplace_back([&, p] {
                cudaSetDevice(dev);
                status[p] = solve_one(problems[p], curves[p], tol, max_iter, diag[p]);
                if (status[p] != SIL_OK) message[p] = sil_last_error();
            });
        }
        for (auto& w : workers) w.join();
    }
    for (int p = 0; p < nproblems; ++p)
        if (status[p] != SIL_OK) return fail(status[p], message[p]);
    return SIL_OK;
}
