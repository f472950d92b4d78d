// hodge_metric.cu -- the discrete Hodge star of an arbitrary (per-node,
// dense) metric on a structured lattice: the per-node tensor SimiLie's
// fill_discrete_hodge_star stores, and its application to a form.
//
// Per node and per canonical source component c, the unit cochain e_c goes
// through DiscreteHodgeStar::run (src/similie/exterior/hodge_star.hpp:227-273):
//   reconstruction (Reconstruction<Primal>, reduction_and_reconstruction.hpp:797-893)
//   -> continuous Hodge star with the metric (hodge_star.hpp:366-450,
//      reduction_and_reconstruction.hpp:350-401)
//   -> circumcentric-dual reduction (reduction_and_reconstruction.hpp:535-647,
//      with the legacy primal/dual volume ratio 403-432 and simplex volumes
//      from Gram determinants, exterior/volume.hpp:55-155);
// the responses fill the Full<k> x Antisym<n-k> tensor (hodge_star.hpp:275-358).
// Small dense matrices use the reference's partial-pivot determinant and
// Gauss-Jordan inverse (misc/small_matrix.hpp:75-198); every step keeps the
// reference's operation order.  One thread per node; this is set-up work
// (the staged operators fill once and apply many times).
#include <cmath>

#include "sil_internal.cuh"

namespace sil {
namespace {

constexpr int kN = kMaxNHodge;  // form dimensions, at most 3
constexpr int kMaxC = 3;        // C(3, k) <= 3

__device__ int binom_d(int n, int k)
{
    if (k < 0 || k > n) return 0;
    int r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

__device__ double factorial_d(int k)
{
    double r = 1.;
    for (int i = 2; i <= k; ++i) r *= i;
    return r;
}

// Lexicographic k-combination of {0..n-1} of a rank, and back.
__device__ void comb_from_rank(int n, int k, int rank, int* ids)
{
    int next = 0;
    for (int i = 0; i < k; ++i) {
        for (int cand = next; cand < n; ++cand) {
            int const remaining = k - i - 1;
            int const count = remaining == 0 ? 1 : binom_d(n - cand - 1, remaining);
            if (rank < count) {
                ids[i] = cand;
                next = cand + 1;
                break;
            }
            rank -= count;
        }
    }
}

__device__ int comb_rank(int n, int k, int const* ids)
{
    int rank = 0, next = 0;
    for (int i = 0; i < k; ++i) {
        for (int cand = next; cand < ids[i]; ++cand) {
            int const remaining = k - i - 1;
            rank += remaining == 0 ? 1 : binom_d(n - cand - 1, remaining);
        }
        next = ids[i] + 1;
    }
    return rank;
}

// Partial-pivot determinant of an n x n matrix (row-major), in place.
__device__ double det_d(double* m, int n)
{
    if (n == 0) return 1.;
    double det = 1.;
    int sign = 1;
    for (int i = 0; i < n; ++i) {
        int pivot = i;
        double pivot_abs = fabs(m[i * n + i]);
        for (int row = i + 1; row < n; ++row) {
            double const cand = fabs(m[row * n + i]);
            if (cand > pivot_abs) {
                pivot = row;
                pivot_abs = cand;
            }
        }
        if (pivot_abs == 0.) return 0.;
        if (pivot != i) {
            sign *= -1;
            for (int col = 0; col < n; ++col) {
                double const t = m[i * n + col];
                m[i * n + col] = m[pivot * n + col];
                m[pivot * n + col] = t;
            }
        }
        double const diagonal = m[i * n + i];
        det *= diagonal;
        for (int row = i + 1; row < n; ++row) {
            double const factor = m[row * n + i] / diagonal;
            for (int col = i + 1; col < n; ++col) m[row * n + col] -= factor * m[i * n + col];
            m[row * n + i] = 0.;
        }
    }
    return sign * det;
}

// Gauss-Jordan inverse with partial pivoting; false (and zeros) if singular.
__device__ bool invert_d(double* inv, double const* m, int n)
{
    double w[kMaxC * kMaxC];
    for (int i = 0; i < n * n; ++i) {
        w[i] = m[i];
        inv[i] = 0.;
    }
    for (int i = 0; i < n; ++i) inv[i * n + i] = 1.;
    for (int i = 0; i < n; ++i) {
        int pivot = i;
        double pivot_abs = fabs(w[i * n + i]);
        for (int row = i + 1; row < n; ++row) {
            double const cand = fabs(w[row * n + i]);
            if (cand > pivot_abs) {
                pivot = row;
                pivot_abs = cand;
            }
        }
        if (pivot_abs == 0.) {
            for (int j = 0; j < n * n; ++j) inv[j] = 0.;
            return false;
        }
        if (pivot != i) {
            for (int col = 0; col < n; ++col) {
                double t = w[i * n + col];
                w[i * n + col] = w[pivot * n + col];
                w[pivot * n + col] = t;
                t = inv[i * n + col];
                inv[i * n + col] = inv[pivot * n + col];
                inv[pivot * n + col] = t;
            }
        }
        double const diagonal = w[i * n + i];
        for (int col = 0; col < n; ++col) {
            w[i * n + col] /= diagonal;
            inv[i * n + col] /= diagonal;
        }
        for (int row = 0; row < n; ++row) {
            if (row == i) continue;
            double const factor = w[row * n + i];
            for (int col = 0; col < n; ++col) {
                w[row * n + col] -= factor * w[i * n + col];
                inv[row * n + col] -= factor * inv[i * n + col];
            }
        }
    }
    return true;
}

__device__ double subdet_d(double const* m, int n, int const* rows, int const* cols, int k)
{
    if (k == 0) return 1.;
    double sub[kMaxC * kMaxC];
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) sub[i * k + j] = m[rows[i] * n + cols[j]];
    return det_d(sub, k);
}

// Cofactor expansion along the first row, k <= 3 (the reference's
// reduction determinant).
__device__ double cofactor_det(double const* m, int k)
{
    if (k == 0) return 1.;
    if (k == 1) return m[0];
    double det = 0.;
    for (int col = 0; col < k; ++col) {
        double minor[(kMaxC - 1) * (kMaxC - 1)];
        for (int row = 1; row < k; ++row) {
            int mc = 0;
            for (int sc = 0; sc < k; ++sc) {
                if (sc == col) continue;
                minor[(row - 1) * (k - 1) + mc] = m[row * k + sc];
                ++mc;
            }
        }
        double md;
        if (k - 1 == 1) {
            md = minor[0];
        } else {  // k - 1 == 2: expand the 2x2 minor the same way
            md = 0.;
            md += 1. * minor[0] * minor[3];
            md += -1. * minor[1] * minor[2];
        }
        double const sign = (col % 2 == 0) ? 1. : -1.;
        det += sign * m[col] * md;
    }
    return det;
}

__device__ bool unique_ids_d(int n, int const* ids, int k)
{
    for (int i = 0; i < k; ++i) {
        if (ids[i] >= n) return false;
        for (int j = i + 1; j < k; ++j)
            if (ids[i] == ids[j]) return false;
    }
    return true;
}

__device__ bool complete_perm_d(int n, int const* a, int ka, int const* b, int kb)
{
    int counts[kN] = {0, 0, 0};
    for (int i = 0; i < ka; ++i) {
        if (a[i] >= n) return false;
        counts[a[i]]++;
    }
    for (int i = 0; i < kb; ++i) {
        if (b[i] >= n) return false;
        counts[b[i]]++;
    }
    for (int i = 0; i < n; ++i)
        if (counts[i] != 1) return false;
    return true;
}

__device__ int perm_sign_d(int const* a, int ka, int const* b, int kb)
{
    int p[2 * kN];
    for (int i = 0; i < ka; ++i) p[i] = a[i];
    for (int i = 0; i < kb; ++i) p[ka + i] = b[i];
    bool odd = false;
    for (int i = 0; i < ka + kb; ++i)
        for (int j = i + 1; j < ka + kb; ++j) odd = (p[i] > p[j]) != odd;
    return odd ? -1 : 1;
}

__device__ int complement_d(int n, int const* ids, int k, int* out)
{
    int m = 0;
    for (int i = 0; i < n; ++i) {
        bool found = false;
        for (int j = 0; j < k; ++j) found = found || ids[j] == i;
        if (!found) out[m++] = i;
    }
    return m;
}

// Position (n components) and metric (n x n, or NULL: identity) fields over
// the form lattice.
struct MetricGeo
{
    int n;
    FieldView pos;
    FieldView met;
    bool has_metric;

    __device__ bool contains(int64_t const* node) const
    {
        for (int d = 0; d < n; ++d)
            if (node[d] < pos.front[d] || node[d] >= pos.front[d] + pos.extent[d]) return false;
        return true;
    }

    __device__ double position(int64_t const* node, int comp) const
    {
        int64_t off = 0;
        for (int d = 0; d < n; ++d) off += (node[d] - pos.front[d]) * pos.stride[d];
        return static_cast<double const*>(pos.data)[off + comp * pos.comp_stride];
    }

    __device__ void metric_at(int64_t const* node, double* g) const
    {
        if (!has_metric) {
            for (int i = 0; i < n * n; ++i) g[i] = 0.;
            for (int i = 0; i < n; ++i) g[i * n + i] = 1.;
            return;
        }
        int64_t off = 0;
        for (int d = 0; d < n; ++d) off += (node[d] - met.front[d]) * met.stride[d];
        double const* p = static_cast<double const*>(met.data) + off;
        for (int i = 0; i < n * n; ++i) g[i] = p[i * met.comp_stride];
    }

    // forward difference of the position (backward at the last node)
    __device__ void edge_vector(int64_t const* node, int dim, double* v) const
    {
        int64_t fwd[kN], bwd[kN];
        for (int d = 0; d < n; ++d) fwd[d] = bwd[d] = node[d];
        fwd[dim] += 1;
        bwd[dim] -= 1;
        bool const has_fwd = contains(fwd);
        bool const has_bwd = contains(bwd);
        for (int c = 0; c < n; ++c) {
            double const center = position(node, c);
            if (has_fwd) v[c] = position(fwd, c) - center;
            else if (has_bwd) v[c] = center - position(bwd, c);
            else v[c] = 0.;
        }
    }

    __device__ double simplex_volume(int64_t const* node, int const* ids, int K) const
    {
        if (K == 0) return 1.;
        double g[kN * kN];
        metric_at(node, g);
        double edges[kN][kN];
        for (int i = 0; i < K; ++i) edge_vector(node, ids[i], edges[i]);
        double gram[kMaxC * kMaxC];
        for (int i = 0; i < K; ++i) {
            for (int j = i; j < K; ++j) {
                double value = 0.;
                for (int a = 0; a < n; ++a)
                    for (int b = 0; b < n; ++b) value += edges[i][a] * g[a * n + b] * edges[j][b];
                gram[i * K + j] = value;
                gram[j * K + i] = value;
            }
        }
        return sqrt(fabs(det_d(gram, K)));
    }

    __device__ double primal_reconstruction_diagonal(int64_t const* node, int const* ids, int K) const
    {
        if (K == 0) return 1.;
        double j[kMaxC * kMaxC];
        for (int row = 0; row < K; ++row)
            for (int col = 0; col < K; ++col) {
                double e[kN];
                edge_vector(node, ids[col], e);
                j[row * K + col] = e[ids[row]];
            }
        double const jac = cofactor_det(j, K);
        if (fabs(jac) < 1e-14) return 0.;
        return 1. / jac;
    }

    __device__ double continuous_hodge_value(int64_t const* node, int const* source, int K, int const* target,
                                             int Q) const
    {
        if (!unique_ids_d(n, source, K) || !unique_ids_d(n, target, Q) || !complete_perm_d(n, source, K, target, Q))
            return 0.;
        int comp[kN];
        int const nc = complement_d(n, target, Q, comp);
        double g[kN * kN], gdet[kN * kN], ginv[kN * kN];
        metric_at(node, g);
        for (int i = 0; i < n * n; ++i) gdet[i] = g[i];
        double const det = det_d(gdet, n);
        if (!invert_d(ginv, g, n)) return 0.;
        return sqrt(fabs(det)) * static_cast<double>(perm_sign_d(comp, nc, target, Q))
               * subdet_d(ginv, n, source, comp, K) / factorial_d(K);
    }

    __device__ double legacy_hodge_value(int64_t const* node, int const* source, int K, int const* target,
                                         int Q) const
    {
        if (!unique_ids_d(n, source, K) || !unique_ids_d(n, target, Q) || !complete_perm_d(n, source, K, target, Q))
            return 0.;
        double const primal_volume = simplex_volume(node, source, K);
        if (primal_volume == 0.) return 0.;
        int comp[kN];
        int const nc = complement_d(n, source, K, comp);
        return static_cast<double>(perm_sign_d(source, K, target, Q)) * simplex_volume(node, comp, nc)
               / (primal_volume * factorial_d(K));
    }

    __device__ void reconstruct(int64_t const* node, int K, double const* cochain, double* rec) const
    {
        if (K == 0) {
            rec[0] = cochain[0];
            return;
        }
        int const nb = binom_d(n, K);
        for (int t = 0; t < nb; ++t) {
            int tids[kN];
            comb_from_rank(n, K, t, tids);
            double value_sum = 0.;
            for (int sidx = 0; sidx < nb; ++sidx) {
                int sids[kN];
                comb_from_rank(n, K, sidx, sids);
                double j[kMaxC * kMaxC];
                for (int row = 0; row < K; ++row)
                    for (int col = 0; col < K; ++col) {
                        double e[kN];
                        edge_vector(node, tids[col], e);
                        j[row * K + col] = e[sids[row]];
                    }
                double const reduction_value = cofactor_det(j, K) / factorial_d(K);
                double value;
                if (sidx != t) value = 0.;
                else if (fabs(reduction_value) < 1e-14) value = 0.;
                else value = 1. / (factorial_d(K) * reduction_value);
                value_sum += value * cochain[sidx];
            }
            rec[t] = value_sum;
        }
    }

    __device__ void continuous_star(int64_t const* node, int K, double const* form, double* out) const
    {
        int const Q = n - K;
        int const nq = binom_d(n, Q);
        int ntuples = 1;
        for (int i = 0; i < K; ++i) ntuples *= n;
        for (int t = 0; t < nq; ++t) {
            int tids[kN];
            comb_from_rank(n, Q, t, tids);
            double acc = 0.;
            for (int tu = 0; tu < ntuples; ++tu) {
                int tuple[kN];
                int r = tu;
                for (int a = K - 1; a >= 0; --a) {
                    tuple[a] = r % n;
                    r /= n;
                }
                double const hs = continuous_hodge_value(node, tuple, K, tids, Q);
                double fv;
                if (K == 0) {
                    fv = form[0];
                } else if (!unique_ids_d(n, tuple, K)) {
                    fv = 0.;
                } else {
                    int sorted[kN];
                    for (int i = 0; i < K; ++i) sorted[i] = tuple[i];
                    for (int i = 0; i < K; ++i)
                        for (int j2 = i + 1; j2 < K; ++j2)
                            if (sorted[j2] < sorted[i]) {
                                int const tmp = sorted[i];
                                sorted[i] = sorted[j2];
                                sorted[j2] = tmp;
                            }
                    fv = perm_sign_d(tuple, K, nullptr, 0) * form[comb_rank(n, K, sorted)];
                }
                acc += hs * fv;
            }
            out[t] = acc;
        }
    }

    __device__ void reduce_dual(int64_t const* node, int Q, double const* form, double* out) const
    {
        int const K = n - Q;
        int const nb = binom_d(n, Q);
        double coeff[kMaxC * kMaxC], cinv[kMaxC * kMaxC], old[kMaxC * kMaxC];
        for (int p = 0; p < nb; ++p) {
            int pids[kN];
            comb_from_rank(n, K, p, pids);
            double const rdiag = primal_reconstruction_diagonal(node, pids, K);
            for (int sidx = 0; sidx < nb; ++sidx) {
                int sids[kN];
                comb_from_rank(n, Q, sidx, sids);
                coeff[sidx * nb + p] = continuous_hodge_value(node, pids, K, sids, Q) * rdiag;
            }
            for (int t = 0; t < nb; ++t) {
                int tids[kN];
                comb_from_rank(n, Q, t, tids);
                old[t * nb + p] = legacy_hodge_value(node, pids, K, tids, Q);
            }
        }
        bool const invertible = invert_d(cinv, coeff, nb);
        for (int t = 0; t < nb; ++t) {
            double reduced = 0.;
            for (int sidx = 0; sidx < nb; ++sidx) {
                double drv = 0.;
                if (invertible)
                    for (int p = 0; p < nb; ++p) drv += old[t * nb + p] * cinv[p * nb + sidx];
                reduced += drv * form[sidx];
            }
            out[t] = reduced;
        }
    }

    __device__ void discrete_star(int64_t const* node, int K, double const* form, double* out) const
    {
        double rec[kMaxC], cont[kMaxC];
        reconstruct(node, K, form, rec);
        continuous_star(node, K, rec, cont);
        reduce_dual(node, n - K, cont, out);
    }
};

// Stored tensor at every node of `hodge` (lattice over the form dims).
__global__ void fill_metric_kernel(MetricGeo geo, FieldView hodge, int K, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int const n = geo.n;
    int64_t node[kN], off = 0, r = flat;
    for (int d = n - 1; d >= 0; --d) {
        int64_t const l = r % hodge.extent[d];
        r /= hodge.extent[d];
        node[d] = hodge.front[d] + l;
        off += l * hodge.stride[d];
    }
    int const Q = n - K;
    int const nk = binom_d(n, K), nq = binom_d(n, Q);
    double resp[kMaxC][kMaxC];
    for (int c = 0; c < nk; ++c) {
        double unit[kMaxC] = {0., 0., 0.};
        unit[c] = 1.;
        geo.discrete_star(node, K, unit, resp[c]);
    }
    int ntuples = 1;
    for (int i = 0; i < K; ++i) ntuples *= n;
    double* o = static_cast<double*>(hodge.data) + off;
    for (int tu = 0; tu < ntuples; ++tu) {
        int tuple[kN];
        int rr = tu;
        for (int a = K - 1; a >= 0; --a) {
            tuple[a] = rr % n;
            rr /= n;
        }
        bool const valid = K <= 1 || unique_ids_d(n, tuple, K);
        bool odd = false;
        for (int i = 0; i < K; ++i)
            for (int j = i + 1; j < K; ++j) odd = (tuple[i] > tuple[j]) != odd;
        int sorted[kN];
        for (int i = 0; i < K; ++i) sorted[i] = tuple[i];
        for (int i = 0; i < K; ++i)
            for (int j = i + 1; j < K; ++j)
                if (sorted[j] < sorted[i]) {
                    int const tmp = sorted[i];
                    sorted[i] = sorted[j];
                    sorted[j] = tmp;
                }
        double const source_factor = (odd ? -1. : 1.) / factorial_d(K);
        int const c = K == 0 ? 0 : comb_rank(n, K, sorted);
        for (int t = 0; t < nq; ++t)
            o[(tu * nq + t) * hodge.comp_stride] = valid ? source_factor * resp[c][t] : 0.;
    }
}

// out[t] = sum over index tuples of form(tuple) * hodge(tuple, t) at every
// node of `out` (the reference's tensor_prod of the stored tensor with a form).
__global__ void apply_stored_kernel(FieldView hodge, FieldView in, FieldView out, int n, int K, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t r = flat, oo = 0, io = 0, ho = 0;
    for (int d = n - 1; d >= 0; --d) {
        int64_t const l = r % out.extent[d];
        r /= out.extent[d];
        int64_t const abs = out.front[d] + l;
        oo += l * out.stride[d];
        io += (abs - in.front[d]) * in.stride[d];
        ho += (abs - hodge.front[d]) * hodge.stride[d];
    }
    double const* h = static_cast<double const*>(hodge.data) + ho;
    double const* f = static_cast<double const*>(in.data) + io;
    double* o = static_cast<double*>(out.data) + oo;
    int const Q = n - K;
    int const nq = binom_d(n, Q);
    int ntuples = 1;
    for (int i = 0; i < K; ++i) ntuples *= n;
    for (int t = 0; t < nq; ++t) {
        double acc = 0.;
        for (int tu = 0; tu < ntuples; ++tu) {
            int tuple[kN];
            int rr = tu;
            for (int a = K - 1; a >= 0; --a) {
                tuple[a] = rr % n;
                rr /= n;
            }
            double fv;
            if (K == 0) {
                fv = f[0];
            } else if (!unique_ids_d(n, tuple, K)) {
                fv = 0.;
            } else {
                int sorted[kN];
                for (int i = 0; i < K; ++i) sorted[i] = tuple[i];
                for (int i = 0; i < K; ++i)
                    for (int j = i + 1; j < K; ++j)
                        if (sorted[j] < sorted[i]) {
                            int const tmp = sorted[i];
                            sorted[i] = sorted[j];
                            sorted[j] = tmp;
                        }
                fv = perm_sign_d(tuple, K, nullptr, 0) * f[comb_rank(n, K, sorted) * in.comp_stride];
            }
            acc += fv * h[(tu * nq + t) * hodge.comp_stride];
        }
        o[t * out.comp_stride] = acc;
    }
}

bool inside(sil_field const& inner, sil_field const& outer, int n)
{
    for (int d = 0; d < n; ++d)
        if (inner.front[d] < outer.front[d] || inner.front[d] + inner.extent[d] > outer.front[d] + outer.extent[d])
            return false;
    return true;
}

} // namespace
} // namespace sil

using namespace sil;

extern "C" {

sil_status sil_fill_discrete_hodge_star_metric(sil_stream stream, int n, int k_in, const sil_field* position,
                                               const sil_field* metric, sil_field* hodge)
{
    if (position == nullptr || hodge == nullptr)
        return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star_metric: NULL field");
    if (n < 1 || n > kN || k_in < 0 || k_in > n)
        return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star_metric: need 1 <= n <= 3 and 0 <= k_in <= n");
    sil_status st = check_field(position, "position", n);
    if (st != SIL_OK) return st;
    st = check_field(hodge, "hodge", static_cast<int>(ipow(n, k_in) * binom(n, n - k_in)));
    if (st != SIL_OK) return st;
    if (metric != nullptr) {
        st = check_field(metric, "metric", n * n);
        if (st != SIL_OK) return st;
    }
    if (position->dtype != SIL_F64 || hodge->dtype != SIL_F64 || (metric != nullptr && metric->dtype != SIL_F64))
        return fail(SIL_ERR_UNSUPPORTED, "sil_fill_discrete_hodge_star_metric: FP64 fields only");
    if (position->ndims != n || hodge->ndims != n || (metric != nullptr && metric->ndims != n))
        return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star_metric: fields must span exactly the n form dims");
    if (!inside(*hodge, *position, n) || (metric != nullptr && !inside(*hodge, *metric, n)))
        return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star_metric: hodge lattice must lie inside position/metric");
    MetricGeo g {};
    g.n = n;
    g.pos = to_view(*position);
    g.has_metric = metric != nullptr;
    if (metric != nullptr) g.met = to_view(*metric);
    int64_t const total = node_count(*hodge);
    if (total == 0) return SIL_OK;
    fill_metric_kernel<<<static_cast<unsigned>((total + 127) / 128), 128, 0, static_cast<cudaStream_t>(stream)>>>(
            g, to_view(*hodge), k_in, total);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status sil_hodge_star_stored(sil_stream stream, int n, int k_in, const sil_field* hodge, const sil_field* in,
                                 sil_field* out)
{
    if (hodge == nullptr || in == nullptr || out == nullptr)
        return fail(SIL_ERR_INVALID, "sil_hodge_star_stored: NULL field");
    if (n < 1 || n > kN || k_in < 0 || k_in > n)
        return fail(SIL_ERR_INVALID, "sil_hodge_star_stored: need 1 <= n <= 3 and 0 <= k_in <= n");
    sil_status st = check_field(hodge, "hodge", static_cast<int>(ipow(n, k_in) * binom(n, n - k_in)));
    if (st == SIL_OK) st = check_field(in, "in", static_cast<int>(binom(n, k_in)));
    if (st == SIL_OK) st = check_field(out, "out", static_cast<int>(binom(n, n - k_in)));
    if (st != SIL_OK) return st;
    if (hodge->dtype != SIL_F64 || in->dtype != SIL_F64 || out->dtype != SIL_F64)
        return fail(SIL_ERR_UNSUPPORTED, "sil_hodge_star_stored: FP64 fields only");
    if (hodge->ndims != n || in->ndims != n || out->ndims != n)
        return fail(SIL_ERR_INVALID, "sil_hodge_star_stored: fields must span exactly the n form dims");
    if (!inside(*out, *in, n) || !inside(*out, *hodge, n))
        return fail(SIL_ERR_INVALID, "sil_hodge_star_stored: output lattice must lie inside the input and the tensor");
    int64_t const total = node_count(*out);
    if (total == 0) return SIL_OK;
    apply_stored_kernel<<<static_cast<unsigned>((total + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            to_view(*hodge), to_view(*in), to_view(*out), n, k_in, total);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

} // extern "C"
