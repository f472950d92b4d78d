// sil_oracle.cpp -- CPU restatement of SimiLie's DEC operators (TEST INFRASTRUCTURE).
//
// This file is the checker the CUDA library is compared against and the timed
// CPU baseline; it is never part of the product path.  Each routine names the
// reference source (paths relative to the SimiLie project root) it restates.
// The restatement keeps the reference's order of floating-point operations
// wherever the reference fixes one (chain order of the coboundary sums, the
// pivoting order of the small-matrix routines, the staged kernel chain).

#include "sil_oracle.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <tuple>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

constexpr int MAXD = SILO_MAX_DIMS;
constexpr int MAXN = 4;  // form dimension limit (tests cover 1D..4D)

// ---------------------------------------------------------------- helpers

int64_t binom(int n, int k)
{
    if (k < 0 || k > n) return 0;
    int64_t r = 1;
    for (int i = 1; i <= k; ++i) r = r * (n - k + i) / i;
    return r;
}

double factorial(int k)
{
    double r = 1.;
    for (int i = 2; i <= k; ++i) r *= i;
    return r;
}

int64_t ipow(int64_t b, int e)
{
    int64_t r = 1;
    for (int i = 0; i < e; ++i) r *= b;
    return r;
}

// Tangent basis of K-simplices over n dims: 0/1 vectors enumerated by
// std::prev_permutation starting from [1..1,0..0].
// Ref: src/similie/exterior/local_chain.hpp:413-437
std::vector<std::array<int, MAXN>> tangent_basis(int n, int k)
{
    std::array<int, MAXN> p {};
    for (int i = 0; i < n; ++i) p[i] = i < k ? 1 : 0;
    std::vector<std::array<int, MAXN>> out;
    do {
        out.push_back(p);
    } while (std::prev_permutation(p.begin(), p.begin() + n));
    return out;
}

// Lexicographic k-combination of {0..n-1} <-> rank.
// Ref: src/similie/exterior/reduction_and_reconstruction.hpp:190-236
std::vector<int> combination_from_rank(int n, int k, int64_t rank)
{
    std::vector<int> ids(k);
    int next_candidate = 0;
    for (int i = 0; i < k; ++i) {
        for (int candidate = next_candidate; candidate < n; ++candidate) {
            int const remaining = k - i - 1;
            int const remaining_space = n - candidate - 1;
            int64_t const count = remaining == 0 ? 1 : binom(remaining_space, remaining);
            if (rank < count) {
                ids[i] = candidate;
                next_candidate = candidate + 1;
                break;
            }
            rank -= count;
        }
    }
    return ids;
}

int64_t combination_rank(int n, std::vector<int> const& ids)
{
    int const k = static_cast<int>(ids.size());
    int64_t rank = 0;
    int next_candidate = 0;
    for (int i = 0; i < k; ++i) {
        for (int candidate = next_candidate; candidate < ids[i]; ++candidate) {
            int const remaining = k - i - 1;
            int const remaining_space = n - candidate - 1;
            rank += remaining == 0 ? 1 : binom(remaining_space, remaining);
        }
        next_candidate = ids[i] + 1;
    }
    return rank;
}

// ---------------------------------------------------------------- simplices

struct Simplex
{
    int n;
    int64_t elem[MAXN];
    int vect[MAXN];
    bool negative;
};

// Constructor with reorientation of -1 entries.
// Ref: src/similie/exterior/simplex.hpp:16-68, 118-129
Simplex make_simplex(int n, int64_t const* elem, int const* vect, bool negative)
{
    Simplex s;
    s.n = n;
    bool neg = negative;
    for (int d = 0; d < n; ++d) {
        s.elem[d] = elem[d];
        s.vect[d] = vect[d];
        if (vect[d] == -1) {
            s.elem[d] -= 1;
            s.vect[d] = 1;
            neg = !neg;
        }
    }
    s.negative = neg;
    return s;
}

// Ref: src/similie/exterior/boundary.hpp:295-317 (generate_local_half_subchain)
void half_subchain(
        int n,
        int K,
        int64_t const* elem,
        int const* vect,
        bool negative,
        std::vector<Simplex>& chain)
{
    int id_dist = -1;
    for (int i = 0; i < K; ++i) {
        int array_[MAXN];
        for (int d = 0; d < n; ++d) array_[d] = vect[d];
        int id = id_dist + 1;
        while (id < n && array_[id] == 0) ++id;
        id_dist = id;
        array_[id] = 0;
        chain.push_back(make_simplex(n, elem, array_, ((negative ? 1 : 0) + i) % 2 != 0));
    }
}

// Boundary of a K-simplex, LocalChain flavour.  Ref: src/similie/exterior/boundary.hpp:426-441
std::vector<Simplex> boundary(int K, Simplex const& s)
{
    std::vector<Simplex> chain;
    half_subchain(s.n, K, s.elem, s.vect, K % 2 != 0, chain);
    int64_t shifted[MAXN];
    int minus[MAXN];
    for (int d = 0; d < s.n; ++d) {
        shifted[d] = s.elem[d] + s.vect[d];
        minus[d] = -s.vect[d];
    }
    half_subchain(s.n, K, shifted, minus, false, chain);
    int const mult = (K % 2 ? 1 : -1) * (s.negative ? -1 : 1);
    if (mult == -1) {
        for (auto& f : chain) f.negative = !f.negative;
    }
    return chain;
}

// One face of the boundary of a basis simplex, as a sampling rule relative
// to the node the simplex starts from.
struct FaceRule
{
    int64_t offset[MAXN];
    int comp;     // index of the face vector in the lower tangent basis
    bool negative;
};

// Face rules for every component of d (Coboundary::run) or of the
// transposed coboundary (TransposedCoboundary::run), with the -2 backward
// shift on the second half-chain for the transposed flavour.
// Ref: src/similie/exterior/coboundary.hpp:359-427 and 523-605
std::vector<std::vector<FaceRule>> face_rules(int n, int k, bool transposed)
{
    auto const chain = tangent_basis(n, k + 1);
    auto const lower = tangent_basis(n, k);
    std::vector<std::vector<FaceRule>> rules;
    int64_t origin[MAXN] = {0, 0, 0, 0};
    for (auto const& v : chain) {
        Simplex const s = make_simplex(n, origin, v.data(), false);
        auto const faces = boundary(k + 1, s);
        std::vector<FaceRule> comp_rules;
        for (std::size_t j = 0; j < faces.size(); ++j) {
            FaceRule r {};
            for (int d = 0; d < n; ++d) r.offset[d] = faces[j].elem[d];
            if (transposed && static_cast<int>(j) >= k + 1) {
                for (int d = 0; d < n; ++d) {
                    if (v[d] != 0 && faces[j].vect[d] == 0) {
                        r.offset[d] -= 2;
                        break;
                    }
                }
            }
            int comp = static_cast<int>(lower.size());
            for (std::size_t c = 0; c < lower.size(); ++c) {
                bool same = true;
                for (int d = 0; d < n; ++d) same = same && (lower[c][d] == faces[j].vect[d]);
                if (same) {
                    comp = static_cast<int>(c);
                    break;
                }
            }
            r.comp = comp;
            r.negative = faces[j].negative;
            comp_rules.push_back(r);
        }
        rules.push_back(comp_rules);
    }
    return rules;
}

// ---------------------------------------------------------------- fields

int64_t num_nodes(silo_field const& f)
{
    int64_t t = 1;
    for (int d = 0; d < f.ndims; ++d) t *= f.extent[d];
    return t;
}

void unravel(silo_field const& f, int64_t flat, int64_t* local)
{
    for (int d = f.ndims - 1; d >= 0; --d) {
        local[d] = flat % f.extent[d];
        flat /= f.extent[d];
    }
}

int64_t offset_local(silo_field const& f, int64_t const* local)
{
    int64_t o = 0;
    for (int d = 0; d < f.ndims; ++d) o += local[d] * f.stride[d];
    return o;
}

bool contains_abs(silo_field const& f, int64_t const* abs)
{
    for (int d = 0; d < f.ndims; ++d) {
        if (abs[d] < f.front[d] || abs[d] > f.front[d] + f.extent[d] - 1) return false;
    }
    return true;
}

int form_dims(uint32_t mask, int ndims, int* dims)
{
    int n = 0;
    for (int d = 0; d < ndims; ++d) {
        if (mask & (1u << d)) dims[n++] = d;
    }
    return n;
}

// d on a k-form with clamped sampling (ClampedTensorEvaluator,
// src/similie/exterior/evaluators.hpp:30-46; misc/clamp_to_domain.hpp:17-47),
// or the transposed coboundary with zero-outside sampling
// (ZeroOutsideTensorEvaluator, evaluators.hpp:48-68; misc/domain_contains.hpp).
// Summation in chain order from 0 (Cochain::integrate, cochain.hpp:187-198).
int coboundary_impl(uint32_t mask, int k, silo_field const* in, silo_field* out, bool transposed)
{
    int dims[MAXD];
    int const n = form_dims(mask, in->ndims, dims);
    if (n < 1 || n > MAXN || k < 0 || k >= n) return -1;
    if (in->ndims != out->ndims) return -1;
    if (in->ncomp != binom(n, k) || out->ncomp != binom(n, k + 1)) return -1;
    auto const rules = face_rules(n, k, transposed);
    int64_t const total = num_nodes(*out);
#pragma omp parallel for schedule(static)
    for (int64_t flat = 0; flat < total; ++flat) {
        int64_t local[MAXD];
        unravel(*out, flat, local);
        int64_t abs[MAXD];
        for (int d = 0; d < out->ndims; ++d) abs[d] = out->front[d] + local[d];
        double* o = out->data + offset_local(*out, local);
        for (std::size_t c = 0; c < rules.size(); ++c) {
            double acc = 0.;
            for (auto const& r : rules[c]) {
                int64_t s[MAXD];
                for (int d = 0; d < in->ndims; ++d) s[d] = abs[d];
                for (int a = 0; a < n; ++a) s[dims[a]] += r.offset[a];
                double v;
                if (!transposed) {
                    for (int d = 0; d < in->ndims; ++d) {
                        s[d] = std::min(std::max(s[d], in->front[d]), in->front[d] + in->extent[d] - 1);
                    }
                    int64_t sl[MAXD];
                    for (int d = 0; d < in->ndims; ++d) sl[d] = s[d] - in->front[d];
                    v = in->data[offset_local(*in, sl) + r.comp * in->comp_stride];
                } else if (!contains_abs(*in, s)) {
                    v = 0.0;
                } else {
                    int64_t sl[MAXD];
                    for (int d = 0; d < in->ndims; ++d) sl[d] = s[d] - in->front[d];
                    v = in->data[offset_local(*in, sl) + r.comp * in->comp_stride];
                }
                acc += (r.negative ? -1 : 1) * v;
            }
            o[c * out->comp_stride] = transposed ? -acc : acc;
        }
    }
    return 0;
}

// ---------------------------------------------------------------- small matrices

// Partial-pivot determinant, in place.  Ref: src/similie/misc/small_matrix.hpp:75-117
double determinant(double* m, int n)
{
    if (n == 0) return 1.;
    double det = 1.;
    int sign = 1;
    for (int i = 0; i < n; ++i) {
        int pivot = i;
        double pivot_abs = std::abs(m[i * n + i]);
        for (int row = i + 1; row < n; ++row) {
            double const cand = std::abs(m[row * n + i]);
            if (cand > pivot_abs) {
                pivot = row;
                pivot_abs = cand;
            }
        }
        if (pivot_abs == 0.) return 0.;
        if (pivot != i) {
            sign *= -1;
            for (int col = 0; col < n; ++col) std::swap(m[i * n + col], m[pivot * n + col]);
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

// Gauss-Jordan inverse with partial pivoting.  Ref: src/similie/misc/small_matrix.hpp:120-180
bool invert(double* inv, double const* m, int n)
{
    std::vector<double> w(m, m + n * n);
    for (int i = 0; i < n * n; ++i) inv[i] = 0.;
    for (int i = 0; i < n; ++i) inv[i * n + i] = 1.;
    for (int i = 0; i < n; ++i) {
        int pivot = i;
        double pivot_abs = std::abs(w[i * n + i]);
        for (int row = i + 1; row < n; ++row) {
            double const cand = std::abs(w[row * n + i]);
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
                std::swap(w[i * n + col], w[pivot * n + col]);
                std::swap(inv[i * n + col], inv[pivot * n + col]);
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

// Ref: src/similie/misc/small_matrix.hpp:183-198
double submatrix_determinant(double const* m, int n, std::vector<int> const& rows, std::vector<int> const& cols)
{
    int const k = static_cast<int>(rows.size());
    if (k == 0) return 1.;
    std::vector<double> sub(k * k);
    for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) sub[i * k + j] = m[rows[i] * n + cols[j]];
    return determinant(sub.data(), k);
}

// Cofactor expansion along the first row.
// Ref: src/similie/exterior/reduction_and_reconstruction.hpp:162-188
double reduction_determinant(std::vector<double> const& m, int k)
{
    if (k == 0) return 1.;
    if (k == 1) return m[0];
    double det = 0.;
    for (int col = 0; col < k; ++col) {
        std::vector<double> minor((k - 1) * (k - 1));
        for (int row = 1; row < k; ++row) {
            int mc = 0;
            for (int sc = 0; sc < k; ++sc) {
                if (sc == col) continue;
                minor[(row - 1) * (k - 1) + mc] = m[row * k + sc];
                ++mc;
            }
        }
        double const sign = (col % 2 == 0) ? 1. : -1.;
        det += sign * m[col] * reduction_determinant(minor, k - 1);
    }
    return det;
}

std::vector<int> complement(int n, std::vector<int> const& ids)
{
    std::vector<int> c;
    for (int i = 0; i < n; ++i) {
        bool found = false;
        for (int id : ids) found = found || id == i;
        if (!found) c.push_back(i);
    }
    return c;
}

bool unique_ids(int n, std::vector<int> const& ids)
{
    for (std::size_t i = 0; i < ids.size(); ++i) {
        if (ids[i] >= n) return false;
        for (std::size_t j = i + 1; j < ids.size(); ++j)
            if (ids[i] == ids[j]) return false;
    }
    return true;
}

bool complete_permutation(int n, std::vector<int> const& a, std::vector<int> const& b)
{
    std::vector<int> counts(n, 0);
    for (int id : a) {
        if (id >= n) return false;
        counts[id]++;
    }
    for (int id : b) {
        if (id >= n) return false;
        counts[id]++;
    }
    for (int c : counts)
        if (c != 1) return false;
    return true;
}

// Ref: src/similie/exterior/reduction_and_reconstruction.hpp:282-304
int permutation_sign(std::vector<int> const& a, std::vector<int> const& b)
{
    std::vector<int> p(a);
    p.insert(p.end(), b.begin(), b.end());
    bool odd = false;
    for (std::size_t i = 0; i < p.size(); ++i)
        for (std::size_t j = i + 1; j < p.size(); ++j) odd = (p[i] > p[j]) != odd;
    return odd ? -1 : 1;
}

// ---------------------------------------------------------------- geometry

struct Geometry
{
    int n;
    silo_field const* position;  // lattice over the form dims, n comps
    silo_field const* metric;    // lattice over the form dims, n*n comps, or nullptr

    void metric_at(int64_t const* node, double* g) const
    {
        if (metric == nullptr) {
            for (int i = 0; i < n * n; ++i) g[i] = 0.;
            for (int i = 0; i < n; ++i) g[i * n + i] = 1.;
            return;
        }
        int64_t local[MAXD];
        for (int d = 0; d < n; ++d) local[d] = node[d] - metric->front[d];
        double const* p = metric->data + offset_local(*metric, local);
        for (int i = 0; i < n * n; ++i) g[i] = p[i * metric->comp_stride];
    }

    double pos(int64_t const* node, int comp) const
    {
        int64_t local[MAXD];
        for (int d = 0; d < n; ++d) local[d] = node[d] - position->front[d];
        return position->data[offset_local(*position, local) + comp * position->comp_stride];
    }

    // Ref: src/similie/exterior/volume.hpp:55-82
    void edge_vector(int64_t const* node, int dim, double* v) const
    {
        int64_t fwd[MAXD], bwd[MAXD];
        for (int d = 0; d < n; ++d) fwd[d] = bwd[d] = node[d];
        fwd[dim] += 1;
        bwd[dim] -= 1;
        bool const has_fwd = contains_abs(*position, fwd);
        bool const has_bwd = contains_abs(*position, bwd);
        for (int c = 0; c < n; ++c) {
            double const center = pos(node, c);
            if (has_fwd) v[c] = pos(fwd, c) - center;
            else if (has_bwd) v[c] = center - pos(bwd, c);
            else v[c] = 0.;
        }
    }

    // Ref: src/similie/exterior/volume.hpp:101-155
    double simplex_volume(int64_t const* node, std::vector<int> const& ids) const
    {
        int const K = static_cast<int>(ids.size());
        if (K == 0) return 1.;
        double g[MAXN * MAXN];
        metric_at(node, g);
        std::vector<std::array<double, MAXN>> edges(K);
        for (int i = 0; i < K; ++i) edge_vector(node, ids[i], edges[i].data());
        std::vector<double> gram(K * K);
        for (int i = 0; i < K; ++i) {
            for (int j = i; j < K; ++j) {
                double value = 0.;
                for (int a = 0; a < n; ++a)
                    for (int b = 0; b < n; ++b) value += edges[i][a] * g[a * n + b] * edges[j][b];
                gram[i * K + j] = value;
                gram[j * K + i] = value;
            }
        }
        return std::sqrt(std::abs(determinant(gram.data(), K)));
    }

    // Ref: src/similie/exterior/reduction_and_reconstruction.hpp:324-348
    double primal_reconstruction_diagonal(int64_t const* node, std::vector<int> const& ids) const
    {
        int const K = static_cast<int>(ids.size());
        if (K == 0) return 1.;
        std::vector<double> j(K * K);
        for (int row = 0; row < K; ++row) {
            for (int col = 0; col < K; ++col) {
                double e[MAXN];
                edge_vector(node, ids[col], e);
                j[row * K + col] = e[ids[row]];
            }
        }
        double const jac = reduction_determinant(j, K);
        if (std::abs(jac) < 1e-14) return 0.;
        return 1. / jac;
    }

    // Ref: src/similie/exterior/reduction_and_reconstruction.hpp:350-401 and hodge_star.hpp:396-450
    double continuous_hodge_value(
            int64_t const* node,
            std::vector<int> const& source,
            std::vector<int> const& target) const
    {
        int const K = static_cast<int>(source.size());
        if (!unique_ids(n, source) || !unique_ids(n, target) || !complete_permutation(n, source, target))
            return 0.;
        std::vector<int> const comp = complement(n, target);
        double g[MAXN * MAXN], gdet[MAXN * MAXN], ginv[MAXN * MAXN];
        metric_at(node, g);
        std::copy(g, g + n * n, gdet);
        double const det = determinant(gdet, n);
        if (!invert(ginv, g, n)) return 0.;
        return std::sqrt(std::abs(det)) * static_cast<double>(permutation_sign(comp, target))
               * submatrix_determinant(ginv, n, source, comp) / factorial(K);
    }

    // Ref: src/similie/exterior/reduction_and_reconstruction.hpp:403-432
    double legacy_hodge_value(
            int64_t const* node,
            std::vector<int> const& source,
            std::vector<int> const& target) const
    {
        int const K = static_cast<int>(source.size());
        if (!unique_ids(n, source) || !unique_ids(n, target) || !complete_permutation(n, source, target))
            return 0.;
        double const primal_volume = simplex_volume(node, source);
        if (primal_volume == 0.) return 0.;
        return static_cast<double>(permutation_sign(source, target)) * simplex_volume(node, complement(n, source))
               / (primal_volume * factorial(K));
    }

    // Reconstruction<Primal>::run: rec[t] = sum_s value(s,t) * cochain[s].
    // Ref: src/similie/exterior/reduction_and_reconstruction.hpp:814-892
    void reconstruct(int64_t const* node, int K, double const* cochain, double* rec) const
    {
        if (K == 0) {
            rec[0] = cochain[0];
            return;
        }
        int64_t const nb = binom(n, K);
        for (int64_t t = 0; t < nb; ++t) {
            auto const tids = combination_from_rank(n, K, t);
            double value_sum = 0.;
            for (int64_t s = 0; s < nb; ++s) {
                auto const sids = combination_from_rank(n, K, s);
                double value;
                // Reduction<Primal>::value with source=sids, target=tids (lines 649-677).
                std::vector<double> j(K * K);
                for (int row = 0; row < K; ++row) {
                    for (int col = 0; col < K; ++col) {
                        double e[MAXN];
                        edge_vector(node, tids[col], e);
                        j[row * K + col] = e[sids[row]];
                    }
                }
                double const reduction_value = reduction_determinant(j, K) / factorial(K);
                if (s != t) value = 0.;
                else if (std::abs(reduction_value) < 1e-14) value = 0.;
                else value = 1. / (factorial(K) * reduction_value);
                value_sum += value * cochain[s];
            }
            rec[t] = value_sum;
        }
    }

    // ContinuousHodgeStar::run: contraction of the Full x Antisym tensor with
    // the K-form over all index tuples.  Ref: src/similie/exterior/hodge_star.hpp:366-394
    void continuous_star(int64_t const* node, int K, double const* form, double* out) const
    {
        int const Q = n - K;
        int64_t const nq = binom(n, Q);
        int64_t const ntuples = ipow(n, K);
        for (int64_t t = 0; t < nq; ++t) {
            auto const tids = combination_from_rank(n, Q, t);
            double acc = 0.;
            for (int64_t tu = 0; tu < ntuples; ++tu) {
                std::vector<int> tuple(K);
                int64_t r = tu;
                for (int a = K - 1; a >= 0; --a) {
                    tuple[a] = static_cast<int>(r % n);
                    r /= n;
                }
                double const hs = continuous_hodge_value(node, tuple, tids);
                double fv;
                if (K == 0) {
                    fv = form[0];
                } else if (!unique_ids(n, tuple)) {
                    fv = 0.;
                } else {
                    std::vector<int> sorted(tuple);
                    std::sort(sorted.begin(), sorted.end());
                    std::vector<int> none;
                    int const sgn = permutation_sign(tuple, none);
                    fv = sgn * form[combination_rank(n, sorted)];
                }
                acc += hs * fv;
            }
            out[t] = acc;
        }
    }

    // Reduction<CircumcentricDual>::run (metric-aware).
    // Ref: src/similie/exterior/reduction_and_reconstruction.hpp:535-647
    void reduce_dual(int64_t const* node, int Q, double const* form, double* out) const
    {
        int const K = n - Q;
        int64_t const nb = binom(n, Q);
        std::vector<double> coeff(nb * nb), cinv(nb * nb), old(nb * nb);
        for (int64_t p = 0; p < nb; ++p) {
            auto const pids = combination_from_rank(n, K, p);
            double const rdiag = primal_reconstruction_diagonal(node, pids);
            for (int64_t s = 0; s < nb; ++s) {
                auto const sids = combination_from_rank(n, Q, s);
                coeff[s * nb + p] = continuous_hodge_value(node, pids, sids) * rdiag;
            }
            for (int64_t t = 0; t < nb; ++t) {
                auto const tids = combination_from_rank(n, Q, t);
                old[t * nb + p] = legacy_hodge_value(node, pids, tids);
            }
        }
        bool const invertible = invert(cinv.data(), coeff.data(), static_cast<int>(nb));
        for (int64_t t = 0; t < nb; ++t) {
            double reduced = 0.;
            for (int64_t s = 0; s < nb; ++s) {
                double drv = 0.;
                if (invertible) {
                    for (int64_t p = 0; p < nb; ++p) drv += old[t * nb + p] * cinv[p * nb + s];
                }
                reduced += drv * form[s];
            }
            out[t] = reduced;
        }
    }

    // DiscreteHodgeStar::run.  Ref: src/similie/exterior/hodge_star.hpp:227-273
    void discrete_star(int64_t const* node, int K, double const* form, double* out) const
    {
        double rec[8], cont[8];
        reconstruct(node, K, form, rec);
        continuous_star(node, K, rec, cont);
        reduce_dual(node, n - K, cont, out);
    }
};

// Per-node stored Hodge tensor, DiscreteHodgeStar::value for every
// (full source tuple, canonical target) pair.  run() depends only on the
// canonical source, so it is evaluated once per canonical component.
// Ref: src/similie/exterior/hodge_star.hpp:275-358, 461-494
void fill_node(Geometry const& geo, int K, int64_t const* node, double* out, int64_t comp_stride)
{
    int const n = geo.n;
    int const Q = n - K;
    int64_t const nk = binom(n, K);
    int64_t const nq = binom(n, Q);
    std::vector<double> responses(nk * nq);
    for (int64_t c = 0; c < nk; ++c) {
        double unit[8] = {0};
        unit[c] = 1.;
        geo.discrete_star(node, K, unit, &responses[c * nq]);
    }
    int64_t const ntuples = ipow(n, K);
    for (int64_t tu = 0; tu < ntuples; ++tu) {
        std::vector<int> tuple(K);
        int64_t r = tu;
        for (int a = K - 1; a >= 0; --a) {
            tuple[a] = static_cast<int>(r % n);
            r /= n;
        }
        bool const valid = K <= 1 || unique_ids(n, tuple);
        bool odd = false;
        for (int i = 0; i < K; ++i)
            for (int j = i + 1; j < K; ++j) odd = (tuple[i] > tuple[j]) != odd;
        std::vector<int> sorted(tuple);
        std::sort(sorted.begin(), sorted.end());
        double const source_factor = (odd ? -1. : 1.) / factorial(K);
        int64_t const c = K == 0 ? 0 : combination_rank(n, sorted);
        for (int64_t t = 0; t < nq; ++t) {
            out[(tu * nq + t) * comp_stride] = valid ? source_factor * responses[c * nq + t] : 0.;
        }
    }
}

// tensor_prod(out, form, hodge): out[t] = sum over tuples form.get(tuple) * hodge(tuple, t).
// Ref: src/similie/tensor/tensor_prod.hpp:108-157
void apply_node(int n, int K, double const* hodge, int64_t hstride, double const* form, int64_t fstride,
                double* out, int64_t ostride)
{
    int const Q = n - K;
    int64_t const nq = binom(n, Q);
    int64_t const ntuples = ipow(n, K);
    for (int64_t t = 0; t < nq; ++t) {
        double acc = 0.;
        for (int64_t tu = 0; tu < ntuples; ++tu) {
            std::vector<int> tuple(K);
            int64_t r = tu;
            for (int a = K - 1; a >= 0; --a) {
                tuple[a] = static_cast<int>(r % n);
                r /= n;
            }
            double fv;
            if (K == 0) {
                fv = form[0];
            } else if (!unique_ids(n, tuple)) {
                fv = 0.;
            } else {
                std::vector<int> sorted(tuple);
                std::sort(sorted.begin(), sorted.end());
                std::vector<int> none;
                fv = permutation_sign(tuple, none) * form[combination_rank(n, sorted) * fstride];
            }
            acc += fv * hodge[(tu * nq + t) * hstride];
        }
        out[t * ostride] = acc;
    }
}

// Stored-Hodge lookup for a node of a field whose form dims are the first
// `n` dims listed in `dims`.
double const* hodge_at(silo_field const& hs, int n, int const* dims, int64_t const* abs)
{
    int64_t local[MAXD];
    for (int a = 0; a < n; ++a) local[a] = abs[dims[a]] - hs.front[a];
    return hs.data + offset_local(hs, local);
}

silo_field make_buffer(silo_field const& like, int ncomp, std::vector<double>& storage)
{
    silo_field f = like;
    int64_t const nodes = num_nodes(like);
    storage.assign(nodes * ncomp, 0.);
    f.data = storage.data();
    f.ncomp = ncomp;
    f.comp_stride = 1;
    int64_t s = ncomp;
    for (int d = like.ndims - 1; d >= 0; --d) {
        f.stride[d] = s;
        s *= like.extent[d];
    }
    return f;
}

silo_field make_hodge_field(silo_field const& lattice, int n, int K, std::vector<double>& storage)
{
    silo_field f {};
    f.ndims = n;
    int const ncomp = static_cast<int>(ipow(n, K) * binom(n, n - K));
    int64_t nodes = 1;
    for (int d = 0; d < n; ++d) {
        f.front[d] = lattice.front[d];
        f.extent[d] = lattice.extent[d];
        nodes *= f.extent[d];
    }
    storage.assign(nodes * ncomp, 0.);
    f.data = storage.data();
    f.ncomp = ncomp;
    f.comp_stride = 1;
    int64_t s = ncomp;
    for (int d = n - 1; d >= 0; --d) {
        f.stride[d] = s;
        s *= f.extent[d];
    }
    return f;
}

int fill_impl(int n, int K, silo_field const* position, silo_field const* metric, silo_field* hodge)
{
    if (n < 1 || n > 3 || K < 0 || K > n) return -1;
    if (hodge->ncomp != ipow(n, K) * binom(n, n - K)) return -1;
    Geometry const geo {n, position, metric};
    int64_t const total = num_nodes(*hodge);
#pragma omp parallel for schedule(static)
    for (int64_t flat = 0; flat < total; ++flat) {
        int64_t local[MAXD], abs[MAXD];
        unravel(*hodge, flat, local);
        for (int d = 0; d < n; ++d) abs[d] = hodge->front[d] + local[d];
        fill_node(geo, K, abs, hodge->data + offset_local(*hodge, local), hodge->comp_stride);
    }
    return 0;
}

// out[node] = hodge[node] . in[node] over every node of `out` (same lattice as in).
void apply_field(int n, int const* dims, int K, silo_field const& hs, silo_field const& in, silo_field& out)
{
    int64_t const total = num_nodes(out);
#pragma omp parallel for schedule(static)
    for (int64_t flat = 0; flat < total; ++flat) {
        int64_t local[MAXD], abs[MAXD], il[MAXD];
        unravel(out, flat, local);
        for (int d = 0; d < out.ndims; ++d) {
            abs[d] = out.front[d] + local[d];
            il[d] = abs[d] - in.front[d];
        }
        apply_node(n, K, hodge_at(hs, n, dims, abs), hs.comp_stride, in.data + offset_local(in, il),
                   in.comp_stride, out.data + offset_local(out, local), out.comp_stride);
    }
}

// dual-side kernel: sample `src` by d^T (zero outside) at each node of `out`,
// then apply the stored Hodge tensor `hs` and the codifferential sign.
// Ref: src/similie/exterior/codifferential.hpp:460-504; laplacian.hpp:110-152
void transpose_star_field(int n, int const* dims, int src_rank, silo_field const& hs, silo_field const& src,
                          silo_field& out, bool negate)
{
    auto const rules = face_rules(n, src_rank, true);
    int const dual_k = src_rank + 1;
    int64_t const total = num_nodes(out);
#pragma omp parallel for schedule(static)
    for (int64_t flat = 0; flat < total; ++flat) {
        int64_t local[MAXD], abs[MAXD];
        unravel(out, flat, local);
        for (int d = 0; d < out.ndims; ++d) abs[d] = out.front[d] + local[d];
        double dual_codiff[8];
        for (std::size_t c = 0; c < rules.size(); ++c) {
            double acc = 0.;
            for (auto const& r : rules[c]) {
                int64_t s[MAXD];
                for (int d = 0; d < src.ndims; ++d) s[d] = abs[d];
                for (int a = 0; a < n; ++a) s[dims[a]] += r.offset[a];
                double v = 0.;
                if (contains_abs(src, s)) {
                    int64_t sl[MAXD];
                    for (int d = 0; d < src.ndims; ++d) sl[d] = s[d] - src.front[d];
                    v = src.data[offset_local(src, sl) + r.comp * src.comp_stride];
                }
                acc += (r.negative ? -1 : 1) * v;
            }
            dual_codiff[c] = -acc;
        }
        double* o = out.data + offset_local(out, local);
        apply_node(n, dual_k, hodge_at(hs, n, dims, abs), hs.comp_stride, dual_codiff, 1, o, out.comp_stride);
        if (negate) {
            for (int c = 0; c < out.ncomp; ++c) o[c * out.comp_stride] *= -1;
        }
    }
}

// First kernel of codifferential_of_coboundary: clamped d then stored Hodge.
// Ref: src/similie/exterior/laplacian.hpp:78-108
void deriv_star_field(int n, int const* dims, int k, silo_field const& hs, silo_field const& in, silo_field& dual)
{
    auto const rules = face_rules(n, k, false);
    int64_t const total = num_nodes(dual);
#pragma omp parallel for schedule(static)
    for (int64_t flat = 0; flat < total; ++flat) {
        int64_t local[MAXD], abs[MAXD];
        unravel(dual, flat, local);
        for (int d = 0; d < dual.ndims; ++d) abs[d] = dual.front[d] + local[d];
        double deriv[8];
        for (std::size_t c = 0; c < rules.size(); ++c) {
            double acc = 0.;
            for (auto const& r : rules[c]) {
                int64_t s[MAXD], sl[MAXD];
                for (int d = 0; d < in.ndims; ++d) s[d] = abs[d];
                for (int a = 0; a < n; ++a) s[dims[a]] += r.offset[a];
                for (int d = 0; d < in.ndims; ++d) {
                    s[d] = std::min(std::max(s[d], in.front[d]), in.front[d] + in.extent[d] - 1);
                    sl[d] = s[d] - in.front[d];
                }
                acc += (r.negative ? -1 : 1) * in.data[offset_local(in, sl) + r.comp * in.comp_stride];
            }
            deriv[c] = acc;
        }
        apply_node(n, k + 1, hodge_at(hs, n, dims, abs), hs.comp_stride, deriv, 1,
                   dual.data + offset_local(dual, local), dual.comp_stride);
    }
}

bool sign_negative(int n, int k_plus_one)
{
    return (n * (k_plus_one + 1) + 1) % 2 == 1;
}

struct LaplacianHodges
{
    silo_field const* h[4];
};

int laplacian_impl(int n, int k, LaplacianHodges const& hs, silo_field const* in, silo_field* out)
{
    int dims[MAXD];
    for (int d = 0; d < n; ++d) dims[d] = d;
    if (in->ndims != n || out->ndims != n) return -1;
    if (in->ncomp != binom(n, k) || out->ncomp != binom(n, k)) return -1;
    std::vector<double> s1, s2, s3, s4;
    if (k < n) {
        // delta d: codifferential_of_coboundary (laplacian.hpp:27-155)
        silo_field dual = make_buffer(*in, static_cast<int>(binom(n, n - k - 1)), s1);
        deriv_star_field(n, dims, k, *hs.h[0], *in, dual);
        transpose_star_field(n, dims, n - k - 1, *hs.h[1], dual, *out, sign_negative(n, k + 1));
    }
    if (k > 0) {
        // d delta: StagedCodifferential::run then deriv (laplacian.hpp:614-631, 793-810)
        silo_field dual = make_buffer(*in, static_cast<int>(binom(n, n - k)), s2);
        apply_field(n, dims, k, *hs.h[2], *in, dual);
        silo_field codiff = make_buffer(*in, static_cast<int>(binom(n, k - 1)), s3);
        transpose_star_field(n, dims, n - k, *hs.h[3], dual, codiff, sign_negative(n, k));
        if (k < n) {
            silo_field cob = make_buffer(*out, out->ncomp, s4);
            coboundary_impl((1u << n) - 1, k - 1, &codiff, &cob, false);
            int64_t const total = num_nodes(*out);
#pragma omp parallel for schedule(static)
            for (int64_t flat = 0; flat < total; ++flat) {
                int64_t local[MAXD];
                unravel(*out, flat, local);
                double* o = out->data + offset_local(*out, local);
                double const* c = cob.data + offset_local(cob, local);
                for (int comp = 0; comp < out->ncomp; ++comp) o[comp * out->comp_stride] += c[comp * cob.comp_stride];
            }
        } else {
            coboundary_impl((1u << n) - 1, k - 1, &codiff, out, false);
        }
    }
    return 0;
}

int hodge_kin(int n, int k, int which)
{
    switch (which) {
    case 0: return k + 1;      // derivative Hodge: (k+1)-form -> (n-k-1)-form
    case 1: return n - k;      // dual derivative Hodge: (n-k)-form -> k-form
    case 2: return k;          // codifferential Hodge: k-form -> (n-k)-form
    case 3: return n - k + 1;  // dual codifferential Hodge: (n-k+1)-form -> (k-1)-form
    default: return -1;
    }
}

bool hodge_needed(int n, int k, int which)
{
    return (which <= 1) ? (k < n) : (k > 0);
}

} // namespace

extern "C" {

int silo_coboundary(uint32_t form_mask, int k, const silo_field* in, silo_field* out)
{
    return coboundary_impl(form_mask, k, in, out, false);
}

int silo_transposed_coboundary(uint32_t form_mask, int k, const silo_field* in, silo_field* out)
{
    return coboundary_impl(form_mask, k, in, out, true);
}

// Reduction<Primal>::run at one node: reduced[t] = sum over the ordered
// source tuples of value(source, t) * form.get(source), value = det(J) / K!
// with J[row][col] = edge_{t[col]}[source[row]] (0 for repeated ids), and
// form.get the antisymmetric tensor's signed component.
// Ref: src/similie/exterior/reduction_and_reconstruction.hpp:472-534, 649-677;
//      volume.hpp:46-53 (complex volume factor 1 on the primal complex)
int silo_reduce_primal(int n, int K, const silo_field* position, const int64_t* node, const double* form, double* out)
{
    if (n < 1 || n > MAXN || K < 0 || K > n) return 1;
    Geometry const G {n, position, nullptr};
    if (K == 0) {
        out[0] = form[0];
        return 0;
    }
    int64_t const nb = binom(n, K);
    int64_t const ntuples = ipow(n, K);
    for (int64_t t = 0; t < nb; ++t) {
        auto const tids = combination_from_rank(n, K, t);
        double reduced = 0.;
        for (int64_t tu = 0; tu < ntuples; ++tu) {
            std::vector<int> tuple(K);
            int64_t rr = tu;
            for (int a = K - 1; a >= 0; --a) {
                tuple[a] = static_cast<int>(rr % n);
                rr /= n;
            }
            double value = 0.;
            double fv = 0.;
            if (unique_ids(n, tuple)) {
                std::vector<double> j(K * K);
                for (int row = 0; row < K; ++row)
                    for (int col = 0; col < K; ++col) {
                        double e[MAXN];
                        G.edge_vector(node, tids[col], e);
                        j[row * K + col] = e[tuple[row]];
                    }
                value = reduction_determinant(j, K) / factorial(K);
                std::vector<int> sorted(tuple);
                std::sort(sorted.begin(), sorted.end());
                std::vector<int> none;
                fv = permutation_sign(tuple, none) * form[combination_rank(n, sorted)];
            }
            reduced += value * fv;
        }
        out[t] = reduced;
    }
    return 0;
}

// Reconstruction<Primal>::run at one node.
// Ref: src/similie/exterior/reduction_and_reconstruction.hpp:814-892
int silo_reconstruct_primal(int n, int K, const silo_field* position, const int64_t* node, const double* cochain,
                            double* out)
{
    if (n < 1 || n > MAXN || K < 0 || K > n) return 1;
    Geometry const G {n, position, nullptr};
    G.reconstruct(node, K, cochain, out);
    return 0;
}

int silo_fill_hodge_star(int n, int k_in, const silo_field* position, const silo_field* metric,
                         silo_field* hodge)
{
    return fill_impl(n, k_in, position, metric, hodge);
}

int silo_apply_hodge_star(int n, int k_in, const silo_field* hodge, const silo_field* in, silo_field* out)
{
    int dims[MAXD];
    for (int d = 0; d < n; ++d) dims[d] = d;
    if (in->ncomp != binom(n, k_in) || out->ncomp != binom(n, n - k_in)) return -1;
    apply_field(n, dims, k_in, *hodge, *in, *out);
    return 0;
}

int silo_hodge_matrix(int n, int k_in, const silo_field* position, const silo_field* metric,
                      const int64_t* node, double* matrix)
{
    if (n < 1 || n > 3 || k_in < 0 || k_in > n) return -1;
    Geometry const geo {n, position, metric};
    int64_t const nk = binom(n, k_in), nq = binom(n, n - k_in);
    for (int64_t c = 0; c < nk; ++c) {
        double unit[8] = {0}, resp[8] = {0};
        unit[c] = 1.;
        geo.discrete_star(node, k_in, unit, resp);
        for (int64_t t = 0; t < nq; ++t) matrix[t * nk + c] = resp[t];
    }
    return 0;
}

int silo_codifferential(int n, int k, const silo_field* position, const silo_field* metric,
                        const silo_field* in, silo_field* out)
{
    if (k < 1 || k > n || n > 3) return -1;
    int dims[MAXD];
    for (int d = 0; d < n; ++d) dims[d] = d;
    std::vector<double> sh, sdh, sdual;
    silo_field hs = make_hodge_field(*position, n, k, sh);
    silo_field dhs = make_hodge_field(*position, n, n - k + 1, sdh);
    fill_impl(n, k, position, metric, &hs);
    fill_impl(n, n - k + 1, position, metric, &dhs);
    silo_field dual = make_buffer(*in, static_cast<int>(binom(n, n - k)), sdual);
    apply_field(n, dims, k, hs, *in, dual);
    transpose_star_field(n, dims, n - k, dhs, dual, *out, sign_negative(n, k));
    return 0;
}

int silo_laplacian_hodge_ncomp(int n, int k, int which)
{
    int const kin = hodge_kin(n, k, which);
    if (kin < 0 || kin > n || !hodge_needed(n, k, which)) return 0;
    return static_cast<int>(ipow(n, kin) * binom(n, n - kin));
}

int silo_laplacian_hodge_kin(int n, int k, int which)
{
    return hodge_kin(n, k, which);
}

int silo_laplacian(int n, int k, const silo_field* position, const silo_field* metric,
                   const silo_field* in, silo_field* out)
{
    if (n < 1 || n > 3 || k < 0 || k > n) return -1;
    std::vector<double> store[4];
    silo_field fields[4];
    LaplacianHodges hs {};
    for (int w = 0; w < 4; ++w) {
        if (!hodge_needed(n, k, w)) {
            hs.h[w] = nullptr;
            continue;
        }
        fields[w] = make_hodge_field(*position, n, hodge_kin(n, k, w), store[w]);
        fill_impl(n, hodge_kin(n, k, w), position, metric, &fields[w]);
        hs.h[w] = &fields[w];
    }
    return laplacian_impl(n, k, hs, in, out);
}

int silo_laplacian_prefilled(int n, int k, const silo_field* const* h, const silo_field* in, silo_field* out)
{
    LaplacianHodges hs {{h[0], h[1], h[2], h[3]}};
    return laplacian_impl(n, k, hs, in, out);
}

// ------------------------------------------------------------------ magnetostatics

// Ref: onelab_interface/magnetostatics_onelab.hpp:4491-4519
void silo_mag2d_node_mu(int64_t nx, int64_t ny, const double* cell_mu, double mu0, double* node_mu)
{
    int64_t const ncx = nx - 1, ncy = ny - 1;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            double acc = 0.;
            int64_t count = 0;
            for (int dj = -1; dj <= 0; ++dj) {
                for (int di = -1; di <= 0; ++di) {
                    int64_t const ci = i + di, cj = j + dj;
                    if (ci < 0 || cj < 0 || ci >= ncx || cj >= ncy) continue;
                    acc += cell_mu[ci + ncx * cj];
                    ++count;
                }
            }
            node_mu[i + nx * j] = count == 0 ? mu0 : acc / static_cast<double>(count);
        }
    }
}

// Ref: onelab_interface/magnetostatics_onelab.hpp:4414-4451
void silo_mag2d_rhs(int64_t nx, int64_t ny, const double* x, const double* y, const double* cell_j, double* rhs)
{
    int64_t const ncx = nx - 1, ncy = ny - 1;
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            bool const boundary = i == 0 || j == 0 || i + 1 == nx || j + 1 == ny;
            if (boundary) {
                rhs[i + nx * j] = 0.;
                continue;
            }
            double acc = 0.;
            for (int dj = -1; dj <= 0; ++dj) {
                for (int di = -1; di <= 0; ++di) {
                    int64_t const ci = i + di, cj = j + dj;
                    if (ci < 0 || cj < 0 || ci >= ncx || cj >= ncy) continue;
                    double const area = (x[ci + 1] - x[ci]) * (y[cj + 1] - y[cj]);
                    acc += 0.25 * area * cell_j[ci + ncx * cj];
                }
            }
            rhs[i + nx * j] = acc;
        }
    }
}

namespace {
inline double m0(int64_t nx, const double* a, int64_t i, int64_t j)
{
    double m = 0.;
    m += -1. * a[i + nx * j];
    m += 1. * a[i + nx * (j + 1)];
    return m;
}
inline double m1(int64_t nx, const double* a, int64_t i, int64_t j)
{
    double m = 0.;
    m += 1. * a[i + nx * j];
    m += -1. * a[(i + 1) + nx * j];
    return m;
}
} // namespace

// Moments criterion (default): residual += c * (moment / mu) over the
// interior sampled nodes whose moment stencil touches the row, in
// ascending sampled-row order, X moments then Y moments.
// Ref: onelab_interface/magnetostatics_onelab.hpp:1095-1258 (stencils), 1271-1426 (apply);
//      src/similie/physics/magnetostatics/magnetostatics_quantities.hpp:100-123
void silo_mag2d_apply(int64_t nx, int64_t ny, const double* mu, const double* a, double* y)
{
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t const row = i + nx * j;
            if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                y[row] = a[row];
                continue;
            }
            double residual = 0.;
            if (j - 1 >= 1) residual -= -1. * (m0(nx, a, i, j - 1) / mu[i + nx * (j - 1)]);
            residual -= 1. * (m0(nx, a, i, j) / mu[row]);
            if (i - 1 >= 1) residual -= 1. * (m1(nx, a, i - 1, j) / mu[(i - 1) + nx * j]);
            residual -= -1. * (m1(nx, a, i, j) / mu[row]);
            y[row] = residual;
        }
    }
}

void silo_mag2d_diagonal(int64_t nx, int64_t ny, const double* mu, double* diag)
{
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t const row = i + nx * j;
            if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                diag[row] = 1.;
                continue;
            }
            double d = 0.;
            if (j - 1 >= 1) d += 1. / mu[i + nx * (j - 1)];
            d += 1. / mu[row];
            if (i - 1 >= 1) d += 1. / mu[(i - 1) + nx * j];
            d += 1. / mu[row];
            diag[row] = d;
        }
    }
}

namespace {
double dot(int64_t n, const double* a, const double* b)
{
    double s = 0.;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}
} // namespace

// Jacobi-preconditioned CG from x0 = 0 with the stopping rule
// ||r_k|| <= tol * ||b|| (Ginkgo Cg + Jacobi + ResidualNorm reduction factor).
// Ref: src/similie/solvers/minimize_strong_formulation_residual.hpp:1028-1304, 1308-1382
int silo_mag2d_cg(int64_t nx, int64_t ny, const double* mu, const double* b, double* x, double tol,
                  int max_iter, double* final_rel)
{
    int64_t const n = nx * ny;
    std::vector<double> r(b, b + n), z(n), p(n), q(n), dinv(n);
    silo_mag2d_diagonal(nx, ny, mu, dinv.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        dinv[i] = 1. / dinv[i];
        x[i] = 0.;
        z[i] = dinv[i] * r[i];
        p[i] = z[i];
    }
    double const bnorm = std::sqrt(dot(n, b, b));
    double rz = dot(n, r.data(), z.data());
    int it = 0;
    double rnorm = bnorm;
    if (bnorm == 0.) {
        if (final_rel) *final_rel = 0.;
        return 0;
    }
    while (it < max_iter) {
        silo_mag2d_apply(nx, ny, mu, p.data(), q.data());
        double const alpha = rz / dot(n, p.data(), q.data());
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        ++it;
        rnorm = std::sqrt(dot(n, r.data(), r.data()));
        if (rnorm <= tol * bnorm) break;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
        double const rz_new = dot(n, r.data(), z.data());
        double const beta = rz_new / rz;
        rz = rz_new;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    if (final_rel) *final_rel = rnorm / bnorm;
    return it;
}

// ------------------------------------------------------------------ magnetostatics 3D

namespace {

// Reference local spacing: one-sided at the ends, central average inside.
// Ref: onelab_interface/magnetostatics_onelab.hpp:856-870
double local_spacing(const double* c, int64_t n, int64_t i)
{
    if (n < 2) return 1.0;
    if (i == 0) return c[1] - c[0];
    if (i + 1 == n) return c[n - 1] - c[n - 2];
    return 0.5 * (c[i + 1] - c[i - 1]);
}

struct Grid3
{
    int64_t nx, ny, nz;
    const double *x, *y, *z;
    bool interior(int64_t i, int64_t j, int64_t k) const
    {
        return i > 0 && j > 0 && k > 0 && i + 1 < nx && j + 1 < ny && k + 1 < nz;
    }
    int64_t node(int64_t i, int64_t j, int64_t k) const { return i + nx * (j + ny * k); }
};

// One entry of a moment stencil: coefficient of A(node, comp).
struct MomentTerm
{
    int64_t node;
    int comp;
    double coeff;
};

// Moment stencils B_m(s) = (curl A)_m at node s (m = x, y, z), as SimiLie's
// Coboundary::value builds them for the 2-form components yz, -(xz), xy,
// visiting the 2x2x2 block (x slowest) and the components in order and
// dropping columns on the Dirichlet boundary.
// Ref: onelab_interface/magnetostatics_onelab.hpp:1815-1900,
//      src/similie/physics/magnetostatics/magnetostatics_quantities.hpp:139-196
std::vector<MomentTerm> moment_stencil(Grid3 const& g, int64_t i, int64_t j, int64_t k, int m)
{
    // coefficients per (di, dj, dk, comp) of the curl component
    double coef[2][2][2][3] = {};
    if (m == 0) {  // B_x = -A_z(s) + A_y(s) + A_z(s+y) - A_y(s+z)
        coef[0][0][0][2] += -1; coef[0][0][0][1] += 1; coef[0][1][0][2] += 1; coef[0][0][1][1] += -1;
    } else if (m == 1) {  // B_y = -[-A_z(s) + A_x(s) + A_z(s+x) - A_x(s+z)]
        coef[0][0][0][2] += 1; coef[0][0][0][0] += -1; coef[1][0][0][2] += -1; coef[0][0][1][0] += 1;
    } else {  // B_z = -A_y(s) + A_x(s) + A_y(s+x) - A_x(s+y)
        coef[0][0][0][1] += -1; coef[0][0][0][0] += 1; coef[1][0][0][1] += 1; coef[0][1][0][0] += -1;
    }
    std::vector<MomentTerm> out;
    for (int di = 0; di < 2; ++di)
        for (int dj = 0; dj < 2; ++dj)
            for (int dk = 0; dk < 2; ++dk)
                for (int c = 0; c < 3; ++c) {
                    double const v = coef[di][dj][dk][c];
                    if (v == 0.0) continue;
                    int64_t const pi = i + di, pj = j + dj, pk = k + dk;
                    if (!g.interior(pi, pj, pk)) continue;
                    out.push_back({g.node(pi, pj, pk), c, v});
                }
    return out;
}

double hodge_b(Grid3 const& g, int64_t i, int64_t j, int64_t k, int m)
{
    double const dx = local_spacing(g.x, g.nx, i), dy = local_spacing(g.y, g.ny, j), dz = local_spacing(g.z, g.nz, k);
    if (m == 0) return dx / (dy * dz);
    if (m == 1) return dy / (dx * dz);
    return dz / (dx * dy);
}

double hodge_a(Grid3 const& g, int64_t i, int64_t j, int64_t k, int c)
{
    double const dx = local_spacing(g.x, g.nx, i), dy = local_spacing(g.y, g.ny, j), dz = local_spacing(g.z, g.nz, k);
    if (c == 0) return dy * dz / dx;
    if (c == 1) return dx * dz / dy;
    return dx * dy / dz;
}

// Transposed stencil lists of every DOF: (sampled node, moment component,
// coefficient), built by visiting the interior sampled nodes in ascending
// order (the reference fills them with atomics, so its order is not fixed).
struct Transposed
{
    std::vector<std::vector<std::tuple<int64_t, int, double>>> rows;
};

Transposed transposed_lists(Grid3 const& g)
{
    Transposed t;
    t.rows.resize(3 * g.nx * g.ny * g.nz);
    for (int64_t k = 1; k + 1 < g.nz; ++k)
        for (int64_t j = 1; j + 1 < g.ny; ++j)
            for (int64_t i = 1; i + 1 < g.nx; ++i)
                for (int m = 0; m < 3; ++m)
                    for (auto const& term : moment_stencil(g, i, j, k, m))
                        t.rows[3 * term.node + term.comp].push_back({g.node(i, j, k), m, term.coeff});
    return t;
}

double moment_value(Grid3 const& g, int64_t s, int m, const double* a)
{
    int64_t const i = s % g.nx, j = (s / g.nx) % g.ny, k = s / (g.nx * g.ny);
    double v = 0.0;
    for (auto const& term : moment_stencil(g, i, j, k, m)) v += term.coeff * a[3 * term.node + term.comp];
    return v;
}

} // namespace

extern "C" {

// Ref: onelab_interface/magnetostatics_onelab.hpp:5030-5067 (node mu, mean of adjacent cells)
void silo_mag3d_node_mu(int64_t nx, int64_t ny, int64_t nz, const double* cell_mu, double mu0, double* node_mu)
{
    int64_t const ncx = nx - 1, ncy = ny - 1, ncz = nz - 1;
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                double acc = 0.0;
                int64_t cnt = 0;
                for (int dk = -1; dk <= 0; ++dk)
                    for (int dj = -1; dj <= 0; ++dj)
                        for (int di = -1; di <= 0; ++di) {
                            int64_t const ci = i + di, cj = j + dj, ck = k + dk;
                            if (ci < 0 || cj < 0 || ck < 0 || ci >= ncx || cj >= ncy || ck >= ncz) continue;
                            acc += cell_mu[ci + ncx * (cj + ncy * ck)];
                            ++cnt;
                        }
                node_mu[i + nx * (j + ny * k)] = cnt == 0 ? mu0 : acc / static_cast<double>(cnt);
            }
}

// Ref: onelab_interface/magnetostatics_onelab.hpp:4919-4975
void silo_mag3d_rhs(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                    const double* cell_j, double* rhs)
{
    int64_t const ncx = nx - 1, ncy = ny - 1, ncz = nz - 1;
    for (int64_t k = 0; k < nz; ++k)
        for (int64_t j = 0; j < ny; ++j)
            for (int64_t i = 0; i < nx; ++i) {
                int64_t const node = i + nx * (j + ny * k);
                bool const boundary = i == 0 || j == 0 || k == 0 || i + 1 == nx || j + 1 == ny || k + 1 == nz;
                for (int c = 0; c < 3; ++c) {
                    double acc = 0.0;
                    if (!boundary) {
                        for (int dk = -1; dk <= 0; ++dk)
                            for (int dj = -1; dj <= 0; ++dj)
                                for (int di = -1; di <= 0; ++di) {
                                    int64_t const ci = i + di, cj = j + dj, ck = k + dk;
                                    if (ci < 0 || cj < 0 || ck < 0 || ci >= ncx || cj >= ncy || ck >= ncz) continue;
                                    double const wx = x[ci + 1] - x[ci], wy = y[cj + 1] - y[cj], wz = z[ck + 1] - z[ck];
                                    double face = wx * wy;
                                    if (c == 0) face = wy * wz;
                                    else if (c == 1) face = wx * wz;
                                    acc += 0.125 * face * cell_j[3 * (ci + ncx * (cj + ncy * ck)) + c];
                                }
                    }
                    rhs[3 * node + c] = acc;
                }
            }
}

// Ref: onelab_interface/magnetostatics_onelab.hpp:2242-2396 (precomputed-stencil apply,
// Coulomb-gauge penalty gamma * H_A * A; y-response sign and divergence gauge at their defaults)
void silo_mag3d_apply(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                      const double* node_mu, double gamma, const double* a, double* out)
{
    Grid3 const g {nx, ny, nz, x, y, z};
    Transposed const t = transposed_lists(g);
    int64_t const nn = nx * ny * nz;
#pragma omp parallel for schedule(static)
    for (int64_t node = 0; node < nn; ++node) {
        int64_t const i = node % nx, j = (node / nx) % ny, k = node / (nx * ny);
        for (int c = 0; c < 3; ++c) {
            int64_t const row = 3 * node + c;
            if (!g.interior(i, j, k)) {
                out[row] = a[row];
                continue;
            }
            double residual = 0.0;
            for (auto const& [s, m, coeff] : t.rows[row]) {
                int64_t const si = s % nx, sj = (s / nx) % ny, sk = s / (nx * ny);
                residual += coeff * hodge_b(g, si, sj, sk, m) * (moment_value(g, s, m, a) / node_mu[s]);
            }
            double const gauge = gamma * hodge_a(g, i, j, k, c) * a[row];
            out[row] = residual + gauge;
        }
    }
}

void silo_mag3d_diagonal(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                         const double* node_mu, double gamma, double* diag)
{
    Grid3 const g {nx, ny, nz, x, y, z};
    Transposed const t = transposed_lists(g);
    int64_t const nn = nx * ny * nz;
    for (int64_t node = 0; node < nn; ++node) {
        int64_t const i = node % nx, j = (node / nx) % ny, k = node / (nx * ny);
        for (int c = 0; c < 3; ++c) {
            int64_t const row = 3 * node + c;
            if (!g.interior(i, j, k)) {
                diag[row] = 1.0;
                continue;
            }
            double d = 0.0;
            for (auto const& [s, m, coeff] : t.rows[row]) {
                int64_t const si = s % nx, sj = (s / nx) % ny, sk = s / (nx * ny);
                d += coeff * coeff * hodge_b(g, si, sj, sk, m) / node_mu[s];
            }
            diag[row] = d + gamma * hodge_a(g, i, j, k, c);
        }
    }
}


} // extern "C"

int silo_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

} // extern "C"

// ------------------------------------------------------------------ magnetostatics 2D, nonlinear material

namespace {

// Interpolated B-H curve: h piecewise linear in b, intervals bracketed by q = b^2.
// Ref: src/similie/physics/magnetostatics/nonlinear_magnetostatics.py:14-181
// (InterpolatedNonlinearBHCurve: constructor, bracket_q, h_from_b,
// dh_db_from_b, h_over_b_from_b and its b- and q-derivatives).
struct BHCurve
{
    int n = 0;
    std::vector<double> b, h, q, dh_db;

    BHCurve(int n_, const double* b_, const double* h_) : n(n_), b(b_, b_ + n_), h(h_, h_ + n_), q(n_), dh_db(n_ - 1)
    {
        for (int i = 0; i < n; ++i) q[i] = b[i] * b[i];
        for (int i = 0; i + 1 < n; ++i) dh_db[i] = (h[i + 1] - h[i]) / (b[i + 1] - b[i]);
    }
    int bracket_q(double qv) const
    {
        if (qv <= q[0]) return 0;
        for (int i = 0; i + 1 < n; ++i)
            if (qv <= q[i + 1]) return i;
        return n - 2;
    }
    double h_from_b(double bv) const
    {
        if (bv <= b[0]) return h[0];
        if (bv >= b[n - 1]) {
            int const k = n - 2;
            return h[k] + dh_db[k] * (bv - b[k]);
        }
        int const k = bracket_q(bv * bv);
        return h[k] + dh_db[k] * (bv - b[k]);
    }
    double dh_db_from_b(double bv) const
    {
        if (bv <= b[0]) return dh_db[0];
        if (bv >= b[n - 1]) return dh_db[n - 2];
        return dh_db[bracket_q(bv * bv)];
    }
    double h_over_b_from_b(double bv) const { return bv == 0.0 ? dh_db_from_b(0.0) : h_from_b(bv) / bv; }
    double d1_b(double bv) const
    {
        if (bv == 0.0) return 0.0;
        return (dh_db_from_b(bv) * bv - h_from_b(bv)) / (bv * bv);
    }
    double d2_b(double bv) const
    {
        if (bv == 0.0) return 0.0;
        double const intercept = h_from_b(bv) - dh_db_from_b(bv) * bv;
        return 2.0 * intercept / (bv * bv * bv);
    }
    double f(double qv) const { return h_over_b_from_b(std::sqrt(qv)); }
    double df(double qv) const
    {
        if (qv == 0.0) return 0.0;
        double const bv = std::sqrt(qv);
        return d1_b(bv) / (2.0 * bv);
    }
    double d2f(double qv) const
    {
        if (qv == 0.0) return 0.0;
        double const bv = std::sqrt(qv);
        return d2_b(bv) / (4.0 * qv) - d1_b(bv) / (4.0 * qv * bv);
    }
};

// dH/dB_c and d2H/dB_r dB_c at a sampled node.  Ferromagnetic nodes use the
// Hamiltonian q F(q) / 2 (F = h/b, q = |B|^2): dH/dB_c = B_c F + q B_c F',
// d2H/dB_r dB_c = delta_rc (F + q F') + 4 B_r B_c F' + 2 q B_r B_c F''; the
// others B_c / mu.
// Ref: onelab_interface/magnetostatics_onelab.hpp:957-1011
// (MaterialMagnetostaticsHamiltonian); the Hamiltonian and its derivatives:
// src/similie/physics/magnetostatics/nonlinear_magnetostatics.py:331-369,
// src/similie/physics/generate_cpp_hamiltonian.py:280-400.
struct NodeLaw
{
    const double* mu;
    const double* ferro;
    BHCurve const* curve;
    void field(int64_t s, double b0, double b1, double* h0, double* h1) const
    {
        if (ferro[s] > 0.5) {
            double const q = b0 * b0 + b1 * b1;
            double const F = curve->f(q), dF = curve->df(q);
            *h0 = b0 * F + q * b0 * dF;
            *h1 = b1 * F + q * b1 * dF;
        } else {
            *h0 = b0 / mu[s];
            *h1 = b1 / mu[s];
        }
    }
    void jacobian(int64_t s, double b0, double b1, double* j00, double* j01, double* j11) const
    {
        if (ferro[s] > 0.5) {
            double const q = b0 * b0 + b1 * b1;
            double const F = curve->f(q), dF = curve->df(q), d2F = curve->d2f(q);
            double const base = F + q * dF;
            *j00 = base + 4.0 * b0 * b0 * dF + 2.0 * q * b0 * b0 * d2F;
            *j11 = base + 4.0 * b1 * b1 * dF + 2.0 * q * b1 * b1 * d2F;
            *j01 = 4.0 * b0 * b1 * dF + 2.0 * q * b0 * b1 * d2F;
        } else {
            *j00 = 1.0 / mu[s];
            *j11 = 1.0 / mu[s];
            *j01 = 0.0;
        }
    }
};

double nrm2(int64_t n, const double* v)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; ++i) s += v[i] * v[i];
    return std::sqrt(s);
}

double dotp(int64_t n, const double* a, const double* b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

// Nonlinear operator, same sampled nodes and order as silo_mag2d_apply.
// Ref: onelab_interface/magnetostatics_onelab.hpp:1271-1426 (moments criterion)
void nl_apply(int64_t nx, int64_t ny, NodeLaw const& law, const double* a, double* y)
{
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t const row = i + nx * j;
            if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                y[row] = a[row];
                continue;
            }
            double residual = 0.0, h0, h1;
            if (j - 1 >= 1) {
                law.field(row - nx, m0(nx, a, i, j - 1), m1(nx, a, i, j - 1), &h0, &h1);
                residual -= -1. * h0;
            }
            law.field(row, m0(nx, a, i, j), m1(nx, a, i, j), &h0, &h1);
            residual -= 1. * h0;
            if (i - 1 >= 1) {
                law.field(row - 1, m0(nx, a, i - 1, j), m1(nx, a, i - 1, j), &h0, &h1);
                residual -= 1. * h1;
            }
            law.field(row, m0(nx, a, i, j), m1(nx, a, i, j), &h0, &h1);
            residual -= -1. * h1;
            y[row] = residual;
        }
    }
}

// Jacobian apply: every sampled node contributes (-outer coefficient) x the
// row (X) or second row (Y) of its 2x2 Jacobian times the moments of x.
// Ref: onelab_interface/magnetostatics_onelab.hpp:2799-2915 (apply_jacobian, 2D)
void nl_jacobian_apply(int64_t nx, int64_t ny, NodeLaw const& law, const double* st, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t const row = i + nx * j;
            if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                y[row] = x[row];
                continue;
            }
            double residual = 0.0, j00, j01, j11;
            auto add = [&](double c, int64_t si, int64_t sj, bool first) {
                law.jacobian(si + nx * sj, m0(nx, st, si, sj), m1(nx, st, si, sj), &j00, &j01, &j11);
                double const d0 = m0(nx, x, si, sj), d1 = m1(nx, x, si, sj);
                residual += c * (first ? (j00 * d0 + j01 * d1) : (j01 * d0 + j11 * d1));
            };
            if (j - 1 >= 1) add(1.0, i, j - 1, true);
            add(-1.0, i, j, true);
            if (i - 1 >= 1) add(-1.0, i - 1, j, false);
            add(1.0, i, j, false);
            y[row] = residual;
        }
    }
}

void nl_jacobian_diagonal(int64_t nx, int64_t ny, NodeLaw const& law, const double* st, double* diag)
{
#pragma omp parallel for schedule(static)
    for (int64_t j = 0; j < ny; ++j) {
        for (int64_t i = 0; i < nx; ++i) {
            int64_t const row = i + nx * j;
            if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                diag[row] = 1.0;
                continue;
            }
            double d = 0.0, j00, j01, j11;
            if (j - 1 >= 1) {
                law.jacobian(row - nx, m0(nx, st, i, j - 1), m1(nx, st, i, j - 1), &j00, &j01, &j11);
                d += j00;
            }
            law.jacobian(row, m0(nx, st, i, j), m1(nx, st, i, j), &j00, &j01, &j11);
            d += j00 - j01;
            if (i - 1 >= 1) {
                law.jacobian(row - 1, m0(nx, st, i - 1, j), m1(nx, st, i - 1, j), &j00, &j01, &j11);
                d += j11;
            }
            law.jacobian(row, m0(nx, st, i, j), m1(nx, st, i, j), &j00, &j01, &j11);
            d += j11 - j01;
            diag[row] = d;
        }
    }
}

} // namespace

void silo_bh_eval(int n, const double* b, const double* h, int count, const double* q, double* f, double* df,
                  double* d2f)
{
    BHCurve const c(n, b, h);
    for (int i = 0; i < count; ++i) {
        f[i] = c.f(q[i]);
        df[i] = c.df(q[i]);
        d2f[i] = c.d2f(q[i]);
    }
}

void silo_mag2d_nl_apply(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                         const double* b, const double* h, const double* a, double* y)
{
    BHCurve const c(n, b, h);
    NodeLaw const law {node_mu, node_ferro, &c};
    nl_apply(nx, ny, law, a, y);
}

void silo_mag2d_nl_jacobian_apply(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                                  const double* b, const double* h, const double* state, const double* x,
                                  double* y)
{
    BHCurve const c(n, b, h);
    NodeLaw const law {node_mu, node_ferro, &c};
    nl_jacobian_apply(nx, ny, law, state, x, y);
}

void silo_mag2d_nl_jacobian_diagonal(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro,
                                     int n, const double* b, const double* h, const double* state, double* diag)
{
    BHCurve const c(n, b, h);
    NodeLaw const law {node_mu, node_ferro, &c};
    nl_jacobian_diagonal(nx, ny, law, state, diag);
}

namespace {

// Newton with a halving line search on F(x) = rhs; every step solves
// J(x) d = r by Jacobi-CG from d = 0 to the relative tolerance.
// Ref: src/similie/solvers/minimize_strong_formulation_residual.hpp:1383-1569
// (nonlinear branch: at most 30 Newton steps; each solves the linearised
// system to the relative tolerance, then a line search of at most 8 steps
// halving alpha from 1 that stops at the first candidate below the current
// residual, else takes the best candidate seen).
// The outer loop: step(x, r, d) solves J(x) d = r from d = 0 and returns its
// CG iterations.
template <class Apply, class Step>
int newton_core(int64_t N, Apply const& apply, Step const& step, const double* rhs, double* x, double tol,
                int* newton_steps, double* final_rel)
{
    std::vector<double> fa(N), r(N), d(N), cand(N), cand_f(N), cand_r(N);
    apply(x, fa.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) r[i] = rhs[i] - fa[i];
    double const r0 = nrm2(N, r.data());
    int total = 0, steps = 0;
    if (r0 == 0.0) {
        *newton_steps = 0;
        *final_rel = 0.0;
        return 0;
    }
    for (int it = 0; it < 30; ++it) {
        double const res = nrm2(N, r.data());
        if (res / r0 <= tol) break;
        ++steps;
        total += step(x, r.data(), d.data());
        // line search
        double const cur = nrm2(N, r.data());
        double alpha = 1.0, best_alpha = 0.0, best = std::numeric_limits<double>::infinity();
        auto candidate = [&](double al) {
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) cand[i] = x[i] + al * d[i];
            apply(cand.data(), cand_f.data());
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < N; ++i) cand_r[i] = rhs[i] - cand_f[i];
            return nrm2(N, cand_r.data());
        };
        for (int ls = 0; ls < 8; ++ls) {
            double const nr = candidate(alpha);
            if (nr < best) {
                best = nr;
                best_alpha = alpha;
            }
            if (nr < cur) break;
            alpha *= 0.5;
        }
        if (best_alpha != alpha) {
            alpha = best_alpha;
            candidate(alpha);
        }
        std::copy(cand.begin(), cand.end(), x);
        r = cand_r;
    }
    *newton_steps = steps;
    *final_rel = nrm2(N, r.data()) / r0;
    return total;
}

// Jacobi-CG on J(x) d = r from d = 0 to the relative tolerance (the
// matrix-free linear solve of the nonlinear branch).
template <class Jacobian, class Diagonal>
int jacobi_cg_step(int64_t N, Jacobian const& jacobian, Diagonal const& diagonal, const double* x, const double* r,
                   double* d, double tol, int max_iter)
{
    std::vector<double> dinv(N), cr(r, r + N), z(N), p(N), q(N);
    diagonal(x, dinv.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) dinv[i] = 1.0 / dinv[i];
    std::fill(d, d + N, 0.0);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < N; ++i) z[i] = dinv[i] * cr[i];
    p = z;
    double rz = dotp(N, cr.data(), z.data());
    double const bn = nrm2(N, r);
    double rn = bn;
    int k = 0;
    while (k < max_iter && rn > tol * bn) {
        jacobian(x, p.data(), q.data());
        double const alpha = rz / dotp(N, p.data(), q.data());
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) {
            d[i] += alpha * p[i];
            cr[i] -= alpha * q[i];
        }
        ++k;
        rn = nrm2(N, cr.data());
        if (rn <= tol * bn) break;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) z[i] = dinv[i] * cr[i];
        double const rz2 = dotp(N, cr.data(), z.data());
        double const beta = rz2 / rz;
        rz = rz2;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < N; ++i) p[i] = z[i] + beta * p[i];
    }
    return k;
}

// Newton with a halving line search on F(x) = rhs; every step solves
// J(x) d = r by Jacobi-CG from d = 0 to the relative tolerance.
// Ref: src/similie/solvers/minimize_strong_formulation_residual.hpp:1383-1569
// (nonlinear branch: at most 30 Newton steps; each solves the linearised
// system to the relative tolerance, then a line search of at most 8 steps
// halving alpha from 1 that stops at the first candidate below the current
// residual, else takes the best candidate seen).
// prepare(x) returns the Jacobian at x with apply(v, out) and diagonal(out);
// its coefficients are evaluated once per Newton step, as on the GPU.
template <class Apply, class Prepare>
int newton_solve(int64_t N, Apply const& apply, Prepare const& prepare, const double* rhs, double* x, double tol,
                 int max_iter, int* newton_steps, double* final_rel)
{
    return newton_core(
            N, apply,
            [&](const double* xs, const double* r, double* d) {
                auto const J = prepare(xs);
                return jacobi_cg_step(
                        N, [&](const double*, const double* v, double* out) { J.apply(v, out); },
                        [&](const double*, double* out) { J.diagonal(out); }, xs, r, d, tol, max_iter);
            },
            rhs, x, tol, newton_steps, final_rel);
}

// The 2D Jacobian with the nodes' 2x2 blocks evaluated once at the state;
// apply and diagonal repeat nl_jacobian_apply / nl_jacobian_diagonal term
// by term.
struct Jac2
{
    int64_t nx, ny;
    std::vector<double> c00, c01, c11;
    Jac2(int64_t nx_, int64_t ny_, NodeLaw const& law, const double* st)
        : nx(nx_), ny(ny_), c00(nx_ * ny_, 0.0), c01(nx_ * ny_, 0.0), c11(nx_ * ny_, 0.0)
    {
#pragma omp parallel for schedule(static)
        for (int64_t j = 1; j < ny - 1; ++j)
            for (int64_t i = 1; i < nx - 1; ++i) {
                int64_t const s = i + nx * j;
                law.jacobian(s, m0(nx, st, i, j), m1(nx, st, i, j), &c00[s], &c01[s], &c11[s]);
            }
    }
    void apply(const double* x, double* y) const
    {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < ny; ++j) {
            for (int64_t i = 0; i < nx; ++i) {
                int64_t const row = i + nx * j;
                if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                    y[row] = x[row];
                    continue;
                }
                double residual = 0.0;
                auto add = [&](double c, int64_t si, int64_t sj, bool first) {
                    int64_t const s = si + nx * sj;
                    double const d0 = m0(nx, x, si, sj), d1 = m1(nx, x, si, sj);
                    residual += c * (first ? (c00[s] * d0 + c01[s] * d1) : (c01[s] * d0 + c11[s] * d1));
                };
                if (j - 1 >= 1) add(1.0, i, j - 1, true);
                add(-1.0, i, j, true);
                if (i - 1 >= 1) add(-1.0, i - 1, j, false);
                add(1.0, i, j, false);
                y[row] = residual;
            }
        }
    }
    void diagonal(double* diag) const
    {
#pragma omp parallel for schedule(static)
        for (int64_t j = 0; j < ny; ++j) {
            for (int64_t i = 0; i < nx; ++i) {
                int64_t const row = i + nx * j;
                if (i == 0 || j == 0 || i + 1 == nx || j + 1 == ny) {
                    diag[row] = 1.0;
                    continue;
                }
                double d = 0.0;
                if (j - 1 >= 1) d += c00[row - nx];
                d += c00[row] - c01[row];
                if (i - 1 >= 1) d += c11[row - 1];
                d += c11[row] - c01[row];
                diag[row] = d;
            }
        }
    }
};

// 3D material law at a sampled node with moments B = (B_x, B_y, B_z):
// the same Hamiltonian as NodeLaw with q = |B|^2 over three components.
struct NodeLaw3
{
    const double* mu;
    const double* ferro;
    BHCurve const* curve;
    void field(int64_t s, const double* B, double* H) const
    {
        if (ferro[s] > 0.5) {
            double const q = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
            double const F = curve->f(q), dF = curve->df(q);
            for (int c = 0; c < 3; ++c) H[c] = B[c] * F + q * B[c] * dF;
        } else {
            for (int c = 0; c < 3; ++c) H[c] = B[c] / mu[s];
        }
    }
    // J[3 * r + c] = d2H / dB_r dB_c
    void jacobian(int64_t s, const double* B, double* J) const
    {
        if (ferro[s] > 0.5) {
            double const q = B[0] * B[0] + B[1] * B[1] + B[2] * B[2];
            double const F = curve->f(q), dF = curve->df(q), d2F = curve->d2f(q);
            double const base = F + q * dF;
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c)
                    J[3 * r + c] = (r == c ? base : 0.0) + 4.0 * B[r] * B[c] * dF + 2.0 * q * B[r] * B[c] * d2F;
        } else {
            for (int r = 0; r < 3; ++r)
                for (int c = 0; c < 3; ++c) J[3 * r + c] = r == c ? 1.0 / mu[s] : 0.0;
        }
    }
};

struct Mag3Nl
{
    Grid3 g;
    Transposed t;
    NodeLaw3 law;
    double gamma;
    // per interior sampled node s and moment m: its stencil terms
    // [sptr[3 s + m], sptr[3 s + m + 1]) in moment_stencil's order, and the
    // Hodge factors hodge_b(s, m), hodge_a(s, c) (3 per node each)
    std::vector<int64_t> sptr;
    std::vector<MomentTerm> sterm;
    std::vector<double> hb, ha;

    void prepare()
    {
        int64_t const nn = g.nx * g.ny * g.nz;
        sptr.assign(3 * nn + 1, 0);
        hb.assign(3 * nn, 0.0);
        ha.assign(3 * nn, 0.0);
        for (int64_t s = 0; s < nn; ++s) {
            int64_t const i = s % g.nx, j = (s / g.nx) % g.ny, k = s / (g.nx * g.ny);
            for (int m = 0; m < 3; ++m) {
                if (g.interior(i, j, k))
                    for (auto const& term : moment_stencil(g, i, j, k, m)) sterm.push_back(term);
                sptr[3 * s + m + 1] = static_cast<int64_t>(sterm.size());
                hb[3 * s + m] = hodge_b(g, i, j, k, m);
                ha[3 * s + m] = hodge_a(g, i, j, k, m);
            }
        }
    }
    double moment(int64_t s, int m, const double* a) const
    {
        double v = 0.0;
        for (int64_t e = sptr[3 * s + m]; e < sptr[3 * s + m + 1]; ++e)
            v += sterm[e].coeff * a[3 * sterm[e].node + sterm[e].comp];
        return v;
    }
    void moments(int64_t s, const double* a, double* B) const
    {
        for (int m = 0; m < 3; ++m) B[m] = moment(s, m, a);
    }
    bool interior_node(int64_t s) const
    {
        return g.interior(s % g.nx, (s / g.nx) % g.ny, s / (g.nx * g.ny));
    }
    // out[row] = sum over the row's transposed moment entries (s, m, coeff)
    // of coeff * hodge_b(s, m) * v[3 s + m] + gamma * hodge_a * a[row];
    // identity rows on the boundary.
    void gather(const double* v, const double* a, double* out) const
    {
        int64_t const nn = g.nx * g.ny * g.nz;
#pragma omp parallel for schedule(static)
        for (int64_t node = 0; node < nn; ++node) {
            int64_t const i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
            for (int c = 0; c < 3; ++c) {
                int64_t const row = 3 * node + c;
                if (!g.interior(i, j, k)) {
                    out[row] = a[row];
                    continue;
                }
                double residual = 0.0;
                for (auto const& [s, m, coeff] : t.rows[row]) residual += coeff * hb[3 * s + m] * v[3 * s + m];
                out[row] = residual + gamma * ha[3 * node + c] * a[row];
            }
        }
    }
    // Nonlinear operator: the linear 3D operator with B_m / mu replaced by
    // the material field H_m(B) at the sampled nodes.
    // Ref: onelab_interface/magnetostatics_onelab.hpp:2241-2396 (3D apply with
    // dpotential_dt of the equations), 957-1011 (material Hamiltonian)
    void apply(const double* a, double* y) const
    {
        int64_t const nn = g.nx * g.ny * g.nz;
        std::vector<double> H(3 * nn, 0.0);
#pragma omp parallel for schedule(static)
        for (int64_t s = 0; s < nn; ++s) {
            if (!interior_node(s)) continue;
            double B[3];
            moments(s, a, B);
            law.field(s, B, &H[3 * s]);
        }
        gather(H.data(), a, y);
    }
    // Jacobian at st applied to x: each sampled node contributes its 3x3
    // Hessian times the moments of x.
    // Ref: onelab_interface/magnetostatics_onelab.hpp:2924-3110 (apply_jacobian, 3D)
    void jacobian(const double* st, const double* x, double* y) const
    {
        int64_t const nn = g.nx * g.ny * g.nz;
        std::vector<double> G(3 * nn, 0.0);
#pragma omp parallel for schedule(static)
        for (int64_t s = 0; s < nn; ++s) {
            if (!interior_node(s)) continue;
            double B[3], D[3], J[9];
            moments(s, st, B);
            moments(s, x, D);
            law.jacobian(s, B, J);
            for (int m = 0; m < 3; ++m) G[3 * s + m] = J[3 * m] * D[0] + J[3 * m + 1] * D[1] + J[3 * m + 2] * D[2];
        }
        gather(G.data(), x, y);
    }
    // The Jacobian at st with every sampled node's 3x3 block evaluated once
    // (the same values jacobian / diagonal compute per call).
    struct Prepared
    {
        Mag3Nl const* op;
        std::vector<double> J;  // 9 per node
        void apply(const double* x, double* y) const
        {
            Mag3Nl const& o = *op;
            int64_t const nn = o.g.nx * o.g.ny * o.g.nz;
            std::vector<double> G(3 * nn, 0.0);
#pragma omp parallel for schedule(static)
            for (int64_t s = 0; s < nn; ++s) {
                if (!o.interior_node(s)) continue;
                double D[3];
                o.moments(s, x, D);
                double const* Js = &J[9 * s];
                for (int m = 0; m < 3; ++m)
                    G[3 * s + m] = Js[3 * m] * D[0] + Js[3 * m + 1] * D[1] + Js[3 * m + 2] * D[2];
            }
            o.gather(G.data(), x, y);
        }
        void diagonal(double* diag) const { op->diagonal_with(J.data(), diag); }
    };
    Prepared prepare_jacobian(const double* st) const
    {
        int64_t const nn = g.nx * g.ny * g.nz;
        Prepared p {this, std::vector<double>(9 * nn, 0.0)};
#pragma omp parallel for schedule(static)
        for (int64_t s = 0; s < nn; ++s) {
            if (!interior_node(s)) continue;
            double B[3];
            moments(s, st, B);
            law.jacobian(s, B, &p.J[9 * s]);
        }
        return p;
    }
    // Diagonal from precomputed node blocks Jn (9 per node): for each entry
    // (s, m, coeff) of the row, coeff * hodge_b(s, m) * sum_c J_mc(s) *
    // (coefficient of the row in B_c(s)); plus the gauge term; 1 on boundary
    // rows.
    void diagonal_with(const double* Jn, double* diag) const
    {
        int64_t const nn = g.nx * g.ny * g.nz;
#pragma omp parallel for schedule(static)
        for (int64_t node = 0; node < nn; ++node) {
            int64_t const i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
            for (int c = 0; c < 3; ++c) {
                int64_t const row = 3 * node + c;
                if (!g.interior(i, j, k)) {
                    diag[row] = 1.0;
                    continue;
                }
                double d = 0.0;
                for (auto const& [s, m, coeff] : t.rows[row]) {
                    double const* J = Jn + 9 * s;
                    double acc = 0.0;
                    for (int cc = 0; cc < 3; ++cc)
                        for (int64_t e = sptr[3 * s + cc]; e < sptr[3 * s + cc + 1]; ++e)
                            if (sterm[e].node == node && sterm[e].comp == c) acc += J[3 * m + cc] * sterm[e].coeff;
                    d += coeff * hb[3 * s + m] * acc;
                }
                diag[row] = d + gamma * ha[3 * node + c];
            }
        }
    }
    // Diagonal of the Jacobian at st: for each entry (s, m, coeff) of the
    // row, coeff * hodge_b(s, m) * sum_c J_mc(s) * (coefficient of the row in
    // B_c(s)); plus the gauge term; 1 on boundary rows.
    void diagonal(const double* st, double* diag) const
    {
        int64_t const nn = g.nx * g.ny * g.nz;
#pragma omp parallel for schedule(static)
        for (int64_t node = 0; node < nn; ++node) {
            int64_t const i = node % g.nx, j = (node / g.nx) % g.ny, k = node / (g.nx * g.ny);
            for (int c = 0; c < 3; ++c) {
                int64_t const row = 3 * node + c;
                if (!g.interior(i, j, k)) {
                    diag[row] = 1.0;
                    continue;
                }
                double d = 0.0;
                for (auto const& [s, m, coeff] : t.rows[row]) {
                    double B[3], J[9];
                    moments(s, st, B);
                    law.jacobian(s, B, J);
                    double acc = 0.0;
                    for (int cc = 0; cc < 3; ++cc)
                        for (int64_t e = sptr[3 * s + cc]; e < sptr[3 * s + cc + 1]; ++e)
                            if (sterm[e].node == node && sterm[e].comp == c) acc += J[3 * m + cc] * sterm[e].coeff;
                    d += coeff * hb[3 * s + m] * acc;
                }
                diag[row] = d + gamma * ha[3 * node + c];
            }
        }
    }
};

Mag3Nl make_mag3nl(Grid3 const& g, NodeLaw3 const& law, double gamma)
{
    Mag3Nl op {g, transposed_lists(g), law, gamma, {}, {}, {}, {}};
    op.prepare();
    return op;
}

} // namespace

// Ref: the linear 3D CG of silo_mag3d_apply (Jacobi, x0 = 0), the
// operator's stencil tables built once per solve.
int silo_mag3d_cg(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                  const double* node_mu, double gamma, const double* b, double* sol, double tol, int max_iter,
                  double* final_rel)
{
    int64_t const n = 3 * nx * ny * nz;
    // the operator of silo_mag3d_apply, its stencil tables built once
    Grid3 const g {nx, ny, nz, x, y, z};
    std::vector<double> const no_ferro(nx * ny * nz, 0.0);
    Mag3Nl const op = make_mag3nl(g, NodeLaw3 {node_mu, no_ferro.data(), nullptr}, gamma);
    std::vector<double> r(b, b + n), zv(n), p(n), q(n), dinv(n);
    silo_mag3d_diagonal(nx, ny, nz, x, y, z, node_mu, gamma, dinv.data());
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
        dinv[i] = 1. / dinv[i];
        sol[i] = 0.;
        zv[i] = dinv[i] * r[i];
        p[i] = zv[i];
    }
    double const bnorm = std::sqrt(dot(n, b, b));
    if (bnorm == 0.) {
        if (final_rel) *final_rel = 0.;
        return 0;
    }
    double rz = dot(n, r.data(), zv.data());
    double rnorm = bnorm;
    int it = 0;
    while (it < max_iter) {
        op.apply(p.data(), q.data());
        double const alpha = rz / dot(n, p.data(), q.data());
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            sol[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        ++it;
        rnorm = std::sqrt(dot(n, r.data(), r.data()));
        if (rnorm <= tol * bnorm) break;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) zv[i] = dinv[i] * r[i];
        double const rz_new = dot(n, r.data(), zv.data());
        double const beta = rz_new / rz;
        rz = rz_new;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = zv[i] + beta * p[i];
    }
    if (final_rel) *final_rel = rnorm / bnorm;
    return it;
}

int silo_mag2d_nl_solve(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                        const double* b, const double* h, const double* rhs, double* x, double tol, int max_iter,
                        int* newton_steps, double* final_rel)
{
    BHCurve const c(n, b, h);
    NodeLaw const law {node_mu, node_ferro, &c};
    return newton_solve(
            nx * ny, [&](const double* v, double* out) { nl_apply(nx, ny, law, v, out); },
            [&](const double* st) { return Jac2(nx, ny, law, st); }, rhs, x, tol, max_iter, newton_steps, final_rel);
}

void silo_mag3d_nl_apply(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                         const double* node_mu, const double* node_ferro, double gamma, int n, const double* b,
                         const double* h, const double* a, double* out)
{
    BHCurve const c(n, b, h);
    Grid3 const g {nx, ny, nz, x, y, z};
    Mag3Nl const op = make_mag3nl(g, NodeLaw3 {node_mu, node_ferro, &c}, gamma);
    op.apply(a, out);
}

void silo_mag3d_nl_jacobian_apply(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y,
                                  const double* z, const double* node_mu, const double* node_ferro, double gamma,
                                  int n, const double* b, const double* h, const double* state, const double* v,
                                  double* out)
{
    BHCurve const c(n, b, h);
    Grid3 const g {nx, ny, nz, x, y, z};
    Mag3Nl const op = make_mag3nl(g, NodeLaw3 {node_mu, node_ferro, &c}, gamma);
    op.jacobian(state, v, out);
}

void silo_mag3d_nl_jacobian_diagonal(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y,
                                     const double* z, const double* node_mu, const double* node_ferro, double gamma,
                                     int n, const double* b, const double* h, const double* state, double* diag)
{
    BHCurve const c(n, b, h);
    Grid3 const g {nx, ny, nz, x, y, z};
    Mag3Nl const op = make_mag3nl(g, NodeLaw3 {node_mu, node_ferro, &c}, gamma);
    op.diagonal(state, diag);
}

int silo_mag3d_nl_solve(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                        const double* node_mu, const double* node_ferro, double gamma, int n, const double* b,
                        const double* h, const double* rhs, double* sol, double tol, int max_iter, int* newton_steps,
                        double* final_rel)
{
    BHCurve const c(n, b, h);
    Grid3 const g {nx, ny, nz, x, y, z};
    Mag3Nl const op = make_mag3nl(g, NodeLaw3 {node_mu, node_ferro, &c}, gamma);
    return newton_solve(
            3 * nx * ny * nz, [&](const double* v, double* out) { op.apply(v, out); },
            [&](const double* st) { return op.prepare_jacobian(st); }, rhs, sol, tol, max_iter, newton_steps,
            final_rel);
}

// ------------------------------------------------------------------ assembled operators
//
// The reference's preconditioner menu on an assembled CSR matrix
// (src/similie/solvers/minimize_strong_formulation_residual.hpp:53-63 names,
// 61-75 defaults, 921-1026 construction through Ginkgo v1.11.0).  Ginkgo's
// source is not available here; each preconditioner restates the published
// algorithm it names:
//   Jacobi            z = D^-1 r (block size 1)
//   SpdIsai           factorized sparse approximate inverse (Kolotilina &
//                     Yeremin): Z with the pattern of tril(A), row i solving
//                     A(P_i, P_i) y = e_i and scaled by 1/sqrt(y_i); M = Z^T Z
//   GeneralIsai       incomplete sparse approximate inverse (Anzt et al. 2018):
//                     M with the pattern of A, (M A)(i, P_i) = e_i per row
//   SymmetricGaussSeidel / Ssor
//                     M = (D - w E) D^-1 (D - w F) / (w (2 - w)), A = D - E - F
//                     (Saad, Iterative Methods for Sparse Linear Systems,
//                     sec. 10.2), w = 1 for Gauss-Seidel; triangular solves
//                     in row order
//   ChebyshevJacobi   k steps of the Chebyshev iteration on the Jacobi-
//                     preconditioned system with eigenvalue bounds [l, u] from
//                     a zero guess (Saad, Algorithm 12.1)
//   IrJacobi          k steps of x += w D^-1 (b - A x) from a zero guess
// The CG is the one of silo_mag3d_cg with the preconditioner in place of
// Jacobi.
namespace {

struct CsrView
{
    int64_t n;
    const int64_t* ptr;
    const int32_t* col;
    const double* val;
    double at(int64_t r, int64_t c) const
    {
        for (int64_t k = ptr[r]; k < ptr[r + 1]; ++k)
            if (col[k] == c) return val[k];
        return 0.0;
    }
};

void spmv(CsrView const& A, const double* x, double* y)
{
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < A.n; ++i) {
        double s = 0.0;
        for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k) s += A.val[k] * x[A.col[k]];
        y[i] = s;
    }
}

// Solves G y = e_t (m x m, row-major) by Gaussian elimination with partial
// pivoting; false if singular.
bool dense_unit_solve(std::vector<double>& G, int m, int t, std::vector<double>& y)
{
    y.assign(m, 0.0);
    y[t] = 1.0;
    for (int c = 0; c < m; ++c) {
        int p = c;
        for (int r = c + 1; r < m; ++r)
            if (std::fabs(G[r * m + c]) > std::fabs(G[p * m + c])) p = r;
        if (G[p * m + c] == 0.0) return false;
        if (p != c) {
            for (int k = 0; k < m; ++k) std::swap(G[c * m + k], G[p * m + k]);
            std::swap(y[c], y[p]);
        }
        for (int r = c + 1; r < m; ++r) {
            double const f = G[r * m + c] / G[c * m + c];
            for (int k = c; k < m; ++k) G[r * m + k] -= f * G[c * m + k];
            y[r] -= f * y[c];
        }
    }
    for (int r = m - 1; r >= 0; --r) {
        double s = y[r];
        for (int k = r + 1; k < m; ++k) s -= G[r * m + k] * y[k];
        y[r] = s / G[r * m + r];
    }
    return true;
}

enum MenuKind
{
    kIdentity = 0,
    kJacobi = 1,
    kSpdIsai = 2,
    kSymGaussSeidel = 3,
    kSsor = 4,
    kChebyshevJacobi = 5,
    kIrJacobi = 6,
    kGeneralIsai = 7
};

struct MenuPrecond
{
    CsrView A;
    int kind;
    double omega;
    int cheb_iters;
    double cheb_lo, cheb_hi;
    int ir_iters;
    double ir_omega;
    std::vector<double> diag, dinv;
    std::vector<int64_t> mptr;  // ISAI factor: Z (SpdIsai, lower) or M (GeneralIsai)
    std::vector<int32_t> mcol;
    std::vector<double> mval;
    bool ok = true;

    void setup()
    {
        int64_t const n = A.n;
        diag.resize(n);
        dinv.resize(n);
        for (int64_t i = 0; i < n; ++i) {
            diag[i] = A.at(i, i);
            dinv[i] = 1.0 / diag[i];
        }
        if (kind != kSpdIsai && kind != kGeneralIsai) return;
        mptr.assign(n + 1, 0);
        for (int64_t i = 0; i < n; ++i) {
            int64_t cnt = 0;
            for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (kind == kGeneralIsai || A.col[k] <= i) ++cnt;
            mptr[i + 1] = mptr[i] + cnt;
        }
        mcol.resize(mptr[n]);
        mval.resize(mptr[n]);
        std::vector<double> G, y;
        for (int64_t i = 0; i < n; ++i) {
            std::vector<int32_t> P;
            for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                if (kind == kGeneralIsai || A.col[k] <= i) P.push_back(A.col[k]);
            int const m = static_cast<int>(P.size());
            G.assign(static_cast<size_t>(m) * m, 0.0);
            int t = 0;
            for (int a = 0; a < m; ++a) {
                if (P[a] == i) t = a;
                for (int b = 0; b < m; ++b)
                    G[a * m + b] = kind == kSpdIsai ? A.at(P[a], P[b]) : A.at(P[b], P[a]);
            }
            if (!dense_unit_solve(G, m, t, y)) {
                ok = false;
                return;
            }
            double const scale = kind == kSpdIsai ? 1.0 / std::sqrt(y[t]) : 1.0;
            for (int a = 0; a < m; ++a) {
                mcol[mptr[i] + a] = P[a];
                mval[mptr[i] + a] = kind == kSpdIsai ? y[a] * scale : y[a];
            }
        }
    }

    void apply(const double* r, double* z) const
    {
        int64_t const n = A.n;
        switch (kind) {
        case kIdentity:
            std::copy(r, r + n, z);
            return;
        case kJacobi:
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) z[i] = dinv[i] * r[i];
            return;
        case kSpdIsai: {
            std::vector<double> t(n, 0.0);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                double s = 0.0;
                for (int64_t k = mptr[i]; k < mptr[i + 1]; ++k) s += mval[k] * r[mcol[k]];
                t[i] = s;
            }
            std::fill(z, z + n, 0.0);
            for (int64_t i = 0; i < n; ++i)
                for (int64_t k = mptr[i]; k < mptr[i + 1]; ++k) z[mcol[k]] += mval[k] * t[i];
            return;
        }
        case kGeneralIsai:
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                double s = 0.0;
                for (int64_t k = mptr[i]; k < mptr[i + 1]; ++k) s += mval[k] * r[mcol[k]];
                z[i] = s;
            }
            return;
        case kSymGaussSeidel:
        case kSsor: {
            double const w = kind == kSsor ? omega : 1.0;
            double const c = w * (2.0 - w);
            std::vector<double> y(n);
            for (int64_t i = 0; i < n; ++i) {
                double s = c * r[i];
                for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                    if (A.col[k] < i) s -= w * A.val[k] * y[A.col[k]];
                y[i] = s / diag[i];
            }
            for (int64_t i = n - 1; i >= 0; --i) {
                double s = diag[i] * y[i];
                for (int64_t k = A.ptr[i]; k < A.ptr[i + 1]; ++k)
                    if (A.col[k] > i) s -= w * A.val[k] * z[A.col[k]];
                z[i] = s / diag[i];
            }
            return;
        }
        case kChebyshevJacobi: {
            double const theta = 0.5 * (cheb_hi + cheb_lo), delta = 0.5 * (cheb_hi - cheb_lo);
            double const sigma = theta / delta;
            double rho = 1.0 / sigma;
            std::vector<double> d(n), res(n), ax(n);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) {
                d[i] = dinv[i] * r[i] / theta;
                z[i] = d[i];
            }
            for (int it = 1; it < cheb_iters; ++it) {
                spmv(A, z, ax.data());
                double const rho1 = 1.0 / (2.0 * sigma - rho);
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < n; ++i) {
                    res[i] = r[i] - ax[i];
                    d[i] = rho1 * rho * d[i] + (2.0 * rho1 / delta) * (dinv[i] * res[i]);
                    z[i] += d[i];
                }
                rho = rho1;
            }
            return;
        }
        case kIrJacobi: {
            std::vector<double> ax(n);
#pragma omp parallel for schedule(static)
            for (int64_t i = 0; i < n; ++i) z[i] = ir_omega * (dinv[i] * r[i]);
            for (int it = 1; it < ir_iters; ++it) {
                spmv(A, z, ax.data());
#pragma omp parallel for schedule(static)
                for (int64_t i = 0; i < n; ++i) z[i] += ir_omega * (dinv[i] * (r[i] - ax[i]));
            }
            return;
        }
        }
    }
};

MenuPrecond make_menu(CsrView A, int kind, const double* params)
{
    MenuPrecond m {A, kind, params[0], static_cast<int>(params[1]), params[2], params[3],
                   static_cast<int>(params[4]), params[5]};
    m.setup();
    return m;
}

} // namespace

// params: sor relaxation factor, Chebyshev iterations, lower bound, upper
// bound, IR iterations, IR relaxation factor.  Returns 0, or -1 when an ISAI
// system is singular.
int silo_csr_precond_apply(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int kind,
                           const double* params, const double* r, double* z)
{
    MenuPrecond const m = make_menu(CsrView {n, ptr, col, val}, kind, params);
    if (!m.ok) return -1;
    m.apply(r, z);
    return 0;
}

// The ISAI factor's values in its pattern (tril(A) for SpdIsai, A for
// GeneralIsai): out_val holds one value per pattern entry in row order.
int silo_csr_isai_values(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int kind,
                         double* out_val)
{
    double const params[6] = {1.2, 8, 0.05, 1.5, 8, 1.0};
    MenuPrecond const m = make_menu(CsrView {n, ptr, col, val}, kind, params);
    if (!m.ok) return -1;
    std::copy(m.mval.begin(), m.mval.end(), out_val);
    return 0;
}

namespace {

int pcg_run(CsrView const& A, MenuPrecond const& m, const double* b, double* x, double tol, int max_iter,
            double* final_rel)
{
    int64_t const n = A.n;
    std::vector<double> r(b, b + n), z(n), p(n), q(n);
    std::fill(x, x + n, 0.0);
    double const bnorm = nrm2(n, b);
    if (bnorm == 0.0) {
        *final_rel = 0.0;
        return 0;
    }
    m.apply(r.data(), z.data());
    p = z;
    double rz = dotp(n, r.data(), z.data());
    double rnorm = bnorm;
    int it = 0;
    while (it < max_iter) {
        spmv(A, p.data(), q.data());
        double const alpha = rz / dotp(n, p.data(), q.data());
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i];
            r[i] -= alpha * q[i];
        }
        ++it;
        rnorm = nrm2(n, r.data());
        if (rnorm <= tol * bnorm) break;
        m.apply(r.data(), z.data());
        double const rz2 = dotp(n, r.data(), z.data());
        double const beta = rz2 / rz;
        rz = rz2;
#pragma omp parallel for schedule(static)
        for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
    }
    *final_rel = rnorm / bnorm;
    return it;
}

// CSR of a linear map whose rows touch only the 3x3 (2D nodes) or 3x3x3
// (3D nodes x 3 components) neighbourhood, by one apply per column colour
// (node coordinates mod 3, and component); exact zeros dropped, columns
// ascending.  The same construction as oracle.assemble2d / assemble3d.
struct OwnedCsr
{
    std::vector<int64_t> ptr;
    std::vector<int32_t> col;
    std::vector<double> val;
    CsrView view(int64_t n) const { return CsrView {n, ptr.data(), col.data(), val.data()}; }
};

template <class Apply>
OwnedCsr probe_csr(int dim, int64_t nx, int64_t ny, int64_t nz, Apply const& apply)
{
    int64_t const n = dim == 2 ? nx * ny : 3 * nx * ny * nz;
    int const ncolors = dim == 2 ? 9 : 81;
    auto color_of = [&](int64_t c) -> int {
        if (dim == 2) return static_cast<int>((c % nx) % 3 + 3 * ((c / nx) % 3));
        int64_t const node = c / 3, comp = c % 3;
        int64_t const i = node % nx, j = (node / nx) % ny, k = node / (nx * ny);
        return static_cast<int>(comp + 3 * (i % 3 + 3 * (j % 3) + 9 * (k % 3)));
    };
    std::vector<std::vector<std::pair<int32_t, double>>> rows(n);
    std::vector<double> probe(n), y(n);
    for (int color = 0; color < ncolors; ++color) {
        for (int64_t c = 0; c < n; ++c) probe[c] = color_of(c) == color ? 1.0 : 0.0;
        apply(probe.data(), y.data());
        for (int64_t r = 0; r < n; ++r) {
            if (y[r] == 0.0) continue;
            int64_t const node = dim == 2 ? r : r / 3;
            int64_t const i = node % nx, j = (node / nx) % ny, k = dim == 2 ? 0 : node / (nx * ny);
            for (int dk = (dim == 2 ? 0 : -1); dk <= (dim == 2 ? 0 : 1); ++dk)
                for (int dj = -1; dj <= 1; ++dj)
                    for (int di = -1; di <= 1; ++di) {
                        int64_t const ii = i + di, jj = j + dj, kk = k + dk;
                        if (ii < 0 || ii >= nx || jj < 0 || jj >= ny || kk < 0 || kk >= (dim == 2 ? 1 : nz)) continue;
                        int64_t const m = ii + nx * (jj + ny * kk);
                        for (int comp = 0; comp < (dim == 2 ? 1 : 3); ++comp) {
                            int64_t const c = dim == 2 ? m : 3 * m + comp;
                            if (color_of(c) == color) rows[r].push_back({static_cast<int32_t>(c), y[r]});
                        }
                    }
        }
    }
    OwnedCsr out;
    out.ptr.assign(n + 1, 0);
    for (int64_t r = 0; r < n; ++r) {
        std::sort(rows[r].begin(), rows[r].end());
        out.ptr[r + 1] = out.ptr[r] + static_cast<int64_t>(rows[r].size());
        for (auto const& [c, v] : rows[r]) {
            out.col.push_back(c);
            out.val.push_back(v);
        }
    }
    return out;
}

// Newton whose linear solves run CG with a menu preconditioner on the
// Jacobian assembled at the state (the reference's nonlinear branch with
// build_matrix(operator_model, solution) + build_preconditioner,
// minimize_strong_formulation_residual.hpp:1432-1436, assembled system).
template <class Apply, class Jacobian>
int newton_menu(int dim, int64_t nx, int64_t ny, int64_t nz, Apply const& apply, Jacobian const& jacobian, int kind,
                const double* params, const double* rhs, double* x, double tol, int max_iter, int* newton_steps,
                double* final_rel)
{
    int64_t const N = dim == 2 ? nx * ny : 3 * nx * ny * nz;
    bool ok = true;
    int const total = newton_core(
            N, apply,
            [&](const double* xs, const double* r, double* d) {
                OwnedCsr const J = probe_csr(dim, nx, ny, nz,
                                             [&](const double* v, double* out) { jacobian(xs, v, out); });
                MenuPrecond const m = make_menu(J.view(N), kind, params);
                if (!m.ok) {
                    ok = false;
                    std::fill(d, d + N, 0.0);
                    return 0;
                }
                double rel = 0.0;
                return pcg_run(J.view(N), m, r, d, tol, max_iter, &rel);
            },
            rhs, x, tol, newton_steps, final_rel);
    return ok ? total : -1;
}

} // namespace

// Preconditioned CG from x = 0 until ||r|| <= tol ||b||; returns the
// iterations (-1 when the preconditioner cannot be built).
int silo_csr_pcg(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int kind, const double* params,
                 const double* b, double* x, double tol, int max_iter, double* final_rel)
{
    CsrView const A {n, ptr, col, val};
    MenuPrecond const m = make_menu(A, kind, params);
    if (!m.ok) return -1;
    return pcg_run(A, m, b, x, tol, max_iter, final_rel);
}

int silo_mag2d_nl_solve_menu(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                             const double* b, const double* h, int kind, const double* params, const double* rhs,
                             double* x, double tol, int max_iter, int* newton_steps, double* final_rel)
{
    BHCurve const c(n, b, h);
    NodeLaw const law {node_mu, node_ferro, &c};
    return newton_menu(
            2, nx, ny, 1, [&](const double* v, double* out) { nl_apply(nx, ny, law, v, out); },
            [&](const double* st, const double* v, double* out) { nl_jacobian_apply(nx, ny, law, st, v, out); },
            kind, params, rhs, x, tol, max_iter, newton_steps, final_rel);
}

int silo_mag3d_nl_solve_menu(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                             const double* node_mu, const double* node_ferro, double gamma, int n, const double* b,
                             const double* h, int kind, const double* params, const double* rhs, double* sol,
                             double tol, int max_iter, int* newton_steps, double* final_rel)
{
    BHCurve const c(n, b, h);
    Grid3 const g {nx, ny, nz, x, y, z};
    Mag3Nl const op = make_mag3nl(g, NodeLaw3 {node_mu, node_ferro, &c}, gamma);
    return newton_menu(
            3, nx, ny, nz, [&](const double* v, double* out) { op.apply(v, out); },
            [&](const double* st, const double* v, double* out) { op.jacobian(st, v, out); }, kind, params, rhs, sol,
            tol, max_iter, newton_steps, final_rel);
}

// ------------------------------------------------------------------ Krylov menu
//
// The reference's SIMILIE_SOLVER alternatives to CG
// (src/similie/solvers/minimize_strong_formulation_residual.hpp:1069-1130:
// Ginkgo's Minres, Fcg, Gmres with Krylov dimension SIMILIE_GMRES_KRYLOV_DIM
// (100), Bicgstab, Gcr with SIMILIE_GCR_KRYLOV_DIM (100), Idr with subspace
// SIMILIE_IDR_SUBSPACE_DIM (8) and a deterministic shadow space), each with
// the menu preconditioner, x0 = 0 and the stop ||r|| <= tol ||b||.  Ginkgo's
// source is not available here; each restates the published method it
// names, preconditioned on the right (x = M^-1 u) except MINRES and FCG,
// which take M^-1 as the symmetric preconditioner of the Lanczos / CG
// recurrences:
//   MINRES    Paige & Saunders (1975), preconditioned Lanczos with Givens
//             rotations; stops on the true residual of its iterate
//   FCG       flexible CG, beta = z_k . (r_k - r_{k-1}) / (z_{k-1} . r_{k-1})
//             (Notay 2000, one stored direction)
//   GMRES(m)  Saad & Schultz (1986), modified Gram-Schmidt Arnoldi, Givens
//             rotations, restart after m; stops on the least-squares residual
//   BiCGSTAB  van der Vorst (1992)
//   GCR(m)    Eisenstat, Elman & Schultz (1983), A-images orthogonalised by
//             modified Gram-Schmidt, restart after m
//   IDR(s)    van Gijzen & Sonneveld (2011), Algorithm 2 (biorthogonal
//             IDR(s)); shadow space: s Gaussian vectors from a fixed seed,
//             orthonormalised
namespace {

enum KrylovKind
{
    kCg = 0,
    kMinres = 1,
    kFcg = 2,
    kGmres = 3,
    kBicgstab = 4,
    kGcr = 5,
    kIdr = 6
};

void axpy(int64_t n, double a, const double* x, double* y)
{
    for (int64_t i = 0; i < n; ++i) y[i] += a * x[i];
}

// returns iterations; x from 0
int krylov_run(CsrView const& A, MenuPrecond const& M, int solver, int dim, const double* b, double* x, double tol,
               int max_iter, double* final_rel)
{
    int64_t const n = A.n;
    std::fill(x, x + n, 0.0);
    double const bn = nrm2(n, b);
    *final_rel = 0.0;
    if (bn == 0.0) return 0;
    double const target = tol * bn;
    std::vector<double> r(b, b + n), z(n), p(n), q(n), t(n);
    auto true_residual = [&]() {
        spmv(A, x, t.data());
        for (int64_t i = 0; i < n; ++i) t[i] = b[i] - t[i];
        return nrm2(n, t.data());
    };
    int it = 0;
    if (solver == kCg) {
        double rel = 0.0;
        it = pcg_run(A, M, b, x, tol, max_iter, &rel);
        *final_rel = rel;
        return it;
    }
    if (solver == kFcg) {
        std::vector<double> r_old(n);
        M.apply(r.data(), z.data());
        p = z;
        double rz = dotp(n, r.data(), z.data());
        double rn = bn;
        while (it < max_iter) {
            spmv(A, p.data(), q.data());
            double const alpha = rz / dotp(n, p.data(), q.data());
            r_old = r;
            for (int64_t i = 0; i < n; ++i) {
                x[i] += alpha * p[i];
                r[i] -= alpha * q[i];
            }
            ++it;
            rn = nrm2(n, r.data());
            if (rn <= target) break;
            M.apply(r.data(), z.data());
            double num = 0.0;
            for (int64_t i = 0; i < n; ++i) num += z[i] * (r[i] - r_old[i]);
            double const beta = num / rz;
            rz = dotp(n, r.data(), z.data());
            for (int64_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        }
        *final_rel = rn / bn;
        return it;
    }
    if (solver == kMinres) {
        // preconditioned Lanczos: v = residual vectors, w = M^-1 v
        std::vector<double> v_old(n, 0.0), v(b, b + n), w(n), v_new(n), d_old(n, 0.0), d_older(n, 0.0), d(n);
        M.apply(v.data(), w.data());
        double beta = std::sqrt(dotp(n, v.data(), w.data()));
        double beta_prev = 1.0;  // multiplies v_old = 0 in the first step
        double eta = beta;
        double c_old = 1.0, s_old = 0.0, c = 1.0, s = 0.0;
        double rn = bn;
        while (it < max_iter && beta > 0.0) {
            for (int64_t i = 0; i < n; ++i) w[i] /= beta;   // w_k = M^-1 v_k / beta_k
            spmv(A, w.data(), q.data());
            double const alpha = dotp(n, w.data(), q.data());
            for (int64_t i = 0; i < n; ++i) v_new[i] = q[i] - (alpha / beta) * v[i] - (beta / beta_prev) * v_old[i];
            std::vector<double> w_new(n);
            M.apply(v_new.data(), w_new.data());
            double const beta_new = std::sqrt(std::max(0.0, dotp(n, v_new.data(), w_new.data())));
            // QR of the tridiagonal by Givens rotations
            double const delta = c * alpha - c_old * s * beta;
            double const rho2 = s * alpha + c_old * c * beta;
            double const rho3 = s_old * beta;
            double const rho1 = std::sqrt(delta * delta + beta_new * beta_new);
            double const c_new = delta / rho1, s_new = beta_new / rho1;
            for (int64_t i = 0; i < n; ++i) d[i] = (w[i] - rho3 * d_older[i] - rho2 * d_old[i]) / rho1;
            axpy(n, c_new * eta, d.data(), x);
            eta = -s_new * eta;
            d_older = d_old;
            d_old = d;
            v_old = v;
            v = v_new;
            w = w_new;
            beta_prev = beta;
            beta = beta_new;
            c_old = c;
            s_old = s;
            c = c_new;
            s = s_new;
            ++it;
            rn = true_residual();
            if (rn <= target) break;
        }
        *final_rel = rn / bn;
        return it;
    }
    if (solver == kGmres) {
        int const m = std::max(1, dim);
        std::vector<std::vector<double>> V(m + 1, std::vector<double>(n));
        std::vector<double> H(static_cast<size_t>(m + 1) * m), cs(m), sn(m), g(m + 1), y(m), u(n);
        double rn = bn;
        while (it < max_iter) {
            double const beta = nrm2(n, r.data());
            if (beta <= target) break;
            for (int64_t i = 0; i < n; ++i) V[0][i] = r[i] / beta;
            std::fill(g.begin(), g.end(), 0.0);
            g[0] = beta;
            int k = 0;
            for (; k < m && it < max_iter; ++k) {
                M.apply(V[k].data(), z.data());
                spmv(A, z.data(), u.data());
                for (int j = 0; j <= k; ++j) {
                    double const h = dotp(n, u.data(), V[j].data());
                    H[j * m + k] = h;
                    axpy(n, -h, V[j].data(), u.data());
                }
                double const hn = nrm2(n, u.data());
                H[(k + 1) * m + k] = hn;
                if (hn != 0.0)
                    for (int64_t i = 0; i < n; ++i) V[k + 1][i] = u[i] / hn;
                for (int j = 0; j < k; ++j) {
                    double const a = H[j * m + k], bb = H[(j + 1) * m + k];
                    H[j * m + k] = cs[j] * a + sn[j] * bb;
                    H[(j + 1) * m + k] = -sn[j] * a + cs[j] * bb;
                }
                double const a = H[k * m + k], bb = H[(k + 1) * m + k];
                double const den = std::sqrt(a * a + bb * bb);
                cs[k] = a / den;
                sn[k] = bb / den;
                H[k * m + k] = den;
                H[(k + 1) * m + k] = 0.0;
                g[k + 1] = -sn[k] * g[k];
                g[k] = cs[k] * g[k];
                ++it;
                rn = std::fabs(g[k + 1]);
                if (rn <= target) {
                    ++k;
                    break;
                }
            }
            // x += M^-1 (V y), H y = g
            for (int j = k - 1; j >= 0; --j) {
                double sacc = g[j];
                for (int l = j + 1; l < k; ++l) sacc -= H[j * m + l] * y[l];
                y[j] = sacc / H[j * m + j];
            }
            std::fill(u.begin(), u.end(), 0.0);
            for (int j = 0; j < k; ++j) axpy(n, y[j], V[j].data(), u.data());
            M.apply(u.data(), z.data());
            axpy(n, 1.0, z.data(), x);
            spmv(A, x, t.data());
            for (int64_t i = 0; i < n; ++i) r[i] = b[i] - t[i];
            if (rn <= target) break;
        }
        *final_rel = rn / bn;
        return it;
    }
    if (solver == kBicgstab) {
        std::vector<double> r0(r), v(n, 0.0), ph(n), sv(n), sh(n), tv(n);
        double rho = 1.0, alpha = 1.0, omega = 1.0, rn = bn;
        std::fill(p.begin(), p.end(), 0.0);
        while (it < max_iter) {
            double const rho_new = dotp(n, r0.data(), r.data());
            double const beta = (rho_new / rho) * (alpha / omega);
            for (int64_t i = 0; i < n; ++i) p[i] = r[i] + beta * (p[i] - omega * v[i]);
            M.apply(p.data(), ph.data());
            spmv(A, ph.data(), v.data());
            alpha = rho_new / dotp(n, r0.data(), v.data());
            for (int64_t i = 0; i < n; ++i) sv[i] = r[i] - alpha * v[i];
            ++it;
            double const sn_ = nrm2(n, sv.data());
            if (sn_ <= target) {
                axpy(n, alpha, ph.data(), x);
                rn = sn_;
                break;
            }
            M.apply(sv.data(), sh.data());
            spmv(A, sh.data(), tv.data());
            omega = dotp(n, tv.data(), sv.data()) / dotp(n, tv.data(), tv.data());
            for (int64_t i = 0; i < n; ++i) {
                x[i] += alpha * ph[i] + omega * sh[i];
                r[i] = sv[i] - omega * tv[i];
            }
            rho = rho_new;
            rn = nrm2(n, r.data());
            if (rn <= target) break;
        }
        *final_rel = rn / bn;
        return it;
    }
    if (solver == kGcr) {
        int const m = std::max(1, dim);
        std::vector<std::vector<double>> P(m, std::vector<double>(n)), Q(m, std::vector<double>(n));
        double rn = bn;
        int k = 0;
        while (it < max_iter) {
            if (k == m) k = 0;
            M.apply(r.data(), P[k].data());
            spmv(A, P[k].data(), Q[k].data());
            for (int j = 0; j < k; ++j) {
                double const h = dotp(n, Q[k].data(), Q[j].data());
                axpy(n, -h, Q[j].data(), Q[k].data());
                axpy(n, -h, P[j].data(), P[k].data());
            }
            double const qn = nrm2(n, Q[k].data());
            for (int64_t i = 0; i < n; ++i) {
                Q[k][i] /= qn;
                P[k][i] /= qn;
            }
            double const alpha = dotp(n, r.data(), Q[k].data());
            axpy(n, alpha, P[k].data(), x);
            axpy(n, -alpha, Q[k].data(), r.data());
            ++k;
            ++it;
            rn = nrm2(n, r.data());
            if (rn <= target) break;
        }
        *final_rel = rn / bn;
        return it;
    }
    if (solver == kIdr) {
        int const s = std::max(1, dim);
        // shadow space: s orthonormalised Gaussian vectors, fixed seed
        std::vector<std::vector<double>> P(s, std::vector<double>(n));
        uint64_t state = 0x9E3779B97F4A7C15ull;
        auto uniform = [&]() {
            state ^= state << 13;
            state ^= state >> 7;
            state ^= state << 17;
            return (static_cast<double>(state >> 11) + 0.5) / 9007199254740992.0;
        };
        for (int j = 0; j < s; ++j) {
            for (int64_t i = 0; i < n; ++i) {
                double const u1 = uniform(), u2 = uniform();
                P[j][i] = std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
            }
            for (int l = 0; l < j; ++l) axpy(n, -dotp(n, P[j].data(), P[l].data()), P[l].data(), P[j].data());
            double const pn = nrm2(n, P[j].data());
            for (int64_t i = 0; i < n; ++i) P[j][i] /= pn;
        }
        std::vector<std::vector<double>> G(s, std::vector<double>(n, 0.0)), U(s, std::vector<double>(n, 0.0));
        std::vector<double> Mm(static_cast<size_t>(s) * s, 0.0), f(s), c(s), vv(n), vh(n), tt(n);
        for (int j = 0; j < s; ++j) Mm[j * s + j] = 1.0;
        double om = 1.0, rn = bn;
        while (it < max_iter) {
            for (int j = 0; j < s; ++j) f[j] = dotp(n, P[j].data(), r.data());
            for (int k = 0; k < s && it < max_iter; ++k) {
                // solve the lower triangular M(k:s, k:s) c = f(k:s)
                for (int i = k; i < s; ++i) {
                    double acc = f[i];
                    for (int j = k; j < i; ++j) acc -= Mm[i * s + j] * c[j];
                    c[i] = acc / Mm[i * s + i];
                }
                vv = r;
                for (int i = k; i < s; ++i) axpy(n, -c[i], G[i].data(), vv.data());
                M.apply(vv.data(), vh.data());
                for (int64_t i = 0; i < n; ++i) {
                    double acc = om * vh[i];
                    for (int j = k; j < s; ++j) acc += c[j] * U[j][i];
                    U[k][i] = acc;
                }
                spmv(A, U[k].data(), G[k].data());
                for (int i = 0; i < k; ++i) {
                    double const a = dotp(n, P[i].data(), G[k].data()) / Mm[i * s + i];
                    axpy(n, -a, G[i].data(), G[k].data());
                    axpy(n, -a, U[i].data(), U[k].data());
                }
                for (int i = k; i < s; ++i) Mm[i * s + k] = dotp(n, P[i].data(), G[k].data());
                double const beta = f[k] / Mm[k * s + k];
                axpy(n, -beta, G[k].data(), r.data());
                axpy(n, beta, U[k].data(), x);
                ++it;
                rn = nrm2(n, r.data());
                if (rn <= target) break;
                for (int i = k + 1; i < s; ++i) f[i] -= beta * Mm[i * s + k];
            }
            if (rn <= target || it >= max_iter) break;
            // the step into the next subspace
            M.apply(r.data(), vh.data());
            spmv(A, vh.data(), tt.data());
            double const tn = dotp(n, tt.data(), tt.data());
            double const tr = dotp(n, tt.data(), r.data());
            om = tr / tn;
            double const rho = std::fabs(tr) / (std::sqrt(tn) * nrm2(n, r.data()));
            if (rho < 0.7) om *= 0.7 / rho;   // the "maintaining the convergence" safeguard
            axpy(n, -om, tt.data(), r.data());
            axpy(n, om, vh.data(), x);
            ++it;
            rn = nrm2(n, r.data());
            if (rn <= target) break;
        }
        *final_rel = rn / bn;
        return it;
    }
    return -1;
}

} // namespace

// solver: 0 cg, 1 minres, 2 fcg, 3 gmres, 4 bicgstab, 5 gcr, 6 idr; dim the
// GMRES / GCR Krylov dimension or the IDR subspace dimension.  Returns the
// iterations (-1: unknown solver or a singular ISAI system).
int silo_csr_krylov(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int solver, int dim,
                    int kind, const double* params, const double* b, double* x, double tol, int max_iter,
                    double* final_rel)
{
    CsrView const A {n, ptr, col, val};
    MenuPrecond const m = make_menu(A, kind, params);
    if (!m.ok) return -1;
    return krylov_run(A, m, solver, dim, b, x, tol, max_iter, final_rel);
}
