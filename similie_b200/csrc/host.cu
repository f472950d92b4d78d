// host.cu -- host-side plumbing: errors, field checks, chain and Hodge rule
// tables, geometry objects.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <string>

#include "sil_internal.cuh"

namespace sil {

namespace {
thread_local std::string g_last_error;
}

void set_error(std::string const& msg)
{
    g_last_error = msg;
}

sil_status fail(sil_status status, std::string const& msg)
{
    set_error(msg);
    return status;
}

sil_status cuda_fail(cudaError_t err, char const* what)
{
    set_error(std::string(what) + ": " + cudaGetErrorString(err));
    return err == cudaErrorMemoryAllocation ? SIL_ERR_ALLOC : SIL_ERR_CUDA;
}

FieldView to_view(sil_field const& f)
{
    FieldView v {};
    v.data = f.data;
    v.ndims = f.ndims;
    v.ncomp = f.ncomp;
    for (int d = 0; d < kMaxDims; ++d) {
        v.front[d] = d < f.ndims ? f.front[d] : 0;
        v.extent[d] = d < f.ndims ? f.extent[d] : 1;
        v.stride[d] = d < f.ndims ? f.stride[d] : 0;
    }
    v.comp_stride = f.comp_stride;
    return v;
}

int64_t node_count(sil_field const& f)
{
    int64_t t = 1;
    for (int d = 0; d < f.ndims; ++d) t *= f.extent[d];
    return t;
}

sil_status check_field(sil_field const* f, char const* name, int expect_ncomp)
{
    if (f == nullptr) return fail(SIL_ERR_INVALID, std::string(name) + " is NULL");
    if (f->ndims < 1 || f->ndims > kMaxDims)
        return fail(SIL_ERR_INVALID, std::string(name) + ": ndims out of range");
    if (f->dtype != SIL_F64 && f->dtype != SIL_F32)
        return fail(SIL_ERR_INVALID, std::string(name) + ": unknown dtype");
    if (expect_ncomp >= 0 && f->ncomp != expect_ncomp)
        return fail(SIL_ERR_INVALID, std::string(name) + ": expected " + std::to_string(expect_ncomp)
                                             + " components, got " + std::to_string(f->ncomp));
    for (int d = 0; d < f->ndims; ++d) {
        if (f->extent[d] < 0) return fail(SIL_ERR_INVALID, std::string(name) + ": negative extent");
    }
    if (node_count(*f) > 0 && f->data == nullptr)
        return fail(SIL_ERR_INVALID, std::string(name) + ": NULL data");
    return SIL_OK;
}

int form_dims(uint32_t mask, int ndims, int* dims)
{
    int n = 0;
    for (int d = 0; d < ndims; ++d) {
        if (mask & (1u << d)) dims[n++] = d;
    }
    return n;
}

std::vector<uint32_t> combinations(int n, int k)
{
    // Lexicographic order of the sorted index lists: walk masks and sort by
    // their element sequences.
    std::vector<uint32_t> out;
    for (uint32_t m = 0; m < (1u << n); ++m) {
        if (__builtin_popcount(m) == k) out.push_back(m);
    }
    std::sort(out.begin(), out.end(), [n](uint32_t a, uint32_t b) {
        for (int d = 0; d < n; ++d) {
            bool const ia = a & (1u << d), ib = b & (1u << d);
            if (ia != ib) return ia;  // the list that holds the smaller index first comes first
        }
        return false;
    });
    return out;
}

namespace {
int comb_index(std::vector<uint32_t> const& combos, uint32_t mask)
{
    for (std::size_t i = 0; i < combos.size(); ++i)
        if (combos[i] == mask) return static_cast<int>(i);
    return -1;
}

// Sign of the permutation that lists the indices of `a` (ascending) then those of `b` (ascending).
int concat_sign(int n, uint32_t a, uint32_t b)
{
    int seq[2 * kMaxN];
    int len = 0;
    for (int d = 0; d < n; ++d)
        if (a & (1u << d)) seq[len++] = d;
    for (int d = 0; d < n; ++d)
        if (b & (1u << d)) seq[len++] = d;
    int inv = 0;
    for (int i = 0; i < len; ++i)
        for (int j = i + 1; j < len; ++j) inv += seq[i] > seq[j];
    return inv % 2 ? -1 : 1;
}
} // namespace

// Oriented boundary of the basis (k+1)-simplex spanned by the directions
// d_0 < ... < d_k from a node.  Face i of the first half removes d_i at the
// node itself; face i of the second half removes d_i at node + e_{d_i} (for
// d^T: node - e_{d_i}).  With K = k + 1, the orientation of SimiLie's chain
// construction (boundary.hpp, simplex.hpp) works out to
//   first half:  negative = ((K + i) odd) xor (K even)
//   second half: negative = ((K - 1 + i) odd) xor (K even)
// and the chain is summed first half then second half, i ascending.
CoboundaryRules make_rules(int n, int k, bool transposed)
{
    CoboundaryRules r {};
    r.n = n;
    r.k = k;
    int const K = k + 1;
    auto const upper = combinations(n, K);
    auto const lower = combinations(n, k);
    r.ncomp_in = static_cast<int>(lower.size());
    r.ncomp_out = static_cast<int>(upper.size());
    r.nfaces = 2 * K;
    bool const even = (K % 2) == 0;
    for (std::size_t c = 0; c < upper.size(); ++c) {
        int dirs[kMaxN];
        int nd = 0;
        for (int d = 0; d < n; ++d)
            if (upper[c] & (1u << d)) dirs[nd++] = d;
        for (int half = 0; half < 2; ++half) {
            for (int i = 0; i < K; ++i) {
                FaceRule& f = r.rule[c][half * K + i];
                for (int d = 0; d < kMaxN; ++d) f.offset[d] = 0;
                uint32_t const face_mask = upper[c] & ~(1u << dirs[i]);
                f.comp = static_cast<int8_t>(comb_index(lower, face_mask));
                bool neg;
                if (half == 0) {
                    neg = ((K + i) % 2 == 1) != even;
                } else {
                    neg = ((K - 1 + i) % 2 == 1) != even;
                    f.offset[dirs[i]] = transposed ? -1 : 1;
                }
                f.negative = neg ? 1 : 0;
            }
        }
    }
    return r;
}

// Diagonal-metric Hodge star of an r-form: output component t (an
// (n-r)-combination) = sign(c, t) * prod_{d in t} h_d / prod_{d in c} h_d
// * input component c, c the complement of t.  This is what SimiLie's
// reconstruction -> continuous star -> circumcentric reduction chain
// (hodge_star.hpp:227-273) evaluates to on an orthogonal grid with the
// identity metric.
StarRule make_star(int n, int r)
{
    StarRule s {};
    s.n = n;
    s.r = r;
    auto const out = combinations(n, n - r);
    auto const in = combinations(n, r);
    s.ncomp_out = static_cast<int>(out.size());
    uint32_t const all = (1u << n) - 1;
    for (std::size_t t = 0; t < out.size(); ++t) {
        uint32_t const c = all & ~out[t];
        s.src[t] = static_cast<int8_t>(comb_index(in, c));
        s.sgn[t] = static_cast<int8_t>(concat_sign(n, c, out[t]));
        s.num_mask[t] = static_cast<uint8_t>(out[t]);
        s.den_mask[t] = static_cast<uint8_t>(c);
    }
    return s;
}

template <class T>
GeoView<T> geo_view(Geometry const& g)
{
    GeoView<T> v {};
    for (int a = 0; a < kMaxNHodge; ++a) {
        if constexpr (sizeof(T) == 8) {
            v.h[a] = g.h[a];
            v.inv_h[a] = g.inv_h[a];
        } else {
            v.h[a] = g.h32[a];
            v.inv_h[a] = g.inv_h32[a];
        }
        v.front[a] = g.front[a];
        v.npoints[a] = g.npoints[a];
    }
    return v;
}

template GeoView<double> geo_view<double>(Geometry const&);
template GeoView<float> geo_view<float>(Geometry const&);

} // namespace sil

using namespace sil;

extern "C" {

const char* sil_status_string(sil_status status)
{
    switch (status) {
    case SIL_OK: return "SIL_OK";
    case SIL_ERR_INVALID: return "SIL_ERR_INVALID";
    case SIL_ERR_UNSUPPORTED: return "SIL_ERR_UNSUPPORTED";
    case SIL_ERR_CUDA: return "SIL_ERR_CUDA";
    case SIL_ERR_ALLOC: return "SIL_ERR_ALLOC";
    case SIL_ERR_NONFINITE: return "SIL_ERR_NONFINITE";
    case SIL_ERR_STALLED: return "SIL_ERR_STALLED";
    case SIL_ERR_BUDGET: return "SIL_ERR_BUDGET";
    }
    return "SIL_UNKNOWN_STATUS";
}

const char* sil_last_error(void)
{
    return g_last_error.c_str();
}

sil_status sil_geometry_create(sil_geometry* geometry, int n, const double* const* coords,
                               const int64_t* npoints, const int64_t* front)
{
    if (geometry == nullptr || coords == nullptr || npoints == nullptr)
        return fail(SIL_ERR_INVALID, "sil_geometry_create: NULL argument");
    *geometry = nullptr;
    if (n < 1 || n > kMaxNHodge) return fail(SIL_ERR_UNSUPPORTED, "sil_geometry_create: n must be 1..3");
    auto* geo = new (std::nothrow) sil_geometry_s();
    if (geo == nullptr) return fail(SIL_ERR_ALLOC, "sil_geometry_create: host allocation");
    Geometry& g = geo->g;
    g.n = n;
    sil_status st = SIL_OK;
    for (int a = 0; a < n && st == SIL_OK; ++a) {
        int64_t const np = npoints[a];
        if (np < 2 || coords[a] == nullptr) {
            st = fail(SIL_ERR_INVALID, "sil_geometry_create: each axis needs >= 2 coordinates");
            break;
        }
        g.npoints[a] = np;
        g.front[a] = front ? front[a] : 0;
        // Pads: edge length 1 and inverse 0 outside the axis, so a Hodge
        // factor evaluated one node outside the lattice vanishes.
        std::vector<double> h(np + 2, 1.0), ih(np + 2, 0.0);
        std::vector<float> h32(np + 2, 1.0f), ih32(np + 2, 0.0f);
        for (int64_t p = 0; p < np; ++p) {
            double const e = p + 1 < np ? coords[a][p + 1] - coords[a][p] : coords[a][p] - coords[a][p - 1];
            h[p + 1] = e;
            ih[p + 1] = 1.0 / e;
            h32[p + 1] = static_cast<float>(e);
            ih32[p + 1] = static_cast<float>(1.0 / e);
        }
        g.host_h[a] = h;
        cudaError_t err = cudaMalloc(&g.h[a], (np + 2) * sizeof(double));
        if (err == cudaSuccess) err = cudaMalloc(&g.inv_h[a], (np + 2) * sizeof(double));
        if (err == cudaSuccess) err = cudaMalloc(&g.h32[a], (np + 2) * sizeof(float));
        if (err == cudaSuccess) err = cudaMalloc(&g.inv_h32[a], (np + 2) * sizeof(float));
        if (err == cudaSuccess) err = cudaMemcpy(g.h[a], h.data(), (np + 2) * sizeof(double), cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(g.inv_h[a], ih.data(), (np + 2) * sizeof(double), cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(g.h32[a], h32.data(), (np + 2) * sizeof(float), cudaMemcpyHostToDevice);
        if (err == cudaSuccess) err = cudaMemcpy(g.inv_h32[a], ih32.data(), (np + 2) * sizeof(float), cudaMemcpyHostToDevice);
        if (err != cudaSuccess) st = cuda_fail(err, "sil_geometry_create");
    }
    if (st != SIL_OK) {
        sil_geometry_destroy(geo);
        return st;
    }
    *geometry = geo;
    return SIL_OK;
}

sil_status sil_geometry_destroy(sil_geometry geometry)
{
    if (geometry == nullptr) return SIL_OK;
    for (int a = 0; a < kMaxNHodge; ++a) {
        cudaFree(geometry->g.h[a]);
        cudaFree(geometry->g.inv_h[a]);
        cudaFree(geometry->g.h32[a]);
        cudaFree(geometry->g.inv_h32[a]);
    }
    delete geometry;
    return SIL_OK;
}

} // extern "C"
