// dec_generic.cu -- table-driven DEC kernels for any rank, 1-4 form
// dimensions (3 for the Hodge-star based operators), any strides, spectator
// dimensions, FP64 and FP32.  They serve every shape the specialised kernels
// do not, and the unfused reference chain.
//
// Each kernel is instantiated for the field rank ND (lattice + spectator
// dims, 1..6) so the index arithmetic unrolls; the sampling rules (faces of
// the basis simplices, Hodge-star factors) come from tables built on the
// host (host.cu).
#include <algorithm>
#include <type_traits>

#include "sil_internal.cuh"

namespace sil {

namespace {

template <int ND>
__device__ __forceinline__ void unravel(FieldView const& f, int64_t flat, int64_t* local)
{
    if (flat < (int64_t(1) << 31)) {
        uint32_t fl = static_cast<uint32_t>(flat);
#pragma unroll
        for (int d = ND - 1; d > 0; --d) {
            uint32_t const e = static_cast<uint32_t>(f.extent[d]);
            local[d] = fl % e;
            fl /= e;
        }
        local[0] = fl;
        return;
    }
#pragma unroll
    for (int d = ND - 1; d > 0; --d) {
        int64_t const e = f.extent[d];
        local[d] = flat % e;
        flat /= e;
    }
    local[0] = flat;
}

// Absolute coordinates of the output node `flat` and its element offset.
template <int ND>
__device__ __forceinline__ int64_t node_setup(FieldView const& out, int64_t flat, int64_t* abs)
{
    int64_t local[ND];
    unravel<ND>(out, flat, local);
    int64_t off = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        abs[d] = out.front[d] + local[d];
        off += local[d] * out.stride[d];
    }
    return off;
}

template <class T, int ND>
__device__ __forceinline__ T load_at(FieldView const& f, int64_t const* abs, int comp)
{
    int64_t off = comp * f.comp_stride;
#pragma unroll
    for (int d = 0; d < ND; ++d) off += (abs[d] - f.front[d]) * f.stride[d];
    return static_cast<T const*>(f.data)[off];
}

template <int ND>
__device__ __forceinline__ bool inside(FieldView const& f, int64_t const* abs)
{
    bool in = true;
#pragma unroll
    for (int d = 0; d < ND; ++d) in = in && abs[d] >= f.front[d] && abs[d] < f.front[d] + f.extent[d];
    return in;
}

template <int ND>
__device__ __forceinline__ void clamp_to(FieldView const& f, int64_t* abs)
{
#pragma unroll
    for (int d = 0; d < ND; ++d) abs[d] = min(max(abs[d], f.front[d]), f.front[d] + f.extent[d] - 1);
}

struct DimMap
{
    int n;
    int dims[kMaxN];
};

template <int ND>
__device__ __forceinline__ void offset_node(DimMap const& dm, int64_t const* abs, FaceRule const& r, int64_t* s)
{
#pragma unroll
    for (int d = 0; d < ND; ++d) s[d] = abs[d];
#pragma unroll
    for (int a = 0; a < kMaxN; ++a) {
        if (a < dm.n) s[dm.dims[a]] += r.offset[a];
    }
}

// ------------------------------------------------------------------ d, d^T

template <class T, bool TRANSPOSED, int ND>
__global__ void coboundary_kernel(FieldView in, FieldView out, CoboundaryRules rules, DimMap dm, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(out.data) + node_setup<ND>(out, flat, abs);
    for (int c = 0; c < rules.ncomp_out; ++c) {
        T acc = T(0);
        for (int f = 0; f < rules.nfaces; ++f) {
            FaceRule const r = rules.rule[c][f];
            int64_t s[ND];
            offset_node<ND>(dm, abs, r, s);
            T v;
            if (!TRANSPOSED) {
                clamp_to<ND>(in, s);
                v = load_at<T, ND>(in, s, r.comp);
            } else {
                v = inside<ND>(in, s) ? load_at<T, ND>(in, s, r.comp) : T(0);
            }
            // Chain-order signed sum from zero: acc + (-1)*v is acc - v exactly.
            acc = r.negative ? acc - v : acc + v;
        }
        o[c * out.comp_stride] = TRANSPOSED ? -acc : acc;
    }
}

// ------------------------------------------------------------------ Hodge star

template <class T>
struct GeoCtx
{
    GeoView<T> geo;
    DimMap dm;
};

// sign * product of edge lengths over `num` * product of inverse lengths over `den`.
template <class T>
__device__ __forceinline__ T star_factor(GeoCtx<T> const& g, int64_t const* abs, uint32_t num, uint32_t den, int sgn)
{
    T f = static_cast<T>(sgn);
#pragma unroll
    for (int a = 0; a < kMaxNHodge; ++a) {
        if (a < g.dm.n) {
            int64_t const p = abs[g.dm.dims[a]] - g.geo.front[a] + 1;
            if (num & (1u << a)) f *= g.geo.h[a][p];
            if (den & (1u << a)) f *= g.geo.inv_h[a][p];
        }
    }
    return f;
}

template <class T, int ND>
__global__ void hodge_kernel(FieldView in, FieldView out, StarRule star, GeoCtx<T> g, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(out.data) + node_setup<ND>(out, flat, abs);
    for (int t = 0; t < star.ncomp_out; ++t) {
        T const v = load_at<T, ND>(in, abs, star.src[t]);
        o[t * out.comp_stride] = star_factor(g, abs, star.num_mask[t], star.den_mask[t], star.sgn[t]) * v;
    }
}

// Dense 3D fast path of the Hodge star: a contiguous [x][y][z][component]
// field over the three form dimensions (no spectators), input and output on
// the same box.  One block covers a run of z along one (x, y) row, so the
// per-node index arithmetic is one add; the factors are formed in the same
// order as star_factor (sign, then h / inv_h per axis), so the result is the
// table-driven kernel's bit for bit.
template <class T>
__global__ void __launch_bounds__(256) hodge3d_dense_kernel(T const* in, T* out, int ncin, int ncout, StarRule star,
                                                            GeoView<T> geo, int64_t fx, int64_t fy, int64_t fz,
                                                            int nx, int ny, int nz, int zchunks)
{
    int const row = blockIdx.x / zchunks;
    int const z = (blockIdx.x - row * zchunks) * blockDim.x + threadIdx.x;
    if (z >= nz) return;
    int const y = row % ny, x = row / ny;
    int64_t const node = (static_cast<int64_t>(row)) * nz + z;
    int64_t const p[3] = {fx + x - geo.front[0] + 1, fy + y - geo.front[1] + 1, fz + z - geo.front[2] + 1};
    T const* src = in + node * ncin;
    T v[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = c < ncin ? src[c] : T(0);
    T* dst = out + node * ncout;
#pragma unroll
    for (int t = 0; t < 3; ++t) {
        if (t >= ncout) break;
        T f = static_cast<T>(star.sgn[t]);
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            if (star.num_mask[t] & (1u << a)) f *= geo.h[a][p[a]];
            if (star.den_mask[t] & (1u << a)) f *= geo.inv_h[a][p[a]];
        }
        dst[t] = f * v[star.src[t]];
    }
}

// Paired variant of the dense 3D row kernel for FP64 fields with three
// components in and out and an even z extent: each thread owns two
// consecutive nodes along z (never split across a row), so its 48 bytes in
// and out move as three 16-byte vector accesses; the pairs of all rows form
// one flat range, so every thread of every block has a pair.
__global__ void __launch_bounds__(256) hodge3d_dense_pair_kernel(double const* in, double* out, StarRule star,
                                                                 GeoView<double> geo, int64_t fx, int64_t fy,
                                                                 int64_t fz, int ny, int nz, uint32_t npairs)
{
    uint32_t const q = blockIdx.x * 256u + threadIdx.x;
    if (q >= npairs) return;
    uint32_t const node0 = 2u * q;
    uint32_t const row = node0 / static_cast<uint32_t>(nz);
    int const z0 = static_cast<int>(node0 - row * static_cast<uint32_t>(nz));
    int const y = static_cast<int>(row % static_cast<uint32_t>(ny)), x = static_cast<int>(row / static_cast<uint32_t>(ny));
    double2 const* src = reinterpret_cast<double2 const*>(in + static_cast<int64_t>(node0) * 3);
    double2 const a = __ldg(src), b = __ldg(src + 1), c = __ldg(src + 2);
    double const v[2][3] = {{a.x, a.y, b.x}, {b.y, c.x, c.y}};
    int64_t const px = fx + x - geo.front[0] + 1, py = fy + y - geo.front[1] + 1;
    int64_t const pz = fz + z0 - geo.front[2] + 1;
    // The spacings this pair can use, loaded once; a factor the rule leaves
    // out multiplies by 1.0, which is exact, so each product is the one the
    // table-driven kernel forms.
    double const hx = __ldg(geo.h[0] + px), ihx = __ldg(geo.inv_h[0] + px);
    double const hy = __ldg(geo.h[1] + py), ihy = __ldg(geo.inv_h[1] + py);
    double const hz[2] = {__ldg(geo.h[2] + pz), __ldg(geo.h[2] + pz + 1)};
    double const ihz[2] = {__ldg(geo.inv_h[2] + pz), __ldg(geo.inv_h[2] + pz + 1)};
    double r[2][3];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        double const hv[3] = {hx, hy, hz[k]}, ihv[3] = {ihx, ihy, ihz[k]};
#pragma unroll
        for (int t = 0; t < 3; ++t) {
            double f = static_cast<double>(star.sgn[t]);
            uint32_t const nm = star.num_mask[t], dm = star.den_mask[t];
#pragma unroll
            for (int ax = 0; ax < 3; ++ax) {
                f *= (nm & (1u << ax)) ? hv[ax] : 1.0;
                f *= (dm & (1u << ax)) ? ihv[ax] : 1.0;
            }
            double const vs = star.src[t] == 0 ? v[k][0] : (star.src[t] == 1 ? v[k][1] : v[k][2]);
            r[k][t] = f * vs;
        }
    }
    double2* dst = reinterpret_cast<double2*>(out + static_cast<int64_t>(node0) * 3);
    __stcs(dst, make_double2(r[0][0], r[0][1]));
    __stcs(dst + 1, make_double2(r[0][2], r[1][0]));
    __stcs(dst + 2, make_double2(r[1][1], r[1][2]));
}

// Stored per-node Hodge tensor (Full<k> x Antisym<n-k>) of the diagonal metric.
template <class T, int ND>
__global__ void fill_hodge_kernel(FieldView out, StarRule star, GeoCtx<T> g, int k, int n, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(out.data) + node_setup<ND>(out, flat, abs);
    int ntuples = 1;
    for (int i = 0; i < k; ++i) ntuples *= n;
    double inv_fact = 1.0;
    for (int i = 2; i <= k; ++i) inv_fact /= i;
    for (int tu = 0; tu < ntuples; ++tu) {
        int ids[kMaxNHodge];
        int r = tu;
        for (int a = k - 1; a >= 0; --a) {
            ids[a] = r % n;
            r /= n;
        }
        uint32_t mask = 0;
        bool unique = true;
        int inv = 0;
        for (int a = 0; a < k; ++a) {
            unique = unique && !(mask & (1u << ids[a]));
            mask |= 1u << ids[a];
            for (int b = a + 1; b < k; ++b) inv += ids[a] > ids[b];
        }
        for (int t = 0; t < star.ncomp_out; ++t) {
            T v = T(0);
            if (unique && star.den_mask[t] == mask) {
                T const m = star_factor(g, abs, star.num_mask[t], star.den_mask[t], star.sgn[t]);
                v = static_cast<T>((inv % 2 ? -1.0 : 1.0) * inv_fact) * m;
            }
            o[(tu * star.ncomp_out + t) * out.comp_stride] = v;
        }
    }
}

// ------------------------------------------------------------------ fused operators

// Everything the fused codifferential / Laplacian kernels need.
template <class T>
struct FusedParams
{
    FieldView in;
    FieldView out;
    GeoCtx<T> g;
    int n;
    int k;
    // delta d (k < n)
    CoboundaryRules d_k;        // d on the k-form (clamped)
    StarRule star_dk;           // (k+1)-form -> (n-k-1)-form
    CoboundaryRules dt_dual;    // d^T on the (n-k-1)-form dual (zero outside)
    StarRule star_dual;         // (n-k)-form -> k-form
    T sign_dd;
    // d delta (k > 0) / codifferential
    StarRule star_k;            // k-form -> (n-k)-form
    CoboundaryRules dt_codiff;  // d^T on the (n-k)-form dual (zero outside)
    StarRule star_codiff;       // (n-k+1)-form -> (k-1)-form
    T sign_codiff;
    CoboundaryRules d_km1;      // d on the (k-1)-form codifferential (clamped)
};

// (star_k w)(q) component c, zero outside the input domain.
template <class T, int ND>
__device__ T dual_of_input(FusedParams<T> const& P, int64_t const* q, int c)
{
    if (!inside<ND>(P.in, q)) return T(0);
    return star_factor(P.g, q, P.star_k.num_mask[c], P.star_k.den_mask[c], P.star_k.sgn[c])
           * load_at<T, ND>(P.in, q, P.star_k.src[c]);
}

// Codifferential of the input at node p (inside the input domain), component t.
template <class T, int ND>
__device__ T codiff_at(FusedParams<T> const& P, int64_t const* p, int t)
{
    int const c = P.star_codiff.src[t];
    T acc = T(0);
    for (int f = 0; f < P.dt_codiff.nfaces; ++f) {
        FaceRule const r = P.dt_codiff.rule[c][f];
        int64_t s[ND];
        offset_node<ND>(P.g.dm, p, r, s);
        T const v = dual_of_input<T, ND>(P, s, r.comp);
        acc = r.negative ? acc - v : acc + v;
    }
    T const dual_codiff = -acc;
    return P.sign_codiff
           * (star_factor(P.g, p, P.star_codiff.num_mask[t], P.star_codiff.den_mask[t], P.star_codiff.sgn[t])
              * dual_codiff);
}

// (star d w)(p) component c1, zero outside the input domain; d samples are clamped.
template <class T, int ND>
__device__ T dual_of_derivative(FusedParams<T> const& P, int64_t const* p, int c1)
{
    if (!inside<ND>(P.in, p)) return T(0);
    int const c0 = P.star_dk.src[c1];
    T acc = T(0);
    for (int f = 0; f < P.d_k.nfaces; ++f) {
        FaceRule const r = P.d_k.rule[c0][f];
        int64_t s[ND];
        offset_node<ND>(P.g.dm, p, r, s);
        clamp_to<ND>(P.in, s);
        T const v = load_at<T, ND>(P.in, s, r.comp);
        acc = r.negative ? acc - v : acc + v;
    }
    return star_factor(P.g, p, P.star_dk.num_mask[c1], P.star_dk.den_mask[c1], P.star_dk.sgn[c1]) * acc;
}

template <class T, bool DELTA_D, bool D_DELTA, int ND>
__global__ void fused_laplacian_kernel(FusedParams<T> P, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(P.out.data) + node_setup<ND>(P.out, flat, abs);
    for (int t = 0; t < P.out.ncomp; ++t) {
        T result = T(0);
        if constexpr (DELTA_D) {
            int const c2 = P.star_dual.src[t];
            T acc = T(0);
            for (int f = 0; f < P.dt_dual.nfaces; ++f) {
                FaceRule const r = P.dt_dual.rule[c2][f];
                int64_t s[ND];
                offset_node<ND>(P.g.dm, abs, r, s);
                T const v = dual_of_derivative<T, ND>(P, s, r.comp);
                acc = r.negative ? acc - v : acc + v;
            }
            T const dual_codiff = -acc;
            result = P.sign_dd
                     * (star_factor(P.g, abs, P.star_dual.num_mask[t], P.star_dual.den_mask[t], P.star_dual.sgn[t])
                        * dual_codiff);
        }
        if constexpr (D_DELTA) {
            T acc = T(0);
            for (int f = 0; f < P.d_km1.nfaces; ++f) {
                FaceRule const r = P.d_km1.rule[t][f];
                int64_t s[ND];
                offset_node<ND>(P.g.dm, abs, r, s);
                clamp_to<ND>(P.in, s);
                T const v = codiff_at<T, ND>(P, s, r.comp);
                acc = r.negative ? acc - v : acc + v;
            }
            result = DELTA_D ? result + acc : acc;
        }
        o[t * P.out.comp_stride] = result;
    }
}

template <class T, int ND>
__global__ void fused_codifferential_kernel(FusedParams<T> P, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(P.out.data) + node_setup<ND>(P.out, flat, abs);
    for (int t = 0; t < P.out.ncomp; ++t) o[t * P.out.comp_stride] = codiff_at<T, ND>(P, abs, t);
}

// Reference kernel 1 of codifferential_of_coboundary: clamped d of an
// r-form followed by the Hodge star of the (r+1)-form, at every node of `out`.
template <class T, int ND>
__global__ void deriv_star_kernel(FieldView in, FieldView out, CoboundaryRules rules, StarRule star, GeoCtx<T> g,
                                  int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(out.data) + node_setup<ND>(out, flat, abs);
    for (int t = 0; t < star.ncomp_out; ++t) {
        int const c0 = star.src[t];
        T acc = T(0);
        for (int f = 0; f < rules.nfaces; ++f) {
            FaceRule const r = rules.rule[c0][f];
            int64_t s[ND];
            offset_node<ND>(g.dm, abs, r, s);
            clamp_to<ND>(in, s);
            T const v = load_at<T, ND>(in, s, r.comp);
            acc = r.negative ? acc - v : acc + v;
        }
        o[t * out.comp_stride] = star_factor(g, abs, star.num_mask[t], star.den_mask[t], star.sgn[t]) * acc;
    }
}

// Reference kernel 2: d^T (zero outside `src`) of an r-form, Hodge star of
// the (r+1)-form, times the codifferential sign.
template <class T, int ND>
__global__ void transpose_star_kernel(FieldView src, FieldView out, CoboundaryRules rules, StarRule star, GeoCtx<T> g,
                                      T sign, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t abs[ND];
    T* o = static_cast<T*>(out.data) + node_setup<ND>(out, flat, abs);
    for (int t = 0; t < star.ncomp_out; ++t) {
        int const c = star.src[t];
        T acc = T(0);
        for (int f = 0; f < rules.nfaces; ++f) {
            FaceRule const r = rules.rule[c][f];
            int64_t s[ND];
            offset_node<ND>(g.dm, abs, r, s);
            T const v = inside<ND>(src, s) ? load_at<T, ND>(src, s, r.comp) : T(0);
            acc = r.negative ? acc - v : acc + v;
        }
        T const dual_codiff = -acc;
        o[t * out.comp_stride] = sign * (star_factor(g, abs, star.num_mask[t], star.den_mask[t], star.sgn[t]) * dual_codiff);
    }
}

// out += add (same shape, any strides).
template <class T, int ND>
__global__ void add_kernel(FieldView out, FieldView add, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t local[ND];
    unravel<ND>(out, flat, local);
    int64_t oo = 0, ao = 0;
#pragma unroll
    for (int d = 0; d < ND; ++d) {
        oo += local[d] * out.stride[d];
        ao += local[d] * add.stride[d];
    }
    for (int c = 0; c < out.ncomp; ++c)
        static_cast<T*>(out.data)[oo + c * out.comp_stride] += static_cast<T const*>(add.data)[ao + c * add.comp_stride];
}

constexpr int kBlock = 256;

unsigned grid_for(int64_t total)
{
    return static_cast<unsigned>((total + kBlock - 1) / kBlock);
}

// Call f(std::integral_constant<int, ND>{}) for the runtime rank nd (1..6).
template <class F>
void with_nd(int nd, F&& f)
{
    switch (nd) {
    case 1: f(std::integral_constant<int, 1>{}); break;
    case 2: f(std::integral_constant<int, 2>{}); break;
    case 3: f(std::integral_constant<int, 3>{}); break;
    case 4: f(std::integral_constant<int, 4>{}); break;
    case 5: f(std::integral_constant<int, 5>{}); break;
    default: f(std::integral_constant<int, 6>{}); break;
    }
}

template <class T>
GeoCtx<T> make_geo_ctx(Geometry const& geo, uint32_t mask, int ndims)
{
    GeoCtx<T> g {};
    g.geo = geo_view<T>(geo);
    g.dm.n = form_dims(mask, ndims, g.dm.dims);
    return g;
}

template <class T>
FusedParams<T> make_fused(Geometry const& geo, uint32_t mask, int k, sil_field const& in, sil_field const& out)
{
    FusedParams<T> P {};
    P.in = to_view(in);
    P.out = to_view(out);
    P.g = make_geo_ctx<T>(geo, mask, in.ndims);
    int const n = P.g.dm.n;
    P.n = n;
    P.k = k;
    if (k < n) {
        P.d_k = make_rules(n, k, false);
        P.star_dk = make_star(n, k + 1);
        P.dt_dual = make_rules(n, n - k - 1, true);
        P.star_dual = make_star(n, n - k);
        P.sign_dd = ((n * (k + 2) + 1) % 2) ? T(-1) : T(1);
    }
    if (k > 0) {
        P.star_k = make_star(n, k);
        P.dt_codiff = make_rules(n, n - k, true);
        P.star_codiff = make_star(n, n - k + 1);
        P.sign_codiff = ((n * (k + 1) + 1) % 2) ? T(-1) : T(1);
        P.d_km1 = make_rules(n, k - 1, false);
    }
    return P;
}

template <class T>
void launch_coboundary_t(cudaStream_t stream, CoboundaryRules const& rules, DimMap const& dm, sil_field const& in,
                         sil_field const& out, bool transposed, int64_t total)
{
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (transposed)
            coboundary_kernel<T, true, ND><<<grid_for(total), kBlock, 0, stream>>>(to_view(in), to_view(out), rules, dm, total);
        else
            coboundary_kernel<T, false, ND><<<grid_for(total), kBlock, 0, stream>>>(to_view(in), to_view(out), rules, dm, total);
    });
}

template <class T>
void launch_fused_t(cudaStream_t stream, Geometry const& geo, uint32_t mask, int k, sil_field const& in,
                    sil_field const& out, int64_t total)
{
    auto P = make_fused<T>(geo, mask, k, in, out);
    bool const dd = k < P.n, dl = k > 0;
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (dd && dl) fused_laplacian_kernel<T, true, true, ND><<<grid_for(total), kBlock, 0, stream>>>(P, total);
        else if (dd) fused_laplacian_kernel<T, true, false, ND><<<grid_for(total), kBlock, 0, stream>>>(P, total);
        else fused_laplacian_kernel<T, false, true, ND><<<grid_for(total), kBlock, 0, stream>>>(P, total);
    });
}

} // namespace

// ------------------------------------------------------------------ launchers

sil_status launch_coboundary(cudaStream_t stream, uint32_t mask, int k, sil_field const& in, sil_field const& out,
                             bool transposed)
{
    DimMap dm {};
    dm.n = form_dims(mask, in.ndims, dm.dims);
    CoboundaryRules const rules = make_rules(dm.n, k, transposed);
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    if (in.dtype == SIL_F64) launch_coboundary_t<double>(stream, rules, dm, in, out, transposed, total);
    else launch_coboundary_t<float>(stream, rules, dm, in, out, transposed, total);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_hodge(cudaStream_t stream, Geometry const& geo, uint32_t mask, int k, sil_field const& in,
                        sil_field const& out)
{
    int dims[kMaxDims];
    int const n = form_dims(mask, in.ndims, dims);
    StarRule const star = make_star(n, k);
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    // dense 3D fields (the 3D magnetostatics / curl-curl layout): row kernel
    auto dense = [](sil_field const& f) {
        return f.ndims == 3 && f.comp_stride == 1 && f.stride[2] == f.ncomp && f.stride[1] == f.extent[2] * f.ncomp
               && f.stride[0] == f.extent[1] * f.extent[2] * f.ncomp;
    };
    bool same_box = in.ndims == 3 && out.ndims == 3;
    for (int d = 0; d < 3 && same_box; ++d) same_box = in.front[d] == out.front[d] && in.extent[d] == out.extent[d];
    if (n == 3 && mask == 7u && same_box && dense(in) && dense(out) && out.extent[0] * out.extent[1] < (int64_t(1) << 30)
        && out.extent[2] < (int64_t(1) << 30)) {
        int const nx = static_cast<int>(out.extent[0]), ny = static_cast<int>(out.extent[1]);
        int const nz = static_cast<int>(out.extent[2]);
        int const zchunks = (nz + 255) / 256;
        int64_t const blocks = static_cast<int64_t>(nx) * ny * zchunks;
        bool const pairable = in.dtype == SIL_F64 && in.ncomp == 3 && out.ncomp == 3 && nz % 2 == 0
                              && reinterpret_cast<uintptr_t>(in.data) % 16 == 0
                              && reinterpret_cast<uintptr_t>(out.data) % 16 == 0;
        if (pairable) {
            int64_t const npairs = static_cast<int64_t>(nx) * ny * (nz / 2);
            if (npairs < (int64_t(1) << 30)) {
                unsigned const b2 = static_cast<unsigned>((npairs + 255) / 256);
                hodge3d_dense_pair_kernel<<<b2, 256, 0, stream>>>(
                        static_cast<double const*>(in.data), static_cast<double*>(out.data), star, geo_view<double>(geo),
                        out.front[0], out.front[1], out.front[2], ny, nz, static_cast<uint32_t>(npairs));
                SIL_CUDA_CHECK(cudaGetLastError());
                return SIL_OK;
            }
        }
        if (blocks < (int64_t(1) << 31)) {
            if (in.dtype == SIL_F64)
                hodge3d_dense_kernel<double><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
                        static_cast<double const*>(in.data), static_cast<double*>(out.data), in.ncomp, out.ncomp, star,
                        geo_view<double>(geo), out.front[0], out.front[1], out.front[2], nx, ny, nz, zchunks);
            else
                hodge3d_dense_kernel<float><<<static_cast<unsigned>(blocks), 256, 0, stream>>>(
                        static_cast<float const*>(in.data), static_cast<float*>(out.data), in.ncomp, out.ncomp, star,
                        geo_view<float>(geo), out.front[0], out.front[1], out.front[2], nx, ny, nz, zchunks);
            SIL_CUDA_CHECK(cudaGetLastError());
            return SIL_OK;
        }
    }
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (in.dtype == SIL_F64)
            hodge_kernel<double, ND><<<grid_for(total), kBlock, 0, stream>>>(to_view(in), to_view(out), star,
                                                                             make_geo_ctx<double>(geo, mask, in.ndims), total);
        else
            hodge_kernel<float, ND><<<grid_for(total), kBlock, 0, stream>>>(to_view(in), to_view(out), star,
                                                                            make_geo_ctx<float>(geo, mask, in.ndims), total);
    });
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_fill_hodge(cudaStream_t stream, Geometry const& geo, int k, sil_field const& out)
{
    int const n = geo.n;
    StarRule const star = make_star(n, k);
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    uint32_t const mask = (1u << n) - 1;
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (out.dtype == SIL_F64)
            fill_hodge_kernel<double, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    to_view(out), star, make_geo_ctx<double>(geo, mask, n), k, n, total);
        else
            fill_hodge_kernel<float, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    to_view(out), star, make_geo_ctx<float>(geo, mask, n), k, n, total);
    });
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_fused_laplacian(cudaStream_t stream, Geometry const& geo, uint32_t mask, int k, sil_field const& in,
                                  sil_field const& out)
{
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    if (in.dtype == SIL_F64) launch_fused_t<double>(stream, geo, mask, k, in, out, total);
    else launch_fused_t<float>(stream, geo, mask, k, in, out, total);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_codifferential(cudaStream_t stream, Geometry const& geo, uint32_t mask, int k, sil_field const& in,
                                 sil_field const& out)
{
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (in.dtype == SIL_F64)
            fused_codifferential_kernel<double, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    make_fused<double>(geo, mask, k, in, out), total);
        else
            fused_codifferential_kernel<float, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    make_fused<float>(geo, mask, k, in, out), total);
    });
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_deriv_star(cudaStream_t stream, Geometry const& geo, uint32_t mask, int r, sil_field const& in,
                             sil_field const& out)
{
    int dims[kMaxDims];
    int const n = form_dims(mask, in.ndims, dims);
    CoboundaryRules const rules = make_rules(n, r, false);
    StarRule const star = make_star(n, r + 1);
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (in.dtype == SIL_F64)
            deriv_star_kernel<double, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    to_view(in), to_view(out), rules, star, make_geo_ctx<double>(geo, mask, in.ndims), total);
        else
            deriv_star_kernel<float, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    to_view(in), to_view(out), rules, star, make_geo_ctx<float>(geo, mask, in.ndims), total);
    });
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_transpose_star(cudaStream_t stream, Geometry const& geo, uint32_t mask, int r, double sign,
                                 sil_field const& src, sil_field const& out)
{
    int dims[kMaxDims];
    int const n = form_dims(mask, src.ndims, dims);
    CoboundaryRules const rules = make_rules(n, r, true);
    StarRule const star = make_star(n, r + 1);
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (src.dtype == SIL_F64)
            transpose_star_kernel<double, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    to_view(src), to_view(out), rules, star, make_geo_ctx<double>(geo, mask, src.ndims), sign, total);
        else
            transpose_star_kernel<float, ND><<<grid_for(total), kBlock, 0, stream>>>(
                    to_view(src), to_view(out), rules, star, make_geo_ctx<float>(geo, mask, src.ndims),
                    static_cast<float>(sign), total);
    });
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

sil_status launch_add(cudaStream_t stream, sil_field const& out, sil_field const& add)
{
    int64_t const total = node_count(out);
    if (total == 0) return SIL_OK;
    with_nd(out.ndims, [&](auto ndc) {
        constexpr int ND = decltype(ndc)::value;
        if (out.dtype == SIL_F64)
            add_kernel<double, ND><<<grid_for(total), kBlock, 0, stream>>>(to_view(out), to_view(add), total);
        else
            add_kernel<float, ND><<<grid_for(total), kBlock, 0, stream>>>(to_view(out), to_view(add), total);
    });
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

} // namespace sil
