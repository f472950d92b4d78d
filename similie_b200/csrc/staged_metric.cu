// staged_metric.cu -- the staged codifferential and Hodge Laplacian built
// from a (metric, position) pair: SimiLie's
//   StagedCodifferential(exec, tensor, metric, position)
//     src/similie/exterior/codifferential.hpp:398-437 (ctor), 439-507 (run)
//   StagedLaplacian(exec, laplacian_tensor, tensor, metric, position)
//     src/similie/exterior/laplacian.hpp:261-310 (rank 0 ctor), 508-597
//     (intermediate ranks), 599-647 (their run), 740-789 (top rank)
// Set-up fills the per-node Hodge tensors the reference stores
// (fill_discrete_hodge_star with the metric, hodge_metric.cu) over the
// position lattice:
//   h[0]  (k+1)-form -> (n-k-1)-form   delta d, after d       (k < n)
//   h[1]  (n-k)-form -> k-form         delta d, after d^T     (k < n)
//   h[2]  k-form -> (n-k)-form         d delta, on the input  (k > 0)
//   h[3]  (n-k+1)-form -> (k-1)-form   d delta, after d^T     (k > 0)
// and every run is ONE kernel: each output node gathers the stored tensors
// and the input at the few neighbouring nodes the reference's passes would
// read back from their intermediate buffers (the dual buffers and the
// codifferential buffer, all over the input lattice), so nothing but the
// input, the stored tensors and the output touches HBM.
//
// The arithmetic follows the reference's order term by term: tensor_prod
// sums the n^K index tuples of the stored Full<K> x Antisym<n-K> tensor in
// order (a tuple with a repeated index contributes 0 * h), d and d^T sum the
// chain's faces first half then second half, d^T negates its sum, and the
// codifferential sign (-1)^{n(k+1)+1} is applied last.  FP64, lattices over
// exactly the n <= 3 form dimensions (no spectator dimensions).
#include <algorithm>
#include <new>

#include "sil_internal.cuh"

namespace sil {

namespace {

constexpr int kN = 3;
constexpr int kTuples = 27;  // n^K for n, K <= 3
constexpr int kC = 3;        // C(n, r) for n <= 3

// The index tuples of a stored tensor of rank K over n dims: tuple tu reads
// canonical component comp[tu] of the form with sign sign[tu] (0: a
// repeated index, the antisymmetric form is zero there).
struct TupleTable
{
    int ntuples;  // n^K
    int nq;       // C(n, n-K), components of the image
    int8_t comp[kTuples];
    int8_t sign[kTuples];
};

TupleTable make_tuples(int n, int K)
{
    TupleTable t {};
    t.ntuples = static_cast<int>(ipow(n, K));
    t.nq = static_cast<int>(binom(n, n - K));
    auto const combos = combinations(n, K);
    for (int tu = 0; tu < t.ntuples; ++tu) {
        int tuple[kN];
        int r = tu;
        for (int a = K - 1; a >= 0; --a) {
            tuple[a] = r % n;
            r /= n;
        }
        uint32_t mask = 0;
        bool repeated = false;
        for (int a = 0; a < K; ++a) {
            repeated = repeated || (mask & (1u << tuple[a]));
            mask |= 1u << tuple[a];
        }
        if (repeated) {
            t.comp[tu] = 0;
            t.sign[tu] = 0;
            continue;
        }
        int inv = 0;
        for (int i = 0; i < K; ++i)
            for (int j = i + 1; j < K; ++j) inv += tuple[i] > tuple[j];
        int c = 0;
        while (combos[c] != mask) ++c;
        t.comp[tu] = static_cast<int8_t>(c);
        t.sign[tu] = static_cast<int8_t>(inv % 2 ? -1 : 1);
    }
    return t;
}

struct StoredParams
{
    FieldView in;
    FieldView out;
    FieldView h[4];
    TupleTable tt[4];
    CoboundaryRules d_k;    // d on the k-form (clamped)
    CoboundaryRules dt_a;   // d^T on the (n-k-1)-form (zero outside)
    CoboundaryRules dt_b;   // d^T on the (n-k)-form (zero outside)
    CoboundaryRules d_km1;  // d on the (k-1)-form (clamped)
    int k;
    int ncomp_in;           // C(n, k)
    int ncomp_out;
    bool neg_dd;            // sign of the codifferential of the (k+1)-form
    bool neg_codiff;        // sign of the codifferential of the k-form
};

template <int N>
__device__ __forceinline__ bool inside_n(FieldView const& f, int64_t const* a)
{
    bool in = true;
#pragma unroll
    for (int d = 0; d < N; ++d) in = in && a[d] >= f.front[d] && a[d] < f.front[d] + f.extent[d];
    return in;
}

template <int N>
__device__ __forceinline__ int64_t offset_n(FieldView const& f, int64_t const* a)
{
    int64_t off = 0;
#pragma unroll
    for (int d = 0; d < N; ++d) off += (a[d] - f.front[d]) * f.stride[d];
    return off;
}

template <int N>
__device__ __forceinline__ void clamp_n(FieldView const& f, int64_t* a)
{
#pragma unroll
    for (int d = 0; d < N; ++d) a[d] = min(max(a[d], f.front[d]), f.front[d] + f.extent[d] - 1);
}

// Index of a face's sample point among {node, node +- e_0, ..., node +- e_{N-1}}:
// 0 for the node itself, a + 1 for a shift along axis a.
template <int N>
__device__ __forceinline__ int face_point(FaceRule const& r)
{
    int j = 0;
#pragma unroll
    for (int a = 0; a < N; ++a) j = r.offset[a] != 0 ? a + 1 : j;
    return j;
}

// Component t of tensor_prod(form, stored tensor at `node`).
// Ref: src/similie/tensor/tensor_prod.hpp:108-157 as the staged operators use it.
template <int N>
__device__ double hodge_dot(FieldView const& h, TupleTable const& tt, int64_t const* node, double const* vals, int t)
{
    double const* hp = static_cast<double const*>(h.data) + offset_n<N>(h, node);
    double acc = 0.;
    for (int tu = 0; tu < tt.ntuples; ++tu) {
        int const sg = tt.sign[tu];
        double const fv = sg == 0 ? 0. : (sg > 0 ? vals[tt.comp[tu]] : -vals[tt.comp[tu]]);
        acc += fv * hp[(tu * tt.nq + t) * h.comp_stride];
    }
    return acc;
}

// Reference kernel 1 of codifferential_of_coboundary at node q: clamped d of
// the input, then the stored star h[0]; zero outside the input lattice (the
// dual buffer spans the input lattice and d^T reads it zero-outside).
// Ref: src/similie/exterior/laplacian.hpp:78-108
template <int N>
__device__ void dual_of_derivative(StoredParams const& P, int64_t const* q, double* dual)
{
    int const nq = P.tt[0].nq;
    if (!inside_n<N>(P.in, q)) {
        for (int c = 0; c < nq; ++c) dual[c] = 0.;
        return;
    }
    double deriv[kC];
    double const* in = static_cast<double const*>(P.in.data);
    for (int c = 0; c < P.d_k.ncomp_out; ++c) {
        double acc = 0.;
        for (int f = 0; f < P.d_k.nfaces; ++f) {
            FaceRule const r = P.d_k.rule[c][f];
            int64_t s[N];
#pragma unroll
            for (int d = 0; d < N; ++d) s[d] = q[d] + r.offset[d];
            clamp_n<N>(P.in, s);
            double const v = in[offset_n<N>(P.in, s) + r.comp * P.in.comp_stride];
            acc = r.negative ? acc - v : acc + v;
        }
        deriv[c] = acc;
    }
    for (int c = 0; c < nq; ++c) dual[c] = hodge_dot<N>(P.h[0], P.tt[0], q, deriv, c);
}

// The codifferential of the input k-form at node q, all C(n, k-1)
// components: star h[2] of the input at q and q - e_a (zero outside the
// input lattice), d^T (negated face sum), star h[3] at q, sign.
// Ref: src/similie/exterior/codifferential.hpp:460-504
template <int N>
__device__ void codiff_vec(StoredParams const& P, int64_t const* q, double* out)
{
    double db[N + 1][kC];
    double const* in = static_cast<double const*>(P.in.data);
    int const nq2 = P.tt[2].nq;
    for (int j = 0; j <= N; ++j) {
        int64_t s[N];
#pragma unroll
        for (int d = 0; d < N; ++d) s[d] = q[d] - (j == d + 1 ? 1 : 0);
        if (!inside_n<N>(P.in, s)) {
            for (int c = 0; c < nq2; ++c) db[j][c] = 0.;
            continue;
        }
        double w[kC];
        int64_t const off = offset_n<N>(P.in, s);
        for (int c = 0; c < P.ncomp_in; ++c) w[c] = in[off + c * P.in.comp_stride];
        for (int c = 0; c < nq2; ++c) db[j][c] = hodge_dot<N>(P.h[2], P.tt[2], s, w, c);
    }
    double dcb[kC];
    for (int c = 0; c < P.dt_b.ncomp_out; ++c) {
        double acc = 0.;
        for (int f = 0; f < P.dt_b.nfaces; ++f) {
            FaceRule const r = P.dt_b.rule[c][f];
            double const v = db[face_point<N>(r)][r.comp];
            acc = r.negative ? acc - v : acc + v;
        }
        dcb[c] = -acc;
    }
    for (int t = 0; t < P.tt[3].nq; ++t) {
        double const v = hodge_dot<N>(P.h[3], P.tt[3], q, dcb, t);
        out[t] = P.neg_codiff ? -v : v;
    }
}

template <int N>
__device__ __forceinline__ int64_t out_node(FieldView const& out, int64_t flat, int64_t* abs)
{
    int64_t off = 0;
#pragma unroll
    for (int d = N - 1; d >= 0; --d) {
        int64_t const l = flat % out.extent[d];
        flat /= out.extent[d];
        abs[d] = out.front[d] + l;
        off += l * out.stride[d];
    }
    return off;
}

// Hodge Laplacian at every node of `out`: delta d (k < n), d delta (k > 0),
// summed in the reference's order (delta d written first, d delta added).
template <int N>
__global__ void __launch_bounds__(128) stored_laplacian_kernel(StoredParams P, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t p[N];
    double* o = static_cast<double*>(P.out.data) + out_node<N>(P.out, flat, p);
    double res[kC] = {0., 0., 0.};
    bool const dd = P.k < N, ddelta = P.k > 0;
    if (dd) {
        // delta of the (k+1)-form d w: dual at p and p - e_a, d^T, star h[1].
        // Ref: src/similie/exterior/laplacian.hpp:110-152
        double da[N + 1][kC];
        for (int j = 0; j <= N; ++j) {
            int64_t s[N];
#pragma unroll
            for (int d = 0; d < N; ++d) s[d] = p[d] - (j == d + 1 ? 1 : 0);
            dual_of_derivative<N>(P, s, da[j]);
        }
        double dc[kC];
        for (int c = 0; c < P.dt_a.ncomp_out; ++c) {
            double acc = 0.;
            for (int f = 0; f < P.dt_a.nfaces; ++f) {
                FaceRule const r = P.dt_a.rule[c][f];
                double const v = da[face_point<N>(r)][r.comp];
                acc = r.negative ? acc - v : acc + v;
            }
            dc[c] = -acc;
        }
        for (int t = 0; t < P.ncomp_out; ++t) {
            double const v = hodge_dot<N>(P.h[1], P.tt[1], p, dc, t);
            res[t] = P.neg_dd ? -v : v;
        }
    }
    if (ddelta) {
        // d of the codifferential, sampled clamped to the input lattice at p
        // and p + e_a.  Ref: src/similie/exterior/laplacian.hpp:614-647
        double cv[N + 1][kC];
        for (int j = 0; j <= N; ++j) {
            int64_t s[N];
#pragma unroll
            for (int d = 0; d < N; ++d) s[d] = p[d] + (j == d + 1 ? 1 : 0);
            clamp_n<N>(P.in, s);
            codiff_vec<N>(P, s, cv[j]);
        }
        for (int t = 0; t < P.ncomp_out; ++t) {
            double acc = 0.;
            for (int f = 0; f < P.d_km1.nfaces; ++f) {
                FaceRule const r = P.d_km1.rule[t][f];
                double const v = cv[face_point<N>(r)][r.comp];
                acc = r.negative ? acc - v : acc + v;
            }
            res[t] = dd ? res[t] + acc : acc;
        }
    }
    for (int t = 0; t < P.ncomp_out; ++t) o[t * P.out.comp_stride] = res[t];
}

// Codifferential of the input k-form at every node of `out`.
template <int N>
__global__ void __launch_bounds__(128) stored_codifferential_kernel(StoredParams P, int64_t total)
{
    int64_t const flat = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (flat >= total) return;
    int64_t p[N];
    double* o = static_cast<double*>(P.out.data) + out_node<N>(P.out, flat, p);
    double cv[kC];
    codiff_vec<N>(P, p, cv);
    for (int t = 0; t < P.ncomp_out; ++t) o[t * P.out.comp_stride] = cv[t];
}

bool lattice_inside(sil_field const& inner, sil_field const& outer, int n)
{
    for (int d = 0; d < n; ++d)
        if (inner.extent[d] > 0 && (inner.front[d] < outer.front[d]
                                    || inner.front[d] + inner.extent[d] > outer.front[d] + outer.extent[d]))
            return false;
    return true;
}

StoredParams make_params(StoredHodges const& H, sil_field const& in, sil_field const& out, int ncomp_out)
{
    int const n = H.n, k = H.k;
    StoredParams P {};
    P.in = to_view(in);
    P.out = to_view(out);
    for (int w = 0; w < 4; ++w) {
        if (H.h[w].data == nullptr) continue;
        P.h[w] = to_view(H.h[w]);
        P.tt[w] = make_tuples(n, H.kin[w]);
    }
    P.k = k;
    P.ncomp_in = static_cast<int>(binom(n, k));
    P.ncomp_out = ncomp_out;
    if (k < n) {
        P.d_k = make_rules(n, k, false);
        P.dt_a = make_rules(n, n - k - 1, true);
    }
    if (k > 0) {
        P.dt_b = make_rules(n, n - k, true);
        P.d_km1 = make_rules(n, k - 1, false);
    }
    P.neg_dd = (n * (k + 2) + 1) % 2 == 1;
    P.neg_codiff = (n * (k + 1) + 1) % 2 == 1;
    return P;
}

sil_status check_metric_fields(int n, int k, sil_field const* position, sil_field const* metric, char const* who)
{
    std::string const w(who);
    if (n < 1 || n > kN) return fail(SIL_ERR_INVALID, w + ": need 1 <= n <= 3");
    if (k < 0 || k > n) return fail(SIL_ERR_INVALID, w + ": rank out of range");
    sil_status st = check_field(position, "position", n);
    if (st == SIL_OK && metric != nullptr) st = check_field(metric, "metric", n * n);
    if (st != SIL_OK) return st;
    if (position->dtype != SIL_F64 || (metric != nullptr && metric->dtype != SIL_F64))
        return fail(SIL_ERR_UNSUPPORTED, w + ": FP64 position and metric only");
    if (position->ndims != n || (metric != nullptr && metric->ndims != n))
        return fail(SIL_ERR_INVALID, w + ": position and metric must span exactly the n form dims");
    if (metric != nullptr && !lattice_inside(*position, *metric, n))
        return fail(SIL_ERR_INVALID, w + ": the metric lattice must cover the position lattice");
    return SIL_OK;
}

sil_status check_run_fields(StoredHodges const& H, sil_field const* in, sil_field const* out, int k_out,
                            char const* who)
{
    std::string const w(who);
    int const n = H.n;
    sil_status st = check_field(in, "in", static_cast<int>(binom(n, H.k)));
    if (st == SIL_OK) st = check_field(out, "out", static_cast<int>(binom(n, k_out)));
    if (st != SIL_OK) return st;
    if (in->dtype != SIL_F64 || out->dtype != SIL_F64) return fail(SIL_ERR_UNSUPPORTED, w + ": FP64 fields only");
    if (in->ndims != n || out->ndims != n)
        return fail(SIL_ERR_INVALID, w + ": fields must span exactly the n form dims (no spectator dims)");
    if (!lattice_inside(*in, H.lattice, n) || !lattice_inside(*out, H.lattice, n))
        return fail(SIL_ERR_INVALID, w + ": fields must lie inside the position lattice the stars were filled on");
    return SIL_OK;
}

template <class Kern>
sil_status launch_n(int n, Kern k1, Kern k2, Kern k3, StoredParams const& P, int64_t total, cudaStream_t s)
{
    if (total == 0) return SIL_OK;
    unsigned const grid = static_cast<unsigned>((total + 127) / 128);
    Kern const k = n == 1 ? k1 : (n == 2 ? k2 : k3);
    k<<<grid, 128, 0, s>>>(P, total);
    SIL_CUDA_CHECK(cudaGetLastError());
    return SIL_OK;
}

} // namespace

sil_status fill_stored_hodges(cudaStream_t stream, int n, int k, sil_field const& position, sil_field const* metric,
                              bool laplacian, void** mem, StoredHodges* out)
{
    *mem = nullptr;
    StoredHodges H {};
    H.n = n;
    H.k = k;
    H.lattice = position;
    int const kin[4] = {k + 1, n - k, k, n - k + 1};
    bool need[4];
    need[0] = need[1] = laplacian && k < n;
    need[2] = need[3] = k > 0;
    int64_t nodes = 1;
    for (int d = 0; d < n; ++d) nodes *= position.extent[d];
    size_t bytes = 0;
    size_t off[4] = {0, 0, 0, 0};
    for (int w = 0; w < 4; ++w) {
        H.kin[w] = kin[w];
        if (!need[w]) continue;
        off[w] = bytes;
        bytes += (static_cast<size_t>(nodes) * ipow(n, kin[w]) * binom(n, n - kin[w]) * sizeof(double) + 255) / 256
                 * 256;
    }
    if (bytes > 0) SIL_CUDA_CHECK(cudaMalloc(mem, bytes));
    for (int w = 0; w < 4; ++w) {
        if (!need[w]) continue;
        sil_field& f = H.h[w];
        f = sil_field {};
        f.data = static_cast<char*>(*mem) + off[w];
        f.dtype = SIL_F64;
        f.ndims = n;
        f.ncomp = static_cast<int32_t>(ipow(n, kin[w]) * binom(n, n - kin[w]));
        f.comp_stride = 1;
        int64_t s = f.ncomp;
        for (int d = n - 1; d >= 0; --d) {
            f.front[d] = position.front[d];
            f.extent[d] = position.extent[d];
            f.stride[d] = s;
            s *= position.extent[d];
        }
        sil_status const st = sil_fill_discrete_hodge_star_metric(stream, n, kin[w], &position, metric, &f);
        if (st != SIL_OK) {
            cudaFree(*mem);
            *mem = nullptr;
            return st;
        }
    }
    *out = H;
    return SIL_OK;
}

sil_status check_stored_laplacian(int n, int k, sil_field const* position, sil_field const* metric)
{
    return check_metric_fields(n, k, position, metric, "sil_laplacian_plan_create_metric");
}

sil_status launch_stored_laplacian(cudaStream_t s, StoredHodges const& H, sil_field const* in, sil_field const* out)
{
    sil_status const st = check_run_fields(H, in, out, H.k, "sil_laplacian_run");
    if (st != SIL_OK) return st;
    StoredParams const P = make_params(H, *in, *out, static_cast<int>(binom(H.n, H.k)));
    return launch_n(H.n, stored_laplacian_kernel<1>, stored_laplacian_kernel<2>, stored_laplacian_kernel<3>, P,
                    node_count(*out), s);
}

} // namespace sil

using namespace sil;

struct sil_codifferential_plan_s
{
    StoredHodges hodges {};
    void* mem = nullptr;
};

extern "C" {

sil_status sil_codifferential_plan_create(sil_codifferential_plan* plan, sil_stream stream, int n, int k,
                                          const sil_field* position, const sil_field* metric)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_codifferential_plan_create: NULL plan");
    *plan = nullptr;
    sil_status st = check_metric_fields(n, k, position, metric, "sil_codifferential_plan_create");
    if (st != SIL_OK) return st;
    if (k < 1) return fail(SIL_ERR_INVALID, "sil_codifferential_plan_create: the codifferential of a 0-form is not defined");
    auto* p = new (std::nothrow) sil_codifferential_plan_s();
    if (p == nullptr) return fail(SIL_ERR_ALLOC, "sil_codifferential_plan_create: host allocation");
    st = fill_stored_hodges(static_cast<cudaStream_t>(stream), n, k, *position, metric, false, &p->mem, &p->hodges);
    if (st != SIL_OK) {
        delete p;
        return st;
    }
    *plan = p;
    return SIL_OK;
}

sil_status sil_codifferential_run(sil_codifferential_plan plan, sil_stream stream, const sil_field* in,
                                  sil_field* out)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_codifferential_run: NULL plan");
    StoredHodges const& H = plan->hodges;
    sil_status const st = check_run_fields(H, in, out, H.k - 1, "sil_codifferential_run");
    if (st != SIL_OK) return st;
    StoredParams const P = make_params(H, *in, *out, static_cast<int>(binom(H.n, H.k - 1)));
    return launch_n(H.n, stored_codifferential_kernel<1>, stored_codifferential_kernel<2>,
                    stored_codifferential_kernel<3>, P, node_count(*out), static_cast<cudaStream_t>(stream));
}

sil_status sil_codifferential_plan_destroy(sil_codifferential_plan plan)
{
    if (plan == nullptr) return SIL_OK;
    cudaFree(plan->mem);
    delete plan;
    return SIL_OK;
}

} // extern "C"
