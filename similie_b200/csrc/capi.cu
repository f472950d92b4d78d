// capi.cu -- C ABI entry points of the DEC operators (see include/sil_b200.h).
#include <algorithm>
#include <cstdlib>
#include <new>
#include <string>

#include "sil_internal.cuh"

namespace sil {

sil_status launch_coboundary(cudaStream_t, uint32_t, int, sil_field const&, sil_field const&, bool);
sil_status launch_hodge(cudaStream_t, Geometry const&, uint32_t, int, sil_field const&, sil_field const&);
sil_status launch_fill_hodge(cudaStream_t, Geometry const&, int, sil_field const&);
sil_status launch_fused_laplacian(cudaStream_t, Geometry const&, uint32_t, int, sil_field const&, sil_field const&);
sil_status launch_codifferential(cudaStream_t, Geometry const&, uint32_t, int, sil_field const&, sil_field const&);
sil_status launch_deriv_star(cudaStream_t, Geometry const&, uint32_t, int, sil_field const&, sil_field const&);
sil_status launch_transpose_star(cudaStream_t, Geometry const&, uint32_t, int, double, sil_field const&,
                                 sil_field const&);
sil_status launch_add(cudaStream_t, sil_field const&, sil_field const&);
bool lap2d_layout_ok(sil_field const&, sil_field const&, int);
bool lap2d_1form_tma_ok(sil_field const&, sil_field const&);
sil_status launch_lap2d_0form(cudaStream_t, Geometry const&, sil_field const&, sil_field const&);
sil_status launch_lap2d_0form(cudaStream_t, Geometry const&, sil_field const&, sil_field const&, int);
sil_status autotune_lap2d_0form(cudaStream_t, Geometry const&, sil_field const&, sil_field const&, int*);
sil_status launch_lap2d_1form_tma(cudaStream_t, Geometry const&, sil_field const&, sil_field const&, int*, int);
sil_status launch_lap2d_1form_tma(cudaStream_t, Geometry const&, sil_field const&, sil_field const&, int*, int, int);
sil_status autotune_lap2d_1form(cudaStream_t, Geometry const&, sil_field const&, sil_field const&, int*, int*, float*);

namespace {

cudaStream_t as_stream(sil_stream s)
{
    return static_cast<cudaStream_t>(s);
}

sil_status check_pair(uint32_t mask, int k, sil_field const* in, sil_field const* out, int n_max, int k_out,
                      char const* what, int* n_out)
{
    sil_status st = check_field(in, "in", -1);
    if (st != SIL_OK) return st;
    st = check_field(out, "out", -1);
    if (st != SIL_OK) return st;
    if (in->ndims != out->ndims) return fail(SIL_ERR_INVALID, std::string(what) + ": in/out ndims differ");
    if (in->dtype != out->dtype) return fail(SIL_ERR_INVALID, std::string(what) + ": in/out dtypes differ");
    if (mask == 0 || (mask >> in->ndims) != 0)
        return fail(SIL_ERR_INVALID, std::string(what) + ": form_mask selects no or nonexistent dims");
    int dims[kMaxDims];
    int const n = form_dims(mask, in->ndims, dims);
    if (n > n_max)
        return fail(SIL_ERR_UNSUPPORTED, std::string(what) + ": at most " + std::to_string(n_max) + " form dims");
    if (k < 0 || k > n) return fail(SIL_ERR_INVALID, std::string(what) + ": rank out of range");
    if (in->ncomp != binom(n, k))
        return fail(SIL_ERR_INVALID, std::string(what) + ": input must hold C(n,k) components");
    if (k_out < 0 || k_out > n || out->ncomp != binom(n, k_out))
        return fail(SIL_ERR_INVALID, std::string(what) + ": output must hold C(n," + std::to_string(k_out) + ") components");
    *n_out = n;
    return SIL_OK;
}

// The geometry must cover every node the operator evaluates a Hodge factor at.
sil_status check_geometry(sil_geometry geometry, uint32_t mask, sil_field const& f, int n, char const* what)
{
    if (geometry == nullptr) return fail(SIL_ERR_INVALID, std::string(what) + ": NULL geometry");
    Geometry const& g = geometry->g;
    if (g.n != n) return fail(SIL_ERR_INVALID, std::string(what) + ": geometry dimension differs from the form dims");
    int dims[kMaxDims];
    form_dims(mask, f.ndims, dims);
    for (int a = 0; a < n; ++a) {
        int64_t const lo = f.front[dims[a]], hi = f.front[dims[a]] + f.extent[dims[a]];
        if (f.extent[dims[a]] > 0 && (lo < g.front[a] || hi > g.front[a] + g.npoints[a]))
            return fail(SIL_ERR_INVALID, std::string(what) + ": field extends beyond the geometry");
    }
    return SIL_OK;
}

sil_field dense_like(sil_field const& like, int ncomp, void* data)
{
    sil_field f = like;
    f.data = data;
    f.ncomp = ncomp;
    f.comp_stride = 1;
    int64_t s = ncomp;
    for (int d = like.ndims - 1; d >= 0; --d) {
        f.stride[d] = s;
        s *= like.extent[d];
    }
    return f;
}

size_t elem_size(int dtype)
{
    return dtype == SIL_F64 ? 8 : 4;
}

} // namespace
} // namespace sil

using namespace sil;

struct sil_laplacian_plan_s
{
    Geometry const* geo = nullptr;
    uint32_t mask = 0;
    int n = 0;
    int k = 0;
    int mode = 0;
    int kernel = 0;  // 0 generic fused, 1 2D 0-form, 2 2D 1-form TMA, 3 unfused chain
    int variant = -1;  // TMA pipeline shape picked by the autotuner (-1: not tuned yet)
    float tuned_ms = 0.f;
    sil_field in_like {};
    sil_field out_like {};
    int* error_flag = nullptr;
    int wait_tries = -1;  // kernel 2's pipeline-wait bound (-1: the default)
    void* scratch = nullptr;
    size_t scratch_bytes = 0;
    sil_field dual_a {}, dual_b {}, codiff {}, cob {};
    StoredHodges hodges {};       // kernel 4: stored general-metric stars
    void* hodge_mem = nullptr;
};

namespace {

bool same_shape(sil_field const& a, sil_field const& b)
{
    if (a.ndims != b.ndims || a.ncomp != b.ncomp || a.dtype != b.dtype || a.comp_stride != b.comp_stride) return false;
    for (int d = 0; d < a.ndims; ++d) {
        if (a.front[d] != b.front[d] || a.extent[d] != b.extent[d] || a.stride[d] != b.stride[d]) return false;
    }
    return true;
}

sil_status run_unfused(sil_laplacian_plan_s const& p, cudaStream_t s, sil_field const& in, sil_field const& out)
{
    Geometry const& g = *p.geo;
    int const n = p.n, k = p.k;
    sil_status st = SIL_OK;
    if (k < n) {
        // delta d: (1) clamped d + star into the dual buffer over the input domain,
        // (2) transposed d + star + sign over the output domain.
        st = launch_deriv_star(s, g, p.mask, k, in, p.dual_a);
        if (st == SIL_OK)
            st = launch_transpose_star(s, g, p.mask, n - k - 1, ((n * (k + 2) + 1) % 2) ? -1.0 : 1.0, p.dual_a, out);
        if (st != SIL_OK) return st;
    }
    if (k > 0) {
        // d delta: (3) star into the dual buffer, (4) transposed d + star + sign
        // into the codifferential buffer, (5) clamped d, (6) accumulate.
        st = launch_hodge(s, g, p.mask, k, in, p.dual_b);
        if (st == SIL_OK)
            st = launch_transpose_star(s, g, p.mask, n - k, ((n * (k + 1) + 1) % 2) ? -1.0 : 1.0, p.dual_b, p.codiff);
        if (st != SIL_OK) return st;
        if (k < n) {
            st = launch_coboundary(s, p.mask, k - 1, p.codiff, p.cob, false);
            if (st == SIL_OK) st = launch_add(s, out, p.cob);
        } else {
            st = launch_coboundary(s, p.mask, k - 1, p.codiff, out, false);
        }
    }
    return st;
}

} // namespace

extern "C" {

sil_status sil_deriv(sil_stream stream, uint32_t form_mask, int k, const sil_field* in, sil_field* out)
{
    int n = 0;
    sil_status st = check_pair(form_mask, k, in, out, kMaxN, k + 1, "sil_deriv", &n);
    if (st != SIL_OK) return st;
    if (k >= n) return fail(SIL_ERR_INVALID, "sil_deriv: d of a top-rank form is not defined");
    return launch_coboundary(as_stream(stream), form_mask, k, *in, *out, false);
}

sil_status sil_transposed_coboundary(sil_stream stream, uint32_t form_mask, int k, const sil_field* in,
                                     sil_field* out)
{
    int n = 0;
    sil_status st = check_pair(form_mask, k, in, out, kMaxN, k + 1, "sil_transposed_coboundary", &n);
    if (st != SIL_OK) return st;
    if (k >= n) return fail(SIL_ERR_INVALID, "sil_transposed_coboundary: rank out of range");
    return launch_coboundary(as_stream(stream), form_mask, k, *in, *out, true);
}

sil_status sil_hodge_star(sil_geometry geometry, sil_stream stream, uint32_t form_mask, int k, const sil_field* in,
                          sil_field* out)
{
    int n = 0;
    sil_status st = SIL_OK;
    if (in != nullptr && out != nullptr && form_mask != 0 && (form_mask >> in->ndims) == 0) {
        int dims[kMaxDims];
        n = form_dims(form_mask, in->ndims, dims);
    }
    st = check_pair(form_mask, k, in, out, kMaxNHodge, n - k, "sil_hodge_star", &n);
    if (st != SIL_OK) return st;
    st = check_geometry(geometry, form_mask, *out, n, "sil_hodge_star");
    if (st != SIL_OK) return st;
    for (int d = 0; d < in->ndims; ++d) {
        if (out->front[d] < in->front[d] || out->front[d] + out->extent[d] > in->front[d] + in->extent[d])
            return fail(SIL_ERR_INVALID, "sil_hodge_star: output lattice must lie inside the input lattice");
    }
    return launch_hodge(as_stream(stream), geometry->g, form_mask, k, *in, *out);
}

sil_status sil_fill_discrete_hodge_star(sil_geometry geometry, sil_stream stream, int k_in, sil_field* hodge)
{
    if (geometry == nullptr) return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star: NULL geometry");
    int const n = geometry->g.n;
    if (k_in < 0 || k_in > n) return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star: rank out of range");
    sil_status st = check_field(hodge, "hodge", static_cast<int>(ipow(n, k_in) * binom(n, n - k_in)));
    if (st != SIL_OK) return st;
    if (hodge->ndims != n) return fail(SIL_ERR_INVALID, "sil_fill_discrete_hodge_star: hodge lattice must span the form dims");
    st = check_geometry(geometry, (1u << n) - 1, *hodge, n, "sil_fill_discrete_hodge_star");
    if (st != SIL_OK) return st;
    return launch_fill_hodge(as_stream(stream), geometry->g, k_in, *hodge);
}

sil_status sil_codifferential(sil_geometry geometry, sil_stream stream, uint32_t form_mask, int k, const sil_field* in,
                              sil_field* out)
{
    int n = 0;
    sil_status st = check_pair(form_mask, k, in, out, kMaxNHodge, k - 1, "sil_codifferential", &n);
    if (st != SIL_OK) return st;
    if (k < 1) return fail(SIL_ERR_INVALID, "sil_codifferential: the codifferential of a 0-form is not defined");
    st = check_geometry(geometry, form_mask, *in, n, "sil_codifferential");
    if (st == SIL_OK) st = check_geometry(geometry, form_mask, *out, n, "sil_codifferential");
    if (st != SIL_OK) return st;
    return launch_codifferential(as_stream(stream), geometry->g, form_mask, k, *in, *out);
}

sil_status sil_laplacian_plan_create(sil_laplacian_plan* plan, sil_geometry geometry, uint32_t form_mask, int k,
                                     const sil_field* in_like, const sil_field* out_like, int mode)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_laplacian_plan_create: NULL plan");
    *plan = nullptr;
    int n = 0;
    sil_status st = check_field(in_like, "in_like", -1);
    if (st == SIL_OK) st = check_field(out_like, "out_like", -1);
    if (st != SIL_OK) return st;
    st = check_pair(form_mask, k, in_like, out_like, kMaxNHodge, k, "sil_laplacian_plan_create", &n);
    if (st != SIL_OK) return st;
    st = check_geometry(geometry, form_mask, *in_like, n, "sil_laplacian_plan_create");
    if (st == SIL_OK) st = check_geometry(geometry, form_mask, *out_like, n, "sil_laplacian_plan_create");
    if (st != SIL_OK) return st;
    if (mode != SIL_LAPLACIAN_FUSED && mode != SIL_LAPLACIAN_UNFUSED)
        return fail(SIL_ERR_INVALID, "sil_laplacian_plan_create: unknown mode");
    auto* p = new (std::nothrow) sil_laplacian_plan_s();
    if (p == nullptr) return fail(SIL_ERR_ALLOC, "sil_laplacian_plan_create: host allocation");
    p->geo = &geometry->g;
    p->mask = form_mask;
    p->n = n;
    p->k = k;
    p->mode = mode;
    p->in_like = *in_like;
    p->out_like = *out_like;
    cudaError_t err = cudaMalloc(&p->error_flag, sizeof(int));
    if (err == cudaSuccess) err = cudaMemset(p->error_flag, 0, sizeof(int));
    if (err != cudaSuccess) {
        sil_laplacian_plan_destroy(p);
        return cuda_fail(err, "sil_laplacian_plan_create");
    }
    bool const all_form = in_like->ndims == n;
    if (mode == SIL_LAPLACIAN_UNFUSED) {
        p->kernel = 3;
        size_t const es = elem_size(in_like->dtype);
        int64_t const in_nodes = node_count(*in_like), out_nodes = node_count(*out_like);
        int const na = k < n ? static_cast<int>(binom(n, n - k - 1)) : 0;
        int const nb = k > 0 ? static_cast<int>(binom(n, n - k)) : 0;
        int const nc = k > 0 ? static_cast<int>(binom(n, k - 1)) : 0;
        int const nd = (k > 0 && k < n) ? static_cast<int>(binom(n, k)) : 0;
        size_t const bytes_a = in_nodes * na * es, bytes_b = in_nodes * nb * es, bytes_c = in_nodes * nc * es,
                     bytes_d = out_nodes * nd * es;
        auto up = [](size_t b) { return (b + 255) / 256 * 256; };
        p->scratch_bytes = up(bytes_a) + up(bytes_b) + up(bytes_c) + up(bytes_d);
        if (p->scratch_bytes > 0) {
            err = cudaMalloc(&p->scratch, p->scratch_bytes);
            if (err != cudaSuccess) {
                sil_laplacian_plan_destroy(p);
                return cuda_fail(err, "sil_laplacian_plan_create: scratch");
            }
        }
        char* base = static_cast<char*>(p->scratch);
        p->dual_a = dense_like(*in_like, na, base);
        base += up(bytes_a);
        p->dual_b = dense_like(*in_like, nb, base);
        base += up(bytes_b);
        p->codiff = dense_like(*in_like, nc, base);
        base += up(bytes_c);
        p->cob = dense_like(*out_like, nd, base);
    } else if (all_form && n == 2 && k == 0 && lap2d_layout_ok(*in_like, *out_like, 1)) {
        p->kernel = 1;
    } else if (all_form && n == 2 && k == 1 && lap2d_1form_tma_ok(*in_like, *out_like)) {
        p->kernel = 2;
    } else {
        p->kernel = 0;
    }
    *plan = p;
    return SIL_OK;
}

sil_status sil_laplacian_plan_create_metric(sil_laplacian_plan* plan, sil_stream stream, int n, int k,
                                            const sil_field* position, const sil_field* metric,
                                            const sil_field* in_like, const sil_field* out_like)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_laplacian_plan_create_metric: NULL plan");
    *plan = nullptr;
    sil_status st = check_stored_laplacian(n, k, position, metric);
    if (st == SIL_OK) st = check_field(in_like, "in_like", static_cast<int>(binom(n, k)));
    if (st == SIL_OK) st = check_field(out_like, "out_like", static_cast<int>(binom(n, k)));
    if (st != SIL_OK) return st;
    if (in_like->dtype != SIL_F64 || out_like->dtype != SIL_F64)
        return fail(SIL_ERR_UNSUPPORTED, "sil_laplacian_plan_create_metric: FP64 fields only");
    if (in_like->ndims != n || out_like->ndims != n)
        return fail(SIL_ERR_INVALID, "sil_laplacian_plan_create_metric: fields must span exactly the n form dims");
    auto* p = new (std::nothrow) sil_laplacian_plan_s();
    if (p == nullptr) return fail(SIL_ERR_ALLOC, "sil_laplacian_plan_create_metric: host allocation");
    p->mask = (1u << n) - 1;
    p->n = n;
    p->k = k;
    p->mode = SIL_LAPLACIAN_FUSED;
    p->kernel = 4;
    p->in_like = *in_like;
    p->out_like = *out_like;
    cudaError_t err = cudaMalloc(&p->error_flag, sizeof(int));
    if (err == cudaSuccess) err = cudaMemset(p->error_flag, 0, sizeof(int));
    if (err != cudaSuccess) {
        sil_laplacian_plan_destroy(p);
        return cuda_fail(err, "sil_laplacian_plan_create_metric");
    }
    st = fill_stored_hodges(as_stream(stream), n, k, *position, metric, true, &p->hodge_mem, &p->hodges);
    if (st != SIL_OK) {
        sil_laplacian_plan_destroy(p);
        return st;
    }
    *plan = p;
    return SIL_OK;
}

sil_status sil_laplacian_run(sil_laplacian_plan plan, sil_stream stream, const sil_field* in, sil_field* out)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_laplacian_run: NULL plan");
    sil_status st = check_field(in, "in", -1);
    if (st == SIL_OK) st = check_field(out, "out", -1);
    if (st != SIL_OK) return st;
    if (!same_shape(*in, plan->in_like) || !same_shape(*out, plan->out_like))
        return fail(SIL_ERR_INVALID, "sil_laplacian_run: fields differ from the plan's shapes");
    cudaStream_t const s = as_stream(stream);
    switch (plan->kernel) {
    case 1: {
        if (plan->variant < 0) {
            // First run: time the block widths on these fields (synchronises the stream once).
            char const* env = std::getenv("SIMILIE_B200_AUTOTUNE");
            if (env != nullptr && env[0] == '0') {
                plan->variant = 2;
            } else {
                sil_status const st = autotune_lap2d_0form(s, *plan->geo, *in, *out, &plan->variant);
                if (st != SIL_OK) return st;
            }
        }
        return launch_lap2d_0form(s, *plan->geo, *in, *out, plan->variant);
    }
    case 2: {
        if (!lap2d_1form_tma_ok(*in, *out)) return launch_fused_laplacian(s, *plan->geo, plan->mask, plan->k, *in, *out);
        if (plan->variant < 0) {
            // First run: time the pipeline shapes on these fields and keep the
            // fastest (synchronises the stream once).
            char const* env = std::getenv("SIMILIE_B200_AUTOTUNE");
            char const* forced = std::getenv("SIMILIE_B200_LAP1_VARIANT");
            if (forced != nullptr && forced[0] >= '0' && forced[0] <= '9') {
                plan->variant = forced[0] - '0';
            } else if (env != nullptr && env[0] == '0') {
                plan->variant = 0;
            } else {
                sil_status const st = autotune_lap2d_1form(s, *plan->geo, *in, *out, plan->error_flag, &plan->variant,
                                                           &plan->tuned_ms);
                if (st != SIL_OK) return st;
            }
        }
        return launch_lap2d_1form_tma(s, *plan->geo, *in, *out, plan->error_flag, plan->variant, plan->wait_tries);
    }
    case 3: return run_unfused(*plan, s, *in, *out);
    case 4: return launch_stored_laplacian(s, plan->hodges, in, out);
    default: return launch_fused_laplacian(s, *plan->geo, plan->mask, plan->k, *in, *out);
    }
}

sil_status sil_laplacian_plan_destroy(sil_laplacian_plan plan)
{
    if (plan == nullptr) return SIL_OK;
    cudaFree(plan->error_flag);
    cudaFree(plan->scratch);
    cudaFree(plan->hodge_mem);
    delete plan;
    return SIL_OK;
}

size_t sil_laplacian_plan_scratch_bytes(sil_laplacian_plan plan)
{
    return plan == nullptr ? 0 : plan->scratch_bytes;
}

int sil_laplacian_plan_kernel(sil_laplacian_plan plan)
{
    return plan == nullptr ? -1 : plan->kernel;
}

int sil_laplacian_plan_variant(sil_laplacian_plan plan)
{
    return plan == nullptr ? -1 : plan->variant;
}

sil_status sil_laplacian_plan_set_wait_bound(sil_laplacian_plan plan, int32_t tries)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_laplacian_plan_set_wait_bound: NULL plan");
    if (tries < -1) return fail(SIL_ERR_INVALID, "sil_laplacian_plan_set_wait_bound: tries must be >= -1");
    plan->wait_tries = tries;
    return SIL_OK;
}

sil_status sil_laplacian_plan_status(sil_laplacian_plan plan)
{
    if (plan == nullptr) return fail(SIL_ERR_INVALID, "sil_laplacian_plan_status: NULL plan");
    int flag = 0;
    SIL_CUDA_CHECK(cudaMemcpy(&flag, plan->error_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag != 0) return fail(SIL_ERR_BUDGET, "a bounded wait in the Laplacian kernel ran out");
    return SIL_OK;
}

sil_status sil_laplacian(sil_geometry geometry, sil_stream stream, uint32_t form_mask, int k, const sil_field* in,
                         sil_field* out)
{
    int n = 0;
    sil_status st = check_pair(form_mask, k, in, out, kMaxNHodge, k, "sil_laplacian", &n);
    if (st != SIL_OK) return st;
    st = check_geometry(geometry, form_mask, *in, n, "sil_laplacian");
    if (st == SIL_OK) st = check_geometry(geometry, form_mask, *out, n, "sil_laplacian");
    if (st != SIL_OK) return st;
    bool const all_form = in->ndims == n;
    if (all_form && n == 2 && k == 0 && lap2d_layout_ok(*in, *out, 1))
        return launch_lap2d_0form(as_stream(stream), geometry->g, *in, *out);
    return launch_fused_laplacian(as_stream(stream), geometry->g, form_mask, k, *in, *out);
}

} // extern "C"
