// ddc_compat.hpp -- the call shapes of SimiLie's exterior-calculus and
// solver entry points, over the sil_b200 C ABI, so that call sites written
// against the reference port line by line:
//
//   reference (src/similie/...)                           here
//   deriv<TagToAdd, CochainTag>(exec, out, in)            deriv<K>(exec, out, in)
//     exterior/coboundary.hpp:698-709
//   transposed_coboundary(exec, out, in)                  transposed_coboundary<K>(exec, out, in)
//     exterior/coboundary.hpp:661-696
//   fill_discrete_hodge_star<Idx1, Idx2>(exec, hodge,     fill_discrete_hodge_star<KIn>(exec, hodge,
//     metric, position)  exterior/hodge_star.hpp:453-494    metric, position)
//   tensor_prod(out, in, hodge) on the stored star        hodge_star_stored<KIn>(exec, out, in, hodge)
//   make_staged_codifferential(...).run(out, in),         codifferential<K>(exec, geometry, out, in)
//   codifferential(...)  exterior/codifferential.hpp:439-656
//   make_staged_codifferential(exec, tensor, metric,      make_staged_codifferential<K>(exec, in, &metric,
//     position).run(out, in)  codifferential.hpp:510-540     position).run(exec, out, in)
//   make_staged_laplacian(exec, out, in, metric,          make_staged_laplacian<K>(exec, geometry, out, in)
//     position).run(out, in)  exterior/laplacian.hpp:327-358   .run(out, in)  (rectilinear, identity metric)
//                                                         make_staged_laplacian<K>(exec, out, in, &metric,
//                                                           position).run(exec, out, in)  (general metric)
//   laplacian(...)  exterior/laplacian.hpp:814-951        laplacian<K>(exec, geometry, out, in)
//   solvers::minimize_strong_formulation_residual(        minimize_strong_formulation_residual(
//     exec, operator_model, rhs, solution, settings)        exec, operator_model, rhs, solution, settings)
//     solvers/minimize_strong_formulation_residual.hpp:1308-1570
//   assemble_matrix_data(operator_model)                  assemble_matrix_data(exec, operator_model)
//     onelab_interface/magnetostatics_onelab.hpp:3120-3748
//
// The reference's tags become the form degree K (a template argument) and
// the dimension (the field's); its DDC tensor spans become Tensor, a
// non-owning view of device memory (sil_field); the Kokkos execution space
// becomes ExecSpace, a CUDA stream.  The metric / position pair of the
// staged operators on a rectilinear grid with the identity metric becomes a
// Geometry built from the node coordinates.  As in the reference the calls
// are asynchronous on the stream (the caller fences), the solver calls are
// synchronous, and errors are thrown (Error, carrying the sil_status).
#pragma once

#include <algorithm>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../sil_b200.h"

namespace sil {
namespace compat {

class Error : public std::runtime_error
{
public:
    Error(sil_status s, std::string const& what) : std::runtime_error(what), status(s) {}
    sil_status status;
};

inline void check(sil_status s, char const* what)
{
    if (s != SIL_OK) throw Error(s, std::string(what) + ": " + sil_status_string(s) + ": " + sil_last_error());
}

// A Kokkos execution-space instance: here a CUDA stream (nullptr: the legacy default stream).
struct ExecSpace
{
    sil_stream stream = nullptr;
};

// Non-owning view of a device field in the reference's DDC layout_right
// ordering: lattice dimensions slowest to fastest, then the form component.
struct Tensor
{
    sil_field field {};

    // extents: lattice points per dimension (the last ones may be spectator
    // dimensions); ncomp: stored form components; front: absolute discrete
    // coordinate of element 0 per dimension (nullptr: all zero).
    static Tensor make(void* data, sil_dtype dtype, std::vector<int64_t> const& extents, int ncomp,
                       int64_t const* front = nullptr)
    {
        if (extents.empty() || extents.size() > SIL_MAX_DIMS) throw Error(SIL_ERR_INVALID, "Tensor: 1 to SIL_MAX_DIMS dimensions");
        Tensor t;
        t.field.data = data;
        t.field.dtype = dtype;
        t.field.ndims = static_cast<int32_t>(extents.size());
        t.field.ncomp = ncomp;
        int64_t stride = ncomp;
        for (int d = static_cast<int>(extents.size()) - 1; d >= 0; --d) {
            t.field.extent[d] = extents[d];
            t.field.stride[d] = stride;
            t.field.front[d] = front != nullptr ? front[d] : 0;
            stride *= extents[d];
        }
        t.field.comp_stride = 1;
        return t;
    }
};

// Rectilinear grid with the identity metric (the metric + position tensors
// of the staged operators): node coordinates per form dimension.
class Geometry
{
public:
    Geometry(std::vector<std::vector<double>> const& coords, std::vector<int64_t> const& front = {})
    {
        std::vector<double const*> c;
        std::vector<int64_t> n;
        for (auto const& v : coords) {
            c.push_back(v.data());
            n.push_back(static_cast<int64_t>(v.size()));
        }
        check(sil_geometry_create(&g_, static_cast<int>(coords.size()), c.data(), n.data(),
                                  front.empty() ? nullptr : front.data()),
              "Geometry");
    }
    Geometry(Geometry const&) = delete;
    Geometry& operator=(Geometry const&) = delete;
    ~Geometry() { sil_geometry_destroy(g_); }
    sil_geometry get() const { return g_; }

private:
    sil_geometry g_ = nullptr;
};

// Every dimension of the field is a form dimension.
inline uint32_t all_form_dims(Tensor const& t) { return (1u << t.field.ndims) - 1u; }

// ------------------------------------------------------------------ exterior calculus

template <int K>
Tensor deriv(ExecSpace exec, Tensor out, Tensor in, uint32_t form_mask = 0)
{
    check(sil_deriv(exec.stream, form_mask ? form_mask : all_form_dims(in), K, &in.field, &out.field), "deriv");
    return out;
}

template <int K>
Tensor transposed_coboundary(ExecSpace exec, Tensor out, Tensor in, uint32_t form_mask = 0)
{
    check(sil_transposed_coboundary(exec.stream, form_mask ? form_mask : all_form_dims(in), K, &in.field,
                                    &out.field),
          "transposed_coboundary");
    return out;
}

template <int K>
Tensor hodge_star(ExecSpace exec, Geometry const& geometry, Tensor out, Tensor in, uint32_t form_mask = 0)
{
    check(sil_hodge_star(geometry.get(), exec.stream, form_mask ? form_mask : all_form_dims(in), K, &in.field,
                         &out.field),
          "hodge_star");
    return out;
}

// General per-node metric (metric == nullptr: identity), n form dimensions.
template <int KIn>
Tensor fill_discrete_hodge_star(ExecSpace exec, Tensor hodge, Tensor const* metric, Tensor position, int n)
{
    check(sil_fill_discrete_hodge_star_metric(exec.stream, n, KIn, &position.field,
                                              metric != nullptr ? &metric->field : nullptr, &hodge.field),
          "fill_discrete_hodge_star");
    return hodge;
}

template <int KIn>
Tensor hodge_star_stored(ExecSpace exec, Tensor out, Tensor in, Tensor hodge, int n)
{
    check(sil_hodge_star_stored(exec.stream, n, KIn, &hodge.field, &in.field, &out.field), "hodge_star_stored");
    return out;
}

template <int K>
Tensor codifferential(ExecSpace exec, Geometry const& geometry, Tensor out, Tensor in, uint32_t form_mask = 0)
{
    check(sil_codifferential(geometry.get(), exec.stream, form_mask ? form_mask : all_form_dims(in), K, &in.field,
                             &out.field),
          "codifferential");
    return out;
}

template <int K>
Tensor laplacian(ExecSpace exec, Geometry const& geometry, Tensor out, Tensor in, uint32_t form_mask = 0)
{
    check(sil_laplacian(geometry.get(), exec.stream, form_mask ? form_mask : all_form_dims(in), K, &in.field,
                        &out.field),
          "laplacian");
    return out;
}

// StagedLaplacian: built once for fields shaped like (out, in), run many times.
template <int K>
class StagedLaplacian
{
public:
    StagedLaplacian(Geometry const& geometry, Tensor out_like, Tensor in_like, bool fused, uint32_t form_mask)
    {
        check(sil_laplacian_plan_create(&plan_, geometry.get(), form_mask ? form_mask : all_form_dims(in_like), K,
                                        &in_like.field, &out_like.field,
                                        fused ? SIL_LAPLACIAN_FUSED : SIL_LAPLACIAN_UNFUSED),
              "make_staged_laplacian");
    }
    StagedLaplacian(StagedLaplacian&& o) noexcept : plan_(std::exchange(o.plan_, nullptr)) {}
    StagedLaplacian(StagedLaplacian const&) = delete;
    ~StagedLaplacian()
    {
        if (plan_ != nullptr) sil_laplacian_plan_destroy(plan_);
    }
    Tensor run(ExecSpace exec, Tensor out, Tensor in) const
    {
        check(sil_laplacian_run(plan_, exec.stream, &in.field, &out.field), "StagedLaplacian::run");
        return out;
    }

private:
    sil_laplacian_plan plan_ = nullptr;
};

template <int K>
StagedLaplacian<K> make_staged_laplacian(ExecSpace, Geometry const& geometry, Tensor out, Tensor in,
                                         bool fused = true, uint32_t form_mask = 0)
{
    return StagedLaplacian<K>(geometry, out, in, fused, form_mask);
}

// The general-metric staged operators: built from the (metric, position)
// tensor pair as in the reference (metric == nullptr: identity), they store
// the per-node Hodge tensors fill_discrete_hodge_star computes and run one
// fused kernel per call.  FP64, fields over exactly the position's n dims.
template <int K>
class MetricStagedLaplacian
{
public:
    MetricStagedLaplacian(ExecSpace exec, Tensor out_like, Tensor in_like, Tensor const* metric, Tensor position)
    {
        check(sil_laplacian_plan_create_metric(&plan_, exec.stream, position.field.ndims, K, &position.field,
                                               metric != nullptr ? &metric->field : nullptr, &in_like.field,
                                               &out_like.field),
              "make_staged_laplacian");
    }
    MetricStagedLaplacian(MetricStagedLaplacian&& o) noexcept : plan_(std::exchange(o.plan_, nullptr)) {}
    MetricStagedLaplacian(MetricStagedLaplacian const&) = delete;
    ~MetricStagedLaplacian()
    {
        if (plan_ != nullptr) sil_laplacian_plan_destroy(plan_);
    }
    Tensor run(ExecSpace exec, Tensor out, Tensor in) const
    {
        check(sil_laplacian_run(plan_, exec.stream, &in.field, &out.field), "StagedLaplacian::run");
        return out;
    }

private:
    sil_laplacian_plan plan_ = nullptr;
};

template <int K>
MetricStagedLaplacian<K> make_staged_laplacian(ExecSpace exec, Tensor out, Tensor in, Tensor const* metric,
                                               Tensor position)
{
    return MetricStagedLaplacian<K>(exec, out, in, metric, position);
}

template <int K>
class MetricStagedCodifferential
{
public:
    MetricStagedCodifferential(ExecSpace exec, Tensor const* metric, Tensor position)
    {
        check(sil_codifferential_plan_create(&plan_, exec.stream, position.field.ndims, K, &position.field,
                                             metric != nullptr ? &metric->field : nullptr),
              "make_staged_codifferential");
    }
    MetricStagedCodifferential(MetricStagedCodifferential&& o) noexcept : plan_(std::exchange(o.plan_, nullptr)) {}
    MetricStagedCodifferential(MetricStagedCodifferential const&) = delete;
    ~MetricStagedCodifferential()
    {
        if (plan_ != nullptr) sil_codifferential_plan_destroy(plan_);
    }
    Tensor run(ExecSpace exec, Tensor out, Tensor in) const
    {
        check(sil_codifferential_run(plan_, exec.stream, &in.field, &out.field), "StagedCodifferential::run");
        return out;
    }

private:
    sil_codifferential_plan plan_ = nullptr;
};

// `tensor` is the input the reference sizes its dual buffer from; the fused
// kernel needs no buffer, so only its rank (K) matters here.
template <int K>
MetricStagedCodifferential<K> make_staged_codifferential(ExecSpace exec, Tensor /*tensor*/, Tensor const* metric,
                                                         Tensor position)
{
    return MetricStagedCodifferential<K>(exec, metric, position);
}

// ------------------------------------------------------------------ solvers

// solvers/minimize_strong_formulation_residual.hpp:53-63: the preconditioner
// menu, in the reference's order and with its spellings.
enum class PreconditionerType
{
    Identity,
    Jacobi,
    SpdIsai,
    SymmetricGaussSeidel,
    Ssor,
    ChebyshevJacobi,
    IrJacobi,
    GeneralIsai,
};

inline PreconditionerType parse_preconditioner(std::string const& name)
{
    struct Entry
    {
        char const* name;
        PreconditionerType type;
    };
    static Entry const table[] = {
            {"Identity", PreconditionerType::Identity},
            {"identity", PreconditionerType::Identity},
            {"Jacobi", PreconditionerType::Jacobi},
            {"jacobi", PreconditionerType::Jacobi},
            {"SpdIsai", PreconditionerType::SpdIsai},
            {"spd-isai", PreconditionerType::SpdIsai},
            {"spd_isai", PreconditionerType::SpdIsai},
            {"SymmetricGaussSeidel", PreconditionerType::SymmetricGaussSeidel},
            {"symmetric-gauss-seidel", PreconditionerType::SymmetricGaussSeidel},
            {"symmetric_gauss_seidel", PreconditionerType::SymmetricGaussSeidel},
            {"Ssor", PreconditionerType::Ssor},
            {"SSOR", PreconditionerType::Ssor},
            {"ssor", PreconditionerType::Ssor},
            {"ChebyshevJacobi", PreconditionerType::ChebyshevJacobi},
            {"chebyshev-jacobi", PreconditionerType::ChebyshevJacobi},
            {"chebyshev_jacobi", PreconditionerType::ChebyshevJacobi},
            {"IrJacobi", PreconditionerType::IrJacobi},
            {"ir-jacobi", PreconditionerType::IrJacobi},
            {"ir_jacobi", PreconditionerType::IrJacobi},
            {"GeneralIsai", PreconditionerType::GeneralIsai},
            {"general-isai", PreconditionerType::GeneralIsai},
            {"general_isai", PreconditionerType::GeneralIsai},
            {"isai", PreconditionerType::GeneralIsai},
    };
    for (Entry const& e : table)
        if (name == e.name) return e.type;
    throw std::runtime_error("unknown strong-formulation preconditioner: " + name);
}

// solvers/minimize_strong_formulation_residual.hpp:61-75: the settings this
// path reads, with the reference's defaults for the menu.
struct StrongFormulationSolverSettings
{
    double relative_tolerance = 1e-10;
    unsigned int max_iterations = 100000;
    // matrix-free Jacobi-CG in FP64 (the reference's default), or FP32 inner
    // CG with FP64 refinement; linear matrix-free solves only.
    bool mixed_precision = false;
    // false, or any preconditioner but Jacobi: the linear solve assembles
    // the operator (sil_mag2d/3d_assemble), a nonlinear solve its Jacobian
    // at every Newton step, and CG runs with the chosen preconditioner.
    bool use_matrix_free = true;
    PreconditionerType preconditioner = PreconditionerType::Jacobi;
    double sor_relaxation_factor = 1.2;
    unsigned int chebyshev_iterations = 8;
    double chebyshev_lower_bound = 0.05;
    double chebyshev_upper_bound = 1.5;
    unsigned int ir_iterations = 8;
    double ir_relaxation_factor = 1.0;
};

// The reference's SIMILIE_* environment overrides
// (solvers/minimize_strong_formulation_residual.hpp:148-218, 932-942,
// 1069-1130, 1510-1515; onelab_interface/magnetostatics_onelab.hpp:796-828).
// Those whose meaning this library implements are applied; those it does not
// (another Krylov solver, a flipped y response, another line search) raise
// SIL_ERR_UNSUPPORTED instead of being ignored.
namespace env {

// set, non-empty and not starting with '0'
inline bool flag(char const* name)
{
    char const* const v = std::getenv(name);
    return v != nullptr && v[0] != '\0' && v[0] != '0';
}

// the value as a number, or `fallback` when unset, empty or not a number
inline double number_or(char const* name, double fallback)
{
    char const* const v = std::getenv(name);
    if (v == nullptr || v[0] == '\0') return fallback;
    char* end = nullptr;
    double const x = std::strtod(v, &end);
    return end == v ? fallback : x;
}

// -1 for a negative number, else 1 (unset, empty, zero or not a number)
inline double sign_or_one(char const* name)
{
    double const x = number_or(name, 0.0);
    return x < 0.0 ? -1.0 : 1.0;
}

}  // namespace env

// SIMILIE_PRECONDITIONER first, then SIMILIE_DISABLE_JACOBI_PRECONDITIONER
// (Identity), else the settings' choice (selected_preconditioner, 932-942).
inline PreconditionerType selected_preconditioner(StrongFormulationSolverSettings const& settings)
{
    char const* const v = std::getenv("SIMILIE_PRECONDITIONER");
    if (v != nullptr && v[0] != '\0') return parse_preconditioner(v);
    if (env::flag("SIMILIE_DISABLE_JACOBI_PRECONDITIONER")) return PreconditionerType::Identity;
    return settings.preconditioner;
}

// SIMILIE_SOLVER: minres, fcg, gmres, bicgstab, gcr or idr; anything else is
// CG (solve_linearized_system, 1069-1130), with the Krylov dimensions of
// SIMILIE_GMRES_KRYLOV_DIM (100), SIMILIE_GCR_KRYLOV_DIM (100) and
// SIMILIE_IDR_SUBSPACE_DIM (8).
struct KrylovChoice
{
    sil_krylov_kind kind = SIL_KRYLOV_CG;
    int dim = 0;
};

inline KrylovChoice selected_solver()
{
    KrylovChoice c;
    char const* const v = std::getenv("SIMILIE_SOLVER");
    std::string const name = v == nullptr ? "" : v;
    if (name == "minres") c.kind = SIL_KRYLOV_MINRES;
    else if (name == "fcg") c.kind = SIL_KRYLOV_FCG;
    else if (name == "gmres") {
        c.kind = SIL_KRYLOV_GMRES;
        c.dim = static_cast<int>(env::number_or("SIMILIE_GMRES_KRYLOV_DIM", 100.0));
    } else if (name == "bicgstab") c.kind = SIL_KRYLOV_BICGSTAB;
    else if (name == "gcr") {
        c.kind = SIL_KRYLOV_GCR;
        c.dim = std::max(1, static_cast<int>(env::number_or("SIMILIE_GCR_KRYLOV_DIM", 100.0)));
    } else if (name == "idr") {
        c.kind = SIL_KRYLOV_IDR;
        c.dim = std::max(1, static_cast<int>(env::number_or("SIMILIE_IDR_SUBSPACE_DIM", 8.0)));
    }
    if (c.dim < 1 && (c.kind == SIL_KRYLOV_GMRES)) c.dim = 1;
    return c;
}

inline void check_supported_environment()
{
    if (env::sign_or_one("SIMILIE_MAGNETIC_Y_RESPONSE_SIGN_3D") < 0.0)
        throw Error(SIL_ERR_UNSUPPORTED, "SIMILIE_MAGNETIC_Y_RESPONSE_SIGN_3D < 0 is not available");
    if (env::number_or("SIMILIE_NONLINEAR_LINE_SEARCH_STEPS", 8.0) != 8.0
        || env::number_or("SIMILIE_NONLINEAR_LINE_SEARCH_REDUCTION", 0.5) != 0.5)
        throw Error(SIL_ERR_UNSUPPORTED, "the line search is fixed at 8 halving steps");
}

// The settings a solve uses: the environment's preconditioner and SOR
// relaxation factor over the caller's.
inline StrongFormulationSolverSettings with_environment(StrongFormulationSolverSettings settings)
{
    check_supported_environment();
    settings.preconditioner = selected_preconditioner(settings);
    settings.sor_relaxation_factor = env::number_or("SIMILIE_SOR_RELAXATION_FACTOR", settings.sor_relaxation_factor);
    return settings;
}

// The solver's stages: an NVTX range around the whole solve (seen by
// profilers, free otherwise) and, with SIMILIE_SOLVER_TIMING, one line per
// stage on stdout.
class StageTimer
{
public:
    StageTimer() : on_(env::flag("SIMILIE_SOLVER_TIMING")), t0_(std::chrono::steady_clock::now())
    {
        nvtxRangePushA("minimize_strong_formulation_residual");
    }
    ~StageTimer() { nvtxRangePop(); }
    StageTimer(StageTimer const&) = delete;
    StageTimer& operator=(StageTimer const&) = delete;
    void done(char const* stage)
    {
        auto const t1 = std::chrono::steady_clock::now();
        if (on_)
            std::printf("SimiLie solver stage: %s duration=%.6f\n", stage,
                        std::chrono::duration<double>(t1 - t0_).count());
        nvtxMarkA(stage);
        t0_ = t1;
    }

private:
    bool on_;
    std::chrono::steady_clock::time_point t0_;
};

struct StrongFormulationSolverDiagnostics
{
    unsigned int iterations = 0;
    bool converged = false;
    double initial_residual_l2 = 0.0;
    double final_residual_l2 = 0.0;
    double final_relative_residual = 0.0;
    unsigned int nonlinear_iterations = 0;  // Newton steps (nonlinear operators)
};

// The OperatorModel concept of the reference (IS_LINEAR, size(), apply,
// apply_jacobian) for the magnetostatics operators; device FP64 arrays.
// magnetostatics_onelab.hpp:1013-1426 (2D), 1625-2700 (3D), 957-1011 and 2799-2915 (nonlinear material).
struct MagnetostaticsOperator2D
{
    static constexpr bool IS_LINEAR = true;
    int64_t nx, ny;
    double const* node_mu;
    int64_t size() const { return nx * ny; }
    void apply(ExecSpace exec, double const* in, double* out) const
    {
        check(sil_mag2d_apply(exec.stream, nx, ny, node_mu, in, out), "MagnetostaticsOperator2D::apply");
    }
};

struct MagnetostaticsOperator3D
{
    static constexpr bool IS_LINEAR = true;
    std::vector<double> x, y, z;  // node coordinates (host)
    double const* node_mu;
    double gauge_penalty = 20.0;
    bool divergence_gauge = false;  // SIMILIE_DIVERGENCE_GAUGE_3D
    int64_t size() const { return 3 * static_cast<int64_t>(x.size() * y.size() * z.size()); }
    sil_mag3d_problem problem(double const* rhs = nullptr, double* solution = nullptr) const
    {
        sil_mag3d_problem p {};
        p.nx = static_cast<int64_t>(x.size());
        p.ny = static_cast<int64_t>(y.size());
        p.nz = static_cast<int64_t>(z.size());
        p.x = x.data();
        p.y = y.data();
        p.z = z.data();
        p.node_mu = node_mu;
        p.rhs = rhs;
        p.solution = solution;
        // SIMILIE_DIVERGENCE_GAUGE_3D selects the divergence gauge, whose
        // factor takes the sign SIMILIE_VECTOR_POTENTIAL_GAUGE_SIGN_3D
        bool const divergence = divergence_gauge || env::flag("SIMILIE_DIVERGENCE_GAUGE_3D");
        p.gauge = divergence ? 1 : 0;
        p.gauge_penalty = divergence ? gauge_penalty * env::sign_or_one("SIMILIE_VECTOR_POTENTIAL_GAUGE_SIGN_3D")
                                     : gauge_penalty;
        return p;
    }
    void apply(ExecSpace exec, double const* in, double* out) const
    {
        sil_mag3d_problem const p = problem();
        check(sil_mag3d_apply(exec.stream, &p, in, out), "MagnetostaticsOperator3D::apply");
    }
};

struct NonlinearMagnetostaticsOperator2D
{
    static constexpr bool IS_LINEAR = false;
    int64_t nx, ny;
    double const* node_mu;
    double const* node_ferro;
    std::vector<double> curve_b, curve_h;  // B-H samples (host)
    int64_t size() const { return nx * ny; }
    sil_mag2d_nl_problem problem(double const* rhs = nullptr, double* solution = nullptr) const
    {
        sil_mag2d_nl_problem p {};
        p.nx = nx;
        p.ny = ny;
        p.node_mu = node_mu;
        p.node_ferro = node_ferro;
        p.curve.n = static_cast<int32_t>(curve_b.size());
        p.curve.b = curve_b.data();
        p.curve.h = curve_h.data();
        p.rhs = rhs;
        p.solution = solution;
        return p;
    }
    void apply(ExecSpace exec, double const* in, double* out) const
    {
        sil_mag2d_nl_problem const p = problem();
        check(sil_mag2d_nl_apply(exec.stream, &p, in, out), "NonlinearMagnetostaticsOperator2D::apply");
    }
    void apply_jacobian(ExecSpace exec, double const* state, double const* in, double* out) const
    {
        sil_mag2d_nl_problem const p = problem();
        check(sil_mag2d_nl_apply_jacobian(exec.stream, &p, state, in, out), "apply_jacobian");
    }
};

struct NonlinearMagnetostaticsOperator3D
{
    static constexpr bool IS_LINEAR = false;
    std::vector<double> x, y, z;  // node coordinates (host)
    double const* node_mu;
    double const* node_ferro;
    std::vector<double> curve_b, curve_h;  // B-H samples (host)
    double gauge_penalty = 20.0;
    bool divergence_gauge = false;  // SIMILIE_DIVERGENCE_GAUGE_3D
    int64_t size() const { return 3 * static_cast<int64_t>(x.size() * y.size() * z.size()); }
    sil_mag3d_nl_problem problem(double const* rhs = nullptr, double* solution = nullptr) const
    {
        sil_mag3d_nl_problem p {};
        p.nx = static_cast<int64_t>(x.size());
        p.ny = static_cast<int64_t>(y.size());
        p.nz = static_cast<int64_t>(z.size());
        p.x = x.data();
        p.y = y.data();
        p.z = z.data();
        p.node_mu = node_mu;
        p.node_ferro = node_ferro;
        p.curve.n = static_cast<int32_t>(curve_b.size());
        p.curve.b = curve_b.data();
        p.curve.h = curve_h.data();
        p.rhs = rhs;
        p.solution = solution;
        bool const divergence = divergence_gauge || env::flag("SIMILIE_DIVERGENCE_GAUGE_3D");
        p.gauge = divergence ? 1 : 0;
        p.gauge_penalty = divergence ? gauge_penalty * env::sign_or_one("SIMILIE_VECTOR_POTENTIAL_GAUGE_SIGN_3D")
                                     : gauge_penalty;
        return p;
    }
    void apply(ExecSpace exec, double const* in, double* out) const
    {
        sil_mag3d_nl_problem const p = problem();
        check(sil_mag3d_nl_apply(exec.stream, &p, in, out), "NonlinearMagnetostaticsOperator3D::apply");
    }
    void apply_jacobian(ExecSpace exec, double const* state, double const* in, double* out) const
    {
        sil_mag3d_nl_problem const p = problem();
        check(sil_mag3d_nl_apply_jacobian(exec.stream, &p, state, in, out), "apply_jacobian");
    }
};

// An assembled operator (the reference's assemble_matrix_data read into a
// Csr<double, int32>); owns the library's matrix.
class CsrMatrix
{
public:
    explicit CsrMatrix(sil_csr m) : m_(m) {}
    CsrMatrix(CsrMatrix&& o) noexcept : m_(o.m_) { o.m_ = nullptr; }
    CsrMatrix& operator=(CsrMatrix&& o) noexcept
    {
        std::swap(m_, o.m_);
        return *this;
    }
    CsrMatrix(CsrMatrix const&) = delete;
    CsrMatrix& operator=(CsrMatrix const&) = delete;
    ~CsrMatrix() { sil_csr_destroy(m_); }
    sil_csr get() const { return m_; }
    int64_t rows() const
    {
        int64_t n = 0;
        check(sil_csr_get(m_, &n, nullptr, nullptr, nullptr, nullptr), "CsrMatrix::rows");
        return n;
    }
    int64_t nonzeros() const
    {
        int64_t nnz = 0;
        check(sil_csr_get(m_, nullptr, &nnz, nullptr, nullptr, nullptr), "CsrMatrix::nonzeros");
        return nnz;
    }
    void apply(ExecSpace exec, double const* in, double* out) const
    {
        check(sil_csr_spmv(exec.stream, m_, in, out), "CsrMatrix::apply");
    }

private:
    sil_csr m_ = nullptr;
};

inline CsrMatrix assemble_matrix_data(ExecSpace exec, MagnetostaticsOperator2D const& op)
{
    sil_csr m = nullptr;
    check(sil_mag2d_assemble(exec.stream, op.nx, op.ny, op.node_mu, &m), "assemble_matrix_data");
    return CsrMatrix(m);
}

inline CsrMatrix assemble_matrix_data(ExecSpace exec, MagnetostaticsOperator3D const& op)
{
    sil_mag3d_problem const p = op.problem();
    sil_csr m = nullptr;
    check(sil_mag3d_assemble(exec.stream, &p, &m), "assemble_matrix_data");
    return CsrMatrix(m);
}

namespace detail {

inline sil_solve_settings to_settings(StrongFormulationSolverSettings const& s)
{
    sil_solve_settings r {};
    r.solver = s.mixed_precision ? SIL_SOLVER_MIXED_IR : SIL_SOLVER_CG_F64;
    r.max_iterations = static_cast<int32_t>(s.max_iterations);
    r.relative_tolerance = s.relative_tolerance;
    return r;
}

inline StrongFormulationSolverDiagnostics to_diagnostics(sil_solve_diagnostics const& d, bool nonlinear)
{
    StrongFormulationSolverDiagnostics r;
    r.iterations = static_cast<unsigned int>(d.iterations);
    r.converged = d.converged != 0;
    r.initial_residual_l2 = d.initial_residual_l2;
    r.final_residual_l2 = d.final_residual_l2;
    r.final_relative_residual = d.final_relative_residual;
    r.nonlinear_iterations = nonlinear ? static_cast<unsigned int>(d.refinements) : 0u;
    return r;
}

inline bool assembled(StrongFormulationSolverSettings const& s)
{
    return !s.use_matrix_free || s.preconditioner != PreconditionerType::Jacobi
           || selected_solver().kind != SIL_KRYLOV_CG;
}

inline sil_menu_settings to_menu(StrongFormulationSolverSettings const& settings)
{
    sil_menu_settings cfg {};
    cfg.kind = static_cast<int32_t>(settings.preconditioner);
    cfg.sor_relaxation_factor = settings.sor_relaxation_factor;
    cfg.chebyshev_iterations = static_cast<int32_t>(settings.chebyshev_iterations);
    cfg.chebyshev_lower_bound = settings.chebyshev_lower_bound;
    cfg.chebyshev_upper_bound = settings.chebyshev_upper_bound;
    cfg.ir_iterations = static_cast<int32_t>(settings.ir_iterations);
    cfg.ir_relaxation_factor = settings.ir_relaxation_factor;
    return cfg;
}

// CG with the chosen preconditioner on the assembled matrix
// (solve_linearized_system with an assembled system matrix).
inline StrongFormulationSolverDiagnostics solve_assembled(ExecSpace exec, CsrMatrix const& m, double const* rhs,
                                                          double* solution,
                                                          StrongFormulationSolverSettings const& settings,
                                                          StageTimer& timer)
{
    sil_menu_settings const cfg = to_menu(settings);
    sil_csr_precond pc = nullptr;
    check(sil_csr_precond_create(exec.stream, m.get(), &cfg, &pc), "build_preconditioner");
    timer.done("preconditioner build");
    sil_solve_settings const s = to_settings(settings);
    sil_solve_diagnostics d {};
    KrylovChoice const k = selected_solver();
    sil_status const st = sil_csr_krylov_solve(exec.stream, m.get(), pc, k.kind, k.dim, rhs, solution, &s, &d);
    sil_csr_precond_destroy(pc);
    check(st, "minimize_strong_formulation_residual");
    timer.done("solve");
    return to_diagnostics(d, false);
}

template <class Operator>
StrongFormulationSolverDiagnostics assemble_and_solve(ExecSpace exec, Operator const& op, double const* rhs,
                                                      double* solution,
                                                      StrongFormulationSolverSettings const& settings)
{
    StageTimer timer;
    CsrMatrix const m = assemble_matrix_data(exec, op);
    timer.done("matrix build");
    return solve_assembled(exec, m, rhs, solution, settings, timer);
}

}  // namespace detail

// The linear solves start from x = 0 (as the reference's); the nonlinear
// one from the content of `solution`.  Synchronous.
inline StrongFormulationSolverDiagnostics minimize_strong_formulation_residual(
        ExecSpace exec, MagnetostaticsOperator2D const& op, double const* rhs, double* solution,
        StrongFormulationSolverSettings const& requested)
{
    StrongFormulationSolverSettings const settings = with_environment(requested);
    if (detail::assembled(settings)) return detail::assemble_and_solve(exec, op, rhs, solution, settings);
    StageTimer timer;
    sil_mag2d_problem p {op.nx, op.ny, op.node_mu, rhs, solution};
    sil_solve_settings const s = detail::to_settings(settings);
    sil_solve_diagnostics d {};
    check(sil_mag2d_solve_batch(&p, 1, &s, &d, exec.stream), "minimize_strong_formulation_residual");
    timer.done("solve");
    return detail::to_diagnostics(d, false);
}

inline StrongFormulationSolverDiagnostics minimize_strong_formulation_residual(
        ExecSpace exec, MagnetostaticsOperator3D const& op, double const* rhs, double* solution,
        StrongFormulationSolverSettings const& requested)
{
    StrongFormulationSolverSettings const settings = with_environment(requested);
    if (detail::assembled(settings)) return detail::assemble_and_solve(exec, op, rhs, solution, settings);
    StageTimer timer;
    sil_mag3d_problem const p = op.problem(rhs, solution);
    sil_solve_settings const s = detail::to_settings(settings);
    sil_solve_diagnostics d {};
    check(sil_mag3d_solve_batch(&p, 1, &s, &d, exec.stream), "minimize_strong_formulation_residual");
    timer.done("solve");
    return detail::to_diagnostics(d, false);
}

inline StrongFormulationSolverDiagnostics minimize_strong_formulation_residual(
        ExecSpace exec, NonlinearMagnetostaticsOperator2D const& op, double const* rhs, double* solution,
        StrongFormulationSolverSettings const& requested)
{
    StrongFormulationSolverSettings const settings = with_environment(requested);
    StageTimer timer;
    sil_mag2d_nl_problem const p = op.problem(rhs, solution);
    sil_solve_settings s = detail::to_settings(settings);
    sil_menu_settings const menu = detail::to_menu(settings);
    if (detail::assembled(settings)) s.jacobian_preconditioner = &menu;
    sil_solve_diagnostics d {};
    check(sil_mag2d_nl_solve_batch(&p, 1, &s, &d, exec.stream), "minimize_strong_formulation_residual");
    timer.done("nonlinear solve");
    return detail::to_diagnostics(d, true);
}

inline StrongFormulationSolverDiagnostics minimize_strong_formulation_residual(
        ExecSpace exec, NonlinearMagnetostaticsOperator3D const& op, double const* rhs, double* solution,
        StrongFormulationSolverSettings const& requested)
{
    StrongFormulationSolverSettings const settings = with_environment(requested);
    StageTimer timer;
    sil_mag3d_nl_problem const p = op.problem(rhs, solution);
    sil_solve_settings s = detail::to_settings(settings);
    sil_menu_settings const menu = detail::to_menu(settings);
    if (detail::assembled(settings)) s.jacobian_preconditioner = &menu;
    sil_solve_diagnostics d {};
    check(sil_mag3d_nl_solve_batch(&p, 1, &s, &d, exec.stream), "minimize_strong_formulation_residual");
    timer.done("nonlinear solve");
    return detail::to_diagnostics(d, true);
}

}  // namespace compat
}  // namespace sil
