// The C++ shim's SIMILIE_* environment layer: which overrides apply and
// which are refused.  No CUDA call is made (runs without a GPU).
#include <cstdio>
#include <cstdlib>

#include "sil/ddc_compat.hpp"

using namespace sil::compat;

namespace {

int failures = 0;

void expect(bool ok, char const* what)
{
    if (!ok) {
        std::printf("FAIL %s\n", what);
        ++failures;
    }
}

bool refused(char const* name, char const* value)
{
    setenv(name, value, 1);
    bool r = false;
    try {
        check_supported_environment();
    } catch (Error const& e) {
        r = e.status == SIL_ERR_UNSUPPORTED;
    }
    unsetenv(name);
    return r;
}

}  // namespace

int main()
{
    StrongFormulationSolverSettings s;
    expect(selected_preconditioner(s) == PreconditionerType::Jacobi, "default Jacobi");
    setenv("SIMILIE_DISABLE_JACOBI_PRECONDITIONER", "1", 1);
    expect(selected_preconditioner(s) == PreconditionerType::Identity, "disable Jacobi -> Identity");
    setenv("SIMILIE_PRECONDITIONER", "spd-isai", 1);
    expect(selected_preconditioner(s) == PreconditionerType::SpdIsai, "SIMILIE_PRECONDITIONER wins");
    unsetenv("SIMILIE_DISABLE_JACOBI_PRECONDITIONER");
    setenv("SIMILIE_PRECONDITIONER", "SSOR", 1);
    setenv("SIMILIE_SOR_RELAXATION_FACTOR", "1.5", 1);
    StrongFormulationSolverSettings const e = with_environment(s);
    expect(e.preconditioner == PreconditionerType::Ssor && e.sor_relaxation_factor == 1.5, "ssor and its factor");
    setenv("SIMILIE_SOR_RELAXATION_FACTOR", "abc", 1);
    expect(with_environment(s).sor_relaxation_factor == 1.2, "unparsable factor keeps the default");
    unsetenv("SIMILIE_SOR_RELAXATION_FACTOR");
    unsetenv("SIMILIE_PRECONDITIONER");
    try {
        setenv("SIMILIE_PRECONDITIONER", "no-such", 1);
        (void)with_environment(s);
        expect(false, "unknown preconditioner throws");
    } catch (std::runtime_error const&) {
    }
    unsetenv("SIMILIE_PRECONDITIONER");

    expect(!refused("SIMILIE_SOLVER", "gmres"), "gmres accepted");
    setenv("SIMILIE_SOLVER", "gmres", 1);
    setenv("SIMILIE_GMRES_KRYLOV_DIM", "30", 1);
    expect(selected_solver().kind == SIL_KRYLOV_GMRES && selected_solver().dim == 30, "gmres and its dimension");
    setenv("SIMILIE_SOLVER", "idr", 1);
    expect(selected_solver().kind == SIL_KRYLOV_IDR && selected_solver().dim == 8, "idr with the default subspace");
    setenv("SIMILIE_SOLVER", "something", 1);
    expect(selected_solver().kind == SIL_KRYLOV_CG, "an unknown name is CG, as in the reference");
    unsetenv("SIMILIE_SOLVER");
    unsetenv("SIMILIE_GMRES_KRYLOV_DIM");
    expect(refused("SIMILIE_MAGNETIC_Y_RESPONSE_SIGN_3D", "-1"), "flipped y response refused");
    expect(!refused("SIMILIE_MAGNETIC_Y_RESPONSE_SIGN_3D", "1"), "y response +1 accepted");
    expect(refused("SIMILIE_NONLINEAR_LINE_SEARCH_STEPS", "4"), "other line search refused");
    expect(!refused("SIMILIE_NONLINEAR_LINE_SEARCH_REDUCTION", "0.5"), "default reduction accepted");

    MagnetostaticsOperator3D op;
    op.x = op.y = op.z = {0.0, 0.5, 1.0};
    op.node_mu = nullptr;
    op.gauge_penalty = 20.0;
    sil_mag3d_problem p = op.problem();
    expect(p.gauge == 0 && p.gauge_penalty == 20.0, "penalty gauge by default");
    setenv("SIMILIE_DIVERGENCE_GAUGE_3D", "1", 1);
    setenv("SIMILIE_VECTOR_POTENTIAL_GAUGE_SIGN_3D", "-3", 1);
    p = op.problem();
    expect(p.gauge == 1 && p.gauge_penalty == -20.0, "divergence gauge with the sign folded in");
    setenv("SIMILIE_DIVERGENCE_GAUGE_3D", "0", 1);
    p = op.problem();
    expect(p.gauge == 0 && p.gauge_penalty == 20.0, "'0' disables, the sign applies to the divergence gauge only");
    std::printf("%s\n", failures == 0 ? "env ok" : "env failed");
    return failures == 0 ? 0 : 1;
}
