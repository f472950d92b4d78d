// A reference-style call site compiled against include/sil/ddc_compat.hpp:
// d of a 0-form, the staged Laplacian of that 0-form, and a 2D
// magnetostatics solve through minimize_strong_formulation_residual.
// Writes its outputs as raw little-endian doubles into the directory given
// as the first argument; tests/test_cpp_shim.py checks them against the
// oracle.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "sil/ddc_compat.hpp"

using namespace sil::compat;

namespace {

double* to_device(std::vector<double> const& h)
{
    double* d = nullptr;
    cudaMalloc(&d, h.size() * sizeof(double));
    cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice);
    return d;
}

std::vector<double> to_host(double const* d, size_t n)
{
    std::vector<double> h(n);
    cudaMemcpy(h.data(), d, n * sizeof(double), cudaMemcpyDeviceToHost);
    return h;
}

void write(std::string const& path, std::vector<double> const& v)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(v.data(), sizeof(double), v.size(), f);
    std::fclose(f);
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    std::string const dir = argv[1];
    ExecSpace const exec {};
    try {
        // d and the Laplacian of a 0-form on a 12 x 9 lattice (x slowest)
        int const nx = 12, ny = 9;
        std::vector<double> phi(nx * ny), xs(nx), ys(ny);
        for (int i = 0; i < nx; ++i) xs[i] = 0.1 * i + 0.002 * i * i;
        for (int j = 0; j < ny; ++j) ys[j] = 0.15 * j;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) phi[i * ny + j] = std::sin(0.3 * i) * std::cos(0.2 * j) + 0.01 * i * j;
        double* d_phi = to_device(phi);
        double* d_dphi = to_device(std::vector<double>(nx * ny * 2, 0.0));
        double* d_lap = to_device(std::vector<double>((nx - 1) * (ny - 1), 0.0));
        Tensor const in = Tensor::make(d_phi, SIL_F64, {nx, ny}, 1);
        Tensor const dout = Tensor::make(d_dphi, SIL_F64, {nx, ny}, 2);
        Tensor const lout = Tensor::make(d_lap, SIL_F64, {nx - 1, ny - 1}, 1);
        deriv<0>(exec, dout, in);
        Geometry const geometry({xs, ys});
        auto const staged = make_staged_laplacian<0>(exec, geometry, lout, in);
        staged.run(exec, lout, in);

        // 2D magnetostatics, 33 x 33 nodes: a permeability-1000 block and a source block
        int const n = 33;
        std::vector<double> mu(n * n, 1.0), rhs(n * n, 0.0);
        for (int j = 10; j < 20; ++j)
            for (int i = 12; i < 24; ++i) mu[i + n * j] = 1000.0;
        for (int j = 5; j < 9; ++j)
            for (int i = 4; i < 9; ++i) rhs[i + n * j] = 1e-3;
        double* d_mu = to_device(mu);
        double* d_rhs = to_device(rhs);
        double* d_sol = to_device(std::vector<double>(n * n, 0.0));
        MagnetostaticsOperator2D const op {n, n, d_mu};
        StrongFormulationSolverSettings settings;
        settings.relative_tolerance = 1e-10;
        StrongFormulationSolverDiagnostics const diag =
                minimize_strong_formulation_residual(exec, op, d_rhs, d_sol, settings);
        cudaDeviceSynchronize();

        write(dir + "/phi.bin", phi);
        write(dir + "/dphi.bin", to_host(d_dphi, nx * ny * 2));
        write(dir + "/lap.bin", to_host(d_lap, (nx - 1) * (ny - 1)));
        write(dir + "/mu.bin", mu);
        write(dir + "/rhs.bin", rhs);
        write(dir + "/sol.bin", to_host(d_sol, n * n));
        std::printf("%u %d %.6e\n", diag.iterations, diag.converged ? 1 : 0, diag.final_relative_residual);

        // errors surface as exceptions carrying the status, as in the reference
        try {
            deriv<3>(exec, dout, in);
            std::printf("no-error\n");
        } catch (Error const& e) {
            std::printf("error %d\n", static_cast<int>(e.status));
        }

        // the same solve on the assembled matrix with the reference's SSOR
        // (SIMILIE_PRECONDITIONER=ssor, use_matrix_free = false)
        StrongFormulationSolverSettings assembled;
        assembled.relative_tolerance = 1e-10;
        assembled.use_matrix_free = false;
        assembled.preconditioner = parse_preconditioner("ssor");
        double* d_sol2 = to_device(std::vector<double>(n * n, 0.0));
        StrongFormulationSolverDiagnostics const diag2 =
                minimize_strong_formulation_residual(exec, op, d_rhs, d_sol2, assembled);
        CsrMatrix const matrix = assemble_matrix_data(exec, op);
        cudaDeviceSynchronize();
        write(dir + "/sol_ssor.bin", to_host(d_sol2, n * n));
        std::printf("assembled %u %d %.6e %lld\n", diag2.iterations, diag2.converged ? 1 : 0,
                    diag2.final_relative_residual, static_cast<long long>(matrix.nonzeros()));

        // the general-metric staged Laplacian of a 1-form on a sheared 10 x 8
        // lattice with a dense metric per node (make_staged_laplacian(exec,
        // out, in, metric, position)), and its codifferential
        int const mx = 10, my = 8;
        std::vector<double> pos(mx * my * 2), met(mx * my * 4), w1(mx * my * 2);
        for (int i = 0; i < mx; ++i)
            for (int j = 0; j < my; ++j) {
                int const node = i * my + j;
                pos[2 * node] = 0.2 * i + 0.05 * j;
                pos[2 * node + 1] = 0.25 * j + 0.01 * i * i;
                double const a = 0.3 * std::sin(0.7 * i + 0.3 * j), b = 0.2 * std::cos(0.4 * i - 0.5 * j);
                met[4 * node] = 1.0 + a * a;
                met[4 * node + 1] = met[4 * node + 2] = a * b;
                met[4 * node + 3] = 1.2 + b * b;
                w1[2 * node] = std::sin(0.5 * i) * std::cos(0.3 * j);
                w1[2 * node + 1] = std::cos(0.2 * i + 0.4 * j);
            }
        double* d_pos = to_device(pos);
        double* d_met = to_device(met);
        double* d_w1 = to_device(w1);
        double* d_lap1 = to_device(std::vector<double>((mx - 1) * (my - 1) * 2, 0.0));
        double* d_cod = to_device(std::vector<double>(mx * my, 0.0));
        Tensor const position = Tensor::make(d_pos, SIL_F64, {mx, my}, 2);
        Tensor const metric = Tensor::make(d_met, SIL_F64, {mx, my}, 4);
        Tensor const w1in = Tensor::make(d_w1, SIL_F64, {mx, my}, 2);
        Tensor const lap1 = Tensor::make(d_lap1, SIL_F64, {mx - 1, my - 1}, 2);
        Tensor const cod = Tensor::make(d_cod, SIL_F64, {mx, my}, 1);
        auto const staged1 = make_staged_laplacian<1>(exec, lap1, w1in, &metric, position);
        staged1.run(exec, lap1, w1in);
        make_staged_codifferential<1>(exec, w1in, &metric, position).run(exec, cod, w1in);
        cudaDeviceSynchronize();
        write(dir + "/pos.bin", pos);
        write(dir + "/met.bin", met);
        write(dir + "/w1.bin", w1);
        write(dir + "/lap1.bin", to_host(d_lap1, (mx - 1) * (my - 1) * 2));
        write(dir + "/cod.bin", to_host(d_cod, mx * my));
        std::printf("metric ok\n");
    } catch (Error const& e) {
        std::fprintf(stderr, "%s\n", e.what());
        return 1;
    }
    return 0;
}
