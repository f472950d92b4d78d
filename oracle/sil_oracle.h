/*
 * sil_oracle.h -- CPU restatement of SimiLie's discrete-exterior-calculus
 * operators and of its 2D magnetostatics residual solve.
 *
 * THIS IS TEST INFRASTRUCTURE. It is the correctness checker and the timed
 * CPU baseline for the CUDA library in similie_b200/. Nothing in the product
 * path links, loads or calls it.
 *
 * Every function follows the reference algorithm step by step (chain
 * construction, boundary orientation, summation order, clamped / zero-outside
 * sampling, stored per-node Hodge-star tensors, staged kernels). The file and
 * line of the reference code each routine restates is given at its
 * definition in sil_oracle.cpp.
 *
 * Field convention: a field is a strided array over up to SILO_MAX_DIMS
 * lattice dimensions plus one component index.  `front` is the absolute
 * lattice coordinate of element 0 along each dimension (DDC's domain front);
 * sampling between fields is done in absolute coordinates, exactly like
 * DDC's DiscreteElement arithmetic.  Form dimensions (those the exterior
 * algebra acts on) are selected by a bit mask; the other dimensions are
 * spectators (batch) and are never shifted.
 */
#ifndef SIL_ORACLE_H
#define SIL_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SILO_MAX_DIMS 6

typedef struct silo_field {
    double* data;
    int32_t ndims;
    int32_t ncomp;
    int64_t front[SILO_MAX_DIMS];
    int64_t extent[SILO_MAX_DIMS];
    int64_t stride[SILO_MAX_DIMS];
    int64_t comp_stride;
} silo_field;

/* Coboundary d on a k-form (clamped sampling).  out has C(n,k+1) comps. */
int silo_coboundary(uint32_t form_mask, int k, const silo_field* in, silo_field* out);

/* Transposed coboundary on a k-form (zero-outside sampling, backward shift,
 * final negation).  out has C(n,k+1) comps. */
int silo_transposed_coboundary(uint32_t form_mask, int k, const silo_field* in, silo_field* out);

/* Fill the stored per-node discrete Hodge star tensor mapping k_in-forms to
 * (n-k_in)-forms: layout per node [n^k_in full tuples][C(n,n-k_in) comps].
 * position: n comps per node; metric: n*n comps per node (row-major) or
 * NULL for the identity metric.  hodge->ncomp must be n^k_in * C(n, n-k_in).
 * The lattice of `hodge`, `position` and `metric` spans the form dims only. */
int silo_fill_hodge_star(int n, int k_in, const silo_field* position, const silo_field* metric,
                         silo_field* hodge);

/* Apply a stored Hodge tensor at every node of `in` (k_in-form) into `out`. */
int silo_apply_hodge_star(int n, int k_in, const silo_field* hodge, const silo_field* in,
                          silo_field* out);

/* Effective per-node Hodge matrix (C(n,n-k) x C(n,k), row-major) at one
 * node, computed by DiscreteHodgeStar::run on unit cochains. */
int silo_hodge_matrix(int n, int k_in, const silo_field* position, const silo_field* metric,
                      const int64_t* node, double* matrix);

/* Staged codifferential of a k-form (k >= 1): reference two-kernel structure. */
int silo_codifferential(int n, int k, const silo_field* position, const silo_field* metric,
                        const silo_field* in, silo_field* out);

/* Staged Hodge Laplacian of a k-form (0 <= k <= n): reference kernel chain
 * (delta d for k = 0, delta d + d delta for 0 < k < n, d delta for k = n). */
int silo_laplacian(int n, int k, const silo_field* position, const silo_field* metric,
                   const silo_field* in, silo_field* out);

/* Same chain with the Hodge tensors supplied by the caller (setup excluded
 * from timing).  hs[0..3] = derivative, dual-derivative, codifferential,
 * dual-codifferential stored Hodge tensors (unused ones may be NULL). */
int silo_laplacian_prefilled(int n, int k, const silo_field* const* hs, const silo_field* in,
                             silo_field* out);

/* Component counts of the stored Hodge tensors silo_laplacian_prefilled needs. */
int silo_laplacian_hodge_ncomp(int n, int k, int which);
int silo_laplacian_hodge_kin(int n, int k, int which);

/* ------------------------------------------------------------------ */
/* 2D linear magnetostatics (x-fastest flat layout row = i + nx*j).     */

/* Node permeability: mean of the (up to 4) adjacent cell values. */
void silo_mag2d_node_mu(int64_t nx, int64_t ny, const double* cell_mu, double mu0,
                        double* node_mu);
/* Right-hand side b_i = sum over adjacent cells of 1/4 * area * J, 0 on the boundary. */
void silo_mag2d_rhs(int64_t nx, int64_t ny, const double* x, const double* y,
                    const double* cell_j, double* rhs);
/* Matrix-free residual operator (moments criterion), identity rows on the boundary. */
void silo_mag2d_apply(int64_t nx, int64_t ny, const double* node_mu, const double* a, double* y);
/* Diagonal of the assembled operator (Jacobi preconditioner). */
void silo_mag2d_diagonal(int64_t nx, int64_t ny, const double* node_mu, double* diag);
/* Jacobi-preconditioned CG from x = 0, stop when ||r|| <= tol * ||b||.
 * Returns iterations; *final_rel receives the recurrence relative residual. */
int silo_mag2d_cg(int64_t nx, int64_t ny, const double* node_mu, const double* rhs,
                  double* x, double tol, int max_iter, double* final_rel);

/* ------------------------------------------------------------------ */
/* 3D linear magnetostatics, curl-curl with the gauge penalty.          */
/* Nodes flat x fastest (node = i + nx*(j + ny*k)), DOF row = 3*node + c. */

/* Node permeability: mean of the (up to 8) adjacent cell values. */
void silo_mag3d_node_mu(int64_t nx, int64_t ny, int64_t nz, const double* cell_mu, double mu0, double* node_mu);
/* b = sum over adjacent cells of 1/8 * dual face * J_c, zero on the boundary.
 * cell_j holds 3 components per cell, cell = ci + ncx*(cj + ncy*ck). */
void silo_mag3d_rhs(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                    const double* cell_j, double* rhs);
/* y = (curl^T W curl + gamma H_A) a on interior DOFs, identity on the boundary. */
void silo_mag3d_apply(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                      const double* node_mu, double gamma, const double* a, double* out);
void silo_mag3d_diagonal(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                         const double* node_mu, double gamma, double* diag);
int silo_mag3d_cg(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                  const double* node_mu, double gamma, const double* rhs, double* sol, double tol, int max_iter,
                  double* final_rel);

/* ------------------------------------------------------------------ */
/* 2D nonlinear magnetostatics: ferromagnetic nodes (node_ferro > 0.5)   */
/* follow an interpolated B-H curve given by n samples (b, h), 2..64.    */

/* F(q) = h(b)/b at b = sqrt(q) and its first two q-derivatives. */
void silo_bh_eval(int n, const double* b, const double* h, int count, const double* q, double* f, double* df,
                  double* d2f);
/* y = nonlinear residual operator (moments criterion), identity rows on the boundary. */
void silo_mag2d_nl_apply(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                         const double* b, const double* h, const double* a, double* y);
/* y = J(state) x, the operator's Jacobian at `state` applied to x. */
void silo_mag2d_nl_jacobian_apply(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                                  const double* b, const double* h, const double* state, const double* x,
                                  double* y);
/* Diagonal of the Jacobian at `state` (1 on boundary rows). */
void silo_mag2d_nl_jacobian_diagonal(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro,
                                     int n, const double* b, const double* h, const double* state, double* diag);
/* Newton with a halving line search from the initial guess in x; every step
 * solves J d = r by Jacobi-CG to the relative tolerance tol.  Returns the
 * CG iterations; newton_steps and final_rel (||r|| / ||r0||) are written. */
int silo_mag2d_nl_solve(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                        const double* b, const double* h, const double* rhs, double* x, double tol, int max_iter,
                        int* newton_steps, double* final_rel);

/* ------------------------------------------------------------------ */
/* 3D nonlinear magnetostatics: the 3D curl-curl + penalty-gauge operator */
/* with the material law of the 2D problem at the sampled nodes.         */

void silo_mag3d_nl_apply(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                         const double* node_mu, const double* node_ferro, double gamma, int n, const double* b,
                         const double* h, const double* a, double* out);
void silo_mag3d_nl_jacobian_apply(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y,
                                  const double* z, const double* node_mu, const double* node_ferro, double gamma,
                                  int n, const double* b, const double* h, const double* state, const double* v,
                                  double* out);
void silo_mag3d_nl_jacobian_diagonal(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y,
                                     const double* z, const double* node_mu, const double* node_ferro, double gamma,
                                     int n, const double* b, const double* h, const double* state, double* diag);
/* Newton as silo_mag2d_nl_solve, on the 3D operator (3 * nx*ny*nz unknowns). */
int silo_mag3d_nl_solve(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                        const double* node_mu, const double* node_ferro, double gamma, int n, const double* b,
                        const double* h, const double* rhs, double* sol, double tol, int max_iter, int* newton_steps,
                        double* final_rel);

/* ------------------------------------------------------------------ */
/* Assembled CSR operators (int64 row pointers, int32 columns) and the   */
/* reference's preconditioner menu: kind 0 Identity, 1 Jacobi, 2 SpdIsai, */
/* 3 SymmetricGaussSeidel, 4 Ssor, 5 ChebyshevJacobi, 6 IrJacobi,         */
/* 7 GeneralIsai.  params: sor relaxation factor, Chebyshev iterations,   */
/* lower and upper bound, IR iterations, IR relaxation factor.            */
int silo_csr_precond_apply(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int kind,
                           const double* params, const double* r, double* z);
int silo_csr_isai_values(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int kind,
                         double* out_val);
int silo_csr_pcg(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int kind, const double* params,
                 const double* b, double* x, double tol, int max_iter, double* final_rel);

/* Newton as silo_mag2d_nl_solve / silo_mag3d_nl_solve, each linear solve a
 * CG with the menu preconditioner `kind` on the Jacobian assembled at the
 * state.  Returns the CG iterations (-1 if a preconditioner cannot be built). */
int silo_mag2d_nl_solve_menu(int64_t nx, int64_t ny, const double* node_mu, const double* node_ferro, int n,
                             const double* b, const double* h, int kind, const double* params, const double* rhs,
                             double* x, double tol, int max_iter, int* newton_steps, double* final_rel);
int silo_mag3d_nl_solve_menu(int64_t nx, int64_t ny, int64_t nz, const double* x, const double* y, const double* z,
                             const double* node_mu, const double* node_ferro, double gamma, int n, const double* b,
                             const double* h, int kind, const double* params, const double* rhs, double* sol,
                             double tol, int max_iter, int* newton_steps, double* final_rel);

/* The reference's SIMILIE_SOLVER menu on a CSR matrix with a menu
 * preconditioner: solver 0 cg, 1 minres, 2 fcg, 3 gmres, 4 bicgstab, 5 gcr,
 * 6 idr; dim = GMRES / GCR Krylov dimension or IDR subspace dimension.
 * x from 0 until ||r|| <= tol ||b||; returns the iterations (-1 on error). */
int silo_csr_krylov(int64_t n, const int64_t* ptr, const int32_t* col, const double* val, int solver, int dim,
                    int kind, const double* params, const double* b, double* x, double tol, int max_iter,
                    double* final_rel);

/* Primal reduction and reconstruction of one node's form / cochain
 * (Reduction<Primal>::run, Reconstruction<Primal>::run); binom(n, K) values
 * in and out.  Return 0, or 1 for a bad rank. */
int silo_reduce_primal(int n, int K, const silo_field* position, const int64_t* node, const double* form, double* out);
int silo_reconstruct_primal(int n, int K, const silo_field* position, const int64_t* node, const double* cochain,
                            double* out);

/* Threads OpenMP uses (for reporting). */
int silo_num_threads(void);

#ifdef __cplusplus
}
#endif

#endif
