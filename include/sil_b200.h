/*
 * sil_b200.h -- C ABI of the B200 (sm_100a) discrete-exterior-calculus library.
 *
 * Drop-in replacement for the device path of SimiLie's exterior-calculus
 * operators and of its 2D magnetostatics residual-minimisation solve.  Every
 * entry point is plain C: raw device pointers, sizes and strides, no C++ or
 * framework types.  All functions are non-throwing and return sil_status.
 * Asynchronous functions enqueue on the given CUDA stream (NULL = legacy
 * default stream) and return once enqueued; the caller synchronises, as a
 * SimiLie caller fences its Kokkos execution space.
 *
 * Fields follow SimiLie's DDC tensor-field layout: up to SIL_MAX_DIMS lattice
 * dimensions with explicit element strides plus one form-component index.
 * `front` is the absolute discrete coordinate of element 0 along each lattice
 * dimension (the DDC domain front); operators sample between fields in
 * absolute coordinates.  Form components are stored in the order of SimiLie's
 * antisymmetric index (lexicographic combinations of the form dimensions).
 * Dimensions not selected by `form_mask` are spectators (batch) dimensions.
 */
#ifndef SIL_B200_H
#define SIL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SIL_MAX_DIMS 6

typedef enum sil_status {
    SIL_OK = 0,
    SIL_ERR_INVALID = 1,      /* bad argument: shape, stride, rank, null pointer */
    SIL_ERR_UNSUPPORTED = 2,  /* valid request this library does not implement */
    SIL_ERR_CUDA = 3,         /* a CUDA runtime/driver call failed */
    SIL_ERR_ALLOC = 4,        /* device allocation failed */
    SIL_ERR_NONFINITE = 5,    /* a solve met NaN/Inf */
    SIL_ERR_STALLED = 6,      /* a solve stopped making progress */
    SIL_ERR_BUDGET = 7        /* a bounded device wait ran out */
} sil_status;

typedef enum sil_dtype { SIL_F64 = 0, SIL_F32 = 1 } sil_dtype;

typedef void* sil_stream; /* a cudaStream_t */

typedef struct sil_field {
    void* data;                    /* device pointer to element 0 */
    int32_t dtype;                 /* sil_dtype */
    int32_t ndims;                 /* lattice (+ spectator) dimensions, 1..SIL_MAX_DIMS */
    int32_t ncomp;                 /* stored form components, C(n, k) */
    int32_t reserved;
    int64_t front[SIL_MAX_DIMS];   /* absolute discrete coordinate of element 0 */
    int64_t extent[SIL_MAX_DIMS];
    int64_t stride[SIL_MAX_DIMS];  /* element strides */
    int64_t comp_stride;           /* element stride of the form-component index */
} sil_field;

/* Human-readable name of a status and the last error message of this thread. */
const char* sil_status_string(sil_status status);
const char* sil_last_error(void);

/* ---------------------------------------------------------------------- */
/* Coboundary and its transpose (bit-exact in FP64 with the reference).    */

/* d on a k-form: (d w)(s) = sum over the oriented boundary faces of each
 * basis (k+1)-simplex, in chain order, of w sampled with clamping to the
 * input domain.  out holds C(n, k+1) components.
 * Replaces: sil::exterior::deriv / coboundary,
 *   src/similie/exterior/coboundary.hpp:614-654, 698-709 (kernel 359-427). */
sil_status sil_deriv(sil_stream stream, uint32_t form_mask, int k, const sil_field* in,
                     sil_field* out);

/* Transposed coboundary on a k-form (zero outside the input domain,
 * backward shift of the second half-chain, negated chain sum).
 * Replaces: sil::exterior::transposed_coboundary,
 *   src/similie/exterior/coboundary.hpp:656-696 (kernel 523-605). */
sil_status sil_transposed_coboundary(sil_stream stream, uint32_t form_mask, int k,
                                     const sil_field* in, sil_field* out);

/* ---------------------------------------------------------------------- */
/* Geometry: a tensor-product (rectilinear) grid with the identity metric.  */
/* The discrete Hodge star on such a grid is diagonal in the component      */
/* basis; its factors are signed ratios of local edge lengths, computed on  */
/* the fly from the per-axis coordinates (no stored per-node tensor).       */

typedef struct sil_geometry_s* sil_geometry;

/* coords[a] points to npoints[a] HOST doubles: node coordinates along form
 * axis a (a = 0..n-1, in the order of the form dimensions).  front[a] is the
 * absolute discrete coordinate of coords[a][0] (may be NULL for all zeros).
 * Replaces the position + metric tensor fields passed to the staged
 * operators (identity metric, position(i,j,...) = (x_i, y_j, ...)). */
sil_status sil_geometry_create(sil_geometry* geometry, int n, const double* const* coords,
                               const int64_t* npoints, const int64_t* front);
sil_status sil_geometry_destroy(sil_geometry geometry);

/* Hodge star of a k-form into an (n-k)-form at every node of `out`.
 * Equivalent to tensor_prod(out, in, hodge) with the tensor that
 * fill_discrete_hodge_star stores: src/similie/exterior/hodge_star.hpp:227-273. */
sil_status sil_hodge_star(sil_geometry geometry, sil_stream stream, uint32_t form_mask, int k,
                          const sil_field* in, sil_field* out);

/* Write the per-node Hodge tensor SimiLie stores (Full<k> x Antisym<n-k>:
 * n^k index tuples x C(n,n-k) components per node, tuple index slowest).
 * Replaces: fill_discrete_hodge_star, src/similie/exterior/hodge_star.hpp:453-494. */
sil_status sil_fill_discrete_hodge_star(sil_geometry geometry, sil_stream stream, int k_in,
                                        sil_field* hodge);

/* General (per-node, dense) metric: fill the stored Hodge tensor from a
 * position field (n components per node) and a metric field (n*n
 * components per node, row-major; NULL for the identity), all FP64 device
 * fields whose lattice spans exactly the n <= 3 form dimensions.  The hodge
 * lattice must lie inside the position and metric lattices (edge vectors are
 * forward differences, backward at the last node of the position field).
 * Same tensor layout as sil_fill_discrete_hodge_star.
 * Replaces: fill_discrete_hodge_star<Idx1, Idx2, CircumcentricDual>(exec, hodge, metric, position),
 *   src/similie/exterior/hodge_star.hpp:453-494 (DiscreteHodgeStar 222-359). */
sil_status sil_fill_discrete_hodge_star_metric(sil_stream stream, int n, int k_in, const sil_field* position,
                                               const sil_field* metric, sil_field* hodge);

/* Apply a stored Hodge tensor (from either fill) to a k-form at every node
 * of `out`: out[t] = sum over index tuples of in(tuple) * hodge(tuple, t).
 * FP64, lattices over the n form dimensions.
 * Replaces: tensor_prod(out, in, hodge), src/similie/tensor/tensor_prod.hpp:108-157,
 *   as the staged operators use it (codifferential.hpp:460-504). */
sil_status sil_hodge_star_stored(sil_stream stream, int n, int k_in, const sil_field* hodge, const sil_field* in,
                                 sil_field* out);

/* Codifferential of a k-form (k >= 1), one fused kernel (star, transposed d,
 * star, sign (-1)^{n(k+1)+1}).
 * Replaces: codifferential / StagedCodifferential::run,
 *   src/similie/exterior/codifferential.hpp:321-508, 542-656. */
sil_status sil_codifferential(sil_geometry geometry, sil_stream stream, uint32_t form_mask, int k,
                              const sil_field* in, sil_field* out);

/* Staged codifferential of a k-form (1 <= k <= n <= 3) built from a
 * (metric, position) pair: position (n components per node) and metric (n*n
 * per node, row-major; NULL for the identity) FP64 fields spanning exactly
 * the n form dims, the metric lattice covering the position lattice.
 * create fills the two Hodge tensors the reference stores (k-form star and
 * (n-k+1)-form star, sil_fill_discrete_hodge_star_metric) over the position
 * lattice and owns them (enqueued on `stream`); run is one fused kernel per
 * call over every node of `out`, FP64, in and out lattices inside the
 * position lattice, no spectator dims.
 * Replaces: make_staged_codifferential(exec, tensor, metric, position) /
 *   StagedCodifferential ctor and run,
 *   src/similie/exterior/codifferential.hpp:398-437, 439-507, 510-540. */
typedef struct sil_codifferential_plan_s* sil_codifferential_plan;
sil_status sil_codifferential_plan_create(sil_codifferential_plan* plan, sil_stream stream, int n, int k,
                                          const sil_field* position, const sil_field* metric);
sil_status sil_codifferential_run(sil_codifferential_plan plan, sil_stream stream, const sil_field* in,
                                  sil_field* out);
sil_status sil_codifferential_plan_destroy(sil_codifferential_plan plan);

/* ---------------------------------------------------------------------- */
/* Hodge Laplacian (delta d for k = 0, delta d + d delta for 0 < k < n,     */
/* d delta for k = n).                                                      */

typedef enum sil_laplacian_mode {
    SIL_LAPLACIAN_FUSED = 0,   /* single pass: each field read once, written once */
    SIL_LAPLACIAN_UNFUSED = 1  /* reference kernel chain with intermediate fields */
} sil_laplacian_mode;

typedef struct sil_laplacian_plan_s* sil_laplacian_plan;

/* Staged Laplacian: precomputes what run() needs for fields shaped like
 * in_like / out_like (data pointers ignored) and owns any scratch.
 * Replaces: make_staged_laplacian / StagedLaplacian ctor,
 *   src/similie/exterior/laplacian.hpp:177-358, 360-648, 650-812. */
sil_status sil_laplacian_plan_create(sil_laplacian_plan* plan, sil_geometry geometry,
                                     uint32_t form_mask, int k, const sil_field* in_like,
                                     const sil_field* out_like, int mode);
/* Staged Laplacian of a k-form (0 <= k <= n <= 3) built from a (metric,
 * position) pair (same fields as sil_codifferential_plan_create): create
 * fills the up to four Hodge tensors the reference stores ((k+1)-, (n-k)-,
 * k- and (n-k+1)-form stars) over the position lattice, enqueued on
 * `stream`; sil_laplacian_run then evaluates delta d + d delta in one fused
 * kernel reading the stored tensors (plan kernel 4).  FP64, in_like and
 * out_like over exactly the n form dims, inside the position lattice.
 * Replaces: make_staged_laplacian(exec, laplacian_tensor, tensor, metric, position),
 *   src/similie/exterior/laplacian.hpp:261-310 (rank 0), 508-597 (intermediate
 *   ranks), 740-789 (top rank), 327-358. */
sil_status sil_laplacian_plan_create_metric(sil_laplacian_plan* plan, sil_stream stream, int n, int k,
                                            const sil_field* position, const sil_field* metric,
                                            const sil_field* in_like, const sil_field* out_like);
/* Replaces: StagedLaplacian::run, laplacian.hpp:312-324, 599-647, 791-811. */
sil_status sil_laplacian_run(sil_laplacian_plan plan, sil_stream stream, const sil_field* in,
                             sil_field* out);
sil_status sil_laplacian_plan_destroy(sil_laplacian_plan plan);
/* Device bytes of scratch the plan owns (0 for the fused mode). */
size_t sil_laplacian_plan_scratch_bytes(sil_laplacian_plan plan);
/* Kernel the plan runs: 0 table-driven fused (any rank / layout), 1 fused 2D
 * 0-form, 2 fused 2D 1-form with TMA-staged tiles, 3 unfused reference chain,
 * 4 fused over stored general-metric Hodge tensors. */
int sil_laplacian_plan_kernel(sil_laplacian_plan plan);
/* Launch shape chosen by the autotuner on the plan's first run (-1 before
 * it): kernel 2's pipeline shape (9 candidates in FP64: 0-5 one column per
 * thread, 6-8 column pairs; 6 in FP32), kernel 1's block width (64, 128 or
 * 256 threads: 0, 1, 2).  The first run times each candidate on the
 * caller's fields (kernel 2: from CUDA graphs of back-to-back launches) and
 * synchronises the stream, so it must not be inside a stream capture: run
 * a plan once before capturing it.  SIMILIE_B200_AUTOTUNE=0 skips the
 * tuning (kernel 2: shape 0, kernel 1: 256 threads),
 * SIMILIE_B200_LAP1_VARIANT=<digit> forces kernel 2's shape. */
int sil_laplacian_plan_variant(sil_laplacian_plan plan);
/* Bound of each pipeline wait of kernel 2, in mbarrier polls (-1: the default,
 * 4,194,304; 0: every wait runs out at once).  A wait that runs out makes the
 * kernel stop, let its loads in flight land and return; the plan's error flag
 * then reports SIL_ERR_BUDGET.  The failure-path tests set a bound of 0; no
 * counterpart in the reference. */
sil_status sil_laplacian_plan_set_wait_bound(sil_laplacian_plan plan, int32_t tries);
/* Synchronising check of the plan's device error flag: SIL_ERR_BUDGET when a
 * bounded wait inside a kernel ran out (the kernel returned early). */
sil_status sil_laplacian_plan_status(sil_laplacian_plan plan);

/* Plan-less Laplacian (free function form).
 * Replaces: sil::exterior::laplacian, src/similie/exterior/laplacian.hpp:814-951. */
sil_status sil_laplacian(sil_geometry geometry, sil_stream stream, uint32_t form_mask, int k,
                         const sil_field* in, sil_field* out);

/* ---------------------------------------------------------------------- */
/* 2D linear magnetostatics: residual operator d^T(nu dA) with identity    */
/* rows on the Dirichlet boundary, flat x-fastest layout row = i + nx*j.     */

/* y = K a for one problem (device pointers, nx*ny doubles each).
 * Replaces: MagnetostaticsOperator2D::apply,
 *   onelab_interface/magnetostatics_onelab.hpp:1271-1426 (stencils 1095-1258). */
sil_status sil_mag2d_apply(sil_stream stream, int64_t nx, int64_t ny, const double* node_mu,
                           const double* a, double* y);

/* Allocation-free variant of sil_mag2d_apply, for callers that must not
 * allocate device memory while they apply the operator: an operator applied
 * inside every iteration of someone else's Krylov loop (a matrix-free linear
 * operator wrapped by a solver library), code running under a memory pool or
 * a device-memory cap owned by its host framework, or a real-time loop where
 * an allocation (even a stream-ordered one, which sil_mag2d_apply makes for
 * its 1/mu scratch) costs an unbounded wait or is not permitted.
 * The scratch is a fixed device array inside the library of 2,097,152 doubles
 * (16 MiB), held by every GPU that loads the library until the process exits;
 * nx*ny above 2,097,152 is rejected with SIL_ERR_INVALID.  The first call on a
 * device looks up that array's device address (once per device, with the
 * device current); make that first call before any stream capture.  All calls
 * share the one array, so calls that overlap on the GPU (e.g. on two streams
 * at once) race; serialise them.  Same result as sil_mag2d_apply.
 * This entry point has no counterpart in the reference. */
sil_status sil_mag2d_apply_noalloc(sil_stream stream, int64_t nx, int64_t ny, const double* node_mu,
                                   const double* a, double* y);

typedef struct sil_mag2d_problem {
    int64_t nx, ny;          /* nodes per axis (>= 3) */
    const double* node_mu;   /* device, nx*ny: node permeability (mean of adjacent cells) */
    const double* rhs;       /* device, nx*ny: right-hand side, 0 on the boundary */
    double* solution;        /* device, nx*ny: written (initial guess is 0) */
} sil_mag2d_problem;

/* Every kind refines on the FP64 true residual r = b - A x: an inner solve
 * of A e = r, x += e, until ||b - A x|| <= tol ||b|| in FP64.  CG_F64 runs a
 * Jacobi-preconditioned CG in FP64 to half the tolerance (further passes only
 * correct recurrence drift); MIXED_IR runs it in FP32 to `inner_tolerance`
 * per pass (dot products in FP64).  LEARNED (2D only, at most 64 problems per call) runs a flexible CG in FP32
 * preconditioned by the learned network (`preconditioner`) inside FP64
 * refinement passes, and hands a problem to the MIXED_IR solver when its
 * preconditioned residual stalls (less than a 10x reduction over
 * `stall_window` iterations) or its inner solve runs out of iterations. */
typedef enum sil_solver_kind {
    SIL_SOLVER_CG_F64 = 0,
    SIL_SOLVER_MIXED_IR = 1,
    SIL_SOLVER_LEARNED = 2
} sil_solver_kind;

typedef struct sil_precond_s* sil_precond;

typedef struct sil_solve_settings {
    int32_t solver;              /* sil_solver_kind */
    int32_t max_iterations;      /* total inner iterations per problem */
    double relative_tolerance;   /* stop when ||b - A x|| <= tol * ||b|| */
    int32_t inner_iterations;    /* MIXED_IR / LEARNED: inner iterations per refinement pass */
    double inner_tolerance;      /* MIXED_IR / LEARNED: inner relative reduction per pass */
    sil_precond preconditioner;  /* LEARNED: the trained network */
    int32_t stall_window;        /* LEARNED: iterations per stall check (0: 200) */
    int32_t flexible_directions; /* LEARNED: directions the flexible CG keeps, 1..16 (0: 8) */
    /* Nonlinear solves: NULL runs every Newton step's linear solve as the
     * matrix-free Jacobi-CG; otherwise the Jacobian is assembled at the state
     * every step and CG runs with this preconditioner of the menu (the
     * reference's nonlinear branch with build_matrix + build_preconditioner,
     * minimize_strong_formulation_residual.hpp:1432-1436). */
    const struct sil_menu_settings* jacobian_preconditioner;
} sil_solve_settings;

typedef struct sil_solve_diagnostics {
    int32_t iterations;          /* inner iterations, all stages together */
    int32_t converged;
    int32_t refinements;         /* FP64 refinement passes */
    int32_t status;              /* sil_status of this problem */
    double initial_residual_l2;
    double final_residual_l2;
    double final_relative_residual;
    int32_t learned_iterations;  /* LEARNED: iterations of the preconditioned solve */
    int32_t fallback;            /* LEARNED: 1 if the plain solver finished the problem */
} sil_solve_diagnostics;

/* Solve a batch of independent problems on one device stream.  Writes one
 * diagnostics record per problem into diag (HOST memory).  Synchronous.
 * Replaces: solvers::minimize_strong_formulation_residual (linear branch),
 *   src/similie/solvers/minimize_strong_formulation_residual.hpp:1308-1382
 *   with the Jacobi-preconditioned Ginkgo CG it runs (1028-1304). */
sil_status sil_mag2d_solve_batch(const sil_mag2d_problem* problems, int nproblems,
                                 const sil_solve_settings* settings, sil_solve_diagnostics* diag,
                                 sil_stream stream);

/* ---------------------------------------------------------------------- */
/* 2D magnetostatics with a nonlinear (saturating) ferromagnetic material.  */
/* A node whose ferromagnetic fraction (share of adjacent cells made of the */
/* material) is above 1/2 follows the B-H curve: at a sampled node with     */
/* moments B = (B0, B1) and q = |B|^2 the field is H_c = B_c (F + q F'),     */
/* F(q) = h(b)/b at b = sqrt(q), and the Jacobian is                        */
/* d_rc (F + q F') + 4 B_r B_c F' + 2 q B_r B_c F''; other nodes keep B/mu.  */
/* Replaces: MaterialMagnetostaticsHamiltonian + InterpolatedNonlinearBHCurve */
/*   onelab_interface/magnetostatics_onelab.hpp:957-1011, 4471-4565;        */
/*   src/similie/physics/magnetostatics/nonlinear_magnetostatics.py:14-369. */

/* B-H curve: n samples (2..64) of b (increasing, b[0] >= 0) and h, HOST
 * arrays; h is interpolated linearly in b and extended linearly beyond the
 * last sample. */
typedef struct sil_bh_curve {
    int32_t n;
    const double* b;
    const double* h;
} sil_bh_curve;

/* One nonlinear problem; device FP64 node arrays of nx*ny (x fastest).
 * node_ferro: ferromagnetic fraction per node.  solution holds the initial
 * guess on entry (zero it for x0 = 0, as the linear solve starts) and the
 * result on exit. */
typedef struct sil_mag2d_nl_problem {
    int64_t nx, ny;
    const double* node_mu;
    const double* node_ferro;
    sil_bh_curve curve;
    const double* rhs;
    double* solution;
} sil_mag2d_nl_problem;

/* y = the nonlinear residual operator applied to a (identity rows on the
 * boundary).  Replaces: MagnetostaticsOperator2D::apply with the material
 * Hamiltonian, magnetostatics_onelab.hpp:1271-1426. */
sil_status sil_mag2d_nl_apply(sil_stream stream, const sil_mag2d_nl_problem* problem, const double* a, double* y);

/* y = J(state) x, the operator's Jacobian at `state` applied to x.
 * Replaces: apply_jacobian (2D), magnetostatics_onelab.hpp:2799-2915. */
sil_status sil_mag2d_nl_apply_jacobian(sil_stream stream, const sil_mag2d_nl_problem* problem, const double* state,
                                       const double* x, double* y);

/* Newton solve of every problem of the batch: at most 30 steps, each
 * solving J(x) d = r by Jacobi-preconditioned CG (FP64) to
 * settings->relative_tolerance (at most settings->max_iterations
 * iterations; with settings->jacobian_preconditioner, CG with that menu
 * preconditioner on the Jacobian assembled at x), then a line search of at most 8 candidates x + alpha d,
 * alpha halving from 1, that stops at the first residual below the current
 * one, else takes the best seen.  Converged when ||b - F(x)|| <= tol *
 * ||b - F(x0)||.  diag: iterations = all CG iterations, refinements =
 * Newton steps.  Synchronous.  settings->solver is ignored.
 * Replaces: solvers::minimize_strong_formulation_residual (nonlinear
 *   branch), src/similie/solvers/minimize_strong_formulation_residual.hpp:1383-1569. */
sil_status sil_mag2d_nl_solve_batch(const sil_mag2d_nl_problem* problems, int nproblems,
                                    const sil_solve_settings* settings, sil_solve_diagnostics* diag,
                                    sil_stream stream);

/* 3D magnetostatics with the nonlinear material: the 3D curl-curl operator
 * with the penalty gauge (sil_mag3d_problem, gauge 0) whose sampled nodes
 * follow the material law above with q = |B|^2 over the three curl moments;
 * the Jacobian applies each sampled node's 3x3 Hessian of the Hamiltonian.
 * Replaces: MagnetostaticsOperator3D with MaterialMagnetostaticsHamiltonian,
 *   magnetostatics_onelab.hpp:5110-5126 (nonlinear dispatch), 2241-2396
 *   (operator, dpotential_dt of the equations), 2924-3110 (apply_jacobian). */
typedef struct sil_mag3d_nl_problem {
    int64_t nx, ny, nz;       /* nodes per axis (>= 3), nx*ny*nz < 2^31 / 9 */
    const double* x;          /* HOST, nx strictly increasing node coordinates */
    const double* y;          /* HOST, ny */
    const double* z;          /* HOST, nz */
    const double* node_mu;    /* device, nx*ny*nz */
    const double* node_ferro; /* device, nx*ny*nz: ferromagnetic fraction per node */
    sil_bh_curve curve;
    const double* rhs;        /* device, 3*nx*ny*nz */
    double* solution;         /* device, 3*nx*ny*nz: initial guess on entry, result on exit */
    double gauge_penalty;     /* gamma: > 0 for the penalty gauge, nonzero for the divergence gauge */
    int32_t gauge;            /* 0: penalty (the default); 1: divergence gauge, as in sil_mag3d_problem */
} sil_mag3d_nl_problem;

/* y = the 3D nonlinear operator applied to a (3*nx*ny*nz doubles, device). */
sil_status sil_mag3d_nl_apply(sil_stream stream, const sil_mag3d_nl_problem* problem, const double* a, double* y);

/* y = J(state) x for the 3D nonlinear operator. */
sil_status sil_mag3d_nl_apply_jacobian(sil_stream stream, const sil_mag3d_nl_problem* problem, const double* state,
                                       const double* x, double* y);

/* Newton solve of every 3D problem of the batch, the scheme of
 * sil_mag2d_nl_solve_batch (Jacobi-CG on the Jacobian, or the settings'
 * jacobian_preconditioner on the assembled Jacobian; halving line search).
 * Synchronous. */
sil_status sil_mag3d_nl_solve_batch(const sil_mag3d_nl_problem* problems, int nproblems,
                                    const sil_solve_settings* settings, sil_solve_diagnostics* diag,
                                    sil_stream stream);

/* ---------------------------------------------------------------------- */
/* Learned multilevel convolutional preconditioner of the 2D solve.        */
/* M(r) = Jacobi step, then a U-Net correction computed at half resolution  */
/* from [r1 / rms(r1), log(nu) / log(1000)], then a Jacobi step; 32          */
/* channels, 3x3 convolutions, BF16 activations and weights with FP32        */
/* accumulation on the tensor cores.  Trained on (source, solution) pairs    */
/* with the loss 1 - (u.b)^2 / ((u.K u)(x.b)), u = M(b): the K-norm error    */
/* left after one optimally scaled preconditioned step.                       */
/* The reference has no learned preconditioner; the entry points below are  */
/* the sil_precond_load/train/save family of its GPU design.                 */

/* (sil_precond is declared with the solver settings above.) */

/* One node grid of a batch: nx x ny nodes, x fastest, starting at element
 * `offset` of the batch's flat FP32 node arrays (nu = 1/mu, r, b, x, out). */
typedef struct sil_precond_sample {
    int32_t nx, ny;
    int64_t offset;
} sil_precond_sample;

int64_t sil_precond_num_params(void);
/* New network with He-normal weights drawn from `seed`. */
sil_status sil_precond_create(sil_precond* out, uint64_t seed, sil_stream stream);
void sil_precond_destroy(sil_precond p);
/* Parameters as FP32 host arrays of sil_precond_num_params() values
 * (save / load); set_params resets the optimiser state. */
sil_status sil_precond_get_params(sil_precond p, float* host);
sil_status sil_precond_set_params(sil_precond p, const float* host, sil_stream stream);
/* The Adam state of training: first and second moments (host FP32
 * [sil_precond_num_params()] each, either may be NULL) and the steps taken.
 * set_params resets it; set_optimizer_state after it restores a checkpoint
 * exactly.  Synchronous.  No counterpart in the reference. */
sil_status sil_precond_get_optimizer_state(sil_precond p, float* m, float* v, int64_t* step);
sil_status sil_precond_set_optimizer_state(sil_precond p, const float* m, const float* v, int64_t step,
                                           sil_stream stream);
/* out = M(r) for 1..64 samples (device arrays). */
sil_status sil_precond_apply(sil_precond p, sil_stream stream, const sil_precond_sample* samples, int n,
                             const float* nu, const float* r, float* out);
/* The same for the samples whose entry of `active` (device, one int32 per
 * sample, read when the kernels run) is nonzero; the others are neither read
 * nor written, so a batched Krylov loop pays only for unconverged samples. */
sil_status sil_precond_apply_active(sil_precond p, sil_stream stream, const sil_precond_sample* samples, int n,
                                    const float* nu, const float* r, const int32_t* active, float* out);
/* Mean loss over the batch for right-hand sides b with solutions x, the
 * per-sample losses (host, may be NULL) and the gradient with respect to
 * every parameter (host FP32, may be NULL).  Synchronous. */
sil_status sil_precond_loss_grad(sil_precond p, sil_stream stream, const sil_precond_sample* samples, int n,
                                 const float* nu, const float* b, const float* x, double* loss,
                                 double* per_sample_loss, float* grad_host);
/* loss_grad followed by one Adam step (beta 0.9 / 0.999, eps 1e-8). */
sil_status sil_precond_train_step(sil_precond p, sil_stream stream, const sil_precond_sample* samples, int n,
                                  const float* nu, const float* b, const float* x, float learning_rate,
                                  double* loss);
/* Diagnostic: copy an intermediate buffer of the last batch to the host as
 * FP32 (which: 0 h, 1 p, 2 g activations of `level`; 3 dh, 4 dg gradients;
 * 5 input features, 6 network output, 7 M(r), 8 network-output gradient). */
sil_status sil_precond_debug_fetch(sil_precond p, int which, int level, float* host, int64_t count);

/* ---------------------------------------------------------------------- */
/* 3D linear magnetostatics: curl-curl residual operator with the Coulomb   */
/* gauge penalty, on a rectilinear grid.  Nodes flat x fastest              */
/* (node = i + nx*(j + ny*k)), unknown row = 3*node + c (c = x, y, z);       */
/* identity rows on the Dirichlet boundary.                                   */

typedef struct sil_mag3d_problem {
    int64_t nx, ny, nz;      /* nodes per axis (>= 3) */
    const double* x;         /* HOST, nx strictly increasing node coordinates */
    const double* y;         /* HOST, ny */
    const double* z;         /* HOST, nz */
    const double* node_mu;   /* device, nx*ny*nz: node permeability (mean of adjacent cells) */
    const double* rhs;       /* device, 3*nx*ny*nz: right-hand side, 0 on the boundary */
    double* solution;        /* device, 3*nx*ny*nz: written (initial guess is 0) */
    double gauge_penalty;    /* gamma > 0 (the reference's default is 20) */
    int32_t gauge;           /* 0: penalty gamma * (star A), the default.  1: divergence gauge
                              * gamma * sum_c w(c) D(c, row) (D A)(c), D the codifferential of the
                              * 1-form A (boundary columns dropped), w(c) the product of the local
                              * spacings at node c (the reference's SIMILIE_DIVERGENCE_GAUGE_3D,
                              * magnetostatics_onelab.hpp:1890-1945, 2355-2392); gamma may then be
                              * negative (SIMILIE_VECTOR_POTENTIAL_GAUGE_SIGN_3D folded in). */
} sil_mag3d_problem;

/* y = K a for one problem (a, y: device, 3*nx*ny*nz doubles; rhs and
 * solution of the problem are not used).
 * Replaces: MagnetostaticsOperator3D::apply_with_precomputed_stencils,
 *   onelab_interface/magnetostatics_onelab.hpp:2241-2396 (Hodge factors 856-910). */
sil_status sil_mag3d_apply(sil_stream stream, const sil_mag3d_problem* problem, const double* a, double* y);

/* The same operator with its set-up done once (device spacing tables,
 * 1/mu, the divergence gauge's coefficient table), as the reference builds
 * its stencils once per operator; an apply is then one kernel on `stream`
 * and may be captured in a CUDA graph.  The permeability is read at create
 * time.  create is synchronous on `stream`.
 * Replaces: the MagnetostaticsOperator3D constructor (precomputed stencils,
 *   onelab_interface/magnetostatics_onelab.hpp:1815-1900) and
 *   apply_with_precomputed_stencils (2241-2396). */
typedef struct sil_mag3d_operator_s* sil_mag3d_operator;
sil_status sil_mag3d_operator_create(sil_mag3d_operator* out, sil_stream stream, const sil_mag3d_problem* problem);
sil_status sil_mag3d_operator_apply(sil_mag3d_operator op, sil_stream stream, const double* a, double* y);
sil_status sil_mag3d_operator_destroy(sil_mag3d_operator op);

/* Batched 3D solve; same settings, diagnostics and refinement scheme as
 * sil_mag2d_solve_batch.  Synchronous.
 * Replaces: solvers::minimize_strong_formulation_residual for
 *   MagnetostaticsOperator3D, minimize_strong_formulation_residual.hpp:1308-1382. */
sil_status sil_mag3d_solve_batch(const sil_mag3d_problem* problems, int nproblems,
                                 const sil_solve_settings* settings, sil_solve_diagnostics* diag,
                                 sil_stream stream);

/* ---------------------------------------------------------------------- */
/* Assembled operators: the magnetostatics operators as CSR matrices, the   */
/* reference's preconditioner menu on them, and a preconditioned CG.       */

/* CSR matrix in device memory (int32 row pointers and columns, FP64
 * values, columns ascending, exact zeros dropped); opaque, owned by the
 * library.
 * Replaces: assemble_matrix_data, magnetostatics_onelab.hpp:3554-3737 (2D),
 *   3120-3534 (3D), read into a gko::matrix::Csr<double, int32>. */
typedef struct sil_csr_s* sil_csr;

/* The 2D operator of sil_mag2d_apply as a CSR matrix.  Synchronous. */
sil_status sil_mag2d_assemble(sil_stream stream, int64_t nx, int64_t ny, const double* node_mu, sil_csr* out);
/* The 3D operator of sil_mag3d_apply (either gauge) as a CSR matrix.  Synchronous. */
sil_status sil_mag3d_assemble(sil_stream stream, const sil_mag3d_problem* problem, sil_csr* out);
/* The Jacobians of the nonlinear operators at `state` (device) as CSR
 * matrices (assemble_matrix_data(operator_model, state)).  Synchronous. */
sil_status sil_mag2d_nl_assemble_jacobian(sil_stream stream, const sil_mag2d_nl_problem* problem,
                                          const double* state, sil_csr* out);
sil_status sil_mag3d_nl_assemble_jacobian(sil_stream stream, const sil_mag3d_nl_problem* problem,
                                          const double* state, sil_csr* out);
/* Size and device arrays of a matrix (any output may be NULL). */
sil_status sil_csr_get(sil_csr m, int64_t* n, int64_t* nnz, const int32_t** row_ptr, const int32_t** col,
                       const double** val);
/* Copies the arrays (n + 1 row pointers, nnz columns and values) to host or
 * device buffers.  Synchronous. */
sil_status sil_csr_copy(sil_stream stream, sil_csr m, int32_t* row_ptr, int32_t* col, double* val);
/* y = A x (device vectors of n doubles). */
sil_status sil_csr_spmv(sil_stream stream, sil_csr m, const double* x, double* y);
void sil_csr_destroy(sil_csr m);

/* The reference's PreconditionerType, in its order
 * (minimize_strong_formulation_residual.hpp:53-63). */
typedef enum sil_pc_kind {
    SIL_PC_IDENTITY = 0,
    SIL_PC_JACOBI = 1,
    SIL_PC_SPD_ISAI = 2,
    SIL_PC_SYMMETRIC_GAUSS_SEIDEL = 3,
    SIL_PC_SSOR = 4,
    SIL_PC_CHEBYSHEV_JACOBI = 5,
    SIL_PC_IR_JACOBI = 6,
    SIL_PC_GENERAL_ISAI = 7
} sil_pc_kind;

/* The menu's parameters; 0 selects the reference's default
 * (StrongFormulationSolverSettings, minimize_strong_formulation_residual.hpp:
 * 61-75): SOR relaxation 1.2, 8 Chebyshev steps on [0.05, 1.5], 8 IR steps
 * with relaxation 1. */
typedef struct sil_menu_settings {
    int32_t kind;                  /* sil_pc_kind */
    double sor_relaxation_factor;  /* Ssor */
    int32_t chebyshev_iterations;
    double chebyshev_lower_bound;  /* eigenvalue bounds of the Jacobi-preconditioned operator */
    double chebyshev_upper_bound;
    int32_t ir_iterations;
    double ir_relaxation_factor;
} sil_menu_settings;

/* A preconditioner built on a matrix (which must outlive it): Jacobi
 * z = D^-1 r; SpdIsai z = Z^T Z r with Z the factorized sparse approximate
 * inverse on the pattern of tril(A); GeneralIsai z = M r with M the
 * incomplete sparse approximate inverse on the pattern of A (ISAI rows of
 * at most 32 entries); SymmetricGaussSeidel / Ssor the symmetric
 * successive over-relaxation M = (D - wE) D^-1 (D - wF) / (w (2 - w)),
 * w = 1 for Gauss-Seidel, its triangular solves run level by level;
 * ChebyshevJacobi / IrJacobi a fixed number of Chebyshev / Richardson steps
 * on the Jacobi-preconditioned system from a zero guess.  Synchronous.
 * Replaces: build_preconditioner, minimize_strong_formulation_residual.hpp:
 *   921-1026 (Ginkgo's Jacobi, SpdIsai, GeneralIsai, GaussSeidel, Sor,
 *   Chebyshev and Ir). */
typedef struct sil_csr_precond_s* sil_csr_precond;
sil_status sil_csr_precond_create(sil_stream stream, sil_csr m, const sil_menu_settings* settings,
                                  sil_csr_precond* out);
/* z = M^-1 r (device vectors).  The preconditioner's scratch is shared by
 * its applies and solves: use one preconditioner on one stream at a time. */
sil_status sil_csr_precond_apply(sil_stream stream, sil_csr_precond p, const double* r, double* z);
void sil_csr_precond_destroy(sil_csr_precond p);

/* Preconditioned CG from x = 0 until ||r|| <= tol ||b|| (recursive
 * residual, as Ginkgo's ResidualNorm with a reduction factor) or
 * settings->max_iterations; diag->iterations, converged, residuals.
 * settings->solver is ignored.  Synchronous.
 * Replaces: solve_linearized_system with the assembled matrix
 *   (use_matrix_free = false), minimize_strong_formulation_residual.hpp:
 *   1028-1304. */
sil_status sil_csr_solve(sil_stream stream, sil_csr m, sil_csr_precond p, const double* rhs, double* x,
                         const sil_solve_settings* settings, sil_solve_diagnostics* diag);

/* The reference's SIMILIE_SOLVER menu on an assembled matrix, in its order:
 * 0 cg, 1 minres, 2 fcg, 3 gmres, 4 bicgstab, 5 gcr, 6 idr. */
typedef enum sil_krylov_kind {
    SIL_KRYLOV_CG = 0,
    SIL_KRYLOV_MINRES = 1,
    SIL_KRYLOV_FCG = 2,
    SIL_KRYLOV_GMRES = 3,
    SIL_KRYLOV_BICGSTAB = 4,
    SIL_KRYLOV_GCR = 5,
    SIL_KRYLOV_IDR = 6
} sil_krylov_kind;

/* x = A^-1 rhs by the chosen Krylov method with the preconditioner p, from
 * x = 0 until ||r|| <= tol ||b|| or settings->max_iterations: MINRES (Paige
 * & Saunders, stopping on its iterate's true residual), flexible CG, GMRES
 * and GCR restarted after `dim` directions (0: 100), BiCGSTAB, IDR(s) with
 * s = `dim` (0: 8) and a fixed-seed shadow space; all but MINRES and FCG
 * preconditioned on the right.  CG is sil_csr_solve.  Scalars are reduced on
 * the host in a fixed order.  Synchronous.
 * Replaces: the SIMILIE_SOLVER choices of solve_linearized_system,
 *   minimize_strong_formulation_residual.hpp:1069-1130 (Ginkgo's Minres, Fcg,
 *   Gmres, Bicgstab, Gcr, Idr; Krylov dimensions 1079-1120). */
sil_status sil_csr_krylov_solve(sil_stream stream, sil_csr m, sil_csr_precond p, int32_t solver, int32_t dim,
                                const double* rhs, double* x, const sil_solve_settings* settings,
                                sil_solve_diagnostics* diag);

#ifdef __cplusplus
}
#endif

#endif /* SIL_B200_H */
