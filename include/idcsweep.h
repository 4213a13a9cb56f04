/*
 * idcsweep — B200 (sm_100a) implementation of the 2-D upwind-DG discrete-ordinates transport sweep of
 * crockatt/idc-transport-solver, behind a plain C ABI.
 *
 * Every entry point takes plain pointers and sizes, returns an int status (IDC_OK == 0) and never
 * aborts.  Arrays use the reference's layouts, halo cells included, so a caller holding the
 * reference's objects passes PointerAtCell(0,0) of each one directly:
 *
 *   psi   [i][j][q][d][e]  (nx+2)*(ny+2)*nq*N doubles   RKDG::OrdinateFlux::Index,   objects/RKDG/OrdinateFlux.hpp:639-700
 *   phi   [i][j][d][e]     (nx+2)*(ny+2)*N doubles      RKDG::DensityFunction::Index, objects/RKDG/DensityFunction.hpp
 *   sigma [i][j]           (nx+2)*(ny+2) doubles        RKDG::CrossSection with DG degree 0 (piecewise constant)
 *
 * with i the x index (0 and nx+1 are ghost cells), j the y index, N = (p+1)^2 for DG degree p, and
 * ordinates sorted into the reference's quadrant ranges (Quadrants(k), utils/Quadrule/OrdinateSet.hpp:352):
 * quadrant 0 xi>0,eta>0; 1 xi>0,eta<0; 2 xi<0,eta>0; 3 xi<0,eta<0.
 *
 * Pointers marked "loc" are host pointers when loc == IDC_LOC_HOST (the library copies them to and from
 * its own device buffers inside the call) and device pointers on the context's GPU when
 * loc == IDC_LOC_DEVICE (the call works on them in place).  Calls are synchronous: when one returns, its
 * results are in place.  A context is not re-entrant: use one context per host thread.
 */
#ifndef IDCSWEEP_H
#define IDCSWEEP_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------------------------------------- */
enum {
    IDC_OK = 0,
    IDC_ERR_ARG = 1,            /* invalid argument (null pointer, bad size, unsorted ordinates, ...)   */
    IDC_ERR_UNSUPPORTED = 2,    /* valid for the reference but not implemented here (e.g. p > 2)        */
    IDC_ERR_CUDA = 3,           /* a CUDA runtime call failed; idc_last_error_message() has the text     */
    IDC_ERR_TIMEOUT = 4,        /* a device-side wait gave up (bounded spin); results are not valid      */
    IDC_ERR_NOT_CONVERGED = 5,  /* an iterative solve stopped at its iteration limit                     */
    IDC_ERR_STATE = 6,          /* call order violated (e.g. sweep before idc_set_ordinates)             */
    IDC_ERR_NOMEM = 7           /* device allocation failed                                              */
};

enum { IDC_LOC_HOST = 0, IDC_LOC_DEVICE = 1 };

/* Arithmetic of a sweep.  IDC_PREC_FP64 restates the reference's FP64 Gaussian elimination.
 * IDC_PREC_FP32_REFINED factors and solves each cell system in FP32 and refines the solution with
 * FP64 residuals of the same cell system (all inputs, outputs and inter-cell traces stay FP64).
 * IDC_PREC_FP32 is the unrefined FP32 solve (FP32 cell arithmetic and moment sums; about 1e-7 relative).
 * IDC_PREC_FP32_IR (idc_gmres_solve only) runs the Krylov iterations with FP32 sweeps inside an FP64
 * iterative refinement of the solve: the right-hand side, every residual and the final psi come from FP64
 * sweeps, so the solution meets the FP64 tolerance. */
enum { IDC_PREC_FP64 = 0, IDC_PREC_FP32_REFINED = 1, IDC_PREC_FP32 = 2, IDC_PREC_FP32_IR = 3 };

typedef struct idc_ctx idc_ctx;

typedef struct idc_problem_desc {
    int64_t nx, ny;          /* interior cells in x and y (DomainDecomposition nx(0), nx(1))            */
    double ax, bx, ay, by;   /* domain [ax,bx] x [ay,by]; dx = (bx-ax)/nx, dy = (by-ay)/ny              */
    int64_t dg_degree;       /* DG degree p of psi and phi (Global::DG_degree): 0..3; 3 runs on the     */
                             /* elimination kernel in FP64 (no FP32, transposed, IDC or batched sweeps) */
    int64_t sigma_degree;    /* DG degree of the cross sections: 0 (piecewise constant) or dg_degree    */
    int32_t device;          /* CUDA device ordinal                                                     */
    int32_t flags;           /* reserved, must be 0                                                     */
} idc_problem_desc;

/* ---- context --------------------------------------------------------------------------------------- */

/* Creates a context for one grid on one GPU.  Replaces the construction of
 * SweepOperator<RKDG::OrdinateFlux> (linear_solvers/Abstract/SweepOperator.cpp:25-49) for the
 * "gpu-wavefront" sweep pattern. */
int idc_ctx_create(const idc_problem_desc *desc, idc_ctx **out);

/* Releases every device resource of the context.  Accepts NULL. */
int idc_ctx_destroy(idc_ctx *ctx);

/* Installs the ordinate set: nq ordinates (xi, eta, w) sorted into the four quadrant ranges
 * quad_bounds[0..4] (quad_bounds[0] = 0, quad_bounds[4] = nq).  Replaces the angular part of the
 * SweepOperator set-up, i.e. the per-ordinate matrices of SweepLinearSolveSpec::ComputeMatrices
 * (linear_solvers/RKDG/SweepCellSolve/SweepLinearSolveSpec.cpp:98-158). */
int idc_set_ordinates(idc_ctx *ctx, int64_t nq, const double *xi, const double *eta, const double *w,
                      const int64_t quad_bounds[5]);

/* Installs sigma_t and sigma_s on the halo-padded cell grid (loc as above): one value per cell when
 * sigma_degree = 0, or, when sigma_degree = dg_degree (high-order cross sections), the (p+1)^2 Legendre
 * moments of each cell, [cell][u][v] as the CrossSection's DensityFunction array holds them.  sigma_s may
 * be NULL (treated as zero).  These are the CrossSection arguments of SweepOperator::Apply and
 * ImplicitSolver::Solve.  High-order cross sections enter as the reference's tensor branches do: the cell
 * matrix of CalcA (linear_solvers/RKDG/SweepCellSolve/SweepLinearSolveSpec.cpp:298-318), Smv and Lmv
 * (operators/RKDG/TransportOperator.cpp:367-386, :1335-1359), with the tensor of Legendre triple products of
 * CrossSection::ComputeTensor (objects/RKDG/CrossSection.cpp:141-230).  They run on the elimination kernel in
 * FP64: sweeps, idc_smv, idc_lmv, source iteration, GMRES (its DSA preconditioner uses the cell averages)
 * and IDC time stepping with implicit scattering; FP32 sweeps, transposed operators, explicit-scattering
 * IDC, batches and reflecting edges return IDC_ERR_UNSUPPORTED. */
int idc_set_sigma(idc_ctx *ctx, const double *sigma_t, const double *sigma_s, int loc);

/* Tile shape of the persistent sweep kernel: G ordinates x R rows per thread block (0 = automatic).
 * A tuning knob only: results do not depend on it.  No reference counterpart (the reference's
 * closest knob is the compile-time SIMD block length, utils/SIMD.hpp). */
int idc_set_tiling(idc_ctx *ctx, int32_t ordinates_per_block, int32_t rows_per_block);

/* ---- the sweep ------------------------------------------------------------------------------------- */

/* In-place transport sweep psi <- (Omega.grad + sigma_t + 1/dt)^{-1} psi over the interior cells,
 * ghost cells of psi_inout carrying the inflow boundary values (they are read, never written).
 * dt = +INFINITY is steady state.  If phi_out is not NULL it receives phi = sum_q w_q psi_q on the
 * interior cells (the fused TransportOperator::Pmv(1, 0, psi, phi)); its ghost cells are zeroed.
 * Replaces SweepOperator<RKDG::OrdinateFlux>::Apply (linear_solvers/Abstract/SweepOperator.cpp:118-135)
 * with SweepPatternUniCartWavefront::Sweep (.../SweepPattern/SweepPatternUniCartWavefront.cpp:121-332). */
int idc_sweep(idc_ctx *ctx, double *psi_inout, double dt, double *phi_out, int precision, int loc);

/* Out-of-place form: result <- (Omega.grad + sigma_t + 1/dt)^{-1} source on the interior cells, the
 * inflow values read from the ghost cells of `source`; result's ghost cells are not written; source is
 * not modified (it must not overlap result unless they are the same pointer).  The shape of
 * SweepPattern::Sweep(source, result, sigma, initial) (.../SweepPattern/SweepPattern.hpp:117-122), of
 * which SweepOperator::Apply is the source == result case. */
int idc_sweep_out(idc_ctx *ctx, const double *source, double *result, double dt, double *phi_out, int precision,
                  int loc);

/* `count` out-of-place sweeps (sources[k] -> results[k], phi_out[k] if phi_out is not NULL), each as
 * idc_sweep_out.  With loc = IDC_LOC_HOST the upload of step k+1, the sweep of step k and the download of
 * step k-1 overlap (three streams, double-buffered device arrays), so a sequence of host-resident steps
 * costs about the slower copy direction per step instead of both; host arrays should be pinned.  A
 * batch-of-right-hand-sides form of SweepPattern::Sweep with no counterpart in the reference. */
int idc_sweep_out_many(idc_ctx *ctx, int64_t count, const double *const *sources, double *const *results,
                       double *const *phi_out, double dt, int precision, int loc);

/* ---- transport operators (operators/RKDG/TransportOperator.hpp:25-43), interior cells ------------ */

/* phi <- beta*phi + alpha * sum_q w_q psi_q.              TransportOperator::Pmv, TransportOperator.cpp:140-158 */
int idc_pmv(idc_ctx *ctx, double alpha, double beta, const double *psi, double *phi, int loc);

/* psi_q <- beta*psi_q + alpha * sigma_s phi / (4 pi).    TransportOperator::Smv, TransportOperator.cpp:317-400 */
int idc_smv(idc_ctx *ctx, double alpha, double beta, const double *phi, double *psi, int loc);

/* y <- beta*y + alpha * (Omega.grad + sigma_t) x.        TransportOperator::Lmv, TransportOperator.cpp:1215-1689 */
int idc_lmv(idc_ctx *ctx, double alpha, double beta, const double *x, double *y, int loc);

/* ---- implicit solvers (linear_solvers/Abstract/ImplicitSolver.hpp:116-122) ------------------------- */

/* Source iteration from a zero initial guess: source_inout holds Q on entry and psi on return.
 * Stops when the absolute l2 change of phi over interior cells is <= abs_tol or after max_its.
 * Replaces SISolver::Solve (linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:190-254).
 * *iters and *final_err (either may be NULL) report the iteration count and last change. */
int idc_source_iteration(idc_ctx *ctx, double *source_inout, double dt, double abs_tol, int64_t max_its,
                         int precision, int loc, int64_t *iters, double *final_err);

/* ---- allocation-free sweep ------------------------------------------------------------------------- */

#define IDC_NOALLOC_MAX_ITEMS 4096      /* work items (row blocks x ordinate chunks) one call can schedule */
#define IDC_NOALLOC_MAX_ORDINATES 1024  /* ordinates one call accepts                                      */

/* The out-of-place sweep of idc_sweep_out for callers that cannot allocate device memory: a host code that
 * owns the whole GPU through its own memory arena, or a loop that cannot pay for cudaMalloc/cudaFree,
 * which may synchronise the device and fail once the memory is reserved.  No counterpart in the
 * reference (its sweep allocates per-thread work space with malloc on every call,
 * SweepPatternUniCartWavefront.cpp:147-170).
 *
 * Everything is passed in: xi, eta, w (nq each), sigma_t, source, result and phi_out (nullable) are DEVICE
 * pointers on desc->device; quad_bounds is a host array.  The call makes no cudaMalloc/cudaFree and uses
 * no context.  As in idc_sweep_out, the inflow values are read from the ghost cells of `source` and only
 * the interior cells of `result` are written (its ghost cells keep what the caller put there).  phi_out
 * receives sum_q w_q result_q on the interior cells, added in ordinate order (bitwise the same on every
 * call), and zero on its ghost cells.  The call reads xi and eta back to check their quadrant signs and
 * synchronises `stream` before it returns; on failure idc_last_error_message() has the reason.  The sweep's own scratch (work-queue head, error word, progress flags, work-item list) is
 * one fixed file-scope device array of about 96 KiB that every GPU loading the library keeps until the
 * process exits; problems needing more than IDC_NOALLOC_MAX_ITEMS work items, or more than
 * IDC_NOALLOC_MAX_ORDINATES ordinates, are rejected with IDC_ERR_ARG (use idc_sweep_out for those).
 * The first call on a device looks up that array's device address (cudaGetSymbolAddress).  All calls
 * share the array and it keeps the last call's contents; each call clears the parts that must start at
 * zero.  Calls whose kernels overlap on the GPU
 * would race on it: calls from one process are serialised by a lock, and the call returns only after its
 * work on `stream` (a cudaStream_t, NULL for the default stream) has finished.  The caller's current
 * device is restored on return. */
int idc_sweep_noalloc(const idc_problem_desc *desc, int64_t nq, const double *xi, const double *eta, const double *w,
                      const int64_t quad_bounds[5], const double *sigma_t, const double *source, double *result,
                      double dt, double *phi_out, int precision, void *stream);

/* GMRES(restart) on the scalar flux, the Peierls form (I - P L^{-1} S) phi = P L^{-1} Q, from a zero
 * initial guess; stops when the residual 2-norm is <= abs_tol (absolute, the reference's default criterion),
 * then psi = L^{-1}(S phi + Q) is returned in source_inout (Q on entry).  Arnoldi (CGS2), Hessenberg least
 * squares and all vectors are FP64; `precision` selects the sweep arithmetic, or IDC_PREC_FP32_IR: FP64
 * iterative refinement whose corrections are GMRES solves with FP32 sweeps (*iters then counts their
 * iterations; each correction adds one FP64 residual sweep).  Replaces
 * PETScPeierlsSolver::Solve with IPLS (linear_solvers/Abstract/ImplicitSolver/PETScPeierlsSolver.cpp:423-572);
 * PETSc's LGMRES augmentation is not reproduced (same fixed point, different iteration counts).  Returns
 * IDC_ERR_NOT_CONVERGED after max_its iterations, as the reference throws. */
int idc_gmres_solve(idc_ctx *ctx, double *source_inout, double dt, double abs_tol, int32_t restart, int64_t max_its,
                    int precision, int loc, int64_t *iters, double *final_resid);

/* Right preconditioner of idc_gmres_solve: 0 = none, 1 = diffusion synthetic acceleration (DSA): a 2-D
 * cell-centred diffusion solve on the cell-average moment, -div(1/(3 sigma_t) grad e) + sigma_a e =
 * sigma_s r_00 with Marshak vacuum boundaries, by inner_steps Jacobi-preconditioned CG steps; GMRES then
 * runs in its flexible form.  The reference has DSA only in 1-D (SIP-DG inside its PETSc Peierls solver,
 * linear_solvers/RKDG/ImplicitSolver/PETScPeierlsSolver.cpp:27-376); the converged solution does not
 * depend on the preconditioner.  The adjoint solve of idc_adjoint_grad uses its transpose (rhs r_00,
 * correction sigma_s e), which gives the adjoint operator the preconditioned spectrum of the forward. */
int idc_set_preconditioner(idc_ctx *ctx, int kind, int32_t inner_steps);

/* ---- time integration ------------------------------------------------------------------------------- */

enum { IDC_SCATTER_EXPLICIT = 0, IDC_SCATTER_IMPLICIT = 1 };

/* IDC time integration of d psi/dt = -(L - S P) psi + q: `steps` steps of size dt from psi_inout (its ghost
 * cells are the inflow values of the initial state) with `source` q constant in time (its ghost cells are
 * the inflow values during the steps).  num_nodes Gauss-Lobatto nodes, num_corrections corrections,
 * non-hybrid update form: IDCIntegrator::Step_Nonhybrid, ComputeResiduals, ComputeSource
 * (time_integrators/RKDG/idc.cpp:846-955, 1657-1740) and SetNodes (:2305-2381).
 * scattering = IDC_SCATTER_IMPLICIT: every substep solves (1/(h dt) + L - S P) with the GPU GMRES
 * (abs_tol, restart, max_its), as the reference does with its implicit solver; high-order cross sections
 * and DG degree 3 are taken here.
 * scattering = IDC_SCATTER_EXPLICIT (IMEX): every substep is one sweep with the scattering lagged to the
 * previous node and corrected by the deferred-correction iterations; with use_graph a step is captured
 * once as a CUDA graph and replayed (lane or modal kernel: DG degree <= 2, piecewise-constant cross
 * sections; at DG degree 1, unless idc_set_tile_shape fixed a shape, a grid too small to give the lane
 * kernel an item for every resident warp runs the step on the modal kernel's (8, 5) shape, the faster one
 * there, and the context's default shape returns afterwards).  Reflecting edges and periodic grids return
 * IDC_ERR_UNSUPPORTED.  Quadrature sums and residuals are FP64; `precision` selects the
 * sweep arithmetic.  *sweeps receives the number of sweeps performed. */
int idc_idc_integrate(idc_ctx *ctx, double *psi_inout, const double *source, double dt, int64_t steps,
                      int32_t num_nodes, int32_t num_corrections, int scattering, int precision, double abs_tol,
                      int32_t restart, int64_t max_its, int use_graph, int loc, int64_t *sweeps);

/* Out-of-place sweep with the fused isotropic scattering source: result = L^{-1}(source +
 * scatter_scale * sigma_s * phi_scatter / (4 pi)) on interior cells, phi_out = P result.  source may be
 * NULL (zero source, vacuum inflow), result may be NULL (not stored), phi_scatter may be NULL (no
 * scattering term); DEVICE pointers only (loc must be IDC_LOC_DEVICE).  The fused form of
 * SISolver::Solve's per-iteration Smv + Apply + Pmv (linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:
 * 190-254) for callers that drive their own iteration, e.g. across GPUs holding disjoint ordinate sets. */
int idc_sweep_fused(idc_ctx *ctx, const double *source, double *result, double dt, const double *phi_scatter,
                    double scatter_scale, double *phi_out, int precision, int loc);

/* ---- tile shapes and batches ------------------------------------------------------------------------- */

/* Tile shape of the sweep kernel: ordinates per row segment (seg: 4, 8, 16 or 32) and compute warps per
 * thread block.  warps = 0 selects the lane-pipelined kernel (every warp sweeps its own row block of 32/seg
 * rows; seg 4, 8 or 16; FP64 sweeps); warps 1..7 the modal kernel with that many compute warps stacked per
 * thread block (at most 5 at DG degree 2 and 7 below, fewer if the shape's shared memory would not fit).
 * 0, 0 restores the default (the lane kernel for FP64, the modal kernel for the FP32 modes; 16-wide lane
 * segments at DG degree 2, 8-wide at degree 1 for up to 24 ordinates per quadrant).  The shape applies to sweeps with a source or a psi output; the moments-only
 * sweeps of the Krylov iterations keep their own default (narrow segments, which suit them).  Results do
 * not depend on it beyond the last bits of the moments. */
int idc_set_tile_shape(idc_ctx *ctx, int32_t seg, int32_t warps);

/* Autotuner: times every tile shape of both kernels on this context's problem with `source` (device psi
 * array; plain sweeps: the IMEX sweeps of idc_idc_integrate may prefer another shape) and keeps the fastest (reported in *seg, *warps; warps = 0: the lane kernel). */
int idc_autotune(idc_ctx *ctx, const double *source, double dt, int precision, int32_t *seg, int32_t *warps);

/* A batch of independent problems (contexts on one GPU) swept together: one persistent launch per DG
 * degree whose work queue interleaves every problem's row blocks.  idc_batch_sweep takes host arrays of
 * device pointers, one entry per added context in order (entries may be NULL: no source / not stored /
 * no moments); FP64 or FP32_REFINED.  idc_batch_autotune picks the tile shape of each degree by timing
 * the batched sweep on the given inputs.  No counterpart in the reference (it sweeps one problem). */
typedef struct idc_batch idc_batch;
int idc_batch_create(idc_batch **out);
int idc_batch_add(idc_batch *b, idc_ctx *ctx);
int idc_batch_sweep(idc_batch *b, const double *const *sources, double *const *results, double *const *phi_out,
                    double dt, int precision);
int idc_batch_autotune(idc_batch *b, const double *const *sources, double *const *results, double dt, int precision);
int idc_batch_last_timing(idc_batch *b, double *ms);
/* The tile shape a batch uses for its problems of DG degree dg_degree at `precision` (what the autotuner
 * picked, the default, or what was set; set 0, 0 to return to the default).  seg 4, 8, 16 or 32 with warps
 * 1..7 is the modal kernel; in FP64, seg 4, 8 or 16 with warps = 0 is the lane kernel (one warp per row
 * block).  The autotuner tries both. */
int idc_batch_set_shape(idc_batch *b, int dg_degree, int precision, int32_t seg, int32_t warps);
int idc_batch_get_shape(idc_batch *b, int dg_degree, int precision, int32_t *seg, int32_t *warps);
/* GMRES(restart) to abs_tol on every member's Peierls system at once (each member's problem as
 * idc_gmres_solve solves it, with the preconditioner set on its context): every Krylov step applies the
 * operators of all unconverged members through one batched sweep and brings their Arnoldi columns back with
 * one synchronisation; converged members drop out of the launches.  psi_inout: host array of device
 * pointers, one per member in order (Q on entry, psi on return); iters and final_resids (nullable): host
 * arrays with one entry per member.  FP64 or FP32_REFINED sweeps.  IDC_ERR_NOT_CONVERGED if a member
 * stopped at max_its.  The batched form of PETScPeierlsSolver::Solve (linear_solvers/Abstract/
 * ImplicitSolver/PETScPeierlsSolver.cpp:423-572) for many independent problems; the reference solves one. */
int idc_batch_gmres_solve(idc_batch *b, double *const *psi_inout, double dt, double abs_tol, int32_t restart,
                          int64_t max_its, int precision, int64_t *iters, double *final_resids);
int idc_batch_destroy(idc_batch *b);

/* ---- discrete adjoint --------------------------------------------------------------------------------- */

/* Transposed sweep: result = L^{-T} source on interior cells, where L^{-1} is the sweep of idc_sweep_out
 * (psi = L^{-1} q with the cell systems divided by dx*dy, so that L^{-T} is the exact transpose of that
 * linear map on interior cells with zero inflow).  Cells are processed downwind-first per quadrant with
 * the transposed cell matrices and face couplings; the source's ghost cells are not read.  moments_out
 * (nullable) receives sum_q result_q (unweighted, interior cells; ghost cells zero).  FP64 and
 * FP32_REFINED only.  No counterpart in the reference (it has no adjoint); it is the transpose of
 * SweepOperator::Apply (linear_solvers/Abstract/SweepOperator.cpp:118-135) restated per cell from
 * SweepLinearSolveSpec.cpp:98-158, 267-321, 473-598. */
int idc_sweep_adjoint(idc_ctx *ctx, const double *source, double *result, double dt, double *moments_out, int precision,
                      int loc);

/* Gradients of the detector response J = sum_{cells, dofs} detector * phi of the transport problem
 * (L - S P) psi = q (the problem idc_gmres_solve solves; psi is its solution, halo layout) with respect to
 * the per-cell sigma_t, sigma_s (halo layout, ghost entries zero) and the isotropic source moments
 * dsource (phi layout; the angular source is dsource-moment / (4 pi) on every ordinate).  The adjoint
 * problem (L - S P)^T lam = P^T detector is solved by GMRES on (I - S^T L^{-T} P^T) mu = detector, then
 * lam = L^{-T} P^T mu; dJ/dsigma_t = -sum_{q,k} lam psi, dJ/dsigma_s = sum_k (sum_q lam)_k phi_k / (4 pi),
 * dJ/dq_k = (sum_q lam)_k / (4 pi) per cell.  Outputs are nullable.  No counterpart in the reference. */
int idc_adjoint_grad(idc_ctx *ctx, const double *psi, const double *detector, double dt, double abs_tol,
                     int32_t restart, int64_t max_its, int precision, double *dsigma_t, double *dsigma_s,
                     double *dsource, int loc, int64_t *iters, double *final_resid);

/* Gradients of J = sum detector * phi(psi^steps) after `steps` implicit-Euler steps
 * (1/dt + L - S P) psi^{n+1} = psi^n / dt + source, psi^0 = psi0 (each step the Peierls GMRES solve of
 * idc_gmres_solve), with respect to the per-cell sigma_t, sigma_s (halo layout), the isotropic source
 * moments dsource (phi layout; source = moment / (4 pi) on every ordinate, constant in time) and the
 * initial angular flux dpsi0 (psi layout, ghost cells zero).  The adjoint steps run backwards,
 * A^T lam^N = P^T detector and A^T lam^n = lam^{n+1} / dt, and the gradients sum the per-step terms of
 * idc_adjoint_grad over n.  The forward states are checkpointed every `checkpoint_every` steps (<= 0: about
 * sqrt(steps)) and recomputed segment by segment in the backward pass, so device memory holds about
 * steps / checkpoint_every + checkpoint_every angular fluxes.  J (nullable) receives the functional;
 * *solves (nullable) the number of forward and adjoint GMRES solves.  Ghost cells of source are the fixed
 * inflow (not differentiated).  Outputs are nullable.  No counterpart in the reference: it is the transpose
 * of the implicit-Euler (DIRK 1) time step of time_integrators/RKDG/dirk.cpp, which is also IDC's
 * prediction step (time_integrators/RKDG/idc.cpp:846-955). */
int idc_adjoint_transient(idc_ctx *ctx, const double *psi0, const double *source, double dt, int64_t steps,
                          const double *detector, int64_t checkpoint_every, double abs_tol, int32_t restart,
                          int64_t max_its, int precision, double *dsigma_t, double *dsigma_s, double *dsource,
                          double *dpsi0, double *J, int loc, int64_t *solves);

/* The same gradients for IDC time stepping with implicit scattering (idc_idc_integrate with
 * IDC_SCATTER_IMPLICIT: num_nodes Gauss-Lobatto nodes, num_corrections correction sweeps, update form, every
 * substep (1/(h dt) + L - S P) psi_n = src_n solved by the Peierls GMRES), J = sum detector * phi(psi^steps).
 * The adjoint runs backwards through every step's correction levels: for each substep the transposed
 * solve A_n^T lam = (the stage's adjoint), which feeds the previous substep's adjoint (lam / (h dt)) and the
 * adjoints of the previous level's residuals (the quadrature weights times lam); those become the previous
 * level's stage adjoints through the transpose of the residual operator, (L - S P)^T (the transposed Lmv).
 * The gradient terms are the solves' (as idc_adjoint_transient) and the residuals' (the same form, opposite
 * sign, no source term).  Checkpointing as idc_adjoint_transient (each step's stages are recomputed from its
 * input in the backward pass); device memory holds about steps / checkpoint_every + checkpoint_every +
 * (num_corrections + 1) num_nodes + 3 num_nodes angular fluxes.  No counterpart in the reference: it is the
 * transpose of IDCIntegrator::Step_Nonhybrid with ComputeResiduals / ComputeSource (update form),
 * time_integrators/RKDG/idc.cpp:846-955, 1657-1740. */
int idc_adjoint_idc(idc_ctx *ctx, const double *psi0, const double *source, double dt, int64_t steps,
                    int32_t num_nodes, int32_t num_corrections, const double *detector, int64_t checkpoint_every,
                    double abs_tol, int32_t restart, int64_t max_its, int precision, double *dsigma_t,
                    double *dsigma_s, double *dsource, double *dpsi0, double *J, int loc, int64_t *solves);

/* y = beta y + alpha L^T x on interior cells (device arrays, psi layout): the transpose of idc_lmv with x's
 * ghost cells taken as zero (boundary data, not unknowns); y's ghost cells are not written.  The transpose of
 * TransportOperator::Lmv (operators/RKDG/TransportOperator.cpp:1215-1689), which the reference has no use for;
 * the IDC adjoint applies it to the residuals' adjoints. */
int idc_lmv_transpose(idc_ctx *ctx, double alpha, double beta, const double *x, double *y, int loc);

/* ---- binary files ------------------------------------------------------------------------------------ */

/* The reference's serial 2-D binary formats, on the halo layouts of this ABI (no GPU involved).
 * .sd2 (scalar flux): SpatialDomain::WriteToDisk (objects/SpatialDomain.cpp:385-411) then
 * DensityFunction::WriteToDisk (objects/RKDG/DensityFunction.cpp:2228-2400): [nx ax bx][ny ay by],
 * dg_degree, byte size, count, density.  .af2 (angular flux): OrdinateFlux::WriteToDisk and ReadFromDisk
 * (objects/RKDG/OrdinateFlux.cpp:2553-2620, 2720-2930): the domain block, the ordinate type name
 * (null-terminated, "#R" appended for symmetric-reduced sets) and ang_order, then dg_degree, byte size,
 * count, density.  Readers with density == NULL return the header only; `count` is the number of doubles. */
int idc_write_sd2(const char *path, int64_t nx, int64_t ny, double ax, double bx, double ay, double by,
                  int64_t dg_degree, const double *density);
int idc_read_sd2(const char *path, int64_t *nx, int64_t *ny, double *ax, double *bx, double *ay, double *by,
                 int64_t *dg_degree, double *density, int64_t capacity, int64_t *count);
int idc_write_af2(const char *path, int64_t nx, int64_t ny, double ax, double bx, double ay, double by,
                  const char *ordinate_type, int64_t ang_order, int64_t dg_degree, int64_t nq, const double *density);
int idc_read_af2(const char *path, int64_t *nx, int64_t *ny, double *ax, double *bx, double *ay, double *by,
                 char *ordinate_type, int64_t type_capacity, int64_t *ang_order, int64_t *dg_degree, double *density,
                 int64_t capacity, int64_t *count);

/* ---- diagnostics ----------------------------------------------------------------------------------- */

/* Text for a status code (static storage). */
const char *idc_strerror(int status);

/* Text of the most recent error on this thread (static per-thread storage). */
const char *idc_last_error_message(void);

/* Bound of every device-side wait of the context's kernels (a wait on another warp's or thread block's
 * progress, polled or blocking in the barrier unit): after `polls` polls the wait gives up, the kernel
 * records the failure in the context's device error word, every warp leaves, and the call returns
 * IDC_ERR_TIMEOUT after re-arming the context's trace buffers, so the next call starts clean.  polls <= 0
 * restores the default (2^22 polls, seconds of waiting; a sweep's waits normally end within microseconds).
 * Meant for failure-detection tests and for callers that want a hung peer reported sooner.  The
 * reference has no counterpart (its OpenMP barriers wait without bound). */
int idc_set_spin_limit(idc_ctx *ctx, int64_t polls);

/* Reflecting boundaries: `edges` as the reference's BoundaryEdge bits (IDC_EDGE_X_MIN 1, IDC_EDGE_X_MAX 2,
 * IDC_EDGE_Y_MIN 4, IDC_EDGE_Y_MAX 8; 0 = none, the default).  With any, every sweep of the context (idc_sweep,
 * idc_source_iteration, idc_gmres_solve) runs the quadrants one after another in the reference's order
 * 3, 2, 1, 0, in place, and after each quadrant refills the reflecting edges' ghost cells of the ordinates
 * entering through them with the first interior cell's values of the reflected ordinate, the mirrored
 * Legendre modes negated (SweepPatternUniCartWavefront::Sweep with sweep_octants_in_sequence,
 * linear_solvers/Abstract/SweepPattern/SweepPatternUniCartWavefront.cpp:186-251, and
 * OrdinateFlux::ReflectBoundaries, objects/RKDG/OrdinateFlux.cpp:1181-1360).  Every ordinate needs its
 * reflection partner in the set (IDC_ERR_ARG otherwise, as the reference's ComputeReflectMap).  The
 * source's ghost cells on the other edges are the inflow; the result's ghost cells on reflecting edges hold
 * the last reflection.  idc_source_iteration follows SISolver::Solve: psi starts at zero and the reflecting
 * edges' ghost cells are not copied from the source, so each sweep reads the reflections of the last.
 * idc_gmres_solve adds the reflecting edges' incoming ghost values to its unknowns and reaches the same fixed
 * point for every edge set.  IDC time stepping with implicit scattering reflects each step's initial stage, as
 * IDCIntegrator::Step_Nonhybrid does (time_integrators/RKDG/idc.cpp:855-859), and solves every substep this
 * way.  FP64 and FP32 sweeps (the lane kernel); IDC_PREC_FP32_IR, transposed sweeps, explicit-scattering
 * IDC, batches and ordinate-partitioned solves with reflecting boundaries return
 * IDC_ERR_UNSUPPORTED. */
/* Periodic boundaries (the reference's Global::periodic, deck key `periodic`): 1 = on, 0 = off (the default).
 * A sweep reads the ghost cells as given, as the reference's does.  idc_source_iteration follows
 * SISolver::Solve on a periodic grid: psi starts at zero; from the second iteration on, each iteration first
 * fills the ghost cells of the four edges with the opposite interior edge's values (DensityFunction::
 * SynchronizeHalos, objects/Abstract/DensityFunction.cpp:927-960) and then copies the source into the interior
 * cells only.  idc_gmres_solve adds the edges' incoming ghost values to its unknowns and reaches the same fixed
 * point.  idc_lmv uses the opposite edges' cells as the upwind neighbours across an edge (Lmv synchronises its
 * input's halos first).  IDC time stepping with implicit scattering synchronises each step's initial stage
 * and solves every substep this way.  Reflecting edges, IDC_PREC_FP32_IR, adjoint solves, transposed
 * operators, explicit-scattering IDC, batches and, for GMRES, ordinate-partitioned solves return
 * IDC_ERR_UNSUPPORTED on a periodic grid. */
int idc_set_periodic(idc_ctx *ctx, int32_t periodic);

#define IDC_EDGE_X_MIN 1
#define IDC_EDGE_X_MAX 2
#define IDC_EDGE_Y_MIN 4
#define IDC_EDGE_Y_MAX 8
int idc_set_reflecting(idc_ctx *ctx, int32_t edges);

/* Ordinate-partitioned solves over several processes (one rank per GPU; each rank's context holds its slice
 * of every quadrant's ordinates, e.g. contiguous near-equal chunks): `fn` sums a moment-sized array of the
 * context's GPU over the ranks, in place, and must give every rank bitwise the same sums (an NCCL or MPI
 * all-reduce does).  Once set, every moment output of the context's sweeps is completed by one call of `fn`
 * before it is used or returned, so idc_source_iteration, idc_gmres_solve (with DSA, and IDC_PREC_FP32_IR)
 * and idc_sweep's phi run the whole quadrature's algorithm: the moment-sized vectors (Krylov basis, DSA
 * state) are replicated and every rank computes the same Arnoldi steps and stopping decisions; psi stays
 * the rank's own ordinates.  The context synchronises its stream before each call; `fn` returns 0 once
 * the sums are in `data`, anything else fails the call with IDC_ERR_STATE.  fn = NULL turns it off.  Not
 * inside CUDA graph captures (idc_idc_integrate with use_graph: IDC_ERR_STATE).  The reference spreads
 * its solves over MPI ranks by space instead (KBA sweeps, linear_solvers/Abstract/SweepPattern/
 * SweepPatternUniCartKBA.cpp, with MPI_Allreduce of the norms, objects/RKDG/DensityFunction.cpp:1154). */
typedef int (*idc_allreduce_fn)(double *data, int64_t n, void *user);
int idc_set_allreduce(idc_ctx *ctx, idc_allreduce_fn fn, void *user);

/* Device time in milliseconds of the last sweep kernel launched by the context (CUDA events on the
 * launching stream), and the number of kernels the last idc_* call launched. */
int idc_last_timing(idc_ctx *ctx, double *sweep_kernel_ms, int64_t *kernels_launched);

#ifdef __cplusplus
}
#endif

#endif /* IDCSWEEP_H */
