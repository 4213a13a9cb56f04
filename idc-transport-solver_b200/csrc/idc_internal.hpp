// Internal declarations shared by the CUDA kernels, the C++ host layer and the C ABI.
#pragma once

#include <cstdint>
#include <cstddef>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace idc {

// Text returned by idc_last_error_message() on the calling thread (abi.cpp), for entry points that
// report errors outside the context-based ABI layer.
void set_last_error(const std::string &msg);

// Device-side error codes written to the context's error word.
enum DeviceError : int {
    kDevOk = 0,
    kDevTimeout = 1,        // a bounded spin on another CTA's progress flag ran out
};

// One unit of work of the persistent wavefront kernel: R consecutive rows (in sweep order) of one
// quadrant, for a chunk of that quadrant's ordinates, swept across all columns.  `dep` is the item
// that owns the R rows just upwind in y (same quadrant and chunk, previous row block), or -1.
struct SweepItem {
    int quadrant;
    int q_begin;
    int q_count;
    int row_block;
    int dep;
    int problem;   // batched modal launch: index into the launch's problem table (0 otherwise)
    int local;     // batched modal launch: the item's index within its problem (trace buffer and moment
                   // slot; `dep` is then a local index too)
};

struct SweepArgs {
    const double *src;         // angular source (read); ghost cells carry the inflow values.  Warp and modal
                               // kernels: null means zero source and vacuum inflow
    const double *src2;        // modal forward sweep: a second angular source added to src as
    double src2_scale;         // fma(src2_scale, src2, src) on interior cells (null: none)
    const double *inflow;      // modal kernel: inflow traces of the ghost cells [nx + ny][nq][P], or null
    double *out;               // psi (written); may equal src (in-place sweep).  Warp kernel: null = not stored
    const double *sigma_t;     // (nx+2)(ny+2), piecewise constant
    const double *sigma_s;     // (nx+2)(ny+2) or null: fused isotropic scattering source (elimination kernels)
    const double *sigma_t_mat; // high-order cross sections (warp kernel, FP64): per cell the N x N term of CalcA,
                               // dx dy / 4 (2d+1)(2e+1) T(d,e; u,v), added to the cell matrix; null: sigma_t per cell
    const double *phi_scatter; // fused scattering source, or null.  Elimination kernels: phi (scaled by sigma_s
                               // / (4 pi) in the kernel).  Modal forward sweep: the per-cell moments
                               // sigma_s phi / (4 pi) of launch_scatter_moments.  Transposed modal sweep: mu
    double *phi;               // fused moment output (atomically accumulated, pre-zeroed), or null
    double *phi_part;          // warp kernel: per-chunk partial moments [phi_slots][stride], or null
    int phi_slots;             // warp kernel: ordinate chunks per row block (items per row block)
    size_t phi_slot_stride;    // warp kernel: doubles per partial-moment slot = (nx+2)(ny+2)N
    const double *xi, *eta, *w;
    int nx, ny, nq;
    double dx, dy, inv_dt;
    double scatter_scale;      // multiplies sigma_s*phi/(4 pi) in the fused source
    const SweepItem *items;
    int n_items;
    int R;                     // rows per item
    int G;                     // ordinate slots per CTA (>= every item's q_count)
    int n_refine;              // FP64 refinement steps of the FP32 cell solve
    int seg;                   // warp kernel: lanes per row segment (power of two >= G); rows per warp = 32/seg
    int wn;                    // warp kernel: compute warps per CTA (rows per CTA = wn * 32/seg)
    double *trace;             // warp / modal kernel: per-item last-row traces [n_items][nx][G][V], V = N (warp)
                               // or P (modal), sentinel-armed
    size_t trace_stride;       // doubles per item in `trace` = nx * G * V
    int *progress;             // per item: columns finished by its last row
    int *next_item;            // dynamic work queue head
    int *error;                // device error word
    long long spin_limit;      // polls before a wait gives up
    int adjoint;               // modal kernel: 1 = transposed sweep (reverse order; phi_scatter is mu and the
                               // fused source is w_q mu; the moments are unweighted sums over ordinates)
    int skip;                  // batched modal launch: 1 = this problem is not swept this time (its items return
                               // at once; nothing of it is read or written)
    int quad_mask;             // lane kernel: quadrants swept by this launch (bit k = quadrant k), 0 = all; items of
                               // the others return at once (reflecting boundaries sweep the quadrants in sequence)
    const double *modal_src;   // lane kernel, moments-only forward sweeps: the packed modal source of every
                               // (cell, quadrant), [(nx+2)(ny+2)][4][N] (launch_modal_sources), or null; the
                               // partial moments are then packed modal sums (launch_reduce_modal_partials)
};

// Launch geometry picked by the host (autotuner or defaults).
struct SweepTiling {
    int G = 0;   // ordinates per CTA
    int R = 0;   // rows per CTA
};

// Kernel launchers (sweep_kernels.cu).  `precision` is one of the IDC_PREC_* values.
cudaError_t launch_sweep(int P, int precision, const SweepArgs &args, int grid, int block, size_t smem,
                         cudaStream_t stream);
cudaError_t sweep_occupancy(int P, int precision, int block, size_t smem, int *blocks_per_sm);
size_t sweep_smem_bytes(int P, int R, int G);

// Warp-pipelined sweep kernel (sweep_warp.cu): same arguments, with seg/wn set and R = wn * 32/seg.
cudaError_t launch_sweep_warp(int P, int precision, const SweepArgs &args, int grid, size_t smem, cudaStream_t stream);
cudaError_t sweep_warp_occupancy(int P, int precision, int threads, size_t smem, int *blocks_per_sm);
size_t sweep_warp_smem_bytes(int P, int wn, int G, int seg);
constexpr int kWarpRingSlots = 8;
constexpr int kModalSolutionSlots = 4;   // modal kernel: step results in flight per compute warp

// Lane-pipelined sweep kernel (sweep_lane.cu): every warp an independent worker on one item of 32/seg rows
// (R = 32/seg, G <= seg); FP64 forward (optionally with src2), transposed or moments-only, and FP32
// (IDC_PREC_FP32) forward or moments-only sweeps; `grid` thread blocks of
// sweep_lane_warps() warps.  Same arguments and trace protocol as the modal kernel.
bool sweep_lane_supports(int P, int precision, int seg);
int sweep_lane_warps();
// A batch's FP64 forward sweep on the lane kernel: the items of several problems of one DG degree (`table`:
// one SweepArgs per problem on the device; items name their problem and carry problem-local indices)
cudaError_t launch_sweep_lane_batched(int P, const SweepArgs &args, const SweepArgs *table, int grid,
                                      cudaStream_t stream);
cudaError_t sweep_lane_batched_occupancy(int P, int seg, int *blocks_per_sm);
cudaError_t launch_sweep_lane(int P, int precision, const SweepArgs &args, int grid, cudaStream_t stream);
cudaError_t sweep_lane_occupancy(int P, int seg, bool src2, int *blocks_per_sm);

// Modal sweep kernel (sweep_modal.cu): same arguments as the warp kernel plus `inflow`, traces of P values.
cudaError_t launch_sweep_modal(int P, int precision, const SweepArgs &args, int grid, size_t smem, cudaStream_t stream);
// Batched modal launch: one persistent kernel over the items of several problems of the same degree P.
// `launch` carries the shared item list, queue head, error word and tile shape (G, seg, wn); `table`
// (device) holds one SweepArgs per problem (its arrays, sizes, trace buffer); items carry their problem
// and problem-local index.  Forward sweeps,
// FP64 or refined precision.
cudaError_t launch_sweep_modal_batched(int P, int precision, const SweepArgs &launch, const SweepArgs *table, int grid,
                                       size_t smem, cudaStream_t stream);
// The batched launch's helpers, one launch each for all `members` problems of the table: inflow traces
// (into each problem's `inflow` from its `src`, packed modal if modal_inflow) and the moment reduction
// (each problem's `phi_part` slots into its `phi`).
cudaError_t launch_batched_helpers(int P, bool modal_inflow, const SweepArgs *table, int members, bool inflow,
                                   bool reduce, cudaStream_t stream);
cudaError_t sweep_modal_occupancy(int P, int precision, int seg, int threads, size_t smem, int *blocks_per_sm);
size_t sweep_modal_smem_bytes(int P, int precision, int wn, int G, int seg);
// shared memory a launch with a second source (SweepArgs::src2) adds to sweep_modal_smem_bytes
size_t sweep_modal_src2_bytes(int P, int wn);
// Modal kernel CTA shape: wn compute warps, one helper warp and one or two aux warps per compute warp;
// at most sweep_modal_max_wn(P) compute warps (the register file holds one CTA).  fit_wn: the largest
// wn <= the given one whose shared memory fits the device.
int sweep_modal_max_wn(int P);
int sweep_modal_default_wn(int P);
int sweep_modal_threads(int P, int wn);
int sweep_modal_fit_wn(int P, int precision, int wn, int G, int seg);
// Inflow traces of the ghost cells of `src` for the modal kernel: out[(k * nq + q) * P + m], k < nx the
// ghost row below column k, k >= nx the ghost column left of row k - nx (sweep order); packed modal
// coefficients if `modal`, else sign-flipped physical traces.
cudaError_t launch_inflow_traces(int P, bool modal, const double *src, const double *xi, const double *eta, int nx,
                                 int ny, int nq, double *out, cudaStream_t stream);
// Bit pattern of an unwritten trace slot: a signalling-NaN payload that floating-point arithmetic never
// produces (arithmetic returns quiet NaNs).
constexpr unsigned long long kTraceSentinel = 0x7FF4DEADBEEFCAFEull;
cudaError_t launch_fill_u64(unsigned long long *p, size_t n, unsigned long long value, cudaStream_t s);

// Operator kernels (ops_kernels.cu).
struct GridDims {
    int nx, ny, nq, P;
    double dx, dy;
};
// Moments-only forward sweeps (no source array, psi not stored) on the lane kernel: the source of a cell is
// the isotropic scattering source, the same for every ordinate of a quadrant, so its packed modal transform
// is formed once per (cell, quadrant): out[(cell * 4 + k) * N + m] = W flip_k(scale * moments) W^T (moments
// = sigma_s phi / (4 pi) of launch_scatter_moments, null for none).  The sweep then sums w_q Z in the packed
// basis per ordinate chunk, and the reduction transforms each quadrant's sum back once per cell:
// phi = sum_k flip_k(V (sum_{slots of k} part) V^T), slots [slot_begin[k], slot_begin[k+1]) of quadrant k,
// interior cells in a fixed order, ghost cells zero.
cudaError_t launch_modal_sources(const GridDims &g, const double *moments, double scale, double *out, cudaStream_t s);
cudaError_t launch_reduce_modal_partials(const GridDims &g, const double *part, const int slot_begin[5], size_t stride,
                                         double *phi, cudaStream_t s);
cudaError_t launch_pmv(const GridDims &g, double alpha, double beta, const double *w, const double *psi,
                       double *phi, cudaStream_t s);
cudaError_t launch_smv(const GridDims &g, double alpha, double beta, const double *sigma_s, const double *phi,
                       double *psi, cudaStream_t s);
// y = beta y + alpha L x (+ gamma sigma_s phi_sc / (4 pi) when phi_sc is given: Lmv and Smv in one pass).
// tensor_t / tensor_s (high-order cross sections): the per-cell tensors T of launch_sigma_tensor take the place
// of sigma_t / sigma_s (the reference's sigma.DG_degree > 0 branches)
cudaError_t launch_lmv(const GridDims &g, double alpha, double beta, const double *sigma_t, const double *xi,
                       const double *eta, const double *x, double *y, cudaStream_t s, double gamma = 0.0,
                       const double *sigma_s = nullptr, const double *phi_sc = nullptr,
                       const double *tensor_t = nullptr, const double *tensor_s = nullptr);

// High-order cross sections (the reference's CrossSection with DG_degree = p, objects/RKDG/CrossSection.cpp).
// tpi[a + P (b + P c)] = integral over [-1, 1] of P_a P_b P_c (Global::TPI, utils/global.cpp:67-110).
struct TripleProducts {
    double v[64];   // P <= 4
};
// Per cell (ghost cells included) from the Legendre moments mom[cell][u][v]: avg[cell] = mom(0, 0) (the cell
// average), tensor[cell][r][c] = T(d,e; u,v) = sum_{m,n} mom(m,n) TPI(d,u,m) TPI(e,v,n) (CrossSection::
// ComputeTensor, :141-230), r = e + P d, c = v + P u, and, when cat is given, cat[cell][r][c] =
// dxdy4 (2d+1)(2e+1) T(d,e; u,v), the cell-matrix term of CalcA (SweepLinearSolveSpec.cpp:298-318).
cudaError_t launch_sigma_tensor(const GridDims &g, const double *mom, const TripleProducts &tpi, double dxdy4,
                                double *avg, double *tensor, double *cat, cudaStream_t s);
// psi(q,i,j,(d,e)) = beta psi + alpha (2d+1)(2e+1)/(16 pi) sum_{u,v} T(d,e; u,v) phi(u,v) on interior cells:
// TransportOperator::Smv with sigma.DG_degree > 0 (operators/RKDG/TransportOperator.cpp:367-386)
cudaError_t launch_smv_tensor(const GridDims &g, double alpha, double beta, const double *tensor_s,
                              const double *phi, double *psi, cudaStream_t s);
// y = beta y + alpha L^T x on interior cells (+ gamma w_q sigma_s zsum / (4 pi) when zsum = sum_q x_q is given:
// gamma = -1 gives (L - S P)^T x); ghost cells of x are not read as unknowns, ghost cells of y not written
cudaError_t launch_lmv_transpose(const GridDims &g, double alpha, double beta, const double *sigma_t, const double *xi,
                                 const double *eta, const double *w, const double *x, double *y, cudaStream_t s,
                                 double gamma = 0.0, const double *sigma_s = nullptr, const double *zsum = nullptr);
// out = w_q m on interior cells (P^T of a moment array as an angular array); ghost cells of out not written
cudaError_t launch_weighted_broadcast(const GridDims &g, const double *w, const double *m, double *out,
                                     cudaStream_t s);
// Reflecting boundaries (OrdinateFlux::ReflectBoundaries, objects/RKDG/OrdinateFlux.cpp:1181-1415): for each
// reflecting edge in `mask` (1 x-min, 2 x-max, 4 y-min, 8 y-max), the ghost cells of the ordinates entering
// through it (at y-max, of every ordinate, as the reference's loop) take the first interior cell's values of
// their reflected ordinate (rmap[q] for x, rmap[nq + q] for y) with the mirrored Legendre modes' signs, (-1)^d
// (x) or (-1)^e (y)
cudaError_t launch_reflect_boundaries(const GridDims &g, int mask, const double *xi, const double *eta,
                                      const int *rmap, double *psi, cudaStream_t s);
// Periodic boundaries (DensityFunction::SynchronizeHalos with Global::periodic, objects/Abstract/
// DensityFunction.cpp:927-960): every value of the edge cells' ghosts from the opposite interior edge,
// (0, j) <- (nx, j), (nx+1, j) <- (1, j), (i, 0) <- (i, ny), (i, ny+1) <- (i, 1); corner cells untouched.
cudaError_t launch_periodic_halos(const GridDims &g, double *psi, cudaStream_t s);
// dst <- src on interior cells only (Copy over OpDomain::Interior); ghost cells of dst untouched
cudaError_t launch_copy_interior(const GridDims &g, const double *src, double *dst, cudaStream_t s);
// The ghost values of the reflecting edges' entering ordinates, packed edge after edge (x-min, x-max, y-min, y-max
// of `mask`), each edge [cell][q][dof]; the entries of ordinates leaving through an edge are 0 in the pack.
// to_packed: packed <- ghosts; else ghosts <- packed (0 for leaving ordinates, and for all when packed is null).
size_t reflect_ghost_len(const GridDims &g, int mask);
cudaError_t launch_reflect_ghosts(const GridDims &g, int mask, const double *xi, const double *eta, double *psi,
                                  double *packed, bool to_packed, cudaStream_t s);
cudaError_t launch_zero_ghost_phi(const GridDims &g, double *phi, cudaStream_t s);
// out = sigma_s phi / (4 pi) per interior cell and moment (the isotropic scattering source of Smv, formed once
// per cell for the modal sweep's fused source; ghost cells of out are not written)
cudaError_t launch_scatter_moments(const GridDims &g, const double *sigma_s, const double *phi, double *out,
                                   cudaStream_t s);
// phi = sum over `slots` partial-moment arrays (interior cells, fixed order); ghost cells of phi zeroed
cudaError_t launch_reduce_phi_partials(const GridDims &g, const double *part, int slots, size_t stride, double *phi,
                                       cudaStream_t s);
// Krylov helpers on flat FP64 vectors of length n (device pointers; `out` arrays are device memory)
// out[k] = V_k . w for k < nv (<= 64), in a fixed order; scratch holds multidot_scratch_doubles() doubles
size_t multidot_scratch_doubles();
cudaError_t launch_multidot(const double *V, int nv, size_t ld, const double *w, size_t n, double *out, double *scratch,
                            cudaStream_t s);
cudaError_t launch_multiaxpy(double *w, const double *V, int nv, size_t ld, const double *c, size_t n, cudaStream_t s);
cudaError_t launch_axpby(double a, const double *x, double b, double *y, size_t n, cudaStream_t s);
cudaError_t launch_dot(const double *x, const double *y, size_t n, double *out, double *scratch, cudaStream_t s);
// adjoint Peierls operator: y = x - sigma_s/(4 pi) lam on interior cells, y = x on ghost cells
cudaError_t launch_adjoint_scatter(const GridDims &g, const double *sigma_s, const double *x, const double *lam,
                                   double *y, cudaStream_t s);
// per-cell gradients of J = c . phi from the forward psi, phi and the adjoint lam, Lam = sum_q lam_q
// (outputs on the halo layouts, interior cells written, any of them nullable)
// (scale multiplies every contribution: -1 for the gradient terms of an explicitly applied operator, e.g.
// the IDC residuals, whose sensitivity enters with the opposite sign of a solve's)
cudaError_t launch_adjoint_gradient(const GridDims &g, const double *psi, const double *lam, const double *phi,
                                    const double *Lam, double *dsig_t, double *dsig_s, double *dq, cudaStream_t s,
                                    bool accumulate = false, double scale = 1.0);
// IDC (ops_kernels.cu): out = sum_k c_k A_k + Q on interior cells, Q on ghost cells (Q nullable = 0)
struct IdcTerms {
    static constexpr int kMax = 10;
    int n;
    const double *a[kMax];
    double c[kMax];
};
cudaError_t launch_idc_source(const GridDims &g, const IdcTerms &t, const double *Q, double *out, cudaStream_t s);
// One IDC correction level's sources but their psi_{n-1} / (h dt) terms: out[n] = Q + sum_l c[n][l] (L - S P)
// stage[l] on interior cells, n = 1 .. M-1, for M nodes (2 .. kIdcFusedMaxNodes); scat[l] =
// sigma_s P stage[l] / (4 pi) per cell (launch_scatter_moments)
constexpr int kIdcFusedMaxNodes = 5;
struct IdcCorr {
    const double *Q;
    const double *stage[kIdcFusedMaxNodes];
    const double *scat[kIdcFusedMaxNodes];
    double *out[kIdcFusedMaxNodes];
    double c[kIdcFusedMaxNodes][kIdcFusedMaxNodes];
};
cudaError_t launch_idc_corrections(const GridDims &g, int M, const IdcCorr &t, const double *sigma_t, const double *xi,
                                   const double *eta, cudaStream_t s);
cudaError_t launch_phi_combine(size_t n, const double *a, const double *b, const double *c, double *out, cudaStream_t s);
// DSA preconditioner (dsa_kernels.cu): workspace size, coefficient setup from the cross sections, and
// out = v + C^{-1}(sigma_s v_00) on the (0,0) moment by cg_steps Jacobi-PCG steps (out may alias v): one
// cooperative kernel (right-hand side and steps) and the correction kernel.  The transposed preconditioner
// (for the adjoint operator) takes rhs = v_00 and corrects by sigma_s x: out = v + E sigma_s C^{-1} R v, the
// transpose of v + E C^{-1} sigma_s R v (C symmetric).  A grid barrier that gives up sets *error.
size_t dsa_workspace_doubles(int nx, int ny);
cudaError_t dsa_setup(const GridDims &g, const double *sigma_t, const double *sigma_s, double *ws, cudaStream_t s);
cudaError_t dsa_precondition(const GridDims &g, const double *sigma_s, const double *v, double *out, int cg_steps,
                             double *ws, bool transpose, int num_sms, int *error, long long spin_limit,
                             cudaStream_t s);
constexpr int kDsaLaunches = 2;
// sum over interior cells of (a - b)^2 into *out (device double), in a fixed order; scratch holds
// multidot_scratch_doubles() doubles
cudaError_t launch_l2dist2(const GridDims &g, const double *a, const double *b, double *out, double *scratch,
                           cudaStream_t s);

}  // namespace idc
