// C++ host layer: the device-resident counterpart of the reference's SweepOperator / TransportOperator /
// SISolver objects for one grid on one GPU.  The C ABI (abi.cpp) validates arguments, moves host data in
// and out, and calls these methods with device pointers.
#pragma once

#include "idc_internal.hpp"
#include "idcsweep.h"

#include <string>
#include <vector>

namespace idc {

// Status carries an IDC_* code and a message.
struct Status {
    int code = IDC_OK;
    std::string msg;
    static Status ok() { return {}; }
    bool good() const { return code == IDC_OK; }
};

Status cuda_status(cudaError_t e, const char *what);

class Context {
public:
    explicit Context(const idc_problem_desc &d);
    ~Context();
    Status init();

    // ---- configuration (SweepOperator construction / SetParameters) ----
    Status set_ordinates(int64_t nq, const double *xi, const double *eta, const double *w, const int64_t qb[5]);
    Status set_sigma(const double *sigma_t, const double *sigma_s, int loc);
    Status set_tiling(int G, int R);   // 0 = automatic
    // fixed tile shape of the modal kernel (segment width seg in {4,8,16,32}, compute warps per CTA wn),
    // set by the autotuner; 0 = the default heuristic
    Status set_tile_shape(int seg, int wn);
    // times the candidate tile shapes on this problem with `src` (device psi array) and keeps the fastest
    Status autotune(const double *src, double dt, int precision, int *seg_out, int *wn_out);

    // ---- operators on device pointers ----
    // Sweep: out <- L^{-1} (src [+ scale * S phi_scatter]); phi (nullable) <- P out.  src may equal out.
    // src2 (modal kernel, forward): the source is src + src2_scale * src2 on interior cells, combined by the
    // sweep's aux warps (or, when its stages do not fit in shared memory, by a kernel into a scratch array)
    Status sweep(const double *src, double *out, double dt, double *phi, int precision,
                 const double *phi_scatter = nullptr, double scatter_scale = 1.0, bool adjoint = false,
                 const double *src2 = nullptr, double src2_scale = 0.0);
    // count out-of-place sweeps of HOST arrays (srcs[k] -> outs[k] interior cells, phis[k] if phis), the
    // upload of step k+1, the sweep of step k and the download of step k-1 overlapped on three streams
    // with double-buffered device arrays
    Status sweep_host_many(int64_t count, const double *const *srcs, double *const *outs, double *const *phis,
                           double dt, int precision);
    cudaError_t copy_interior_d2h(double *host, const double *dev, cudaStream_t s) const;
    Status pmv(double alpha, double beta, const double *psi, double *phi);
    Status smv(double alpha, double beta, const double *phi, double *psi);
    Status lmv(double alpha, double beta, const double *x, double *y);
    Status transport_residual(const double *psi, const double *phi, double *res);   // (L - S P) psi, phi = P psi
    Status l2dist(const double *a, const double *b, double *out_host);
    Status source_iteration(const double *src, double *psi_out, double dt, double abs_tol, int64_t max_its,
                            int precision, int64_t *iters, double *err);
    // phi_guess (optional, moment-sized, device): GMRES starts from it instead of zero (reflecting or periodic
    // edges and IDC_PREC_FP32_IR start from zero)
    Status gmres_peierls(const double *src, double *psi_out, double dt, double abs_tol, int restart, int64_t max_its,
                         int precision, int64_t *iters, double *resid, const double *phi_guess = nullptr);
    Status apply_peierls(const double *x, double *y, double *tmp_phi, double dt, int precision);
    // precision IDC_PREC_FP32_IR of gmres_peierls: FP32 Krylov solves inside FP64 iterative refinement
    Status gmres_peierls_ir(const double *src, double *psi_out, double dt, double abs_tol, int restart,
                            int64_t max_its, int64_t *iters, double *resid);
    int ir_corrections = 0;   // corrections (FP64 residual sweeps) of the last refined solve
    // GMRES(restart) from x = 0 on A x = b for an operator on moment-sized vectors; *converged reports
    // whether the residual reached abs_tol (the caller decides whether that is an error)
    // whether the residual reached abs_tol (the caller decides whether that is an error).  n_extra unknowns
    // follow the moments in every vector (the reflecting edges' ghost values); the preconditioner leaves them.
    template <typename Op>
    Status gmres(Op apply, const double *b, double *x, double abs_tol, int restart, int64_t max_its, int64_t *iters,
                 double *resid, bool *converged, int dsa_mode = 0,   // 0 none, 1 DSA, 2 transposed DSA
                 size_t n_extra = 0, bool warm = false);   // warm: x holds the initial guess
    Status set_preconditioner(int kind, int inner_steps);   // 0 none, 1 DSA
    // IDC time integration (idc.cpp): psi (device, in/out) advanced `steps` steps of size dt with M
    // Gauss-Lobatto nodes and K corrections; scattering 0 = explicit (IMEX, one sweep per substep, CUDA
    // graph when use_graph), 1 = implicit (GMRES per substep)
    Status idc_integrate(double *psi, const double *Q, double dt, int64_t steps, int M, int K, int scattering,
                         int precision, double abs_tol, int restart, int64_t max_its, bool use_graph,
                         int64_t *sweeps);
    // transposed (adjoint) problem: (L - S P)^T lam = P^T c, via (I - S^T L^{-T} P^T) mu = c
    Status apply_peierls_adjoint(const double *x, double *y, double *tmp_phi, double dt, int precision);
    Status adjoint_solve(const double *detector, double *lam_out, double *Lam_out, double dt, double abs_tol,
                         int restart, int64_t max_its, int precision, int64_t *iters, double *resid);
    Status adjoint_gradient(const double *psi, const double *detector, double dt, double abs_tol, int restart,
                            int64_t max_its, int precision, double *dsig_t, double *dsig_s, double *dq,
                            int64_t *iters, double *resid);
    // (L' - S P)^T lam = b for a psi-sized b (interior cells): with nu = S^T lam, (I - S^T L'^{-T} P^T) nu =
    // S^T L'^{-T} b by GMRES, then lam = L'^{-T} (b + P^T nu); Lam_out = sum_q lam_q
    Status adjoint_solve_psi(const double *b, double *lam_out, double *Lam_out, double dt, double abs_tol, int restart,
                             int64_t max_its, int precision, int64_t *iters);
    // gradients of J = c . P psi^steps for implicit-Euler steps (1/dt + L - S P) psi^{n+1} = psi^n / dt + Q
    // (device arrays), states kept every `checkpoint_every` steps and recomputed segment by segment
    Status adjoint_transient(const double *psi0, const double *Q, double dt, int64_t steps, const double *detector,
                             int64_t checkpoint_every, double abs_tol, int restart, int64_t max_its, int precision,
                             double *dsig_t, double *dsig_s, double *dq, double *dpsi0, double *J, int64_t *solves);
    // gradients of J = c . P psi^steps for implicit-scattering IDC steps (idc_integrate with scattering 1: M
    // Gauss-Lobatto nodes, K corrections, update form), the same checkpointing
    Status adjoint_idc(const double *psi0, const double *Q, double dt, int64_t steps, int M, int K,
                       const double *detector, int64_t checkpoint_every, double abs_tol, int restart, int64_t max_its,
                       int precision, double *dsig_t, double *dsig_s, double *dq, double *dpsi0, double *J,
                       int64_t *solves);
    // y = (L - S P)^T z on interior cells (the transpose of transport_residual); zsum: a moment-sized scratch
    Status transport_residual_transpose(const double *z, double *y, double *zsum);
    Status lmv_transpose(double alpha, double beta, const double *x, double *y);   // y = beta y + alpha L^T x
    Status dot_host(const double *x, const double *y, size_t n, double *out);

    // ---- buffers ----
    Status ensure_psi_buffers(int count);   // device scratch psi-sized buffers
    Status ensure_phi_buffers(int count);
    double *psi_buf(int k) { return psi_bufs_[k]; }
    double *phi_buf(int k) { return phi_bufs_[k]; }
    Status check_device_error();   // reads and clears the device error word

    size_t psi_len() const { return (size_t)(nx + 2) * (ny + 2) * (size_t)nq * N; }
    size_t phi_len() const { return (size_t)(nx + 2) * (ny + 2) * (size_t)N; }
    size_t sig_len() const { return (size_t)(nx + 2) * (ny + 2); }
    GridDims dims() const { return GridDims{(int)nx, (int)ny, (int)nq, P, dx, dy}; }

    idc_problem_desc desc;
    int64_t nx = 0, ny = 0;
    int P = 0, N = 0;
    double dx = 0, dy = 0;
    int device = 0;
    int num_sms = 0;
    int lane_src2_blocks_[2] = {-1, -1};   // resident blocks per SM of the lane kernel's second-source
                                           // instance at DG degree 1, segments 8 and 4 (-1: not queried yet)
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    int64_t nq = 0;
    int64_t quad[5] = {0, 0, 0, 0, 0};
    double *d_xi = nullptr, *d_eta = nullptr, *d_w = nullptr;
    double *d_sigma_t = nullptr, *d_sigma_s = nullptr;
    bool have_ordinates = false, have_sigma = false;
    // high-order cross sections (desc.sigma_degree = p): d_sigma_t / d_sigma_s hold the cell averages (the DSA
    // preconditioner's coefficients); the operators use the tensors T (launch_sigma_tensor) and CalcA's term
    bool high_order_sigma() const { return desc.sigma_degree > 0; }
    double *d_sig_mom_ = nullptr;                               // staging of one set of moments
    double *d_tens_t_ = nullptr, *d_tens_s_ = nullptr, *d_cat_t_ = nullptr;
    double *d_work_psi_ = nullptr;   // psi-sized array in which a sweep's scattering source is formed
    Status sweep_tensor_source(const double *src, double *out, double dt, double *phi, int precision,
                               const double *phi_scatter, double scatter_scale);

    // sweep schedule
    SweepTiling tiling;
    int user_G = 0, user_R = 0;
    int tune_seg = 0, tune_wn = 0;
    SweepItem *d_items = nullptr;
    int n_items = 0;
    int *d_sync = nullptr;        // [0] queue head, [1] error word, [2..] progress per item
    // sweep kernel: lane-pipelined (sweep_lane.cu, default; FP64 sweeps), modal (sweep_modal.cu; every
    // precision, and the FP32 modes when kLane is selected), warp-pipelined with elimination (sweep_warp.cu)
    // or row-synchronous (sweep_kernels.cu)
    enum Kernel { kRowSync = 0, kWarp = 1, kModal = 2, kLane = 3 };
    int kernel = kLane;
    int active = kLane;            // the kernel the current schedule was built for (kernel_for(precision))
    bool use_warp_kernel = true;   // kernel is kWarp, kModal or kLane (same trace protocol)
    // the modal cell arithmetic (modal or lane kernel): the transposed sweep, IDC, batches
    // the lane and modal kernels (their cell arithmetic diagonalises a Kronecker cell matrix): DG degree <= 2,
    // piecewise-constant cross sections
    bool modal_family() const { return (kernel == kModal || kernel == kLane) && P <= 3 && !high_order_sigma(); }
    int kernel_for(int precision) const;
    int seg = 0, wn = 0;           // warp kernel tiling
    double *d_trace = nullptr;     // warp / modal kernel: per-item last-row traces (sentinel-armed)
    double *d_inflow = nullptr;    // modal kernel: inflow traces of the ghost cells
    size_t inflow_len = 0;
    double *d_scat = nullptr;      // modal kernel: the fused scattering source's moments sigma_s phi / (4 pi)
    size_t scat_len = 0;
    double *d_src2mix = nullptr;   // src + scale src2 when the second source's stages do not fit
    double *d_msrc = nullptr;      // lane kernel, moments-only sweeps: packed modal sources [(nx+2)(ny+2)][4][N]
    size_t msrc_len = 0;
    bool moments_fast_path = true;
    int quad_slots[5] = {0, 0, 0, 0, 0};   // partial-moment slots of each quadrant within a row block
    size_t src2mix_len = 0;
    size_t trace_len = 0;
    int items_per_rb = 0;          // work items per row block (= ordinate chunks over all quadrants)
    double *d_phi_part = nullptr;  // warp kernel: per-chunk partial moments
    size_t phi_part_len = 0;
    int grid = 0, block = 0;
    size_t smem = 0;
    int occupancy_precision = -1;
    size_t sync_cap_ = 0;          // ints allocated at d_sync (shared by both schedules below)
    // Two cached schedules, one per sweep variant: 0 = sweeps with a source or a psi output, 1 = the moments-only
    // Krylov sweeps (no source, psi not stored).  They want different tile widths (the full lane sweep at DG
    // degree 2 is fastest with 16-wide segments, the moments-only one with narrow ones), and GMRES alternates
    // between them, so the members above hold the current variant's schedule and `other_sched_` the other's;
    // `use_schedule` swaps them.  d_sync (the error word and progress flags) is shared.
    struct ScheduleSlot {
        SweepTiling tiling{};
        SweepItem *d_items = nullptr;
        double *d_trace = nullptr;
        size_t trace_len = 0, smem = 0;
        int n_items = 0, items_per_rb = 0, quad_slots[5] = {0, 0, 0, 0, 0}, seg = 0, wn = 0, active = 3, grid = 0,
            block = 0, occupancy_precision = -1;
    };
    ScheduleSlot other_sched_;
    int sched_variant_ = 0;
    void use_schedule(int variant);
    void invalidate_schedules() {
        n_items = 0;
        occupancy_precision = -1;
        other_sched_.n_items = 0;
        other_sched_.occupancy_precision = -1;
    }

    float last_sweep_ms = 0.f;
    bool capturing = false;   // a CUDA graph capture is open on `stream`: no timing events, no host syncs
    int64_t launches = 0;
    static constexpr long long kDefaultSpinLimit = 1ll << 22;
    long long spin_limit = kDefaultSpinLimit;   // polls before a device-side wait gives up (idc_set_spin_limit)
    // ordinate-partitioned solves: sums every moment output of a sweep over the ranks, in place (device memory);
    // 0 on success (idc_set_allreduce)
    int (*allreduce_fn)(double *data, int64_t n, void *user) = nullptr;
    void *allreduce_user = nullptr;
    // reflecting boundaries (idc_set_reflecting): the reference's BoundaryEdge bits, the reflection partners
    // [2][nq] on the device, and the state of a sequential-quadrant sweep in progress
    int reflect_mask = 0;
    int *d_rmap = nullptr;
    int quad_mask_ = 0;
    bool skip_reduce_ = false, in_reflect_ = false;
    double *d_reflect_ = nullptr;   // psi-sized work array of reflecting sweeps that return no psi
    double *d_reflect_g_ = nullptr;  // the reflecting edges' ghost values, packed (source iteration)
    size_t reflect_g_len_ = 0;
    double *d_reflect_vec_ = nullptr;   // GMRES vectors [moments; packed ghost values]: b, x, work
    size_t reflect_vec_len_ = 0;
    Status set_reflecting(int mask);
    Status update_reflect_map();
    Status sweep_reflecting(const double *src, double *out, double dt, double *phi, int precision,
                            const double *phi_scatter, double scatter_scale, bool adjoint, const double *src2);
    Status reflect_quadrants(double *w, double dt, double *phi, int precision);
    Status reflect_ghosts(double *psi, double *packed, bool to_packed);
    Status source_iteration_reflecting(const double *src, double *psi_out, double dt, double abs_tol,
                                       int64_t max_its, int precision, int64_t *iters, double *err);
    // periodic boundaries (idc_set_periodic, the reference's Global::periodic): the sweep reads the ghost
    // cells as given; source iteration and GMRES carry them from the opposite edges between sweeps
    bool periodic_ = false;
    Status set_periodic(bool on);
    Status source_iteration_periodic(const double *src, double *psi_out, double dt, double abs_tol,
                                     int64_t max_its, int precision, int64_t *iters, double *err);
    // edges whose ghost values the solvers carry: the reflecting ones, or all four when periodic
    int ghost_mask() const { return periodic_ ? 15 : reflect_mask; }
    Status boundary_sweep(double *w, double dt, double *phi, int precision);
    Status apply_peierls_boundary(const double *x, double *y, double *tmp, double dt, int precision);
    Status gmres_peierls_boundary(const double *src, double *psi_out, double dt, double abs_tol, int restart,
                                  int64_t max_its, int precision, int64_t *iters, double *resid);

    double *d_krylov = nullptr;    // GMRES basis, (restart + 1) phi-sized vectors (+ restart for flexible GMRES)
    int precond_kind = 0;          // 0 none, 1 DSA (right preconditioner of the forward Peierls GMRES)
    int dsa_steps = 30;            // Jacobi-PCG steps per DSA application
    double *d_dsa_ws = nullptr;    // DSA workspace
    size_t dsa_ws_len = 0;
    cudaStream_t copy_in = nullptr, copy_out = nullptr;   // sweep_host_many's copy streams
    cudaEvent_t ev_in[2] = {}, ev_done[2] = {}, ev_out[2] = {};
    size_t krylov_len = 0;
    double *d_small = nullptr;     // GMRES Hessenberg column / coefficients (device)
    double *h_small = nullptr;     // GMRES: pinned host copy of the column, the new vector's norm and the error
                                   // word (one copy and one synchronisation per Arnoldi step)

private:
    Status build_schedule(int precision);
    std::vector<double *> psi_bufs_, phi_bufs_;
    std::vector<double *> transient_bufs_;   // adjoint_transient: checkpoints, segment states, lam, b, source
    std::vector<double *> adj_idc_bufs_;    // adjoint_idc: checkpoints, step inputs, stages, adjoint states
    double *d_ones_ = nullptr;              // nq ones: unweighted moment sums through the Pmv kernel
    std::vector<double *> idc_psi_, idc_phi_;
    double *d_scalar_ = nullptr;
};

}  // namespace idc
