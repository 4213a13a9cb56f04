// Krylov solver on the GPU: the reference's Peierls-form GMRES (PETScPeierlsSolver,
// linear_solvers/Abstract/ImplicitSolver/PETScPeierlsSolver.cpp:423-572) with the operator application
// done by the fused sweep and the Arnoldi process, Hessenberg least squares and all vectors in FP64.
#include "context.hpp"

#include <algorithm>
#include <cstring>
#include <cmath>
#include <vector>

namespace idc {

#define IDC_TRY_CUDA(expr)                                    \
    do {                                                      \
        cudaError_t e_ = (expr);                              \
        if (e_ != cudaSuccess) return cuda_status(e_, #expr); \
    } while (0)

#define IDC_TRY(expr)              \
    do {                           \
        Status s_ = (expr);        \
        if (!s_.good()) return s_; \
    } while (0)

namespace {

Status bad(int code, const std::string &m) {
    Status s;
    s.code = code;
    s.msg = m;
    return s;
}

}  // namespace

Status Context::dot_host(const double *x, const double *y, size_t n, double *out) {
    IDC_TRY_CUDA(launch_dot(x, y, n, d_scalar_, d_scalar_ + 4, stream));
    launches += 2;
    IDC_TRY_CUDA(cudaMemcpyAsync(out, d_scalar_, sizeof(double), cudaMemcpyDeviceToHost, stream));
    IDC_TRY_CUDA(cudaStreamSynchronize(stream));
    return Status::ok();
}

// y = x - P L^{-1} S x  (IPLS, PETScPeierlsSolver.cpp:529-572): one sweep with no angular source and
// vacuum inflow, the scattering source built from x on the fly, psi not stored.
Status Context::apply_peierls(const double *x, double *y, double *tmp_phi, double dt, int precision) {
    IDC_TRY(sweep(nullptr, nullptr, dt, tmp_phi, precision, x, 1.0));
    IDC_TRY_CUDA(launch_axpby(1.0, x, 0.0, y, phi_len(), stream));
    IDC_TRY_CUDA(launch_axpby(-1.0, tmp_phi, 1.0, y, phi_len(), stream));
    launches += 2;
    return Status::ok();
}

// GMRES(restart) from a zero initial guess on A x = b (moment-sized vectors), stopping when the residual
// 2-norm (the Arnoldi estimate, as PETSc reports it) is <= abs_tol.  Classical Gram-Schmidt with one
// re-orthogonalisation pass (CGS2), Givens rotations on the host, restarts from the true residual.
// PETSc's LGMRES adds error-approximation vectors to the restart; it converges to the same solution, so
// iteration counts may differ but the solution does not.  With `dsa`, flexible GMRES with the DSA right
// preconditioner M: the basis Z_j = M V_j is kept (M is a fixed number of CG steps, so it is not exactly
// linear) and x = Z y.
template <typename Op>
Status Context::gmres(Op apply, const double *b, double *x, double abs_tol, int restart, int64_t max_its,
                      int64_t *iters_out, double *resid_out, bool *converged_out, int dsa_mode, size_t n_extra,
                      bool warm) {
    const bool dsa = dsa_mode != 0;
    if (restart < 1 || restart > 60) return bad(IDC_ERR_ARG, "gmres restart must be in 1..60");
    const size_t n = phi_len() + n_extra;
    const int m = restart;
    const size_t need = (size_t)(dsa ? 2 * m + 1 : m + 1) * n;
    if (krylov_len < need) {
        cudaFree(d_krylov);
        d_krylov = nullptr;
        krylov_len = 0;
        IDC_TRY_CUDA(cudaMalloc(&d_krylov, sizeof(double) * need));
        krylov_len = need;
    }
    if (!d_small) IDC_TRY_CUDA(cudaMalloc(&d_small, sizeof(double) * (128 + multidot_scratch_doubles())));
    if (!h_small) IDC_TRY_CUDA(cudaMallocHost(&h_small, sizeof(double) * 129));
    double *dot_scratch = d_small + 128;
    double *V = d_krylov;
    auto Vc = [&](int k) { return V + (size_t)k * n; };
    auto Zc = [&](int k) { return V + (size_t)(m + 1 + k) * n; };
    if (dsa) {
        const size_t wl = dsa_workspace_doubles((int)nx, (int)ny);
        if (dsa_ws_len < wl) {
            cudaFree(d_dsa_ws);
            d_dsa_ws = nullptr;
            dsa_ws_len = 0;
            IDC_TRY_CUDA(cudaMalloc(&d_dsa_ws, sizeof(double) * wl));
            dsa_ws_len = wl;
        }
        IDC_TRY_CUDA(dsa_setup(dims(), d_sigma_t, d_sigma_s, d_dsa_ws, stream));
        launches += 2;
    }

    if (warm) {   // r = b - A x for the caller's initial guess
        IDC_TRY(apply(x, Vc(0)));
        IDC_TRY_CUDA(launch_axpby(1.0, b, -1.0, Vc(0), n, stream));
        launches += 1;
    } else {      // r = b - A x = b for the zero initial guess
        IDC_TRY_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
        IDC_TRY_CUDA(cudaMemcpyAsync(Vc(0), b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    }
    double beta = 0.0;
    IDC_TRY(dot_host(Vc(0), Vc(0), n, &beta));
    beta = std::sqrt(beta);

    std::vector<double> H((size_t)(m + 1) * m, 0.0), cs(m), sn(m), g(m + 1), yv(m);
    int64_t its = 0;
    double resid = beta;
    bool converged = resid <= abs_tol;
    while (!converged && its < max_its) {
        IDC_TRY_CUDA(launch_axpby(0.0, Vc(0), 1.0 / beta, Vc(0), n, stream));
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int k = 0;   // columns built in this cycle
        for (int j = 0; j < m && its < max_its; ++j) {
            if (dsa) {
                IDC_TRY_CUDA(dsa_precondition(dims(), d_sigma_s, Vc(j), Zc(j), dsa_steps, d_dsa_ws, dsa_mode == 2,
                                              num_sms, d_sync + 1, spin_limit, stream));
                launches += kDsaLaunches;
                if (n_extra)
                    IDC_TRY_CUDA(cudaMemcpyAsync(Zc(j) + phi_len(), Vc(j) + phi_len(), sizeof(double) * n_extra,
                                                 cudaMemcpyDeviceToDevice, stream));
                IDC_TRY(apply(Zc(j), Vc(j + 1)));
            } else {
                IDC_TRY(apply(Vc(j), Vc(j + 1)));
            }
            // CGS2: h = V^T w, w -= V h, twice; then |w|^2.  The two coefficient columns (d_small[0..], [64..]),
            // the squared norm (d_small[127]) and the device error word reach the host in one pinned copy
            // with one synchronisation.
            IDC_TRY_CUDA(launch_multidot(V, j + 1, n, Vc(j + 1), n, d_small, dot_scratch, stream));
            IDC_TRY_CUDA(launch_multiaxpy(Vc(j + 1), V, j + 1, n, d_small, n, stream));
            IDC_TRY_CUDA(launch_multidot(V, j + 1, n, Vc(j + 1), n, d_small + 64, dot_scratch, stream));
            IDC_TRY_CUDA(launch_multiaxpy(Vc(j + 1), V, j + 1, n, d_small + 64, n, stream));
            IDC_TRY_CUDA(launch_dot(Vc(j + 1), Vc(j + 1), n, d_small + 127, dot_scratch, stream));
            launches += 8;
            IDC_TRY_CUDA(cudaMemcpyAsync(h_small, d_small, sizeof(double) * 128, cudaMemcpyDeviceToHost, stream));
            IDC_TRY_CUDA(cudaMemcpyAsync(h_small + 128, d_sync + 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
            IDC_TRY_CUDA(cudaStreamSynchronize(stream));
            int dev_err = 0;
            std::memcpy(&dev_err, h_small + 128, sizeof(int));
            if (dev_err != kDevOk) IDC_TRY(check_device_error());   // re-arms the sweep state, returns the error
            double hn = std::sqrt(h_small[127]);
            for (int i = 0; i <= j; ++i) H[(size_t)i * m + j] = h_small[i] + h_small[64 + i];
            H[(size_t)(j + 1) * m + j] = hn;
            if (hn > 0.0) {
                IDC_TRY_CUDA(launch_axpby(0.0, Vc(j + 1), 1.0 / hn, Vc(j + 1), n, stream));
                launches += 1;
            }
            // apply the previous rotations to the new column, then a new one
            for (int i = 0; i < j; ++i) {
                const double a = H[(size_t)i * m + j], c = H[(size_t)(i + 1) * m + j];
                H[(size_t)i * m + j] = cs[i] * a + sn[i] * c;
                H[(size_t)(i + 1) * m + j] = -sn[i] * a + cs[i] * c;
            }
            const double a = H[(size_t)j * m + j], c = H[(size_t)(j + 1) * m + j];
            const double r = std::hypot(a, c);
            cs[j] = r > 0.0 ? a / r : 1.0;
            sn[j] = r > 0.0 ? c / r : 0.0;
            H[(size_t)j * m + j] = r;
            H[(size_t)(j + 1) * m + j] = 0.0;
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            resid = std::fabs(g[j + 1]);
            ++its;
            k = j + 1;
            if (resid <= abs_tol || hn == 0.0) break;
        }
        // y = H^{-1} g, x += V y
        for (int i = k - 1; i >= 0; --i) {
            double sum = g[i];
            for (int l = i + 1; l < k; ++l) sum -= H[(size_t)i * m + l] * yv[l];
            yv[i] = sum / H[(size_t)i * m + i];
        }
        for (int i = 0; i < k; ++i) yv[i] = -yv[i];   // multiaxpy subtracts
        IDC_TRY_CUDA(cudaMemcpyAsync(d_small, yv.data(), sizeof(double) * k, cudaMemcpyHostToDevice, stream));
        IDC_TRY_CUDA(launch_multiaxpy(x, dsa ? Zc(0) : V, k, n, d_small, n, stream));
        launches += 1;
        if (resid <= abs_tol) {
            converged = true;
            break;
        }
        // restart from the true residual r = b - A x
        IDC_TRY(apply(x, Vc(0)));
        IDC_TRY_CUDA(launch_axpby(1.0, b, -1.0, Vc(0), n, stream));
        launches += 1;
        IDC_TRY(dot_host(Vc(0), Vc(0), n, &beta));
        beta = std::sqrt(beta);
        resid = beta;
        converged = resid <= abs_tol;
        if (beta == 0.0) break;
    }
    if (iters_out) *iters_out = its;
    if (resid_out) *resid_out = resid;
    if (converged_out) *converged_out = converged;
    return Status::ok();
}

// The sweep of a prepared array w in place with the boundary treatment of source iteration: with reflecting
// edges the quadrants in sequence with the reflections between them (the reflections of the last quadrant are
// the ghost values it leaves); on a periodic grid one sweep, then the halos synchronised from the opposite edges.
Status Context::boundary_sweep(double *w, double dt, double *phi, int precision) {
    if (reflect_mask) return reflect_quadrants(w, dt, phi, precision);
    IDC_TRY(sweep(w, w, dt, phi, precision));
    IDC_TRY_CUDA(launch_periodic_halos(dims(), w, stream));
    launches += 1;
    return Status::ok();
}

// The Peierls operator with reflecting or periodic edges, on x = [phi; g], g the ghost values of those edges'
// entering ordinates at the start of a sweep (packed as launch_reflect_ghosts packs them): the boundary sweep
// of the scattering source S phi with vacuum inflow on the other edges and g on these, y = x - [P psi; g(psi)],
// g(psi) the ghost values that the sweep leaves.  Source iteration with such edges is the fixed-point iteration
// of exactly this map (the ghost values left by one sweep are the next sweep's inflow), so GMRES on it reaches
// the source-iteration fixed point.  The reference's Peierls operator (PETScPeierlsSolver.cpp:529-572) starts
// every sweep from zero ghost cells instead (Smv over OpDomain::All of a scalar flux unpacked with zero halos):
// the same solution only where one sweep needs no ghost value from the sweep before (reflecting x-min and y-min
// edges), a different one elsewhere (other reflecting edges, periodic grids).
Status Context::apply_peierls_boundary(const double *x, double *y, double *tmp, double dt, int precision) {
    const size_t np = phi_len(), n = np + reflect_ghost_len(dims(), ghost_mask());
    double *w = d_reflect_;
    IDC_TRY_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * psi_len(), stream));
    IDC_TRY(reflect_ghosts(w, const_cast<double *>(x) + np, false));
    IDC_TRY(smv(1.0, 1.0, x, w));
    IDC_TRY(boundary_sweep(w, dt, tmp, precision));
    IDC_TRY(reflect_ghosts(w, tmp + np, true));
    IDC_TRY_CUDA(launch_axpby(1.0, x, 0.0, y, n, stream));
    IDC_TRY_CUDA(launch_axpby(-1.0, tmp, 1.0, y, n, stream));
    launches += 2;
    return Status::ok();
}

// GMRES on (I - K) [phi; g] = b with K the map above and b the boundary sweep of Q (its own inflow on the other
// edges, zero ghost values on these); then psi is the boundary sweep of Q + S phi with g in those ghost cells.
Status Context::gmres_peierls_boundary(const double *src, double *psi_out, double dt, double abs_tol, int restart,
                                       int64_t max_its, int precision, int64_t *iters_out, double *resid_out) {
    if (precision == IDC_PREC_FP32_IR)
        return bad(IDC_ERR_UNSUPPORTED, "reflecting or periodic edges: GMRES with FP64 or FP32 sweeps");
    if (reflect_mask && kernel_for(precision) != kLane)
        return bad(IDC_ERR_UNSUPPORTED,
                   "reflecting boundaries need the lane kernel: FP64 or FP32 sweeps at a lane tile shape");
    if (allreduce_fn)
        return bad(IDC_ERR_UNSUPPORTED, "reflecting or periodic edges with ordinates partitioned over ranks");
    const size_t np = phi_len(), ng = reflect_ghost_len(dims(), ghost_mask()), n = np + ng;
    if (capturing && (!d_reflect_ || reflect_vec_len_ < 3 * n))
        return bad(IDC_ERR_STATE, "boundary-solve buffer allocation inside a stream capture");
    if (!d_reflect_) IDC_TRY_CUDA(cudaMalloc(&d_reflect_, sizeof(double) * psi_len()));
    if (reflect_vec_len_ < 3 * n) {
        cudaFree(d_reflect_vec_);
        d_reflect_vec_ = nullptr;
        reflect_vec_len_ = 0;
        IDC_TRY_CUDA(cudaMalloc(&d_reflect_vec_, sizeof(double) * 3 * n));
        reflect_vec_len_ = 3 * n;
    }
    double *b = d_reflect_vec_, *x = b + n, *tmp = x + n;
    double *w = d_reflect_;
    IDC_TRY_CUDA(cudaMemcpyAsync(w, src, sizeof(double) * psi_len(), cudaMemcpyDeviceToDevice, stream));
    IDC_TRY(reflect_ghosts(w, nullptr, false));
    IDC_TRY(boundary_sweep(w, dt, b, precision));
    IDC_TRY(reflect_ghosts(w, b + np, true));
    bool converged = false;
    double resid = 0.0;
    auto op = [&](const double *in, double *out) { return apply_peierls_boundary(in, out, tmp, dt, precision); };
    IDC_TRY(gmres(op, b, x, abs_tol, restart, max_its, iters_out, &resid, &converged, precond_kind == 1 ? 1 : 0,
                  ng));
    IDC_TRY_CUDA(cudaMemcpyAsync(psi_out, src, sizeof(double) * psi_len(), cudaMemcpyDeviceToDevice, stream));
    IDC_TRY(reflect_ghosts(psi_out, x + np, false));
    IDC_TRY(smv(1.0, 1.0, x, psi_out));
    IDC_TRY(boundary_sweep(psi_out, dt, nullptr, precision));
    IDC_TRY(check_device_error());
    if (resid_out) *resid_out = resid;
    if (!converged)
        return bad(IDC_ERR_NOT_CONVERGED, "GMRES transport solve failed to converge (max_its reached, residual " +
                                              std::to_string(resid) + ")");
    return Status::ok();
}

// (I - P L^{-1} S) phi = P L^{-1} Q (PETScPeierlsSolver.cpp:423-572), then psi = L^{-1}(S phi + Q).
Status Context::gmres_peierls(const double *src, double *psi_out, double dt, double abs_tol, int restart,
                              int64_t max_its, int precision, int64_t *iters_out, double *resid_out,
                              const double *phi_guess) {
    if (!use_warp_kernel) return bad(IDC_ERR_UNSUPPORTED, "GMRES needs the warp-pipelined sweep kernel");
    if (reflect_mask || periodic_)
        return gmres_peierls_boundary(src, psi_out, dt, abs_tol, restart, max_its, precision, iters_out, resid_out);
    if (precision == IDC_PREC_FP32_IR) return gmres_peierls_ir(src, psi_out, dt, abs_tol, restart, max_its, iters_out,
                                                               resid_out);
    IDC_TRY(ensure_phi_buffers(6));
    double *b = phi_buf(3), *x = phi_buf(4), *tmp = phi_buf(5);
    // right-hand side b = P L^{-1} Q (PETScPeierlsSolver.cpp:461-466)
    IDC_TRY(sweep(src, nullptr, dt, b, precision));
    bool converged = false;
    double resid = 0.0;
    auto op = [&](const double *in, double *out) { return apply_peierls(in, out, tmp, dt, precision); };
    if (phi_guess)
        IDC_TRY_CUDA(cudaMemcpyAsync(x, phi_guess, sizeof(double) * phi_len(), cudaMemcpyDeviceToDevice, stream));
    IDC_TRY(gmres(op, b, x, abs_tol, restart, max_its, iters_out, &resid, &converged, precond_kind == 1 ? 1 : 0, 0,
                  phi_guess != nullptr));
    // psi = L^{-1} (S phi + Q)  (PETScPeierlsSolver.cpp:504-505)
    IDC_TRY(sweep(src, psi_out, dt, nullptr, precision, x, 1.0));
    IDC_TRY(check_device_error());
    if (resid_out) *resid_out = resid;
    if (!converged)
        return bad(IDC_ERR_NOT_CONVERGED, "GMRES transport solve failed to converge (max_its reached, residual " +
                                              std::to_string(resid) + ")");
    return Status::ok();
}

// FP64 iterative refinement of the Peierls system A phi = b (A = I - P L^{-1} S, b = P L^{-1} Q) around FP32
// Krylov solves: b, every residual r = b - A phi and the final psi = L^{-1}(S phi + Q) come from FP64 sweeps;
// each correction A d = r is solved by GMRES (with the DSA preconditioner if set) whose sweeps run in FP32
// arithmetic, to kIrInnerReduction of |r| (the FP32 operator is accurate to about 1e-7 relative), and
// phi += d.  Stops when |r| <= abs_tol (the same absolute criterion as the FP64 solve).  *iters_out counts the
// FP32 Krylov iterations, the FP64 residual sweeps come on top (one per correction).
Status Context::gmres_peierls_ir(const double *src, double *psi_out, double dt, double abs_tol, int restart,
                                 int64_t max_its, int64_t *iters_out, double *resid_out) {
    constexpr double kIrInnerReduction = 1e-5;
    constexpr int kIrMaxCorrections = 20;
    IDC_TRY(ensure_phi_buffers(9));
    double *b = phi_buf(3), *x = phi_buf(4), *tmp = phi_buf(5), *r = phi_buf(6), *d = phi_buf(7), *ax = phi_buf(8);
    const size_t n = phi_len();
    IDC_TRY(sweep(src, nullptr, dt, b, IDC_PREC_FP64));
    IDC_TRY_CUDA(cudaMemsetAsync(x, 0, sizeof(double) * n, stream));
    IDC_TRY_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
    auto op32 = [&](const double *in, double *out) { return apply_peierls(in, out, tmp, dt, IDC_PREC_FP32); };
    int64_t total = 0;
    double resid = 0.0;
    bool converged = false;
    ir_corrections = 0;
    for (int k = 0;; ++k) {
        double rr = 0.0;
        IDC_TRY(dot_host(r, r, n, &rr));
        resid = std::sqrt(rr);
        if (resid <= abs_tol) {
            converged = true;
            break;
        }
        if (k >= kIrMaxCorrections || total >= max_its) break;
        int64_t its = 0;
        double ires = 0.0;
        bool iconv = false;
        IDC_TRY(gmres(op32, r, d, std::max(abs_tol, kIrInnerReduction * resid), restart, max_its - total, &its, &ires,
                      &iconv, precond_kind == 1 ? 1 : 0));
        total += its;
        ++ir_corrections;
        IDC_TRY_CUDA(launch_axpby(1.0, d, 1.0, x, n, stream));            // phi += d
        IDC_TRY(apply_peierls(x, ax, tmp, dt, IDC_PREC_FP64));             // r = b - A phi in FP64
        IDC_TRY_CUDA(cudaMemcpyAsync(r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, stream));
        IDC_TRY_CUDA(launch_axpby(-1.0, ax, 1.0, r, n, stream));
        launches += 3;
    }
    IDC_TRY(sweep(src, psi_out, dt, nullptr, IDC_PREC_FP64, x, 1.0));
    IDC_TRY(check_device_error());
    if (iters_out) *iters_out = total;
    if (resid_out) *resid_out = resid;
    if (!converged)
        return bad(IDC_ERR_NOT_CONVERGED, "GMRES iterative refinement failed to converge (residual " +
                                              std::to_string(resid) + ")");
    return Status::ok();
}

Status Context::set_preconditioner(int kind, int inner_steps) {
    if (kind < 0 || kind > 1) return bad(IDC_ERR_ARG, "unknown preconditioner");
    if (kind == 1 && (inner_steps < 1 || inner_steps > 10000)) return bad(IDC_ERR_ARG, "DSA steps must be in 1..10000");
    precond_kind = kind;
    if (kind == 1) dsa_steps = inner_steps;
    return Status::ok();
}

// y = x - S^T L^{-T} P^T x: one transposed sweep with the fused source w_q x, no psi stored, the unweighted
// moment sums scaled by sigma_s / (4 pi).
Status Context::apply_peierls_adjoint(const double *x, double *y, double *tmp_phi, double dt, int precision) {
    if (periodic_ || reflect_mask)
        return bad(IDC_ERR_UNSUPPORTED, "adjoint solves with periodic or reflecting edges");
    IDC_TRY(sweep(nullptr, nullptr, dt, tmp_phi, precision, x, 1.0, true));
    IDC_TRY_CUDA(launch_adjoint_scatter(dims(), d_sigma_s, x, tmp_phi, y, stream));
    launches += 1;
    return Status::ok();
}

// The discrete adjoint of the steady (or implicit-step) transport problem F = L' psi - Q - S P psi = 0
// with the functional J = c . P psi: (L' - S P)^T lam = P^T c.  With mu = c + S^T lam the equation reads
// (I - S^T L'^{-T} P^T) mu = c (GMRES), then lam = L'^{-T} P^T mu (one more transposed sweep).
// lam_out (psi-sized, nullable) and Lam_out = sum_q lam_q (moment-sized) are device arrays.
Status Context::adjoint_solve(const double *detector, double *lam_out, double *Lam_out, double dt, double abs_tol,
                              int restart, int64_t max_its, int precision, int64_t *iters, double *resid_out) {
    if (!modal_family()) return bad(IDC_ERR_UNSUPPORTED, "the adjoint needs the modal sweep kernel");
    IDC_TRY(ensure_phi_buffers(8));
    double *mu = phi_buf(6), *tmp = phi_buf(7);
    bool converged = false;
    double resid = 0.0;
    auto op = [&](const double *in, double *out) { return apply_peierls_adjoint(in, out, tmp, dt, precision); };
    // the transposed DSA preconditions the adjoint operator (the same spectrum as the forward one)
    IDC_TRY(gmres(op, detector, mu, abs_tol, restart, max_its, iters, &resid, &converged, precond_kind == 1 ? 2 : 0));
    IDC_TRY(sweep(nullptr, lam_out, dt, Lam_out, precision, mu, 1.0, true));
    IDC_TRY(check_device_error());
    if (resid_out) *resid_out = resid;
    if (!converged)
        return bad(IDC_ERR_NOT_CONVERGED, "adjoint GMRES failed to converge (max_its reached, residual " +
                                              std::to_string(resid) + ")");
    return Status::ok();
}

Status Context::adjoint_gradient(const double *psi, const double *detector, double dt, double abs_tol, int restart,
                                 int64_t max_its, int precision, double *dsig_t, double *dsig_s, double *dq,
                                 int64_t *iters, double *resid) {
    IDC_TRY(ensure_psi_buffers(1));
    IDC_TRY(ensure_phi_buffers(10));
    double *lam = psi_buf(0), *Lam = phi_buf(8), *phi = phi_buf(9);
    IDC_TRY(adjoint_solve(detector, lam, Lam, dt, abs_tol, restart, max_its, precision, iters, resid));
    IDC_TRY(pmv(1.0, 0.0, psi, phi));
    if (dsig_t) IDC_TRY_CUDA(cudaMemsetAsync(dsig_t, 0, sizeof(double) * sig_len(), stream));
    if (dsig_s) IDC_TRY_CUDA(cudaMemsetAsync(dsig_s, 0, sizeof(double) * sig_len(), stream));
    if (dq) IDC_TRY_CUDA(cudaMemsetAsync(dq, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(launch_adjoint_gradient(dims(), psi, lam, phi, Lam, dsig_t, dsig_s, dq, stream));
    launches += 1;
    return Status::ok();
}

Status Context::adjoint_solve_psi(const double *b, double *lam_out, double *Lam_out, double dt, double abs_tol,
                                  int restart, int64_t max_its, int precision, int64_t *iters) {
    if (!modal_family()) return bad(IDC_ERR_UNSUPPORTED, "the adjoint needs the modal sweep kernel");
    IDC_TRY(ensure_phi_buffers(9));
    double *nu = phi_buf(6), *tmp = phi_buf(7), *rhs = phi_buf(8);
    // rhs = S^T L'^{-T} b: the transposed sweep's moment sums, scaled by sigma_s / (4 pi); ghost cells zero
    IDC_TRY(sweep(b, nullptr, dt, tmp, precision, nullptr, 1.0, true));
    IDC_TRY_CUDA(cudaMemsetAsync(rhs, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(launch_scatter_moments(dims(), d_sigma_s, tmp, rhs, stream));
    launches += 1;
    bool converged = false;
    double resid = 0.0;
    auto op = [&](const double *in, double *out) { return apply_peierls_adjoint(in, out, tmp, dt, precision); };
    IDC_TRY(gmres(op, rhs, nu, abs_tol, restart, max_its, iters, &resid, &converged, precond_kind == 1 ? 2 : 0));
    IDC_TRY(sweep(b, lam_out, dt, Lam_out, precision, nu, 1.0, true));   // lam = L'^{-T} (b + P^T nu)
    IDC_TRY(check_device_error());
    if (!converged)
        return bad(IDC_ERR_NOT_CONVERGED, "adjoint GMRES failed to converge (max_its reached, residual " +
                                              std::to_string(resid) + ")");
    return Status::ok();
}

// Discrete adjoint of implicit-Euler time stepping (the reference's `dirk` integrator with the `euler`
// table, time_integrators/RKDG/dirk.cpp; equally IDC's prediction sweeps, time_integrators/RKDG/idc.cpp:
// 846-955): A psi^{n+1} = psi^n / dt + Q with A = 1/dt + L - S P, each step solved by the Peierls GMRES, and
// J = c . P psi^N.  The adjoint runs backwards: A^T lam^N = P^T c, A^T lam^n = lam^{n+1} / dt, and
//     dJ/dsigma_t = -sum_n sum_{q,k} lam^n psi^n,   dJ/dsigma_s = sum_n sum_k Lam^n_k phi^n_k / (4 pi),
//     dJ/dq_k = sum_n Lam^n_k / (4 pi),             dJ/dpsi^0 = lam^1 / dt
// per cell (Q = q / (4 pi) on every ordinate, constant in time).  Checkpointing: the forward pass keeps
// psi^{mK} (K = checkpoint_every); the backward pass recomputes each segment's states from its checkpoint
// (the same deterministic solves, so the states are bitwise those of the forward pass) and runs the
// segment's adjoint steps, so memory holds N/K + K states instead of N.  Inflow (ghost cells of Q) is data,
// not differentiated.
Status Context::adjoint_transient(const double *psi0, const double *Q, double dt, int64_t steps,
                                  const double *detector, int64_t checkpoint_every, double abs_tol, int restart,
                                  int64_t max_its, int precision, double *dsig_t, double *dsig_s, double *dq,
                                  double *dpsi0, double *J, int64_t *solves) {
    if (!have_ordinates || !have_sigma) return bad(IDC_ERR_STATE, "transient adjoint before ordinates and sigma");
    if (!modal_family()) return bad(IDC_ERR_UNSUPPORTED, "the adjoint needs the modal sweep kernel");
    if (steps < 1) return bad(IDC_ERR_ARG, "transient adjoint needs at least one step");
    if (!(dt > 0) || !std::isfinite(dt)) return bad(IDC_ERR_ARG, "transient adjoint needs a finite positive dt");
    const int64_t K = checkpoint_every > 0 ? std::min(checkpoint_every, steps)
                                           : std::max<int64_t>(1, (int64_t)std::ceil(std::sqrt((double)steps)));
    const int64_t M = (steps + K - 1) / K;   // segments; checkpoints psi^{mK}, m = 0..M-1
    const size_t np = psi_len(), nm = phi_len();
    const int need = (int)(M + K + 3);
    IDC_TRY_CUDA(cudaSetDevice(device));
    while ((int)transient_bufs_.size() < need) {   // zeroed once: the sweeps write interior cells only, so the
        double *p = nullptr;                        // ghost cells of every state stay zero
        IDC_TRY_CUDA(cudaMalloc(&p, sizeof(double) * np));
        IDC_TRY_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * np, stream));
        transient_bufs_.push_back(p);
    }
    auto ckpt = [&](int64_t m) { return transient_bufs_[(size_t)m]; };
    auto seg = [&](int64_t k) { return transient_bufs_[(size_t)(M + k - 1)]; };   // k = 1..K
    double *lam = transient_bufs_[(size_t)(M + K)], *b = transient_bufs_[(size_t)(M + K + 1)];
    double *src = transient_bufs_[(size_t)(M + K + 2)];
    IDC_TRY(ensure_phi_buffers(16));   // 15: the warm-start moments of each step's solve
    double *Lam = phi_buf(9), *phi = phi_buf(10);
    int64_t nsolve = 0;

    // one step: out = A^{-1} (in / dt + Q), GMRES from the moments of `in` (the previous step's solution)
    auto step = [&](const double *in, double *out) -> Status {
        IdcTerms tm{};
        tm.n = 1;
        tm.a[0] = in;
        tm.c[0] = 1.0 / dt;
        IDC_TRY_CUDA(launch_idc_source(dims(), tm, Q, src, stream));
        launches += 1;
        IDC_TRY(pmv(1.0, 0.0, in, phi_buf(15)));
        int64_t its = 0;
        double r = 0.0;
        IDC_TRY(gmres_peierls(src, out, dt, abs_tol, restart, max_its, precision, &its, &r, phi_buf(15)));
        ++nsolve;
        return Status::ok();
    };

    // forward pass: checkpoints, and psi^N in the last segment slot for J
    IDC_TRY_CUDA(cudaMemcpyAsync(ckpt(0), psi0, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
    const double *cur = ckpt(0);
    for (int64_t n = 1; n <= steps; ++n) {
        double *out = (n % K == 0 && n / K < M) ? ckpt(n / K) : seg(1);
        IDC_TRY(step(cur, out));
        cur = out;
    }
    IDC_TRY(pmv(1.0, 0.0, cur, phi));
    if (J) IDC_TRY(dot_host(phi, detector, nm, J));

    if (dsig_t) IDC_TRY_CUDA(cudaMemsetAsync(dsig_t, 0, sizeof(double) * sig_len(), stream));
    if (dsig_s) IDC_TRY_CUDA(cudaMemsetAsync(dsig_s, 0, sizeof(double) * sig_len(), stream));
    if (dq) IDC_TRY_CUDA(cudaMemsetAsync(dq, 0, sizeof(double) * nm, stream));
    // backward pass, one segment (m K, min((m+1) K, N)] at a time
    for (int64_t m = M - 1; m >= 0; --m) {
        const int64_t n0 = m * K, n1 = std::min(steps, n0 + K);
        for (int64_t k = 1; k <= n1 - n0; ++k) IDC_TRY(step(k == 1 ? ckpt(m) : seg(k - 1), seg(k)));
        for (int64_t n = n1; n > n0; --n) {
            int64_t its = 0;
            if (n == steps) {   // A^T lam^N = P^T c
                double resid = 0.0;
                IDC_TRY(adjoint_solve(detector, lam, Lam, dt, abs_tol, restart, max_its, precision, &its, &resid));
            } else {            // A^T lam^n = lam^{n+1} / dt
                IDC_TRY_CUDA(launch_axpby(1.0 / dt, lam, 0.0, b, np, stream));
                launches += 1;
                IDC_TRY(adjoint_solve_psi(b, lam, Lam, dt, abs_tol, restart, max_its, precision, &its));
            }
            ++nsolve;
            const double *psin = seg(n - n0);
            IDC_TRY(pmv(1.0, 0.0, psin, phi));
            IDC_TRY_CUDA(launch_adjoint_gradient(dims(), psin, lam, phi, Lam, dsig_t, dsig_s, dq, stream, true));
            launches += 1;
        }
    }
    if (dpsi0) {   // lam^1 / dt on interior cells, zero ghost cells
        IdcTerms tm{};
        tm.n = 1;
        tm.a[0] = lam;
        tm.c[0] = 1.0 / dt;
        IDC_TRY_CUDA(launch_idc_source(dims(), tm, nullptr, dpsi0, stream));
        launches += 1;
    }
    IDC_TRY(check_device_error());
    if (solves) *solves = nsolve;
    return Status::ok();
}

}  // namespace idc
