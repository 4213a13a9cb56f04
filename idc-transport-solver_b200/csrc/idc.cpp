// IDC (integral deferred correction) time stepping of the transport equation on the GPU:
//     d psi / dt = -(L - S P) psi + Q,
// non-hybrid, "update" form (IDCIntegrator::Step_Nonhybrid and ComputeResiduals / ComputeSource,
// time_integrators/RKDG/idc.cpp:846-955, 1657-1740), on Gauss-Lobatto nodes (SetNodes, :2305-2381).
//
// Two treatments of scattering:
//  * implicit (the reference's): every substep solves (1/(h dt) + L - S P) psi_n = src_n with the GPU
//    GMRES (Peierls form); the prediction is implicit Euler, and a correction's source is
//    src_n = sum_l (delta_nl - W(n,l)/h) res_l + psi_{n-1}/(h dt) + Q,  res_l = (L - S P) psi_l.
//  * explicit (IMEX): every substep is one sweep, (1/(h dt) + L) psi_n = src_n + S phi_s, with the
//    scattering lagged to the previous node: the prediction uses phi_s = phi_{n-1}; a correction uses
//    src_n = psi_{n-1}^new/(h dt) + Q + res_n^old - (1/h) sum_l W(n,l) res_l^old and
//    phi_s = phi_{n-1}^new - phi_{n-1}^old + phi_n^old, so that the implicit part L psi_n and the
//    explicit part S P psi_{n-1} are both corrected against the previous level (IMEX deferred correction).
//    A whole IMEX step is a fixed sequence of kernels with no host synchronisation, so it is captured once
//    as a CUDA graph and replayed.
// The quadrature sums, residuals and sources are FP64; `precision` selects the sweep arithmetic.
#include "context.hpp"

#include <algorithm>
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

// Legendre P_n(x) and P_n'(x).
void legendre(int n, double x, double *p, double *dp) {
    double p0 = 1.0, p1 = x;
    if (n == 0) {
        *p = 1.0;
        *dp = 0.0;
        return;
    }
    for (int k = 2; k <= n; ++k) {
        const double pk = ((2 * k - 1) * x * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = pk;
    }
    *p = p1;
    *dp = (std::fabs(x) < 1.0) ? n * (x * p1 - p0) / (x * x - 1.0) : 0.5 * n * (n + 1) * (x > 0 ? 1.0 : ((n & 1) ? 1.0 : -1.0));
}

// Gauss-Legendre nodes / weights on [-1, 1] (Newton on P_m).
void gauss_legendre(int m, std::vector<double> &x, std::vector<double> &w) {
    x.assign(m, 0.0);
    w.assign(m, 0.0);
    for (int k = 0; k < m; ++k) {
        double z = std::cos(M_PI * (k + 0.75) / (m + 0.5));
        for (int it = 0; it < 100; ++it) {
            double p, dp;
            legendre(m, z, &p, &dp);
            const double dz = p / dp;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        double p, dp;
        legendre(m, z, &p, &dp);
        x[k] = z;
        w[k] = 2.0 / ((1.0 - z * z) * dp * dp);
    }
}

// Gauss-Lobatto nodes on [0, 1] (M >= 2): the endpoints and the roots of P'_{M-1}.
std::vector<double> lobatto_nodes(int M) {
    std::vector<double> t(M);
    const int n = M - 1;
    t[0] = 0.0;
    t[M - 1] = 1.0;
    for (int k = 1; k < n; ++k) {
        double z = -std::cos(M_PI * k / n);
        for (int it = 0; it < 100; ++it) {
            double p, dp;
            legendre(n, z, &p, &dp);
            const double d2p = (2.0 * z * dp - n * (n + 1) * p) / (1.0 - z * z);
            const double dz = dp / d2p;
            z -= dz;
            if (std::fabs(dz) < 1e-16) break;
        }
        t[k] = 0.5 * (z + 1.0);
    }
    return t;
}

// W[i][j] = integral over [t_{i-1}, t_i] (i >= 1) or [0, 1] (i = 0) of the Lagrange basis l_j of the nodes.
std::vector<double> integration_weights(const std::vector<double> &t) {
    const int M = (int)t.size();
    std::vector<double> gx, gw, W((size_t)M * M, 0.0);
    gauss_legendre(M, gx, gw);   // exact for degree 2M-1 >= M-1
    for (int i = 0; i < M; ++i) {
        const double a = i == 0 ? 0.0 : t[i - 1], b = i == 0 ? 1.0 : t[i];
        for (int j = 0; j < M; ++j) {
            double acc = 0.0;
            for (int q = 0; q < M; ++q) {
                const double x = 0.5 * (a + b) + 0.5 * (b - a) * gx[q];
                double l = 1.0;
                for (int m = 0; m < M; ++m)
                    if (m != j) l *= (x - t[m]) / (t[j] - t[m]);
                acc += gw[q] * l;
            }
            W[(size_t)i * M + j] = 0.5 * (b - a) * acc;
        }
    }
    return W;
}

}  // namespace

void idc_nodes_and_weights(int M, std::vector<double> &t, std::vector<double> &W) {
    t = lobatto_nodes(M);
    W = integration_weights(t);
}

Status Context::idc_integrate(double *psi, const double *Q, double dt, int64_t steps, int M, int K, int scattering,
                              int precision, double abs_tol, int restart, int64_t max_its, bool use_graph,
                              int64_t *sweeps_out) {
    if (!have_ordinates || !have_sigma) return bad(IDC_ERR_STATE, "IDC before ordinates and sigma");
    if (M < 2 || M > 8) return bad(IDC_ERR_ARG, "IDC nodes must be in 2..8");
    if (K < 0 || K > 16) return bad(IDC_ERR_ARG, "IDC corrections must be in 0..16");
    if (!(dt > 0) || !std::isfinite(dt)) return bad(IDC_ERR_ARG, "IDC needs a finite positive dt");
    if (steps < 0) return bad(IDC_ERR_ARG, "negative step count");
    if (scattering != 0 && scattering != 1) return bad(IDC_ERR_ARG, "scattering must be 0 (explicit) or 1 (implicit)");
    if (scattering == 0 && (reflect_mask || periodic_))
        return bad(IDC_ERR_UNSUPPORTED, "IDC with explicit scattering on reflecting or periodic edges; implicit "
                                        "scattering takes them");
    // explicit scattering: the lane or modal kernel's second source and the fused correction kernel (piecewise-
    // constant sigma, DG degree <= 2); implicit scattering (GMRES substeps) takes every input the solver takes
    if (scattering == 0 && !modal_family())
        return bad(IDC_ERR_UNSUPPORTED, "IDC with explicit scattering needs the lane or modal kernel (DG degree <= 2, "
                                        "piecewise-constant cross sections); implicit scattering takes these inputs");
    std::vector<double> t, W;
    idc_nodes_and_weights(M, t, W);
    // The IMEX sweeps (a second source and the scattering term) at DG degree 1 run on the lane kernel's default
    // shape when its work queue has an item for every resident warp, else on the modal (8, 5) shape.  Measured
    // per step (lattice, Q1 S12): 512^2 (1536 lane items for 1184 resident warps) lane 22.2 ms, modal 23.7 ms;
    // 256^2 (768 items) lane 8.9 ms, modal 7.7 ms.  Without a tile shape of the caller's, the modal shape is
    // set for the call and the default comes back when it returns, on every path (the schedules are rebuilt:
    // ~0.8 ms per call at these sizes).
    struct TileRestore {
        Context *c = nullptr;
        ~TileRestore() {
            if (c) c->set_tile_shape(0, 0);
        }
    } tile_restore;
    if (scattering == 0 && P == 2 && tune_seg == 0 && tune_wn == 0 && kernel_for(precision) == kLane) {
        int counts[4], qmax = 0;
        for (int k = 0; k < 4; ++k) qmax = std::max(qmax, counts[k] = (int)(quad[k + 1] - quad[k]));
        const int seg = qmax <= 24 ? 8 : 4, rows = 32 / seg;
        int64_t items = 0;
        for (int k = 0; k < 4; ++k) items += (int64_t)((counts[k] + seg - 1) / seg) * ((ny + rows - 1) / rows);
        int &per_sm = lane_src2_blocks_[seg == 8 ? 0 : 1];   // queried once per context
        if (per_sm < 0) IDC_TRY_CUDA(sweep_lane_occupancy(P, seg, true, &per_sm));
        if (items < (int64_t)per_sm * sweep_lane_warps() * num_sms) {
            IDC_TRY(set_tile_shape(8, 5));
            tile_restore.c = this;
        }
    }

    // buffers: M stages, M residuals, one source (psi-sized); M moments, M previous-level moments, one
    // scattering combination (moment-sized)
    const size_t np = psi_len(), nm = phi_len();
    const int need_psi = 2 * M + 1, need_phi = 3 * M + 1;
    IDC_TRY_CUDA(cudaSetDevice(device));
    while ((int)idc_psi_.size() < need_psi) {
        double *p = nullptr;
        IDC_TRY_CUDA(cudaMalloc(&p, sizeof(double) * np));
        idc_psi_.push_back(p);
    }
    while ((int)idc_phi_.size() < need_phi) {
        double *p = nullptr;
        IDC_TRY_CUDA(cudaMalloc(&p, sizeof(double) * nm));
        IDC_TRY_CUDA(cudaMemset(p, 0, sizeof(double) * nm));
        idc_phi_.push_back(p);
    }
    auto stage = [&](int l) { return idc_psi_[l]; };
    auto res = [&](int l) { return idc_psi_[M + l]; };
    double *src = idc_psi_[2 * M];
    auto phi = [&](int l) { return idc_phi_[l]; };
    auto phi_old = [&](int l) { return idc_phi_[M + l]; };
    double *phi_s = idc_phi_[2 * M];
    auto scat = [&](int l) { return idc_phi_[2 * M + 1 + l]; };   // sigma_s phi_l / (4 pi)
    int64_t sweeps = 0;

    auto residual = [&](int l) -> Status {   // res_l = (L - S P) psi_l  (ComputeResiduals, idc.cpp:1657-1667)
        IDC_TRY(pmv(1.0, 0.0, stage(l), phi(l)));
        IDC_TRY(transport_residual(stage(l), phi(l), res(l)));
        return Status::ok();
    };
    auto source = [&](int n, bool correction, bool imex) -> Status {
        const double h = t[n] - t[n - 1];
        IdcTerms tm{};
        tm.n = 0;
        tm.a[tm.n] = stage(n - 1);
        tm.c[tm.n++] = 1.0 / (h * dt);
        if (correction) {
            for (int l = 0; l < M; ++l) {
                tm.a[tm.n] = res(l);
                tm.c[tm.n++] = (n == l ? 1.0 : 0.0) - W[(size_t)n * M + l] / h;
            }
        }
        (void)imex;
        IDC_TRY_CUDA(launch_idc_source(dims(), tm, Q, src, stream));
        launches += 1;
        return Status::ok();
    };

    // one IMEX step: only stream work, so it can be captured
    auto imex_step = [&]() -> Status {
        IDC_TRY(pmv(1.0, 0.0, stage(0), phi(0)));
        for (int n = 1; n < M; ++n) {   // prediction: IMEX Euler, source Q + psi_{n-1} / (h dt) formed in the sweep
            const double h = t[n] - t[n - 1];
            IDC_TRY(sweep(Q, stage(n), h * dt, phi(n), precision, phi(n - 1), 1.0, false, stage(n - 1), 1.0 / (h * dt)));
            ++sweeps;
        }
        const bool fused = M <= kIdcFusedMaxNodes;
        for (int p = 0; p < K; ++p) {
            if (fused) {   // every substep's residual terms in one pass over the stages (into res(1 .. M-1))
                IdcCorr cr{};
                cr.Q = Q;
                for (int l = 0; l < M; ++l) {
                    IDC_TRY_CUDA(launch_scatter_moments(dims(), d_sigma_s, phi(l), scat(l), stream));
                    cr.stage[l] = stage(l);
                    cr.scat[l] = scat(l);
                }
                for (int n = 1; n < M; ++n) {
                    cr.out[n] = res(n);
                    const double h = t[n] - t[n - 1];
                    for (int l = 0; l < M; ++l) cr.c[n][l] = (n == l ? 1.0 : 0.0) - W[(size_t)n * M + l] / h;
                }
                IDC_TRY_CUDA(launch_idc_corrections(dims(), M, cr, d_sigma_t, d_xi, d_eta, stream));
                launches += M + 1;
            }
            for (int l = 0; l < M; ++l) {
                if (!fused) IDC_TRY(transport_residual(stage(l), phi(l), res(l)));
                IDC_TRY_CUDA(cudaMemcpyAsync(phi_old(l), phi(l), sizeof(double) * nm, cudaMemcpyDeviceToDevice, stream));
            }
            for (int n = 1; n < M; ++n) {
                const double h = t[n] - t[n - 1];
                if (!fused) IDC_TRY(source(n, true, true));
                IDC_TRY_CUDA(launch_phi_combine(nm, phi(n - 1), phi_old(n - 1), phi_old(n), phi_s, stream));
                launches += 1;
                if (fused)   // src_n = (Q + the residual terms, with Q's ghost cells) + psi_{n-1} / (h dt)
                    IDC_TRY(sweep(res(n), stage(n), h * dt, phi(n), precision, phi_s, 1.0, false, stage(n - 1),
                                  1.0 / (h * dt)));
                else
                    IDC_TRY(sweep(src, stage(n), h * dt, phi(n), precision, phi_s, 1.0));
                ++sweeps;
            }
        }
        IDC_TRY_CUDA(cudaMemcpyAsync(stage(0), stage(M - 1), sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
        return Status::ok();
    };

    // stage ghost cells hold the inflow values (Q's ghost cells), as the reference's in-place solves leave
    // them; the sweeps write interior cells only, so they stay.  Lmv reads them for the boundary residuals.
    IDC_TRY_CUDA(cudaMemcpyAsync(stage(0), psi, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
    for (int l = 1; l < M; ++l)
        IDC_TRY_CUDA(cudaMemcpyAsync(stage(l), Q, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
    // the fused IMEX corrections write interior cells of res(1 .. M-1) only: their ghost cells hold Q's (the
    // inflow), which the substep sources copy
    if (scattering == 0 && M <= kIdcFusedMaxNodes)
        for (int l = 1; l < M; ++l)
            IDC_TRY_CUDA(cudaMemcpyAsync(res(l), Q, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
    if (scattering == 0) {
        if (use_graph && steps > 0) {
            // first step uncaptured (builds the sweep schedule, allocates nothing inside the capture), then
            // capture one step and replay it
            IDC_TRY(imex_step());
            IDC_TRY(check_device_error());
            if (steps > 1) {
                cudaGraph_t graph = nullptr;
                cudaGraphExec_t exec = nullptr;
                capturing = true;
                const int64_t s0 = sweeps, l0 = launches;
                IDC_TRY_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
                Status st = imex_step();
                cudaError_t ce = cudaStreamEndCapture(stream, &graph);
                capturing = false;
                if (!st.good()) {
                    if (graph) cudaGraphDestroy(graph);
                    return st;
                }
                IDC_TRY_CUDA(ce);
                const int64_t per_sweeps = sweeps - s0, per_launch = launches - l0;
                sweeps = s0;
                launches = l0;
                ce = cudaGraphInstantiate(&exec, graph, 0);
                if (ce != cudaSuccess) {
                    cudaGraphDestroy(graph);
                    return cuda_status(ce, "cudaGraphInstantiate");
                }
                for (int64_t s = 1; s < steps; ++s) {
                    ce = cudaGraphLaunch(exec, stream);
                    if (ce != cudaSuccess) break;
                    sweeps += per_sweeps;
                    launches += per_launch;
                }
                cudaGraphExecDestroy(exec);
                cudaGraphDestroy(graph);
                IDC_TRY_CUDA(ce);
            }
        } else {
            for (int64_t s = 0; s < steps; ++s) IDC_TRY(imex_step());
        }
        IDC_TRY(check_device_error());
    } else {
        // implicit: GMRES per substep (host-driven; the reference's Step_Nonhybrid, update form); a guess costs
        // one operator application where it is used
        const bool warm_start = !(reflect_mask || periodic_ || precision == IDC_PREC_FP32_IR);
        for (int64_t s = 0; s < steps; ++s) {
            // the step's initial stage with its boundary ghosts made consistent, as Step_Nonhybrid reflects it
            // (idc.cpp:855-859) and Lmv synchronises periodic halos before reading them; the stages the
            // substep solves return carry their reflections or periodic images already
            if (reflect_mask) {
                IDC_TRY_CUDA(launch_reflect_boundaries(dims(), reflect_mask, d_xi, d_eta, d_rmap, stage(0), stream));
                launches += 1;
            } else if (periodic_) {
                IDC_TRY_CUDA(launch_periodic_halos(dims(), stage(0), stream));
                launches += 1;
            }
            // GMRES starts from the previous node's moments in the prediction and from the same node's moments one
            // level down in the corrections (the reference's source iteration keeps its psi between substeps)
            for (int n = 1; n < M; ++n) {
                const double h = t[n] - t[n - 1];
                IDC_TRY(source(n, false, false));
                IDC_TRY(pmv(1.0, 0.0, stage(n - 1), phi(n)));
                int64_t its = 0;
                double r = 0;
                IDC_TRY(gmres_peierls(src, stage(n), h * dt, abs_tol, restart, max_its, precision, &its, &r, phi(n)));
                sweeps += its + (warm_start ? 3 : 2);
            }
            for (int p = 0; p < K; ++p) {
                for (int l = 0; l < M; ++l) IDC_TRY(residual(l));
                for (int n = 1; n < M; ++n) {   // phi(n) = P stage(n) of the level before (residual)
                    const double h = t[n] - t[n - 1];
                    IDC_TRY(source(n, true, false));
                    int64_t its = 0;
                    double r = 0;
                    IDC_TRY(gmres_peierls(src, stage(n), h * dt, abs_tol, restart, max_its, precision, &its, &r,
                                          phi(n)));
                    sweeps += its + (warm_start ? 3 : 2);
                }
            }
            IDC_TRY_CUDA(cudaMemcpyAsync(stage(0), stage(M - 1), sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
        }
    }
    IDC_TRY_CUDA(cudaMemcpyAsync(psi, stage(0), sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
    IDC_TRY_CUDA(cudaStreamSynchronize(stream));
    if (sweeps_out) *sweeps_out = sweeps;
    return Status::ok();
}

}  // namespace idc

namespace idc {

// Discrete adjoint of implicit-scattering IDC time stepping (idc_integrate with scattering = 1, the reference's
// IDCIntegrator::Step_Nonhybrid in update form, time_integrators/RKDG/idc.cpp:846-955, 1657-1740).  One step
// from psi_in, with A_n = 1/(h_n dt) + T, T = L - S P (transport_residual) and c_nl = delta_nl - W(n,l)/h_n:
//     level 0:  A_n u^0_n = u^0_{n-1} / (h_n dt) + Q                                (n = 1..M-1, u^p_0 = psi_in)
//     level p:  A_n u^p_n = u^p_{n-1} / (h_n dt) + sum_l c_nl T u^{p-1}_l + Q       (p = 1..K)
//     psi_out = u^K_{M-1}.
// Backwards through a step, ubar being the adjoint of the stages and rbar that of the residuals T u^{p-1}_l:
//     for p = K..0, n = M-1..1:  A_n^T lam = ubar_n (adjoint_solve_psi);  ubar_{n-1} += lam / (h_n dt);
//                                 rbar_l += c_nl lam;  the solve's gradient terms (-lam^T dA u, lam^T dQ);
//     then ubar^{p-1}_l = T^T rbar_l (lmvt_kernel; l = 0 feeds psi_in's adjoint) and the residuals' gradient
//     terms +rbar^T dT u^{p-1}_l (the solve's form with the opposite sign and no source term).
// psi_in's adjoint (every level's first substep and its l = 0 residual) becomes the previous step's psi_out
// adjoint; J = c . P psi^N starts the last step with P^T c.  Checkpointing as in adjoint_transient: psi at
// every CK-th step boundary; the backward pass recomputes a segment's step inputs, then each step's stages
// (bitwise those of the forward pass: every solve is reproducible).  Inflow (Q's ghost cells) is data.
Status Context::adjoint_idc(const double *psi0, const double *Q, double dt, int64_t steps, int M, int K,
                            const double *detector, int64_t checkpoint_every, double abs_tol, int restart,
                            int64_t max_its, int precision, double *dsig_t, double *dsig_s, double *dq, double *dpsi0,
                            double *J, int64_t *solves) {
    if (!have_ordinates || !have_sigma) return bad(IDC_ERR_STATE, "IDC adjoint before ordinates and sigma");
    if (!modal_family()) return bad(IDC_ERR_UNSUPPORTED, "the adjoint needs the modal sweep kernel");
    if (steps < 1) return bad(IDC_ERR_ARG, "IDC adjoint needs at least one step");
    if (!(dt > 0) || !std::isfinite(dt)) return bad(IDC_ERR_ARG, "IDC adjoint needs a finite positive dt");
    if (M < 2 || M > 8) return bad(IDC_ERR_ARG, "IDC nodes must be in 2..8");
    if (K < 0 || K > 16) return bad(IDC_ERR_ARG, "IDC corrections must be in 0..16");
    std::vector<double> t, W;
    idc_nodes_and_weights(M, t, W);
    const int64_t CK = checkpoint_every > 0 ? std::min(checkpoint_every, steps)
                                            : std::max<int64_t>(1, (int64_t)std::ceil(std::sqrt((double)steps)));
    const int64_t NS = (steps + CK - 1) / CK;
    const size_t np = psi_len(), nm = phi_len();
    const int64_t n_stage = (int64_t)(K + 1) * M;
    const int64_t need = NS + CK + n_stage + 3 * (int64_t)M + 6;
    IDC_TRY_CUDA(cudaSetDevice(device));
    while ((int64_t)adj_idc_bufs_.size() < need) {   // zeroed once: the kernels below write interior cells only
        double *p = nullptr;
        IDC_TRY_CUDA(cudaMalloc(&p, sizeof(double) * np));
        IDC_TRY_CUDA(cudaMemsetAsync(p, 0, sizeof(double) * np, stream));
        adj_idc_bufs_.push_back(p);
    }
    auto ckpt = [&](int64_t m) { return adj_idc_bufs_[(size_t)m]; };
    auto inp = [&](int64_t k) { return adj_idc_bufs_[(size_t)(NS + k)]; };   // k = 0..CK-1
    auto stage = [&](int p, int n) { return adj_idc_bufs_[(size_t)(NS + CK + (int64_t)p * M + n)]; };
    const size_t b0 = (size_t)(NS + CK + n_stage);
    auto res = [&](int l) { return adj_idc_bufs_[b0 + l]; };
    auto ubar = [&](int l) { return adj_idc_bufs_[b0 + M + l]; };
    auto rbar = [&](int l) { return adj_idc_bufs_[b0 + 2 * M + l]; };
    double *lam = adj_idc_bufs_[b0 + 3 * M], *tmp = adj_idc_bufs_[b0 + 3 * M + 1];
    double *src = adj_idc_bufs_[b0 + 3 * M + 2], *pbar = adj_idc_bufs_[b0 + 3 * M + 3];
    double *inbar = adj_idc_bufs_[b0 + 3 * M + 4], *zsum = adj_idc_bufs_[b0 + 3 * M + 5];   // zsum: moment-sized use
    IDC_TRY(ensure_phi_buffers(16));   // 15: the warm-start moments of each solve
    double *Lam = phi_buf(9), *phi = phi_buf(10), *guess = phi_buf(15);
    int64_t nsolve = 0;
    // stage ghost cells hold the inflow (Q's ghost cells), as in idc_integrate; the solves write interiors only
    for (int p = 0; p <= K; ++p)
        for (int n = 1; n < M; ++n)
            IDC_TRY_CUDA(cudaMemcpyAsync(stage(p, n), Q, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));

    auto solve = [&](int p, int n) -> Status {   // A_n u^p_n = u^p_{n-1}/(h dt) [+ sum_l c_nl res_l] + Q
        const double h = t[n] - t[n - 1];
        IdcTerms tm{};
        tm.n = 0;
        tm.a[tm.n] = stage(p, n - 1);
        tm.c[tm.n++] = 1.0 / (h * dt);
        if (p > 0)
            for (int l = 0; l < M; ++l) {
                tm.a[tm.n] = res(l);
                tm.c[tm.n++] = (n == l ? 1.0 : 0.0) - W[(size_t)n * M + l] / h;
            }
        IDC_TRY_CUDA(launch_idc_source(dims(), tm, Q, src, stream));
        launches += 1;
        // GMRES from the moments idc_integrate starts from: the previous node's stage (prediction), the same
        // node's stage one level down (corrections)
        IDC_TRY(pmv(1.0, 0.0, p == 0 ? stage(0, n - 1) : stage(p - 1, n), guess));
        int64_t its = 0;
        double r = 0.0;
        IDC_TRY(gmres_peierls(src, stage(p, n), h * dt, abs_tol, restart, max_its, precision, &its, &r, guess));
        ++nsolve;
        return Status::ok();
    };
    // one forward step from `in`, every level's stages kept; the result is stage(K, M - 1)
    auto step_store = [&](const double *in) -> Status {
        for (int p = 0; p <= K; ++p)
            IDC_TRY_CUDA(cudaMemcpyAsync(stage(p, 0), in, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
        for (int n = 1; n < M; ++n) IDC_TRY(solve(0, n));
        for (int p = 1; p <= K; ++p) {
            for (int l = 0; l < M; ++l) {   // res_l = (L - S P) u^{p-1}_l
                IDC_TRY(pmv(1.0, 0.0, stage(p - 1, l), phi));
                IDC_TRY(transport_residual(stage(p - 1, l), phi, res(l)));
            }
            for (int n = 1; n < M; ++n) IDC_TRY(solve(p, n));
        }
        return Status::ok();
    };
    auto axpy = [&](double a, const double *x, double *y) -> Status {
        IDC_TRY_CUDA(launch_axpby(a, x, 1.0, y, np, stream));
        launches += 1;
        return Status::ok();
    };

    // forward pass: checkpoints at the segment boundaries, J from psi^N
    IDC_TRY_CUDA(cudaMemcpyAsync(ckpt(0), psi0, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
    const double *cur = ckpt(0);
    for (int64_t s = 1; s <= steps; ++s) {
        IDC_TRY(step_store(cur));
        cur = stage(K, M - 1);
        if (s % CK == 0 && s / CK < NS) {
            IDC_TRY_CUDA(cudaMemcpyAsync(ckpt(s / CK), cur, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
            cur = ckpt(s / CK);
        }
    }
    IDC_TRY(pmv(1.0, 0.0, cur, phi));
    if (J) IDC_TRY(dot_host(phi, detector, nm, J));

    if (dsig_t) IDC_TRY_CUDA(cudaMemsetAsync(dsig_t, 0, sizeof(double) * sig_len(), stream));
    if (dsig_s) IDC_TRY_CUDA(cudaMemsetAsync(dsig_s, 0, sizeof(double) * sig_len(), stream));
    if (dq) IDC_TRY_CUDA(cudaMemsetAsync(dq, 0, sizeof(double) * nm, stream));
    IDC_TRY_CUDA(launch_weighted_broadcast(dims(), d_w, detector, pbar, stream));   // P^T c
    launches += 1;

    // the adjoint of one step: pbar (psi_out's adjoint) -> pbar (psi_in's adjoint), stages of the step in place
    auto adjoint_step = [&]() -> Status {
        for (int l = 0; l < M; ++l) IDC_TRY_CUDA(cudaMemsetAsync(ubar(l), 0, sizeof(double) * np, stream));
        IDC_TRY_CUDA(cudaMemcpyAsync(ubar(M - 1), pbar, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
        IDC_TRY_CUDA(cudaMemsetAsync(inbar, 0, sizeof(double) * np, stream));
        for (int p = K; p >= 0; --p) {
            if (p > 0)
                for (int l = 0; l < M; ++l) IDC_TRY_CUDA(cudaMemsetAsync(rbar(l), 0, sizeof(double) * np, stream));
            for (int n = M - 1; n >= 1; --n) {
                const double h = t[n] - t[n - 1];
                int64_t its = 0;
                IDC_TRY(adjoint_solve_psi(ubar(n), lam, Lam, h * dt, abs_tol, restart, max_its, precision, &its));
                ++nsolve;
                IDC_TRY(pmv(1.0, 0.0, stage(p, n), phi));
                IDC_TRY_CUDA(launch_adjoint_gradient(dims(), stage(p, n), lam, phi, Lam, dsig_t, dsig_s, dq, stream,
                                                     true, 1.0));
                launches += 1;
                IDC_TRY(axpy(1.0 / (h * dt), lam, n == 1 ? inbar : ubar(n - 1)));
                if (p > 0)
                    for (int l = 0; l < M; ++l) {
                        const double c = (n == l ? 1.0 : 0.0) - W[(size_t)n * M + l] / h;
                        if (c != 0.0) IDC_TRY(axpy(c, lam, rbar(l)));
                    }
            }
            if (p > 0)
                for (int l = 0; l < M; ++l) {   // res_l = T u^{p-1}_l: the adjoint of level p-1's stage l
                    double *y = l == 0 ? tmp : ubar(l);
                    IDC_TRY(transport_residual_transpose(rbar(l), y, zsum));
                    if (l == 0) IDC_TRY(axpy(1.0, tmp, inbar));
                    IDC_TRY(pmv(1.0, 0.0, stage(p - 1, l), phi));
                    IDC_TRY_CUDA(launch_adjoint_gradient(dims(), stage(p - 1, l), rbar(l), phi, zsum, dsig_t, dsig_s,
                                                         nullptr, stream, true, -1.0));
                    launches += 1;
                }
        }
        IDC_TRY_CUDA(cudaMemcpyAsync(pbar, inbar, sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
        return Status::ok();
    };

    // backward pass, one segment (m CK, min((m+1) CK, steps)] at a time
    for (int64_t m = NS - 1; m >= 0; --m) {
        const int64_t n0 = m * CK, n1 = std::min(steps, n0 + CK);
        IDC_TRY_CUDA(cudaMemcpyAsync(inp(0), ckpt(m), sizeof(double) * np, cudaMemcpyDeviceToDevice, stream));
        for (int64_t k = 1; k < n1 - n0; ++k) {   // the segment's step inputs
            IDC_TRY(step_store(inp(k - 1)));
            IDC_TRY_CUDA(cudaMemcpyAsync(inp(k), stage(K, M - 1), sizeof(double) * np, cudaMemcpyDeviceToDevice,
                                         stream));
        }
        for (int64_t s = n1; s > n0; --s) {
            IDC_TRY(step_store(inp(s - n0 - 1)));
            IDC_TRY(adjoint_step());
        }
    }
    if (dpsi0) {   // interior cells; zero ghost cells
        IdcTerms tm{};
        tm.n = 1;
        tm.a[0] = pbar;
        tm.c[0] = 1.0;
        IDC_TRY_CUDA(launch_idc_source(dims(), tm, nullptr, dpsi0, stream));
        launches += 1;
    }
    IDC_TRY(check_device_error());
    if (solves) *solves = nsolve;
    return Status::ok();
}

}  // namespace idc
