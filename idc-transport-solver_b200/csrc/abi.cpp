// The extern "C" boundary declared in include/idcsweep.h: argument checks, host <-> device staging,
// status codes.  Nothing here throws across the boundary.
#include "batch.hpp"
#include "context.hpp"
#include "idcsweep.h"

#include <cmath>
#include <cstring>
#include <new>
#include <string>

struct idc_batch {
    idc::Batch impl;
};

struct idc_ctx {
    idc::Context impl;
    explicit idc_ctx(const idc_problem_desc &d) : impl(d) {}
};

namespace {

thread_local std::string g_last_error;

}  // namespace

namespace idc {
void set_last_error(const std::string &msg) { g_last_error = msg; }
}  // namespace idc

namespace {

int fail(const idc::Status &s) {
    g_last_error = s.msg;
    return s.code;
}

int fail(int code, const char *msg) {
    g_last_error = msg;
    return code;
}

#define ABI_TRY(expr)                        \
    do {                                     \
        idc::Status s_ = (expr);             \
        if (!s_.good()) return fail(s_);     \
    } while (0)

#define ABI_TRY_CUDA(expr) ABI_TRY(idc::cuda_status((expr), #expr))

#define ABI_GUARD_BEGIN try {
#define ABI_GUARD_END                                                      \
    }                                                                      \
    catch (const std::bad_alloc &) { return fail(IDC_ERR_NOMEM, "host allocation failed"); } \
    catch (...) { return fail(IDC_ERR_CUDA, "unexpected exception in idcsweep"); }

bool valid_loc(int loc) { return loc == IDC_LOC_HOST || loc == IDC_LOC_DEVICE; }

}  // namespace

namespace {

// The staging shared by the time-dependent adjoints: inputs to the device, the solve, gradients back.
template <typename Run>
int adjoint_time_abi(const char *name, idc_ctx *ctx, const double *psi0, const double *source, const double *detector,
                     double abs_tol, int64_t max_its, double *dsigma_t, double *dsigma_s, double *dsource,
                     double *dpsi0, double *J, int loc, int64_t *solves, Run run) {
    ABI_GUARD_BEGIN
    if (!ctx || !psi0 || !source || !detector) return fail(IDC_ERR_ARG, (std::string(name) + ": null argument").c_str());
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    if (max_its < 0 || !(abs_tol >= 0)) return fail(IDC_ERR_ARG, (std::string(name) + ": bad tolerance").c_str());
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates || !c.have_sigma) return fail(IDC_ERR_STATE, (std::string(name) + " before ordinates and sigma").c_str());
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    ABI_TRY(c.ensure_psi_buffers(3));
    ABI_TRY(c.ensure_phi_buffers(15));
    const double *d_psi0 = psi0, *d_src = source;
    double *d_det = c.phi_buf(11);
    double *d_gt = dsigma_t, *d_gs = dsigma_s, *d_gq = dsource, *d_p0 = dpsi0;
    const cudaMemcpyKind in = loc == IDC_LOC_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (loc == IDC_LOC_HOST) {
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(0), psi0, sizeof(double) * c.psi_len(), in, c.stream));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(1), source, sizeof(double) * c.psi_len(), in, c.stream));
        d_psi0 = c.psi_buf(0);
        d_src = c.psi_buf(1);
        d_gt = dsigma_t ? c.phi_buf(12) : nullptr;   // sigma-sized results fit a moment-sized buffer
        d_gs = dsigma_s ? c.phi_buf(13) : nullptr;
        d_gq = dsource ? c.phi_buf(14) : nullptr;
        d_p0 = dpsi0 ? c.psi_buf(2) : nullptr;
    }
    ABI_TRY_CUDA(cudaMemcpyAsync(d_det, detector, sizeof(double) * c.phi_len(), in, c.stream));
    ABI_TRY_CUDA(idc::launch_zero_ghost_phi(c.dims(), d_det, c.stream));
    double jv = 0.0;
    int64_t ns = 0;
    idc::Status st = run(c, d_psi0, d_src, d_det, d_gt, d_gs, d_gq, d_p0, &jv, &ns);
    if (solves) *solves = ns;
    if (!st.good()) return fail(st);
    if (J) *J = jv;
    if (loc == IDC_LOC_HOST) {
        if (dsigma_t)
            ABI_TRY_CUDA(cudaMemcpyAsync(dsigma_t, d_gt, sizeof(double) * c.sig_len(), cudaMemcpyDeviceToHost, c.stream));
        if (dsigma_s)
            ABI_TRY_CUDA(cudaMemcpyAsync(dsigma_s, d_gs, sizeof(double) * c.sig_len(), cudaMemcpyDeviceToHost, c.stream));
        if (dsource)
            ABI_TRY_CUDA(cudaMemcpyAsync(dsource, d_gq, sizeof(double) * c.phi_len(), cudaMemcpyDeviceToHost, c.stream));
        if (dpsi0)
            ABI_TRY_CUDA(cudaMemcpyAsync(dpsi0, d_p0, sizeof(double) * c.psi_len(), cudaMemcpyDeviceToHost, c.stream));
    }
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

}  // namespace

extern "C" {

const char *idc_strerror(int status) {
    switch (status) {
        case IDC_OK: return "ok";
        case IDC_ERR_ARG: return "invalid argument";
        case IDC_ERR_UNSUPPORTED: return "unsupported configuration";
        case IDC_ERR_CUDA: return "CUDA error";
        case IDC_ERR_TIMEOUT: return "device-side wait timed out";
        case IDC_ERR_NOT_CONVERGED: return "iterative solve did not converge";
        case IDC_ERR_STATE: return "call made in the wrong state";
        case IDC_ERR_NOMEM: return "out of memory";
        default: return "unknown status";
    }
}

const char *idc_last_error_message(void) { return g_last_error.c_str(); }

int idc_ctx_create(const idc_problem_desc *desc, idc_ctx **out) {
    ABI_GUARD_BEGIN
    if (!desc || !out) return fail(IDC_ERR_ARG, "idc_ctx_create: null argument");
    *out = nullptr;
    if (desc->nx < 1 || desc->ny < 1) return fail(IDC_ERR_ARG, "idc_ctx_create: nx and ny must be >= 1");
    if (desc->nx > (1 << 20) || desc->ny > (1 << 20)) return fail(IDC_ERR_ARG, "idc_ctx_create: grid too large");
    if (!(desc->bx > desc->ax) || !(desc->by > desc->ay) || !std::isfinite(desc->bx - desc->ax) ||
        !std::isfinite(desc->by - desc->ay))
        return fail(IDC_ERR_ARG, "idc_ctx_create: empty or non-finite domain");
    if (desc->dg_degree < 0) return fail(IDC_ERR_ARG, "idc_ctx_create: negative DG degree");
    if (desc->dg_degree > 3) return fail(IDC_ERR_UNSUPPORTED, "idc_ctx_create: DG degree > 3 not implemented");
    if (desc->sigma_degree != 0 && desc->sigma_degree != desc->dg_degree)
        return fail(IDC_ERR_ARG, "idc_ctx_create: sigma_degree must be 0 (piecewise constant) or the DG degree");
    if (desc->flags != 0) return fail(IDC_ERR_ARG, "idc_ctx_create: flags must be 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return fail(IDC_ERR_CUDA, "idc_ctx_create: no CUDA device available");
    if (desc->device < 0 || desc->device >= ndev) return fail(IDC_ERR_ARG, "idc_ctx_create: bad device ordinal");
    auto *c = new idc_ctx(*desc);
    idc::Status s = c->impl.init();
    if (!s.good()) {
        delete c;
        return fail(s);
    }
    *out = c;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_ctx_destroy(idc_ctx *ctx) {
    ABI_GUARD_BEGIN
    delete ctx;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_ordinates(idc_ctx *ctx, int64_t nq, const double *xi, const double *eta, const double *w,
                      const int64_t quad_bounds[5]) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    ABI_TRY(ctx->impl.set_ordinates(nq, xi, eta, w, quad_bounds));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_sigma(idc_ctx *ctx, const double *sigma_t, const double *sigma_s, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    ABI_TRY(ctx->impl.set_sigma(sigma_t, sigma_s, loc));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_tiling(idc_ctx *ctx, int32_t ordinates_per_block, int32_t rows_per_block) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    if (ordinates_per_block > 320 || rows_per_block > 320 ||
        (int64_t)ordinates_per_block * rows_per_block > 320)
        return fail(IDC_ERR_ARG, "idc_set_tiling: more than 320 threads per block");
    ABI_TRY(ctx->impl.set_tiling(ordinates_per_block, rows_per_block));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_sweep(idc_ctx *ctx, double *psi_inout, double dt, double *phi_out, int precision, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !psi_inout) return fail(IDC_ERR_ARG, "idc_sweep: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_sweep before idc_set_ordinates");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        ABI_TRY(c.sweep(psi_inout, psi_inout, dt, phi_out, precision));
        ABI_TRY(c.check_device_error());
    } else {
        ABI_TRY(c.ensure_psi_buffers(1));
        ABI_TRY(c.ensure_phi_buffers(3));
        double *d_psi = c.psi_buf(0);
        double *d_phi = phi_out ? c.phi_buf(2) : nullptr;
        ABI_TRY_CUDA(cudaMemcpyAsync(d_psi, psi_inout, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY(c.sweep(d_psi, d_psi, dt, d_phi, precision));
        ABI_TRY_CUDA(cudaMemcpyAsync(psi_inout, d_psi, sizeof(double) * c.psi_len(), cudaMemcpyDeviceToHost, c.stream));
        if (phi_out)
            ABI_TRY_CUDA(cudaMemcpyAsync(phi_out, d_phi, sizeof(double) * c.phi_len(), cudaMemcpyDeviceToHost, c.stream));
        ABI_TRY(c.check_device_error());
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.ev0, c.ev1) == cudaSuccess) c.last_sweep_ms = ms;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_sweep_out(idc_ctx *ctx, const double *source, double *result, double dt, double *phi_out, int precision,
                  int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !source || !result) return fail(IDC_ERR_ARG, "idc_sweep_out: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_sweep_out before idc_set_ordinates");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        ABI_TRY(c.sweep(source, result, dt, phi_out, precision));
        ABI_TRY(c.check_device_error());
    } else {
        ABI_TRY(c.ensure_psi_buffers(2));
        ABI_TRY(c.ensure_phi_buffers(3));
        double *d_src = c.psi_buf(1), *d_res = c.psi_buf(0);
        double *d_phi = phi_out ? c.phi_buf(2) : nullptr;
        ABI_TRY_CUDA(cudaMemcpyAsync(d_src, source, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY(c.sweep(d_src, d_res, dt, d_phi, precision));
        // interior cells only; the caller's ghost cells of result stay as they were
        ABI_TRY_CUDA(c.copy_interior_d2h(result, d_res, c.stream));
        if (phi_out)
            ABI_TRY_CUDA(cudaMemcpyAsync(phi_out, d_phi, sizeof(double) * c.phi_len(), cudaMemcpyDeviceToHost, c.stream));
        ABI_TRY(c.check_device_error());
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.ev0, c.ev1) == cudaSuccess) c.last_sweep_ms = ms;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_sweep_out_many(idc_ctx *ctx, int64_t count, const double *const *sources, double *const *results,
                       double *const *phi_out, double dt, int precision, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || count < 0 || (count > 0 && (!sources || !results))) return fail(IDC_ERR_ARG, "idc_sweep_out_many: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    for (int64_t k = 0; k < count; ++k)
        if (!sources[k] || !results[k]) return fail(IDC_ERR_ARG, "idc_sweep_out_many: null source or result");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_sweep_out_many before idc_set_ordinates");
    if (!c.have_sigma) return fail(IDC_ERR_STATE, "idc_sweep_out_many before idc_set_sigma");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        for (int64_t k = 0; k < count; ++k) ABI_TRY(c.sweep(sources[k], results[k], dt, phi_out ? phi_out[k] : nullptr, precision));
        ABI_TRY(c.check_device_error());
    } else {
        ABI_TRY(c.sweep_host_many(count, sources, results, phi_out, dt, precision));
    }
    return IDC_OK;
    ABI_GUARD_END
}

// Operators: stage through the context's buffers when loc is host.
int idc_pmv(idc_ctx *ctx, double alpha, double beta, const double *psi, double *phi, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !psi || !phi) return fail(IDC_ERR_ARG, "idc_pmv: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_pmv before idc_set_ordinates");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        ABI_TRY(c.pmv(alpha, beta, psi, phi));
    } else {
        ABI_TRY(c.ensure_psi_buffers(1));
        ABI_TRY(c.ensure_phi_buffers(3));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(0), psi, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.phi_buf(2), phi, sizeof(double) * c.phi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY(c.pmv(alpha, beta, c.psi_buf(0), c.phi_buf(2)));
        ABI_TRY_CUDA(cudaMemcpyAsync(phi, c.phi_buf(2), sizeof(double) * c.phi_len(), cudaMemcpyDeviceToHost, c.stream));
    }
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_smv(idc_ctx *ctx, double alpha, double beta, const double *phi, double *psi, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !psi || !phi) return fail(IDC_ERR_ARG, "idc_smv: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_smv before idc_set_ordinates");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        ABI_TRY(c.smv(alpha, beta, phi, psi));
    } else {
        ABI_TRY(c.ensure_psi_buffers(1));
        ABI_TRY(c.ensure_phi_buffers(3));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(0), psi, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.phi_buf(2), phi, sizeof(double) * c.phi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY(c.smv(alpha, beta, c.phi_buf(2), c.psi_buf(0)));
        ABI_TRY_CUDA(cudaMemcpyAsync(psi, c.psi_buf(0), sizeof(double) * c.psi_len(), cudaMemcpyDeviceToHost, c.stream));
    }
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_lmv(idc_ctx *ctx, double alpha, double beta, const double *x, double *y, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !x || !y) return fail(IDC_ERR_ARG, "idc_lmv: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_lmv before idc_set_ordinates");
    if (x == y) return fail(IDC_ERR_ARG, "idc_lmv: x and y must not alias");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        ABI_TRY(c.lmv(alpha, beta, x, y));
    } else {
        ABI_TRY(c.ensure_psi_buffers(2));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(0), x, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(1), y, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY(c.lmv(alpha, beta, c.psi_buf(0), c.psi_buf(1)));
        ABI_TRY_CUDA(cudaMemcpyAsync(y, c.psi_buf(1), sizeof(double) * c.psi_len(), cudaMemcpyDeviceToHost, c.stream));
    }
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_source_iteration(idc_ctx *ctx, double *source_inout, double dt, double abs_tol, int64_t max_its, int precision,
                         int loc, int64_t *iters, double *final_err) {
    ABI_GUARD_BEGIN
    if (!ctx || !source_inout) return fail(IDC_ERR_ARG, "idc_source_iteration: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    if (max_its < 0 || !(abs_tol >= 0)) return fail(IDC_ERR_ARG, "idc_source_iteration: bad tolerance");
    idc::Context &c = ctx->impl;
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    ABI_TRY(c.ensure_psi_buffers(2));
    double *d_src = c.psi_buf(1), *d_psi = c.psi_buf(0);
    const cudaMemcpyKind in = loc == IDC_LOC_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out = loc == IDC_LOC_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    ABI_TRY_CUDA(cudaMemcpyAsync(d_src, source_inout, sizeof(double) * c.psi_len(), in, c.stream));
    // psi starts as the source so that its ghost cells hold the inflow values (SISolver copies
    // Interior|Boundary from the source every iteration, SISolver.cpp:226)
    ABI_TRY_CUDA(cudaMemcpyAsync(d_psi, d_src, sizeof(double) * c.psi_len(), cudaMemcpyDeviceToDevice, c.stream));
    int64_t its = 0;
    double err = 0;
    ABI_TRY(c.source_iteration(d_src, d_psi, dt, abs_tol, max_its, precision, &its, &err));
    ABI_TRY_CUDA(cudaMemcpyAsync(source_inout, d_psi, sizeof(double) * c.psi_len(), out, c.stream));
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    if (iters) *iters = its;
    if (final_err) *final_err = err;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_gmres_solve(idc_ctx *ctx, double *source_inout, double dt, double abs_tol, int32_t restart, int64_t max_its,
                    int precision, int loc, int64_t *iters, double *final_resid) {
    ABI_GUARD_BEGIN
    if (!ctx || !source_inout) return fail(IDC_ERR_ARG, "idc_gmres_solve: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    if (max_its < 0 || !(abs_tol >= 0)) return fail(IDC_ERR_ARG, "idc_gmres_solve: bad tolerance");
    idc::Context &c = ctx->impl;
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    ABI_TRY(c.ensure_psi_buffers(2));
    double *d_src = c.psi_buf(1), *d_psi = c.psi_buf(0);
    const cudaMemcpyKind in = loc == IDC_LOC_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind out = loc == IDC_LOC_HOST ? cudaMemcpyDeviceToHost : cudaMemcpyDeviceToDevice;
    ABI_TRY_CUDA(cudaMemcpyAsync(d_src, source_inout, sizeof(double) * c.psi_len(), in, c.stream));
    ABI_TRY_CUDA(cudaMemcpyAsync(d_psi, d_src, sizeof(double) * c.psi_len(), cudaMemcpyDeviceToDevice, c.stream));
    int64_t its = 0;
    double res = 0;
    idc::Status st = c.gmres_peierls(d_src, d_psi, dt, abs_tol, restart, max_its, precision, &its, &res);
    if (iters) *iters = its;
    if (final_resid) *final_resid = res;
    if (!st.good()) return fail(st);
    ABI_TRY_CUDA(cudaMemcpyAsync(source_inout, d_psi, sizeof(double) * c.psi_len(), out, c.stream));
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_preconditioner(idc_ctx *ctx, int kind, int32_t inner_steps) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    ABI_TRY(ctx->impl.set_preconditioner(kind, inner_steps));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_idc_integrate(idc_ctx *ctx, double *psi_inout, const double *source, double dt, int64_t steps,
                      int32_t num_nodes, int32_t num_corrections, int scattering, int precision, double abs_tol,
                      int32_t restart, int64_t max_its, int use_graph, int loc, int64_t *sweeps) {
    ABI_GUARD_BEGIN
    if (!ctx || !psi_inout || !source) return fail(IDC_ERR_ARG, "idc_idc_integrate: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    double *d_psi = psi_inout;
    const double *d_src = source;
    if (loc == IDC_LOC_HOST) {
        ABI_TRY(c.ensure_psi_buffers(2));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(0), psi_inout, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice,
                                     c.stream));
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(1), source, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice,
                                     c.stream));
        d_psi = c.psi_buf(0);
        d_src = c.psi_buf(1);
    }
    int64_t n_sweeps = 0;
    idc::Status st = c.idc_integrate(d_psi, d_src, dt, steps, num_nodes, num_corrections, scattering, precision,
                                     abs_tol, restart, max_its, use_graph != 0, &n_sweeps);
    if (sweeps) *sweeps = n_sweeps;
    if (!st.good()) return fail(st);
    if (loc == IDC_LOC_HOST)
        ABI_TRY_CUDA(cudaMemcpyAsync(psi_inout, d_psi, sizeof(double) * c.psi_len(), cudaMemcpyDeviceToHost, c.stream));
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_sweep_fused(idc_ctx *ctx, const double *source, double *result, double dt, const double *phi_scatter,
                    double scatter_scale, double *phi_out, int precision, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "idc_sweep_fused: null context");
    if (loc != IDC_LOC_DEVICE) return fail(IDC_ERR_ARG, "idc_sweep_fused takes device pointers only");
    idc::Context &c = ctx->impl;
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    ABI_TRY(c.sweep(source, result, dt, phi_out, precision, phi_scatter, scatter_scale));
    ABI_TRY(c.check_device_error());
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.ev0, c.ev1) == cudaSuccess) c.last_sweep_ms = ms;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_tile_shape(idc_ctx *ctx, int32_t seg, int32_t warps) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    ABI_TRY(ctx->impl.set_tile_shape(seg, warps));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_autotune(idc_ctx *ctx, const double *source, double dt, int precision, int32_t *seg, int32_t *warps) {
    ABI_GUARD_BEGIN
    if (!ctx || !source) return fail(IDC_ERR_ARG, "idc_autotune: null argument");
    idc::Context &c = ctx->impl;
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    int s = 0, w = 0;
    ABI_TRY(c.autotune(source, dt, precision, &s, &w));
    if (seg) *seg = s;
    if (warps) *warps = w;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_create(idc_batch **out) {
    ABI_GUARD_BEGIN
    if (!out) return fail(IDC_ERR_ARG, "idc_batch_create: null argument");
    *out = new (std::nothrow) idc_batch();
    if (!*out) return fail(IDC_ERR_NOMEM, "idc_batch_create: out of host memory");
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_add(idc_batch *b, idc_ctx *ctx) {
    ABI_GUARD_BEGIN
    if (!b || !ctx) return fail(IDC_ERR_ARG, "idc_batch_add: null argument");
    ABI_TRY(b->impl.add(&ctx->impl));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_sweep(idc_batch *b, const double *const *sources, double *const *results, double *const *phi_out,
                    double dt, int precision) {
    ABI_GUARD_BEGIN
    if (!b) return fail(IDC_ERR_ARG, "idc_batch_sweep: null batch");
    ABI_TRY(b->impl.sweep(sources, results, nullptr, 1.0, phi_out, dt, precision));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_autotune(idc_batch *b, const double *const *sources, double *const *results, double dt, int precision) {
    ABI_GUARD_BEGIN
    if (!b) return fail(IDC_ERR_ARG, "idc_batch_autotune: null batch");
    ABI_TRY(b->impl.autotune(sources, results, dt, precision));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_set_shape(idc_batch *b, int dg_degree, int precision, int32_t seg, int32_t warps) {
    ABI_GUARD_BEGIN
    if (!b) return fail(IDC_ERR_ARG, "null batch");
    ABI_TRY(b->impl.set_shape((int)dg_degree + 1, precision, seg, warps));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_get_shape(idc_batch *b, int dg_degree, int precision, int32_t *seg, int32_t *warps) {
    if (!b || !seg || !warps) return fail(IDC_ERR_ARG, "idc_batch_get_shape: null argument");
    int s = 0, w = 0;
    b->impl.get_shape((int)dg_degree + 1, precision, &s, &w);
    *seg = s;
    *warps = w;
    return IDC_OK;
}

int idc_batch_last_timing(idc_batch *b, double *ms) {
    if (!b) return fail(IDC_ERR_ARG, "null batch");
    if (ms) *ms = b->impl.last_ms;
    return IDC_OK;
}

int idc_batch_gmres_solve(idc_batch *b, double *const *psi_inout, double dt, double abs_tol, int32_t restart,
                          int64_t max_its, int precision, int64_t *iters, double *final_resids) {
    ABI_GUARD_BEGIN
    if (!b || !psi_inout) return fail(IDC_ERR_ARG, "idc_batch_gmres_solve: null argument");
    if (max_its < 0 || !(abs_tol >= 0)) return fail(IDC_ERR_ARG, "idc_batch_gmres_solve: bad tolerance");
    ABI_TRY(b->impl.gmres_solve(psi_inout, dt, abs_tol, restart, max_its, precision, iters, final_resids));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_batch_destroy(idc_batch *b) {
    delete b;
    return IDC_OK;
}

int idc_sweep_adjoint(idc_ctx *ctx, const double *source, double *result, double dt, double *moments_out, int precision,
                      int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !source || !result) return fail(IDC_ERR_ARG, "idc_sweep_adjoint: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates) return fail(IDC_ERR_STATE, "idc_sweep_adjoint before idc_set_ordinates");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    if (loc == IDC_LOC_DEVICE) {
        ABI_TRY(c.sweep(source, result, dt, moments_out, precision, nullptr, 1.0, true));
        ABI_TRY(c.check_device_error());
    } else {
        ABI_TRY(c.ensure_psi_buffers(2));
        ABI_TRY(c.ensure_phi_buffers(3));
        double *d_src = c.psi_buf(1), *d_res = c.psi_buf(0);
        double *d_mom = moments_out ? c.phi_buf(2) : nullptr;
        ABI_TRY_CUDA(cudaMemcpyAsync(d_src, source, sizeof(double) * c.psi_len(), cudaMemcpyHostToDevice, c.stream));
        ABI_TRY(c.sweep(d_src, d_res, dt, d_mom, precision, nullptr, 1.0, true));
        ABI_TRY_CUDA(c.copy_interior_d2h(result, d_res, c.stream));
        if (moments_out)
            ABI_TRY_CUDA(cudaMemcpyAsync(moments_out, d_mom, sizeof(double) * c.phi_len(), cudaMemcpyDeviceToHost,
                                         c.stream));
        ABI_TRY(c.check_device_error());
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, c.ev0, c.ev1) == cudaSuccess) c.last_sweep_ms = ms;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_adjoint_grad(idc_ctx *ctx, const double *psi, const double *detector, double dt, double abs_tol,
                     int32_t restart, int64_t max_its, int precision, double *dsigma_t, double *dsigma_s,
                     double *dsource, int loc, int64_t *iters, double *final_resid) {
    ABI_GUARD_BEGIN
    if (!ctx || !psi || !detector) return fail(IDC_ERR_ARG, "idc_adjoint_grad: null argument");
    if (!valid_loc(loc)) return fail(IDC_ERR_ARG, "bad loc");
    if (max_its < 0 || !(abs_tol >= 0)) return fail(IDC_ERR_ARG, "idc_adjoint_grad: bad tolerance");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates || !c.have_sigma) return fail(IDC_ERR_STATE, "idc_adjoint_grad before ordinates and sigma");
    ABI_TRY_CUDA(cudaSetDevice(c.device));
    c.launches = 0;
    ABI_TRY(c.ensure_psi_buffers(2));
    ABI_TRY(c.ensure_phi_buffers(14));
    const double *d_psi = psi;
    double *d_det = c.phi_buf(10);
    double *d_gt = dsigma_t, *d_gs = dsigma_s, *d_gq = dsource;
    const cudaMemcpyKind in = loc == IDC_LOC_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (loc == IDC_LOC_HOST) {
        ABI_TRY_CUDA(cudaMemcpyAsync(c.psi_buf(1), psi, sizeof(double) * c.psi_len(), in, c.stream));
        d_psi = c.psi_buf(1);
        d_gt = dsigma_t ? c.phi_buf(11) : nullptr;   // sigma-sized results fit a moment-sized buffer
        d_gs = dsigma_s ? c.phi_buf(12) : nullptr;
        d_gq = dsource ? c.phi_buf(13) : nullptr;
    }
    ABI_TRY_CUDA(cudaMemcpyAsync(d_det, detector, sizeof(double) * c.phi_len(), in, c.stream));
    ABI_TRY_CUDA(idc::launch_zero_ghost_phi(c.dims(), d_det, c.stream));
    int64_t its = 0;
    double res = 0;
    idc::Status st = c.adjoint_gradient(d_psi, d_det, dt, abs_tol, restart, max_its, precision, d_gt, d_gs, d_gq, &its,
                                        &res);
    if (iters) *iters = its;
    if (final_resid) *final_resid = res;
    if (!st.good()) return fail(st);
    if (loc == IDC_LOC_HOST) {
        if (dsigma_t)
            ABI_TRY_CUDA(cudaMemcpyAsync(dsigma_t, d_gt, sizeof(double) * c.sig_len(), cudaMemcpyDeviceToHost, c.stream));
        if (dsigma_s)
            ABI_TRY_CUDA(cudaMemcpyAsync(dsigma_s, d_gs, sizeof(double) * c.sig_len(), cudaMemcpyDeviceToHost, c.stream));
        if (dsource)
            ABI_TRY_CUDA(cudaMemcpyAsync(dsource, d_gq, sizeof(double) * c.phi_len(), cudaMemcpyDeviceToHost, c.stream));
    }
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}


int idc_adjoint_transient(idc_ctx *ctx, const double *psi0, const double *source, double dt, int64_t steps,
                          const double *detector, int64_t checkpoint_every, double abs_tol, int32_t restart,
                          int64_t max_its, int precision, double *dsigma_t, double *dsigma_s, double *dsource,
                          double *dpsi0, double *J, int loc, int64_t *solves) {
    return adjoint_time_abi(
        "idc_adjoint_transient", ctx, psi0, source, detector, abs_tol, max_its, dsigma_t, dsigma_s, dsource, dpsi0, J,
        loc, solves,
        [&](idc::Context &c, const double *p0, const double *q, const double *det, double *gt, double *gs, double *gq,
            double *gp, double *jv, int64_t *ns) {
            return c.adjoint_transient(p0, q, dt, steps, det, checkpoint_every, abs_tol, restart, max_its, precision,
                                       gt, gs, gq, gp, jv, ns);
        });
}

int idc_adjoint_idc(idc_ctx *ctx, const double *psi0, const double *source, double dt, int64_t steps,
                    int32_t num_nodes, int32_t num_corrections, const double *detector, int64_t checkpoint_every,
                    double abs_tol, int32_t restart, int64_t max_its, int precision, double *dsigma_t,
                    double *dsigma_s, double *dsource, double *dpsi0, double *J, int loc, int64_t *solves) {
    return adjoint_time_abi(
        "idc_adjoint_idc", ctx, psi0, source, detector, abs_tol, max_its, dsigma_t, dsigma_s, dsource, dpsi0, J, loc,
        solves,
        [&](idc::Context &c, const double *p0, const double *q, const double *det, double *gt, double *gs, double *gq,
            double *gp, double *jv, int64_t *ns) {
            return c.adjoint_idc(p0, q, dt, steps, num_nodes, num_corrections, det, checkpoint_every, abs_tol, restart,
                                 max_its, precision, gt, gs, gq, gp, jv, ns);
        });
}

int idc_lmv_transpose(idc_ctx *ctx, double alpha, double beta, const double *x, double *y, int loc) {
    ABI_GUARD_BEGIN
    if (!ctx || !x || !y) return fail(IDC_ERR_ARG, "idc_lmv_transpose: null argument");
    if (loc != IDC_LOC_DEVICE) return fail(IDC_ERR_ARG, "idc_lmv_transpose: device arrays only");
    idc::Context &c = ctx->impl;
    if (!c.have_ordinates || !c.have_sigma) return fail(IDC_ERR_STATE, "idc_lmv_transpose before ordinates and sigma");
    ABI_TRY(c.lmv_transpose(alpha, beta, x, y));
    ABI_TRY_CUDA(cudaStreamSynchronize(c.stream));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_spin_limit(idc_ctx *ctx, int64_t polls) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    ctx->impl.spin_limit = polls > 0 ? (long long)polls : idc::Context::kDefaultSpinLimit;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_periodic(idc_ctx *ctx, int32_t periodic) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    if (periodic != 0 && periodic != 1) return fail(IDC_ERR_ARG, "idc_set_periodic: 0 or 1");
    ABI_TRY(ctx->impl.set_periodic(periodic == 1));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_reflecting(idc_ctx *ctx, int32_t edges) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    ABI_TRY(ctx->impl.set_reflecting((int)edges));
    return IDC_OK;
    ABI_GUARD_END
}

int idc_set_allreduce(idc_ctx *ctx, idc_allreduce_fn fn, void *user) {
    ABI_GUARD_BEGIN
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    ctx->impl.allreduce_fn = fn;
    ctx->impl.allreduce_user = fn ? user : nullptr;
    return IDC_OK;
    ABI_GUARD_END
}

int idc_last_timing(idc_ctx *ctx, double *sweep_kernel_ms, int64_t *kernels_launched) {
    if (!ctx) return fail(IDC_ERR_ARG, "null context");
    if (sweep_kernel_ms) *sweep_kernel_ms = ctx->impl.last_sweep_ms;
    if (kernels_launched) *kernels_launched = ctx->impl.launches;
    return IDC_OK;
}

}  // extern "C"
