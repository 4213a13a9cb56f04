// C++ host layer, see context.hpp.
#include "context.hpp"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace idc {

Status cuda_status(cudaError_t e, const char *what) {
    if (e == cudaSuccess) return Status::ok();
    Status s;
    s.code = (e == cudaErrorMemoryAllocation) ? IDC_ERR_NOMEM : IDC_ERR_CUDA;
    s.msg = std::string(what) + ": " + cudaGetErrorString(e);
    return s;
}

#define IDC_TRY_CUDA(expr)                                   \
    do {                                                     \
        cudaError_t e_ = (expr);                             \
        if (e_ != cudaSuccess) return cuda_status(e_, #expr); \
    } while (0)

#define IDC_TRY(expr)                     \
    do {                                  \
        Status s_ = (expr);               \
        if (!s_.good()) return s_;        \
    } while (0)

static Status bad(int code, const std::string &m) {
    Status s;
    s.code = code;
    s.msg = m;
    return s;
}

Context::Context(const idc_problem_desc &d) : desc(d) {}

Context::~Context() {
    if (device >= 0) cudaSetDevice(device);
    for (double *p : psi_bufs_) cudaFree(p);
    for (double *p : phi_bufs_) cudaFree(p);
    for (double *p : idc_psi_) cudaFree(p);
    for (double *p : idc_phi_) cudaFree(p);
    for (double *p : transient_bufs_) cudaFree(p);
    for (double *p : adj_idc_bufs_) cudaFree(p);
    cudaFree(d_ones_);
    cudaFree(d_rmap);
    cudaFree(d_reflect_);
    cudaFree(d_reflect_g_);
    cudaFree(d_reflect_vec_);
    cudaFree(d_scalar_);
    cudaFree(d_xi);
    cudaFree(d_eta);
    cudaFree(d_w);
    cudaFree(d_sigma_t);
    cudaFree(d_sigma_s);
    cudaFree(other_sched_.d_items);
    cudaFree(other_sched_.d_trace);
    cudaFree(d_sig_mom_);
    cudaFree(d_tens_t_);
    cudaFree(d_tens_s_);
    cudaFree(d_cat_t_);
    cudaFree(d_work_psi_);
    cudaFree(d_items);
    cudaFree(d_sync);
    cudaFree(d_phi_part);
    cudaFree(d_trace);
    cudaFree(d_inflow);
    cudaFree(d_scat);
    cudaFree(d_src2mix);
    cudaFree(d_msrc);
    cudaFree(d_krylov);
    cudaFree(d_small);
    cudaFreeHost(h_small);
    cudaFree(d_dsa_ws);
    for (int b = 0; b < 2; ++b) {
        if (ev_in[b]) cudaEventDestroy(ev_in[b]);
        if (ev_done[b]) cudaEventDestroy(ev_done[b]);
        if (ev_out[b]) cudaEventDestroy(ev_out[b]);
    }
    if (copy_in) cudaStreamDestroy(copy_in);
    if (copy_out) cudaStreamDestroy(copy_out);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
}

Status Context::init() {
    nx = desc.nx;
    ny = desc.ny;
    P = (int)desc.dg_degree + 1;
    N = P * P;
    dx = (desc.bx - desc.ax) / (double)nx;
    dy = (desc.by - desc.ay) / (double)ny;
    device = desc.device;
    IDC_TRY_CUDA(cudaSetDevice(device));
    IDC_TRY_CUDA(cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device));
    IDC_TRY_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    IDC_TRY_CUDA(cudaEventCreate(&ev0));
    IDC_TRY_CUDA(cudaEventCreate(&ev1));
    IDC_TRY_CUDA(cudaMalloc(&d_scalar_, sizeof(double) * (4 + multidot_scratch_doubles())));   // + dot scratch
    // IDC_SWEEP_KERNEL=modal|warp|rowsync selects another sweep kernel than the lane-pipelined one
    if (const char *k = std::getenv("IDC_SWEEP_KERNEL")) {
        const std::string v(k);
        kernel = v == "rowsync" ? kRowSync : v == "warp" ? kWarp : v == "modal" ? kModal : kLane;
    }
    use_warp_kernel = kernel != kRowSync;
    // IDC_MOMENTS_FAST_PATH=0 sweeps the Krylov iterations through the per-ordinate transforms as well
    if (const char *f = std::getenv("IDC_MOMENTS_FAST_PATH")) moments_fast_path = std::string(f) != "0";
    return Status::ok();
}

Status Context::set_ordinates(int64_t nq_in, const double *xi, const double *eta, const double *w,
                              const int64_t qb[5]) {
    if (nq_in <= 0 || !xi || !eta || !w || !qb) return bad(IDC_ERR_ARG, "set_ordinates: null or empty input");
    if (qb[0] != 0 || qb[4] != nq_in) return bad(IDC_ERR_ARG, "set_ordinates: quad_bounds must run 0..nq");
    for (int k = 0; k < 4; ++k)
        if (qb[k + 1] < qb[k]) return bad(IDC_ERR_ARG, "set_ordinates: quad_bounds not monotone");
    // every ordinate must lie strictly inside its quadrant (OrdinateSet::SetSigns, OrdinateSet.cpp:658-700)
    for (int k = 0; k < 4; ++k)
        for (int64_t q = qb[k]; q < qb[k + 1]; ++q) {
            const bool xneg = k >= 2, yneg = (k & 1) != 0;
            if (!(std::isfinite(xi[q]) && std::isfinite(eta[q]) && std::isfinite(w[q])))
                return bad(IDC_ERR_ARG, "set_ordinates: non-finite ordinate");
            if ((xneg ? !(xi[q] < 0) : !(xi[q] > 0)) || (yneg ? !(eta[q] < 0) : !(eta[q] > 0)))
                return bad(IDC_ERR_ARG, "set_ordinates: ordinate " + std::to_string(q) + " outside quadrant " +
                                            std::to_string(k));
        }
    IDC_TRY_CUDA(cudaSetDevice(device));
    cudaFree(d_xi);
    cudaFree(d_eta);
    cudaFree(d_w);
    d_xi = d_eta = d_w = nullptr;
    IDC_TRY_CUDA(cudaMalloc(&d_xi, sizeof(double) * nq_in));
    IDC_TRY_CUDA(cudaMalloc(&d_eta, sizeof(double) * nq_in));
    IDC_TRY_CUDA(cudaMalloc(&d_w, sizeof(double) * nq_in));
    IDC_TRY_CUDA(cudaMemcpy(d_xi, xi, sizeof(double) * nq_in, cudaMemcpyHostToDevice));
    IDC_TRY_CUDA(cudaMemcpy(d_eta, eta, sizeof(double) * nq_in, cudaMemcpyHostToDevice));
    IDC_TRY_CUDA(cudaMemcpy(d_w, w, sizeof(double) * nq_in, cudaMemcpyHostToDevice));
    if (nq_in != nq) {
        // psi-sized buffers (and the unweighted-sum weights) depend on nq
        for (auto *v : {&psi_bufs_, &idc_psi_, &transient_bufs_, &adj_idc_bufs_}) {
            for (double *p : *v) cudaFree(p);
            v->clear();
        }
        cudaFree(d_ones_);
        d_ones_ = nullptr;
        cudaFree(d_reflect_);
        d_reflect_ = nullptr;
        cudaFree(d_reflect_g_);   // sized by nq and the reflecting edges
        d_reflect_g_ = nullptr;
        reflect_g_len_ = 0;
        cudaFree(d_reflect_vec_);
        d_reflect_vec_ = nullptr;
        reflect_vec_len_ = 0;
        cudaFree(d_work_psi_);
        d_work_psi_ = nullptr;
    }
    nq = nq_in;
    for (int k = 0; k < 5; ++k) quad[k] = qb[k];
    have_ordinates = true;
    invalidate_schedules();   // rebuilt lazily
    if (reflect_mask) return update_reflect_map();
    return Status::ok();
}

// The reflection partner of every ordinate in x (-xi, eta) and in y (xi, -eta), found as the reference's
// OrdinateData::ComputeReflectMap finds it (utils/Quadrule/OrdinateSet.cpp:1093-1140: coordinates equal
// within 1e-14).
Status Context::update_reflect_map() {
    std::vector<double> xi(nq), eta(nq);
    IDC_TRY_CUDA(cudaMemcpy(xi.data(), d_xi, sizeof(double) * nq, cudaMemcpyDeviceToHost));
    IDC_TRY_CUDA(cudaMemcpy(eta.data(), d_eta, sizeof(double) * nq, cudaMemcpyDeviceToHost));
    std::vector<int> map(2 * (size_t)nq, -1);
    for (int dim = 0; dim < 2; ++dim)
        for (int64_t q = 0; q < nq; ++q) {
            for (int64_t k = 0; k < nq; ++k) {
                const double dx_ = dim == 0 ? xi[q] + xi[k] : xi[q] - xi[k];
                const double dy_ = dim == 1 ? eta[q] + eta[k] : eta[q] - eta[k];
                if (std::fabs(dx_) < 1e-14 && std::fabs(dy_) < 1e-14) {
                    map[(size_t)dim * nq + q] = (int)k;
                    break;
                }
            }
            if (map[(size_t)dim * nq + q] < 0)
                return bad(IDC_ERR_ARG, "reflecting boundaries: ordinate " + std::to_string(q) +
                                            " has no reflection partner in dimension " + std::to_string(dim));
        }
    cudaFree(d_rmap);
    d_rmap = nullptr;
    IDC_TRY_CUDA(cudaMalloc(&d_rmap, sizeof(int) * map.size()));
    IDC_TRY_CUDA(cudaMemcpy(d_rmap, map.data(), sizeof(int) * map.size(), cudaMemcpyHostToDevice));
    return Status::ok();
}

Status Context::set_reflecting(int mask) {
    if (mask < 0 || mask > 15) return bad(IDC_ERR_ARG, "reflecting edges: bits 1 x-min, 2 x-max, 4 y-min, 8 y-max");
    if (mask && periodic_) return bad(IDC_ERR_UNSUPPORTED, "reflecting edges on a periodic grid");
    IDC_TRY_CUDA(cudaSetDevice(device));
    const int old = reflect_mask;
    reflect_mask = mask;
    if (mask && have_ordinates) {
        Status st = update_reflect_map();
        if (!st.good()) {
            reflect_mask = old;
            return st;
        }
    }
    return Status::ok();
}

// A sweep whose source carries the scattering term with high-order cross sections: the term is formed by the
// tensor Smv into the array first, as the reference's solvers apply Smv into the array before Apply
// (SISolver.cpp:226-232, PETScPeierlsSolver.cpp:504-505 and :551-552), then the array is swept in place.
Status Context::sweep_tensor_source(const double *src, double *out, double dt, double *phi, int precision,
                                    const double *phi_scatter, double scatter_scale) {
    double *w = out;
    if (!w) {
        if (!d_work_psi_) {
            if (capturing) return bad(IDC_ERR_STATE, "work array allocation inside a stream capture");
            IDC_TRY_CUDA(cudaMalloc(&d_work_psi_, sizeof(double) * psi_len()));
        }
        w = d_work_psi_;
    }
    if (src) {
        if (w != src)
            IDC_TRY_CUDA(cudaMemcpyAsync(w, src, sizeof(double) * psi_len(), cudaMemcpyDeviceToDevice, stream));
    } else {
        IDC_TRY_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * psi_len(), stream));
    }
    IDC_TRY_CUDA(launch_smv_tensor(dims(), scatter_scale, 1.0, d_tens_s_, phi_scatter, w, stream));
    launches += 1;
    return sweep(w, out, dt, phi, precision);
}

// A sweep with reflecting boundaries, as the reference's SweepPatternUniCartWavefront::Sweep makes it
// (linear_solvers/Abstract/SweepPattern/SweepPatternUniCartWavefront.cpp:186-251): the quadrants one after
// another in its default order 3, 2, 1, 0 (SweepPatternUniCart.cpp:33-36), in place, and after each the
// reflecting edges' ghost cells refilled from the current interior values (OrdinateFlux::ReflectBoundaries).
// The array starts as the reference's in-place array does: the source, with the fused scattering term
// materialised (the reference applies Smv into the array before Apply), so a quadrant swept before its
// reflection partner reads the ghost values the array came with.
Status Context::sweep_reflecting(const double *src, double *out, double dt, double *phi, int precision,
                                 const double *phi_scatter, double scatter_scale, bool adjoint, const double *src2) {
    if (adjoint || src2)
        return bad(IDC_ERR_UNSUPPORTED, "reflecting boundaries: forward sweeps with one source only");
    if (kernel_for(precision) != kLane)
        return bad(IDC_ERR_UNSUPPORTED,
                   "reflecting boundaries need the lane kernel: FP64 or FP32 sweeps at a lane tile shape");
    if (allreduce_fn)
        return bad(IDC_ERR_UNSUPPORTED, "reflecting boundaries with ordinates partitioned over ranks");
    double *w = out;
    if (!w) {
        if (!d_reflect_) {
            if (capturing) return bad(IDC_ERR_STATE, "reflecting-sweep buffer allocation inside a stream capture");
            IDC_TRY_CUDA(cudaMalloc(&d_reflect_, sizeof(double) * psi_len()));
        }
        w = d_reflect_;
    }
    if (src) {
        if (w != src)
            IDC_TRY_CUDA(cudaMemcpyAsync(w, src, sizeof(double) * psi_len(), cudaMemcpyDeviceToDevice, stream));
    } else {
        IDC_TRY_CUDA(cudaMemsetAsync(w, 0, sizeof(double) * psi_len(), stream));
    }
    if (phi_scatter) {   // TransportOperator::Smv(scale, 1, sigma_s, phi -> w)
        IDC_TRY_CUDA(launch_smv(dims(), scatter_scale, 1.0, d_sigma_s, phi_scatter, w, stream));
        launches += 1;
    }
    return reflect_quadrants(w, dt, phi, precision);
}

// The reference's quadrant sequence 3, 2, 1, 0 (a reflection after each) in as few launches as give the same
// result.  Quadrant k (0: xi > 0, eta > 0; 1: xi > 0, eta < 0; 2: xi < 0, eta > 0; 3: xi < 0, eta < 0) reads
// ghost cells on its x-inflow edge (x-min if xi > 0) and y-inflow edge (y-min if eta > 0); where that edge
// reflects, the reference hands it the mirror of partner quadrant k ^ 2 (x) or k ^ 1 (y) as the partner stands
// after the quadrants swept before k.  Launch levels L (a reflection after each launch) keep that when
//   * a partner swept before k in the reference is in an earlier launch: L(k) > L(partner);
//   * a partner swept after k is not in an earlier launch: L(partner) >= L(k) (k must see it unswept);
//   * k other than the first quadrant, 3, with a reflecting inflow is not in the first launch: the first
//     launch reads the input's ghost cells, k reads a reflection.
// Quadrants of one launch read nothing another of them writes, and the reflection after a launch is that of
// the current interior, as after the reference's last quadrant.  The least levels meeting these (a fixed
// point; quadrant 3 stays at 0) give, e.g., all edges: {3}, {2, 1}, {0}; x-min: {3, 2}, {1, 0}; y-min: {3, 1},
// {2, 0}.  Returns the launches' quadrant masks in order.
static std::vector<int> reflect_launches(int mask) {
    auto before = [](int p, int k) { return p > k; };   // the reference sweeps 3, 2, 1, 0
    int L[4] = {0, 0, 0, 0};
    for (int k = 0; k < 4; ++k) {
        const int xedge = (k & 2) ? 2 : 1, yedge = (k & 1) ? 8 : 4;   // xi < 0: x-max; eta < 0: y-max
        if (k != 3 && (mask & (xedge | yedge))) L[k] = 1;
    }
    for (bool changed = true; changed;) {
        changed = false;
        for (int k = 0; k < 4; ++k) {
            const int xedge = (k & 2) ? 2 : 1, yedge = (k & 1) ? 8 : 4;
            for (int e = 0; e < 2; ++e) {
                if (!(mask & (e == 0 ? xedge : yedge))) continue;
                const int p = e == 0 ? (k ^ 2) : (k ^ 1);
                if (before(p, k) && L[k] < L[p] + 1) {
                    L[k] = L[p] + 1;
                    changed = true;
                }
                if (!before(p, k) && L[p] < L[k]) {
                    L[p] = L[k];
                    changed = true;
                }
            }
        }
    }
    std::vector<int> groups;
    for (int level = 0; level < 4; ++level) {
        int m = 0;
        for (int k = 0; k < 4; ++k)
            if (L[k] == level) m |= 1 << k;
        if (m) groups.push_back(m);
    }
    return groups;
}

// The sequential-quadrant sweep proper, in place on a prepared array w; phi (optional) gets the moments of
// all four quadrants.
Status Context::reflect_quadrants(double *w, double dt, double *phi, int precision) {
    in_reflect_ = true;
    Status st = Status::ok();
    const std::vector<int> launches_q = reflect_launches(reflect_mask);
    for (size_t g = 0; g < launches_q.size(); ++g) {
        const int mask = launches_q[g];
        quad_mask_ = mask;
        skip_reduce_ = g + 1 < launches_q.size();   // the chunk partials of every quadrant are summed after the last
        st = sweep(w, w, dt, phi, precision);
        if (!st.good()) break;
        cudaError_t e = launch_reflect_boundaries(dims(), reflect_mask, d_xi, d_eta, d_rmap, w, stream);
        if (e != cudaSuccess) {
            st = cuda_status(e, "launch_reflect_boundaries");
            break;
        }
        launches += 1;
    }
    in_reflect_ = false;
    quad_mask_ = 0;
    skip_reduce_ = false;
    return st;
}

Status Context::reflect_ghosts(double *psi, double *packed, bool to_packed) {
    IDC_TRY_CUDA(launch_reflect_ghosts(dims(), ghost_mask(), d_xi, d_eta, psi, packed, to_packed, stream));
    launches += 1;
    return Status::ok();
}

Status Context::set_periodic(bool on) {
    if (on && reflect_mask) return bad(IDC_ERR_UNSUPPORTED, "reflecting edges on a periodic grid");
    periodic_ = on;
    return Status::ok();
}

// SISolver::Solve with Global::periodic: psi starts at zero, and each iteration first synchronises the halos
// that the last sweep left dirty (SISolver.cpp:223; SynchronizeHalos copies the opposite interior edge into
// every ghost cell of the four edges, objects/Abstract/DensityFunction.cpp:927-960), then copies the source
// with OpDomain::Interior | OpDomain::Boundary, which on a periodic grid is the interior alone
// (DomainDecomposition::DetermineOffsets, objects/DomainDecomposition.cpp:271-330).  The sweep then reads the
// last iterate's periodic images as its inflow.
Status Context::source_iteration_periodic(const double *src, double *psi_out, double dt, double abs_tol,
                                          int64_t max_its, int precision, int64_t *iters, double *err) {
    if (src == psi_out) return bad(IDC_ERR_ARG, "source iteration: source and psi must be different arrays");
    IDC_TRY(ensure_phi_buffers(2));
    double *phi_cur = phi_buf(0), *phi_last = phi_buf(1);
    IDC_TRY_CUDA(cudaMemsetAsync(phi_cur, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(cudaMemsetAsync(phi_last, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(cudaMemsetAsync(psi_out, 0, sizeof(double) * psi_len(), stream));
    int64_t it = 0;
    double e = INFINITY;
    while (it < max_its && e > abs_tol) {
        ++it;
        std::swap(phi_cur, phi_last);
        if (it > 1) IDC_TRY_CUDA(launch_periodic_halos(dims(), psi_out, stream));
        IDC_TRY_CUDA(launch_copy_interior(dims(), src, psi_out, stream));
        launches += it > 1 ? 2 : 1;
        IDC_TRY(smv(1.0, 1.0, phi_last, psi_out));
        IDC_TRY(sweep(psi_out, psi_out, dt, phi_cur, precision));
        IDC_TRY(l2dist(phi_cur, phi_last, &e));
        IDC_TRY(check_device_error());
    }
    if (iters) *iters = it;
    if (err) *err = e;
    return Status::ok();
}

// SISolver::Solve (linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:190-254) with reflecting edges.  psi
// starts at zero (SetInitialGuess(nullptr)), and each iteration copies the source with OpDomain::Interior |
// OpDomain::Boundary, which leaves out the reflecting edges' ghost cells (DomainDecomposition::DetermineOffsets,
// objects/DomainDecomposition.cpp:271-330): the reflections left by one sweep are the inflow that the next
// sweep's quadrants read before their partners are swept.  The fixed point is the reflecting problem's solution.
Status Context::source_iteration_reflecting(const double *src, double *psi_out, double dt, double abs_tol,
                                            int64_t max_its, int precision, int64_t *iters, double *err) {
    if (src == psi_out) return bad(IDC_ERR_ARG, "source iteration: source and psi must be different arrays");
    const size_t ng = reflect_ghost_len(dims(), reflect_mask);
    if (reflect_g_len_ < ng) {
        if (capturing) return bad(IDC_ERR_STATE, "reflecting-sweep buffer allocation inside a stream capture");
        cudaFree(d_reflect_g_);
        d_reflect_g_ = nullptr;
        reflect_g_len_ = 0;
        IDC_TRY_CUDA(cudaMalloc(&d_reflect_g_, sizeof(double) * ng));
        reflect_g_len_ = ng;
    }
    IDC_TRY(ensure_phi_buffers(2));
    double *phi_cur = phi_buf(0), *phi_last = phi_buf(1);
    IDC_TRY_CUDA(cudaMemsetAsync(phi_cur, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(cudaMemsetAsync(phi_last, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(cudaMemsetAsync(psi_out, 0, sizeof(double) * psi_len(), stream));
    int64_t it = 0;
    double e = INFINITY;
    while (it < max_its && e > abs_tol) {
        ++it;
        std::swap(phi_cur, phi_last);
        IDC_TRY(reflect_ghosts(psi_out, d_reflect_g_, true));    // keep the reflections of the last sweep
        IDC_TRY_CUDA(cudaMemcpyAsync(psi_out, src, sizeof(double) * psi_len(), cudaMemcpyDeviceToDevice, stream));
        IDC_TRY(reflect_ghosts(psi_out, d_reflect_g_, false));
        IDC_TRY_CUDA(launch_smv(dims(), 1.0, 1.0, d_sigma_s, phi_last, psi_out, stream));
        launches += 1;
        IDC_TRY(reflect_quadrants(psi_out, dt, phi_cur, precision));
        IDC_TRY(l2dist(phi_cur, phi_last, &e));
        IDC_TRY(check_device_error());
    }
    if (iters) *iters = it;
    if (err) *err = e;
    return Status::ok();
}

namespace {

// The integrals over [-1, 1] of P_a P_b P_c for degrees a, b, c < P (Global::TPI, utils/global.cpp:67-110, which
// evaluates them by Gauss-Legendre quadrature): here from the monomial coefficients of the Legendre polynomials
// (Bonnet's recurrence) and the exact monomial integrals 2 / (k + 1) for even k; values below 5e-16 are zero,
// as the reference clears them.
TripleProducts triple_products(int P) {
    const double c[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {-0.5, 0, 1.5, 0}, {0, -1.5, 0, 2.5}};   // P_0..P_3
    TripleProducts t{};
    for (int a = 0; a < P; ++a)
        for (int b = 0; b < P; ++b)
            for (int cc = 0; cc < P; ++cc) {
                double v = 0.0;
                for (int i = 0; i < 4; ++i)
                    for (int j = 0; j < 4; ++j)
                        for (int k = 0; k < 4; ++k) {
                            const int deg = i + j + k;
                            if (deg % 2 == 0) v += c[a][i] * c[b][j] * c[cc][k] * (2.0 / (deg + 1));
                        }
                t.v[a + P * (b + P * cc)] = std::fabs(v) < 5e-16 ? 0.0 : v;
            }
    return t;
}

}  // namespace

Status Context::set_sigma(const double *sigma_t, const double *sigma_s, int loc) {
    if (!sigma_t) return bad(IDC_ERR_ARG, "set_sigma: sigma_t is null");
    IDC_TRY_CUDA(cudaSetDevice(device));
    if (!d_sigma_t) IDC_TRY_CUDA(cudaMalloc(&d_sigma_t, sizeof(double) * sig_len()));
    if (!d_sigma_s) IDC_TRY_CUDA(cudaMalloc(&d_sigma_s, sizeof(double) * sig_len()));
    const cudaMemcpyKind kind = loc == IDC_LOC_HOST ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToDevice;
    if (high_order_sigma()) {   // Legendre moments [cell][u][v] of both cross sections
        const size_t nm = sig_len() * N, nt = sig_len() * N * N;
        if (!d_sig_mom_) IDC_TRY_CUDA(cudaMalloc(&d_sig_mom_, sizeof(double) * nm));
        if (!d_tens_t_) IDC_TRY_CUDA(cudaMalloc(&d_tens_t_, sizeof(double) * nt));
        if (!d_tens_s_) IDC_TRY_CUDA(cudaMalloc(&d_tens_s_, sizeof(double) * nt));
        if (!d_cat_t_) IDC_TRY_CUDA(cudaMalloc(&d_cat_t_, sizeof(double) * nt));
        const TripleProducts tpi = triple_products(P);
        IDC_TRY_CUDA(cudaMemcpyAsync(d_sig_mom_, sigma_t, sizeof(double) * nm, kind, stream));
        IDC_TRY_CUDA(launch_sigma_tensor(dims(), d_sig_mom_, tpi, dx * dy / 4.0, d_sigma_t, d_tens_t_, d_cat_t_, stream));
        if (sigma_s)
            IDC_TRY_CUDA(cudaMemcpyAsync(d_sig_mom_, sigma_s, sizeof(double) * nm, kind, stream));
        else
            IDC_TRY_CUDA(cudaMemsetAsync(d_sig_mom_, 0, sizeof(double) * nm, stream));
        IDC_TRY_CUDA(launch_sigma_tensor(dims(), d_sig_mom_, tpi, 0.0, d_sigma_s, d_tens_s_, nullptr, stream));
        IDC_TRY_CUDA(cudaStreamSynchronize(stream));
        have_sigma = true;
        return Status::ok();
    }
    IDC_TRY_CUDA(cudaMemcpy(d_sigma_t, sigma_t, sizeof(double) * sig_len(), kind));
    if (sigma_s)
        IDC_TRY_CUDA(cudaMemcpy(d_sigma_s, sigma_s, sizeof(double) * sig_len(), kind));
    else
        IDC_TRY_CUDA(cudaMemset(d_sigma_s, 0, sizeof(double) * sig_len()));
    have_sigma = true;
    return Status::ok();
}

Status Context::set_tiling(int G, int R) {
    if (G < 0 || R < 0) return bad(IDC_ERR_ARG, "set_tiling: negative tile size");
    user_G = G;
    user_R = R;
    invalidate_schedules();
    return Status::ok();
}

// The kernel of a sweep at `precision`: with the default (kLane) the one the tile shape names (warps = 0:
// the lane kernel, else the modal kernel), and without a tile shape the lane kernel; the lane kernel
// sweeps in FP64 only, the FP32 modes run on the modal kernel.  IDC_SWEEP_KERNEL fixes another kernel.
int Context::kernel_for(int precision) const {
    if (high_order_sigma() || P > 3) return kWarp;   // the elimination kernel takes a full cell matrix
    if (kernel != kLane) return kernel;
    if (tune_seg > 0 && tune_wn > 0) return kModal;
    return sweep_lane_supports(P, precision, tune_seg > 0 ? tune_seg : 4) ? kLane : kModal;
}

Status Context::set_tile_shape(int s, int w) {
    if (s == 0 && w == 0) {
        tune_seg = tune_wn = 0;
    } else {
        if ((s != 4 && s != 8 && s != 16 && s != 32) || w < 0 || w > 7 || (w == 0 && s == 32))
            return bad(IDC_ERR_ARG, "tile shape: seg must be 4, 8, 16 or 32 and wn in 0..7 (0: the lane kernel, "
                                    "seg 4, 8 or 16)");
        tune_seg = s;
        tune_wn = w;
    }
    invalidate_schedules();
    return Status::ok();
}

// Candidate tile shapes, timed with CUDA events on this problem (best of three sweeps after a warm-up).
Status Context::autotune(const double *src, double dt, int precision, int *seg_out, int *wn_out) {
    if (high_order_sigma()) return bad(IDC_ERR_UNSUPPORTED, "high-order cross sections use the elimination kernel");
    if (!modal_family()) return bad(IDC_ERR_UNSUPPORTED, "the autotuner tunes the lane and modal kernels");
    IDC_TRY(ensure_psi_buffers(1));
    IDC_TRY(ensure_phi_buffers(1));
    float best = 1e30f;
    int bs = 0, bw = 0;
    // candidates: the lane kernel's segment widths (warps = 0; FP64 and the default kernel choice only), then
    // the modal kernel's segment widths and compute-warp counts
    const bool lane = kernel == kLane && sweep_lane_supports(P, precision, 4);
    const int mw = sweep_modal_max_wn(P);
    for (int cs : {4, 8, 16, 32})
        for (int cw = lane ? 0 : std::max(1, mw - 3); cw <= mw; cw = cw == 0 ? std::max(1, mw - 3) : cw + 1) {
            if (cw == 0 && !sweep_lane_supports(P, precision, cs)) continue;
            IDC_TRY(set_tile_shape(cs, cw));
            float ms = 1e30f;
            for (int rep = 0; rep < 4; ++rep) {   // one warm-up, then the best of three
                IDC_TRY(sweep(src, psi_buf(0), dt, phi_buf(0), precision));
                IDC_TRY(check_device_error());
                float t = 0.f;
                IDC_TRY_CUDA(cudaEventElapsedTime(&t, ev0, ev1));
                if (rep > 0) ms = std::min(ms, t);
            }
            if (ms < best) {
                best = ms;
                bs = cs;
                bw = cw;
            }
        }
    IDC_TRY(set_tile_shape(bs, bw));
    if (seg_out) *seg_out = bs;
    if (wn_out) *wn_out = bw;
    return Status::ok();
}

Status Context::ensure_psi_buffers(int count) {
    IDC_TRY_CUDA(cudaSetDevice(device));
    while ((int)psi_bufs_.size() < count) {
        double *p = nullptr;
        IDC_TRY_CUDA(cudaMalloc(&p, sizeof(double) * psi_len()));
        psi_bufs_.push_back(p);
    }
    return Status::ok();
}

Status Context::ensure_phi_buffers(int count) {
    IDC_TRY_CUDA(cudaSetDevice(device));
    while ((int)phi_bufs_.size() < count) {
        double *p = nullptr;
        IDC_TRY_CUDA(cudaMalloc(&p, sizeof(double) * phi_len()));
        IDC_TRY_CUDA(cudaMemset(p, 0, sizeof(double) * phi_len()));
        phi_bufs_.push_back(p);
    }
    return Status::ok();
}

// Tile shape of the warp and modal kernels: ordinates of a quadrant are split into nch chunks of at most
// G ordinates, each chunk on a row segment of `seg` lanes (a power of two, at least 4); a warp holds
// 32/seg rows and a CTA wn compute warps (at most max_wn, default default_wn; the modal kernel adds a
// helper warp and its aux warps, the warp kernel the helper warp).  The warp kernel prefers wide
// segments; the modal kernel the narrowest segment with the best lane use (4 lanes, 8 rows per warp:
// measured fastest on B200 at S4..S16).
static void choose_warp_tiling(int qmax, int user_G, int user_rows, int max_wn, int default_wn, bool narrow,
                               int *G_out, int *seg_out, int *wn_out) {
    int seg = 16, G = 0;
    if (user_G > 0) {
        G = std::min(user_G, 32);
        seg = 4;
        while (seg < G) seg <<= 1;
    } else {
        // from wide to narrow: a narrower segment must use its lanes clearly better (> 10 points) to win,
        // since every extra chunk adds moment atomics and work items
        double best = -1.0;
        for (int k = 0; k < 4; ++k) {
            const int cand = narrow ? (4 << k) : (32 >> k);
            const int nch = (qmax + cand - 1) / cand;
            const int g = (qmax + nch - 1) / nch;
            const double eff = (double)qmax / (nch * cand);
            if (eff > best + (narrow ? 1e-9 : 0.1)) {
                best = eff;
                seg = cand;
                G = g;
            }
        }
    }
    const int rw = 32 / seg;
    int wn = user_rows > 0 ? std::max(1, user_rows / rw) : default_wn;
    wn = std::min(wn, max_wn);
    *G_out = G;
    *seg_out = seg;
    *wn_out = wn;
}

// Work items in row-block-major order: (row block, quadrant, ordinate chunk).
void Context::use_schedule(int variant) {
    if (variant == sched_variant_) return;
    ScheduleSlot &o = other_sched_;
    std::swap(tiling, o.tiling);
    std::swap(d_items, o.d_items);
    std::swap(d_trace, o.d_trace);
    std::swap(trace_len, o.trace_len);
    std::swap(smem, o.smem);
    std::swap(n_items, o.n_items);
    std::swap(items_per_rb, o.items_per_rb);
    for (int k = 0; k < 5; ++k) std::swap(quad_slots[k], o.quad_slots[k]);
    std::swap(seg, o.seg);
    std::swap(wn, o.wn);
    std::swap(active, o.active);
    std::swap(grid, o.grid);
    std::swap(block, o.block);
    std::swap(occupancy_precision, o.occupancy_precision);
    sched_variant_ = variant;
}

Status Context::build_schedule(int precision) {
    if (n_items > 0 && occupancy_precision == precision) return Status::ok();
    // the lane kernel's schedule does not depend on the precision (the same tiling rules, traces and grid for
    // its FP64 and FP32 instances): a switch between them, as FP32 Krylov sweeps inside FP64 refinement make
    // on every refinement pass, keeps it instead of reallocating and re-arming the traces
    if (n_items > 0 && active == kLane && kernel_for(precision) == kLane) {
        occupancy_precision = precision;
        return Status::ok();
    }
    int qmax = 0;
    for (int k = 0; k < 4; ++k) qmax = std::max<int>(qmax, (int)(quad[k + 1] - quad[k]));
    if (qmax == 0) return bad(IDC_ERR_ARG, "no ordinates");
    int G = 0, R = 0;
    active = kernel_for(precision);
    const int max_wn = active == kModal ? sweep_modal_max_wn(P) : active == kLane ? 1 : 7;
    const bool modal_like = active == kModal || active == kLane;
    // a fixed or autotuned tile shape is the full sweeps'; the moments-only sweeps keep the default rule
    if (use_warp_kernel && tune_seg > 0 && sched_variant_ == 0) {
        seg = tune_seg;
        if (active == kLane && !sweep_lane_supports(P, precision, seg)) seg = 16;
        wn = tune_wn > 0 ? std::min(tune_wn, max_wn) : (active == kModal ? sweep_modal_default_wn(P) : 1);
        const int nch = (qmax + seg - 1) / seg;
        G = (qmax + nch - 1) / nch;
        if (active == kModal) wn = sweep_modal_fit_wn(P, precision, wn, G, seg);
        R = wn * (32 / seg);
    } else if (use_warp_kernel) {
        choose_warp_tiling(qmax, user_G, user_R, max_wn, active == kModal ? sweep_modal_default_wn(P) : max_wn,
                           modal_like, &G, &seg, &wn);
        if (active == kLane && sched_variant_ == 0 && user_G == 0 && user_R == 0 && (P == 3 || (P == 2 && qmax <= 24))) {
            // full lane sweeps: at DG degree 2 16-wide segments (fewer row blocks, 16-wide moment sums) were the
            // fastest at S8, S12 and S16 on 256^2 grids; at degree 1 8-wide ones for up to 24 ordinates per quadrant
            // (S8, S12: 4-7% ahead of 4-wide, also on the 64^2 lattice), while S16's 36 keep the 4-wide rule
            seg = P == 3 ? 16 : 8;
            const int nch = (qmax + seg - 1) / seg;
            G = (qmax + nch - 1) / nch;
        }
        if (active == kLane && !sweep_lane_supports(P, precision, seg)) {   // 32 lanes: 16 and two chunks
            seg = 16;
            const int nch = (qmax + seg - 1) / seg;
            G = (qmax + nch - 1) / nch;
        }
        if (active == kModal) wn = sweep_modal_fit_wn(P, precision, wn, G, seg);
        if (active == kWarp) {   // fewer warps per block where the rings outgrow shared memory (DG degree 3)
            int limit = 0;
            IDC_TRY_CUDA(cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
            while (wn > 1 && sweep_warp_smem_bytes(P, wn, G, seg) > (size_t)limit) --wn;
        }
        R = wn * (32 / seg);
    } else {
        const int max_threads = 320;
        G = user_G > 0 ? user_G : std::min(qmax, P == 3 ? 36 : 64);
        if (G > max_threads) G = max_threads;
        R = user_R > 0 ? user_R : std::max(1, std::min(16, max_threads / G));
        if (G * R > max_threads) R = std::max(1, max_threads / G);
        if (R > ny) R = (int)ny;
    }
    tiling.G = G;
    tiling.R = R;
    const int nrb = (int)((ny + R - 1) / R);

    std::vector<SweepItem> items;
    // chunks of each quadrant, balanced: ceil(count / G) chunks of near-equal size
    std::vector<std::vector<std::pair<int, int>>> chunks(4);
    for (int k = 0; k < 4; ++k) {
        const int cnt = (int)(quad[k + 1] - quad[k]);
        if (cnt == 0) continue;
        const int nch = (cnt + G - 1) / G;
        int beg = (int)quad[k];
        for (int c = 0; c < nch; ++c) {
            const int sz = cnt / nch + (c < cnt % nch ? 1 : 0);
            chunks[k].push_back({beg, sz});
            beg += sz;
        }
    }
    quad_slots[0] = 0;   // the partial-moment slots (items of a row block) of each quadrant
    for (int k = 0; k < 4; ++k) quad_slots[k + 1] = quad_slots[k] + (int)chunks[k].size();
    std::vector<int> prev_index;   // index of the same (quadrant, chunk) in the previous row block
    for (int rb = 0; rb < nrb; ++rb) {
        std::vector<int> cur_index;
        int slot = 0;
        for (int k = 0; k < 4; ++k)
            for (auto &ch : chunks[k]) {
                SweepItem it;
                it.quadrant = k;
                it.q_begin = ch.first;
                it.q_count = ch.second;
                it.row_block = rb;
                it.dep = rb == 0 ? -1 : prev_index[slot];
                cur_index.push_back((int)items.size());
                items.push_back(it);
                ++slot;
            }
        prev_index = cur_index;
    }
    n_items = (int)items.size();
    items_per_rb = n_items / nrb;

    IDC_TRY_CUDA(cudaSetDevice(device));
    cudaFree(d_items);
    d_items = nullptr;
    IDC_TRY_CUDA(cudaMalloc(&d_items, sizeof(SweepItem) * items.size()));
    IDC_TRY_CUDA(cudaMemcpy(d_items, items.data(), sizeof(SweepItem) * items.size(), cudaMemcpyHostToDevice));
    if (sync_cap_ < 2 + items.size()) {   // shared by both schedules: the larger one's progress flags
        int err_word = 0;
        if (d_sync) IDC_TRY_CUDA(cudaMemcpy(&err_word, d_sync + 1, sizeof(int), cudaMemcpyDeviceToHost));
        cudaFree(d_sync);
        d_sync = nullptr;
        sync_cap_ = 0;
        IDC_TRY_CUDA(cudaMalloc(&d_sync, sizeof(int) * (2 + items.size())));
        sync_cap_ = 2 + items.size();
        IDC_TRY_CUDA(cudaMemset(d_sync, 0, sizeof(int) * sync_cap_));
        IDC_TRY_CUDA(cudaMemcpy(d_sync + 1, &err_word, sizeof(int), cudaMemcpyHostToDevice));   // kept until checked
    }

    if (use_warp_kernel) {
        cudaFree(d_trace);
        d_trace = nullptr;
        const size_t tl = (size_t)n_items * nx * G * (modal_like ? P : N);
        IDC_TRY_CUDA(cudaMalloc(&d_trace, sizeof(double) * tl));
        trace_len = tl;
        IDC_TRY_CUDA(launch_fill_u64(reinterpret_cast<unsigned long long *>(d_trace), tl, kTraceSentinel, stream));
        IDC_TRY_CUDA(cudaStreamSynchronize(stream));
    }

    int per_sm = 0;
    if (active == kLane) {
        block = sweep_lane_warps() * 32;
        smem = 0;   // fixed per kernel instance (set by the launcher)
        IDC_TRY_CUDA(sweep_lane_occupancy(P, seg, false, &per_sm));
    } else if (active == kModal) {
        block = sweep_modal_threads(P, wn);
        smem = sweep_modal_smem_bytes(P, precision, wn, G, seg);
        IDC_TRY_CUDA(sweep_modal_occupancy(P, precision, seg, block, smem, &per_sm));
    } else if (active == kWarp) {
        block = (wn + 1) * 32;
        smem = sweep_warp_smem_bytes(P, wn, G, seg);
        IDC_TRY_CUDA(sweep_warp_occupancy(P, precision, block, smem, &per_sm));
    } else {
        block = ((G * R + 31) / 32) * 32;
        smem = sweep_smem_bytes(P, R, G);
        IDC_TRY_CUDA(sweep_occupancy(P, precision, block, smem, &per_sm));
    }
    if (per_sm < 1) return bad(IDC_ERR_UNSUPPORTED, "sweep kernel does not fit on an SM with this tiling");
    if (active == kLane)   // one item per warp at a time
        grid = std::min((n_items + sweep_lane_warps() - 1) / sweep_lane_warps(), per_sm * num_sms);
    else
        grid = std::min(n_items, per_sm * num_sms);
    occupancy_precision = precision;
    return Status::ok();
}

// The interior cells of a psi array, device -> host, as one strided copy: nx runs of ny cells (the
// interior j range of one column i), (ny + 2) cells apart in both arrays.
cudaError_t Context::copy_interior_d2h(double *host, const double *dev, cudaStream_t s) const {
    const size_t cell = (size_t)nq * N * sizeof(double);
    const size_t off = ((size_t)1 * (ny + 2) + 1) * (size_t)nq * N;
    return cudaMemcpy2DAsync(host + off, (ny + 2) * cell, dev + off, (ny + 2) * cell, ny * cell, (size_t)nx,
                             cudaMemcpyDeviceToHost, s);
}

Status Context::sweep_host_many(int64_t count, const double *const *srcs, double *const *outs,
                                double *const *phis, double dt, int precision) {
    if (count < 1) return Status::ok();
    IDC_TRY_CUDA(cudaSetDevice(device));
    IDC_TRY(ensure_psi_buffers(4));   // sources in 0, 1; results in 2, 3
    IDC_TRY(ensure_phi_buffers(5));   // moments in 3, 4
    if (!copy_in) {
        IDC_TRY_CUDA(cudaStreamCreateWithFlags(&copy_in, cudaStreamNonBlocking));
        IDC_TRY_CUDA(cudaStreamCreateWithFlags(&copy_out, cudaStreamNonBlocking));
        for (int b = 0; b < 2; ++b) {
            IDC_TRY_CUDA(cudaEventCreateWithFlags(&ev_in[b], cudaEventDisableTiming));
            IDC_TRY_CUDA(cudaEventCreateWithFlags(&ev_done[b], cudaEventDisableTiming));
            IDC_TRY_CUDA(cudaEventCreateWithFlags(&ev_out[b], cudaEventDisableTiming));
        }
    }
    for (int64_t k = 0; k < count; ++k) {
        const int b = (int)(k & 1);
        double *d_src = psi_buf(b), *d_res = psi_buf(2 + b), *d_phi = phis ? phi_buf(3 + b) : nullptr;
        // upload, once the sweep two steps back has read this source buffer
        if (k >= 2) IDC_TRY_CUDA(cudaStreamWaitEvent(copy_in, ev_done[b], 0));
        IDC_TRY_CUDA(cudaMemcpyAsync(d_src, srcs[k], sizeof(double) * psi_len(), cudaMemcpyHostToDevice, copy_in));
        IDC_TRY_CUDA(cudaEventRecord(ev_in[b], copy_in));
        // sweep, once the source is in and the download two steps back has read this result buffer
        IDC_TRY_CUDA(cudaStreamWaitEvent(stream, ev_in[b], 0));
        if (k >= 2) IDC_TRY_CUDA(cudaStreamWaitEvent(stream, ev_out[b], 0));
        IDC_TRY(sweep(d_src, d_res, dt, d_phi, precision));
        IDC_TRY_CUDA(cudaEventRecord(ev_done[b], stream));
        // download the interior cells (the caller's ghost cells stay as they were) and the moments
        IDC_TRY_CUDA(cudaStreamWaitEvent(copy_out, ev_done[b], 0));
        IDC_TRY_CUDA(copy_interior_d2h(outs[k], d_res, copy_out));
        if (phis && phis[k])
            IDC_TRY_CUDA(cudaMemcpyAsync(phis[k], d_phi, sizeof(double) * phi_len(), cudaMemcpyDeviceToHost, copy_out));
        IDC_TRY_CUDA(cudaEventRecord(ev_out[b], copy_out));
    }
    IDC_TRY_CUDA(cudaStreamSynchronize(copy_out));
    IDC_TRY_CUDA(cudaStreamSynchronize(copy_in));
    return check_device_error();
}

Status Context::check_device_error() {
    int err = 0;
    IDC_TRY_CUDA(cudaMemcpyAsync(&err, d_sync + 1, sizeof(int), cudaMemcpyDeviceToHost, stream));
    IDC_TRY_CUDA(cudaStreamSynchronize(stream));
    if (err != kDevOk) {
        IDC_TRY_CUDA(cudaMemsetAsync(d_sync + 1, 0, sizeof(int), stream));
        if (d_trace)
            IDC_TRY_CUDA(launch_fill_u64(reinterpret_cast<unsigned long long *>(d_trace), trace_len, kTraceSentinel, stream));
        if (other_sched_.d_trace)   // the other variant's schedule: its sweeps may have been the abandoned ones
            IDC_TRY_CUDA(launch_fill_u64(reinterpret_cast<unsigned long long *>(other_sched_.d_trace),
                                         other_sched_.trace_len, kTraceSentinel, stream));
        IDC_TRY_CUDA(cudaStreamSynchronize(stream));
        return bad(IDC_ERR_TIMEOUT, "a device-side wait gave up (bounded spin); the sweep was abandoned");
    }
    return Status::ok();
}

Status Context::sweep(const double *src, double *out, double dt, double *phi, int precision,
                      const double *phi_scatter, double scatter_scale, bool adjoint, const double *src2,
                      double src2_scale) {
    if (!have_ordinates) return bad(IDC_ERR_STATE, "sweep before idc_set_ordinates");
    if (!have_sigma) return bad(IDC_ERR_STATE, "sweep before idc_set_sigma");
    if (precision < 0 || precision > 2) return bad(IDC_ERR_ARG, "unknown precision");
    if (!(dt > 0)) return bad(IDC_ERR_ARG, "dt must be positive (+inf for steady state)");
    if ((!src || !out) && !use_warp_kernel)
        return bad(IDC_ERR_UNSUPPORTED, "a sweep without source or output array needs the warp-pipelined kernel");
    if (adjoint && (!modal_family() || precision == IDC_PREC_FP32))
        return bad(IDC_ERR_UNSUPPORTED, "the transposed sweep needs the modal kernel in FP64 or refined precision");
    if (src2 && (adjoint || !modal_family() || !src))
        return bad(IDC_ERR_UNSUPPORTED, "a second source needs a forward modal sweep with a first source");
    if (P > 3 && precision != IDC_PREC_FP64)
        return bad(IDC_ERR_UNSUPPORTED, "DG degree 3: FP64 sweeps (the elimination kernel)");
    if (high_order_sigma()) {
        if (precision != IDC_PREC_FP64)
            return bad(IDC_ERR_UNSUPPORTED, "high-order cross sections: FP64 sweeps (the elimination kernel)");
        if (adjoint || src2)
            return bad(IDC_ERR_UNSUPPORTED, "high-order cross sections: forward sweeps with one source only");
        if (phi_scatter) return sweep_tensor_source(src, out, dt, phi, precision, phi_scatter, scatter_scale);
    }
    if (reflect_mask && !in_reflect_)
        return sweep_reflecting(src, out, dt, phi, precision, phi_scatter, scatter_scale, adjoint, src2);
    use_schedule((!src && !out && phi && !adjoint && !src2 && moments_fast_path) ? 1 : 0);
    IDC_TRY(build_schedule(precision));
    IDC_TRY_CUDA(cudaSetDevice(device));

    size_t launch_smem = smem;
    if (src2 && active == kLane && precision == IDC_PREC_FP64) {
        // the lane kernel has its own instance with the second source's stages
    } else if (src2) {
        int limit = 0;
        IDC_TRY_CUDA(cudaDeviceGetAttribute(&limit, cudaDevAttrMaxSharedMemoryPerBlockOptin, device));
        if (precision != IDC_PREC_FP32 && smem + sweep_modal_src2_bytes(P, wn) <= (size_t)limit) {
            launch_smem = smem + sweep_modal_src2_bytes(P, wn);
        } else {   // no in-sweep variant for this precision, or its stages do not fit: combine first
            if (src2mix_len < psi_len()) {
                if (capturing) return bad(IDC_ERR_STATE, "source buffer allocation inside a stream capture");
                cudaFree(d_src2mix);
                d_src2mix = nullptr;
                src2mix_len = 0;
                IDC_TRY_CUDA(cudaMalloc(&d_src2mix, sizeof(double) * psi_len()));
                src2mix_len = psi_len();
            }
            IdcTerms tm{};
            tm.n = 1;
            tm.a[0] = src2;
            tm.c[0] = src2_scale;
            IDC_TRY_CUDA(launch_idc_source(dims(), tm, src, d_src2mix, stream));
            launches += 1;
            src = d_src2mix;
            src2 = nullptr;
        }
    }

    SweepArgs a{};
    a.src = src;
    a.src2 = src2;
    a.src2_scale = src2_scale;
    a.out = out;
    a.sigma_t = d_sigma_t;
    a.sigma_s = d_sigma_s;
    a.sigma_t_mat = high_order_sigma() ? d_cat_t_ : nullptr;
    a.phi_scatter = phi_scatter;
    a.scatter_scale = scatter_scale;
    a.phi = phi;
    a.xi = d_xi;
    a.eta = d_eta;
    a.w = d_w;
    a.nx = (int)nx;
    a.ny = (int)ny;
    a.nq = (int)nq;
    a.dx = dx;
    a.dy = dy;
    a.inv_dt = 1.0 / dt;
    a.items = d_items;
    a.n_items = n_items;
    a.R = tiling.R;
    a.G = tiling.G;
    a.quad_mask = quad_mask_;
    a.n_refine = 1;
    a.seg = seg;
    a.wn = wn;
    a.trace = d_trace;
    a.trace_stride = (size_t)nx * tiling.G * ((active == kModal || active == kLane) ? P : N);
    a.next_item = d_sync;
    a.error = d_sync + 1;
    a.progress = d_sync + 2;
    a.spin_limit = spin_limit;
    a.adjoint = adjoint ? 1 : 0;

    // the warp kernel writes per-chunk partial moments, summed afterwards in a fixed order
    if (use_warp_kernel && phi) {
        const size_t need = (size_t)items_per_rb * phi_len();
        if (phi_part_len < need) {
            cudaFree(d_phi_part);
            d_phi_part = nullptr;
            phi_part_len = 0;
            IDC_TRY_CUDA(cudaMalloc(&d_phi_part, sizeof(double) * need));
            phi_part_len = need;
        }
        a.phi = nullptr;
        a.phi_part = d_phi_part;
        a.phi_slots = items_per_rb;
        a.phi_slot_stride = phi_len();
    }

    // moments-only forward sweeps (the Krylov iterations) on the lane kernel: no per-ordinate transforms
    const bool phi_only = active == kLane && !src && !out && phi && !adjoint && !src2 && a.phi_part && moments_fast_path;

    // queue head and progress flags start at zero; the error word is kept until checked
    IDC_TRY_CUDA(cudaMemsetAsync(d_sync, 0, sizeof(int), stream));
    IDC_TRY_CUDA(cudaMemsetAsync(d_sync + 2, 0, sizeof(int) * n_items, stream));
    if (a.phi) IDC_TRY_CUDA(cudaMemsetAsync(phi, 0, sizeof(double) * phi_len(), stream));
    if (active != kModal && active != kLane && !capturing) IDC_TRY_CUDA(cudaEventRecord(ev0, stream));
    if (active == kModal || active == kLane) {
        if (src && !adjoint) {   // inflow traces of the ghost cells (packed modal, or physical for the refined mode)
            const size_t need = (size_t)(nx + ny) * nq * P;
            if (inflow_len < need) {
                cudaFree(d_inflow);
                d_inflow = nullptr;
                inflow_len = 0;
                IDC_TRY_CUDA(cudaMalloc(&d_inflow, sizeof(double) * need));
                inflow_len = need;
            }
            IDC_TRY_CUDA(launch_inflow_traces(P, precision != IDC_PREC_FP32_REFINED, src, d_xi, d_eta, (int)nx,
                                              (int)ny, (int)nq, d_inflow, stream));
            launches += 1;
            a.inflow = d_inflow;
        }
        if (phi_scatter && !adjoint) {   // the scattering source's moments, once per cell instead of per ordinate
            if (scat_len < phi_len()) {
                if (capturing) return bad(IDC_ERR_STATE, "scattering buffer allocation inside a stream capture");
                cudaFree(d_scat);
                d_scat = nullptr;
                scat_len = 0;
                IDC_TRY_CUDA(cudaMalloc(&d_scat, sizeof(double) * phi_len()));
                scat_len = phi_len();
            }
            IDC_TRY_CUDA(launch_scatter_moments(dims(), d_sigma_s, phi_scatter, d_scat, stream));
            launches += 1;
            a.phi_scatter = d_scat;
            a.sigma_s = nullptr;
        }
        if (phi_only) {   // the scattering source in the packed modal basis, once per (cell, quadrant)
            const size_t need = sig_len() * 4 * N;
            if (msrc_len < need) {
                if (capturing) return bad(IDC_ERR_STATE, "modal source buffer allocation inside a stream capture");
                cudaFree(d_msrc);
                d_msrc = nullptr;
                msrc_len = 0;
                IDC_TRY_CUDA(cudaMalloc(&d_msrc, sizeof(double) * need));
                msrc_len = need;
            }
            IDC_TRY_CUDA(launch_modal_sources(dims(), a.phi_scatter, scatter_scale, d_msrc, stream));
            launches += 1;
            a.modal_src = d_msrc;
            a.phi_scatter = nullptr;
        }
        if (!capturing) IDC_TRY_CUDA(cudaEventRecord(ev0, stream));   // the timing covers the sweep kernel alone
        if (active == kLane)
            IDC_TRY_CUDA(launch_sweep_lane(P, precision, a, grid, stream));
        else
            IDC_TRY_CUDA(launch_sweep_modal(P, precision, a, grid, launch_smem, stream));
    } else if (active == kWarp)
        IDC_TRY_CUDA(launch_sweep_warp(P, precision, a, grid, smem, stream));
    else
        IDC_TRY_CUDA(launch_sweep(P, precision, a, grid, block, smem, stream));
    if (!capturing) IDC_TRY_CUDA(cudaEventRecord(ev1, stream));
    launches += 1;
    if (a.phi_part && phi_only) {
        IDC_TRY_CUDA(launch_reduce_modal_partials(dims(), d_phi_part, quad_slots, phi_len(), phi, stream));
        launches += 1;
    } else if (a.phi_part && !skip_reduce_) {
        IDC_TRY_CUDA(launch_reduce_phi_partials(dims(), d_phi_part, items_per_rb, phi_len(), phi, stream));
        launches += 1;
    }
    if (phi && allreduce_fn) {   // this rank's ordinates gave partial moments: complete them over the ranks
        if (capturing) return bad(IDC_ERR_STATE, "an all-reduce hook cannot run inside a stream capture");
        IDC_TRY_CUDA(cudaStreamSynchronize(stream));
        const int rc = allreduce_fn(phi, (int64_t)phi_len(), allreduce_user);
        if (rc != 0) return bad(IDC_ERR_STATE, "the all-reduce hook failed (returned " + std::to_string(rc) + ")");
    }
    return Status::ok();
}

Status Context::pmv(double alpha, double beta, const double *psi, double *phi) {
    if (!have_ordinates) return bad(IDC_ERR_STATE, "pmv before idc_set_ordinates");
    IDC_TRY_CUDA(cudaSetDevice(device));
    IDC_TRY_CUDA(launch_pmv(dims(), alpha, beta, d_w, psi, phi, stream));
    launches += 1;
    return Status::ok();
}

Status Context::smv(double alpha, double beta, const double *phi, double *psi) {
    if (!have_ordinates) return bad(IDC_ERR_STATE, "smv before idc_set_ordinates");
    if (!have_sigma) return bad(IDC_ERR_STATE, "smv before idc_set_sigma");
    IDC_TRY_CUDA(cudaSetDevice(device));
    if (high_order_sigma())
        IDC_TRY_CUDA(launch_smv_tensor(dims(), alpha, beta, d_tens_s_, phi, psi, stream));
    else
        IDC_TRY_CUDA(launch_smv(dims(), alpha, beta, d_sigma_s, phi, psi, stream));
    launches += 1;
    return Status::ok();
}

Status Context::lmv(double alpha, double beta, const double *x, double *y) {
    if (!have_ordinates) return bad(IDC_ERR_STATE, "lmv before idc_set_ordinates");
    if (!have_sigma) return bad(IDC_ERR_STATE, "lmv before idc_set_sigma");
    IDC_TRY_CUDA(cudaSetDevice(device));
    if (periodic_) {   // the upwind neighbours across an edge are the opposite edge's cells (Lmv synchronises
                       // its input's halos first, TransportOperator.cpp:1232): a copy of x with its halos synced
        if (!d_work_psi_) {
            if (capturing) return bad(IDC_ERR_STATE, "work array allocation inside a stream capture");
            IDC_TRY_CUDA(cudaMalloc(&d_work_psi_, sizeof(double) * psi_len()));
        }
        IDC_TRY_CUDA(cudaMemcpyAsync(d_work_psi_, x, sizeof(double) * psi_len(), cudaMemcpyDeviceToDevice, stream));
        IDC_TRY_CUDA(launch_periodic_halos(dims(), d_work_psi_, stream));
        launches += 1;
        x = d_work_psi_;
    }
    IDC_TRY_CUDA(launch_lmv(dims(), alpha, beta, d_sigma_t, d_xi, d_eta, x, y, stream, 0.0, nullptr, nullptr,
                            high_order_sigma() ? d_tens_t_ : nullptr));
    launches += 1;
    return Status::ok();
}

// res = (L - S P) psi given phi = P psi: Lmv(1, 0) then Smv(-1, 1) in one pass over psi, rounded alike
Status Context::transport_residual(const double *psi, const double *phi, double *res) {
    IDC_TRY_CUDA(launch_lmv(dims(), 1.0, 0.0, d_sigma_t, d_xi, d_eta, psi, res, stream, -1.0, d_sigma_s, phi,
                            high_order_sigma() ? d_tens_t_ : nullptr, high_order_sigma() ? d_tens_s_ : nullptr));
    launches += 1;
    return Status::ok();
}

Status Context::lmv_transpose(double alpha, double beta, const double *x, double *y) {
    if (periodic_ || reflect_mask) return bad(IDC_ERR_UNSUPPORTED, "the transposed operators with periodic or reflecting edges");
    if (high_order_sigma()) return bad(IDC_ERR_UNSUPPORTED, "the transposed operators with high-order cross sections");
    IDC_TRY_CUDA(cudaSetDevice(device));
    IDC_TRY_CUDA(launch_lmv_transpose(dims(), alpha, beta, d_sigma_t, d_xi, d_eta, d_w, x, y, stream));
    launches += 1;
    return Status::ok();
}

Status Context::transport_residual_transpose(const double *z, double *y, double *zsum) {
    if (high_order_sigma()) return bad(IDC_ERR_UNSUPPORTED, "the transposed operators with high-order cross sections");
    if (!d_ones_) {
        std::vector<double> ones((size_t)nq, 1.0);
        IDC_TRY_CUDA(cudaMalloc(&d_ones_, sizeof(double) * nq));
        IDC_TRY_CUDA(cudaMemcpy(d_ones_, ones.data(), sizeof(double) * nq, cudaMemcpyHostToDevice));
    }
    IDC_TRY_CUDA(launch_pmv(dims(), 1.0, 0.0, d_ones_, z, zsum, stream));   // sum_q z_q
    IDC_TRY_CUDA(launch_lmv_transpose(dims(), 1.0, 0.0, d_sigma_t, d_xi, d_eta, d_w, z, y, stream, -1.0, d_sigma_s,
                                      zsum));
    launches += 2;
    return Status::ok();
}

Status Context::l2dist(const double *a, const double *b, double *out_host) {
    IDC_TRY_CUDA(launch_l2dist2(dims(), a, b, d_scalar_, d_scalar_ + 4, stream));
    launches += 2;
    double v = 0;
    IDC_TRY_CUDA(cudaMemcpyAsync(&v, d_scalar_, sizeof(double), cudaMemcpyDeviceToHost, stream));
    IDC_TRY_CUDA(cudaStreamSynchronize(stream));
    *out_host = std::sqrt(v);
    return Status::ok();
}

// SISolver::Solve, linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:190-254.  The copy of the
// source into psi, Smv(1, 1, sigma_s, phi_last -> psi) and Pmv(1, 0, psi -> phi) of each iteration are
// fused into the sweep (source read + scattering term on the fly, moments in the epilogue).
Status Context::source_iteration(const double *src, double *psi_out, double dt, double abs_tol, int64_t max_its,
                                 int precision, int64_t *iters, double *err) {
    if (reflect_mask) return source_iteration_reflecting(src, psi_out, dt, abs_tol, max_its, precision, iters, err);
    if (periodic_) return source_iteration_periodic(src, psi_out, dt, abs_tol, max_its, precision, iters, err);
    IDC_TRY(ensure_phi_buffers(2));
    double *phi_cur = phi_buf(0), *phi_last = phi_buf(1);
    IDC_TRY_CUDA(cudaMemsetAsync(phi_cur, 0, sizeof(double) * phi_len(), stream));
    IDC_TRY_CUDA(cudaMemsetAsync(phi_last, 0, sizeof(double) * phi_len(), stream));
    int64_t it = 0;
    double e = INFINITY;
    while (it < max_its && e > abs_tol) {
        ++it;
        std::swap(phi_cur, phi_last);
        IDC_TRY(sweep(src, psi_out, dt, phi_cur, precision, phi_last, 1.0));
        IDC_TRY(l2dist(phi_cur, phi_last, &e));
        IDC_TRY(check_device_error());
    }
    // Like the reference, reaching max_its is not an error: the caller reads *err.
    if (iters) *iters = it;
    if (err) *err = e;
    return Status::ok();
}

}  // namespace idc
