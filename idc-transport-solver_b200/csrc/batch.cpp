// Batched sweeps: several independent problems (contexts on one GPU) in one persistent launch per DG
// degree, and the tile-shape autotuner for a batch.
//
// The problems of a degree share the launch's tile shape (row-segment width seg, compute warps wn) and
// item queue.  Each problem keeps its own arrays, chunks its quadrants' ordinates by seg, and gets its
// own trace buffer, partial-moment slots and inflow traces; its descriptor (a SweepArgs)
// sits in a device table that the kernel reads per item.  Row blocks of all problems are interleaved in
// the queue (row block 0 of every problem, then row block 1, ...), so every problem's wavefront starts at
// once and every dependency is dequeued before its consumer.
#include "batch.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>

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

// Default shape: the single problem's default kernel and rule.  FP64: the lane kernel (warps = 0) with 16-wide
// segments at DG degree 2, 8-wide at degree 1 for up to 24 ordinates per quadrant, else the narrowest segment
// with the best lane use.  FP32_REFINED: the modal kernel, narrowest best segment, its default warps.
void default_shape(int P, int precision, int qmax, int *seg, int *wn) {
    const bool lane = precision == IDC_PREC_FP64;
    double best = -1.0;
    for (int cand : {4, 8, 16, 32}) {
        if (lane && cand == 32) break;
        const int nch = (qmax + cand - 1) / cand;
        const double eff = (double)qmax / (nch * cand);
        if (eff > best + 1e-9) {
            best = eff;
            *seg = cand;
        }
    }
    if (lane && (P == 3 || (P == 2 && qmax <= 24))) *seg = P == 3 ? 16 : 8;
    *wn = lane ? 0 : sweep_modal_default_wn(P);
}

int qmax_of(const Context &c) {
    int q = 0;
    for (int k = 0; k < 4; ++k) q = std::max<int>(q, (int)(c.quad[k + 1] - c.quad[k]));
    return q;
}

}  // namespace

Batch::~Batch() { release(); }

void Batch::release() {
    for (auto &g : groups) {
        cudaFree(g.d_items);
        cudaFree(g.d_sync);
        cudaFree(g.d_table);
        cudaFreeHost(g.h_table);
        if (g.upload_done) cudaEventDestroy(g.upload_done);
        for (double *p : g.trace) cudaFree(p);
        for (double *p : g.phi_part) cudaFree(p);
        for (double *p : g.inflow) cudaFree(p);
    }
    groups.clear();
}

Status Batch::add(Context *c) {
    if (!c) return bad(IDC_ERR_ARG, "null context");
    if (!c->have_ordinates || !c->have_sigma) return bad(IDC_ERR_STATE, "batch member without ordinates or sigma");
    if (!c->modal_family())
        return bad(IDC_ERR_UNSUPPORTED, "batched sweeps need the lane or modal kernel (DG degree <= 2, piecewise-"
                                        "constant cross sections)");
    if (c->reflect_mask) return bad(IDC_ERR_UNSUPPORTED, "batched sweeps with reflecting boundaries");
    if (c->high_order_sigma()) return bad(IDC_ERR_UNSUPPORTED, "batched sweeps with high-order cross sections");
    if (c->periodic_) return bad(IDC_ERR_UNSUPPORTED, "batched solves on a periodic grid");
    if (!members.empty() && c->device != members[0]->device) return bad(IDC_ERR_ARG, "batch members on different GPUs");
    members.push_back(c);
    release();
    return Status::ok();
}

Status Batch::build_group(Group &g, int precision) {
    Context &c0 = *members[g.members[0]];
    g.G = g.seg;
    const bool lane = g.wn == 0;   // the lane kernel (FP64): one warp per item, 32 / seg rows
    if (lane && (precision != IDC_PREC_FP64 || !sweep_lane_supports(c0.P, 0, g.seg)))
        return bad(IDC_ERR_UNSUPPORTED, "batched lane sweeps: FP64, seg 4, 8 or 16");
    if (!lane) g.wn = sweep_modal_fit_wn(c0.P, precision, g.wn, g.G, g.seg);
    const int seg = g.seg, wn = g.wn, rw = 32 / seg, rows_cta = lane ? rw : wn * rw;
    std::vector<std::vector<SweepItem>> per(g.members.size());
    std::vector<int> nrb(g.members.size()), ipr(g.members.size());
    for (size_t m = 0; m < g.members.size(); ++m) {
        const Context &c = *members[g.members[m]];
        // chunks of each quadrant (near-equal, at most seg ordinates)
        std::vector<int> qk, qb, qc;
        for (int k = 0; k < 4; ++k) {
            const int cnt = (int)(c.quad[k + 1] - c.quad[k]);
            if (!cnt) continue;
            const int nch = (cnt + seg - 1) / seg;
            int beg = (int)c.quad[k];
            for (int h = 0; h < nch; ++h) {
                const int sz = cnt / nch + (h < cnt % nch ? 1 : 0);
                qk.push_back(k);
                qb.push_back(beg);
                qc.push_back(sz);
                beg += sz;
            }
        }
        ipr[m] = (int)qk.size();
        nrb[m] = (int)((c.ny + rows_cta - 1) / rows_cta);
        for (int rb = 0; rb < nrb[m]; ++rb)
            for (int s = 0; s < ipr[m]; ++s)
                per[m].push_back(
                    SweepItem{qk[s], qb[s], qc[s], rb, rb == 0 ? -1 : (rb - 1) * ipr[m] + s, (int)m, rb * ipr[m] + s});
    }
    // interleave row blocks (items keep their problem-local index and local dependency)
    std::vector<SweepItem> items;
    const int max_rb = *std::max_element(nrb.begin(), nrb.end());
    for (int rb = 0; rb < max_rb; ++rb)
        for (size_t m = 0; m < g.members.size(); ++m)
            if (rb < nrb[m])
                for (int s = 0; s < ipr[m]; ++s) items.push_back(per[m][(size_t)rb * ipr[m] + s]);
    g.n_items = (int)items.size();
    g.items_per_rb = ipr;
    IDC_TRY_CUDA(cudaSetDevice(c0.device));
    IDC_TRY_CUDA(cudaMalloc(&g.d_items, sizeof(SweepItem) * items.size()));
    IDC_TRY_CUDA(cudaMemcpy(g.d_items, items.data(), sizeof(SweepItem) * items.size(), cudaMemcpyHostToDevice));
    IDC_TRY_CUDA(cudaMalloc(&g.d_sync, sizeof(int) * 2));
    IDC_TRY_CUDA(cudaMemset(g.d_sync, 0, sizeof(int) * 2));
    IDC_TRY_CUDA(cudaMalloc(&g.d_table, sizeof(SweepArgs) * g.members.size()));
    IDC_TRY_CUDA(cudaMallocHost(&g.h_table, sizeof(SweepArgs) * g.members.size()));
    IDC_TRY_CUDA(cudaEventCreateWithFlags(&g.upload_done, cudaEventDisableTiming));
    g.uploaded.clear();
    g.trace.assign(g.members.size(), nullptr);
    g.trace_len.assign(g.members.size(), 0);
    g.phi_part.assign(g.members.size(), nullptr);
    g.inflow.assign(g.members.size(), nullptr);
    for (size_t m = 0; m < g.members.size(); ++m) {
        const Context &c = *members[g.members[m]];
        const size_t tl = per[m].size() * (size_t)c.nx * g.G * c.P;   // one trace row per item of the member
        IDC_TRY_CUDA(cudaMalloc(&g.trace[m], sizeof(double) * tl));
        g.trace_len[m] = tl;
        IDC_TRY_CUDA(launch_fill_u64(reinterpret_cast<unsigned long long *>(g.trace[m]), tl, kTraceSentinel, stream()));
        IDC_TRY_CUDA(cudaMalloc(&g.phi_part[m], sizeof(double) * (size_t)ipr[m] * c.phi_len()));
        IDC_TRY_CUDA(cudaMalloc(&g.inflow[m], sizeof(double) * (size_t)(c.nx + c.ny) * c.nq * c.P));
    }
    int per_sm = 0;
    if (lane) {   // shared memory fixed per kernel instance (set by the launcher); one item per warp at a time
        g.smem = 0;
        IDC_TRY_CUDA(sweep_lane_batched_occupancy(c0.P, seg, &per_sm));
        if (per_sm < 1) return bad(IDC_ERR_UNSUPPORTED, "batched sweep kernel does not fit on an SM");
        g.grid = std::min((g.n_items + sweep_lane_warps() - 1) / sweep_lane_warps(), per_sm * c0.num_sms);
    } else {
        g.smem = sweep_modal_smem_bytes(c0.P, precision, wn, g.G, seg);
        IDC_TRY_CUDA(sweep_modal_occupancy(c0.P, precision, seg, sweep_modal_threads(c0.P, wn), g.smem, &per_sm));
        if (per_sm < 1) return bad(IDC_ERR_UNSUPPORTED, "batched sweep kernel does not fit on an SM");
        g.grid = std::min(g.n_items, per_sm * c0.num_sms);
    }
    g.precision = precision;
    IDC_TRY_CUDA(cudaStreamSynchronize(stream()));
    return Status::ok();
}

Status Batch::launch_group(Group &g, const double *const *srcs, double *const *outs, const double *const *phi_sc,
                           double scale, double *const *phis, double dt, const std::vector<char> *active) {
    Context &c0 = *members[g.members[0]];
    cudaStream_t st = stream();
    std::vector<SweepArgs> table(g.members.size());
    for (size_t m = 0; m < g.members.size(); ++m) {
        const int p = g.members[m];
        Context &c = *members[p];
        SweepArgs &a = table[m];
        a = SweepArgs{};
        a.src = srcs ? srcs[p] : nullptr;
        a.out = outs ? outs[p] : nullptr;
        a.sigma_t = c.d_sigma_t;
        a.sigma_s = nullptr;   // the modal kernel's fused source takes ready scattering moments
        a.phi_scatter = phi_sc ? phi_sc[p] : nullptr;
        a.scatter_scale = scale;
        a.xi = c.d_xi;
        a.eta = c.d_eta;
        a.w = c.d_w;
        a.nx = (int)c.nx;
        a.ny = (int)c.ny;
        a.nq = (int)c.nq;
        a.dx = c.dx;
        a.dy = c.dy;
        a.inv_dt = 1.0 / dt;
        a.items = g.d_items;
        a.n_items = g.n_items;
        a.G = g.G;
        a.n_refine = 1;
        a.seg = g.seg;
        a.wn = g.wn;
        a.R = (g.wn == 0 ? 1 : g.wn) * (32 / g.seg);
        a.trace = g.trace[m];
        a.trace_stride = (size_t)c.nx * g.G * c.P;
        a.next_item = g.d_sync;
        a.error = g.d_sync + 1;
        a.spin_limit = c.spin_limit;
        if (phis && phis[p]) {
            a.phi_part = g.phi_part[m];
            a.phi_slots = g.items_per_rb[m];
            a.phi_slot_stride = c.phi_len();
            a.phi = phis[p];   // the batched reduction's output (the sweep kernel writes the slots)
        }
        if (a.src) a.inflow = g.inflow[m];
        if (active && !(*active)[p]) {   // left out: its items return at once, the helpers see no arrays
            a.skip = 1;
            a.src = nullptr;
            a.out = nullptr;
            a.phi_scatter = nullptr;
            a.phi = nullptr;
            a.phi_part = nullptr;
            a.inflow = nullptr;
        }
    }
    bool any_src = false, any_phi = false;
    for (const auto &a : table) {
        any_src |= a.src != nullptr;
        any_phi |= a.phi != nullptr;
    }
    // upload the table only when it changed (pinned source: no stream synchronisation)
    const size_t bytes = sizeof(SweepArgs) * table.size();
    if (g.uploaded.size() != table.size() || std::memcmp(g.uploaded.data(), table.data(), bytes) != 0) {
        IDC_TRY_CUDA(cudaEventSynchronize(g.upload_done));   // the previous upload no longer reads h_table
        std::memcpy(g.h_table, table.data(), bytes);
        IDC_TRY_CUDA(cudaMemcpyAsync(g.d_table, g.h_table, bytes, cudaMemcpyHostToDevice, st));
        IDC_TRY_CUDA(cudaEventRecord(g.upload_done, st));
        g.uploaded = table;
    }
    SweepArgs launch = table[0];   // the launch-wide fields (items, queue, error, tile shape) are common
    // three launches per degree, whatever the number of problems: inflow traces, the sweep, the moments
    if (any_src)
        IDC_TRY_CUDA(launch_batched_helpers(c0.P, g.precision != IDC_PREC_FP32_REFINED, g.d_table, (int)table.size(),
                                            true, false, st));
    IDC_TRY_CUDA(cudaMemsetAsync(g.d_sync, 0, sizeof(int), st));
    if (g.wn == 0)
        IDC_TRY_CUDA(launch_sweep_lane_batched(c0.P, launch, g.d_table, g.grid, st));
    else
        IDC_TRY_CUDA(launch_sweep_modal_batched(c0.P, g.precision, launch, g.d_table, g.grid, g.smem, st));
    if (any_phi)
        IDC_TRY_CUDA(launch_batched_helpers(c0.P, false, g.d_table, (int)table.size(), false, true, st));
    return Status::ok();
}

Status Batch::sweep(const double *const *srcs, double *const *outs, const double *const *phi_sc, double scale,
                    double *const *phis, double dt, int precision, const std::vector<char> *active) {
    if (members.empty()) return bad(IDC_ERR_STATE, "empty batch");
    if (precision != IDC_PREC_FP64 && precision != IDC_PREC_FP32_REFINED)
        return bad(IDC_ERR_UNSUPPORTED, "batched sweeps run in FP64 or refined precision");
    if (!(dt > 0)) return bad(IDC_ERR_ARG, "dt must be positive");
    Context &c0 = *members[0];
    IDC_TRY_CUDA(cudaSetDevice(c0.device));
    if (groups.empty() || groups[0].precision != precision) {
        release();
        for (int P : {1, 2, 3}) {
            Group g;
            for (size_t m = 0; m < members.size(); ++m)
                if (members[m]->P == P) g.members.push_back((int)m);
            if (g.members.empty()) continue;
            g.P = P;
            int qmax = 0;
            for (int m : g.members) qmax = std::max(qmax, qmax_of(*members[m]));
            const auto key = std::make_pair(P, precision);
            if (tuned.count(key)) {
                g.seg = tuned[key].first;
                g.wn = std::min(tuned[key].second, sweep_modal_max_wn(P));
            } else {
                default_shape(P, precision, qmax, &g.seg, &g.wn);
            }
            g.precision = precision;
            groups.push_back(g);
        }
        for (auto &g : groups) IDC_TRY(build_group(g, precision));
    }
    IDC_TRY_CUDA(cudaEventRecord(c0.ev0, c0.stream));
    for (auto &g : groups) IDC_TRY(launch_group(g, srcs, outs, phi_sc, scale, phis, dt, active));
    IDC_TRY_CUDA(cudaEventRecord(c0.ev1, c0.stream));
    IDC_TRY_CUDA(cudaStreamSynchronize(c0.stream));
    for (auto &g : groups) {
        int err = 0;
        IDC_TRY_CUDA(cudaMemcpy(&err, g.d_sync + 1, sizeof(int), cudaMemcpyDeviceToHost));
        if (err != kDevOk) {
            IDC_TRY_CUDA(cudaMemset(g.d_sync + 1, 0, sizeof(int)));
            for (size_t m = 0; m < g.members.size(); ++m)
                IDC_TRY_CUDA(launch_fill_u64(reinterpret_cast<unsigned long long *>(g.trace[m]), g.trace_len[m],
                                             kTraceSentinel, c0.stream));
            IDC_TRY_CUDA(cudaStreamSynchronize(c0.stream));
            return bad(IDC_ERR_TIMEOUT, "a device-side wait gave up in a batched sweep");
        }
    }
    float ms = 0.f;
    IDC_TRY_CUDA(cudaEventElapsedTime(&ms, c0.ev0, c0.ev1));
    last_ms = ms;
    return Status::ok();
}

// Batched GMRES: Context::gmres_peierls's algorithm (CGS2 Arnoldi, Givens rotations on the host, restarts
// from the true residual, flexible GMRES with the member's DSA preconditioner) run on every member in lock
// step.  A step applies the Peierls operator of every unconverged member, A v = v - P L^{-1} S v, through
// ONE batched sweep (members that have converged are skipped inside the launch), then queues each member's
// orthogonalisation on the device and brings every member's Hessenberg column back with one
// synchronisation.  A member whose cycle ends restarts from its true residual in the next step's sweep.
Status Batch::gmres_solve(double *const *psi_inout, double dt, double abs_tol, int restart, int64_t max_its,
                          int precision, int64_t *iters_out, double *resids_out) {
    if (members.empty()) return bad(IDC_ERR_STATE, "empty batch");
    if (restart < 1 || restart > 60) return bad(IDC_ERR_ARG, "gmres restart must be in 1..60");
    if (!psi_inout) return bad(IDC_ERR_ARG, "null psi arrays");
    const size_t M = members.size();
    for (size_t p = 0; p < M; ++p)
        if (!psi_inout[p]) return bad(IDC_ERR_ARG, "null psi array of a batch member");
    Context &c0 = *members[0];
    IDC_TRY_CUDA(cudaSetDevice(c0.device));
    cudaStream_t st = stream();
    const int m = restart;

    struct State {
        Context *c;
        size_t n;
        int m;
        bool dsa;
        double *V, *b, *x, *tmp, *scat;
        std::vector<double> H, cs, sn, g, yv;
        double beta = 0, resid = 0;
        int j = 0;
        int64_t its = 0;
        bool done = false, converged = false, restart_pending = false;
        double *in = nullptr, *out = nullptr;
        double *Vc(int k) const { return V + (size_t)k * n; }
        double *Zc(int k) const { return V + (size_t)(m + 1 + k) * n; }   // flexible GMRES: Z after V_0 .. V_m
    };
    int *d_err = nullptr;   // one device error word per member for its DSA grid barriers
    IDC_TRY_CUDA(cudaMalloc(&d_err, sizeof(int) * M));
    struct Free {
        int *p;
        ~Free() { cudaFree(p); }
    } free_err{d_err};
    IDC_TRY_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int) * M, st));
    std::vector<State> S(M);
    for (size_t p = 0; p < M; ++p) {
        Context &c = *members[p];
        State &z = S[p];
        z.c = &c;
        z.n = c.phi_len();
        z.m = m;
        z.dsa = c.precond_kind == 1;
        const size_t need = (size_t)(z.dsa ? 2 * m + 1 : m + 1) * z.n;
        if (c.krylov_len < need) {
            cudaFree(c.d_krylov);
            c.d_krylov = nullptr;
            c.krylov_len = 0;
            IDC_TRY_CUDA(cudaMalloc(&c.d_krylov, sizeof(double) * need));
            c.krylov_len = need;
        }
        if (!c.d_small) IDC_TRY_CUDA(cudaMalloc(&c.d_small, sizeof(double) * (128 + multidot_scratch_doubles())));
        if (!c.h_small) IDC_TRY_CUDA(cudaMallocHost(&c.h_small, sizeof(double) * 129));
        IDC_TRY(c.ensure_phi_buffers(7));
        z.V = c.d_krylov;
        z.b = c.phi_buf(3);
        z.x = c.phi_buf(4);
        z.tmp = c.phi_buf(5);
        z.scat = c.phi_buf(6);
        z.H.assign((size_t)(m + 1) * m, 0.0);
        z.cs.assign(m, 0.0);
        z.sn.assign(m, 0.0);
        z.g.assign(m + 1, 0.0);
        z.yv.assign(m, 0.0);
        if (z.dsa) {
            const size_t wl = dsa_workspace_doubles((int)c.nx, (int)c.ny);
            if (c.dsa_ws_len < wl) {
                cudaFree(c.d_dsa_ws);
                c.d_dsa_ws = nullptr;
                c.dsa_ws_len = 0;
                IDC_TRY_CUDA(cudaMalloc(&c.d_dsa_ws, sizeof(double) * wl));
                c.dsa_ws_len = wl;
            }
            IDC_TRY_CUDA(dsa_setup(c.dims(), c.d_sigma_t, c.d_sigma_s, c.d_dsa_ws, st));
        }
        IDC_TRY_CUDA(cudaMemsetAsync(z.x, 0, sizeof(double) * z.n, st));
    }
    std::vector<const double *> srcs(M), scats(M);
    std::vector<double *> outs(M, nullptr), bs(M), tmps(M);
    for (size_t p = 0; p < M; ++p) {
        srcs[p] = psi_inout[p];
        bs[p] = S[p].b;
        tmps[p] = S[p].tmp;
        scats[p] = S[p].scat;
    }
    // right-hand sides b = P L^{-1} Q of every member in one batched sweep, then r = b, beta = |b|
    IDC_TRY(sweep(srcs.data(), nullptr, nullptr, 1.0, bs.data(), dt, precision));
    for (auto &z : S) {
        IDC_TRY_CUDA(cudaMemcpyAsync(z.Vc(0), z.b, sizeof(double) * z.n, cudaMemcpyDeviceToDevice, st));
        IDC_TRY_CUDA(launch_dot(z.Vc(0), z.Vc(0), z.n, z.c->d_small + 127, z.c->d_small + 128, st));
        IDC_TRY_CUDA(cudaMemcpyAsync(z.c->h_small + 127, z.c->d_small + 127, sizeof(double), cudaMemcpyDeviceToHost, st));
    }
    IDC_TRY_CUDA(cudaStreamSynchronize(st));
    auto start_cycle = [&](State &z) -> Status {
        IDC_TRY_CUDA(launch_axpby(0.0, z.Vc(0), 1.0 / z.beta, z.Vc(0), z.n, st));
        std::fill(z.g.begin(), z.g.end(), 0.0);
        z.g[0] = z.beta;
        z.j = 0;
        return Status::ok();
    };
    for (auto &z : S) {
        z.beta = std::sqrt(z.c->h_small[127]);
        z.resid = z.beta;
        z.converged = z.resid <= abs_tol;
        z.done = z.converged || z.beta == 0.0 || max_its == 0;
        if (!z.done) IDC_TRY(start_cycle(z));
    }
    std::vector<char> active(M);
    for (;;) {
        bool any = false;
        for (size_t p = 0; p < M; ++p) {
            active[p] = !S[p].done;
            any |= !S[p].done;
        }
        if (!any) break;
        // the vectors to apply A to: x (a restart's true residual) or the next basis (preconditioned) vector
        for (size_t p = 0; p < M; ++p) {
            State &z = S[p];
            if (z.done) continue;
            Context &c = *z.c;
            if (z.restart_pending) {
                z.in = z.x;
                z.out = z.Vc(0);
            } else {
                if (z.dsa) {
                    IDC_TRY_CUDA(dsa_precondition(c.dims(), c.d_sigma_s, z.Vc(z.j), z.Zc(z.j), c.dsa_steps, c.d_dsa_ws,
                                                  false, c.num_sms, d_err + p, c.spin_limit, st));
                    z.in = z.Zc(z.j);
                } else {
                    z.in = z.Vc(z.j);
                }
                z.out = z.Vc(z.j + 1);
            }
            IDC_TRY_CUDA(launch_scatter_moments(c.dims(), c.d_sigma_s, z.in, z.scat, st));
        }
        IDC_TRY(sweep(nullptr, nullptr, scats.data(), 1.0, tmps.data(), dt, precision, &active));
        for (size_t p = 0; p < M; ++p) {
            State &z = S[p];
            if (z.done) continue;
            Context &c = *z.c;
            const size_t n = z.n;
            IDC_TRY_CUDA(launch_axpby(1.0, z.in, 0.0, z.out, n, st));     // A in = in - P L^{-1} S in
            IDC_TRY_CUDA(launch_axpby(-1.0, z.tmp, 1.0, z.out, n, st));
            double *ds = c.d_small, *scratch = c.d_small + 128;
            if (z.restart_pending) {   // r = b - A x
                IDC_TRY_CUDA(launch_axpby(1.0, z.b, -1.0, z.Vc(0), n, st));
                IDC_TRY_CUDA(launch_dot(z.Vc(0), z.Vc(0), n, ds + 127, scratch, st));
            } else {                   // CGS2 against V_0 .. V_j, then |w|^2
                const int j = z.j;
                IDC_TRY_CUDA(launch_multidot(z.V, j + 1, n, z.Vc(j + 1), n, ds, scratch, st));
                IDC_TRY_CUDA(launch_multiaxpy(z.Vc(j + 1), z.V, j + 1, n, ds, n, st));
                IDC_TRY_CUDA(launch_multidot(z.V, j + 1, n, z.Vc(j + 1), n, ds + 64, scratch, st));
                IDC_TRY_CUDA(launch_multiaxpy(z.Vc(j + 1), z.V, j + 1, n, ds + 64, n, st));
                IDC_TRY_CUDA(launch_dot(z.Vc(j + 1), z.Vc(j + 1), n, ds + 127, scratch, st));
            }
            IDC_TRY_CUDA(cudaMemcpyAsync(c.h_small, ds, sizeof(double) * 128, cudaMemcpyDeviceToHost, st));
            IDC_TRY_CUDA(cudaMemcpyAsync(c.h_small + 128, d_err + p, sizeof(int), cudaMemcpyDeviceToHost, st));
        }
        IDC_TRY_CUDA(cudaStreamSynchronize(st));
        for (size_t p = 0; p < M; ++p) {
            State &z = S[p];
            if (z.done) continue;
            const double *h = z.c->h_small;
            int dev_err = 0;
            std::memcpy(&dev_err, h + 128, sizeof(int));
            if (dev_err != kDevOk)
                return bad(IDC_ERR_TIMEOUT, "a DSA grid barrier gave up in a batched GMRES solve");
            if (z.restart_pending) {
                z.restart_pending = false;
                z.beta = std::sqrt(h[127]);
                z.resid = z.beta;
                z.converged = z.resid <= abs_tol;
                z.done = z.converged || z.beta == 0.0 || z.its >= max_its;
                if (!z.done) IDC_TRY(start_cycle(z));
                continue;
            }
            const int j = z.j;
            const double hn = std::sqrt(h[127]);
            for (int i = 0; i <= j; ++i) z.H[(size_t)i * m + j] = h[i] + h[64 + i];
            z.H[(size_t)(j + 1) * m + j] = hn;
            if (hn > 0.0) IDC_TRY_CUDA(launch_axpby(0.0, z.Vc(j + 1), 1.0 / hn, z.Vc(j + 1), z.n, st));
            for (int i = 0; i < j; ++i) {
                const double a = z.H[(size_t)i * m + j], c = z.H[(size_t)(i + 1) * m + j];
                z.H[(size_t)i * m + j] = z.cs[i] * a + z.sn[i] * c;
                z.H[(size_t)(i + 1) * m + j] = -z.sn[i] * a + z.cs[i] * c;
            }
            const double a = z.H[(size_t)j * m + j], c = z.H[(size_t)(j + 1) * m + j];
            const double r = std::hypot(a, c);
            z.cs[j] = r > 0.0 ? a / r : 1.0;
            z.sn[j] = r > 0.0 ? c / r : 0.0;
            z.H[(size_t)j * m + j] = r;
            z.H[(size_t)(j + 1) * m + j] = 0.0;
            z.g[j + 1] = -z.sn[j] * z.g[j];
            z.g[j] = z.cs[j] * z.g[j];
            z.resid = std::fabs(z.g[j + 1]);
            ++z.its;
            const bool cycle_end = z.resid <= abs_tol || hn == 0.0 || j + 1 == m || z.its >= max_its;
            if (!cycle_end) {
                z.j = j + 1;
                continue;
            }
            // y = H^{-1} g, x += Z y (or V y)
            const int k = j + 1;
            for (int i = k - 1; i >= 0; --i) {
                double sum = z.g[i];
                for (int l = i + 1; l < k; ++l) sum -= z.H[(size_t)i * m + l] * z.yv[l];
                z.yv[i] = sum / z.H[(size_t)i * m + i];
            }
            for (int i = 0; i < k; ++i) z.yv[i] = -z.yv[i];   // multiaxpy subtracts
            IDC_TRY_CUDA(cudaMemcpyAsync(z.c->d_small, z.yv.data(), sizeof(double) * k, cudaMemcpyHostToDevice, st));
            IDC_TRY_CUDA(launch_multiaxpy(z.x, z.dsa ? z.Zc(0) : z.V, k, z.n, z.c->d_small, z.n, st));
            if (z.resid <= abs_tol) {
                z.converged = true;
                z.done = true;
            } else if (z.its >= max_its || hn == 0.0) {
                z.done = true;
            } else {
                z.restart_pending = true;
            }
        }
    }
    // psi = L^{-1}(S phi + Q) of every member in one batched sweep (in place: Q in, psi out)
    for (auto &z : S) IDC_TRY_CUDA(launch_scatter_moments(z.c->dims(), z.c->d_sigma_s, z.x, z.scat, st));
    IDC_TRY(sweep(srcs.data(), psi_inout, scats.data(), 1.0, nullptr, dt, precision));
    bool all = true;
    for (size_t p = 0; p < M; ++p) {
        if (iters_out) iters_out[p] = S[p].its;
        if (resids_out) resids_out[p] = S[p].resid;
        all &= S[p].converged;
    }
    if (!all) return bad(IDC_ERR_NOT_CONVERGED, "a batched GMRES solve stopped at its iteration limit");
    return Status::ok();
}

Status Batch::set_shape(int P, int precision, int seg, int wn) {
    const auto key = std::make_pair(P, precision);
    if (seg == 0 && wn == 0) {
        tuned.erase(key);
    } else {
        const bool lane = wn == 0 && precision == IDC_PREC_FP64 && (seg == 4 || seg == 8 || seg == 16);
        if (!lane && ((seg != 4 && seg != 8 && seg != 16 && seg != 32) || wn < 1 || wn > 7))
            return bad(IDC_ERR_ARG, "batch tile shape: seg 4, 8, 16 or 32 with wn in 1..7 (the modal kernel), or "
                                    "seg 4, 8 or 16 with wn 0 (the lane kernel, FP64)");
        tuned[key] = {seg, wn};
    }
    release();
    return Status::ok();
}

void Batch::get_shape(int P, int precision, int *seg, int *wn) const {
    const auto it = tuned.find(std::make_pair(P, precision));
    if (it != tuned.end()) {
        *seg = it->second.first;
        *wn = it->second.second;
        return;
    }
    int qmax = 0;
    for (auto *c : members)
        if (c->P == P) qmax = std::max(qmax, qmax_of(*c));
    if (qmax == 0) {
        *seg = *wn = 0;
        return;
    }
    default_shape(P, precision, qmax, seg, wn);
}

Status Batch::autotune(const double *const *srcs, double *const *outs, double dt, int precision) {
    if (members.empty()) return bad(IDC_ERR_STATE, "empty batch");
    for (int P : {1, 2, 3}) {
        bool any = false;
        for (auto *c : members) any |= c->P == P;
        if (!any) continue;
        float best = 1e30f;
        std::pair<int, int> bsh{0, 0};
        // the modal kernel's shapes, and in FP64 the lane kernel's (wn 0)
        std::vector<std::pair<int, int>> cands;
        for (int cs : {4, 8, 16, 32})
            for (int cw = std::max(1, sweep_modal_max_wn(P) - 3); cw <= sweep_modal_max_wn(P); ++cw)
                cands.push_back({cs, cw});
        if (precision == IDC_PREC_FP64)
            for (int cs : {4, 8, 16}) cands.push_back({cs, 0});
        for (const auto &cand : cands) {
            tuned[std::make_pair(P, precision)] = cand;
            release();
            float ms = 1e30f;
            for (int rep = 0; rep < 4; ++rep) {   // one warm-up, then the best of three
                IDC_TRY(sweep(srcs, outs, nullptr, 1.0, nullptr, dt, precision));
                if (rep > 0) ms = std::min(ms, last_ms);
            }
            // the timing covers every degree's launch; the other degrees' shapes stay fixed meanwhile
            if (ms < best) {
                best = ms;
                bsh = cand;
            }
        }
        tuned[std::make_pair(P, precision)] = bsh;
        release();
    }
    return Status::ok();
}

}  // namespace idc
