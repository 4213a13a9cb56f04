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

// Default shape: the narrowest segment with the best lane use, the single problem's default warps.
void default_shape(int P, int qmax, int *seg, int *wn) {
    double best = -1.0;
    for (int cand : {4, 8, 16, 32}) {
        const int nch = (qmax + cand - 1) / cand;
        const double eff = (double)qmax / (nch * cand);
        if (eff > best + 1e-9) {
            best = eff;
            *seg = cand;
        }
    }
    *wn = sweep_modal_default_wn(P);
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
    if (!c->modal_family()) return bad(IDC_ERR_UNSUPPORTED, "batched sweeps need the modal kernel");
    if (!members.empty() && c->device != members[0]->device) return bad(IDC_ERR_ARG, "batch members on different GPUs");
    members.push_back(c);
    release();
    return Status::ok();
}

Status Batch::build_group(Group &g, int precision) {
    Context &c0 = *members[g.members[0]];
    g.G = g.seg;
    g.wn = sweep_modal_fit_wn(c0.P, precision, g.wn, g.G, g.seg);
    const int seg = g.seg, wn = g.wn, rw = 32 / seg, rows_cta = wn * rw;
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
    g.smem = sweep_modal_smem_bytes(c0.P, precision, wn, g.G, seg);
    IDC_TRY_CUDA(sweep_modal_occupancy(c0.P, precision, seg, sweep_modal_threads(c0.P, wn), g.smem, &per_sm));
    if (per_sm < 1) return bad(IDC_ERR_UNSUPPORTED, "batched sweep kernel does not fit on an SM");
    g.grid = std::min(g.n_items, per_sm * c0.num_sms);
    g.precision = precision;
    IDC_TRY_CUDA(cudaStreamSynchronize(stream()));
    return Status::ok();
}

Status Batch::launch_group(Group &g, const double *const *srcs, double *const *outs, const double *const *phi_sc,
                           double scale, double *const *phis, double dt) {
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
        a.R = g.wn * (32 / g.seg);
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
    IDC_TRY_CUDA(launch_sweep_modal_batched(c0.P, g.precision, launch, g.d_table, g.grid, g.smem, st));
    if (any_phi)
        IDC_TRY_CUDA(launch_batched_helpers(c0.P, false, g.d_table, (int)table.size(), false, true, st));
    return Status::ok();
}

Status Batch::sweep(const double *const *srcs, double *const *outs, const double *const *phi_sc, double scale,
                    double *const *phis, double dt, int precision) {
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
                default_shape(P, qmax, &g.seg, &g.wn);
            }
            g.precision = precision;
            groups.push_back(g);
        }
        for (auto &g : groups) IDC_TRY(build_group(g, precision));
    }
    IDC_TRY_CUDA(cudaEventRecord(c0.ev0, c0.stream));
    for (auto &g : groups) IDC_TRY(launch_group(g, srcs, outs, phi_sc, scale, phis, dt));
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

Status Batch::set_shape(int P, int precision, int seg, int wn) {
    const auto key = std::make_pair(P, precision);
    if (seg == 0 && wn == 0) {
        tuned.erase(key);
    } else {
        if ((seg != 4 && seg != 8 && seg != 16 && seg != 32) || wn < 1 || wn > 7)
            return bad(IDC_ERR_ARG, "batch tile shape: seg must be 4, 8, 16 or 32 and wn in 1..7");
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
    default_shape(P, qmax, seg, wn);
}

Status Batch::autotune(const double *const *srcs, double *const *outs, double dt, int precision) {
    if (members.empty()) return bad(IDC_ERR_STATE, "empty batch");
    for (int P : {1, 2, 3}) {
        bool any = false;
        for (auto *c : members) any |= c->P == P;
        if (!any) continue;
        float best = 1e30f;
        std::pair<int, int> bsh{0, 0};
        for (int cs : {4, 8, 16, 32})
            for (int cw = std::max(1, sweep_modal_max_wn(P) - 3); cw <= sweep_modal_max_wn(P); ++cw) {
                tuned[std::make_pair(P, precision)] = {cs, cw};
                release();
                float ms = 1e30f;
                for (int rep = 0; rep < 4; ++rep) {   // one warm-up, then the best of three
                    IDC_TRY(sweep(srcs, outs, nullptr, 1.0, nullptr, dt, precision));
                    if (rep > 0) ms = std::min(ms, last_ms);
                }
                // the timing covers every degree's launch; the other degrees' shapes stay fixed meanwhile
                if (ms < best) {
                    best = ms;
                    bsh = {cs, cw};
                }
            }
        tuned[std::make_pair(P, precision)] = bsh;
        release();
    }
    return Status::ok();
}

}  // namespace idc
