// Modal persistent wavefront sweep for sm_100a.
//
// Replaces SweepPatternUniCartWavefront::Sweep (linear_solvers/Abstract/SweepPattern/
// SweepPatternUniCartWavefront.cpp:121-332) with the per-cell CalcB / CalcA / GE / StoreResult of
// SweepCellSolveBase::ConstructAndSolve (linear_solvers/RKDG/SweepCellSolve/SweepCellSolve.hpp:312-353),
// solving each (cell, ordinate) system in the packed modal basis of modal_cell.cuh.  What travels from
// a cell to its downwind neighbours is its face trace (P values per ordinate and face), not its N dofs.
//
//   * a compute warp owns Rw = 32/seg consecutive rows; lane (rr, o) = (lane / seg, lane % seg) owns
//     ordinate q_begin + o on row rr.  Row rr runs one column behind row rr-1; its y trace is row rr-1's
//     outgoing trace of the previous step, moved by __shfl_up.  The x trace stays in the lane.
//   * the Wn compute warps of a CTA are stacked in y; warp w's last row hands its outgoing y traces to
//     warp w+1 through a ring of kWarpRingSlots shared-memory slots guarded by full/empty mbarriers.
//   * between CTAs: the CTA's last warp writes its last row's traces, column by column, into the item's
//     trace buffer with relaxed stores, and the helper warp of the item below polls the values
//     themselves (a slot holds a NaN-payload sentinel that arithmetic never produces; 8-byte accesses
//     are single-copy atomic), copies ready columns into ring 0 and re-arms the slots.  The first row
//     block's helper copies the inflow traces of the ghost row (inflow_traces_kernel) instead.
//   * the loop over columns is instantiated per quadrant, so the quadrant's sign flips are constants.
//   * each compute warp has one or two aux warps and a ring of kModalSolutionSlots step slots: an aux
//     warp loads a step's source (cp.async), prepares its inputs (modal source, reciprocals) into the
//     slot, and after the compute warp has left the step result there, transforms it back to the cell
//     dofs, stores psi and forms the moments.  A compute warp's step is thus only the inputs' wait,
//     receive, cell step and send: the cell-to-cell dependency chain and little else.
//   * the fused moments phi = sum_q w_q psi_q: a row segment's weighted values meet in shared memory and
//     one partial moment per (cell, dof, ordinate chunk) is stored; reduce_phi_partials (ops_kernels.cu)
//     adds the chunks in a fixed order, so phi is bitwise reproducible.
//
// Transposed sweep (ADJ): the same schedule in reverse traversal order per quadrant, the transposed cell
// operator and rank-one coupling of modal_cell.cuh, zero inflow, the fused source w_q * mu (the
// transpose of Pmv applied to a moment array mu) and unweighted moment sums (the transpose of Smv's
// broadcast).
//
// Precision: MODE 0 computes in FP64.  MODE 2 computes the modal step in FP32 (traces in FP32).
// MODE 1 keeps FP64 physical traces and right-hand sides and solves each cell by FP32 modal solves
// with FP64 residual corrections (iterative refinement per cell).
//
// Work items (row blocks x quadrant x ordinate chunk) are dequeued in row-block order from an atomic
// counter, so every item's producer is held by a CTA that is already running.  Every wait (mbarrier or
// trace poll) is bounded; on expiry the warp records kDevTimeout in the device error word and leaves,
// and every other warp leaves as soon as it sees the word.  After an error the trace buffer may hold
// values instead of sentinels; the host re-arms it before the next sweep.
// This header holds the kernel templates; sweep_modal_f64.cu, sweep_modal_f32r.cu and sweep_modal_f32.cu
// instantiate them per precision (compiled in parallel) and sweep_modal.cu dispatches.
#pragma once

#include "device_sync.cuh"
#include "idc_internal.hpp"
#include "modal_cell.cuh"

#include <cstdint>
#include <type_traits>

namespace idc {
namespace modal {

constexpr int kS = kWarpRingSlots;
constexpr int kZ = kModalSolutionSlots;

// Warps per CTA: Wn compute warps, the helper warp and nA aux warps per compute warp (the most of 4, 2, 1
// that fit; kZ is a multiple of each), at most 16 warps: one CTA per SM, 128 registers a thread.
__host__ __device__ constexpr int max_warps(int) { return 16; }
__host__ __device__ constexpr int max_compute_warps(int P) { return (max_warps(P) - 1) / 2; }
__host__ __device__ constexpr int aux_per_compute(int P, int wn) {
    return 5 * wn + 1 <= max_warps(P) ? 4 : (3 * wn + 1 <= max_warps(P) ? 2 : 1);
}
__host__ __device__ constexpr int cta_warps(int P, int wn) { return wn * (1 + aux_per_compute(P, wn)) + 1; }

__device__ __forceinline__ int T_steps(int nx, int Rw) { return nx + Rw - 1; }

// Source prefetch depth of an aux warp (cells ahead per lane, in its own steps, which are nA steps apart;
// the loads are issued two of its steps ahead, well beyond the HBM latency at every nA).
__host__ __device__ constexpr int prefetch_depth(int) { return 3; }

// Inputs of one cell step.  MODE 0 / 2: packed modal source and reciprocal denominators.  MODE 1: the
// sign-flipped physical source, FP32 reciprocals and s = sigma_t + 1/dt.
template <int P, int MODE>
struct CellIn {
    using TS = std::conditional_t<MODE == 0, double, float>;
    std::conditional_t<MODE == 1, double, TS> v[P * P];
    ModalRecip<P, TS> r;
    double s;
};
// What an aux warp hands the compute warp per step: the source part and s.  The compute warp forms the
// reciprocals itself (it has slack; the aux warps pace the pipeline), which halves the slot traffic.
template <int P, int MODE>
struct CellSrc {
    using TS = std::conditional_t<MODE == 0, double, float>;
    std::conditional_t<MODE == 1, double, TS> v[P * P];
    double s;
};
template <int P, int MODE>
__host__ __device__ constexpr int slot_words() {
    static_assert(sizeof(CellSrc<P, MODE>) % 8 == 0, "CellSrc is a whole number of 8-byte words");
    return (int)(sizeof(CellSrc<P, MODE>) / 8);
}

struct Layout {
    uint64_t *full, *empty;      // [Wn+1][kS]: y-trace rings
    uint64_t *in_full, *z_full;  // [Wn][kZ]: step slots (inputs ready / result ready)
    double *ring;                // [Wn+1][kS][G][P]: y traces
    double *slot;                // [Wn][kZ][CW + N][32]: a step's inputs (CW 8-byte words) and result
    double *src;                 // [Wn*nA][D][32][N]: an aux warp's prefetched cell source dofs
    double *cellst;              // [Wn*nA][D][32/seg][N+1]: per row: sigma_t, then the fused source's moments[N]
    double *w;                   // [G]
    double *red;                 // [Wn*nA][32][N]: an aux warp's weighted values for the moment reduction
    double *src2;                // [Wn*nA][D][32][N]: the second source's stages (launches with src2 only; the
                                 // launch adds src2_layout_bytes to the shared memory)
};

__host__ __device__ constexpr size_t layout_bytes(int wn, int na, int G, int P, int D, int rw, int cw) {
    return sizeof(uint64_t) * (size_t)(2 * (wn + 1) * kS + 2 * wn * kZ) +
           sizeof(double) * ((size_t)(wn + 1) * kS * G * P + (size_t)wn * kZ * (cw + P * P) * 32 +
                             (size_t)wn * na * D * 32 * P * P + (size_t)wn * na * D * rw * (P * P + 1) +
                             (size_t)((G + 1) & ~1) + (size_t)wn * na * 32 * P * P);
}

// Shared memory of the second source's stages (after the rest of the layout).
__host__ __device__ constexpr size_t src2_layout_bytes(int wn, int na, int P, int D) {
    return sizeof(double) * (size_t)wn * na * D * 32 * P * P;
}

__device__ __forceinline__ Layout carve(unsigned char *raw, int wn, int na, int G, int P, int D, int rw, int cw) {
    const int N = P * P;
    Layout L;
    L.full = reinterpret_cast<uint64_t *>(raw);
    L.empty = L.full + (wn + 1) * kS;
    L.in_full = L.empty + (wn + 1) * kS;
    L.z_full = L.in_full + wn * kZ;
    L.ring = reinterpret_cast<double *>(L.z_full + wn * kZ);
    L.slot = L.ring + (size_t)(wn + 1) * kS * G * P;
    L.src = L.slot + (size_t)wn * kZ * (cw + N) * 32;
    L.cellst = L.src + (size_t)wn * na * D * 32 * N;
    L.w = L.cellst + (size_t)wn * na * D * rw * (N + 1);
    L.red = L.w + ((G + 1) & ~1);
    L.src2 = L.red + (size_t)wn * na * 32 * N;
    return L;
}

template <int P, int MODE, bool XN, bool YN, bool ADJ, bool RECIP = true, bool SRC2 = false>
__device__ __forceinline__ void prep_cell(CellIn<P, MODE> &in, const double *sp, const double *sp2, const double *cp,
                                          const SweepArgs &a,
                                          const ModalOrdinate<P, typename CellIn<P, MODE>::TS> &od, double wq) {
    constexpr int N = P * P;
    using TS = typename CellIn<P, MODE>::TS;
    double src[N];
#pragma unroll
    for (int k = 0; k < N; ++k) src[k] = a.src ? sp[k] : 0.0;
    if constexpr (SRC2) {   // the second source, as the IDC source kernel combines it
#pragma unroll
        for (int k = 0; k < N; ++k) src[k] = fma(a.src2_scale, sp2[k], src[k]);
    }
    if (a.phi_scatter) {
        if constexpr (!ADJ) {   // fused TransportOperator::Smv(scale, 1, sigma_s, phi -> src); the moments
                                // sigma_s phi / (4 pi) come from launch_scatter_moments (no division here)
#pragma unroll
            for (int k = 0; k < N; ++k) src[k] = fma(a.scatter_scale, cp[1 + k], src[k]);
        } else {                // adjoint: the transpose of Pmv, w_q * mu
#pragma unroll
            for (int k = 0; k < N; ++k) src[k] = fma(wq, cp[1 + k], src[k]);
        }
    }
    in.s = cp[0] + a.inv_dt;
    if constexpr (RECIP) in.r = modal_recip<P, TS>(od, TS(in.s));
    if constexpr (MODE != 1) {
        TS v[N];
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = TS(src[k]);
        modal_forward<P, XN, YN, TS, ADJ>(in.v, v);
    } else {
#pragma unroll
        for (int d = 0; d < P; ++d)
#pragma unroll
            for (int e = 0; e < P; ++e) in.v[e + P * d] = flip_sign<XN>(d) * flip_sign<YN>(e) * src[e + P * d];
    }
}

// MODE 1 cell step in the flipped physical frame: B = src' + ax u (x) f + ay g (x) u in FP64, solved by an
// FP32 modal solve and n_refine FP64 residual corrections; f <- outgoing x trace, g_out <- outgoing y trace.
template <int P, bool ADJ>
__device__ __forceinline__ void refined_step(double (&xp)[P * P], const CellIn<P, 1> &in, double (&f)[P],
                                             const double (&g)[P], double (&g_out)[P], double axd, double ayd,
                                             int n_refine) {
    constexpr int N = P * P;
    // coupling vector of the incoming traces (u forward, ones for the transpose) and weights of the
    // outgoing traces (ones forward, u for the transpose)
    auto u = [](int d) { return (d & 1) ? -double(2 * d + 1) : double(2 * d + 1); };
    auto cin = [&](int d) { return ADJ ? 1.0 : u(d); };
    auto tout = [&](int d) { return ADJ ? u(d) : 1.0; };
    double B[N], res[N];
    float bf[N], xf[N];
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e) B[e + P * d] = fma(axd * cin(d), f[e], fma(ayd * cin(e), g[d], in.v[e + P * d]));
#pragma unroll
    for (int k = 0; k < N; ++k) bf[k] = float(B[k]);
    modal_solve_phys<P, float, ADJ>(xf, bf, in.r);
#pragma unroll
    for (int k = 0; k < N; ++k) xp[k] = double(xf[k]);
    for (int it = 0; it < n_refine; ++it) {
        phys_residual<P, ADJ>(res, B, xp, axd, ayd, in.s);
#pragma unroll
        for (int k = 0; k < N; ++k) bf[k] = float(res[k]);
        modal_solve_phys<P, float, ADJ>(xf, bf, in.r);
#pragma unroll
        for (int k = 0; k < N; ++k) xp[k] += double(xf[k]);
    }
#pragma unroll
    for (int e = 0; e < P; ++e) {
        double acc = tout(0) * xp[e];
#pragma unroll
        for (int d = 1; d < P; ++d) acc = fma(tout(d), xp[e + P * d], acc);
        f[e] = acc;
    }
#pragma unroll
    for (int d = 0; d < P; ++d) {
        double acc = tout(0) * xp[P * d];
#pragma unroll
        for (int e = 1; e < P; ++e) acc = fma(tout(e), xp[e + P * d], acc);
        g_out[d] = acc;
    }
}

// Compute warp.  Per column step s the loop runs: wait for the step's prepared inputs (slot s % kZ),
// receive the y trace, the cell step (the only part on the cell-to-cell dependency chain), send the
// outgoing y trace and leave the step result in the slot for the aux warp.  Lanes without a cell this
// step compute on stale inputs; nothing is stored for them.
template <int P, int MODE, int SEG, bool XN, bool YN, bool ADJ>
__device__ __forceinline__ void modal_rows(const SweepArgs &a, const SweepItem &item, const Layout &L, int w,
                                           int lane, bool has_consumer, int it_index) {
    constexpr int N = P * P;
    constexpr int CW = slot_words<P, MODE>();
    using TS = std::conditional_t<MODE == 0, double, float>;   // modal solve type
    using TR = std::conditional_t<MODE == 2, float, double>;   // trace type
    using TZ = std::conditional_t<MODE == 1, double, TS>;      // step result (modal Z, or MODE 1 dofs)
    constexpr int seg = SEG, Rw = 32 / SEG;
    const int G = a.G, rows_cta = a.wn * Rw;
    const int rr = lane / seg, o = lane - rr * seg;
    const int row = item.row_block * rows_cta + w * Rw + rr;
    const bool act = (o < item.q_count) && row < a.ny;
    const int q = item.q_begin + (act ? o : 0);
    const bool last_warp = w == a.wn - 1;

    double axd = 0.0, ayd = 0.0;
    TR f[P];   // x trace (modal, or physical in MODE 1) entering the next cell of this row
#pragma unroll
    for (int m = 0; m < P; ++m) f[m] = TR(0);
    if (act) {
        axd = fabs(a.xi[q]) / a.dx;
        ayd = fabs(a.eta[q]) / a.dy;
        if (a.inflow) {
            const double *in = a.inflow + ((size_t)(a.nx + row) * a.nq + q) * P;
#pragma unroll
            for (int m = 0; m < P; ++m) f[m] = TR(in[m]);
        }
    }
    const ModalOrdinate<P, TS> od = modal_ordinate<P, TS, ADJ>(axd, ayd);
    TR gprev[P];   // this lane's outgoing y trace of the previous step
#pragma unroll
    for (int m = 0; m < P; ++m) gprev[m] = TR(0);
    const unsigned long long *slots = reinterpret_cast<const unsigned long long *>(L.slot) +
                                      (size_t)w * kZ * (CW + N) * 32 + lane;

    const int T = T_steps(a.nx, Rw);
    for (int s = 0; s < T; ++s) {
        const int c = s - rr;
        const bool valid = act && c >= 0 && c < a.nx;
        const int zs = s % kZ;

        // the step's inputs, prepared by the aux warp (word-major in the slot: conflict-free)
        if (!mbar_wait(L.in_full + w * kZ + zs, (uint32_t)((s / kZ) & 1), a.error, a.spin_limit)) break;
        CellIn<P, MODE> cur;
        {
            unsigned long long wv[CW];
            const unsigned long long *sp = slots + (size_t)zs * (CW + N) * 32;
#pragma unroll
            for (int k = 0; k < CW; ++k) wv[k] = sp[k * 32];
            CellSrc<P, MODE> cs;
            memcpy(&cs, wv, sizeof(cs));
#pragma unroll
            for (int k = 0; k < N; ++k) cur.v[k] = cs.v[k];
            cur.s = cs.s;
            cur.r = modal_recip<P, TS>(od, TS(cs.s));
        }

        // y trace: rows rr > 0 from the lane seg below in the warp (previous step), row 0 from the ring
        TR g[P];
#pragma unroll
        for (int m = 0; m < P; ++m) g[m] = __shfl_up_sync(kFullMask, gprev[m], seg);
        if (s < a.nx) {   // warp-uniform: row 0 needs column s
            const int slot = s % kS;
            if (!mbar_wait(L.full + w * kS + slot, (uint32_t)((s / kS) & 1), a.error, a.spin_limit)) break;
            if (rr == 0 && o < G) {
                const double *rp = L.ring + (((size_t)w * kS + slot) * G + o) * P;
#pragma unroll
                for (int m = 0; m < P; ++m) g[m] = TR(rp[m]);
            }
            __syncwarp();
            mbar_arrive(L.empty + w * kS + slot);
        }

        // the cell step: the dependency chain from cell to cell
        TZ Z[N];
        TR fn[P], gout[P];
#pragma unroll
        for (int m = 0; m < P; ++m) fn[m] = f[m];
        if constexpr (MODE != 1)
            modal_step<P, TS, ADJ>(Z, cur.v, fn, g, gout, od, cur.r);
        else
            refined_step<P, ADJ>(Z, cur, fn, g, gout, axd, ayd, a.n_refine);
#pragma unroll
        for (int m = 0; m < P; ++m) {
            f[m] = valid ? fn[m] : f[m];
            gout[m] = valid ? gout[m] : TR(0);
            gprev[m] = gout[m];
        }

        // last row (column s - (Rw-1)): its y traces to ring w+1, or, from the CTA's last warp, to the
        // item's trace buffer that the item below polls (relaxed stores, no fence: each value is its flag)
        const int cout = s - (Rw - 1);
        if (last_warp) {
            if (has_consumer && rr == Rw - 1 && o < item.q_count && cout >= 0 && cout < a.nx) {
                double *tp = a.trace + (size_t)it_index * a.trace_stride + ((size_t)cout * G + o) * P;
#pragma unroll
                for (int m = 0; m < P; ++m) st_relaxed_f64(tp + m, double(gout[m]));
            }
        } else if (cout >= 0 && cout < a.nx) {   // warp-uniform
            const int slot = cout % kS;
            uint64_t *emp = L.empty + (w + 1) * kS + slot;
            if (!mbar_wait(emp, (uint32_t)(((cout / kS) & 1) ^ 1), a.error, a.spin_limit)) break;
            if (rr == Rw - 1 && o < G) {
                double *rp = L.ring + (((size_t)(w + 1) * kS + slot) * G + o) * P;
#pragma unroll
                for (int m = 0; m < P; ++m) rp[m] = double(gout[m]);
            }
            __syncwarp();
            mbar_arrive(L.full + (w + 1) * kS + slot);
        }

        // the step result into the slot (the aux warp reuses the slot for step s + kZ after reading it)
        TZ *zp = reinterpret_cast<TZ *>(L.slot + ((size_t)(w * kZ + zs) * (CW + N) + CW) * 32) + lane;
#pragma unroll
        for (int k = 0; k < N; ++k) zp[k * 32] = Z[k];
        mbar_arrive(L.z_full + w * kZ + zs);
    }
}

// Aux warp k of compute warp w (of na): owns the steps s = k (mod na), so the slots s % kZ with the same
// residue (kZ is a multiple of na).  It prepares the inputs of its first steps, then per owned step s:
// waits for the result, finishes the cell (cell dofs from the backward modal transform or the MODE 1
// sign flips, the psi store, the moments) and prepares step s + kZ in the freed slot.  The source is
// prefetched with cp.async, prefetch_depth() of the warp's own steps ahead, into a per-warp stage ring
// (lane o == 0 of a row also loads sigma_t and the fused source's moments).  A row segment's weighted
// values meet in shared memory; the warp's Rw x N (row, dof) sums over each segment's ordinates are
// spread over the lanes, each a fixed pairwise tree, and stored into this chunk's partial moments.
template <int P, int MODE, int SEG, bool XN, bool YN, bool ADJ, bool SRC2 = false>
__device__ __forceinline__ void modal_aux(const SweepArgs &a, const SweepItem &item, const Layout &L, int w,
                                          int k0, int na, int lane, int it_index) {
    constexpr int N = P * P;
    constexpr int CW = slot_words<P, MODE>();
    using TS = std::conditional_t<MODE == 0, double, float>;
    using TZ = std::conditional_t<MODE == 1, double, TS>;
    constexpr int seg = SEG, Rw = 32 / SEG;
    constexpr int D = prefetch_depth(P);
    constexpr int NC = N + 1;
    const int rr = lane / seg, o = lane - rr * seg;
    const int row_w = item.row_block * a.wn * Rw + w * Rw;
    const int row = row_w + rr;
    const bool row_valid = row < a.ny;
    const bool act = (o < item.q_count) && row_valid;
    const int q = item.q_begin + (act ? o : 0);
    constexpr bool TX = XN != ADJ, TY = YN != ADJ;
    const int j = TY ? (a.ny - row) : (1 + row);
    const size_t plane = (size_t)a.nq * N;
    const size_t istride = (size_t)(a.ny + 2) * plane;
    double axd = 0.0, ayd = 0.0, wq = 0.0;
    if (act) {
        axd = fabs(a.xi[q]) / a.dx;
        ayd = fabs(a.eta[q]) / a.dy;
        wq = L.w[o];
    }
    const ModalOrdinate<P, TS> od = modal_ordinate<P, TS, ADJ>(axd, ayd);
    const int phi_slot = a.phi_slots > 0 ? it_index % a.phi_slots : 0;
    const int ai = w * na + k0;   // this aux warp among the CTA's
    double *red = L.red + (size_t)ai * 32 * N;
    double *my_src = L.src + ((size_t)ai * D * 32 + lane) * N;     // stage b at + b*32*N
    double *my_src2 = L.src2 + ((size_t)ai * D * 32 + lane) * N;   // (launches with src2)
    double *my_cell = L.cellst + ((size_t)ai * D * Rw + rr) * NC;  // stage b at + b*Rw*NC
    const int T = T_steps(a.nx, Rw);

    // the warp's own steps in order: target i is step k0 + i na; one cp.async group per target
    auto prefetch = [&](int i) {
        const int s = k0 + i * na;
        const int c = s - rr;
        if (s < T && row_valid && c >= 0 && c < a.nx) {
            const int ci = TX ? a.nx - c : 1 + c;
            if (act && a.src) {
                const double *g = a.src + (size_t)ci * istride + (size_t)j * plane + (size_t)q * N;
                double *d = my_src + (size_t)(i % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, g + k);
            }
            if (SRC2 && act) {
                const double *g = a.src2 + (size_t)ci * istride + (size_t)j * plane + (size_t)q * N;
                double *d = my_src2 + (size_t)(i % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, g + k);
            }
            if (o == 0) {
                const size_t cidx = (size_t)ci * (a.ny + 2) + j;
                double *d = my_cell + (size_t)(i % D) * Rw * NC;
                cp_async8(d, a.sigma_t + cidx);
                if (a.phi_scatter) {
#pragma unroll
                    for (int k = 0; k < N; ++k) cp_async8(d + 1 + k, a.phi_scatter + cidx * N + k);
                }
            }
        }
        cp_commit();
    };
    // target i's inputs: wait for its stage (one cp.async group per target, in order), form them
    auto stage_in = [&](int i, CellIn<P, MODE> &cur) {
        __syncwarp();   // the row segment's reads of the cell-data stage that lane o == 0 refills are done
        prefetch(i + D - 1);
        cp_wait<D - 2>();   // target i has landed
        __syncwarp();       // lane o == 0's cell-data copies are visible to its row segment
        prep_cell<P, MODE, XN, YN, ADJ, false, SRC2>(cur, my_src + (size_t)(i % D) * 32 * N, my_src2 + (size_t)(i % D) * 32 * N,
                                               my_cell + (size_t)(i % D) * Rw * NC, a, od, wq);
    };
    // ...into its slot, released to the compute warp
    auto publish = [&](int i, const CellIn<P, MODE> &cur) {
        const int s = k0 + i * na;
        CellSrc<P, MODE> cs;
#pragma unroll
        for (int k = 0; k < N; ++k) cs.v[k] = cur.v[k];
        cs.s = cur.s;
        unsigned long long wv[CW];
        memcpy(wv, &cs, sizeof(cs));
        unsigned long long *sp = reinterpret_cast<unsigned long long *>(L.slot) +
                                 ((size_t)(w * kZ + s % kZ) * (CW + N)) * 32 + lane;
#pragma unroll
        for (int k = 0; k < CW; ++k) sp[k * 32] = wv[k];
        mbar_arrive(L.in_full + w * kZ + s % kZ);
    };

#pragma unroll
    for (int i = 0; i < D - 1; ++i) prefetch(i);
    const int ahead = kZ / na;   // targets in flight: the slots this warp owns
    for (int i = 0; i < ahead; ++i) {
        CellIn<P, MODE> cur;
        stage_in(i, cur);
        if (k0 + i * na < T) publish(i, cur);
    }

    for (int i = 0; k0 + i * na < T; ++i) {
        const int s = k0 + i * na;
        const int zs = s % kZ;
        if (!mbar_wait(L.z_full + w * kZ + zs, (uint32_t)((s / kZ) & 1), a.error, a.spin_limit)) break;
        TZ Z[N];
        const TZ *zp = reinterpret_cast<const TZ *>(L.slot + ((size_t)(w * kZ + zs) * (CW + N) + CW) * 32) + lane;
#pragma unroll
        for (int k = 0; k < N; ++k) Z[k] = zp[k * 32];
        // the slot's next step (target i + ahead; a dummy past the last step) and this step's cell dofs:
        // two independent transforms with no barrier between them, so their instructions interleave
        CellIn<P, MODE> nxt;
        stage_in(i + ahead, nxt);
        const int c = s - rr;
        const bool valid = act && c >= 0 && c < a.nx;
        double x[N];
        if constexpr (MODE != 1) {
            TS xv[N];
            modal_backward<P, XN, YN, TS, ADJ>(xv, Z);
#pragma unroll
            for (int k = 0; k < N; ++k) x[k] = double(xv[k]);
        } else {
#pragma unroll
            for (int d = 0; d < P; ++d)
#pragma unroll
                for (int e = 0; e < P; ++e) x[e + P * d] = flip_sign<XN>(d) * flip_sign<YN>(e) * Z[e + P * d];
        }
        // its inputs overwrite nothing the compute warp still reads; the result was read above
        if (k0 + (i + ahead) * na < T) publish(i + ahead, nxt);
        if (a.out && valid) {
            double *op = a.out + (size_t)(TX ? a.nx - c : 1 + c) * istride + (size_t)j * plane + (size_t)q * N;
#pragma unroll
            for (int k = 0; k < N; ++k) op[k] = x[k];
        }
        if (a.phi_part) {
            __syncwarp();   // the previous step's reads of the stage are done
#pragma unroll
            for (int k = 0; k < N; ++k) red[lane * N + k] = valid ? (ADJ ? x[k] : wq * x[k]) : 0.0;
            __syncwarp();
            constexpr int kSums = Rw * N;
#pragma unroll
            for (int m = 0; m < (kSums + 31) / 32; ++m) {
                const int t = lane + 32 * m;
                const int r2 = t / N, k = t - (t / N) * N;
                const int c2 = s - r2, row2 = row_w + r2;
                if (t < kSums && row2 < a.ny && c2 >= 0 && c2 < a.nx) {
                    const double *sr = red + (size_t)r2 * SEG * N + k;
                    double v[SEG];
#pragma unroll
                    for (int oo = 0; oo < SEG; ++oo) v[oo] = sr[oo * N];
#pragma unroll
                    for (int h = 1; h < SEG; h <<= 1)
#pragma unroll
                        for (int oo = 0; oo < SEG; oo += 2 * h) v[oo] += v[oo + h];
                    const int i2 = TX ? a.nx - c2 : 1 + c2, j2 = TY ? (a.ny - row2) : (1 + row2);
                    a.phi_part[(size_t)phi_slot * a.phi_slot_stride + ((size_t)i2 * (a.ny + 2) + j2) * N + k] = v[0];
                }
            }
        }
    }
    cp_wait<0>();
}

// Helper warp: feeds ring 0 with the y traces entering the item's first row -- the ghost row's inflow
// traces for the first row block, otherwise the traces the item above writes column by column (ready
// when none of a column's values is the sentinel; the helper writes the sentinel back for the next
// sweep).  The helper blocks in the barrier unit until the ring slot of its next column is free, then
// loads that column and every further column with a free slot (up to kS): lane l holds values
// l, l + 32, l + 64 of each column, all loads issued before any value is used.
template <int P>
__device__ void modal_helper(const SweepArgs &a, const SweepItem &item, const Layout &L, int lane) {
    constexpr int kV = (32 * P + 31) / 32;   // values per lane and column: chunk <= 32 P
    const int G = a.G;
    const bool has_dep = item.dep >= 0;
    const int chunk = item.q_count * P;   // values per column
    const size_t col_stride = has_dep ? (size_t)G * P : (size_t)a.nq * P;
    double *trace = has_dep ? a.trace + (size_t)item.dep * a.trace_stride : nullptr;
    const double *src = has_dep ? trace : (a.inflow ? a.inflow + (size_t)item.q_begin * P : nullptr);

    int fetch = 0;
    long long idle = 0;
    while (fetch < a.nx) {
        // block (bounded, in the barrier unit) until the slot of column `fetch` is free, then count the
        // free slots after it without blocking
        if (!mbar_wait(L.empty + fetch % kS, (uint32_t)(((fetch / kS) & 1) ^ 1), a.error, a.spin_limit)) break;
        int n = 1;
        if (lane == 0)
            while (n < kS && fetch + n < a.nx &&
                   mbar_test(L.empty + (fetch + n) % kS, (uint32_t)((((fetch + n) / kS) & 1) ^ 1)))
                ++n;
        n = __shfl_sync(kFullMask, n, 0);

        // the item above: wait until the first value of column `fetch` is written before loading the
        // columns (one load per poll, with a bounded back-off, so that many waiting items do not flood L2)
        if (has_dep) {
            int ok = 1;
            if (lane == 0) {
                unsigned ns = 0;
                for (long long poll = 0;; ++poll) {
                    if (!is_sentinel(ld_relaxed_f64(trace + (size_t)fetch * col_stride))) break;
                    if ((poll & 63) == 63 && ld_relaxed(a.error) != kDevOk) {
                        ok = 0;
                        break;
                    }
                    if (poll > a.spin_limit) {
                        atomicCAS(a.error, kDevOk, kDevTimeout);
                        ok = 0;
                        break;
                    }
                    if (ns) __nanosleep(ns);
                    ns = ns ? min(ns * 2, 1024u) : 32u;
                }
            }
            if (!__shfl_sync(kFullMask, ok, 0)) break;
        }

        double v[kS][kV];
        unsigned col_ok = (1u << n) - 1u;   // bit t: column fetch + t complete in this lane
#pragma unroll
        for (int t = 0; t < kS; ++t)
#pragma unroll
            for (int k = 0; k < kV; ++k) {
                const int e = lane + 32 * k;
                v[t][k] = 0.0;
                if (t < n && e < chunk && src) {
                    const double *p = src + (size_t)(fetch + t) * col_stride + e;
                    if (has_dep) {
                        v[t][k] = ld_relaxed_f64(p);
                        if (is_sentinel(v[t][k])) col_ok &= ~(1u << t);
                    } else {
                        v[t][k] = *p;
                    }
                }
            }
        // leading columns that every lane has complete
        const unsigned all_ok = __reduce_and_sync(kFullMask, col_ok);
        int ready = __ffs(~all_ok) - 1;
        if (ready < 0 || ready > n) ready = n;
#pragma unroll
        for (int t = 0; t < kS; ++t)
#pragma unroll
            for (int k = 0; k < kV; ++k) {
                const int e = lane + 32 * k;
                if (t < ready && e < chunk) {
                    L.ring[(size_t)((fetch + t) % kS) * G * P + e] = v[t][k];
                    if (has_dep) st_relaxed_f64(trace + (size_t)(fetch + t) * col_stride + e, sentinel_value());
                }
            }
        if (ready > 0) {
            __syncwarp();
            for (int t = 0; t < ready; ++t) mbar_arrive(L.full + (fetch + t) % kS);
            fetch += ready;
        } else {   // the item above has not written column `fetch` yet: poll again (each poll is an L2
                   // round trip), bounded
            if (((++idle) & 63) == 0 && ld_relaxed(a.error) != kDevOk) break;
            if (idle > a.spin_limit) {
                if (lane == 0) atomicCAS(a.error, kDevOk, kDevTimeout);
                break;
            }
        }
    }
}

template <int P, int MODE, int SEG, bool ADJ, bool BATCHED, bool SRC2 = false>
__global__ void __launch_bounds__(max_warps(P) * 32, 1) sweep_modal_kernel(const SweepArgs a0,
                                                                           const SweepArgs *__restrict__ table) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ int s_stop;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int na = aux_per_compute(P, a0.wn);
    const Layout L = carve(smem_raw, a0.wn, na, a0.G, P, prefetch_depth(P), 32 / SEG, slot_words<P, MODE>());
    const int rows_cta = a0.wn * (32 / SEG);
    __shared__ __align__(16) SweepArgs s_args;   // batched: the current item's problem descriptor

    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(a0.next_item, 1);
            s_item = it;
            s_stop = (it >= a0.n_items) || (ld_relaxed(a0.error) != kDevOk);
            if (!s_stop) {
                for (int b = 0; b < (a0.wn + 1) * kS; ++b) {
                    mbar_init(L.full + b, 32);
                    mbar_init(L.empty + b, 32);
                }
                for (int b = 0; b < a0.wn * kZ; ++b) {
                    mbar_init(L.in_full + b, 32);
                    mbar_init(L.z_full + b, 32);
                }
            }
        }
        __syncthreads();
        const int it = s_item;
        if (s_stop) return;
        const SweepItem item = a0.items[it];
        if constexpr (BATCHED) {
            const unsigned long long *sw = reinterpret_cast<const unsigned long long *>(table + item.problem);
            unsigned long long *dw = reinterpret_cast<unsigned long long *>(&s_args);
            for (int k = threadIdx.x; k < (int)(sizeof(SweepArgs) / 8); k += blockDim.x) dw[k] = sw[k];
            __syncthreads();
            if (s_args.skip) {   // a problem left out of this sweep (block-uniform): take the next item
                __syncthreads();
                continue;
            }
        }
        const SweepArgs &a = BATCHED ? s_args : a0;
        // the item's index within its problem (its trace buffer and partial-moment slot)
        const int local = BATCHED ? item.local : it;
        if ((int)threadIdx.x < item.q_count) L.w[threadIdx.x] = a.w[item.q_begin + threadIdx.x];
        __syncthreads();
        const bool has_consumer = (item.row_block + 1) * rows_cta < a.ny;
        if (warp < a0.wn) {
            switch (item.quadrant) {
                case 0: modal_rows<P, MODE, SEG, false, false, ADJ>(a, item, L, warp, lane, has_consumer, local); break;
                case 1: modal_rows<P, MODE, SEG, false, true, ADJ>(a, item, L, warp, lane, has_consumer, local); break;
                case 2: modal_rows<P, MODE, SEG, true, false, ADJ>(a, item, L, warp, lane, has_consumer, local); break;
                default: modal_rows<P, MODE, SEG, true, true, ADJ>(a, item, L, warp, lane, has_consumer, local); break;
            }
        } else if (warp == a0.wn) {
            modal_helper<P>(a, item, L, lane);
        } else {
            const int ax = warp - a0.wn - 1, w = ax / na, k0 = ax - w * na;   // aux warp k0 of compute warp w
            switch (item.quadrant) {
                case 0: modal_aux<P, MODE, SEG, false, false, ADJ, SRC2>(a, item, L, w, k0, na, lane, local); break;
                case 1: modal_aux<P, MODE, SEG, false, true, ADJ, SRC2>(a, item, L, w, k0, na, lane, local); break;
                case 2: modal_aux<P, MODE, SEG, true, false, ADJ, SRC2>(a, item, L, w, k0, na, lane, local); break;
                default: modal_aux<P, MODE, SEG, true, true, ADJ, SRC2>(a, item, L, w, k0, na, lane, local); break;
            }
        }
        __syncthreads();
    }
}

template <int P, int MODE, int SEG, bool ADJ>
cudaError_t launch_seg(const SweepArgs &args, int grid, size_t smem, cudaStream_t stream) {
    // the second source has its own instantiation (forward, FP64 and refined precision), so the other
    // launches run the kernel without it
    auto kern = sweep_modal_kernel<P, MODE, SEG, ADJ, false>;
    if constexpr (!ADJ && MODE != 2) {
        if (args.src2) kern = sweep_modal_kernel<P, MODE, SEG, false, false, true>;
    } else {
        if (args.src2) return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, cta_warps(P, args.wn) * 32, smem, stream>>>(args, nullptr);
    return cudaGetLastError();
}

template <int P, int MODE, int SEG>
cudaError_t launch_seg_batched(const SweepArgs &launch, const SweepArgs *table, int grid, size_t smem,
                               cudaStream_t stream) {
    auto kern = sweep_modal_kernel<P, MODE, SEG, false, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, cta_warps(P, launch.wn) * 32, smem, stream>>>(launch, table);
    return cudaGetLastError();
}

template <int P, int MODE, int SEG, bool ADJ>
cudaError_t occ_seg(int threads, size_t smem, int *n) {
    auto kern = sweep_modal_kernel<P, MODE, SEG, ADJ, false>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, kern, threads, smem);
}

}  // namespace modal
}  // namespace idc

// Explicit instantiation (or extern declaration, DECL = extern) of the launchers of one precision and
// direction for every degree and row-segment width.
#define IDC_MODAL_LAUNCHERS(DECL, MODE, ADJ)                                                                  \
    DECL template cudaError_t idc::modal::launch_seg<1, MODE, 4, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg<1, MODE, 8, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg<1, MODE, 16, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg<1, MODE, 32, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg<2, MODE, 4, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg<2, MODE, 8, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg<2, MODE, 16, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg<2, MODE, 32, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg<3, MODE, 4, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg<3, MODE, 8, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg<3, MODE, 16, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg<3, MODE, 32, ADJ>(const idc::SweepArgs &, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::occ_seg<1, MODE, 4, ADJ>(int, size_t, int *);                             \
    DECL template cudaError_t idc::modal::occ_seg<1, MODE, 8, ADJ>(int, size_t, int *);                             \
    DECL template cudaError_t idc::modal::occ_seg<1, MODE, 16, ADJ>(int, size_t, int *);                            \
    DECL template cudaError_t idc::modal::occ_seg<1, MODE, 32, ADJ>(int, size_t, int *);                            \
    DECL template cudaError_t idc::modal::occ_seg<2, MODE, 4, ADJ>(int, size_t, int *);                             \
    DECL template cudaError_t idc::modal::occ_seg<2, MODE, 8, ADJ>(int, size_t, int *);                             \
    DECL template cudaError_t idc::modal::occ_seg<2, MODE, 16, ADJ>(int, size_t, int *);                            \
    DECL template cudaError_t idc::modal::occ_seg<2, MODE, 32, ADJ>(int, size_t, int *);                            \
    DECL template cudaError_t idc::modal::occ_seg<3, MODE, 4, ADJ>(int, size_t, int *);                             \
    DECL template cudaError_t idc::modal::occ_seg<3, MODE, 8, ADJ>(int, size_t, int *);                             \
    DECL template cudaError_t idc::modal::occ_seg<3, MODE, 16, ADJ>(int, size_t, int *);                            \
    DECL template cudaError_t idc::modal::occ_seg<3, MODE, 32, ADJ>(int, size_t, int *);

#define IDC_MODAL_BATCHED(DECL, MODE)                                                                              \
    DECL template cudaError_t idc::modal::launch_seg_batched<1, MODE, 4>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg_batched<1, MODE, 8>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg_batched<1, MODE, 16>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg_batched<1, MODE, 32>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg_batched<2, MODE, 4>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg_batched<2, MODE, 8>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg_batched<2, MODE, 16>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg_batched<2, MODE, 32>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg_batched<3, MODE, 4>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg_batched<3, MODE, 8>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);  \
    DECL template cudaError_t idc::modal::launch_seg_batched<3, MODE, 16>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t); \
    DECL template cudaError_t idc::modal::launch_seg_batched<3, MODE, 32>(const idc::SweepArgs &, const idc::SweepArgs *, int, size_t, cudaStream_t);
