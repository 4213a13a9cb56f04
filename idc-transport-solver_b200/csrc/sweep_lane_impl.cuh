// Lane-pipelined persistent wavefront sweep for sm_100a.
//
// Replaces SweepPatternUniCartWavefront::Sweep (linear_solvers/Abstract/SweepPattern/
// SweepPatternUniCartWavefront.cpp:121-332) with the per-cell CalcB / CalcA / GE / StoreResult of
// SweepCellSolveBase::ConstructAndSolve (linear_solvers/RKDG/SweepCellSolve/SweepCellSolve.hpp:312-353),
// in the packed modal basis of modal_cell.cuh (the same cell arithmetic as sweep_modal_impl.cuh).
//
// Every warp is an independent worker with its own work item: Rw = 32/SEG consecutive rows (in sweep
// order) of one quadrant for one chunk of <= SEG ordinates, swept across all columns.  Lane (rr, o) =
// (lane / SEG, lane % SEG) owns ordinate q_begin + o on row rr; row rr runs one column behind row rr-1 and
// takes its y trace by __shfl_up, the x trace stays in the lane.  A step of the warp does, for every lane,
// everything that cell needs, so there is no hand-off between warps inside a thread block at all:
//   * the chain: the y trace in, the modal cell step, the traces out (the only cell-to-cell dependency);
//   * the inputs of the next step: its source dofs (staged in shared memory by cp.async, kStages steps
//     ahead), sigma_t, the fused scattering moments and second source, the forward modal transform and
//     the reciprocal denominators -- independent of the chain, so the compiler interleaves them with it;
//   * the finish of this step: the backward transform, the psi store and the row segment's moment sums
//     (one partial per ordinate chunk, added in a fixed order by reduce_phi_partials: bitwise
//     reproducible).
// A warp has few neighbours on its SM sub-partition (four warps per thread block, one per sub-partition,
// one or two blocks per SM), so it may hold up to 255 registers and its step is one long stretch of
// independent instructions around a short dependency chain.
//
// Between row blocks: the warp's last row writes its outgoing y traces, column by column, into the item's
// trace buffer with relaxed 8-byte stores; the warp of the item below loads them kTraceAhead steps before
// it needs them (the loop is unrolled by that depth so that the values stay in registers), finds a slot
// still holding the NaN-payload sentinel only if it caught up with its producer (then it polls that
// column, bounded), and writes the sentinel back after use.  The first row block reads the ghost row's
// inflow traces (inflow_traces_kernel) instead.  Items are dequeued per warp in row-block order from an
// atomic counter, so an item's producer is always held by a running warp: no deadlock, and no thread
// block needs any other to be resident.  Every wait is bounded (spin_limit); on expiry the warp records
// kDevTimeout in the device error word and leaves, and every other warp leaves when it sees the word.
//
// Transposed sweep (ADJ): reverse traversal order per quadrant, the transposed cell operator and coupling
// of modal_cell.cuh, zero inflow, the fused source w_q * mu and unweighted moment sums (the transposes of
// Smv's broadcast and of Pmv).  SRC2 adds a second source, fma(src2_scale, src2, src), as the IDC source
// kernel combines them.  FP64 arithmetic (the reference's).
#pragma once

#include "device_sync.cuh"
#include "idc_internal.hpp"
#include "modal_cell.cuh"

#include <cstdint>

namespace idc {
namespace lane {

constexpr int kWarps = 4;        // warps per thread block: one per SM sub-partition
constexpr int kStages = 6;       // source stages in shared memory: a step's inputs are loaded this many steps ahead
constexpr int kTraceAhead = 4;   // row 0's y traces are loaded this many steps before use

// Shared memory of one warp, in doubles: source stages [kStages][32][N] (lane-major, conflict-free),
// the second source's stages (launches with one), cell-data stages [kStages][Rw][1 + N] (sigma_t and the
// fused scattering moments, loaded by lane o == 0 of each row) and the moment reduction buffer [32][N].
__host__ __device__ constexpr size_t warp_doubles(int P, int seg, bool src2) {
    return (size_t)kStages * 32 * P * P * (src2 ? 2 : 1) + (size_t)kStages * (32 / seg) * (P * P + 1) +
           (size_t)32 * P * P;
}
__host__ __device__ constexpr size_t block_smem_bytes(int P, int seg, bool src2) {
    return sizeof(double) * warp_doubles(P, seg, src2) * kWarps;
}

template <int P, int SEG, bool XN, bool YN, bool ADJ, bool SRC2>
__device__ __forceinline__ void run_item(const SweepArgs &a, const SweepItem &item, int it_index, double *wsm,
                                         int lane) {
    constexpr int N = P * P, Rw = 32 / SEG, D = kStages, K = kTraceAhead, NC = N + 1;
    constexpr bool TX = XN != ADJ, TY = YN != ADJ;
    const int rr = lane / SEG, o = lane - rr * SEG;
    const int row_w = item.row_block * Rw;
    const int row = row_w + rr;
    const bool row_valid = row < a.ny;
    const bool act = (o < item.q_count) && row_valid;
    const int q = item.q_begin + (act ? o : 0);
    const int j = TY ? (a.ny - row) : (1 + row);
    const int nx = a.nx, G = a.G;
    const size_t plane = (size_t)a.nq * N;
    const size_t istride = (size_t)(a.ny + 2) * plane;
    const bool has_dep = item.dep >= 0;
    const bool has_consumer = row_w + Rw < a.ny;
    const int T = nx + Rw - 1;

    double *stage = wsm + (size_t)lane * N;                           // step t at + (t % D) * 32 * N
    double *stage2 = wsm + (size_t)D * 32 * N + (size_t)lane * N;     // (SRC2 launches only)
    double *cell = wsm + (size_t)D * 32 * N * (SRC2 ? 2 : 1) + (size_t)rr * NC;   // + (t % D) * Rw * NC
    double *red = cell - (size_t)rr * NC + (size_t)D * Rw * NC;      // [32][N]

    double axd = 0.0, ayd = 0.0, wq = 0.0;
    if (act) {
        axd = fabs(a.xi[q]) / a.dx;
        ayd = fabs(a.eta[q]) / a.dy;
        wq = a.w[q];
    }
    const ModalOrdinate<P, double> od = modal_ordinate<P, double, ADJ>(axd, ayd);

    // the row's x trace entering its first column (ghost-column inflow; zero for the transposed sweep)
    double f[P];
#pragma unroll
    for (int m = 0; m < P; ++m) f[m] = 0.0;
    if (act && a.inflow && !ADJ) {
        const double *in = a.inflow + ((size_t)(nx + row) * a.nq + q) * P;
#pragma unroll
        for (int m = 0; m < P; ++m) f[m] = in[m];
    }

    // where row 0 of this item reads its y traces: the item above (sentinel-armed) or the ghost row's inflow
    const bool reader = rr == 0 && o < item.q_count && row_valid;
    double *dep_trace = has_dep ? a.trace + (size_t)item.dep * a.trace_stride + (size_t)o * P : nullptr;
    const double *inflow_y = (!has_dep && a.inflow && !ADJ) ? a.inflow + (size_t)q * P : nullptr;
    auto load_trace = [&](int c, double (&v)[P]) {
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = 0.0;
        if (reader && c < nx) {
            if (has_dep) {
#pragma unroll
                for (int m = 0; m < P; ++m) v[m] = ld_relaxed_f64(dep_trace + (size_t)c * G * P + m);
            } else if (inflow_y) {
#pragma unroll
                for (int m = 0; m < P; ++m) v[m] = inflow_y[(size_t)c * a.nq * P + m];
            }
        }
    };
    double *out_trace = a.trace + (size_t)it_index * a.trace_stride + (size_t)o * P;
    const bool writer = has_consumer && rr == Rw - 1 && o < item.q_count;

    // step t's inputs into stage t % D: the source dofs (every active lane its own), sigma_t and the fused
    // scattering moments (lane o == 0 of the row); one cp.async group per step, empty past the last
    auto prefetch = [&](int t) {
        const int c = t - rr;
        if (t < T && row_valid && c >= 0 && c < nx) {
            const int ci = TX ? nx - c : 1 + c;
            const size_t base = (size_t)ci * istride + (size_t)j * plane + (size_t)q * N;
            if (act && a.src) {
                double *d = stage + (size_t)(t % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, a.src + base + k);
            }
            if (SRC2 && act) {
                double *d = stage2 + (size_t)(t % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, a.src2 + base + k);
            }
            if (o == 0) {
                const size_t cidx = (size_t)ci * (a.ny + 2) + j;
                double *d = cell + (size_t)(t % D) * Rw * NC;
                cp_async8(d, a.sigma_t + cidx);
                if (a.phi_scatter) {
#pragma unroll
                    for (int k = 0; k < N; ++k) cp_async8(d + 1 + k, a.phi_scatter + cidx * N + k);
                }
            }
        }
        cp_commit();
    };

    // step t's modal source and reciprocals from its landed stage
    auto prepare = [&](int t, double (&S)[N], ModalRecip<P, double> &r) {
        const double *sp = stage + (size_t)(t % D) * 32 * N;
        const double *cp = cell + (size_t)(t % D) * Rw * NC;
        double src[N];
#pragma unroll
        for (int k = 0; k < N; ++k) src[k] = a.src ? sp[k] : 0.0;
        if constexpr (SRC2) {
            const double *sp2 = stage2 + (size_t)(t % D) * 32 * N;
#pragma unroll
            for (int k = 0; k < N; ++k) src[k] = fma(a.src2_scale, sp2[k], src[k]);
        }
        if (a.phi_scatter) {
            if constexpr (!ADJ) {   // fused TransportOperator::Smv(scale, 1, sigma_s, phi -> src)
#pragma unroll
                for (int k = 0; k < N; ++k) src[k] += a.scatter_scale * cp[1 + k];
            } else {                // the transpose of Pmv: w_q * mu
#pragma unroll
                for (int k = 0; k < N; ++k) src[k] = fma(wq, cp[1 + k], src[k]);
            }
        }
        r = modal_recip<P, double>(od, cp[0] + a.inv_dt);
        modal_forward<P, XN, YN, double, ADJ>(S, src);
    };

    const int phi_slot = a.phi_slots > 0 ? it_index % a.phi_slots : 0;
    long long polls = 0;
    bool failed = false;

    // prologue: stages 0 .. D-2 in flight, step 0 prepared, row 0's traces of columns 0 .. K-1 loaded
#pragma unroll
    for (int t = 0; t < D - 1; ++t) prefetch(t);
    cp_wait<D - 2>();
    __syncwarp();
    double S[N];
    ModalRecip<P, double> r;
    prepare(0, S, r);
    double tr[K][P];
#pragma unroll
    for (int u = 0; u < K; ++u) load_trace(u, tr[u]);
    double gprev[P];
#pragma unroll
    for (int m = 0; m < P; ++m) gprev[m] = 0.0;

    for (int s0 = 0; s0 < T && !failed; s0 += K) {
#pragma unroll
        for (int u = 0; u < K; ++u) {
            const int s = s0 + u;
            if (s >= T || failed) break;   // warp-uniform
            const int c = s - rr;
            const bool valid = act && c >= 0 && c < nx;

            // ---- the y trace in: from the lane seg below (previous step), row 0 from the item above ----
            double g[P];
#pragma unroll
            for (int m = 0; m < P; ++m) g[m] = __shfl_up_sync(kFullMask, gprev[m], SEG);
            if (has_dep && s < nx) {   // row 0 consumes column s of the item above
                bool bad = false;
#pragma unroll
                for (int m = 0; m < P; ++m) bad |= reader && is_sentinel(tr[u][m]);
                if (__any_sync(kFullMask, bad)) {   // caught up with the producer: poll this column, bounded
                    unsigned ns = 32;
                    for (;;) {
                        bool still = false;
                        if (reader) {
#pragma unroll
                            for (int m = 0; m < P; ++m) {
                                if (is_sentinel(tr[u][m])) tr[u][m] = ld_relaxed_f64(dep_trace + (size_t)s * G * P + m);
                                still |= is_sentinel(tr[u][m]);
                            }
                        }
                        if (!__any_sync(kFullMask, still)) break;
                        ++polls;
                        if ((polls & 63) == 63 && ld_relaxed(a.error) != kDevOk) {
                            failed = true;
                            break;
                        }
                        if (polls > a.spin_limit) {
                            if (lane == 0) atomicCAS(a.error, kDevOk, kDevTimeout);
                            failed = true;
                            break;
                        }
                        __nanosleep(ns);
                        ns = ns < 1024 ? ns * 2 : 1024;
                    }
                    if (failed) break;
                }
            }
            if (rr == 0) {
#pragma unroll
                for (int m = 0; m < P; ++m) g[m] = tr[u][m];
            }

            // ---- the cell step: the chain from cell to cell ----
            double Z[N], fn[P], gout[P];
#pragma unroll
            for (int m = 0; m < P; ++m) fn[m] = f[m];
            modal_step<P, double, ADJ>(Z, S, fn, g, gout, od, r);
#pragma unroll
            for (int m = 0; m < P; ++m) {
                f[m] = valid ? fn[m] : f[m];
                gprev[m] = valid ? gout[m] : 0.0;
            }

            // ---- traces out (relaxed stores: each value is its own flag) and row 0's trace bookkeeping ----
            const int cout = s - (Rw - 1);
            if (writer && cout >= 0 && cout < nx) {
#pragma unroll
                for (int m = 0; m < P; ++m) st_relaxed_f64(out_trace + (size_t)cout * G * P + m, gout[m]);
            }
            if (reader && has_dep && s < nx) {   // re-arm the consumed column for the next sweep
#pragma unroll
                for (int m = 0; m < P; ++m) st_relaxed_f64(dep_trace + (size_t)s * G * P + m, sentinel_value());
            }
            load_trace(s + K, tr[u]);

            // ---- the next step's inputs (independent of the chain) ----
            prefetch(s + D - 1);   // into the stage step s - 1 used (read while preparing it, a step ago)
            cp_wait<D - 2>();      // step s + 1's group has landed
            __syncwarp();   // lane o == 0's cell data of step s + 1 is visible to its row
            prepare(s + 1, S, r);

            // ---- this step's finish: cell dofs, psi, moments ----
            double x[N];
            modal_backward<P, XN, YN, double, ADJ>(x, Z);
            if (a.out && valid) {
                double *op = a.out + (size_t)(TX ? nx - c : 1 + c) * istride + (size_t)j * plane + (size_t)q * N;
#pragma unroll
                for (int k = 0; k < N; ++k) op[k] = x[k];
            }
            if (a.phi_part) {
#pragma unroll
                for (int k = 0; k < N; ++k) red[lane * N + k] = valid ? (ADJ ? x[k] : wq * x[k]) : 0.0;
                __syncwarp();
                constexpr int kSums = Rw * N;
#pragma unroll
                for (int mm = 0; mm < (kSums + 31) / 32; ++mm) {
                    const int t = lane + 32 * mm;
                    const int r2 = t / N, k = t - (t / N) * N;
                    const int c2 = s - r2, row2 = row_w + r2;
                    if (t < kSums && row2 < a.ny && c2 >= 0 && c2 < nx) {
                        const double *sr = red + (size_t)r2 * SEG * N + k;
                        double v[SEG];
#pragma unroll
                        for (int oo = 0; oo < SEG; ++oo) v[oo] = sr[oo * N];
#pragma unroll
                        for (int h = 1; h < SEG; h <<= 1)
#pragma unroll
                            for (int oo = 0; oo < SEG; oo += 2 * h) v[oo] += v[oo + h];
                        const int i2 = TX ? nx - c2 : 1 + c2, j2 = TY ? (a.ny - row2) : (1 + row2);
                        a.phi_part[(size_t)phi_slot * a.phi_slot_stride + ((size_t)i2 * (a.ny + 2) + j2) * N + k] = v[0];
                    }
                }
                __syncwarp();   // the sums are read before the next step overwrites the buffer
            }
        }
    }
    cp_wait<0>();
    __syncwarp();
}

template <int P, int SEG, bool ADJ, bool SRC2>
__global__ void __launch_bounds__(kWarps * 32, 1) sweep_lane_kernel(const SweepArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double *wsm = reinterpret_cast<double *>(smem_raw) + warp_doubles(P, SEG, SRC2) * warp;
    for (;;) {
        int it = 0;
        if (lane == 0) {
            it = atomicAdd(a.next_item, 1);
            if (ld_relaxed(a.error) != kDevOk) it = a.n_items;
        }
        it = __shfl_sync(kFullMask, it, 0);
        if (it >= a.n_items) return;
        const SweepItem item = a.items[it];
        switch (item.quadrant) {
            case 0: run_item<P, SEG, false, false, ADJ, SRC2>(a, item, it, wsm, lane); break;
            case 1: run_item<P, SEG, false, true, ADJ, SRC2>(a, item, it, wsm, lane); break;
            case 2: run_item<P, SEG, true, false, ADJ, SRC2>(a, item, it, wsm, lane); break;
            default: run_item<P, SEG, true, true, ADJ, SRC2>(a, item, it, wsm, lane); break;
        }
    }
}

template <int P, int SEG, bool ADJ, bool SRC2>
cudaError_t launch(const SweepArgs &args, int grid, cudaStream_t stream) {
    auto kern = sweep_lane_kernel<P, SEG, ADJ, SRC2>;
    const size_t smem = block_smem_bytes(P, SEG, SRC2);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kWarps * 32, smem, stream>>>(args);
    return cudaGetLastError();
}

template <int P, int SEG, bool ADJ, bool SRC2>
cudaError_t occupancy(int *blocks_per_sm) {
    auto kern = sweep_lane_kernel<P, SEG, ADJ, SRC2>;
    const size_t smem = block_smem_bytes(P, SEG, SRC2);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, kWarps * 32, smem);
}

}  // namespace lane
}  // namespace idc
