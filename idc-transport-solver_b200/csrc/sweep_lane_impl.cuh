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
// takes its y trace by __shfl_up, the x trace stays in the lane.  Iteration s of a warp does, for every
// lane, all the work of three cells, with no barrier between them, so the compiler can interleave their
// instructions and each hides the others' latencies:
//   * the chain of step s: the y trace in, the modal cell step, the traces out (the only dependency from
//     cell to cell, so the only part whose latency sits on the wavefront's critical path);
//   * the finish of step s - 1: the backward transform, the psi store, and the row segment's moment sums
//     by a butterfly of shuffles (one partial per ordinate chunk, each sum a fixed tree, added in a fixed
//     order by reduce_phi_partials: bitwise reproducible);
//   * the inputs of step s + 1: its source dofs and sigma_t (and the second source), copied into shared
//     memory by cp.async kStages - 1 steps ahead, each lane its own (lane o == 0 of a row copies the fused
//     scattering moments and hands them to its row by shuffles), the forward modal transform and the
//     reciprocal denominators.
// The loop body is one iteration for every quadrant (the quadrant's sign flips are applied to the cell
// values at run time as sign-bit flips, exact), so the hot loop stays small for the instruction caches.
// Four warps per thread block, one per SM sub-partition; a warp may hold up to 255 registers.  Measured on
// B200: one warp with enough independent work issues FP64 at the sub-partition's full rate.
//
// Between row blocks: the warp's last row writes its outgoing y traces, column by column, into the item's
// trace buffer with relaxed 8-byte stores; row 0 of the item below loads column s + 1 with relaxed loads
// at iteration s (a whole iteration, longer than an L2 round trip, before use).  A value still holding the
// NaN-payload sentinel means the consumer has caught up with its producer: it then polls (bounded) until
// the producer is two columns further, which gives it slack for the next loads.  The consumer writes the
// sentinel back after use.  The first row block reads the ghost row's inflow traces (inflow_traces_kernel)
// the same way.  Items are dequeued per warp in row-block order from an atomic counter, so an item's
// producer is always held by a running warp: no deadlock, and no thread block needs any other to be
// resident.  Every wait is bounded (spin_limit); on expiry the warp records kDevTimeout in the device
// error word and leaves, and every other warp leaves when it sees the word.
//
// Transposed sweep (ADJ): reverse traversal order per quadrant, the transposed cell operator and coupling
// of modal_cell.cuh, zero inflow, the fused source w_q * mu and unweighted moment sums (the transposes of
// Smv's broadcast and of Pmv).  SRC2 adds a second source, fma(src2_scale, src2, src), as the IDC source
// kernel combines them.  PHI: the moments-only forward sweep of the Krylov iterations (no source array,
// psi not stored): the cell's source is its isotropic scattering source, the same for every ordinate of a
// quadrant, read already in the packed modal basis (launch_modal_sources, once per cell and quadrant), and
// the moments are summed in the packed basis (launch_reduce_modal_partials transforms each quadrant's sum
// back once per cell), so neither modal transform is done per ordinate.  TC is the arithmetic: double (the
// reference's FP64) or float (the unrefined FP32 sweep of IDC_PREC_FP32: FP32 cell arithmetic and moment
// sums, FP64 arrays and traces), forward sweeps only.
#pragma once

#include "device_sync.cuh"
#include "idc_internal.hpp"
#include "modal_cell.cuh"

#include <cstdint>

namespace idc {
namespace lane {

constexpr int kWarps = 4;    // warps per thread block: one per SM sub-partition
constexpr int kStages = 8;   // stages in shared memory (a power of two): a step's inputs are copied this many steps minus one ahead

// Doubles per (column, ordinate) slot of the trace buffer.
__host__ __device__ constexpr int trace_slot(int P) { return P; }

// Shared memory of one warp, in doubles: source stages [kStages][32][N] (lane-major, conflict-free), the
// second source's stages (launches with one), sigma_t stages [kStages][32] (each lane its own copy) and the
// fused scattering moments' stages [kStages][Rw][N] (copied by lane o == 0 of each row).
__host__ __device__ constexpr size_t warp_doubles(int P, int seg, bool src2) {
    return (size_t)kStages * 32 * P * P * (src2 ? 2 : 1) + (size_t)kStages * 32 + (size_t)kStages * (32 / seg) * P * P;
}
__host__ __device__ constexpr size_t block_smem_bytes(int P, int seg, bool src2) {
    return sizeof(double) * warp_doubles(P, seg, src2) * kWarps;
}

// x with its sign bit flipped where `mask` has it (mask: 0 or 0x80000000, the sign bit of a float or of a
// double's high word).
__device__ __forceinline__ double flip_by(double x, unsigned mask) {
    return __hiloint2double(__double2hiint(x) ^ (int)mask, __double2loint(x));
}
__device__ __forceinline__ float flip_by(float x, unsigned mask) { return __int_as_float(__float_as_int(x) ^ (int)mask); }

// Sums of v[0 .. N) over the SEG lanes of a row segment (o = lane % SEG) by recursive halving: at the
// stage of distance h a lane keeps the lower half of its current range if bit h of o is clear, the upper
// half otherwise, and adds its partner's copy of it (the halves always sit in slots 0 .. len-1).  After
// log2(SEG) stages lane o holds the sums of k in [*lo, *hi) in slots 0 .. *hi - *lo.  Every sum is a fixed
// tree over the segment's lanes.
template <int N, int SEG, int LEN = N, int H = SEG / 2, typename T>
__device__ __forceinline__ void segment_sums(T (&v)[N], int o, int *lo, int *hi) {
    if constexpr (H >= 1) {
        constexpr int HALF = (LEN + 1) / 2;
        const bool upper = (o & H) != 0;
#pragma unroll
        for (int i = 0; i < HALF; ++i) {
            const T keep = upper ? (i + HALF < LEN ? v[i + HALF] : T(0)) : v[i];
            const T give = upper ? v[i] : (i + HALF < LEN ? v[i + HALF] : T(0));
            v[i] = keep + __shfl_xor_sync(kFullMask, give, H);
        }
        const int mid = *lo + HALF;
        if (upper)
            *lo = mid < *hi ? mid : *hi;
        else
            *hi = mid < *hi ? mid : *hi;
        segment_sums<N, SEG, HALF, H / 2, T>(v, o, lo, hi);
    }
}

// The consumer caught up with its producer (a value of column s still held the sentinel): wait until the
// producer has written column `last` and all of column s, bounded.  Returns false if the wait gave up or
// another warp has failed (the error word is then set).  Out of line: the hot loop stays small.
template <int P>
__device__ __noinline__ bool wait_for_producer(const double *dep_trace, int s, int last, bool reader, int G,
                                               int *error, long long spin_limit, long long *polls, int lane) {
    const size_t col = (size_t)G * P;
    for (int want = last;;) {
        bool still = false;
        if (reader) {
#pragma unroll
            for (int m = 0; m < P; ++m) still |= is_sentinel(ld_relaxed_f64(dep_trace + (size_t)want * col + m));
        }
        if (!__any_sync(kFullMask, still)) {
            if (want == s) return true;
            want = s;
            continue;
        }
        ++*polls;
        if ((*polls & 63) == 63 && ld_relaxed(error) != kDevOk) return false;
        if (*polls > spin_limit) {
            if (lane == 0) atomicCAS(error, kDevOk, kDevTimeout);
            return false;
        }
        __nanosleep(64);
    }
}

template <int P, int SEG, bool ADJ, bool SRC2, bool PHI, typename TC>
__device__ __forceinline__ void run_item(const SweepArgs &a, const SweepItem &item, int it_index, double *wsm,
                                         int lane) {
    constexpr int N = P * P, Rw = 32 / SEG, D = kStages;
    // quadrant signs: flips of the cell values (exact), traversal directions (reversed for the transpose)
    const bool XN = item.quadrant >= 2, YN = (item.quadrant & 1) != 0;
    const bool TX = XN != ADJ, TY = YN != ADJ;
    const int rr = lane / SEG, o = lane - rr * SEG;
    const int row_w = item.row_block * Rw;
    const int row = row_w + rr;
    const bool row_valid = row < a.ny;
    const bool act = (o < item.q_count) && row_valid;
    const int q = item.q_begin + (act ? o : 0);
    const int j = TY ? (a.ny - row) : (1 + row);
    const int nx = a.nx;
    const size_t plane = (size_t)a.nq * N;
    const size_t istride = (size_t)(a.ny + 2) * plane;
    const bool has_dep = item.dep >= 0;
    const bool has_consumer = row_w + Rw < a.ny;
    const int T = nx + Rw - 1;
    const size_t tcol = (size_t)a.G * P;   // doubles per trace column
    const int xi0 = TX ? nx : 1, xis = TX ? -1 : 1;   // array x index of sweep column c: xi0 + xis * c
    const unsigned xm = XN ? 0x80000000u : 0u, ym = YN ? 0x80000000u : 0u;
    auto fmask = [&](int k) { return ((k / P) & 1 ? xm : 0u) ^ ((k % P) & 1 ? ym : 0u); };   // k = e + P d

    double *stage = wsm + (size_t)lane * N;                            // step t at + (t % D) * 32 * N
    double *stage2 = wsm + (size_t)D * 32 * N + (size_t)lane * N;      // (SRC2 launches only)
    double *sig = wsm + (size_t)D * 32 * N * (SRC2 ? 2 : 1) + lane;    // + (t % D) * 32
    double *mom = wsm + (size_t)D * 32 * N * (SRC2 ? 2 : 1) + (size_t)D * 32 + (size_t)rr * N;   // + (t % D) * Rw * N

    double axd = 0.0, ayd = 0.0, wq = 0.0;
    if (act) {
        axd = fabs(a.xi[q]) / a.dx;
        ayd = fabs(a.eta[q]) / a.dy;
        wq = a.w[q];
    }
    const ModalOrdinate<P, TC> od = modal_ordinate<P, TC, ADJ>(axd, ayd);

    // the row's x trace entering its first column (ghost-column inflow; zero for the transposed sweep)
    TC f[P];
#pragma unroll
    for (int m = 0; m < P; ++m) f[m] = TC(0);
    if (act && a.inflow && !ADJ) {
        const double *in = a.inflow + ((size_t)(nx + row) * a.nq + q) * P;
#pragma unroll
        for (int m = 0; m < P; ++m) f[m] = TC(in[m]);
    }

    // row 0 reads its y traces from the item above (sentinel-armed) or the ghost row's inflow
    const bool reader = rr == 0 && o < item.q_count && row_valid;
    double *dep_trace = has_dep ? a.trace + (size_t)item.dep * a.trace_stride + (size_t)o * P : nullptr;
    const double *inflow_y = (!has_dep && a.inflow && !ADJ) ? a.inflow + (size_t)q * P : nullptr;
    double *out_trace = a.trace + (size_t)it_index * a.trace_stride + (size_t)o * P;
    const bool writer = has_consumer && rr == Rw - 1 && o < item.q_count;
    auto load_trace = [&](int c, double (&v)[P]) {
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = 0.0;
        if (reader && c < nx) {
            if (has_dep) {
#pragma unroll
                for (int m = 0; m < P; ++m) v[m] = ld_relaxed_f64(dep_trace + (size_t)c * tcol + m);
            } else if (inflow_y) {
#pragma unroll
                for (int m = 0; m < P; ++m) v[m] = inflow_y[(size_t)c * a.nq * P + m];
            }
        }
    };

    // step t's inputs into stage t % D, one cp.async group per step (empty past the last step)
    auto prefetch = [&](int t) {
        const int c = t - rr;
        if (t < T && row_valid && c >= 0 && c < nx) {
            const int ci = xi0 + xis * c;
            const size_t base = (size_t)ci * istride + (size_t)j * plane + (size_t)q * N;
            const size_t cidx = (size_t)ci * (a.ny + 2) + j;
            if (PHI && act) {   // the cell's packed modal source of this quadrant (the same for the row segment)
                double *d = stage + (size_t)(t % D) * 32 * N;
                const double *g = a.modal_src + (cidx * 4 + item.quadrant) * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, g + k);
            }
            if (!PHI && act && a.src) {
                double *d = stage + (size_t)(t % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, a.src + base + k);
            }
            if (SRC2 && act) {
                double *d = stage2 + (size_t)(t % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, a.src2 + base + k);
            }
            cp_async8(sig + (size_t)(t % D) * 32, a.sigma_t + cidx);
            if (!PHI && o == 0 && a.phi_scatter) {
                double *d = mom + (size_t)(t % D) * Rw * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, a.phi_scatter + cidx * N + k);
            }
        }
        cp_commit();
    };

    // step t's modal source and reciprocals from its landed stage (the caller has waited for its group)
    auto prepare = [&](int t, TC (&S)[N], ModalRecip<P, TC> &r) {
        const double *sp = stage + (size_t)(t % D) * 32 * N;
        if constexpr (PHI) {
#pragma unroll
            for (int k = 0; k < N; ++k) S[k] = TC(sp[k]);
            r = modal_recip<P, TC>(od, TC(sig[(size_t)(t % D) * 32] + a.inv_dt));
            return;
        }
        double src[N];
#pragma unroll
        for (int k = 0; k < N; ++k) src[k] = a.src ? sp[k] : 0.0;
        if constexpr (SRC2) {
            const double *sp2 = stage2 + (size_t)(t % D) * 32 * N;
#pragma unroll
            for (int k = 0; k < N; ++k) src[k] = fma(a.src2_scale, sp2[k], src[k]);
        }
        if (!PHI && a.phi_scatter) {   // lane o == 0's copy of the cell's moments, handed to its row segment
            const double *mp = mom + (size_t)(t % D) * Rw * N;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const double mk = __shfl_sync(kFullMask, o == 0 ? mp[k] : 0.0, rr * SEG);
                if constexpr (!ADJ)   // fused TransportOperator::Smv(scale, 1, sigma_s, phi -> src)
                    src[k] = fma(a.scatter_scale, mk, src[k]);
                else                  // the transpose of Pmv: w_q * mu
                    src[k] = fma(wq, mk, src[k]);
            }
        }
        r = modal_recip<P, TC>(od, TC(sig[(size_t)(t % D) * 32] + a.inv_dt));
        TC sv[N];
#pragma unroll
        for (int k = 0; k < N; ++k) sv[k] = flip_by(TC(src[k]), fmask(k));
        modal_forward<P, false, false, TC, ADJ>(S, sv);
    };

    const int phi_slot = a.phi_slots > 0 ? it_index % a.phi_slots : 0;
    long long polls = 0;

    // prologue: stages 0 .. D-2 in flight, step 0 prepared, row 0's trace of column 0 loaded
#pragma unroll
    for (int t = 0; t < D - 1; ++t) prefetch(t);
    cp_wait<D - 2>();
    TC S[N];
    ModalRecip<P, TC> r;
    prepare(0, S, r);
    double tnext[P];
    load_trace(0, tnext);
    TC gprev[P], Zp[N];
#pragma unroll
    for (int m = 0; m < P; ++m) gprev[m] = TC(0);
#pragma unroll
    for (int k = 0; k < N; ++k) Zp[k] = TC(0);

    // iteration s: chain of step s (s < T), finish of step s - 1 (s >= 1), inputs of step s + 1
    for (int s = 0; s <= T; ++s) {
        const int c = s - rr;
        const bool valid = act && c >= 0 && c < nx;

        // ---- the y trace in: from the row below (previous step); row 0 from the item above ----
        TC g[P];
#pragma unroll
        for (int m = 0; m < P; ++m) g[m] = __shfl_up_sync(kFullMask, gprev[m], SEG);
        if (s < nx) {   // row 0 consumes column s (loaded an iteration ago)
            if (has_dep) {
                bool bad = false;
#pragma unroll
                for (int m = 0; m < P; ++m) bad |= reader && is_sentinel(tnext[m]);
                if (__any_sync(kFullMask, bad)) {   // caught up with the producer: wait for two columns of slack
                    if (!wait_for_producer<P>(dep_trace, s, min(s + 2, nx - 1), reader, a.G, a.error, a.spin_limit,
                                              &polls, lane))
                        break;
                    load_trace(s, tnext);
                }
                if (reader) {   // re-arm the consumed column for the next sweep
#pragma unroll
                    for (int m = 0; m < P; ++m) st_relaxed_f64(dep_trace + (size_t)s * tcol + m, sentinel_value());
                }
            }
            if (rr == 0) {
#pragma unroll
                for (int m = 0; m < P; ++m) g[m] = TC(tnext[m]);
            }
        }
        load_trace(s + 1, tnext);

        // ---- the chain of step s ----
        TC Z[N], fn[P], gout[P];
#pragma unroll
        for (int m = 0; m < P; ++m) fn[m] = f[m];
        modal_step<P, TC, ADJ>(Z, S, fn, g, gout, od, r);
#pragma unroll
        for (int m = 0; m < P; ++m) {
            f[m] = valid ? fn[m] : f[m];
            gprev[m] = valid ? gout[m] : TC(0);
        }
        const int cout = s - (Rw - 1);   // traces out: relaxed stores, each value its own flag
        if (writer && cout >= 0 && cout < nx) {
#pragma unroll
            for (int m = 0; m < P; ++m) st_relaxed_f64(out_trace + (size_t)cout * tcol + m, double(gout[m]));
        }

        // ---- the finish of step s - 1: cell dofs, psi, moments (PHI: the packed modal moments) ----
        {   // (at s = 0 nothing is valid: Zp is zero and no store is made)
            const int cp = c - 1;
            const bool vp = act && cp >= 0 && cp < nx;
            TC x[N];
            if constexpr (PHI) {
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = Zp[k];
            } else {
                modal_backward<P, false, false, TC, ADJ>(x, Zp);
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = flip_by(x[k], fmask(k));
            }
            if (!PHI && a.out && vp) {
                double *op = a.out + (size_t)(xi0 + xis * cp) * istride + (size_t)j * plane + (size_t)q * N;
#pragma unroll
                for (int k = 0; k < N; ++k) op[k] = double(x[k]);
            }
            if (a.phi_part) {
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = vp ? (ADJ ? x[k] : TC(wq) * x[k]) : TC(0);
                int lo = 0, hi = N;
                segment_sums<N, SEG>(x, o, &lo, &hi);
                if (row_valid && cp >= 0 && cp < nx) {
                    double *pp = a.phi_part + (size_t)phi_slot * a.phi_slot_stride +
                                 ((size_t)(xi0 + xis * cp) * (a.ny + 2) + j) * N;
#pragma unroll
                    for (int i = 0; i < (N + SEG - 1) / SEG; ++i)
                        if (lo + i < hi) pp[lo + i] = double(x[i]);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < N; ++k) Zp[k] = Z[k];

        // ---- the inputs of step s + 1 ----
        prefetch(s + D - 1);   // into the stage of step s - 1 (read an iteration ago)
        cp_wait<D - 2>();      // step s + 1's group has landed
        prepare(s + 1, S, r);
    }
    cp_wait<0>();
}

template <int P, int SEG, bool ADJ, bool SRC2, bool PHI, typename TC>
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
        run_item<P, SEG, ADJ, SRC2, PHI, TC>(a, a.items[it], it, wsm, lane);
    }
}

template <int P, int SEG, bool ADJ, bool SRC2, bool PHI = false, typename TC = double>
cudaError_t launch(const SweepArgs &args, int grid, cudaStream_t stream) {
    auto kern = sweep_lane_kernel<P, SEG, ADJ, SRC2, PHI, TC>;
    const size_t smem = block_smem_bytes(P, SEG, SRC2);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kWarps * 32, smem, stream>>>(args);
    return cudaGetLastError();
}

template <int P, int SEG, bool ADJ, bool SRC2>
cudaError_t occupancy(int *blocks_per_sm) {
    auto kern = sweep_lane_kernel<P, SEG, ADJ, SRC2, false, double>;
    const size_t smem = block_smem_bytes(P, SEG, SRC2);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, kWarps * 32, smem);
}

}  // namespace lane
}  // namespace idc
