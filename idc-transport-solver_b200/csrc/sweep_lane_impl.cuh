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
// lane, the work of three cells:
//   * the chain of step s: the y trace in, the modal cell step, the traces out (the only dependency from
//     cell to cell, so the only part whose latency sits on the wavefront's critical path);
//   * the finish of step s - 1: the backward transform; psi through a per-warp shared buffer whose rows are
//     the reference's contiguous row segments, one bulk copy (cp.async.bulk) per row segment; the row
//     segment's moment sums (a shuffle butterfly for 4- and 8-wide segments, sums over a k-major shared
//     buffer for 16-wide ones), one partial per ordinate chunk, each a fixed tree, added in a fixed order by
//     reduce_phi_partials: bitwise reproducible;
//   * the inputs of step s + 1: the forward modal transform and the reciprocal denominators of its source
//     dofs and sigma_t (and second source, and fused scattering moments), which were copied into shared
//     memory by cp.async kStages - 2 iterations earlier.
// After the y trace's arrival (and, rarely, a wait for the producer) the chain, the finish and the transform
// are one basic block with the chain first: every global access in it is predicated instead of branched
// around, so the scheduler interleaves the three cells' instructions.  The loads and copies for later steps
// and the work behind uniform branches (scattering moments, psi rows that are not 16-byte aligned) follow in
// a tail section.  Measured on B200 at 256x256 Q2 S16 (FP64): the branchy form of the same work ran its
// phases one after another (the per-phase times summed to the iteration time) and scattered 8-byte psi
// stores, 32 sectors per instruction, were a third of the kernel's time.  The loop body is one iteration for
// every quadrant (the quadrant's sign flips are applied to the cell values at run time as sign-bit flips,
// exact), so the hot loop stays small for the instruction caches.  Four warps per thread block, one per SM
// sub-partition.
//
// Between row blocks: the warp's last row writes its outgoing y traces, column by column, into the item's
// trace buffer with relaxed 8-byte stores; row 0 of the item below loads column s + 1 with relaxed loads at
// iteration s.  A value still holding the NaN-payload sentinel means the consumer has caught up with its
// producer: it then polls (bounded) until the producer has written that column, and no further, which
// keeps the lag between row blocks at its minimum.  The consumer writes the sentinel back after use.  The
// first row block reads the ghost row's inflow traces (inflow_traces_kernel) the same way.  Items are
// dequeued per warp in row-block order from an atomic counter, so an item's producer is always held by a
// running warp: no deadlock, and no thread block needs any other to be resident.  Every wait is bounded
// (spin_limit); on expiry the warp records kDevTimeout in the device error word and leaves, and every other
// warp leaves when it sees the word.
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
constexpr int kStages = 6;   // stages in shared memory: a step's inputs are copied this many steps minus one ahead
constexpr int kOutBufs = 2;  // psi leaves through a ring of this many per-warp buffers
constexpr int kMomStride = 34;   // doubles per moment index k in the moment buffer (32 lanes + 2: conflict-free sums)
// Polls per round of the producer wait below, by DG degree + 1, chosen by measurement on B200 (interleaved
// A/B).  At DG degree 1 the three-poll form is 6-8% faster (512x512 Q1 S12 1.015-1.039 -> 0.950 ms; two: no
// gain).  ptxas places its poll array in local memory (a 48-byte stack frame), so its loads do not stay in
// flight together as the loop is written; variants with the polls in registers (overlapping), with one poll
// and a 256 ns sleep, or waiting for 2 or 4 columns of slack all lose the gain (1.02-1.18 ms), so where the
// gain comes from is not established.  At DG degree 2 three polls cost 2-3% (0.695 -> 0.714 ms): one.
template <int P>
constexpr int kPollDepth = P >= 3 ? 1 : 3;

// Doubles per (column, ordinate) slot of the trace buffer.
__host__ __device__ constexpr int trace_slot(int P) { return P; }

// Shared memory of one warp, in doubles: source stages [kStages][32][N] (lane-major, conflict-free), the
// second source's stages (launches with one), sigma_t stages [kStages][32] (each lane its own copy), the
// fused scattering moments' stages [kStages][Rw][N] (copied by lane o == 0 of each row) and the psi out
// buffers [kOutBufs][32][N] (lane-major: row rr's SEG ordinates are the reference's contiguous row segment)
// and, for 16-wide segments, the weighted moment values [N][kMomStride] (k-major: a row segment's SEG values
// of one k are adjacent).
// Every part is an even number of doubles, so each starts on a 16-byte boundary.
__host__ __device__ constexpr size_t warp_doubles(int P, int seg, bool src2) {
    return (size_t)kStages * 32 * P * P * (src2 ? 2 : 1) + (size_t)kStages * 32 + (size_t)kStages * (32 / seg) * P * P +
           (size_t)kOutBufs * 32 * P * P + (seg >= 16 ? (size_t)P * P * kMomStride : 0);
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

// Global accesses under a predicate instead of a branch, so that the loop body stays one basic block and
// the scheduler can interleave the three cells' work.  An access whose predicate is false is not made.
__device__ __forceinline__ void st_f64_if(double *p, double v, bool pred) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.global.f64 [%0], %1;\n\t}" ::"l"(p), "d"(v),
                 "r"((int)pred));
}
__device__ __forceinline__ void st_relaxed_f64_if(double *p, double v, bool pred) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q st.relaxed.gpu.global.f64 [%0], %1;\n\t}" ::"l"(p),
                 "d"(v), "r"((int)pred));
}
// 0.0 where the predicate is false
__device__ __forceinline__ double ld_relaxed_f64_if(const double *p, bool pred) {
    double v;
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\tmov.f64 %0, 0d0000000000000000;\n\t"
                 "@q ld.relaxed.gpu.global.f64 %0, [%1];\n\t}"
                 : "=d"(v)
                 : "l"(p), "r"((int)pred));
    return v;
}
// 8-byte cp.async that writes zeros into dst where the predicate is false (source size 0: nothing is read;
// callers still pass a source inside a valid allocation)
__device__ __forceinline__ void cp_async8_zfill(void *dst, const void *src, bool pred) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(saddr(dst)), "l"(src), "r"(pred ? 8 : 0));
}
// 16-byte cp.async (through L2) with the same zero fill; dst and src 16-byte aligned
__device__ __forceinline__ void cp_async16_zfill(void *dst, const void *src, bool pred) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(saddr(dst)), "l"(src), "r"(pred ? 16 : 0));
}
// n doubles (n even: 16-byte copies when `wide`, both addresses then 16-byte aligned; else 8-byte copies)
template <int n>
__device__ __forceinline__ void cp_async_doubles(double *dst, const double *src, bool pred, bool wide) {
    if constexpr (n % 2 == 0) {
        if (wide) {
#pragma unroll
            for (int h = 0; h < n / 2; ++h) cp_async16_zfill(dst + 2 * h, src + 2 * h, pred);
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < n; ++k) cp_async8_zfill(dst + k, src + k, pred);
}
__device__ __forceinline__ void cp_async8_if(void *dst, const void *src, bool pred) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %2, 0;\n\t@q cp.async.ca.shared.global [%0], [%1], 8;\n\t}" ::"r"(
                     saddr(dst)),
                 "l"(src), "r"((int)pred));
}

// Bulk copies shared -> global (the copy engine reads the buffer after the issuing thread moves on): one
// per row segment of psi.  The writes into the buffer are made visible to the copy engine by the proxy fence.
__device__ __forceinline__ void bulk_store_if(double *dst, const double *src, unsigned bytes, bool pred) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %3, 0;\n\t@q cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n\t}" ::"l"(dst),
                 "r"(saddr(src)), "r"(bytes), "r"((int)pred)
                 : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
template <int n>
__device__ __forceinline__ void bulk_wait_read() {
    asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(n) : "memory");
}
template <int n>
__device__ __forceinline__ void bulk_wait() {
    asm volatile("cp.async.bulk.wait_group %0;" ::"n"(n) : "memory");
}
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// The consumer caught up with its producer (a value of column s still held the sentinel): wait, bounded,
// until the producer has written column s.  Waiting for no more than that keeps the lag between row blocks
// at its minimum (measured on B200: waiting for two more columns of slack, to wait less often, made the
// 256x256 Q2 S16 sweep 10-20% slower).  The poll that finds the column complete has read its values, which
// are returned with the poll count, so the consumer does not load them again (one L2 round trip less on the
// row-block handoff); polls = -1 if the wait gave up or another warp has failed (the error word is then
// set).  Out of line: the hot loop stays small; every argument is a register.
template <int P>
struct ProducerWait {
    long long polls;
    double v[P];   // column s as the last poll read it; 0.0 in lanes that do not read (as load_trace gives)
};
template <int P>
__device__ __noinline__ ProducerWait<P> wait_for_producer(const double *dep_trace, int s, bool reader, int G,
                                                          int *error, long long spin_limit, long long polls,
                                                          int lane) {
    const double *col = dep_trace + (size_t)s * G * P;
    ProducerWait<P> r;
    // kPollDepth<P> polls per round: each checked poll is reissued at once
    double v[kPollDepth<P>][P];
#pragma unroll
    for (int d = 0; d < kPollDepth<P>; ++d)
#pragma unroll
        for (int m = 0; m < P; ++m) v[d][m] = ld_relaxed_f64_if(col + m, reader);
    for (;;) {
#pragma unroll
        for (int d = 0; d < kPollDepth<P>; ++d) {
            bool still = false;
#pragma unroll
            for (int m = 0; m < P; ++m) still |= reader && is_sentinel(v[d][m]);
            r.polls = polls;
            if (!__any_sync(kFullMask, still)) {
#pragma unroll
                for (int m = 0; m < P; ++m) r.v[m] = v[d][m];
                return r;
            }
            ++polls;
            if ((polls & 63) == 63 && ld_relaxed(error) != kDevOk) {
                r.polls = -1;
                return r;
            }
            if (polls > spin_limit) {
                if (lane == 0) atomicCAS(error, kDevOk, kDevTimeout);
                r.polls = -1;
                return r;
            }
#pragma unroll
            for (int m = 0; m < P; ++m) v[d][m] = ld_relaxed_f64_if(col + m, reader);
        }
    }
}

// The backward transform of one cell, x = Vb Z Vb^T, and the forward transform of another, S = Wb v Wb^T
// (modal_backward and modal_forward of modal_cell.cuh with no flips: the same operations in the same order,
// so the results are bitwise theirs), emitted statement by statement side by side: the two independent FMA
// chains are adjacent in the instruction stream, and each FMA of one can issue while the other's previous
// result is still in the pipe.
template <int P, typename T, bool ADJ>
__device__ __forceinline__ void modal_backward_forward(T (&x)[P * P], const T (&Z)[P * P], T (&S)[P * P],
                                                       const T (&v)[P * P]) {
    T tb[P * P], tf[P * P];
#pragma unroll
    for (int i = 0; i < P; ++i)
#pragma unroll
        for (int k = 0; k < P; ++k) {
            // backward: tb(d = i, b = k) = sum_a Vb(d,a) Z(a,b); forward: tf(a = i, e = k) = sum_d Wb(a,d) v(d,e)
            T ab = Z[k] * T(basis_v<P, ADJ>(i, 0));
            T af = v[k] * T(basis_w<P, ADJ>(i, 0));
#pragma unroll
            for (int m = 1; m < P; ++m) {
                ab = fma(T(basis_v<P, ADJ>(i, m)), Z[k + P * m], ab);
                af = fma(T(basis_w<P, ADJ>(i, m)), v[k + P * m], af);
            }
            tb[k + P * i] = ab;
            tf[k + P * i] = af;
        }
#pragma unroll
    for (int i = 0; i < P; ++i)
#pragma unroll
        for (int k = 0; k < P; ++k) {
            // backward: x(d = i, e = k) = sum_b Vb(e,b) tb(d,b); forward: S(a = i, b = k) = sum_e Wb(b,e) tf(a,e)
            T ab = tb[P * i] * T(basis_v<P, ADJ>(k, 0));
            T af = tf[P * i] * T(basis_w<P, ADJ>(k, 0));
#pragma unroll
            for (int m = 1; m < P; ++m) {
                ab = fma(T(basis_v<P, ADJ>(k, m)), tb[m + P * i], ab);
                af = fma(T(basis_w<P, ADJ>(k, m)), tf[m + P * i], af);
            }
            x[k + P * i] = ab;
            S[k + P * i] = af;
        }
}

template <int P, int SEG, bool ADJ, bool SRC2, bool PHI, typename TC>
__device__ __forceinline__ void run_item(const SweepArgs &a, const SweepItem &item, int it_index, double *wsm,
                                         int lane) {
    constexpr int N = P * P, Rw = 32 / SEG, D = kStages;
    if (a.quad_mask != 0 && ((a.quad_mask >> item.quadrant) & 1) == 0) return;   // another quadrant's launch
    // quadrant signs: flips of the cell values (exact), traversal directions (reversed for the transpose)
    const bool XN = item.quadrant >= 2, YN = (item.quadrant & 1) != 0;
    const bool TX = XN != ADJ, TY = YN != ADJ;
    const int quadrant = item.quadrant;
    const int rr = lane / SEG, o = lane - rr * SEG;
    const int row_w = item.row_block * Rw;
    const int row = row_w + rr;
    const bool row_valid = row < a.ny;
    const bool act = (o < item.q_count) && row_valid;
    const int q = item.q_begin + (act ? o : 0);
    const int j = row_valid ? (TY ? (a.ny - row) : (1 + row)) : 1;
    const int nx = a.nx;
    const size_t plane = (size_t)a.nq * N;
    const size_t istride = (size_t)(a.ny + 2) * plane;
    const size_t cstride = (size_t)(a.ny + 2);
    const bool has_dep = item.dep >= 0;
    const bool has_consumer = row_w + Rw < a.ny;
    const bool has_scatter = !PHI && a.phi_scatter != nullptr;
    const int T = nx + Rw - 1;
    const size_t tcol = (size_t)a.G * P;   // doubles per trace column
    const int xi0 = TX ? nx : 1, xis = TX ? -1 : 1;   // array x index of sweep column c: xi0 + xis * c
    const unsigned xm = XN ? 0x80000000u : 0u, ym = YN ? 0x80000000u : 0u;
    auto fmask = [&](int k) { return ((k / P) & 1 ? xm : 0u) ^ ((k % P) & 1 ? ym : 0u); };   // k = e + P d
    const double *valid_addr = a.sigma_t;   // a source address for accesses that are not made

    double *stage = wsm + (size_t)lane * N;                            // step t at + (t % D) * 32 * N
    double *stage2 = wsm + (size_t)D * 32 * N + (size_t)lane * N;      // (SRC2 launches only)
    double *sig = wsm + (size_t)D * 32 * N * (SRC2 ? 2 : 1) + lane;    // + (t % D) * 32
    double *mom = wsm + (size_t)D * 32 * N * (SRC2 ? 2 : 1) + (size_t)D * 32 + (size_t)rr * N;   // + (t % D) * Rw * N
    double *obuf = wsm + (size_t)D * 32 * N * (SRC2 ? 2 : 1) + (size_t)D * 32 + (size_t)D * Rw * N;   // + b * 32 * N
    double *mbuf = obuf + (size_t)kOutBufs * 32 * N;   // [N][kMomStride]
    // psi rows leave by bulk copies when every row segment starts and ends on a 16-byte boundary
    const bool bulk_out = a.out != nullptr && ((size_t)a.out & 15) == 0 && ((size_t)a.nq * N) % 2 == 0 &&
                          ((size_t)item.q_begin * N) % 2 == 0 && ((size_t)item.q_count * N) % 2 == 0;

    // an inactive lane runs the cell step of a unit ordinate (finite values) with moment weight zero, so that
    // the moment sums need no selects
    double axd = 1.0, ayd = 1.0, wq = 0.0;
    if (act) {
        axd = fabs(a.xi[q]) / a.dx;
        ayd = fabs(a.eta[q]) / a.dy;
        wq = a.w[q];
    }
    const ModalOrdinate<P, TC> od = modal_ordinate<P, TC, ADJ>(axd, ayd);
    const TC wv = act ? (ADJ ? TC(1) : TC(wq)) : TC(0);   // moment weight (the transpose sums unweighted)

    // the row's x trace entering its first column (ghost-column inflow; zero for the transposed sweep)
    TC f[P];
#pragma unroll
    for (int m = 0; m < P; ++m) f[m] = TC(0);
    if (act && a.inflow && !ADJ) {
        const double *in = a.inflow + ((size_t)(nx + row) * a.nq + q) * P;
#pragma unroll
        for (int m = 0; m < P; ++m) f[m] = TC(in[m]);
    }

    // row 0 reads its y traces from the item above (sentinel-armed) or the ghost row's inflow, the same way
    const bool reader = rr == 0 && o < item.q_count && row_valid;
    double *dep_trace = has_dep ? a.trace + (size_t)item.dep * a.trace_stride + (size_t)o * P : nullptr;
    const double *tin = has_dep ? dep_trace : ((a.inflow && !ADJ) ? a.inflow + (size_t)q * P : nullptr);
    const size_t tin_col = has_dep ? tcol : (size_t)a.nq * P;
    const bool tin_ok = reader && tin != nullptr;
    double *out_trace = a.trace + (size_t)it_index * a.trace_stride + (size_t)o * P;
    const bool writer = has_consumer && rr == Rw - 1 && o < item.q_count;
    auto load_trace = [&](int c, long long off, double (&v)[P]) {   // off = c * tin_col
        const bool p = tin_ok && c < nx;
        const double *ptr = p ? tin + off : valid_addr;
#pragma unroll
        for (int m = 0; m < P; ++m) v[m] = ld_relaxed_f64_if(ptr + m, p);
    };

    // Column addresses advance by a fixed stride per step: the prefetch of step t reads column t - rr, whose
    // cell index (xi0 + xis (t - rr)) cstride + j and psi offset are kept running (prefetches come in step order).
    const long long dcol = (long long)xis * (long long)cstride;   // cells between consecutive columns
    const long long dsoff = dcol * (long long)plane;              // psi doubles between them
    long long pf_cidx = ((long long)xi0 - (long long)xis * rr) * (long long)cstride + j;   // step 0's column
    long long pf_soff = pf_cidx * (long long)plane + (long long)q * N;

    // step t's inputs into stage slot = t % D, one cp.async group per step; a cell outside the row gets zeros.
    // With an even number of dofs per cell (DG degree 1) every (cell, ordinate) block starts on a 16-byte
    // boundary of an aligned array, and the copies are 16 bytes wide (half the copy instructions; measured on
    // B200 at DG degree 1: see the lane kernel's notes); the stage slots are 16-byte aligned by layout.
    const bool wide_ok = N % 2 == 0 && ((size_t)valid_addr & 15) == 0;
    const bool src16 = wide_ok && ((size_t)a.src & 15) == 0;
    const bool src2_16 = wide_ok && (!SRC2 || ((size_t)a.src2 & 15) == 0);
    const bool modal16 = wide_ok && (!PHI || ((size_t)a.modal_src & 15) == 0);
    auto prefetch = [&](int t, int slot) {
        const int c = t - rr;
        const bool in = row_valid && c >= 0 && c < nx;
        const size_t cidx = in ? (size_t)pf_cidx : 0;
        double *d = stage + (size_t)slot * 32 * N;
        if constexpr (PHI) {   // the cell's packed modal source of this quadrant (the same for the row segment)
            const double *g = a.modal_src + (cidx * 4 + quadrant) * N;
            cp_async_doubles<N>(d, g, in && act, modal16);
        } else {
            const bool ps = in && act && a.src != nullptr;
            const double *g = ps ? a.src + pf_soff : valid_addr;
            cp_async_doubles<N>(d, g, ps, src16);
        }
        if constexpr (SRC2) {
            double *d2 = stage2 + (size_t)slot * 32 * N;
            const double *g2 = (in && act) ? a.src2 + pf_soff : valid_addr;
            cp_async_doubles<N>(d2, g2, in && act, src2_16);
        }
        cp_async8_zfill(sig + (size_t)slot * 32, a.sigma_t + cidx, in);
        if (has_scatter) {   // lane o == 0 of a row copies the cell's fused scattering moments (one copy per row)
            const bool pm = in && o == 0;
            const double *gm = pm ? a.phi_scatter + cidx * N : valid_addr;
            double *dm = mom + (size_t)slot * Rw * N;
#pragma unroll
            for (int k = 0; k < N; ++k) cp_async8_if(dm + k, gm + k, pm);
        }
        cp_commit();
        pf_cidx += dcol;
        pf_soff += dsoff;
    };

    // step t's raw inputs from its landed stage: the source (with the second source and the fused scattering
    // source) and sigma_t + 1/dt
    auto load_inputs = [&](int slot, double (&src)[N], double &st) {   // slot = t % D of step t
        const double *sp = stage + (size_t)slot * 32 * N;
#pragma unroll
        for (int k = 0; k < N; ++k) src[k] = sp[k];
        if constexpr (SRC2) {
            const double *sp2 = stage2 + (size_t)slot * 32 * N;
#pragma unroll
            for (int k = 0; k < N; ++k) src[k] = fma(a.src2_scale, sp2[k], src[k]);
        }
        st = sig[(size_t)slot * 32] + a.inv_dt;
        if (has_scatter) {   // lane o == 0's copy of the cell's moments, handed to its row segment
            const double *mp = mom + (size_t)slot * Rw * N;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const double mk = __shfl_sync(kFullMask, o == 0 ? mp[k] : 0.0, rr * SEG);
                if constexpr (!ADJ)   // fused TransportOperator::Smv(scale, 1, sigma_s, phi -> src)
                    src[k] = fma(a.scatter_scale, mk, src[k]);
                else                  // the transpose of Pmv: w_q * mu
                    src[k] = fma(wq, mk, src[k]);
            }
        }
    };
    // the modal source and the reciprocal denominators of the raw inputs (the prologue's step; in the loop the
    // forward transform runs beside the previous step's backward transform)
    auto transform = [&](const double (&src)[N], double st, TC (&S)[N], ModalRecip<P, TC> &r) {
        r = modal_recip<P, TC>(od, TC(st));
        if constexpr (PHI) {
#pragma unroll
            for (int k = 0; k < N; ++k) S[k] = TC(src[k]);
        } else {
            TC sv[N];
#pragma unroll
            for (int k = 0; k < N; ++k) sv[k] = flip_by(TC(src[k]), fmask(k));
            modal_forward<P, false, false, TC, ADJ>(S, sv);
        }
    };

    // psi of step t from its out buffer (filled at iteration t + 1) with per-lane stores (row segments that are
    // not 16-byte aligned)
    auto store_psi_lanes = [&](int t) {
        const int ct = t - rr;
        const bool ps = act && ct >= 0 && ct < nx;
        const double *ob = obuf + (size_t)((t + 1) & (kOutBufs - 1)) * 32 * N + (size_t)lane * N;
        double *op = ps ? a.out + ((size_t)(xi0 + xis * ct) * cstride + j) * plane + (size_t)q * N : out_trace;
#pragma unroll
        for (int k = 0; k < N; ++k) st_f64_if(op + k, ob[k], ps);
    };
    const bool lane_out = !PHI && a.out != nullptr && !bulk_out;

    const int phi_slot = a.phi_slots > 0 ? it_index % a.phi_slots : 0;
    double *phi_base = a.phi_part ? a.phi_part + (size_t)phi_slot * a.phi_slot_stride : nullptr;
    long long polls = 0;

    // prologue: stages 0 .. D-1 in flight, step 0 prepared, step 1's raw inputs loaded, row 0's trace of
    // column 0 loaded
#pragma unroll
    for (int t = 0; t < D - 1; ++t) prefetch(t, t);
    cp_wait<D - 2>();
    TC S[N];
    ModalRecip<P, TC> r;
    {
        double src0[N], st0;
        load_inputs(0, src0, st0);   // slot 0
        transform(src0, st0, S, r);
    }
    double srcn[N], stn;
    cp_wait<D - 3>();
    load_inputs(1, srcn, stn);   // slot 1
    prefetch(D - 1, D - 1);
    double tnext[P];
    load_trace(0, 0, tnext);
    // per-step running values of the loop: the stage slots of steps s + D (= s % D) and s + 2, the trace column
    // offsets s * tcol and (s + 1) * tin_col, and the finish column (s - rr - 1)'s cell index and psi offset
    int sl = 0, sl2 = 2 % D;
    long long s_tcol = 0, lt_off = (long long)tin_col;
    const long long out_lag = (long long)(Rw - 1) * (long long)tcol;
    long long fin_cidx = ((long long)xi0 - (long long)xis * (rr + 1)) * (long long)cstride + j;
    long long fin_ooff = fin_cidx * (long long)plane + (long long)item.q_begin * N;
    TC gprev[P], Zp[N];
#pragma unroll
    for (int m = 0; m < P; ++m) gprev[m] = TC(0);
#pragma unroll
    for (int k = 0; k < N; ++k) Zp[k] = TC(0);

    // Iteration s: the y trace in (and the wait for a producer, rarely taken); then one basic block with the
    // chain of step s (s < T) first, as it is the wavefront's critical path, the finish of step s - 1 and the
    // transform of step s + 1's inputs; then the loads and copies for later steps.
    for (int s = 0; s <= T; ++s) {
        const int c = s - rr;
        const bool valid = act && c >= 0 && c < nx;

        // ---- the y trace in: from the row below (previous step); row 0 from the item above ----
        TC g[P];
#pragma unroll
        for (int m = 0; m < P; ++m) g[m] = __shfl_up_sync(kFullMask, gprev[m], SEG);
        if (has_dep) {
            bool bad = false;
#pragma unroll
            for (int m = 0; m < P; ++m) bad |= reader && s < nx && is_sentinel(tnext[m]);
            if (__any_sync(kFullMask, bad)) {   // caught up with the producer: wait for column s
                const ProducerWait<P> w =
                    wait_for_producer<P>(dep_trace, s, reader, a.G, a.error, a.spin_limit, polls, lane);
                polls = w.polls;
                if (polls < 0) break;
#pragma unroll
                for (int m = 0; m < P; ++m) tnext[m] = w.v[m];
            }
        }
        {   // re-arm the consumed column for the next sweep
            const bool p = has_dep && reader && s < nx;
            double *ptr = p ? dep_trace + s_tcol : out_trace;
#pragma unroll
            for (int m = 0; m < P; ++m) st_relaxed_f64_if(ptr + m, sentinel_value(), p);
        }
#pragma unroll
        for (int m = 0; m < P; ++m) g[m] = (rr == 0) ? TC(tnext[m]) : g[m];
        load_trace(s + 1, lt_off, tnext);

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
        {   // traces out: relaxed stores, each value its own flag
            const int cout = s - (Rw - 1);
            const bool p = writer && cout >= 0 && cout < nx;
            double *ptr = p ? out_trace + (s_tcol - out_lag) : out_trace;
#pragma unroll
            for (int m = 0; m < P; ++m) st_relaxed_f64_if(ptr + m, double(gout[m]), p);
        }

        // ---- the finish of step s - 1: cell dofs, psi, moments (PHI: the packed modal moments) ----
        {   // (at s = 0 nothing is valid: Zp is zero and no store is made)
            const int cp = c - 1;
            const bool inrow = row_valid && cp >= 0 && cp < nx;
            const size_t cidx = inrow ? (size_t)fin_cidx : 0;
            TC x[N];
            if constexpr (PHI) {
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = Zp[k];
#pragma unroll
                for (int k = 0; k < N; ++k) S[k] = TC(srcn[k]);
            } else {   // this step's backward transform beside step s + 1's forward transform
                TC sv[N];
#pragma unroll
                for (int k = 0; k < N; ++k) sv[k] = flip_by(TC(srcn[k]), fmask(k));
                modal_backward_forward<P, TC, ADJ>(x, Zp, S, sv);
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = flip_by(x[k], fmask(k));
            }
            r = modal_recip<P, TC>(od, TC(stn));
            double *ob = obuf + (size_t)(s & (kOutBufs - 1)) * 32 * N;
            if constexpr (!PHI) bulk_wait_read<kOutBufs - 1>();   // the copy that read this buffer is done
            __syncwarp();   // and every lane's reads of the buffers in the previous iterations
            if constexpr (!PHI) {
#pragma unroll
                for (int k = 0; k < N; ++k) ob[(size_t)lane * N + k] = double(x[k]);
            }
            if constexpr (SEG >= 16) {
#pragma unroll
                for (int k = 0; k < N; ++k) mbuf[k * kMomStride + lane] = double(wv * x[k]);
            }
            if constexpr (!PHI) fence_proxy_async_smem();
            __syncwarp();
            if constexpr (!PHI) {   // row rr's segment: one bulk copy by lane o == 0
                const bool pb = bulk_out && o == 0 && inrow;
                double *dst = pb ? a.out + fin_ooff : out_trace;
                bulk_store_if(dst, ob + (size_t)rr * SEG * N, (unsigned)(item.q_count * N * sizeof(double)), pb);
                bulk_commit();
            }
            // the moments of row rr: sums of the SEG weighted values in fixed trees, one partial per ordinate
            // chunk (added in a fixed order by the reduction kernel: bitwise reproducible).  16-wide segments
            // sum moment k = o from the shared buffer in a pairwise tree over ordinate order (the sequential
            // sum's 15 dependent adds cost 4% of the 256x256 Q2 S16 sweep on B200); narrower ones by a shuffle
            // butterfly (measured on B200: each is the faster one at its width).
            const bool pp = inrow && phi_base != nullptr;
            double *pt = pp ? phi_base + cidx * N : out_trace;
            if constexpr (SEG >= 16) {
                const int k = o < N ? o : N - 1;
                const double2 *mv = reinterpret_cast<const double2 *>(mbuf + k * kMomStride + rr * SEG);
                double part[SEG / 2];   // a pairwise tree in ordinate order: 4 dependent adds, not 15
#pragma unroll
                for (int h = 0; h < SEG / 2; ++h) {
                    const double2 v = mv[h];
                    part[h] = v.x + v.y;
                }
#pragma unroll
                for (int w = SEG / 4; w >= 1; w /= 2)
#pragma unroll
                    for (int h = 0; h < w; ++h) part[h] = part[2 * h] + part[2 * h + 1];
                st_f64_if(pt + k, part[0], pp && o < N);
            } else {
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = wv * x[k];
                int lo = 0, hi = N;
                segment_sums<N, SEG>(x, o, &lo, &hi);
#pragma unroll
                for (int i = 0; i < (N + SEG - 1) / SEG; ++i) st_f64_if(pt + lo + i, double(x[i]), pp && lo + i < hi);
            }
        }
#pragma unroll
        for (int k = 0; k < N; ++k) Zp[k] = Z[k];


        // ---- step s + 2's raw inputs (copied D - 2 iterations ago), the copies of step s + D ----
        if (lane_out) store_psi_lanes(s - 1);
        cp_wait<D - 3>();
        load_inputs(sl2, srcn, stn);   // step s + 2
        prefetch(s + D, sl);           // into the stage of step s (read two iterations ago)
        sl = sl + 1 == D ? 0 : sl + 1;
        sl2 = sl2 + 1 == D ? 0 : sl2 + 1;
        s_tcol += (long long)tcol;
        lt_off += (long long)tin_col;
        fin_cidx += dcol;
        fin_ooff += dsoff;
    }
    cp_wait<0>();
    bulk_wait<0>();
}

// BATCHED: the items of several problems in one launch (a batch's problems of one DG degree, FP64 forward
// sweeps); each item names its problem in `table` and carries its index within that problem (`local`: its trace
// row and moment slot, `dep` is local too).  A warp copies its item's entry into shared memory; a problem left
// out of the launch (`skip`) has its items return at once.
template <int P, int SEG, bool ADJ, bool SRC2, bool PHI, typename TC, bool BATCHED>
__global__ void __launch_bounds__(kWarps * 32, 1) sweep_lane_kernel(const SweepArgs a,
                                                                    const SweepArgs *__restrict__ table) {
    static_assert(sizeof(SweepArgs) % 8 == 0, "SweepArgs is copied in 8-byte words");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ __align__(16) SweepArgs s_args[BATCHED ? kWarps : 1];
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
        if constexpr (BATCHED) {
            const unsigned long long *sw = reinterpret_cast<const unsigned long long *>(table + item.problem);
            unsigned long long *dw = reinterpret_cast<unsigned long long *>(&s_args[warp]);
            for (int k = lane; k < (int)(sizeof(SweepArgs) / 8); k += 32) dw[k] = sw[k];
            __syncwarp();
            if (!s_args[warp].skip) run_item<P, SEG, ADJ, SRC2, PHI, TC>(s_args[warp], item, item.local, wsm, lane);
            __syncwarp();   // every lane is done with the entry before the next item's copy
        } else {
            run_item<P, SEG, ADJ, SRC2, PHI, TC>(a, item, it, wsm, lane);
        }
    }
}

template <int P, int SEG, bool ADJ, bool SRC2, bool PHI = false, typename TC = double>
cudaError_t launch(const SweepArgs &args, int grid, cudaStream_t stream) {
    auto kern = sweep_lane_kernel<P, SEG, ADJ, SRC2, PHI, TC, false>;
    const size_t smem = block_smem_bytes(P, SEG, SRC2);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kWarps * 32, smem, stream>>>(args, nullptr);
    return cudaGetLastError();
}

// A batch's FP64 forward sweep (items of several problems; `table` on the device, one entry per problem)
template <int P, int SEG>
cudaError_t launch_batched(const SweepArgs &args, const SweepArgs *table, int grid, cudaStream_t stream) {
    auto kern = sweep_lane_kernel<P, SEG, false, false, false, double, true>;
    const size_t smem = block_smem_bytes(P, SEG, false);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, kWarps * 32, smem, stream>>>(args, table);
    return cudaGetLastError();
}

template <int P, int SEG>
cudaError_t occupancy_batched(int *blocks_per_sm) {
    auto kern = sweep_lane_kernel<P, SEG, false, false, false, double, true>;
    const size_t smem = block_smem_bytes(P, SEG, false);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, kWarps * 32, smem);
}

template <int P, int SEG, bool ADJ, bool SRC2>
cudaError_t occupancy(int *blocks_per_sm) {
    auto kern = sweep_lane_kernel<P, SEG, ADJ, SRC2, false, double, false>;
    const size_t smem = block_smem_bytes(P, SEG, SRC2);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(blocks_per_sm, kern, kWarps * 32, smem);
}

}  // namespace lane
}  // namespace idc
