// Warp-pipelined persistent wavefront sweep for sm_100a.
//
// Same contract as sweep_kernel (sweep_kernels.cu) -- it replaces SweepPatternUniCartWavefront::Sweep
// (linear_solvers/Abstract/SweepPattern/SweepPatternUniCartWavefront.cpp:121-332) with the per-cell
// CalcB/CalcA/GE/StoreResult of SweepCellSolveBase::ConstructAndSolve -- but without CTA-wide
// barriers on the per-step path:
//
//   * a compute warp owns Rw = 32/seg consecutive rows; lane (rr, o) = (lane / seg, lane % seg) owns
//     ordinate q_begin + o on row rr.  Row rr runs one column behind row rr-1 (the anti-diagonal skew
//     inside the warp); its y-upwind trace is row rr-1's previous result, moved by one __shfl_up.
//   * the Wn compute warps of a CTA are stacked in y.  Warp w's last row hands its results to warp w+1
//     through a ring of kWarpRingSlots shared-memory slots guarded by full/empty mbarriers, so the warps
//     run as a software pipeline, each one Rw columns behind the one above, with no __syncthreads.
//   * between CTAs there is no flag and no fence: the CTA's last warp writes its last row, column by
//     column, into the item's trace buffer with relaxed stores, and the helper warp of the item below
//     polls those values themselves (a slot holds a NaN-payload sentinel that arithmetic never produces
//     until it is written; 8-byte accesses are single-copy atomic).  The helper copies ready columns
//     into ring 0 and re-arms the slots with the sentinel for the next sweep.  The first row block's
//     helper copies the ghost row (inflow values) instead.
//   * each lane prefetches its next cells' source and sigma_t with cp.async, prefetch_depth(P) cells
//     ahead, into a per-warp ring of shared-memory stages: nothing on the per-cell path waits on L2/HBM.
//   * the fused phi = sum_q w_q psi_q reduction sums a row segment's ordinates through shared memory and
//     stores one partial moment per (cell, dof, ordinate chunk); reduce_phi_partials (ops_kernels.cu)
//     adds the chunks in a fixed order, so phi is bitwise reproducible.
//
// Work items (row blocks of Wn*Rw rows x quadrant x ordinate chunk) are dequeued in row-block order
// from an atomic counter, so every item's producer is held by a CTA that is already running.  Every wait
// (mbarrier or trace poll) is bounded; on expiry the warp records kDevTimeout in the device error word,
// leaves its loop, and every other warp leaves as soon as it sees the word.  After an error the trace
// buffer may hold values instead of sentinels; the host re-arms it before the next sweep.
#include "cell_solve.cuh"
#include "idc_internal.hpp"

#include <cstdint>

namespace idc {

namespace {

constexpr int kS = kWarpRingSlots;
constexpr int kMaxWarps = 8;   // up to 7 compute warps + 1 helper (256 threads: P=3 FP64 fits in registers)
constexpr unsigned kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t saddr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(saddr(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ bool mbar_test(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(saddr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ int ld_acquire(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ double ld_relaxed_f64(const double *p) {
    double v;
    asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_f64(double *p, double v) {
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ bool is_sentinel(double v) {
    return (unsigned long long)__double_as_longlong(v) == kTraceSentinel;
}
__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(saddr(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int n>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(n) : "memory");
}

// Bounded, warp-uniform wait on an mbarrier phase.  Returns false if the wait gave up or another warp
// has recorded an error; in both cases the device error word is non-zero afterwards.
__device__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *error, long long limit) {
    for (long long n = 0;; ++n) {
        if (mbar_try(bar, parity)) return true;
        if ((n & 63) == 63 && ld_relaxed(error) != kDevOk) return false;
        if (n > limit) {
            atomicCAS(error, kDevOk, kDevTimeout);
            return false;
        }
    }
}

__device__ __forceinline__ int T_steps(int nx, int Rw) { return nx + Rw - 1; }

template <int N>
__device__ __forceinline__ double pick(const double (&v)[N], int k) {
    double r = 0.0;
#pragma unroll
    for (int t = 0; t < N; ++t) r = (t == k) ? v[t] : r;
    return r;
}

// Source prefetch depth (cells ahead per lane): enough to cover HBM latency under load with the
// per-step time of each DG degree, within the shared-memory budget.
__host__ __device__ constexpr int prefetch_depth(int P) { return P >= 4 ? 3 : P == 3 ? 4 : 8; }

struct Layout {
    uint64_t *full, *empty;   // [Wn+1][kS]
    double *ring;             // [Wn+1][kS][G][N]
    double *src;              // [Wn][D][32][N]: each lane's cell source dofs
    double *cellst;           // [Wn][D][32/seg][N+2]: per row: sigma_t, sigma_s, phi_scatter[N]
    double *w;                // [G]
    double *red;              // [Wn][32][N]: per-lane weighted values for the moment reduction
};

__device__ __forceinline__ Layout carve(unsigned char *raw, int wn, int G, int N, int D, int rw) {
    Layout L;
    L.full = reinterpret_cast<uint64_t *>(raw);
    L.empty = L.full + (wn + 1) * kS;
    L.ring = reinterpret_cast<double *>(L.empty + (wn + 1) * kS);
    L.src = L.ring + (size_t)(wn + 1) * kS * G * N;
    L.cellst = L.src + (size_t)wn * D * 32 * N;
    L.w = L.cellst + (size_t)wn * D * rw * (N + 2);
    L.red = L.w + ((G + 1) & ~1);
    return L;
}

template <int P, int MODE>
__device__ void compute_warp(const SweepArgs &a, const SweepItem &item, const Layout &L, int w, int lane,
                             bool has_consumer, int it_index) {
    constexpr int N = P * P;
    const int seg = a.seg, Rw = 32 / seg, G = a.G, rows_cta = a.wn * Rw;
    const int rr = lane / seg, o = lane - rr * seg;
    const int row0 = item.row_block * rows_cta;
    const int rrow = w * Rw + rr;
    const bool xneg = item.quadrant >= 2, yneg = (item.quadrant & 1) != 0;
    const bool row_valid = row0 + rrow < a.ny;
    const bool act = (o < item.q_count) && row_valid;
    const int q = item.q_begin + (act ? o : 0);
    const int j = yneg ? (a.ny - (row0 + rrow)) : (1 + row0 + rrow);
    const size_t plane = (size_t)a.nq * N;
    const size_t istride = (size_t)(a.ny + 2) * plane;
    const bool last_warp = w == a.wn - 1;

    double xi = 0.0, eta = 0.0, xc = 0.0, ec = 0.0, wq = 0.0;
    double xup[N], xprev[N];
#pragma unroll
    for (int k = 0; k < N; ++k) xup[k] = xprev[k] = 0.0;
    if (act) {
        xi = a.xi[q];
        eta = a.eta[q];
        xc = a.dy * xi;
        ec = a.dx * eta;
        wq = L.w[o];
        if (a.src) {   // inflow ghost column; a null source means zero source and vacuum inflow
            const int ig = xneg ? a.nx + 1 : 0;
            const double *g = a.src + (size_t)ig * istride + (size_t)j * plane + (size_t)q * N;
#pragma unroll
            for (int k = 0; k < N; ++k) xup[k] = g[k];
        }
    }
    constexpr int D = prefetch_depth(P);
    constexpr int NC = N + 2;
    double *my_red = L.red + ((size_t)w * 32 + lane) * N;
    const int phi_slot = a.phi_slots > 0 ? it_index % a.phi_slots : 0;
    double *my_src = L.src + ((size_t)w * D * 32 + lane) * N;    // stage b at + b*32*N
    double *my_cell = L.cellst + ((size_t)w * D * Rw + rr) * NC;  // stage b at + b*Rw*NC

    // One cp.async group per step (possibly empty), D - 1 steps in flight ahead of the current one.
    // Every lane copies its own source dofs; lane o == 0 of a row copies that cell's sigma_t (and
    // sigma_s, phi for the fused scattering source) for the whole row segment.
    auto prefetch = [&](int s) {
        const int c = s - rr;
        if (s < T_steps(a.nx, Rw) && row_valid && c >= 0 && c < a.nx) {
            const int i = xneg ? a.nx - c : 1 + c;
            if (act && a.src) {
                const double *g = a.src + (size_t)i * istride + (size_t)j * plane + (size_t)q * N;
                double *d = my_src + (size_t)(s % D) * 32 * N;
#pragma unroll
                for (int k = 0; k < N; ++k) cp_async8(d + k, g + k);
            }
            if (o == 0) {
                const size_t cidx = (size_t)i * (a.ny + 2) + j;
                double *d = my_cell + (size_t)(s % D) * Rw * NC;
                cp_async8(d, a.sigma_t + cidx);
                if (a.phi_scatter) {
                    cp_async8(d + 1, a.sigma_s + cidx);
#pragma unroll
                    for (int k = 0; k < N; ++k) cp_async8(d + 2 + k, a.phi_scatter + cidx * N + k);
                }
            }
        }
        cp_commit();
    };

    const int T = T_steps(a.nx, Rw);
#pragma unroll
    for (int s = 0; s < D - 1; ++s) prefetch(s);
    for (int s = 0; s < T; ++s) {
        prefetch(s + D - 1);
        cp_wait<D - 1>();
        __syncwarp();   // lane o == 0's cell-data copies are visible to its row segment
        const int c = s - rr;

        // y-upwind trace: rows rr > 0 from the lane Rw.. above (previous step), row 0 from the ring
        double yup[N];
#pragma unroll
        for (int k = 0; k < N; ++k) yup[k] = __shfl_up_sync(kFull, xprev[k], seg);
        if (s < a.nx) {   // warp-uniform: row 0 needs column s
            const int slot = s % kS;
            if (!mbar_wait(L.full + w * kS + slot, (uint32_t)((s / kS) & 1), a.error, a.spin_limit)) break;
            if (rr == 0 && o < G) {
                const double *rp = L.ring + (((size_t)w * kS + slot) * G + o) * N;
#pragma unroll
                for (int k = 0; k < N; ++k) yup[k] = rp[k];
            }
            __syncwarp();
            mbar_arrive(L.empty + w * kS + slot);
        }

        double x[N];
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = 0.0;
        const bool valid = act && c >= 0 && c < a.nx;
        if (valid) {
            const size_t cell = (size_t)(xneg ? a.nx - c : 1 + c) * istride + (size_t)j * plane + (size_t)q * N;
            const double *sp = my_src + (size_t)(s % D) * 32 * N;
            const double *cp = my_cell + (size_t)(s % D) * Rw * NC;
            double src[N], B[N];
#pragma unroll
            for (int k = 0; k < N; ++k) src[k] = a.src ? sp[k] : 0.0;
            if (a.phi_scatter) {   // fused TransportOperator::Smv(scale, 1, sigma_s, phi -> src)
                const double sv = cp[1];
#pragma unroll
                for (int k = 0; k < N; ++k) src[k] += a.scatter_scale * (sv * cp[2 + k] / (4.0 * M_PI));
            }
            build_cell_rhs<P>(B, src, xup, yup, a.dx, a.dy, xi, eta, xneg, yneg);
            if (MODE == 0 && a.sigma_t_mat) {
                // high-order cross sections: CalcA's tensor branch (SweepLinearSolveSpec.cpp:298-318), the
                // dx dy / dt diagonal and then the cell's N x N absorption term
                const int ic = xneg ? a.nx - c : 1 + c;
                const double *Mt = a.sigma_t_mat + ((size_t)ic * (a.ny + 2) + j) * N * N;
                double A[N][N];
                build_cell_matrix<P, double>(A, xc, ec, xneg, yneg, a.dx * a.dy * a.inv_dt);
#pragma unroll
                for (int r = 0; r < N; ++r)
#pragma unroll
                    for (int cc = 0; cc < N; ++cc) A[r][cc] += __ldg(Mt + r * N + cc);
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] = B[k];
                ge_solve<P, double>(A, x);
            } else {
                const double sdiag = (cp[0] + a.inv_dt) * a.dx * a.dy;
                cell_solve<P, MODE>(x, B, xc, ec, xneg, yneg, sdiag, a.n_refine);
            }
            if (a.out) {
                double *dst = a.out + cell;
#pragma unroll
                for (int k = 0; k < N; ++k) dst[k] = x[k];
            }
#pragma unroll
            for (int k = 0; k < N; ++k) xup[k] = x[k];
        }
#pragma unroll
        for (int k = 0; k < N; ++k) xprev[k] = x[k];

        // fused moments: the row segment's weighted values meet in shared memory; lane o sums dof
        // k = o, o + seg, ... over the segment's ordinates and stores it into this chunk's partial
        // moments (plain stores; the chunks are summed in a fixed order by reduce_phi_partials)
        if (a.phi_part) {
            __syncwarp();
#pragma unroll
            for (int k = 0; k < N; ++k) my_red[k] = valid ? wq * x[k] : 0.0;
            __syncwarp();
            const bool row_ok = (row0 + rrow < a.ny) && c >= 0 && c < a.nx;
            if (row_ok) {
                const int i = xneg ? a.nx - c : 1 + c;
                double *ph = a.phi_part + ((size_t)phi_slot * a.phi_slot_stride) + ((size_t)i * (a.ny + 2) + j) * N;
                const double *seg_red = L.red + ((size_t)w * 32 + rr * seg) * N;
                for (int k = o; k < N; k += seg) {
                    double sum = 0.0;
                    for (int oo = 0; oo < item.q_count; ++oo) sum += seg_red[(size_t)oo * N + k];
                    ph[k] = sum;
                }
            }
        }

        // last row (column s - (Rw-1)): to ring w+1, or, from the CTA's last warp, to the item's trace
        // buffer that the item below polls (plain relaxed stores, no fence: each value is its own flag)
        const int cout = s - (Rw - 1);
        if (last_warp) {
            if (has_consumer && rr == Rw - 1 && o < item.q_count && cout >= 0 && cout < a.nx) {
                double *tp = a.trace + (size_t)it_index * a.trace_stride + ((size_t)cout * G + o) * N;
#pragma unroll
                for (int k = 0; k < N; ++k) st_relaxed_f64(tp + k, x[k]);
            }
        } else if (cout >= 0 && cout < a.nx) {   // warp-uniform
            const int slot = cout % kS;
            uint64_t *emp = L.empty + (w + 1) * kS + slot;
            if (!mbar_wait(emp, (uint32_t)(((cout / kS) & 1) ^ 1), a.error, a.spin_limit)) break;
            if (rr == Rw - 1 && o < G) {
                double *rp = L.ring + (((size_t)(w + 1) * kS + slot) * G + o) * N;
#pragma unroll
                for (int k = 0; k < N; ++k) rp[k] = x[k];
            }
            __syncwarp();
            mbar_arrive(L.full + (w + 1) * kS + slot);
        }
    }
    cp_wait<0>();
}

// Helper warp: feeds ring 0 with the y-upwind row of the item's first row -- the ghost row (inflow
// values) for the first row block, otherwise the trace the item above writes column by column.  A trace
// slot holds kTraceSentinel until its value is written, so a column is ready when none of its values
// is the sentinel; the helper copies ready columns into the ring and writes the sentinel back for the
// next sweep.  Up to kS columns are loaded per pass, all loads issued before any value is used.
__device__ void helper_warp(const SweepArgs &a, const SweepItem &item, const Layout &L, int lane, int N) {
    const int seg = a.seg, Rw = 32 / seg, G = a.G, rows_cta = a.wn * Rw;
    const bool xneg = item.quadrant >= 2, yneg = (item.quadrant & 1) != 0;
    const int row0 = item.row_block * rows_cta;
    const size_t plane = (size_t)a.nq * N;
    const size_t istride = (size_t)(a.ny + 2) * plane;
    const bool has_dep = item.dep >= 0;
    const int j_up = yneg ? (a.ny - row0 + 1) : row0;   // row just upwind of the item's first row
    const int chunk = item.q_count * N;                 // values per column
    const size_t qoff = (size_t)item.q_begin * N;
    const int max_cols = max(1, (16 * 32) / chunk);   // columns whose values fit the 16-entry buffer
    double *trace = has_dep ? a.trace + (size_t)item.dep * a.trace_stride : nullptr;

    int fetch = 0;
    long long idle = 0;
    unsigned ns = 32;
    while (fetch < a.nx) {
        int n = 0;
        if (lane == 0)
            while (n < kS && n < max_cols && fetch + n < a.nx &&
                   mbar_test(L.empty + (fetch + n) % kS, (uint32_t)((((fetch + n) / kS) & 1) ^ 1)))
                ++n;
        n = __shfl_sync(kFull, n, 0);
        int ready = 0;
        if (n > 0) {
            // element m of this lane is flat index lane + 32 m of the n columns x chunk values; (t, e)
            // advance incrementally so the register buffer is indexed statically
            const int total = n * chunk;
            double v[16];
            unsigned col_ok = (n >= 32) ? ~0u : ((1u << n) - 1u);   // bit t: column t complete in this lane
            int t = lane / chunk, e = lane - (lane / chunk) * chunk;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int idx = lane + 32 * m;
                v[m] = 0.0;
                if (idx < total) {
                    const int col = fetch + t;
                    if (has_dep) {
                        v[m] = ld_relaxed_f64(trace + (size_t)col * G * N + e);
                        if (is_sentinel(v[m])) col_ok &= ~(1u << t);
                    } else if (a.src) {
                        const int i = xneg ? a.nx - col : 1 + col;
                        v[m] = a.src[(size_t)i * istride + (size_t)j_up * plane + qoff + e];
                    }
                }
                e += 32;
                while (e >= chunk) {
                    e -= chunk;
                    ++t;
                }
            }
            // leading columns that every lane has complete
            const unsigned all_ok = __reduce_and_sync(kFull, col_ok);
            ready = __ffs(~all_ok) - 1;
            if (ready < 0 || ready > n) ready = n;
            t = lane / chunk;
            e = lane - t * chunk;
#pragma unroll
            for (int m = 0; m < 16; ++m) {
                const int idx = lane + 32 * m;
                if (idx < total && t < ready) {
                    const int col = fetch + t;
                    L.ring[(size_t)(col % kS) * G * N + e] = v[m];
                    if (has_dep)
                        st_relaxed_f64(trace + (size_t)col * G * N + e, __longlong_as_double((long long)kTraceSentinel));
                }
                e += 32;
                while (e >= chunk) {
                    e -= chunk;
                    ++t;
                }
            }
            if (ready > 0) {
                __syncwarp();
                for (int tt = 0; tt < ready; ++tt) mbar_arrive(L.full + (fetch + tt) % kS);
                fetch += ready;
            }
        }
        if (ready > 0) {
            ns = 32;
        } else {
            if (((++idle) & 63) == 0 && ld_relaxed(a.error) != kDevOk) break;
            if (idle > a.spin_limit) {
                if (lane == 0) atomicCAS(a.error, kDevOk, kDevTimeout);
                break;
            }
            __nanosleep(ns);
            if (ns < 128) ns <<= 1;
        }
    }
}

template <int P, int MODE>
__global__ void __launch_bounds__(kMaxWarps * 32, 1) sweep_warp_kernel(const SweepArgs a) {
    constexpr int N = P * P;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ int s_stop;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Layout L = carve(smem_raw, a.wn, a.G, N, prefetch_depth(P), 32 / a.seg);
    const int rows_cta = a.wn * (32 / a.seg);

    for (;;) {
        if (threadIdx.x == 0) {
            const int it = atomicAdd(a.next_item, 1);
            s_item = it;
            s_stop = (it >= a.n_items) || (ld_relaxed(a.error) != kDevOk);
            if (!s_stop)
                for (int b = 0; b < (a.wn + 1) * kS; ++b) {
                    mbar_init(L.full + b, 32);
                    mbar_init(L.empty + b, 32);
                }
        }
        __syncthreads();
        const int it = s_item;
        if (s_stop) return;
        const SweepItem item = a.items[it];
        if ((int)threadIdx.x < item.q_count) L.w[threadIdx.x] = a.w[item.q_begin + threadIdx.x];
        __syncthreads();
        const bool has_consumer = (item.row_block + 1) * rows_cta < a.ny;
        if (warp < a.wn)
            compute_warp<P, MODE>(a, item, L, warp, lane, has_consumer, it);
        else
            helper_warp(a, item, L, lane, N);
        __syncthreads();
    }
}

template <int P, int MODE>
cudaError_t launch_t(const SweepArgs &args, int grid, size_t smem, cudaStream_t stream) {
    auto kern = sweep_warp_kernel<P, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, (args.wn + 1) * 32, smem, stream>>>(args);
    return cudaGetLastError();
}

template <int P, int MODE>
cudaError_t occ_t(int threads, size_t smem, int *n) {
    auto kern = sweep_warp_kernel<P, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, kern, threads, smem);
}

}  // namespace

size_t sweep_warp_smem_bytes(int P, int wn, int G, int seg) {
    const int N = P * P;
    return sizeof(uint64_t) * 2 * (wn + 1) * kS +
           sizeof(double) * ((size_t)(wn + 1) * kS * G * N + (size_t)wn * prefetch_depth(P) * 32 * N +
                             (size_t)wn * prefetch_depth(P) * (32 / seg) * (N + 2) + (size_t)((G + 1) & ~1) +
                             (size_t)wn * 32 * N);
}

#define IDC_WDISPATCH(P_, FN, ...)                  \
    switch (precision) {                            \
        case 0: return FN<P_, 0>(__VA_ARGS__);      \
        case 1: return FN<P_, 1>(__VA_ARGS__);      \
        case 2: return FN<P_, 2>(__VA_ARGS__);      \
        default: return cudaErrorInvalidValue;      \
    }

cudaError_t launch_sweep_warp(int P, int precision, const SweepArgs &args, int grid, size_t smem,
                              cudaStream_t stream) {
    if (args.wn < 1 || args.wn + 1 > kMaxWarps || !args.trace || args.seg < 1 || args.seg > 32 || (args.seg & (args.seg - 1)) ||
        args.G > args.seg)
        return cudaErrorInvalidValue;
    switch (P) {
        case 1: IDC_WDISPATCH(1, launch_t, args, grid, smem, stream);
        case 2: IDC_WDISPATCH(2, launch_t, args, grid, smem, stream);
        case 3: IDC_WDISPATCH(3, launch_t, args, grid, smem, stream);
        case 4: return precision == 0 ? launch_t<4, 0>(args, grid, smem, stream) : cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t sweep_warp_occupancy(int P, int precision, int threads, size_t smem, int *blocks_per_sm) {
    switch (P) {
        case 1: IDC_WDISPATCH(1, occ_t, threads, smem, blocks_per_sm);
        case 2: IDC_WDISPATCH(2, occ_t, threads, smem, blocks_per_sm);
        case 3: IDC_WDISPATCH(3, occ_t, threads, smem, blocks_per_sm);
        case 4: return precision == 0 ? occ_t<4, 0>(threads, smem, blocks_per_sm) : cudaErrorInvalidValue;
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace idc
