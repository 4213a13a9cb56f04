// Persistent wavefront sweep kernel for sm_100a.
//
// Replaces SweepPatternUniCartWavefront::Sweep (linear_solvers/Abstract/SweepPattern/
// SweepPatternUniCartWavefront.cpp:121-332) + SweepCellSolveBase::ConstructAndSolve
// (linear_solvers/Abstract/SweepCellSolve/SweepCellSolveBase.cpp:86-103).
//
// Decomposition.  Work items (host-built, SweepItem) are R consecutive rows of one quadrant for a
// chunk of G ordinates of that quadrant.  A CTA of G*R threads owns an item; thread (o, r) owns
// ordinate q_begin+o on row r and walks the columns upwind -> downwind, row r lagging row r-1 by one
// step, so after step t the CTA has solved the anti-diagonal {(r, t - r)} of its R x nx block:
//   * the x-upwind trace of a thread is its own previous result (registers);
//   * the y-upwind trace of row r > 0 is row r-1's result of the previous step, exchanged through a
//     double-buffered shared-memory stage;
//   * the y-upwind trace of row 0 is the last row of the item `dep` (previous row block), read from
//     global memory (L2) once that item's progress flag says the column is done; row block 0 reads
//     the ghost row, i.e. the inflow boundary values.
// Items are handed out by an atomic queue in row-block order, so every item's producer was taken
// earlier by a CTA that is already running: no CTA can wait on one that has not started.  Waits are
// bounded: after `spin_limit` polls the CTA sets the device error word and leaves; every other CTA
// leaves as soon as it sees the word.
//
// The four quadrants run concurrently (the reference's "simultaneous" branch, :235-300), which is
// valid for vacuum/inflow boundaries.  The moment reduction phi = sum_q w_q psi_q (TransportOperator::
// Pmv) is fused: after each step the CTA reduces its G ordinates per cell and adds the partial sum
// to phi with one FP64 atomic per (cell, dof).  The isotropic scattering source (TransportOperator::
// Smv) can be fused into the source read.
#include "cell_solve.cuh"
#include "idc_internal.hpp"

#include <cstdio>

namespace idc {

constexpr int kMaxSweepThreads = 320;

__device__ __forceinline__ int ld_acquire_gpu(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ int ld_relaxed_gpu(const int *p) {
    int v;
    asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_gpu(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Waits until *flag >= target.  Returns false (and records kDevTimeout) after `limit` polls, or as
// soon as another CTA has recorded an error.
__device__ bool wait_at_least(const int *flag, int target, int *error, long long limit) {
    unsigned ns = 32;
    for (long long n = 0;; ++n) {
        if (ld_acquire_gpu(flag) >= target) return true;
        if (ld_relaxed_gpu(error) != kDevOk) return false;
        if (n >= limit) {
            atomicCAS(error, kDevOk, kDevTimeout);
            return false;
        }
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
}

template <int P, int MODE>
__global__ void __launch_bounds__(kMaxSweepThreads) sweep_kernel(const SweepArgs a) {
    constexpr int N = P * P;
    extern __shared__ __align__(16) double smem[];
    __shared__ int s_item;
    __shared__ int s_abort;

    const int tid = threadIdx.x;
    const int G = a.G, R = a.R;
    const int o = tid % G;
    const int r = tid / G;                 // >= R for the padding threads of the last warp
    double *stage = smem;                  // [2][R][G][N]
    double *s_w = smem + 2 * R * G * N;    // [G]
    const size_t plane = (size_t)a.nq * N;               // doubles per cell
    const size_t istride = (size_t)(a.ny + 2) * plane;   // doubles per x index
    const double dxdy = a.dx * a.dy;

    for (;;) {
        if (tid == 0) {
            s_item = atomicAdd(a.next_item, 1);
            s_abort = ld_relaxed_gpu(a.error) != kDevOk;
        }
        __syncthreads();
        const int it = s_item;
        const bool stop = s_abort || it >= a.n_items;
        __syncthreads();
        if (stop) return;

        const SweepItem item = a.items[it];
        const bool xneg = item.quadrant >= 2;
        const bool yneg = (item.quadrant & 1) != 0;
        const int row0 = item.row_block * R;
        const int R_eff = min(R, a.ny - row0);
        const bool active = (o < item.q_count) && (r < R_eff);
        const int q = item.q_begin + (active ? o : 0);
        const int j = yneg ? (a.ny - (row0 + r)) : (1 + row0 + r);
        const ptrdiff_t ystep = yneg ? (ptrdiff_t)plane : -(ptrdiff_t)plane;   // (i, j) -> (i, j + yoff)

        if (tid < item.q_count) s_w[tid] = a.w[item.q_begin + tid];

        double xi = 0.0, eta = 0.0, xc = 0.0, ec = 0.0;
        double xup[N];
#pragma unroll
        for (int k = 0; k < N; ++k) xup[k] = 0.0;
        if (active) {
            xi = a.xi[q];
            eta = a.eta[q];
            xc = a.dy * xi;
            ec = a.dx * eta;
            const int ig = xneg ? a.nx + 1 : 0;   // inflow ghost column
            const double *g = a.src + (size_t)ig * istride + (size_t)j * plane + (size_t)q * N;
#pragma unroll
            for (int k = 0; k < N; ++k) xup[k] = g[k];
        }
        __syncthreads();

        const int T = a.nx + R_eff - 1;
        for (int t = 0; t < T; ++t) {
            if (item.dep >= 0 && t < a.nx) {
                if (tid == 0 && !wait_at_least(a.progress + item.dep, t + 1, a.error, a.spin_limit)) s_abort = 1;
                __syncthreads();
                if (s_abort) return;
            }
            const int c = t - r;
            double *st_cur = stage + (size_t)(t & 1) * R * G * N;
            const double *st_prev = stage + (size_t)((t + 1) & 1) * R * G * N;
            if (active && c >= 0 && c < a.nx) {
                const int i = xneg ? a.nx - c : 1 + c;
                const size_t cell = (size_t)i * istride + (size_t)j * plane + (size_t)q * N;
                double src[N], yup[N], B[N], x[N];
#pragma unroll
                for (int k = 0; k < N; ++k) src[k] = a.src[cell + k];
                if (a.phi_scatter) {   // fused TransportOperator::Smv(scale, 1, sigma_s, phi -> src)
                    const size_t cidx = (size_t)i * (a.ny + 2) + j;
                    const double sv = a.sigma_s[cidx];
                    const double *ph = a.phi_scatter + cidx * N;
#pragma unroll
                    for (int k = 0; k < N; ++k) src[k] += a.scatter_scale * (sv * ph[k] / (4.0 * M_PI));
                }
                if (r == 0) {
                    if (item.dep >= 0) {
                        const double *yp = a.out + (ptrdiff_t)cell + ystep;
#pragma unroll
                        for (int k = 0; k < N; ++k) yup[k] = __ldcg(yp + k);
                    } else {
                        const double *yp = a.src + (ptrdiff_t)cell + ystep;   // ghost row
#pragma unroll
                        for (int k = 0; k < N; ++k) yup[k] = yp[k];
                    }
                } else {
                    const double *yp = st_prev + ((size_t)(r - 1) * G + o) * N;
#pragma unroll
                    for (int k = 0; k < N; ++k) yup[k] = yp[k];
                }
                build_cell_rhs<P>(B, src, xup, yup, a.dx, a.dy, xi, eta, xneg, yneg);
                const double s = (a.sigma_t[(size_t)i * (a.ny + 2) + j] + a.inv_dt) * a.dx * a.dy;
                cell_solve<P, MODE>(x, B, xc, ec, xneg, yneg, s, a.n_refine);
                double *dst = a.out + cell;
                double *sp = st_cur + ((size_t)r * G + o) * N;
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    dst[k] = x[k];
                    sp[k] = x[k];
                    xup[k] = x[k];
                }
            }
            __syncthreads();

            if (a.phi) {
                for (int idx = tid; idx < R_eff * N; idx += blockDim.x) {
                    const int rr = idx / N, k = idx - rr * N, cc = t - rr;
                    if (cc >= 0 && cc < a.nx) {
                        double sum = 0.0;
                        const double *sp = st_cur + (size_t)rr * G * N + k;
                        for (int oo = 0; oo < item.q_count; ++oo) sum += s_w[oo] * sp[(size_t)oo * N];
                        const int ii = xneg ? a.nx - cc : 1 + cc;
                        const int jj = yneg ? (a.ny - (row0 + rr)) : (1 + row0 + rr);
                        atomicAdd(a.phi + ((size_t)ii * (a.ny + 2) + jj) * N + k, sum);
                    }
                }
            }

            const int c_last = t - (R_eff - 1);
            if (tid == 0 && c_last >= 0) {
                __threadfence();
                st_release_gpu(a.progress + it, c_last + 1);
            }
        }
        (void)dxdy;
    }
}

size_t sweep_smem_bytes(int P, int R, int G) {
    return sizeof(double) * ((size_t)2 * R * G * P * P + (size_t)G);
}

template <int P, int MODE>
static cudaError_t launch_one(const SweepArgs &args, int grid, int block, size_t smem, cudaStream_t stream) {
    auto kern = sweep_kernel<P, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<grid, block, smem, stream>>>(args);
    return cudaGetLastError();
}

template <int P, int MODE>
static cudaError_t occ_one(int block, size_t smem, int *n) {
    auto kern = sweep_kernel<P, MODE>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(n, kern, block, smem);
}

#define IDC_DISPATCH(P_, FN, ...)                                   \
    switch (precision) {                                            \
        case 0: return FN<P_, 0>(__VA_ARGS__);                      \
        case 1: return FN<P_, 1>(__VA_ARGS__);                      \
        case 2: return FN<P_, 2>(__VA_ARGS__);                      \
        default: return cudaErrorInvalidValue;                      \
    }

cudaError_t launch_sweep(int P, int precision, const SweepArgs &args, int grid, int block, size_t smem,
                         cudaStream_t stream) {
    if (block > kMaxSweepThreads) return cudaErrorInvalidValue;
    switch (P) {
        case 1: IDC_DISPATCH(1, launch_one, args, grid, block, smem, stream);
        case 2: IDC_DISPATCH(2, launch_one, args, grid, block, smem, stream);
        case 3: IDC_DISPATCH(3, launch_one, args, grid, block, smem, stream);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t sweep_occupancy(int P, int precision, int block, size_t smem, int *blocks_per_sm) {
    switch (P) {
        case 1: IDC_DISPATCH(1, occ_one, block, smem, blocks_per_sm);
        case 2: IDC_DISPATCH(2, occ_one, block, smem, blocks_per_sm);
        case 3: IDC_DISPATCH(3, occ_one, block, smem, blocks_per_sm);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace idc
