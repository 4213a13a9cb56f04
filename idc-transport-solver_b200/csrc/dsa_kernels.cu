// Diffusion synthetic acceleration (DSA) for the Peierls-form GMRES: a 2-D cell-centred finite-volume
// diffusion operator on the cell-average moment and a fixed number of Jacobi-preconditioned conjugate
// gradient steps, all scalars on the device (no host round trip per step).
//
// The reference has DSA only in 1-D (a SIP-DG diffusion solve inside its PETSc Peierls solver,
// linear_solvers/RKDG/ImplicitSolver/PETScPeierlsSolver.cpp:27-376); this is a 2-D design.  The
// preconditioner M r = r + C^{-1} (sigma_s r_00) on the (0,0) moment, with
//     C u = -div(D grad u) + sigma_a u,   D = 1 / (3 sigma_t),   sigma_a = sigma_t - sigma_s,
// is the classic DSA correction: for the flat mode of an infinite medium, (I - P L^{-1} S)^{-1} =
// 1 + sigma_s / sigma_a exactly.  Faces use the harmonic mean of the two cells' D (uniform grid); a
// boundary face is a Marshak vacuum condition, flux = u_b / 2 with D (u - u_b) / (h/2) = u_b / 2.
// The right-hand side and all Jacobi-PCG steps run in one cooperative kernel (every block resident) with
// two grid barriers per step; each block adds the per-block partial sums in the same fixed order, so the
// step lengths are identical on every block and the result is bitwise reproducible.  The barrier waits
// are bounded: on expiry the device error word is set and every block leaves.
#include "device_sync.cuh"
#include "idc_internal.hpp"

namespace idc {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double face_coef(double Da, double Db) { return 2.0 * Da * Db / (Da + Db); }

// Diagonal of C (for the Jacobi preconditioner).
__global__ void dsa_diag_kernel(int nx, int ny, double dx, double dy, const double *__restrict__ Dc,
                                const double *__restrict__ sa, double *__restrict__ dinv) {
    const int n = nx * ny;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t / ny, j = t - (t / ny) * ny;
        const double D = Dc[t];
        const double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy);
        double acc = sa[t];
        acc += (i > 0) ? face_coef(D, Dc[t - ny]) * ix2 : D / (2.0 * D + 0.25 * dx) / dx;
        acc += (i < nx - 1) ? face_coef(D, Dc[t + ny]) * ix2 : D / (2.0 * D + 0.25 * dx) / dx;
        acc += (j > 0) ? face_coef(D, Dc[t - 1]) * iy2 : D / (2.0 * D + 0.25 * dy) / dy;
        acc += (j < ny - 1) ? face_coef(D, Dc[t + 1]) * iy2 : D / (2.0 * D + 0.25 * dy) / dy;
        dinv[t] = 1.0 / acc;
    }
}

// D = 1/(3 sigma_t), sigma_a = sigma_t - sigma_s (clamped at 0) on interior cells, from the halo arrays.
__global__ void dsa_coef_kernel(int nx, int ny, const double *__restrict__ st, const double *__restrict__ ss,
                                double *__restrict__ Dc, double *__restrict__ sa) {
    const int n = nx * ny;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t / ny, j = t - (t / ny) * ny;
        const size_t c = (size_t)(i + 1) * (ny + 2) + (j + 1);
        const double sigt = fmax(st[c], 1e-12);
        Dc[t] = 1.0 / (3.0 * sigt);
        sa[t] = fmax(st[c] - ss[c], 0.0);
    }
}


// out = v, out_00 += x (forward) or sigma_s x (transposed, ss non-null) on interior cells (phi layout).
__global__ void dsa_correct_kernel(int nx, int ny, int N, const double *v, const double *__restrict__ x,
                                   const double *__restrict__ ss, double *out) {
    const size_t total = (size_t)(nx + 2) * (ny + 2) * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t c = t / N;
        const int k = (int)(t - c * N);
        const int i = (int)(c / (ny + 2)), j = (int)(c % (ny + 2));
        double val = v[t];
        if (k == 0 && i >= 1 && i <= nx && j >= 1 && j <= ny) {
            const double xc = x[(size_t)(i - 1) * ny + (j - 1)];
            val += ss ? ss[c] * xc : xc;
        }
        out[t] = val;
    }
}

inline int blocks_for(size_t n) {
    size_t b = (n + kThreads - 1) / kThreads;
    if (b > 148 * 4) b = 148 * 4;
    return (int)(b == 0 ? 1 : b);
}

constexpr int kPcgThreads = 512;
constexpr int kMaxPcgBlocks = 1024;   // partial sums per reduction (the grid is at most one block per SM)

__device__ __forceinline__ unsigned ld_acquire_u32(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_u32(unsigned *p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Grid barrier of a cooperative launch: bar[0] counts arrivals, bar[1] is the generation.  Bounded: a block
// that waits longer than `limit` polls records kDevTimeout; a block that sees an error leaves.  Returns false
// (in every thread of the block) when the block must leave.
__device__ bool grid_barrier(unsigned *bar, int *error, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        const unsigned gen = ld_acquire_u32(bar + 1);
        __threadfence();
        if (atomicAdd(bar, 1u) == gridDim.x - 1) {
            atomicExch(bar, 0u);
            __threadfence();
            st_release_u32(bar + 1, gen + 1u);
        } else {
            for (long long n = 0; ld_acquire_u32(bar + 1) == gen; ++n) {
                if ((n & 63) == 63 && ld_relaxed(error) != kDevOk) {
                    ok = 0;
                    break;
                }
                if (n > limit) {
                    atomicCAS(error, kDevOk, kDevTimeout);
                    ok = 0;
                    break;
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Fixed-order sum of per-thread values into part[blockIdx.x] (warp trees, then the warps in order).
__device__ __forceinline__ void block_partial(double v, double *part) {
    __shared__ double w[kPcgThreads / 32];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFullMask, v, off);
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        double acc = w[0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) acc += w[k];
        part[blockIdx.x] = acc;
    }
}

// Sum of part[0 .. gridDim.x) in one fixed order, the same value in every block.
__device__ __forceinline__ double grid_total(const double *part) {
    __shared__ double s_tot;
    if (threadIdx.x < 32) {
        double v = 0.0;
        for (int k = threadIdx.x; k < (int)gridDim.x; k += 32) v += __ldcg(part + k);
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFullMask, v, off);
        if (threadIdx.x == 0) s_tot = v;
    }
    __syncthreads();
    const double t = s_tot;
    __syncthreads();
    return t;
}

struct PcgArgs {
    int nx, ny, N, scale, cg_steps;
    double dx, dy;
    const double *ss, *v, *Dc, *sa, *dinv;
    double *x, *r, *z, *p0, *p1, *q, *part_a, *part_b;
    unsigned *bar;
    int *error;
    long long spin_limit;
};

// x = C^{-1} f by cg_steps Jacobi-PCG steps from x = 0, f = sigma_s v_00 (scale) or v_00.  Per step k:
//   p <- z + beta p (beta = 0 at k = 0, where p = z), q = C p, alpha = r.z / p.q     (barrier)
//   x += alpha p, r -= alpha q, z = dinv r, beta = r.z_new / r.z                    (barrier)
// p alternates between two buffers so that a block forms its neighbours' new p itself (from the old p and
// z, both complete at the barrier) without waiting for their owners.
__global__ void __launch_bounds__(kPcgThreads) dsa_pcg_kernel(const PcgArgs a) {
    const int nx = a.nx, ny = a.ny, n = nx * ny;
    const int stride = gridDim.x * blockDim.x;
    const double ix2 = 1.0 / (a.dx * a.dx), iy2 = 1.0 / (a.dy * a.dy);

    double dot = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {   // right-hand side
        const int i = t / ny, j = t - (t / ny) * ny;
        const size_t c = (size_t)(i + 1) * (ny + 2) + (j + 1);
        const double f = a.scale ? a.ss[c] * a.v[c * a.N] : a.v[c * a.N];
        const double zt = a.dinv[t] * f;
        a.x[t] = 0.0;
        a.r[t] = f;
        a.z[t] = zt;
        a.p0[t] = zt;
        dot = fma(f, zt, dot);
    }
    block_partial(dot, a.part_b);
    if (!grid_barrier(a.bar, a.error, a.spin_limit)) return;

    double rz = 0.0;
    for (int k = 0; k < a.cg_steps; ++k) {
        const double *pc = (k & 1) ? a.p1 : a.p0;
        double *pn = (k & 1) ? a.p0 : a.p1;
        const double rz_new = grid_total(a.part_b);
        const double beta = k == 0 ? 0.0 : (rz != 0.0 ? rz_new / rz : 0.0);
        rz = rz_new;
        const double *z = a.z;
        // neighbours' values were written by other blocks before the barrier: read them from L2
        auto pv = [&](int c) { return fma(beta, __ldcg(pc + c), __ldcg(z + c)); };
        dot = 0.0;
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
            const int i = t / ny, j = t - (t / ny) * ny;
            const double D = a.Dc[t], ui = pv(t);
            pn[t] = ui;
            double acc = a.sa[t] * ui;
            acc += (i > 0) ? face_coef(D, a.Dc[t - ny]) * ix2 * (ui - pv(t - ny)) : ui * D / (2.0 * D + 0.25 * a.dx) / a.dx;
            acc += (i < nx - 1) ? face_coef(D, a.Dc[t + ny]) * ix2 * (ui - pv(t + ny)) : ui * D / (2.0 * D + 0.25 * a.dx) / a.dx;
            acc += (j > 0) ? face_coef(D, a.Dc[t - 1]) * iy2 * (ui - pv(t - 1)) : ui * D / (2.0 * D + 0.25 * a.dy) / a.dy;
            acc += (j < ny - 1) ? face_coef(D, a.Dc[t + 1]) * iy2 * (ui - pv(t + 1)) : ui * D / (2.0 * D + 0.25 * a.dy) / a.dy;
            a.q[t] = acc;
            dot = fma(ui, acc, dot);
        }
        block_partial(dot, a.part_a);
        if (!grid_barrier(a.bar, a.error, a.spin_limit)) return;

        const double pq = grid_total(a.part_a);
        const double alpha = pq != 0.0 ? rz / pq : 0.0;
        dot = 0.0;
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += stride) {
            a.x[t] = fma(alpha, pn[t], a.x[t]);
            const double rt = fma(-alpha, a.q[t], a.r[t]);
            a.r[t] = rt;
            const double zt = a.dinv[t] * rt;
            a.z[t] = zt;
            dot = fma(rt, zt, dot);
        }
        if (k + 1 == a.cg_steps) break;   // x is final; the kernel's end orders it before the correction
        block_partial(dot, a.part_b);
        if (!grid_barrier(a.bar, a.error, a.spin_limit)) return;
    }
}

// Workspace: Dc, sa, dinv, x, r, z, p0, p1, q (n each), two partial-sum arrays, the barrier words.
struct DsaWs {
    double *Dc, *sa, *dinv, *x, *r, *z, *p0, *p1, *q, *part_a, *part_b;
    unsigned *bar;
    DsaWs(double *ws, int n) {
        Dc = ws, sa = ws + n, dinv = ws + 2 * (size_t)n, x = ws + 3 * (size_t)n, r = ws + 4 * (size_t)n;
        z = ws + 5 * (size_t)n, p0 = ws + 6 * (size_t)n, p1 = ws + 7 * (size_t)n, q = ws + 8 * (size_t)n;
        part_a = ws + 9 * (size_t)n, part_b = part_a + kMaxPcgBlocks;
        bar = reinterpret_cast<unsigned *>(part_b + kMaxPcgBlocks);
    }
};

}  // namespace

size_t dsa_workspace_doubles(int nx, int ny) { return (size_t)nx * ny * 9 + 2 * kMaxPcgBlocks + 2; }

// Coefficients and the Jacobi diagonal from the cross sections; the barrier words start at zero (also after
// a barrier that gave up).
cudaError_t dsa_setup(const GridDims &g, const double *sigma_t, const double *sigma_s, double *ws, cudaStream_t s) {
    const int n = g.nx * g.ny;
    const DsaWs w(ws, n);
    dsa_coef_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, sigma_t, sigma_s, w.Dc, w.sa);
    dsa_diag_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, g.dx, g.dy, w.Dc, w.sa, w.dinv);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(w.bar, 0, 2 * sizeof(unsigned), s);
    return e;
}

cudaError_t dsa_precondition(const GridDims &g, const double *sigma_s, const double *v, double *out, int cg_steps,
                             double *ws, bool transpose, int num_sms, int *error, long long spin_limit,
                             cudaStream_t s) {
    const int n = g.nx * g.ny;
    const DsaWs w(ws, n);
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, dsa_pcg_kernel, kPcgThreads, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorCooperativeLaunchTooLarge;
    int blocks = (n + kPcgThreads - 1) / kPcgThreads;
    blocks = blocks < 1 ? 1 : blocks;
    blocks = blocks < num_sms ? blocks : num_sms;   // one block per SM at most: cheap barriers
    blocks = blocks < kMaxPcgBlocks ? blocks : kMaxPcgBlocks;
    PcgArgs a{};
    a.nx = g.nx;
    a.ny = g.ny;
    a.N = g.P * g.P;
    a.scale = transpose ? 0 : 1;
    a.cg_steps = cg_steps;
    a.dx = g.dx;
    a.dy = g.dy;
    a.ss = sigma_s;
    a.v = v;
    a.Dc = w.Dc;
    a.sa = w.sa;
    a.dinv = w.dinv;
    a.x = w.x;
    a.r = w.r;
    a.z = w.z;
    a.p0 = w.p0;
    a.p1 = w.p1;
    a.q = w.q;
    a.part_a = w.part_a;
    a.part_b = w.part_b;
    a.bar = w.bar;
    a.error = error;
    a.spin_limit = spin_limit;
    void *args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void *)dsa_pcg_kernel, dim3(blocks), dim3(kPcgThreads), args, 0, s);
    if (e != cudaSuccess) return e;
    const size_t tot = (size_t)(g.nx + 2) * (g.ny + 2) * g.P * g.P;
    dsa_correct_kernel<<<blocks_for(tot), kThreads, 0, s>>>(g.nx, g.ny, g.P * g.P, v, w.x,
                                                            transpose ? sigma_s : nullptr, out);
    return cudaGetLastError();
}

}  // namespace idc

