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
// The right-hand side and all Jacobi-PCG steps run in one cooperative kernel (every block resident), in
// the Chronopoulos-Gear form of CG with one global reduction and one grid barrier per step; each block adds
// the per-block partial sums in the same fixed order, so the step lengths are identical on every block and
// the result is bitwise reproducible.  The barrier waits are bounded: on expiry the device error word is
// set and every block leaves.
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
// It also re-arms the PCG kernel's barrier counter (zero at the start of every launch).
__global__ void dsa_correct_kernel(int nx, int ny, int N, const double *v, const double *__restrict__ x,
                                   const double *__restrict__ ss, double *out, unsigned *count) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *count = 0u;
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

// Grid barrier number e (0, 1, ...) of a cooperative launch on an arrival counter that is zero when the
// kernel starts: each block adds one, then waits until the counter reaches (e + 1) blocks.  Bounded: a block
// that waits longer than `limit` polls records kDevTimeout; a block that sees an error leaves.  Returns false
// (in every thread of the block) when the block must leave.
__device__ bool grid_barrier(unsigned *count, unsigned e, int *error, long long limit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(count, 1u);
        const unsigned target = (e + 1u) * gridDim.x;
        for (long long n = 0; (int)(ld_acquire_u32(count) - target) < 0; ++n) {
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
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Fixed-order sums of per-thread values (a, b) into part[blockIdx.x] and part[gridDim.x + blockIdx.x].
__device__ __forceinline__ void block_partial2(double a, double b, double *part) {
    __shared__ double w[2][kPcgThreads / 32];
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(kFullMask, a, off);
        b += __shfl_down_sync(kFullMask, b, off);
    }
    if ((threadIdx.x & 31) == 0) {
        w[0][threadIdx.x >> 5] = a;
        w[1][threadIdx.x >> 5] = b;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double acc = w[threadIdx.x][0];
        for (int k = 1; k < (int)(blockDim.x >> 5); ++k) acc += w[threadIdx.x][k];
        part[threadIdx.x * gridDim.x + blockIdx.x] = acc;
    }
}

// Sums of part[0 .. gridDim.x) and part[gridDim.x .. 2 gridDim.x) in one fixed order: the same values in
// every block.  The partial sums were written by other blocks before the barrier: read from L2.
__device__ __forceinline__ void grid_totals(const double *part, double &a, double &b) {
    __shared__ double s_tot[2];
    if (threadIdx.x < 64) {
        const int h = threadIdx.x >> 5, l = threadIdx.x & 31;
        double v = 0.0;
        for (int k = l; k < (int)gridDim.x; k += 32) v += __ldcg(part + h * gridDim.x + k);
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(kFullMask, v, off);
        if (l == 0) s_tot[h] = v;
    }
    __syncthreads();
    a = s_tot[0];
    b = s_tot[1];
    __syncthreads();
}

struct PcgArgs {
    int nx, ny, N, scale, cg_steps;
    double dx, dy;
    const double *ss, *v, *Dc, *sa, *dinv;
    double *x, *p, *r[2], *u[2], *w[2], *s[2], *part;
    unsigned *count;
    int *error;
    long long spin_limit;
};

// y = (C u)(t) for cell t = (i, j) given u at t (ut) and at any cell (uv).
template <typename U>
__device__ __forceinline__ double apply_c(const PcgArgs &a, int t, int i, int j, double ut, U uv) {
    const int nx = a.nx, ny = a.ny;
    const double ix2 = 1.0 / (a.dx * a.dx), iy2 = 1.0 / (a.dy * a.dy);
    const double D = a.Dc[t];
    double acc = a.sa[t] * ut;
    acc += (i > 0) ? face_coef(D, a.Dc[t - ny]) * ix2 * (ut - uv(t - ny)) : ut * D / (2.0 * D + 0.25 * a.dx) / a.dx;
    acc += (i < nx - 1) ? face_coef(D, a.Dc[t + ny]) * ix2 * (ut - uv(t + ny)) : ut * D / (2.0 * D + 0.25 * a.dx) / a.dx;
    acc += (j > 0) ? face_coef(D, a.Dc[t - 1]) * iy2 * (ut - uv(t - 1)) : ut * D / (2.0 * D + 0.25 * a.dy) / a.dy;
    acc += (j < ny - 1) ? face_coef(D, a.Dc[t + 1]) * iy2 * (ut - uv(t + 1)) : ut * D / (2.0 * D + 0.25 * a.dy) / a.dy;
    return acc;
}

// x = C^{-1} f by cg_steps Jacobi-preconditioned CG steps from x = 0, f = sigma_s v_00 (scale) or v_00, in
// the Chronopoulos-Gear form (one global reduction per step; the same iterates as standard PCG in exact
// arithmetic).  With u = M r and w = C u:
//   gamma = r.u, delta = w.u, beta = gamma / gamma_old (0 at the first step),
//   alpha = gamma / (delta - beta gamma / alpha_old),
//   p = u + beta p, s = w + beta s, x += alpha p, r -= alpha s, u = M r, w = C u.
// r, u, w, s alternate between two buffers: a block forms its neighbours' new u from their old r, w, s
// (complete at the barrier, never overwritten in the same step) instead of waiting for their owners, so a
// step has one grid barrier.
__global__ void __launch_bounds__(kPcgThreads) dsa_pcg_kernel(const PcgArgs a) {
    const int nx = a.nx, ny = a.ny, n = nx * ny;
    const int stride = gridDim.x * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    (void)nx;
    auto rhs = [&](int t) {
        const int i = t / ny, j = t - (t / ny) * ny;
        const size_t c = (size_t)(i + 1) * (ny + 2) + (j + 1);
        return a.scale ? a.ss[c] * a.v[c * a.N] : a.v[c * a.N];
    };
    // r = f, u = M f, w = C u, x = p = s = 0; partial r.u and w.u
    double g = 0.0, d = 0.0;
    for (int t = t0; t < n; t += stride) {
        const int i = t / ny, j = t - (t / ny) * ny;
        const double f = rhs(t), ut = a.dinv[t] * f;
        const double wt = apply_c(a, t, i, j, ut, [&](int c) { return a.dinv[c] * rhs(c); });
        a.r[0][t] = f;
        a.u[0][t] = ut;
        a.w[0][t] = wt;
        a.s[0][t] = 0.0;
        a.x[t] = 0.0;
        a.p[t] = 0.0;
        g = fma(f, ut, g);
        d = fma(wt, ut, d);
    }
    block_partial2(g, d, a.part);
    unsigned e = 0;
    if (!grid_barrier(a.count, e++, a.error, a.spin_limit)) return;

    double gamma_old = 0.0, alpha_old = 1.0;
    for (int k = 0; k < a.cg_steps; ++k) {
        const int c0 = k & 1, c1 = c0 ^ 1;
        const double *rc = a.r[c0], *wc = a.w[c0], *sc = a.s[c0], *uc = a.u[c0];
        double *rn = a.r[c1], *wn = a.w[c1], *sn = a.s[c1], *un = a.u[c1];
        double gamma, delta;
        grid_totals(a.part + (size_t)2 * kMaxPcgBlocks * c0, gamma, delta);   // partials alternate halves
        const double beta = k == 0 ? 0.0 : (gamma_old != 0.0 ? gamma / gamma_old : 0.0);
        const double den = delta - (k == 0 ? 0.0 : beta * gamma / alpha_old);
        const double alpha = den != 0.0 ? gamma / den : 0.0;
        gamma_old = gamma;
        alpha_old = alpha != 0.0 ? alpha : 1.0;
        const bool last = k + 1 == a.cg_steps;
        // the new u of any cell from its old r, w, s (read from L2: other blocks wrote them)
        auto unew = [&](int c) {
            const double sv = fma(beta, __ldcg(sc + c), __ldcg(wc + c));
            return a.dinv[c] * fma(-alpha, sv, __ldcg(rc + c));
        };
        g = 0.0;
        d = 0.0;
        for (int t = t0; t < n; t += stride) {
            const double pt = fma(beta, a.p[t], uc[t]);
            const double st = fma(beta, sc[t], wc[t]);
            a.p[t] = pt;
            a.x[t] = fma(alpha, pt, a.x[t]);
            if (last) continue;   // x is final; the kernel's end orders it before the correction
            const double rt = fma(-alpha, st, rc[t]);
            const double ut = a.dinv[t] * rt;
            const int i = t / ny, j = t - (t / ny) * ny;
            const double wt = apply_c(a, t, i, j, ut, unew);
            sn[t] = st;
            rn[t] = rt;
            un[t] = ut;
            wn[t] = wt;
            g = fma(rt, ut, g);
            d = fma(wt, ut, d);
        }
        if (last) break;
        block_partial2(g, d, a.part + (size_t)2 * kMaxPcgBlocks * (c1));
        if (!grid_barrier(a.count, e++, a.error, a.spin_limit)) return;
    }
}

// Workspace: Dc, sa, dinv, x, p, r[2], u[2], w[2], s[2] (n each), partial sums, the barrier counter.
struct DsaWs {
    double *Dc, *sa, *dinv, *x, *p, *r[2], *u[2], *w[2], *s[2], *part;
    unsigned *count;
    DsaWs(double *ws, int n) {
        double *q = ws;
        auto take = [&]() { double *o = q; q += n; return o; };
        Dc = take(), sa = take(), dinv = take(), x = take(), p = take();
        for (int b = 0; b < 2; ++b) r[b] = take(), u[b] = take(), w[b] = take(), s[b] = take();
        part = q;
        count = reinterpret_cast<unsigned *>(part + 4 * kMaxPcgBlocks);
    }
};

}  // namespace

size_t dsa_workspace_doubles(int nx, int ny) { return (size_t)nx * ny * 13 + 4 * kMaxPcgBlocks + 2; }

// Coefficients and the Jacobi diagonal from the cross sections; the barrier words start at zero (also after
// a barrier that gave up).
cudaError_t dsa_setup(const GridDims &g, const double *sigma_t, const double *sigma_s, double *ws, cudaStream_t s) {
    const int n = g.nx * g.ny;
    const DsaWs w(ws, n);
    dsa_coef_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, sigma_t, sigma_s, w.Dc, w.sa);
    dsa_diag_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, g.dx, g.dy, w.Dc, w.sa, w.dinv);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemsetAsync(w.count, 0, sizeof(unsigned), s);
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
    a.p = w.p;
    for (int b = 0; b < 2; ++b) a.r[b] = w.r[b], a.u[b] = w.u[b], a.w[b] = w.w[b], a.s[b] = w.s[b];
    a.part = w.part;
    a.count = w.count;
    a.error = error;
    a.spin_limit = spin_limit;
    void *args[] = {&a};
    e = cudaLaunchCooperativeKernel((const void *)dsa_pcg_kernel, dim3(blocks), dim3(kPcgThreads), args, 0, s);
    if (e != cudaSuccess) return e;
    const size_t tot = (size_t)(g.nx + 2) * (g.ny + 2) * g.P * g.P;
    dsa_correct_kernel<<<blocks_for(tot), kThreads, 0, s>>>(g.nx, g.ny, g.P * g.P, v, w.x,
                                                            transpose ? sigma_s : nullptr, out, w.count);
    return cudaGetLastError();
}

}  // namespace idc

