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
// CG updates read their step lengths from device memory written by single-block reduction kernels, so
// the partial sums are added in a fixed order and the result is bitwise reproducible.
#include "idc_internal.hpp"

namespace idc {

namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ double face_coef(double Da, double Db) { return 2.0 * Da * Db / (Da + Db); }

// Fixed-order block sum of per-thread values into part[blockIdx.x].
__device__ __forceinline__ void block_sum(double acc, double *part) {
    __shared__ double s[kThreads];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = s[0];
}

// y = C u on the nx x ny cell-average array (row-major [i][j], i the x index); part <- block sums of u . y.
__global__ void dsa_apply_kernel(int nx, int ny, double dx, double dy, const double *__restrict__ Dc,
                                 const double *__restrict__ sa, const double *__restrict__ u, double *__restrict__ y,
                                 double *__restrict__ part) {
    const int n = nx * ny;
    double dot = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t / ny, j = t - (t / ny) * ny;
        const double D = Dc[t], ui = u[t];
        const double ix2 = 1.0 / (dx * dx), iy2 = 1.0 / (dy * dy);
        double acc = sa[t] * ui;
        // x faces
        acc += (i > 0) ? face_coef(D, Dc[t - ny]) * ix2 * (ui - u[t - ny]) : ui * D / (2.0 * D + 0.25 * dx) / dx;
        acc += (i < nx - 1) ? face_coef(D, Dc[t + ny]) * ix2 * (ui - u[t + ny]) : ui * D / (2.0 * D + 0.25 * dx) / dx;
        // y faces
        acc += (j > 0) ? face_coef(D, Dc[t - 1]) * iy2 * (ui - u[t - 1]) : ui * D / (2.0 * D + 0.25 * dy) / dy;
        acc += (j < ny - 1) ? face_coef(D, Dc[t + 1]) * iy2 * (ui - u[t + 1]) : ui * D / (2.0 * D + 0.25 * dy) / dy;
        y[t] = acc;
        dot = fma(ui, acc, dot);
    }
    block_sum(dot, part);
}

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


// Scalars of one CG step.  sc[0] = r.z (current), sc[1] = alpha, sc[2] = beta.
// mode 0: r.z <- sum(part)  (initialisation);  mode 1: alpha = r.z / sum(part) (part = p.Cp);
// mode 2: beta = sum(part) / r.z, r.z <- sum(part)  (part = r_new . z_new).
__global__ void cg_scalar_kernel(int nparts, const double *__restrict__ part, double *__restrict__ sc, int mode) {
    __shared__ double s[kThreads];
    double acc = 0.0;
    for (int t = threadIdx.x; t < nparts; t += blockDim.x) acc += part[t];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int h = kThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        const double v = s[0];
        if (mode == 0) {
            sc[0] = v;
        } else if (mode == 1) {
            sc[1] = v != 0.0 ? sc[0] / v : 0.0;
        } else {
            sc[2] = sc[0] != 0.0 ? v / sc[0] : 0.0;
            sc[0] = v;
        }
    }
}

// x += alpha p; r -= alpha q; z = dinv r; part <- block sums of r . z
__global__ void cg_update_kernel(int n, const double *__restrict__ sc, const double *__restrict__ p,
                                 const double *__restrict__ q, const double *__restrict__ dinv, double *__restrict__ x,
                                 double *__restrict__ r, double *__restrict__ z, double *__restrict__ part) {
    const double alpha = sc[1];
    double dot = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        x[t] = fma(alpha, p[t], x[t]);
        const double rt = fma(-alpha, q[t], r[t]);
        r[t] = rt;
        const double zt = dinv[t] * rt;
        z[t] = zt;
        dot = fma(rt, zt, dot);
    }
    block_sum(dot, part);
}

// p = z + beta p
__global__ void cg_dir_kernel(int n, const double *__restrict__ sc, const double *__restrict__ z, double *__restrict__ p) {
    const double beta = sc[2];
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) p[t] = fma(beta, p[t], z[t]);
}

// Initial state for x = 0: r = f = sigma_s * v_00 (interior), z = p = dinv r, x = 0; part <- block sums of r . z.
// rhs f = sigma_s v_00 (forward), or v_00 (transposed: sigma_s is applied to the solution instead)
__global__ void dsa_rhs_kernel(int nx, int ny, int N, const double *__restrict__ ss, int scale, const double *__restrict__ v,
                               const double *__restrict__ dinv, double *__restrict__ x, double *__restrict__ r,
                               double *__restrict__ z, double *__restrict__ p, double *__restrict__ part) {
    const int n = nx * ny;
    double dot = 0.0;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
        const int i = t / ny, j = t - (t / ny) * ny;
        const size_t c = (size_t)(i + 1) * (ny + 2) + (j + 1);
        const double f = scale ? ss[c] * v[c * N] : v[c * N];
        const double zt = dinv[t] * f;
        x[t] = 0.0;
        r[t] = f;
        z[t] = zt;
        p[t] = zt;
        dot = fma(f, zt, dot);
    }
    block_sum(dot, part);
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

}  // namespace

size_t dsa_workspace_doubles(int nx, int ny) { return (size_t)nx * ny * 8 + 148 * 4 + 8; }

cudaError_t dsa_setup(const GridDims &g, const double *sigma_t, const double *sigma_s, double *ws, cudaStream_t s) {
    const int n = g.nx * g.ny;
    double *Dc = ws, *sa = ws + n, *dinv = ws + 2 * (size_t)n;
    dsa_coef_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, sigma_t, sigma_s, Dc, sa);
    dsa_diag_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, g.dx, g.dy, Dc, sa, dinv);
    return cudaGetLastError();
}

// out = v + e_00 with C e = sigma_s v_00 approximated by cg_steps Jacobi-PCG steps from e = 0 (out may
// alias v).  5 kernels per step; returns the number of launches in *launches.
namespace {
struct DsaWs {
    double *Dc, *sa, *dinv, *x, *r, *z, *p, *q, *part, *sc;
    DsaWs(double *ws, int n) {
        Dc = ws, sa = ws + n, dinv = ws + 2 * (size_t)n, x = ws + 3 * (size_t)n, r = ws + 4 * (size_t)n;
        z = ws + 5 * (size_t)n, p = ws + 6 * (size_t)n, q = ws + 7 * (size_t)n;
        part = ws + 8 * (size_t)n, sc = part + 148 * 4;
    }
};
}  // namespace

cudaError_t dsa_rhs(const GridDims &g, const double *sigma_s, const double *v, double *ws, cudaStream_t s,
                    bool transpose) {
    const int n = g.nx * g.ny;
    const DsaWs w(ws, n);
    dsa_rhs_kernel<<<blocks_for(n), kThreads, 0, s>>>(g.nx, g.ny, g.P * g.P, sigma_s, transpose ? 0 : 1, v, w.dinv,
                                                      w.x, w.r, w.z, w.p, w.part);
    return cudaGetLastError();
}

cudaError_t dsa_cg(const GridDims &g, int cg_steps, double *ws, cudaStream_t s) {
    const int n = g.nx * g.ny;
    const DsaWs w(ws, n);
    const int nb = blocks_for(n);
    cg_scalar_kernel<<<1, kThreads, 0, s>>>(nb, w.part, w.sc, 0);
    for (int it = 0; it < cg_steps; ++it) {
        dsa_apply_kernel<<<nb, kThreads, 0, s>>>(g.nx, g.ny, g.dx, g.dy, w.Dc, w.sa, w.p, w.q, w.part);
        cg_scalar_kernel<<<1, kThreads, 0, s>>>(nb, w.part, w.sc, 1);
        cg_update_kernel<<<nb, kThreads, 0, s>>>(n, w.sc, w.p, w.q, w.dinv, w.x, w.r, w.z, w.part);
        cg_scalar_kernel<<<1, kThreads, 0, s>>>(nb, w.part, w.sc, 2);
        cg_dir_kernel<<<nb, kThreads, 0, s>>>(n, w.sc, w.z, w.p);
    }
    return cudaGetLastError();
}

int dsa_cg_launches(int cg_steps) { return 1 + 5 * cg_steps; }

cudaError_t dsa_correct(const GridDims &g, const double *v, double *ws, double *out, cudaStream_t s,
                        const double *sigma_s_after) {
    const int n = g.nx * g.ny;
    const DsaWs w(ws, n);
    const size_t tot = (size_t)(g.nx + 2) * (g.ny + 2) * g.P * g.P;
    dsa_correct_kernel<<<blocks_for(tot), kThreads, 0, s>>>(g.nx, g.ny, g.P * g.P, v, w.x, sigma_s_after, out);
    return cudaGetLastError();
}

cudaError_t dsa_apply(const GridDims &g, const double *sigma_s, const double *v, double *out, int cg_steps, double *ws,
                      cudaStream_t s, int *launches) {
    cudaError_t e = dsa_rhs(g, sigma_s, v, ws, s, false);
    if (e == cudaSuccess) e = dsa_cg(g, cg_steps, ws, s);
    if (e == cudaSuccess) e = dsa_correct(g, v, ws, out, s, nullptr);
    if (launches) *launches = 2 + dsa_cg_launches(cg_steps);
    return e;
}

}  // namespace idc
