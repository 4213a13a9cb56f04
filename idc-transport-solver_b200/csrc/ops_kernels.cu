// Streaming transport operators on the reference's layouts (operators/RKDG/TransportOperator.cpp):
// Pmv (moment reduction), Smv (isotropic scattering source), Lmv (explicit advection-absorption), plus
// the l2 distance used by source iteration.  All of them touch interior cells only, as the reference
// does with OpDomain::Interior.  HBM-bound streaming kernels: one pass over psi, coalesced.
#include "cell_solve.cuh"
#include "idc_internal.hpp"

namespace idc {

namespace {

constexpr int kThreads = 256;

inline int blocks_for(size_t n, int threads = kThreads) {
    size_t b = (n + threads - 1) / threads;
    if (b > (size_t)148 * 32) b = (size_t)148 * 32;   // grid-stride beyond 32 waves of 148 SMs
    return (int)(b == 0 ? 1 : b);
}

// phi(i,j,k) <- beta*phi + alpha * sum_q w_q psi(q,i,j,k): TransportOperator::Pmv, :140-158.
// In this file a zero beta means the output's old values are not read (BLAS convention), so an
// uninitialised output array never leaks NaN through 0 * NaN.
// One thread per (interior cell, dof).
__global__ void pmv_kernel(GridDims g, double alpha, double beta, const double *__restrict__ w,
                           const double *__restrict__ psi, double *__restrict__ phi) {
    const int N = g.P * g.P;
    const size_t total = (size_t)g.nx * g.ny * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % N);
        const size_t cell = t / N;
        const int i = 1 + (int)(cell / g.ny), j = 1 + (int)(cell % g.ny);
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        const double *ps = psi + cidx * (size_t)g.nq * N + k;
        double acc = beta == 0.0 ? 0.0 : phi[cidx * N + k] * beta;   // beta = 0: phi is not read
        for (int q = 0; q < g.nq; ++q) acc += alpha * w[q] * ps[(size_t)q * N];
        phi[cidx * N + k] = acc;
    }
}

// psi(q,i,j,k) <- beta*psi + alpha*sigma_s(i,j)*phi(i,j,k)/(4 pi): TransportOperator::Smv, :317-400.
// One thread per (interior cell, ordinate): the cell's sigma_s phi / (4 pi) is formed once and written to
// the ordinate's N dofs.  IDX is the index type (32-bit whenever nx ny nq fits).
template <typename IDX>
__global__ void smv_kernel(GridDims g, double alpha, double beta, const double *__restrict__ sigma_s,
                           const double *__restrict__ phi, double *__restrict__ psi) {
    const int N = g.P * g.P;
    const IDX total = (IDX)g.nx * g.ny * g.nq;
    for (IDX t = blockIdx.x * (IDX)blockDim.x + threadIdx.x; t < total; t += (IDX)gridDim.x * blockDim.x) {
        const IDX cell = t / (IDX)g.nq;
        const int q = (int)(t - cell * (IDX)g.nq);
        const int i = 1 + (int)(cell / (IDX)g.ny), j = 1 + (int)(cell - (cell / (IDX)g.ny) * (IDX)g.ny);
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        const double ss = sigma_s[cidx];
        double *out = psi + (cidx * g.nq + q) * N;
        for (int k = 0; k < N; ++k) {
            const double v = (ss * phi[cidx * N + k] / (4.0 * M_PI)) * alpha;
            out[k] = beta == 0.0 ? v : beta * out[k] + v;   // beta = 0: psi is not read
        }
    }
}

// y <- beta*y + alpha*(Omega.grad + sigma_t) x: TransportOperator::Lmv, :1215-1480 (piecewise-constant
// sigma).  One thread per (interior cell, ordinate).  With phi_sc, the scattering term of Smv is added in
// the same pass, y += (sigma_s phi_sc / (4 pi)) gamma, rounded as Lmv followed by Smv(gamma, 1) would
// round it (the IDC residual (L - S P) psi in one pass over psi).
// v = p[0 .. n): 16-byte loads when n is even and `wide` (p 16-byte aligned), else 8-byte loads.  A cell's
// dofs of one ordinate start on a 16-byte boundary of an aligned array when n is even (DG degree 1).
template <int n>
__device__ __forceinline__ void load_dofs(const double *__restrict__ p, double (&v)[n], bool wide) {
    if constexpr (n % 2 == 0) {
        if (wide) {
#pragma unroll
            for (int h = 0; h < n / 2; ++h) {
                const double2 t = reinterpret_cast<const double2 *>(p)[h];
                v[2 * h] = t.x;
                v[2 * h + 1] = t.y;
            }
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < n; ++k) v[k] = p[k];
}
template <int n>
__device__ __forceinline__ void store_dofs(double *__restrict__ p, const double (&v)[n], bool wide) {
    if constexpr (n % 2 == 0) {
        if (wide) {
#pragma unroll
            for (int h = 0; h < n / 2; ++h) reinterpret_cast<double2 *>(p)[h] = make_double2(v[2 * h], v[2 * h + 1]);
            return;
        }
    }
#pragma unroll
    for (int k = 0; k < n; ++k) p[k] = v[k];
}
__device__ __forceinline__ bool aligned16(const void *p) { return ((size_t)p & 15) == 0; }

// (Omega.grad + sigma_t) x at one interior (cell, ordinate): TransportOperator::Lmv, :1215-1480 (piecewise
// constant sigma), with x's dofs of the cell at x + base and its upwind neighbours' at +-istride, +-plane.
// With tens (high-order cross sections) the absorption term is 1/4 (2d+1)(2e+1) sum_{u,v} T(d,e; u,v) x(u,v)
// (TransportOperator::Lmv, :1335-1359) in place of s x(d,e).
template <int P>
__device__ __forceinline__ void lmv_point(const GridDims &g, const double *__restrict__ x, size_t base, size_t istride,
                                          size_t plane, double xi, double eta, double s, double (&x3)[P * P],
                                          const double *__restrict__ tens = nullptr) {
    constexpr int N = P * P;
    const bool xneg = xi <= 0.0, yneg = eta <= 0.0;
    const double *X0 = x + base;
    const double *X1 = x + base + (xneg ? (ptrdiff_t)istride : -(ptrdiff_t)istride);
    const double *X2 = x + base + (yneg ? (ptrdiff_t)plane : -(ptrdiff_t)plane);
    double x0[N], x1[N], x2[N];
    const bool wide = aligned16(x);
    load_dofs<N>(X0, x0, wide);
    load_dofs<N>(X1, x1, wide);
    load_dofs<N>(X2, x2, wide);
    if (tens) {
#pragma unroll
        for (int d = 0; d < P; ++d)
#pragma unroll
            for (int e = 0; e < P; ++e) {
                double acc = 0.0;
#pragma unroll
                for (int c = 0; c < N; ++c)
                    acc += 0.25 * double(2 * d + 1) * double(2 * e + 1) * tens[(e + P * d) * N + c] * x0[c];
                x3[e + P * d] = acc;
            }
    } else {
#pragma unroll
        for (int k = 0; k < N; ++k) x3[k] = s * x0[k];
    }
    double cv = xi / g.dx;
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int a = 0; a < P; ++a)
#pragma unroll
            for (int e = 0; e < P; ++e) {
                const double f = xneg ? (neg1pow(a) * x1[e + P * a] + neg1pow(d + a + 1) * x0[e + P * a])
                                      : (x0[e + P * a] + neg1pow(d + 1) * x1[e + P * a]);
                x3[e + P * d] += cv * double(2 * d + 1) * f;
            }
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int a = d - 1; a >= 0; a -= 2)
#pragma unroll
            for (int e = 0; e < P; ++e) x3[e + P * d] -= double(2 * (2 * d + 1)) * cv * x0[e + P * a];
    cv = eta / g.dy;
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e)
#pragma unroll
            for (int b = 0; b < P; ++b) {
                const double f = yneg ? (neg1pow(b) * x2[b + P * d] + neg1pow(e + b + 1) * x0[b + P * d])
                                      : (x0[b + P * d] + neg1pow(e + 1) * x2[b + P * d]);
                x3[e + P * d] += cv * double(2 * e + 1) * f;
            }
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e)
#pragma unroll
            for (int b = e - 1; b >= 0; b -= 2) x3[e + P * d] -= double(2 * (2 * e + 1)) * cv * x0[b + P * d];
}

// (Omega.grad + sigma_t)^T x at one interior (cell, ordinate): the transpose of lmv_point's stencil.  Cell c's
// row of L couples c with its upwind neighbours, so c's row of L^T gathers c's own value through the transposed
// cell matrix and the values of the cells downwind of c (whose upwind neighbour c is) through the transposed
// face matrices; a downwind neighbour outside the interior contributes nothing (`dn_x`, `dn_y` false): the
// ghost cells hold boundary data, not unknowns.
template <int P>
__device__ __forceinline__ void lmvt_point(const GridDims &g, const double *__restrict__ x, size_t base, size_t istride,
                                           size_t plane, double xi, double eta, double s, bool dn_x, bool dn_y,
                                           double (&y)[P * P]) {
    constexpr int N = P * P;
    const bool xneg = xi <= 0.0, yneg = eta <= 0.0;
    const double *X0 = x + base;
    const double *XD = x + base + (xneg ? -(ptrdiff_t)istride : (ptrdiff_t)istride);   // downwind in x
    const double *YD = x + base + (yneg ? -(ptrdiff_t)plane : (ptrdiff_t)plane);       // downwind in y
    double x0[N], xd[N], yd[N];
#pragma unroll
    for (int k = 0; k < N; ++k) {
        x0[k] = X0[k];
        xd[k] = dn_x ? XD[k] : 0.0;
        yd[k] = dn_y ? YD[k] : 0.0;
    }
#pragma unroll
    for (int k = 0; k < N; ++k) y[k] = s * x0[k];
    double cv = xi / g.dx;
    // lmv_point: row (d,e) += cv (2d+1) [own(d,a) x0(a,e) + up(d,a) x_up(a,e)], and -2(2d+1) cv x0(a,e) for
    // a = d-1, d-3, ...; the transpose moves each coefficient to row (a,e), column (d,e)
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int a = 0; a < P; ++a) {
            const double own = cv * double(2 * d + 1) * (xneg ? neg1pow(d + a + 1) : 1.0);
            const double up = cv * double(2 * d + 1) * (xneg ? neg1pow(a) : neg1pow(d + 1));
#pragma unroll
            for (int e = 0; e < P; ++e) y[e + P * a] += own * x0[e + P * d] + up * xd[e + P * d];
        }
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int a = d - 1; a >= 0; a -= 2)
#pragma unroll
            for (int e = 0; e < P; ++e) y[e + P * a] -= double(2 * (2 * d + 1)) * cv * x0[e + P * d];
    cv = eta / g.dy;
#pragma unroll
    for (int e = 0; e < P; ++e)
#pragma unroll
        for (int b = 0; b < P; ++b) {
            const double own = cv * double(2 * e + 1) * (yneg ? neg1pow(e + b + 1) : 1.0);
            const double up = cv * double(2 * e + 1) * (yneg ? neg1pow(b) : neg1pow(e + 1));
#pragma unroll
            for (int d = 0; d < P; ++d) y[b + P * d] += own * x0[e + P * d] + up * yd[e + P * d];
        }
#pragma unroll
    for (int e = 0; e < P; ++e)
#pragma unroll
        for (int b = e - 1; b >= 0; b -= 2)
#pragma unroll
            for (int d = 0; d < P; ++d) y[b + P * d] -= double(2 * (2 * e + 1)) * cv * x0[e + P * d];
}

// y <- beta*y + alpha*L^T x on interior cells, plus gamma * w_q sigma_s zsum / (4 pi) when zsum (the
// unweighted moment sums of x, sum_q x_q) is given: with gamma = -1 that is (L - S P)^T x, the transpose of
// the IDC residual operator (S P x puts sigma_s sum_q w_q x_q / (4 pi) on every ordinate; its transpose puts
// w_q sigma_s sum_q' x_q' / (4 pi) on ordinate q).  Ghost cells of y are not written.
template <int P, typename IDX>
__global__ void lmvt_kernel(GridDims g, double alpha, double beta, const double *__restrict__ sigma_t,
                            const double *__restrict__ xi_a, const double *__restrict__ eta_a,
                            const double *__restrict__ w_a, const double *__restrict__ x, double *__restrict__ y,
                            double gamma, const double *__restrict__ sigma_s, const double *__restrict__ zsum) {
    constexpr int N = P * P;
    const size_t plane = (size_t)g.nq * N;
    const size_t istride = (size_t)(g.ny + 2) * plane;
    const IDX total = (IDX)g.nx * g.ny * g.nq;
    for (IDX t = blockIdx.x * (IDX)blockDim.x + threadIdx.x; t < total; t += (IDX)gridDim.x * blockDim.x) {
        const IDX cell = t / (IDX)g.nq;
        const int q = (int)(t - cell * (IDX)g.nq);
        const int i = 1 + (int)(cell / (IDX)g.ny), j = 1 + (int)(cell - (cell / (IDX)g.ny) * (IDX)g.ny);
        const double xi = xi_a[q], eta = eta_a[q];
        const int id = i + (xi <= 0.0 ? -1 : 1), jd = j + (eta <= 0.0 ? -1 : 1);
        const size_t base = (size_t)i * istride + (size_t)j * plane + (size_t)q * N;
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        double y3[N];
        lmvt_point<P>(g, x, base, istride, plane, xi, eta, sigma_t[cidx], id >= 1 && id <= g.nx, jd >= 1 && jd <= g.ny,
                      y3);
        if (zsum) {
            const double c = gamma * w_a[q] * sigma_s[cidx] / (4.0 * M_PI);
#pragma unroll
            for (int k = 0; k < N; ++k) y3[k] = fma(c, zsum[cidx * N + k], y3[k]);
        }
        double *Y = y + base;
#pragma unroll
        for (int k = 0; k < N; ++k) Y[k] = beta == 0.0 ? alpha * y3[k] : beta * Y[k] + alpha * y3[k];
    }
}

// out(q, cell, k) = w_q m(cell, k) on interior cells: P^T m, the adjoint of the moment functional m . P psi as
// an angular array.  Ghost cells of out are not written.
__global__ void weighted_broadcast_kernel(GridDims g, const double *__restrict__ w, const double *__restrict__ m,
                                          double *__restrict__ out) {
    const int N = g.P * g.P;
    const size_t total = (size_t)g.nx * g.ny * g.nq * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t cell = t / ((size_t)g.nq * N);
        const size_t rest = t - cell * ((size_t)g.nq * N);
        const int q = (int)(rest / N), k = (int)(rest - (size_t)q * N);
        const int i = 1 + (int)(cell / g.ny), j = 1 + (int)(cell % g.ny);
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        out[(cidx * g.nq + q) * N + k] = w[q] * m[cidx * N + k];
    }
}

// One thread per (edge cell, ordinate, dof) of the reflecting edges: see launch_reflect_boundaries.
__global__ void reflect_kernel(GridDims g, int mask, const double *__restrict__ xi, const double *__restrict__ eta,
                               const int *__restrict__ rmap, double *__restrict__ psi) {
    const int N = g.P * g.P;
    const size_t nxe = (size_t)g.ny * g.nq * N, nye = (size_t)g.nx * g.nq * N;   // per x edge, per y edge
    const size_t total = 2 * nxe + 2 * nye;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int edge = t < nxe ? 0 : t < 2 * nxe ? 1 : t < 2 * nxe + nye ? 2 : 3;   // x-min, x-max, y-min, y-max
        if (!((mask >> edge) & 1)) continue;
        size_t r = edge < 2 ? t - edge * nxe : t - 2 * nxe - (edge - 2) * nye;
        const int k = (int)(r % N);
        r /= N;
        const int q = (int)(r % g.nq);
        const int cell = (int)(r / g.nq);   // j - 1 (x edges) or i - 1 (y edges)
        // ordinates entering through the edge: xi > 0 at x-min, xi < 0 at x-max, eta > 0 at y-min; at y-max the
        // reference's loop takes every quadrant (OrdinateFlux.cpp:1399), so the ghost values of the ordinates
        // leaving there, which no sweep reads, are written as well
        const bool in = edge == 0 ? xi[q] > 0.0 : edge == 1 ? xi[q] < 0.0 : edge == 2 ? eta[q] > 0.0 : true;
        if (!in) continue;
        const int d = k / g.P, e = k - (k / g.P) * g.P;
        int ig, jg, ii, jj, qr;
        double sgn;
        if (edge < 2) {
            jg = jj = cell + 1;
            ig = edge == 0 ? 0 : g.nx + 1;
            ii = edge == 0 ? 1 : g.nx;
            qr = rmap[q];
            sgn = (d & 1) ? -1.0 : 1.0;
        } else {
            ig = ii = cell + 1;
            jg = edge == 2 ? 0 : g.ny + 1;
            jj = edge == 2 ? 1 : g.ny;
            qr = rmap[g.nq + q];
            sgn = (e & 1) ? -1.0 : 1.0;
        }
        const size_t src = (((size_t)ii * (g.ny + 2) + jj) * g.nq + qr) * N + k;
        const size_t dst = (((size_t)ig * (g.ny + 2) + jg) * g.nq + q) * N + k;
        psi[dst] = sgn * psi[src];
    }
}

// One thread per (edge cell, value of the cell): see launch_periodic_halos.
__global__ void periodic_halos_kernel(GridDims g, double *__restrict__ psi) {
    const size_t per = (size_t)g.nq * g.P * g.P;   // values of a cell: every ordinate's dofs
    const size_t nxe = (size_t)g.ny * per, nye = (size_t)g.nx * per;
    const size_t total = nxe + nye;
    const size_t istride = (size_t)(g.ny + 2) * per;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        if (t < nye) {   // the y edges of column i: (i, 0) <- (i, ny), (i, ny + 1) <- (i, 1)
            const size_t i = 1 + t / per, l = t % per;
            double *col = psi + i * istride + l;
            col[0] = col[(size_t)g.ny * per];
            col[(size_t)(g.ny + 1) * per] = col[per];
        } else {         // the x edges of row j: (0, j) <- (nx, j), (nx + 1, j) <- (1, j)
            const size_t r = t - nye, j = 1 + r / per, l = r % per;
            double *row = psi + j * per + l;
            row[0] = row[(size_t)g.nx * istride];
            row[(size_t)(g.nx + 1) * istride] = row[istride];
        }
    }
}

// One thread per interior value: see launch_copy_interior.
__global__ void copy_interior_kernel(GridDims g, const double *__restrict__ src, double *__restrict__ dst) {
    const size_t per = (size_t)g.nq * g.P * g.P;
    const size_t total = (size_t)g.nx * g.ny * per;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t cell = t / per, l = t % per;
        const size_t i = 1 + cell / g.ny, j = 1 + cell % g.ny;
        const size_t at = (i * (g.ny + 2) + j) * per + l;
        dst[at] = src[at];
    }
}

// One thread per (edge cell, ordinate, dof) of the reflecting edges, packed edge after edge (x-min, x-max, y-min,
// y-max; absent edges take no room): see launch_reflect_ghosts.
__global__ void reflect_ghosts_kernel(GridDims g, int mask, const double *__restrict__ xi,
                                      const double *__restrict__ eta, double *__restrict__ psi,
                                      double *__restrict__ packed, int to_packed) {
    const int N = g.P * g.P;
    const size_t nxe = (size_t)g.ny * g.nq * N, nye = (size_t)g.nx * g.nq * N;
    size_t len[4], total = 0;
    for (int e = 0; e < 4; ++e) {
        len[e] = ((mask >> e) & 1) ? (e < 2 ? nxe : nye) : 0;
        total += len[e];
    }
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        int edge = 0;
        size_t r = t;
        while (r >= len[edge]) r -= len[edge++];
        const int k = (int)(r % N);
        r /= N;
        const int q = (int)(r % g.nq);
        const int cell = (int)(r / g.nq);
        const bool in = edge == 0 ? xi[q] > 0.0 : edge == 1 ? xi[q] < 0.0 : edge == 2 ? eta[q] > 0.0 : eta[q] < 0.0;
        const int ig = edge < 2 ? (edge == 0 ? 0 : g.nx + 1) : cell + 1;
        const int jg = edge < 2 ? cell + 1 : (edge == 2 ? 0 : g.ny + 1);
        const size_t gi = (((size_t)ig * (g.ny + 2) + jg) * g.nq + q) * N + k;
        if (to_packed)
            packed[t] = in ? psi[gi] : 0.0;
        else
            psi[gi] = (in && packed) ? packed[t] : 0.0;
    }
}

template <int P, typename IDX>
__global__ void lmv_kernel(GridDims g, double alpha, double beta, const double *__restrict__ sigma_t,
                           const double *__restrict__ xi_a, const double *__restrict__ eta_a,
                           const double *__restrict__ x, double *__restrict__ y, double gamma,
                           const double *__restrict__ sigma_s, const double *__restrict__ phi_sc,
                           const double *__restrict__ tensor_t, const double *__restrict__ tensor_s) {
    constexpr int N = P * P;
    const size_t plane = (size_t)g.nq * N;
    const size_t istride = (size_t)(g.ny + 2) * plane;
    const IDX total = (IDX)g.nx * g.ny * g.nq;
    for (IDX t = blockIdx.x * (IDX)blockDim.x + threadIdx.x; t < total; t += (IDX)gridDim.x * blockDim.x) {
        const IDX cell = t / (IDX)g.nq;
        const int q = (int)(t - cell * (IDX)g.nq);
        const int i = 1 + (int)(cell / (IDX)g.ny), j = 1 + (int)(cell - (cell / (IDX)g.ny) * (IDX)g.ny);
        const double xi = xi_a[q], eta = eta_a[q];
        const size_t base = (size_t)i * istride + (size_t)j * plane + (size_t)q * N;
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        double x3[N];
        lmv_point<P>(g, x, base, istride, plane, xi, eta, tensor_t ? 0.0 : sigma_t[cidx], x3,
                     tensor_t ? tensor_t + cidx * N * N : nullptr);
        double *Y = y + base;
        if (!phi_sc) {
#pragma unroll
            for (int k = 0; k < N; ++k) Y[k] = beta == 0.0 ? alpha * x3[k] : beta * Y[k] + alpha * x3[k];
        } else {
            double sc[N];   // the scattering source of Smv(gamma, 1) at this cell
            if (tensor_s) {
                const double *T = tensor_s + cidx * N * N;
#pragma unroll
                for (int d = 0; d < P; ++d)
#pragma unroll
                    for (int e = 0; e < P; ++e) {
                        double acc = 0.0;
#pragma unroll
                        for (int c = 0; c < N; ++c) acc += T[(e + P * d) * N + c] * phi_sc[cidx * N + c];
                        sc[e + P * d] = (acc * (double((2 * d + 1) * (2 * e + 1)) / (16.0 * M_PI))) * gamma;
                    }
            } else {
                const double ss = sigma_s[cidx];
#pragma unroll
                for (int k = 0; k < N; ++k) sc[k] = (ss * phi_sc[cidx * N + k] / (4.0 * M_PI)) * gamma;
            }
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const double lv = beta == 0.0 ? __dmul_rn(alpha, x3[k]) : beta * Y[k] + alpha * x3[k];
                Y[k] = __dadd_rn(lv, sc[k]);
            }
        }
    }
}

// One thread per cell of the halo-padded grid: see launch_sigma_tensor.
template <int P>
__global__ void sigma_tensor_kernel(GridDims g, const double *__restrict__ mom, TripleProducts tpi, double dxdy4,
                                    double *__restrict__ avg, double *__restrict__ tensor, double *__restrict__ cat) {
    constexpr int N = P * P;
    const size_t cells = (size_t)(g.nx + 2) * (g.ny + 2);
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < cells; c += (size_t)gridDim.x * blockDim.x) {
        const double *m = mom + c * N;
        avg[c] = m[0];
#pragma unroll
        for (int d = 0; d < P; ++d)
#pragma unroll
            for (int e = 0; e < P; ++e)
#pragma unroll
                for (int u = 0; u < P; ++u)
#pragma unroll
                    for (int v = 0; v < P; ++v) {
                        // ComputeTensor's sum over the moments (mu, nu) in its order, each term (m TPI) TPI
                        double t = 0.0;
#pragma unroll
                        for (int mu = 0; mu < P; ++mu)
#pragma unroll
                            for (int nu = 0; nu < P; ++nu)
                                t += m[nu + P * mu] * tpi.v[d + P * (u + P * mu)] * tpi.v[e + P * (v + P * nu)];
                        const size_t at = c * N * N + (size_t)(e + P * d) * N + (v + P * u);
                        tensor[at] = t;
                        if (cat) cat[at] = dxdy4 * double(2 * d + 1) * double(2 * e + 1) * t;
                    }
    }
}

// One thread per (interior cell, dof (d,e)): the cell's scattering value for (d,e), written to every ordinate.
template <int P>
__global__ void smv_tensor_kernel(GridDims g, double alpha, double beta, const double *__restrict__ tensor_s,
                                  const double *__restrict__ phi, double *__restrict__ psi) {
    constexpr int N = P * P;
    const size_t total = (size_t)g.nx * g.ny * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % N);
        const size_t cell = t / N;
        const int i = 1 + (int)(cell / g.ny), j = 1 + (int)(cell % g.ny);
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        const int d = k / P, e = k - (k / P) * P;
        const double *T = tensor_s + cidx * N * N + (size_t)k * N;
        double acc = 0.0;
#pragma unroll
        for (int c = 0; c < N; ++c) acc += T[c] * phi[cidx * N + c];
        const double v = (acc * (double((2 * d + 1) * (2 * e + 1)) / (16.0 * M_PI))) * alpha;
        double *out = psi + cidx * (size_t)g.nq * N + k;
        for (int q = 0; q < g.nq; ++q) {
            double *o = out + (size_t)q * N;
            *o = beta == 0.0 ? v : beta * *o + v;   // beta = 0: psi is not read
        }
    }
}

// Every IDC correction source of one correction level but its psi_{n-1} / (h dt) term, in one pass over the
// stages:
//     out_n = Q + sum_l c[n][l] res_l,   res_l = (L - S P) psi_l = Lmv(psi_l) - scat_l,
// scat_l = sigma_s phi_l / (4 pi) per cell (scatter_moments_kernel), n = 1 .. M-1, l = 0 .. M-1
// (IDCIntegrator::ComputeResiduals / ComputeSource, time_integrators/RKDG/idc.cpp:1657-1740), each res_l
// rounded as Lmv followed by Smv rounds it.  The residuals are never stored: a level reads its M stages once
// (neighbours from L2) and writes M-1 arrays, where stored residuals cost M reads and M writes, then M reads
// per source.  Interior cells only.  (At most 128 registers for P <= 2, two blocks per SM: the loads of a
// stage wait on the previous stage's arithmetic, so bandwidth comes from resident warps.)
template <int P, int M, typename IDX>
__global__ void __launch_bounds__(kThreads, P <= 2 ? 2 : 1)
    idc_corr_kernel(GridDims g, IdcCorr t, const double *__restrict__ sigma_t, const double *__restrict__ xi_a,
                    const double *__restrict__ eta_a) {
    constexpr int N = P * P;
    const size_t plane = (size_t)g.nq * N;
    const size_t istride = (size_t)(g.ny + 2) * plane;
    const IDX total = (IDX)g.nx * g.ny * g.nq;
    const IDX e = blockIdx.x * (IDX)blockDim.x + threadIdx.x;
    if (e >= total) return;
    const IDX cell = e / (IDX)g.nq;
    const int q = (int)(e - cell * (IDX)g.nq);
    const int i = 1 + (int)(cell / (IDX)g.ny), j = 1 + (int)(cell - (cell / (IDX)g.ny) * (IDX)g.ny);
    const double xi = xi_a[q], eta = eta_a[q];
    const size_t cidx = (size_t)i * (g.ny + 2) + j;
    const size_t base = (size_t)i * istride + (size_t)j * plane + (size_t)q * N;
    const double st = sigma_t[cidx];
    double acc[M - 1][N];
    double q0[N];
    load_dofs<N>(t.Q + base, q0, aligned16(t.Q));
#pragma unroll
    for (int n = 0; n < M - 1; ++n)
#pragma unroll
        for (int k = 0; k < N; ++k) acc[n][k] = q0[k];
#pragma unroll
    for (int l = 0; l < M; ++l) {
        double x3[N];
        lmv_point<P>(g, t.stage[l], base, istride, plane, xi, eta, st, x3);
        double sm[N];
        load_dofs<N>(t.scat[l] + cidx * N, sm, aligned16(t.scat[l]));
#pragma unroll
        for (int k = 0; k < N; ++k) {
            const double r = __dadd_rn(__dmul_rn(1.0, x3[k]), sm[k] * -1.0);
#pragma unroll
            for (int n = 0; n < M - 1; ++n) acc[n][k] = fma(t.c[n + 1][l], r, acc[n][k]);
        }
    }
#pragma unroll
    for (int n = 0; n < M - 1; ++n) store_dofs<N>(t.out[n + 1] + base, acc[n], aligned16(t.out[n + 1]));
}

// out = sigma_s phi / (4 pi) on interior cells, rounded as TransportOperator::Smv rounds its scattering term
// (operators/RKDG/TransportOperator.cpp:317-400): the modal sweep adds scale * out to its source.
__global__ void scatter_moments_kernel(GridDims g, const double *__restrict__ sigma_s, const double *__restrict__ phi,
                                       double *__restrict__ out) {
    const int N = g.P * g.P;
    const size_t total = (size_t)g.nx * g.ny * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t cell = t / N;
        const int k = (int)(t - cell * N);
        const size_t cidx = (size_t)(1 + cell / g.ny) * (g.ny + 2) + 1 + cell % g.ny;
        out[cidx * N + k] = sigma_s[cidx] * phi[cidx * N + k] / (4.0 * M_PI);
    }
}

__global__ void zero_ghost_phi_kernel(GridDims g, double *phi) {
    const int N = g.P * g.P;
    const int nxg = g.nx + 2, nyg = g.ny + 2;
    const size_t perim = (size_t)2 * nyg + (size_t)2 * g.nx;   // ghost cells
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < perim * N; t += (size_t)gridDim.x * blockDim.x) {
        const size_t c = t / N;
        const int k = (int)(t % N);
        int i, j;
        if (c < (size_t)nyg) { i = 0; j = (int)c; }
        else if (c < (size_t)2 * nyg) { i = nxg - 1; j = (int)(c - nyg); }
        else if (c < (size_t)2 * nyg + g.nx) { i = 1 + (int)(c - 2 * nyg); j = 0; }
        else { i = 1 + (int)(c - 2 * nyg - g.nx); j = nyg - 1; }
        phi[((size_t)i * nyg + j) * N + k] = 0.0;
    }
}

// phi(cell, k) = sum_{slot} part[slot](cell, k) for interior cells, ghosts zero; one thread per
// (cell, dof), slots summed in index order.
__global__ void reduce_phi_partials_kernel(GridDims g, const double *__restrict__ part, int slots, size_t stride,
                                           double *__restrict__ phi) {
    const int N = g.P * g.P;
    const size_t total = (size_t)(g.nx + 2) * (g.ny + 2) * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t cell = t / N;
        const int i = (int)(cell / (g.ny + 2)), j = (int)(cell % (g.ny + 2));
        double acc = 0.0;
        if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny)
            for (int sl = 0; sl < slots; ++sl) acc += part[(size_t)sl * stride + t];
        phi[t] = acc;
    }
}

__global__ void fill_u64_kernel(unsigned long long *p, size_t n, unsigned long long v) {
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x)
        p[t] = v;
}

__global__ void l2dist2_kernel(GridDims g, const double *__restrict__ a, const double *__restrict__ b,
                               double *__restrict__ out) {
    const int N = g.P * g.P;
    const size_t total = (size_t)g.nx * g.ny * N;
    double acc = 0.0;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const int k = (int)(t % N);
        const size_t cell = t / N;
        const int i = 1 + (int)(cell / g.ny), j = 1 + (int)(cell % g.ny);
        const size_t idx = ((size_t)i * (g.ny + 2) + j) * N + k;
        const double d = a[idx] - b[idx];
        acc += d * d;
    }
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    __shared__ double warp_sums[kThreads / 32];
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x < 32) {
        acc = threadIdx.x < (blockDim.x >> 5) ? warp_sums[threadIdx.x] : 0.0;
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
        if (threadIdx.x == 0) out[blockIdx.x] = acc;   // per-block partial, added in a fixed order afterwards
    }
}

// Partial dot products V_k . w for the vectors k = 4 blockIdx.y .. +3 (< nv) over this block's share of i
// (grid-stride in x), each a fixed-order block sum, into part[k * gridDim.x + blockIdx.x].  w is read once
// per four vectors.
constexpr int kMaxDots = 64;
constexpr int kDotBlocks = 2 * 148;
__global__ void multidot_partial_kernel(const double *__restrict__ V, int nv, size_t ld, const double *__restrict__ w,
                                        size_t n, double *__restrict__ part) {
    __shared__ double red[4][kThreads / 32];
    const int k0 = 4 * blockIdx.y;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const double wi = w[i];
#pragma unroll
        for (int m = 0; m < 4; ++m)
            if (k0 + m < nv) acc[m] = fma(V[(size_t)(k0 + m) * ld + i], wi, acc[m]);
    }
#pragma unroll
    for (int m = 0; m < 4; ++m) {
        double v = acc[m];
        for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
        if ((threadIdx.x & 31) == 0) red[m][threadIdx.x >> 5] = v;
    }
    __syncthreads();
    if (threadIdx.x < 4 && k0 + (int)threadIdx.x < nv) {
        double v = red[threadIdx.x][0];
        for (int t = 1; t < (int)(blockDim.x >> 5); ++t) v += red[threadIdx.x][t];
        part[(size_t)(k0 + threadIdx.x) * gridDim.x + blockIdx.x] = v;
    }
}

// out[k] = sum over the nb partial sums of vector k (one warp per k, fixed order).
__global__ void multidot_final_kernel(const double *__restrict__ part, int nb, double *__restrict__ out) {
    const int k = blockIdx.x;
    double v = 0.0;
    for (int b = threadIdx.x; b < nb; b += 32) v += part[(size_t)k * nb + b];
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xffffffffu, v, off);
    if (threadIdx.x == 0) out[k] = v;
}

// w[i] -= sum_k c[k] V[k*ld + i]
__global__ void multiaxpy_kernel(double *__restrict__ w, const double *__restrict__ V, int nv, size_t ld,
                                 const double *__restrict__ c, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        double acc = w[i];
        for (int k = 0; k < nv; ++k) acc -= c[k] * V[(size_t)k * ld + i];
        w[i] = acc;
    }
}

// y = a*x + b*y
__global__ void axpby_kernel(double a, const double *__restrict__ x, double b, double *__restrict__ y, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        // BLAS convention: a zero coefficient means the operand is not read (so 0 * NaN never leaks in)
        y[i] = b == 0.0 ? a * x[i] : (a == 0.0 ? b * y[i] : a * x[i] + b * y[i]);
}

// out[0] += sum x*y



// ---- IDC helpers ----

// out = sum_k c_k A_k + Q on interior cells, out = Q on ghost cells (the inflow values), psi layout:
// the FP64 source of an IDC substep (IDCIntegrator::ComputeSource, time_integrators/RKDG/idc.cpp:1691-1740).
__global__ void idc_source_kernel(GridDims g, IdcTerms t, const double *__restrict__ Q, double *__restrict__ out) {
    const size_t cell = (size_t)g.nq * g.P * g.P;
    const size_t total = (size_t)(g.nx + 2) * (g.ny + 2) * cell;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t c = e / cell;
        const int i = (int)(c / (g.ny + 2)), j = (int)(c % (g.ny + 2));
        double v = Q ? Q[e] : 0.0;
        if (i >= 1 && i <= g.nx && j >= 1 && j <= g.ny)
            for (int k = 0; k < t.n; ++k) v = fma(t.c[k], t.a[k][e], v);
        out[e] = v;
    }
}

// out = a - b + c (moment arrays, all cells)
__global__ void phi_combine_kernel(size_t n, const double *__restrict__ a, const double *__restrict__ b,
                                   const double *__restrict__ c, double *__restrict__ out) {
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
        out[e] = a[e] - b[e] + c[e];
}

// ---- adjoint helpers ----

// y = x - sigma_s / (4 pi) * lam on interior cells, y = x on ghost cells: the adjoint Peierls operator
// (I - S^T L^{-T} P^T) applied to x, given lam = sum_q (L^{-T} P^T x)_q.
__global__ void adjoint_scatter_kernel(GridDims g, const double *__restrict__ sigma_s, const double *__restrict__ x,
                                       const double *__restrict__ lam, double *__restrict__ y) {
    const int N = g.P * g.P;
    const size_t total = (size_t)(g.nx + 2) * (g.ny + 2) * N;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < total; t += (size_t)gridDim.x * blockDim.x) {
        const size_t cidx = t / N;
        const int i = (int)(cidx / (g.ny + 2)), j = (int)(cidx % (g.ny + 2));
        const bool interior = i >= 1 && i <= g.nx && j >= 1 && j <= g.ny;
        y[t] = interior ? x[t] - sigma_s[cidx] / (4.0 * M_PI) * lam[t] : x[t];
    }
}

// Gradients of J = c . phi per interior cell (one warp per cell; the cell's nq*N values are contiguous):
// dJ/dsigma_t = -sum_{q,k} lam psi, dJ/dsigma_s = sum_k Lam_k phi_k / (4 pi), dJ/dq_k = Lam_k / (4 pi),
// with Lam = sum_q lam_q and q the isotropic source moments (angular source q / (4 pi)).
// With `accumulate` the contributions are added to the outputs (sums over time steps).
__global__ void adjoint_gradient_kernel(GridDims g, const double *__restrict__ psi, const double *__restrict__ lam,
                                        const double *__restrict__ phi, const double *__restrict__ Lam,
                                        double *__restrict__ dsig_t, double *__restrict__ dsig_s, double *__restrict__ dq,
                                        int accumulate, double scale) {
    const int N = g.P * g.P;
    const int lane = threadIdx.x & 31;
    const size_t warps = (size_t)gridDim.x * (blockDim.x / 32);
    const size_t cells = (size_t)g.nx * g.ny;
    for (size_t c = blockIdx.x * (size_t)(blockDim.x / 32) + (threadIdx.x >> 5); c < cells; c += warps) {
        const int i = 1 + (int)(c / g.ny), j = 1 + (int)(c % g.ny);
        const size_t cidx = (size_t)i * (g.ny + 2) + j;
        const size_t base = cidx * (size_t)g.nq * N;
        double acc = 0.0;
        for (int t = lane; t < g.nq * N; t += 32) acc = fma(lam[base + t], psi[base + t], acc);
        for (int off = 16; off > 0; off >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, off);
        double accs = 0.0;
        if (lane < N) {
            const double L = Lam[cidx * N + lane];
            accs = L * phi[cidx * N + lane];
            if (dq) dq[cidx * N + lane] = (accumulate ? dq[cidx * N + lane] : 0.0) + scale * (L / (4.0 * M_PI));
        }
        for (int off = 16; off > 0; off >>= 1) accs += __shfl_xor_sync(0xffffffffu, accs, off);
        if (lane == 0) {
            if (dsig_t) dsig_t[cidx] = (accumulate ? dsig_t[cidx] : 0.0) - scale * acc;
            if (dsig_s) dsig_s[cidx] = (accumulate ? dsig_s[cidx] : 0.0) + scale * (accs / (4.0 * M_PI));
        }
    }
}

}  // namespace

size_t multidot_scratch_doubles() { return (size_t)kMaxDots * kDotBlocks; }

cudaError_t launch_multidot(const double *V, int nv, size_t ld, const double *w, size_t n, double *out, double *scratch,
                            cudaStream_t s) {
    if (nv < 1 || nv > kMaxDots) return cudaErrorInvalidValue;
    int bx = blocks_for(n);
    if (bx > kDotBlocks) bx = kDotBlocks;
    multidot_partial_kernel<<<dim3(bx, (nv + 3) / 4), kThreads, 0, s>>>(V, nv, ld, w, n, scratch);
    multidot_final_kernel<<<nv, 32, 0, s>>>(scratch, bx, out);
    return cudaGetLastError();
}
cudaError_t launch_multiaxpy(double *w, const double *V, int nv, size_t ld, const double *c, size_t n, cudaStream_t s) {
    multiaxpy_kernel<<<blocks_for(n), kThreads, 0, s>>>(w, V, nv, ld, c, n);
    return cudaGetLastError();
}

cudaError_t launch_axpby(double a, const double *x, double b, double *y, size_t n, cudaStream_t s) {
    axpby_kernel<<<blocks_for(n), kThreads, 0, s>>>(a, x, b, y, n);
    return cudaGetLastError();
}

cudaError_t launch_dot(const double *x, const double *y, size_t n, double *out, double *scratch, cudaStream_t s) {
    return launch_multidot(x, 1, n, y, n, out, scratch, s);   // fixed order: bitwise reproducible
}

cudaError_t launch_pmv(const GridDims &g, double alpha, double beta, const double *w, const double *psi, double *phi,
                       cudaStream_t s) {
    const size_t n = (size_t)g.nx * g.ny * g.P * g.P;
    pmv_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, w, psi, phi);
    return cudaGetLastError();
}

cudaError_t launch_smv(const GridDims &g, double alpha, double beta, const double *sigma_s, const double *phi,
                       double *psi, cudaStream_t s) {
    const size_t n = (size_t)g.nx * g.ny * g.nq;
    if (n < (size_t)INT32_MAX)
        smv_kernel<int32_t><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, sigma_s, phi, psi);
    else
        smv_kernel<size_t><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, sigma_s, phi, psi);
    return cudaGetLastError();
}

template <int P>
static void lmv_p(const GridDims &g, size_t n, double alpha, double beta, const double *sigma_t, const double *xi,
                  const double *eta, const double *x, double *y, double gamma, const double *sigma_s,
                  const double *phi_sc, const double *tensor_t, const double *tensor_s, cudaStream_t s) {
    if (n < (size_t)INT32_MAX)
        lmv_kernel<P, int32_t><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, sigma_t, xi, eta, x, y, gamma, sigma_s,
                                                                   phi_sc, tensor_t, tensor_s);
    else
        lmv_kernel<P, size_t><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, sigma_t, xi, eta, x, y, gamma, sigma_s,
                                                                  phi_sc, tensor_t, tensor_s);
}

template <int P>
static void lmvt_p(const GridDims &g, size_t n, double alpha, double beta, const double *sigma_t, const double *xi,
                   const double *eta, const double *w, const double *x, double *y, double gamma,
                   const double *sigma_s, const double *zsum, cudaStream_t s) {
    if (n < (size_t)INT32_MAX)
        lmvt_kernel<P, int32_t><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, sigma_t, xi, eta, w, x, y, gamma,
                                                                    sigma_s, zsum);
    else
        lmvt_kernel<P, size_t><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, sigma_t, xi, eta, w, x, y, gamma,
                                                                   sigma_s, zsum);
}

cudaError_t launch_lmv_transpose(const GridDims &g, double alpha, double beta, const double *sigma_t, const double *xi,
                                 const double *eta, const double *w, const double *x, double *y, cudaStream_t s,
                                 double gamma, const double *sigma_s, const double *zsum) {
    const size_t n = (size_t)g.nx * g.ny * g.nq;
    switch (g.P) {
        case 1: lmvt_p<1>(g, n, alpha, beta, sigma_t, xi, eta, w, x, y, gamma, sigma_s, zsum, s); break;
        case 2: lmvt_p<2>(g, n, alpha, beta, sigma_t, xi, eta, w, x, y, gamma, sigma_s, zsum, s); break;
        case 3: lmvt_p<3>(g, n, alpha, beta, sigma_t, xi, eta, w, x, y, gamma, sigma_s, zsum, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_weighted_broadcast(const GridDims &g, const double *w, const double *m, double *out,
                                     cudaStream_t s) {
    weighted_broadcast_kernel<<<blocks_for((size_t)g.nx * g.ny * g.nq * g.P * g.P), kThreads, 0, s>>>(g, w, m, out);
    return cudaGetLastError();
}

cudaError_t launch_reflect_boundaries(const GridDims &g, int mask, const double *xi, const double *eta,
                                      const int *rmap, double *psi, cudaStream_t s) {
    const size_t total = 2 * (size_t)(g.nx + g.ny) * g.nq * g.P * g.P;
    reflect_kernel<<<blocks_for(total), kThreads, 0, s>>>(g, mask, xi, eta, rmap, psi);
    return cudaGetLastError();
}

cudaError_t launch_periodic_halos(const GridDims &g, double *psi, cudaStream_t s) {
    const size_t total = (size_t)(g.nx + g.ny) * g.nq * g.P * g.P;
    periodic_halos_kernel<<<blocks_for(total), kThreads, 0, s>>>(g, psi);
    return cudaGetLastError();
}

cudaError_t launch_copy_interior(const GridDims &g, const double *src, double *dst, cudaStream_t s) {
    const size_t total = (size_t)g.nx * g.ny * g.nq * g.P * g.P;
    copy_interior_kernel<<<blocks_for(total), kThreads, 0, s>>>(g, src, dst);
    return cudaGetLastError();
}

size_t reflect_ghost_len(const GridDims &g, int mask) {
    const size_t per = (size_t)g.nq * g.P * g.P;
    return per * ((mask & 1 ? g.ny : 0) + (mask & 2 ? g.ny : 0) + (mask & 4 ? g.nx : 0) + (mask & 8 ? g.nx : 0));
}

cudaError_t launch_reflect_ghosts(const GridDims &g, int mask, const double *xi, const double *eta, double *psi,
                                  double *packed, bool to_packed, cudaStream_t s) {
    const size_t total = reflect_ghost_len(g, mask);
    if (total == 0) return cudaSuccess;
    reflect_ghosts_kernel<<<blocks_for(total), kThreads, 0, s>>>(g, mask, xi, eta, psi, packed, to_packed ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_lmv(const GridDims &g, double alpha, double beta, const double *sigma_t, const double *xi,
                       const double *eta, const double *x, double *y, cudaStream_t s, double gamma,
                       const double *sigma_s, const double *phi_sc, const double *tensor_t, const double *tensor_s) {
    const size_t n = (size_t)g.nx * g.ny * g.nq;
    switch (g.P) {
        case 1: lmv_p<1>(g, n, alpha, beta, sigma_t, xi, eta, x, y, gamma, sigma_s, phi_sc, tensor_t, tensor_s, s); break;
        case 2: lmv_p<2>(g, n, alpha, beta, sigma_t, xi, eta, x, y, gamma, sigma_s, phi_sc, tensor_t, tensor_s, s); break;
        case 3: lmv_p<3>(g, n, alpha, beta, sigma_t, xi, eta, x, y, gamma, sigma_s, phi_sc, tensor_t, tensor_s, s); break;
        case 4: lmv_p<4>(g, n, alpha, beta, sigma_t, xi, eta, x, y, gamma, sigma_s, phi_sc, tensor_t, tensor_s, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_sigma_tensor(const GridDims &g, const double *mom, const TripleProducts &tpi, double dxdy4,
                                double *avg, double *tensor, double *cat, cudaStream_t s) {
    const size_t cells = (size_t)(g.nx + 2) * (g.ny + 2);
    switch (g.P) {
        case 1: sigma_tensor_kernel<1><<<blocks_for(cells), kThreads, 0, s>>>(g, mom, tpi, dxdy4, avg, tensor, cat); break;
        case 2: sigma_tensor_kernel<2><<<blocks_for(cells), kThreads, 0, s>>>(g, mom, tpi, dxdy4, avg, tensor, cat); break;
        case 3: sigma_tensor_kernel<3><<<blocks_for(cells), kThreads, 0, s>>>(g, mom, tpi, dxdy4, avg, tensor, cat); break;
        case 4: sigma_tensor_kernel<4><<<blocks_for(cells), kThreads, 0, s>>>(g, mom, tpi, dxdy4, avg, tensor, cat); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_smv_tensor(const GridDims &g, double alpha, double beta, const double *tensor_s,
                              const double *phi, double *psi, cudaStream_t s) {
    const size_t n = (size_t)g.nx * g.ny * g.P * g.P;
    switch (g.P) {
        case 1: smv_tensor_kernel<1><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, tensor_s, phi, psi); break;
        case 2: smv_tensor_kernel<2><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, tensor_s, phi, psi); break;
        case 3: smv_tensor_kernel<3><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, tensor_s, phi, psi); break;
        case 4: smv_tensor_kernel<4><<<blocks_for(n), kThreads, 0, s>>>(g, alpha, beta, tensor_s, phi, psi); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_scatter_moments(const GridDims &g, const double *sigma_s, const double *phi, double *out,
                                   cudaStream_t s) {
    const size_t total = (size_t)g.nx * g.ny * g.P * g.P;
    scatter_moments_kernel<<<blocks_for(total), kThreads, 0, s>>>(g, sigma_s, phi, out);
    return cudaGetLastError();
}

cudaError_t launch_zero_ghost_phi(const GridDims &g, double *phi, cudaStream_t s) {
    const size_t n = ((size_t)2 * (g.ny + 2) + (size_t)2 * g.nx) * g.P * g.P;
    zero_ghost_phi_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, phi);
    return cudaGetLastError();
}

cudaError_t launch_reduce_phi_partials(const GridDims &g, const double *part, int slots, size_t stride, double *phi,
                                       cudaStream_t s) {
    const size_t n = (size_t)(g.nx + 2) * (g.ny + 2) * g.P * g.P;
    reduce_phi_partials_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, part, slots, stride, phi);
    return cudaGetLastError();
}

cudaError_t launch_fill_u64(unsigned long long *p, size_t n, unsigned long long value, cudaStream_t s) {
    fill_u64_kernel<<<blocks_for(n), kThreads, 0, s>>>(p, n, value);
    return cudaGetLastError();
}

cudaError_t launch_l2dist2(const GridDims &g, const double *a, const double *b, double *out, double *scratch,
                           cudaStream_t s) {
    const size_t total = (size_t)g.nx * g.ny * g.P * g.P;
    int blocks = blocks_for(total);
    if (blocks > kDotBlocks) blocks = kDotBlocks;
    l2dist2_kernel<<<blocks, kThreads, 0, s>>>(g, a, b, scratch);
    multidot_final_kernel<<<1, 32, 0, s>>>(scratch, blocks, out);   // fixed order: bitwise reproducible
    return cudaGetLastError();
}

cudaError_t launch_adjoint_scatter(const GridDims &g, const double *sigma_s, const double *x, const double *lam,
                                   double *y, cudaStream_t s) {
    const size_t n = (size_t)(g.nx + 2) * (g.ny + 2) * g.P * g.P;
    adjoint_scatter_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, sigma_s, x, lam, y);
    return cudaGetLastError();
}

cudaError_t launch_adjoint_gradient(const GridDims &g, const double *psi, const double *lam, const double *phi,
                                    const double *Lam, double *dsig_t, double *dsig_s, double *dq, cudaStream_t s,
                                    bool accumulate, double scale) {
    const size_t warps = (size_t)g.nx * g.ny;
    adjoint_gradient_kernel<<<blocks_for(warps * 32), kThreads, 0, s>>>(g, psi, lam, phi, Lam, dsig_t, dsig_s, dq,
                                                                        accumulate ? 1 : 0, scale);
    return cudaGetLastError();
}

template <int P, int M>
static void idc_corr_pm(const GridDims &g, const IdcCorr &t, const double *sigma_t, const double *xi, const double *eta,
                        cudaStream_t s) {
    // one thread per element and no grid stride: blocks run in index order, so the resident ones cover a
    // contiguous front of cell rows and an x-neighbour row is still in L2 when it is read again
    const size_t n = (size_t)g.nx * g.ny * g.nq;
    const size_t blocks = (n + kThreads - 1) / kThreads;
    if (n < (size_t)INT32_MAX)
        idc_corr_kernel<P, M, int32_t><<<(unsigned)blocks, kThreads, 0, s>>>(g, t, sigma_t, xi, eta);
    else
        idc_corr_kernel<P, M, size_t><<<(unsigned)blocks, kThreads, 0, s>>>(g, t, sigma_t, xi, eta);
}

template <int P>
static cudaError_t idc_corr_p(const GridDims &g, int M, const IdcCorr &t, const double *sigma_t, const double *xi,
                              const double *eta, cudaStream_t s) {
    switch (M) {
        case 2: idc_corr_pm<P, 2>(g, t, sigma_t, xi, eta, s); break;
        case 3: idc_corr_pm<P, 3>(g, t, sigma_t, xi, eta, s); break;
        case 4: idc_corr_pm<P, 4>(g, t, sigma_t, xi, eta, s); break;
        case 5: idc_corr_pm<P, 5>(g, t, sigma_t, xi, eta, s); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_idc_corrections(const GridDims &g, int M, const IdcCorr &t, const double *sigma_t, const double *xi,
                                   const double *eta, cudaStream_t s) {
    switch (g.P) {
        case 1: return idc_corr_p<1>(g, M, t, sigma_t, xi, eta, s);
        case 2: return idc_corr_p<2>(g, M, t, sigma_t, xi, eta, s);
        case 3: return idc_corr_p<3>(g, M, t, sigma_t, xi, eta, s);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_idc_source(const GridDims &g, const IdcTerms &t, const double *Q, double *out, cudaStream_t s) {
    if (t.n < 0 || t.n > IdcTerms::kMax) return cudaErrorInvalidValue;
    const size_t n = (size_t)(g.nx + 2) * (g.ny + 2) * g.nq * g.P * g.P;
    idc_source_kernel<<<blocks_for(n), kThreads, 0, s>>>(g, t, Q, out);
    return cudaGetLastError();
}

cudaError_t launch_phi_combine(size_t n, const double *a, const double *b, const double *c, double *out, cudaStream_t s) {
    phi_combine_kernel<<<blocks_for(n), kThreads, 0, s>>>(n, a, b, c, out);
    return cudaGetLastError();
}

}  // namespace idc
