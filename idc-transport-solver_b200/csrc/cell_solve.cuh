// Per-cell arithmetic of the upwind-DG sweep, one (cell, ordinate) system per thread.
//
// Conventions (reference: linear_solvers/RKDG/SweepCellSolve/SweepCellSolve.hpp:312-353):
//   a cell system has N = P*P unknowns, P = p + 1; the unknown / equation for the Legendre pair
//   (d, e) (degree d in x, e in y) has index k = e + P*d, the same order as the psi layout;
//   row = test function, column = basis function.
#pragma once

#include <cuda_runtime.h>

namespace idc {

__host__ __device__ constexpr double neg1pow(int n) { return (n & 1) ? -1.0 : 1.0; }

// x-direction coupling constant of the cell matrix, entry (row (d,e), column (a,e)), divided by
// xi_coeff = dy * xi.  SweepLinearSolveSpec::ComputeMatrices, SweepLinearSolveSpec.cpp:123-138:
// -2(2d+1) for a = d-1, d-3, ..., plus the upwind face term (2d+1) (xi >= 0) or
// (-1)^(d+a+1) (2d+1) (xi < 0).  The same constant describes the y direction with (e, b).
__host__ __device__ constexpr double face_matrix_coeff(int d, int a, bool neg) {
    return ((a < d && ((d - a) & 1)) ? -2.0 * (2 * d + 1) : 0.0) +
           (neg ? neg1pow(d + a + 1) * (2 * d + 1) : double(2 * d + 1));
}

// Upwind-neighbour coupling constant of the right-hand side, CalcB, SweepLinearSolveSpec.cpp:544-598:
// B(d,e) += coeff(d,a) * (dy xi) * psi_up(a,e), coeff = (-1)^(a+1)(2d+1) (xi <= 0) or (-1)^d (2d+1).
__host__ __device__ constexpr double face_rhs_coeff(int d, int a, bool neg) {
    return neg ? neg1pow(a + 1) * (2 * d + 1) : neg1pow(d) * (2 * d + 1);
}

// Dense cell matrix A = Aq + s I in row-major registers A[row][col], built in the reference's order
// (ComputeMatrices, then CalcA's diagonal term).  xc = dy*xi, ec = dx*eta, s = (sigma_t + 1/dt) dx dy.
template <int P, typename T>
__device__ __forceinline__ void build_cell_matrix(T (&A)[P * P][P * P], T xc, T ec, bool xneg, bool yneg, T s) {
    constexpr int N = P * P;
#pragma unroll
    for (int r = 0; r < N; ++r)
#pragma unroll
        for (int c = 0; c < N; ++c) A[r][c] = T(0);
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e) {
            const int r = e + P * d;
#pragma unroll
            for (int a = d - 1; a >= 0; a -= 2) A[r][e + P * a] -= T(2) * xc * T(2 * d + 1);
#pragma unroll
            for (int a = 0; a < P; ++a)
                A[r][e + P * a] += xneg ? T(neg1pow(d + a + 1)) * xc * T(2 * d + 1) : xc * T(2 * d + 1);
#pragma unroll
            for (int b = e - 1; b >= 0; b -= 2) A[r][b + P * d] -= T(2) * ec * T(2 * e + 1);
#pragma unroll
            for (int b = 0; b < P; ++b)
                A[r][b + P * d] += yneg ? T(neg1pow(e + b + 1)) * ec * T(2 * e + 1) : ec * T(2 * e + 1);
        }
#pragma unroll
    for (int k = 0; k < N; ++k) A[k][k] += s;
}

// Right-hand side of CalcB, SweepLinearSolveSpec.cpp:511-598:
// B = dx dy * src + upwind x trace * (dy xi) + upwind y trace * (dx eta), FP64.
template <int P>
__device__ __forceinline__ void build_cell_rhs(double (&B)[P * P], const double (&src)[P * P],
                                               const double (&xup)[P * P], const double (&yup)[P * P], double dx,
                                               double dy, double xi, double eta, bool xneg, bool yneg) {
    constexpr int N = P * P;
    double W0[N], W1[N];
    const double xs = dy * xi, ys = dx * eta, dxdy = dx * dy;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        W0[k] = xup[k] * xs;
        W1[k] = yup[k] * ys;
        B[k] = dxdy * src[k];
    }
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e)
#pragma unroll
            for (int a = 0; a < P; ++a) B[e + P * d] += W0[e + P * a] * face_rhs_coeff(d, a, xneg);
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e)
#pragma unroll
            for (int b = 0; b < P; ++b) B[e + P * d] += W1[b + P * d] * face_rhs_coeff(e, b, yneg);
}

__device__ __forceinline__ double recip(double x) { return __drcp_rn(x); }
__device__ __forceinline__ float recip(float x) { return __frcp_rn(x); }

// Unpivoted Gaussian elimination with the reference's multiplier convention
// (SIMD_GaussianElimination_CM, linear_solvers/SIMD_LinearAlgebra.hpp:74-112): forward elimination
// applied to b as it goes, then back substitution.  Pivots are inverted once each.
template <int P, typename T>
__device__ __forceinline__ void ge_solve(T (&A)[P * P][P * P], T (&b)[P * P]) {
    constexpr int N = P * P;
    T rd[N];
#pragma unroll
    for (int j = 0; j < N; ++j) {
        const T rj = recip(A[j][j]);
        rd[j] = rj;
#pragma unroll
        for (int i = j + 1; i < N; ++i) {
            A[i][j] = A[i][j] * (-rj);
            b[i] = fma(A[i][j], b[j], b[i]);
        }
#pragma unroll
        for (int k = j + 1; k < N; ++k)
#pragma unroll
            for (int i = j + 1; i < N; ++i) A[i][k] = fma(A[i][j], A[j][k], A[i][k]);
    }
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        b[i] = b[i] * rd[i];
#pragma unroll
        for (int j = 0; j < i; ++j) b[j] = fma(-A[j][i], b[i], b[j]);
    }
}

// LU factorisation in place (same elimination as ge_solve, no right-hand side); rd = 1/U(j,j).
template <int P, typename T>
__device__ __forceinline__ void lu_factor(T (&A)[P * P][P * P], T (&rd)[P * P]) {
    constexpr int N = P * P;
#pragma unroll
    for (int j = 0; j < N; ++j) {
        const T rj = recip(A[j][j]);
        rd[j] = rj;
#pragma unroll
        for (int i = j + 1; i < N; ++i) A[i][j] = A[i][j] * (-rj);
#pragma unroll
        for (int k = j + 1; k < N; ++k)
#pragma unroll
            for (int i = j + 1; i < N; ++i) A[i][k] = fma(A[i][j], A[j][k], A[i][k]);
    }
}

template <int P, typename T>
__device__ __forceinline__ void lu_solve(const T (&A)[P * P][P * P], const T (&rd)[P * P], T (&b)[P * P]) {
    constexpr int N = P * P;
#pragma unroll
    for (int j = 0; j < N; ++j)
#pragma unroll
        for (int i = j + 1; i < N; ++i) b[i] = fma(A[i][j], b[j], b[i]);
#pragma unroll
    for (int i = N - 1; i >= 0; --i) {
        b[i] = b[i] * rd[i];
#pragma unroll
        for (int j = 0; j < i; ++j) b[j] = fma(-A[j][i], b[i], b[j]);
    }
}

// r = B - A x in FP64 without forming A: A = xc (Mx (x) I) + ec (I (x) My) + s I, the Kronecker
// structure of ComputeMatrices + CalcA.
template <int P>
__device__ __forceinline__ void cell_residual(double (&r)[P * P], const double (&B)[P * P], const double (&x)[P * P],
                                              double xc, double ec, bool xneg, bool yneg, double s) {
#pragma unroll
    for (int d = 0; d < P; ++d)
#pragma unroll
        for (int e = 0; e < P; ++e) {
            double ax = 0.0, ay = 0.0;
#pragma unroll
            for (int a = 0; a < P; ++a) ax = fma(face_matrix_coeff(d, a, xneg), x[e + P * a], ax);
#pragma unroll
            for (int b = 0; b < P; ++b) ay = fma(face_matrix_coeff(e, b, yneg), x[b + P * d], ay);
            const double ax_full = fma(xc, ax, fma(ec, ay, s * x[e + P * d]));
            r[e + P * d] = B[e + P * d] - ax_full;
        }
}

// Solves one cell system.  MODE 0: FP64 elimination.  MODE 1: FP32 LU + n_refine FP64 residual
// corrections.  MODE 2: FP32 only.
template <int P, int MODE>
__device__ __forceinline__ void cell_solve(double (&x)[P * P], const double (&B)[P * P], double xc, double ec, bool xneg,
                                           bool yneg, double s, int n_refine) {
    constexpr int N = P * P;
    if constexpr (MODE == 0) {
        double A[N][N];
        build_cell_matrix<P, double>(A, xc, ec, xneg, yneg, s);
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = B[k];
        ge_solve<P, double>(A, x);
    } else {
        float A[N][N], rd[N], v[N];
        build_cell_matrix<P, float>(A, float(xc), float(ec), xneg, yneg, float(s));
        lu_factor<P, float>(A, rd);
#pragma unroll
        for (int k = 0; k < N; ++k) v[k] = float(B[k]);
        lu_solve<P, float>(A, rd, v);
#pragma unroll
        for (int k = 0; k < N; ++k) x[k] = double(v[k]);
        if constexpr (MODE == 1) {
            for (int it = 0; it < n_refine; ++it) {
                double r[N];
                cell_residual<P>(r, B, x, xc, ec, xneg, yneg, s);
#pragma unroll
                for (int k = 0; k < N; ++k) v[k] = float(r[k]);
                lu_solve<P, float>(A, rd, v);
#pragma unroll
                for (int k = 0; k < N; ++k) x[k] += double(v[k]);
            }
        }
    }
}

}  // namespace idc
