/*
 * CPU restatement of the reference's 2-D upwind-DG sweep (see sweep_oracle.h).  TEST INFRASTRUCTURE
 * ONLY: the checker for the CUDA path, never part of it.
 */
#include "sweep_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define MAXP 4
#define MAXN (MAXP * MAXP)

static double neg1pow(int64_t n) { return (n % 2 == 0) ? 1.0 : -1.0; }

static size_t psi_index(const oracle_grid *g, int64_t q, int64_t i, int64_t j, int64_t d, int64_t e) {
    const int64_t P = g->p + 1;
    return (size_t)(e + P * (d + P * (q + g->nq * (j + (g->ny + 2) * i))));
}

static size_t phi_index(const oracle_grid *g, int64_t i, int64_t j, int64_t d, int64_t e) {
    const int64_t P = g->p + 1;
    return (size_t)(e + P * (d + P * (j + (g->ny + 2) * i)));
}

static size_t cell_index(const oracle_grid *g, int64_t i, int64_t j) { return (size_t)(j + (g->ny + 2) * i); }

/* Row/column index of a (degree x, degree y) pair inside the N x N cell matrix.  Column-major
 * storage A[r + N*c], row = test function, column = basis function
 * (MatIdx_CM, linear_solvers/RKDG/SweepCellSolve/SweepCellSolve.hpp:312-353). */
#define RC(P, d, e) ((e) + (P) * (d))

/* Angular part of the cell matrix for one ordinate: SweepLinearSolveSpec<RKDG>::ComputeMatrices,
 * linear_solvers/RKDG/SweepCellSolve/SweepLinearSolveSpec.cpp:98-158 (the same entries, same order). */
static void compute_aq(int64_t p, double dx, double dy, double xi, double eta, double *A) {
    const int64_t P = p + 1, N = P * P;
    const double xi_coeff = dy * xi;
    const double eta_coeff = dx * eta;
    memset(A, 0, sizeof(double) * (size_t)(N * N));
    for (int64_t d = 0; d <= p; ++d) {
        for (int64_t e = 0; e <= p; ++e) {
            const int64_t r = RC(P, d, e);
            for (int64_t a = d - 1; a >= 0; a -= 2) A[r + N * RC(P, a, e)] -= 2.0 * xi_coeff * (double)(2 * d + 1);
            if (xi < 0) {
                for (int64_t a = 0; a <= p; ++a)
                    A[r + N * RC(P, a, e)] += neg1pow(d + a + 1) * xi_coeff * (double)(2 * d + 1);
            } else {
                for (int64_t a = 0; a <= p; ++a) A[r + N * RC(P, a, e)] += xi_coeff * (double)(2 * d + 1);
            }
            for (int64_t b = e - 1; b >= 0; b -= 2) A[r + N * RC(P, d, b)] -= 2.0 * eta_coeff * (double)(2 * e + 1);
            if (eta < 0) {
                for (int64_t b = 0; b <= p; ++b)
                    A[r + N * RC(P, d, b)] += neg1pow(e + b + 1) * eta_coeff * (double)(2 * e + 1);
            } else {
                for (int64_t b = 0; b <= p; ++b) A[r + N * RC(P, d, b)] += eta_coeff * (double)(2 * e + 1);
            }
        }
    }
}

/* SIMD_GaussianElimination_CM, linear_solvers/SIMD_LinearAlgebra.hpp:45-118 (one lane): unpivoted
 * column-major elimination with multipliers A(i,j) /= -A(j,j), then back substitution. */
static void gauss_eliminate(int64_t N, double *A, double *b) {
#define IM(i, j) A[(i) + N * (j)]
    for (int64_t j = 0; j < N; ++j) {
        for (int64_t i = j + 1; i < N; ++i) {
            IM(i, j) /= -IM(j, j);
            b[i] += IM(i, j) * b[j];
        }
        for (int64_t k = j + 1; k < N; ++k)
            for (int64_t i = j + 1; i < N; ++i) IM(i, k) += IM(i, j) * IM(j, k);
    }
    for (int64_t i = N - 1; i >= 0; --i) {
        b[i] /= IM(i, i);
        for (int64_t j = 0; j < i; ++j) b[j] -= IM(j, i) * b[i];
    }
#undef IM
}

/* One ordinate over the whole grid, upwind to downwind.  Each cell is CalcB
 * (SweepLinearSolveSpec.cpp:473-598), CalcA for piecewise-constant sigma (:286-298), GE and
 * StoreResult (RKDG/SweepCellSolve/SweepCellSolve.cpp:93-99).  Cells are visited i-major from the
 * upwind corner; any order that visits both upwind neighbours first gives the same arithmetic as the
 * reference's diagonal wavefront (SweepPatternUniCartWavefront.cpp:205-230). */
static void sweep_ordinate(const oracle_grid *g, int64_t q, const double *sigma_t, double dt, double *psi) {
    const int64_t p = g->p, P = p + 1, N = P * P;
    const double xi = g->xi[q], eta = g->eta[q];
    double Aq[MAXN * MAXN], A[MAXN * MAXN], B[MAXN], W0[MAXN], W1[MAXN];
    compute_aq(p, g->dx, g->dy, xi, eta, Aq);

    const int xneg = xi <= 0.0, yneg = eta <= 0.0;          /* all_xi_negative / all_eta_negative */
    const int64_t xoff = xneg ? +1 : -1, yoff = yneg ? +1 : -1;
    const double dxdy = g->dx * g->dy;

    for (int64_t ii = 1; ii <= g->nx; ++ii) {
        const int64_t i = (xi < 0) ? g->nx - ii + 1 : ii;  /* SetSigns mirroring, :283-288 */
        for (int64_t jj = 1; jj <= g->ny; ++jj) {
            const int64_t j = (eta < 0) ? g->ny - jj + 1 : jj;

            /* CalcB */
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e) {
                    W0[RC(P, d, e)] = psi[psi_index(g, q, i + xoff, j, d, e)];
                    W1[RC(P, d, e)] = psi[psi_index(g, q, i, j + yoff, d, e)];
                }
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e) {
                    W0[RC(P, d, e)] *= g->dy * xi;
                    W1[RC(P, d, e)] *= g->dx * eta;
                }
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e) B[RC(P, d, e)] = dxdy * psi[psi_index(g, q, i, j, d, e)];
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e)
                    for (int64_t a = 0; a <= p; ++a) {
                        const double c = xneg ? neg1pow(a + 1) * (double)(2 * d + 1) : neg1pow(d) * (double)(2 * d + 1);
                        B[RC(P, d, e)] += W0[RC(P, a, e)] * c;
                    }
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e)
                    for (int64_t b = 0; b <= p; ++b) {
                        const double c = yneg ? neg1pow(b + 1) * (double)(2 * e + 1) : neg1pow(e) * (double)(2 * e + 1);
                        B[RC(P, d, e)] += W1[RC(P, d, b)] * c;
                    }

            /* CalcA, piecewise-constant sigma */
            memcpy(A, Aq, sizeof(double) * (size_t)(N * N));
            const double coeff = (sigma_t[cell_index(g, i, j)] + 1.0 / dt) * g->dx * g->dy;
            for (int64_t k = 0; k < N; ++k) A[k + N * k] += coeff;

            gauss_eliminate(N, A, B);

            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e) psi[psi_index(g, q, i, j, d, e)] = B[RC(P, d, e)];
        }
    }
}

int oracle_sweep(const oracle_grid *g, const double *sigma_t, double dt, double *psi_inout) {
    if (g->p < 0 || g->p >= MAXP) return 1;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < g->nq; ++q) sweep_ordinate(g, q, sigma_t, dt, psi_inout);
    return 0;
}

/* Transposed cell solve by unpivoted GE on A^T. */
static void sweep_ordinate_adjoint(const oracle_grid *g, int64_t q, const double *sigma_t, double dt,
                                   double *psi) {
    const int64_t p = g->p, P = p + 1, N = P * P;
    const double xi = g->xi[q], eta = g->eta[q];
    double Aq[MAXN * MAXN], A[MAXN * MAXN], B[MAXN];
    compute_aq(p, g->dx, g->dy, xi, eta, Aq);
    const int xneg = xi <= 0.0, yneg = eta <= 0.0;
    /* forward sweep: cell (i,j) reads (i+xoff, j) and (i, j+yoff); the transpose runs the other way and
     * the cell that a forward cell fed now feeds it. */
    const int64_t xoff = xneg ? +1 : -1, yoff = yneg ? +1 : -1;
    const double dxdy = g->dx * g->dy;
    for (int64_t ii = g->nx; ii >= 1; --ii) {
        const int64_t i = (xi < 0) ? g->nx - ii + 1 : ii;
        for (int64_t jj = g->ny; jj >= 1; --jj) {
            const int64_t j = (eta < 0) ? g->ny - jj + 1 : jj;
            /* rhs: dxdy * source, plus the transposed coupling of the downwind neighbours that read this cell.
             * Forward: B_down(d,e) += c_x(d,a) * (dy xi) * psi_here(a,e)  with c_x as in CalcB.
             * Adjoint: rhs_here(a,e) += c_x(d,a) * (dy xi) * lambda_down(d,e). */
            for (int64_t k = 0; k < N; ++k) B[k] = dxdy * psi[psi_index(g, q, i, j, k / P, k % P)];
            const int64_t id = i - xoff, jd = j - yoff;   /* downwind neighbours */
            if (id >= 1 && id <= g->nx) {
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e)
                        for (int64_t a = 0; a <= p; ++a) {
                            const double c = xneg ? neg1pow(a + 1) * (double)(2 * d + 1) : neg1pow(d) * (double)(2 * d + 1);
                            B[RC(P, a, e)] += c * g->dy * xi * psi[psi_index(g, q, id, j, d, e)];
                        }
            }
            if (jd >= 1 && jd <= g->ny) {
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e)
                        for (int64_t b = 0; b <= p; ++b) {
                            const double c = yneg ? neg1pow(b + 1) * (double)(2 * e + 1) : neg1pow(e) * (double)(2 * e + 1);
                            B[RC(P, d, b)] += c * g->dx * eta * psi[psi_index(g, q, i, jd, d, e)];
                        }
            }
            /* A^T */
            for (int64_t r = 0; r < N; ++r)
                for (int64_t c = 0; c < N; ++c) A[r + N * c] = Aq[c + N * r];
            const double coeff = (sigma_t[cell_index(g, i, j)] + 1.0 / dt) * g->dx * g->dy;
            for (int64_t k = 0; k < N; ++k) A[k + N * k] += coeff;
            gauss_eliminate(N, A, B);
            /* the system was scaled by dx*dy on the rhs: lambda solves A^T lambda = dxdy*src + coupling,
             * which is the transpose of the forward scaling, so lambda is the adjoint of psi w.r.t. the
             * unscaled source. */
            for (int64_t k = 0; k < N; ++k) psi[psi_index(g, q, i, j, k / P, k % P)] = B[k];
        }
    }
}

int oracle_sweep_adjoint(const oracle_grid *g, const double *sigma_t, double dt, double *psi_inout) {
    if (g->p < 0 || g->p >= MAXP) return 1;
    /* Downwind order needs every downwind cell solved first; process each ordinate serially. */
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t q = 0; q < g->nq; ++q) sweep_ordinate_adjoint(g, q, sigma_t, dt, psi_inout);
    return 0;
}

/* TransportOperator::Pmv, operators/RKDG/TransportOperator.cpp:140-158, OpDomain::Interior. */
void oracle_pmv(const oracle_grid *g, double alpha, double beta, const double *psi, double *phi) {
    const int64_t p = g->p;
#pragma omp parallel for collapse(2)
    for (int64_t i = 1; i <= g->nx; ++i)
        for (int64_t j = 1; j <= g->ny; ++j) {
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e) phi[phi_index(g, i, j, d, e)] *= beta;
            for (int64_t q = 0; q < g->nq; ++q)
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e)
                        phi[phi_index(g, i, j, d, e)] += alpha * g->w[q] * psi[psi_index(g, q, i, j, d, e)];
        }
}

/* TransportOperator::Smv, operators/RKDG/TransportOperator.cpp:317-400, PWC branch, OpDomain::Interior. */
void oracle_smv(const oracle_grid *g, double alpha, double beta, const double *sigma_s, const double *phi,
                double *psi) {
    const int64_t p = g->p, P = p + 1;
#pragma omp parallel for collapse(2)
    for (int64_t i = 1; i <= g->nx; ++i)
        for (int64_t j = 1; j <= g->ny; ++j) {
            double val[MAXN];
            for (int64_t d = 0; d <= p; ++d)
                for (int64_t e = 0; e <= p; ++e) {
                    double v = sigma_s[cell_index(g, i, j)] * phi[phi_index(g, i, j, d, e)] / (4.0 * M_PI);
                    val[d + P * e] = v * alpha;
                }
            for (int64_t q = 0; q < g->nq; ++q)
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e) {
                        const size_t k = psi_index(g, q, i, j, d, e);
                        psi[k] = beta * psi[k] + val[d + P * e];
                    }
        }
}

/* TransportOperator::Lmv, operators/RKDG/TransportOperator.cpp:1215-1480 (full-block branch, PWC
 * sigma): y <- beta*y + alpha*[ sigma x + xi/dx (...) + eta/dy (...) ] per interior cell and ordinate. */
void oracle_lmv(const oracle_grid *g, double alpha, double beta, const double *sigma_t, const double *x,
                double *y) {
    const int64_t p = g->p, P = p + 1;
#pragma omp parallel for collapse(2)
    for (int64_t i = 1; i <= g->nx; ++i)
        for (int64_t j = 1; j <= g->ny; ++j)
            for (int64_t q = 0; q < g->nq; ++q) {
                const double xi = g->xi[q], eta = g->eta[q];
                const int xneg = xi <= 0.0, yneg = eta <= 0.0;
                const int64_t xoff = xneg ? +1 : -1, yoff = yneg ? +1 : -1;
                double X0[MAXN], X1[MAXN], X2[MAXN], X3[MAXN];
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e) {
                        X0[RC(P, d, e)] = x[psi_index(g, q, i, j, d, e)];
                        X1[RC(P, d, e)] = x[psi_index(g, q, i + xoff, j, d, e)];
                        X2[RC(P, d, e)] = x[psi_index(g, q, i, j + yoff, d, e)];
                        X3[RC(P, d, e)] = 0.0;
                    }
                const double s = sigma_t[cell_index(g, i, j)];
                for (int64_t k = 0; k < P * P; ++k) X3[k] += s * X0[k];
                double cv = xi / g->dx;
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t a = 0; a <= p; ++a)
                        for (int64_t e = 0; e <= p; ++e) {
                            if (xneg)
                                X3[RC(P, d, e)] += cv * (double)(2 * d + 1) *
                                                   (neg1pow(a) * X1[RC(P, a, e)] + neg1pow(d + a + 1) * X0[RC(P, a, e)]);
                            else
                                X3[RC(P, d, e)] += cv * (double)(2 * d + 1) *
                                                   (X0[RC(P, a, e)] + neg1pow(d + 1) * X1[RC(P, a, e)]);
                        }
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t a = d - 1; a >= 0; a -= 2)
                        for (int64_t e = 0; e <= p; ++e)
                            X3[RC(P, d, e)] -= (double)(2 * (2 * d + 1)) * cv * X0[RC(P, a, e)];
                cv = eta / g->dy;
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e)
                        for (int64_t b = 0; b <= p; ++b) {
                            if (yneg)
                                X3[RC(P, d, e)] += cv * (double)(2 * e + 1) *
                                                   (neg1pow(b) * X2[RC(P, d, b)] + neg1pow(e + b + 1) * X0[RC(P, d, b)]);
                            else
                                X3[RC(P, d, e)] += cv * (double)(2 * e + 1) *
                                                   (X0[RC(P, d, b)] + neg1pow(e + 1) * X2[RC(P, d, b)]);
                        }
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e)
                        for (int64_t b = e - 1; b >= 0; b -= 2)
                            X3[RC(P, d, e)] -= (double)(2 * (2 * e + 1)) * cv * X0[RC(P, d, b)];
                for (int64_t d = 0; d <= p; ++d)
                    for (int64_t e = 0; e <= p; ++e) {
                        const size_t k = psi_index(g, q, i, j, d, e);
                        y[k] = beta * y[k] + alpha * X3[RC(P, d, e)];
                    }
            }
}

/* SISolver::Solve, linear_solvers/Abstract/ImplicitSolver/SISolver.cpp:190-254, zero initial guess. */
int64_t oracle_si(const oracle_grid *g, const double *sigma_t, const double *sigma_s, double dt,
                  double abs_tol, int64_t max_its, double *source_inout, double *err_out) {
    const int64_t P = g->p + 1, N = P * P;
    const size_t npsi = (size_t)(g->nx + 2) * (size_t)(g->ny + 2) * (size_t)(g->nq * N);
    const size_t nphi = (size_t)(g->nx + 2) * (size_t)(g->ny + 2) * (size_t)N;
    double *psi = calloc(npsi, sizeof(double));
    double *phi_cur = calloc(nphi, sizeof(double));
    double *phi_last = calloc(nphi, sizeof(double));
    int64_t iter = 0;
    double err = INFINITY;
    oracle_pmv(g, 1.0, 0.0, psi, phi_cur);
    while (iter < max_its && err > abs_tol) {
        ++iter;
        double *t = phi_cur; phi_cur = phi_last; phi_last = t;
        memcpy(psi, source_inout, npsi * sizeof(double));
        oracle_smv(g, 1.0, 1.0, sigma_s, phi_last, psi);
        oracle_sweep(g, sigma_t, dt, psi);
        oracle_pmv(g, 1.0, 0.0, psi, phi_cur);
        double s = 0.0;
        for (int64_t i = 1; i <= g->nx; ++i)
            for (int64_t j = 1; j <= g->ny; ++j)
                for (int64_t k = 0; k < N; ++k) {
                    const size_t idx = (size_t)k + (size_t)N * cell_index(g, i, j);
                    const double d = phi_cur[idx] - phi_last[idx];
                    s += d * d;
                }
        err = sqrt(s);
    }
    memcpy(source_inout, psi, npsi * sizeof(double));
    free(psi); free(phi_cur); free(phi_last);
    if (err_out) *err_out = err;
    return iter;
}
