/*
 * CPU restatement of the reference's 2-D upwind-DG transport sweep and the operators around it.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the tests and bench.py's CPU-baseline leg check the
 * CUDA path against; nothing in the product links or calls it.  Each routine cites the reference
 * (crockatt/idc-transport-solver) file:line whose arithmetic it restates.  It is pinned against the
 * reference itself: tests/test_oracle_pin.py compares it with the reference compiled from source
 * (oracle/Makefile.ref) and tests/test_oracle_golden.py with fixtures that reference produced
 * (tests/golden/make_golden.py).
 *
 * Array layouts are the reference's (halo cells 0 and n+1 in each direction):
 *   psi   [i][j][q][d][e]   idx = e + P*(d + P*(q + nq*(j + (ny+2)*i)))     objects/RKDG/OrdinateFlux.hpp:639-700
 *   phi   [i][j][d][e]      idx = e + P*(d + P*(j + (ny+2)*i))              objects/RKDG/DensityFunction.hpp
 *   sigma [i][j]            idx = j + (ny+2)*i   (piecewise-constant, DG degree 0)
 * with P = p + 1 (DG degree p, tensor Q_p) and N = P*P dofs per cell.
 */
#ifndef IDC_SWEEP_ORACLE_H
#define IDC_SWEEP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_grid {
    int64_t nx, ny;        /* interior cells */
    double dx, dy;         /* cell widths */
    int64_t p;             /* DG degree */
    int64_t nq;            /* ordinates */
    const double *xi, *eta, *w;
    int64_t quad[5];       /* quadrant ranges [quad[k], quad[k+1]) */
} oracle_grid;

/* SweepOperator::Apply (in place, psi_inout: source in, psi out).  Returns 0. */
int oracle_sweep(const oracle_grid *g, const double *sigma_t, double dt, double *psi_inout);

/* Transposed (adjoint) sweep: solves (L + 1/dt)^T psi = source cell by cell in downwind order. */
int oracle_sweep_adjoint(const oracle_grid *g, const double *sigma_t, double dt, double *psi_inout);

/* TransportOperator::Pmv over interior cells: phi <- beta*phi + alpha * sum_q w_q psi_q. */
void oracle_pmv(const oracle_grid *g, double alpha, double beta, const double *psi, double *phi);

/* TransportOperator::Smv over interior cells (PWC sigma_s): psi_q <- beta*psi_q + alpha*sigma_s*phi/(4 pi). */
void oracle_smv(const oracle_grid *g, double alpha, double beta, const double *sigma_s, const double *phi,
                double *psi);

/* TransportOperator::Lmv over interior cells: y <- beta*y + alpha*(Omega.grad + sigma_t) x. */
void oracle_lmv(const oracle_grid *g, double alpha, double beta, const double *sigma_t, const double *x,
                double *y);

/* SISolver::Solve from a zero initial guess.  source_inout: Q in, psi out.  Returns the number of
 * iterations; *err receives the final absolute l2 change in phi. */
int64_t oracle_si(const oracle_grid *g, const double *sigma_t, const double *sigma_s, double dt,
                  double abs_tol, int64_t max_its, double *source_inout, double *err);

#ifdef __cplusplus
}
#endif

#endif
