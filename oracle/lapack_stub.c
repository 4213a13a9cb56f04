/* LAPACK/BLAS symbols that the reference's sources reference, for the reference build in oracle/_ref
 * (test infrastructure only; LAPACK itself is not installed here).
 *
 * dgesv_ is implemented: the reference's Quadrule::ComputeQuadratureWeights (utils/Quadrule/Quadrule.cpp:
 * 1200-1250) solves a small Vandermonde system with it when the IDC integrator sets up its node weights.
 * It follows LAPACK's documented DGESV contract (A = P L U by Gaussian elimination with partial pivoting,
 * the first row of largest magnitude as pivot, then forward and back substitution for every right-hand
 * side; column-major A[lda x n], B[ldb x nrhs], 1-based IPIV, INFO = i > 0 for an exactly zero pivot
 * U(i,i)); it is the textbook algorithm, not LAPACK's blocked code, so results can differ from a LAPACK
 * build in the last bits.
 *
 * The rest abort: they serve off-path solvers (LAPACK-LU and Hessenberg cell solves, the relabel
 * operator) that the oracle never drives; if one were called, the oracle stops loudly instead of returning
 * garbage. */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>

int dgesv_(int *n_, int *nrhs_, double *a, int *lda_, int *ipiv, double *b, int *ldb_, int *info) {
    const int n = *n_, nrhs = *nrhs_, lda = *lda_, ldb = *ldb_;
    *info = 0;
    if (n < 0) *info = -1;
    else if (nrhs < 0) *info = -2;
    else if (lda < (n > 1 ? n : 1)) *info = -4;
    else if (ldb < (n > 1 ? n : 1)) *info = -7;
    if (*info != 0) return 0;
#define A(i, j) a[(size_t)(j) * lda + (i)]
#define B(i, j) b[(size_t)(j) * ldb + (i)]
    for (int k = 0; k < n; ++k) {
        int p = k;
        for (int i = k + 1; i < n; ++i)
            if (fabs(A(i, k)) > fabs(A(p, k))) p = i;
        ipiv[k] = p + 1;
        if (A(p, k) == 0.0) {
            if (*info == 0) *info = k + 1;
            continue;
        }
        if (p != k)
            for (int j = 0; j < n; ++j) {
                const double t = A(k, j);
                A(k, j) = A(p, j);
                A(p, j) = t;
            }
        const double inv = 1.0 / A(k, k);
        for (int i = k + 1; i < n; ++i) A(i, k) *= inv;
        for (int j = k + 1; j < n; ++j)
            for (int i = k + 1; i < n; ++i) A(i, j) -= A(i, k) * A(k, j);
    }
    if (*info != 0) return 0;
    for (int r = 0; r < nrhs; ++r) {
        for (int k = 0; k < n; ++k) {   /* row interchanges, in order */
            const int p = ipiv[k] - 1;
            if (p != k) {
                const double t = B(k, r);
                B(k, r) = B(p, r);
                B(p, r) = t;
            }
        }
        for (int k = 0; k < n; ++k)      /* L y = P b, unit diagonal */
            for (int i = k + 1; i < n; ++i) B(i, r) -= A(i, k) * B(k, r);
        for (int k = n - 1; k >= 0; --k) {   /* U x = y */
            B(k, r) /= A(k, k);
            for (int i = 0; i < k; ++i) B(i, r) -= A(i, k) * B(k, r);
        }
    }
#undef A
#undef B
    return 0;
}

#define STUB(name) void name(void) { fprintf(stderr, "oracle: LAPACK stub '" #name "' called\n"); abort(); }
STUB(dgehrd_) STUB(dgemm_) STUB(dgemv_) STUB(dgesdd_) STUB(dorghr_) STUB(dormhr_)
STUB(dlacpy_) STUB(dlange_)
