/* Abort-stubs for the LAPACK/BLAS routines that the reference's off-path solvers (LAPACK-LU and
 * Hessenberg cell solves, relabel operator) reference.  The oracle only drives the Gaussian-elimination
 * sweep, so none of these is ever called; if one were, the oracle stops loudly instead of returning
 * garbage.  Test infrastructure only. */
#include <stdio.h>
#include <stdlib.h>
#define STUB(name) void name(void) { fprintf(stderr, "oracle: LAPACK stub '" #name "' called\n"); abort(); }
STUB(dgehrd_) STUB(dgemm_) STUB(dgemv_) STUB(dgesdd_) STUB(dgesv_) STUB(dorghr_) STUB(dormhr_)
STUB(dlacpy_) STUB(dlange_)
