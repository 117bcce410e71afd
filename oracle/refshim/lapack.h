/* LAPACK prototypes (ILP64, numpy's OpenBLAS).  Test infrastructure. */
#ifndef REFSHIM_LAPACK_H
#define REFSHIM_LAPACK_H
#include <stddef.h>
#define dpotrf scipy_dpotrf_64_
#define dpotrs scipy_dpotrs_64_
#define dgesv scipy_dgesv_64_
void dpotrf(char *uplo, ptrdiff_t *n, double *a, ptrdiff_t *lda, ptrdiff_t *info);
void dpotrs(char *uplo, ptrdiff_t *n, ptrdiff_t *nrhs, double *a, ptrdiff_t *lda, double *b,
            ptrdiff_t *ldb, ptrdiff_t *info);
void dgesv(ptrdiff_t *n, ptrdiff_t *nrhs, double *a, ptrdiff_t *lda, ptrdiff_t *ipiv, double *b,
           ptrdiff_t *ldb, ptrdiff_t *info);
#endif
