/* BLAS prototypes with MATLAB's ptrdiff_t integers, bound to the ILP64 OpenBLAS that numpy
 * ships (symbol prefix scipy_, suffix _64_).  Test infrastructure. */
#ifndef REFSHIM_BLAS_H
#define REFSHIM_BLAS_H
#include <stddef.h>
#define dgemm scipy_dgemm_64_
#define dgemv scipy_dgemv_64_
#define daxpy scipy_daxpy_64_
#define dcopy scipy_dcopy_64_
void dgemm(char *ta, char *tb, ptrdiff_t *m, ptrdiff_t *n, ptrdiff_t *k, double *alpha, double *a,
           ptrdiff_t *lda, double *b, ptrdiff_t *ldb, double *beta, double *c, ptrdiff_t *ldc);
void dgemv(char *t, ptrdiff_t *m, ptrdiff_t *n, double *alpha, double *a, ptrdiff_t *lda, double *x,
           ptrdiff_t *incx, double *beta, double *y, ptrdiff_t *incy);
void daxpy(ptrdiff_t *n, double *a, double *x, ptrdiff_t *incx, double *y, ptrdiff_t *incy);
void dcopy(ptrdiff_t *n, double *x, ptrdiff_t *incx, double *y, ptrdiff_t *incy);
#endif
