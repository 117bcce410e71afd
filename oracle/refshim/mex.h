/* Minimal MATLAB MEX emulation so the reference's MEX C sources compile and run outside
 * MATLAB (test infrastructure; written for this project).  Arrays are plain column-major
 * double buffers with a dimension vector; the harness (oracle/refshim/mexharness.c) builds
 * them from caller pointers and calls the reference's mexFunction. */
#ifndef REFSHIM_MEX_H
#define REFSHIM_MEX_H
#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>

typedef ptrdiff_t mwSize;
typedef ptrdiff_t mwIndex;
typedef int mxClassID;
typedef int mxComplexity;
#define mxDOUBLE_CLASS 6
#define mxREAL 0

typedef struct mxArray_tag {
    double *pr;
    mwSize ndim;
    mwSize dims[8];
    int owns;
} mxArray;

double *mxGetPr(const mxArray *a);
const mwSize *mxGetDimensions(const mxArray *a);
mwSize mxGetNumberOfDimensions(const mxArray *a);
mwSize mxGetM(const mxArray *a);
mwSize mxGetN(const mxArray *a);
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID c, mxComplexity x);
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x);
void mexErrMsgTxt(const char *msg);
#define mexPrintf printf
#endif
