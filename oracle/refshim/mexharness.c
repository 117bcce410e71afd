/* MEX emulation runtime + a C entry point that runs one reference mexFunction on caller
 * buffers (test infrastructure).  ref_call(nrhs, in_ptrs, in_ndims, in_dims, nlhs, out_ptrs)
 * copies each output mxArray into out_ptrs[i] (caller-sized) and frees it. */
#include <string.h>
#include "mex.h"

double *mxGetPr(const mxArray *a) { return a->pr; }
const mwSize *mxGetDimensions(const mxArray *a) { return a->dims; }
mwSize mxGetNumberOfDimensions(const mxArray *a) { return a->ndim; }
mwSize mxGetM(const mxArray *a) { return a->dims[0]; }
mwSize mxGetN(const mxArray *a) { mwSize n = 1; for (int i = 1; i < a->ndim; i++) n *= a->dims[i]; return n; }
mxArray *mxCreateNumericArray(mwSize ndim, const mwSize *dims, mxClassID c, mxComplexity x)
{
    (void)c; (void)x;
    mxArray *a = calloc(1, sizeof(mxArray));
    mwSize n = 1;
    a->ndim = ndim;
    for (int i = 0; i < ndim; i++) { a->dims[i] = dims[i]; n *= dims[i]; }
    a->pr = calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    a->owns = 1;
    return a;
}
mxArray *mxCreateDoubleMatrix(mwSize m, mwSize n, mxComplexity x)
{
    mwSize d[2] = {m, n};
    return mxCreateNumericArray(2, d, mxDOUBLE_CLASS, x);
}
static char g_err[512];
void mexErrMsgTxt(const char *msg) { strncpy(g_err, msg, sizeof(g_err) - 1); fprintf(stderr, "mexErrMsgTxt: %s\n", msg); }
const char *ref_last_error(void) { return g_err; }

void mexFunction(int nlhs, mxArray *plhs[], int nrhs, const mxArray *prhs[]);

int ref_call(int nrhs, double **in, const int *in_ndims, const long long *in_dims,
             int nlhs, double **out, long long *out_numel)
{
    mxArray ins[16];
    const mxArray *pin[16];
    mxArray *pout[8] = {0};
    long long off = 0;
    g_err[0] = 0;
    for (int i = 0; i < nrhs; i++) {
        ins[i].pr = in[i]; ins[i].ndim = in_ndims[i]; ins[i].owns = 0;
        for (int d = 0; d < in_ndims[i]; d++) ins[i].dims[d] = (mwSize)in_dims[off + d];
        off += in_ndims[i];
        pin[i] = &ins[i];
    }
    mexFunction(nlhs, pout, nrhs, pin);
    if (g_err[0]) return -1;
    for (int i = 0; i < nlhs; i++) {
        if (!pout[i]) return -2;
        mwSize n = 1;
        for (int d = 0; d < pout[i]->ndim; d++) n *= pout[i]->dims[d];
        out_numel[i] = n;
        if (out[i]) memcpy(out[i], pout[i]->pr, sizeof(double) * (size_t)n);
        free(pout[i]->pr); free(pout[i]);
    }
    return 0;
}
