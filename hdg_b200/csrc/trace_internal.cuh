// trace_internal.cuh -- declarations shared by the translation units of the condensed-system
// path (trace_system.cu defines the kernels; capi_trace.cu the host helpers; dense_block.cu and
// noalloc.cu use both).  One definition of GmresState: it is a __global__ kernel parameter, so
// every unit must see the same layout.
#pragma once
#include <cuda_runtime.h>
#include "hdgx_common.cuh"

namespace hdgx {

// Device state of restarted GMRES: Hessenberg H[(m+1), m] column-major, the Givens rotations
// cs / sn [m+1], the rotated right-hand side g [m+1], the least-squares solution y [m+1],
// scal = [beta, |g_{j+1}|, scratch norm, ...], and (when not NULL) hist[m], the residual norm
// |g_{j+1}| after each step j of the current cycle.
struct GmresState {
    double *H, *cs, *sn, *g, *y;
    double *scal;
    double *hist;
};

__global__ void givens_kernel(GmresState, int, int);
__global__ void hess_solve_kernel(GmresState, int, int);
__global__ void gmres_init_kernel(GmresState, int);
__global__ void dot_partial_kernel(size_t, const double *, const double *, double *);
__global__ void dot_final_kernel(int, const double *, double *, int);
__global__ void axpy_kernel(size_t, const double *, double, const double *, double *);
__global__ void scale_div_kernel(size_t, const double *, const double *, double *);
__global__ void sub_kernel(size_t, const double *, const double *, double *);
__global__ void axpby_kernel(size_t, double, const double *, double, double *);

// y = Hg x with the block-size specialised kernels (kernel/matvec.m).
int trace_matvec(const hdgx_bsr *A, const double *Hg, const double *x, double *y, cudaStream_t st);

// v = (L U)^{-1} x (kernel/applyBILU0.m); y [bs*nf] is the forward sweep's output.  Single-launch
// level sweeps when A->sweep_plan is set, flag-scheduled sweeps when A->ncolors == 0, one launch
// per colour otherwise.  Allocates nothing.
int trace_bilu0_apply(const hdgx_bsr *A, const double *Mg, const double *x, double *y, double *v, cudaStream_t st);

// The same sweeps with the factors stored in FP32 (every sum in FP64); only the single-launch
// level sweeps of A->sweep_plan are offered in this form (-2 otherwise).
int trace_bilu0_apply_f32(const hdgx_bsr *A, const float *Mg32, const double *x, double *y, double *v,
                          cudaStream_t st);

// Restarted left-preconditioned GMRES (kernel/gmres_bilu0.m) with every scratch array carved from
// `mem` (hdgx_gmres_workspace_bytes(A, restart) bytes, 8-byte aligned).  The preconditioner is the
// FP64 factors Mg, or, when Mg32 is not NULL, the same factors stored in FP32.  Allocates nothing;
// the host scalars live on the caller's stack.  Returns 0 or a status of include/hdgx.h.
int gmres_bilu0_run(const hdgx_bsr *A, const double *Hg, const double *Mg, const float *Mg32, const double *b,
                    double *x, int restart, double tol, int maxit, int *iters, int *flag, double *relres,
                    double *history, void *mem, cudaStream_t st);

}  // namespace hdgx
