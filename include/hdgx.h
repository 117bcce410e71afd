/*
 * hdgx.h -- C ABI of the B200 (sm_100a) HDG elemental hot path.
 *
 * Every entry point takes caller-owned DEVICE pointers (cudaMalloc'd or cudaMallocAsync'd;
 * pinned host memory is not accepted for the compute calls) in the reference's MATLAB
 * column-major layouts with the element index last, plus explicit dimensions instead of
 * mxArray introspection, and runs on the caller's CUDA stream.  Index arrays (perm, elcon,
 * t2f, bf, colind) stay 1-based as the reference stores them.  Every function returns an
 * int status: 0 ok, < 0 bad argument / unsupported size / CUDA error (see hdgx_status_str).
 * Per-element numerical failures (zero or non-finite pivot) are reported through the
 * optional `status[ne]` array (0 ok, 1 singular mass matrix, 2 singular local system,
 * 3 unsupported boundary type) and counted in the return value of hdgx_status_count.
 *
 * Reference call surface each entry point replaces (paths relative to the reference tree):
 *   hdgx_elemental   kernel/hdg_elemental.m:1   [AE,FE,DUDG,DUDG_DUH] = hdg_elemental(master,app,dgnodes,bf,UDG,UH,SH)
 *   hdgx_schur_uq    kernel/schur_uq.c:193      [DUDG,DUDG_DUH,AE,FE] = schur_uq(M,C,E,BD,F,GK,H,Rq,Ru,Rh)
 *   hdgx_schur_u     kernel/schur_u.c:82        [DUDG,DUDG_DUH,AE,FE] = schur_u(BD,F,GK,H,Ru,Rh)
 *   hdgx_globalassembly   kernel/globalassembly.m:1  [Hg,Rg] = globalassembly(mesh,AE,FE)
 *   hdgx_matvec           kernel/matvec.m:1          Xg = matvec(mesh,Hg,Rg)
 *   hdgx_bilu0_factor     kernel/computeBILU0.m:1    Mg = computeBILU0(mesh,Hg)
 *   hdgx_bilu0_apply      kernel/applyBILU0.m:1      v  = applyBILU0(mesh,Mg,x)
 *   hdgx_gmres_bilu0      kernel/gmres_bilu0.m:1     [x,flags,iter,rev] = gmres_bilu0(mesh,M,A,b,x,restart,tol,maxit)
 *   hdgx_backsub          kernel/hdg_solve.m:119-121 DUDGT = DUDG + mapContractK(DUDG_DUH, DUH(elcon))
 *   hdgx_gather_uh        kernel/hdg_assemble.m:34   uh = reshape(UH(:,elcon),[ncu npf*nfe ne])
 */
#ifndef HDGX_H
#define HDGX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *hdgx_stream_t;   /* a cudaStream_t; NULL = legacy default stream */

/* Master element tables (master/mkmaster.m + util/preprocess.m:23-55), DEVICE pointers. */
typedef struct {
    int nd, porder, npv, npf, nfe, ngv, ngf;
    const double *shapvt;   /* [ngv, npv, nd+1]  shape functions/derivatives at volume Gauss points */
    const double *shapvg;   /* [npv, ngv, nd+1]  the same times the Gauss weights */
    const double *shapmv;   /* [ngv, npv, nd+1]  geometry shape functions (morder = porder) */
    const double *shapft;   /* [ngf, npf, nd]    face shape functions at face Gauss points */
    const double *shapfg;   /* [npf, ngf, nd]    the same times the face Gauss weights */
    const double *shapmf;   /* [ngf, npf, nd]    face geometry shape functions */
    const int *perm;        /* [npf, nfe]        1-based volume node of face node (master.perm) */
} hdgx_master;

#define HDGX_MAX_BND 16

/* Physics (app struct fields read by volint/faceint), passed BY VALUE. */
typedef struct {
    int nd, ncu, nc;        /* nc = ncu*(nd+1) for the (u,q) form */
    int localsolve;         /* 1: (u,q) form (only form the fused kernel supports) */
    int getdqdg;            /* 1: DUDG/DUDG_DUH carry all nc components (reference default) */
    double fc_q, fc_u;      /* fc_u and tdep are accepted; the steady path uses tdep = 0 */
    int tdep;
    double param[8];        /* [gam, epslm, Re, Pr, Minf, tau]; Re = +inf gives Euler */
    int nbnd;               /* number of boundary indices (bf = -1..-nbnd) */
    int bcm[HDGX_MAX_BND];  /* fbou type per boundary index: 5 periodic, 6 Dirichlet */
    double bcs[HDGX_MAX_BND * 5];  /* boundary state per index, row-major [nbnd][ncu] */
} hdgx_app;

/* Library identity and error strings. */
int hdgx_version(void);
const char *hdgx_status_str(int code);

/* Number of nonzero entries of a device status[n] array (synchronises the stream). */
int hdgx_status_count(const int *status, int n, hdgx_stream_t stream);

/* Fused FP64 elemental kernel: volume + face integrals + local (u,q) Schur elimination.
 * Inputs : dgnodes[npv,nd,ne], bf[nfe,ne] (int32), UDG[npv,nc,ne], UH[ncu,npf*nfe,ne]
 *          (element-gathered trace), SH[npv,nc,ne].
 * Outputs: AE[ncu,ndf,ncu,ndf,ne], FE[ncu,ndf,ne], DUDG[npv,nc,ne], DUDG_DUH[npv,nc,ncu,ndf,ne]
 *          (ndf = npf*nfe), status[ne] (may be NULL).
 * Supported (nd, porder): 2D 1..4, 3D 1..2; returns -3 otherwise. */
int hdgx_elemental(const hdgx_master *master, const hdgx_app *app, int ne,
                   const double *dgnodes, const int *bf, const double *UDG, const double *UH,
                   const double *SH, double *AE, double *FE, double *DUDG, double *DUDG_DUH,
                   int *status, hdgx_stream_t stream);

/* Batched local (u,q) Schur complement on the reference MEX layouts (kernel/schur_uq.c):
 * M[npv,npv,ne] C[npv,npv,nd,ne] E[npv,ndf,nd,ne] BD[npv,ncu,npv,nc,ne] F[npv,ncu,ncu,ndf,ne]
 * GK[ncu,ndf,npv,nc,ne] H[ncu,ndf,ncu,ndf,ne] Rq[npv,ncu,nd,ne] Ru[npv,ncu,ne] Rh[ncu,ndf,ne]
 * -> DUDG[npv,nc,ne] DUDG_DUH[npv,nc,ncu,ndf,ne] AE[ncu,ndf,ncu,ndf,ne] FE[ncu,ndf,ne].
 * Inputs are read-only (the reference MEX overwrites M, C, E, BD, F, Rq, Ru in place). */
int hdgx_schur_uq(int nd, int npv, int ncu, int ndf, int ne,
                  const double *M, const double *C, const double *E, const double *BD,
                  const double *F, const double *GK, const double *H, const double *Rq,
                  const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                  double *AE, double *FE, int *status, hdgx_stream_t stream);

/* Batched u-only Schur complement (kernel/schur_u.c): BD[npv,ncu,npv,nc,ne] (only the
 * first ncu component columns are read), F, GK[ncu,ndf,npv,nc,ne], H, Ru, Rh ->
 * DUDG[npv,nc,ne], DUDG_DUH[npv,nc,ncu,ndf,ne] (components >= ncu set to 0), AE, FE. */
int hdgx_schur_u(int npv, int ncu, int nc, int ndf, int ne,
                 const double *BD, const double *F, const double *GK, const double *H,
                 const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                 double *AE, double *FE, int *status, hdgx_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* HDGX_H */
