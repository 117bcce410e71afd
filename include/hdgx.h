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
 * 3 boundary type outside the app's fbou family) and counted in the return value of hdgx_status_count.
 *
 * Reference call surface each entry point replaces (paths relative to the reference tree):
 *   hdgx_elemental   kernel/hdg_elemental.m:1   [AE,FE,DUDG,DUDG_DUH] = hdg_elemental(master,app,dgnodes,bf,UDG,UH,SH)
 *   hdgx_elemental_host   kernel/hdg_elemental.m:1   the same call on host arrays (copies overlapped)
 *   hdgx_schur_uq    kernel/schur_uq.c:193      [DUDG,DUDG_DUH,AE,FE] = schur_uq(M,C,E,BD,F,GK,H,Rq,Ru,Rh)
 *   hdgx_schur_u     kernel/schur_u.c:82        [DUDG,DUDG_DUH,AE,FE] = schur_u(BD,F,GK,H,Ru,Rh)
 *   hdgx_getq        kernel/getq.m:1            QDG = getq(master,mesh,UDG,UH,SH,fc_q)
 *   hdgx_residual    kernel/cuda_residual.m:1   Ru = cuda_residual(...): Ru at q = getq(u, uh)
 *   hdgx_schur_uq_adjoint  kernel/schur_uq_adjoint.c:300  [DUDG,DUDG_DUH,AE,FE] = schur_uq_adjoint(M,C,E,BD,F,GK,H,Rq,Ru,Rh)
 *   hdgx_schur_u_adjoint   kernel/schur_u_adjoint.c:145   [DUDG,DUDG_DUH,AE,FE] = schur_u_adjoint(BD,F,GK,H,Ru,Rh)
 *   hdgx_globalassembly   kernel/globalassembly.m:1  [Hg,Rg] = globalassembly(mesh,AE,FE)
 *   hdgx_matvec           kernel/matvec.m:1          Xg = matvec(mesh,Hg,Rg)
 *   hdgx_bilu0_factor     kernel/computeBILU0.m:1    Mg = computeBILU0(mesh,Hg)
 *   hdgx_bilu0_apply      kernel/applyBILU0.m:1      v  = applyBILU0(mesh,Mg,x)
 *   hdgx_gmres_bilu0      kernel/gmres_bilu0.m:1     [x,flags,iter,rev] = gmres_bilu0(mesh,M,A,b,x,restart,tol,maxit)
 *   hdgx_gmres_bilu0_mixed kernel/gmres_bilu0.m:1    the same with the factors M stored in FP32
 *   hdgx_backsub          kernel/hdg_solve.m:119-121 DUDGT = DUDG + mapContractK(DUDG_DUH, DUH(elcon))
 *   hdgx_gather_uh        kernel/hdg_assemble.m:34   uh = reshape(UH(:,elcon),[ncu npf*nfe ne])
 *   hdgx_solve            kernel/hdg_solve.m:1       [UDG,UH] = hdg_solve(master,mesh,app,UDG,UH,SH)
 *   hdgx_arraymul         kernel/arraymul.c:11       C = arraymul(A,B)
 *   hdgx_dense_block_system kernel/mkDenseBlockSystem.m:9  [K,F] = mkDenseBlockSystem(AE,FE,f,t2f,elcon)
 *   hdgx_dense_matvec     kernel/gmres.m:40-44       d = x + arraymul(K, gather(x, f2f))
 *   hdgx_gmres_dense      kernel/gmres.m:1           [x,flags,iter,rev] = gmres(K,F,f2f,x,restart,tol,maxit)
 */
#ifndef HDGX_H
#define HDGX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st *hdgx_stream_t;   /* a cudaStream_t; NULL = legacy default stream */
typedef struct hdgx_combiner hdgx_combiner;  /* shared elemental launches of concurrent solves */

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
    int getdqdg;            /* 1: DUDG/DUDG_DUH carry all nc components (reference default); 0: the u
                               components only, q is recovered with hdgx_getq (hdg_solve.m:129-132) */
    double fc_q, fc_u;      /* fc_u: time-derivative coefficient of a DIRK stage (tdep = 1) */
    int tdep;               /* 1: time-dependent residual of kernel/volint.m:180-221 (dtcoef = 1, no
                               axisymmetry): source SH_u - fc_u u, Jacobian -fc_u on the u components */
    double param[8];        /* [gam, epslm, Re, Pr, Minf, tau]; Re = +inf gives Euler */
    int nbnd;               /* number of boundary indices (bf = -1..-nbnd) */
    int bcm[HDGX_MAX_BND];  /* fbou type per boundary index (the case labels of the family's fbou.m) */
    double bcs[HDGX_MAX_BND * 5];  /* boundary state per index, row-major [nbnd][ncu] */
    int fbou;               /* boundary-flux family, the app's physics folder (faceint.m:171-268 calls
                               app.fbou of application/FM/<physics>):
                               0 ns    (ns/fbou.m, fbou3d.m): 1 far field (Roe matrices of getan.m),
                                       2 adiabatic wall, 3 isothermal wall, 4 prescribed pressure,
                                       5 periodic (fhat), 6 Dirichlet uh - uinf;
                               1 euler (euler/fbou.m): 1 far field (local Lax-Friedrichs scalars of
                                       euler/getan.m), 2 slip wall, 3 and 4 prescribed pressure,
                                       5 density and energy extrapolated, 6 Dirichlet as for ns.
                               Other types give element status 3. */
} hdgx_app;

/* Library identity and error strings. */
int hdgx_version(void);

/* How host threads wait for the GPU where a solve reads a scalar back (each GMRES iteration's
 * residual, |F| after each assembly, the MDF block norms): 0 (default) as CUDA does, the thread
 * spinning until the copy completes; 1 the thread sleeps on a blocking-synchronisation event first
 * (taken from a per-device pool the library keeps).  Mode 1 is for processes that run many solves
 * at once, one host thread each (a serving loop): spinning threads then occupy as many cores and
 * slow each other down.  Process-wide; no counterpart in the reference.  -1 for another mode. */
int hdgx_set_host_wait(int mode);
int hdgx_get_host_wait(void);
const char *hdgx_status_str(int code);

/* Number of nonzero entries of a device status[n] array (synchronises the stream). */
int hdgx_status_count(const int *status, int n, hdgx_stream_t stream);

/* Fused FP64 elemental kernel: volume + face integrals + local (u,q) Schur elimination.
 * Inputs : dgnodes[npv,nd,ne], bf[nfe,ne] (int32), UDG[npv,nc,ne], UH[ncu,npf*nfe,ne]
 *          (element-gathered trace), SH[npv,nc,ne].
 * Outputs: AE[ncu,ndf,ncu,ndf,ne], FE[ncu,ndf,ne], DUDG[npv,nco,ne], DUDG_DUH[npv,nco,ncu,ndf,ne]
 *          (ndf = npf*nfe; nco = nc, or ncu when app->getdqdg = 0: the u rows only, as
 *          hdg_elemental.m:20-26 sizes them), status[ne] (may be NULL).
 * Supported (nd, porder): 2D 1..4, 3D 1..2, with the drivers' quadrature order pgauss = 2 porder
 * (mkmaster(mesh, 2*porder)); returns -3, before anything is launched, for any other (nd, porder)
 * and for a master whose npv, npf, ngv or ngf differ from that element's (e.g. one built by
 * mkmaster(mesh, pgauss) with pgauss != 2 porder).  hdgx_elemental_mixed, _host, _buckets,
 * hdgx_getq, hdgx_residual and hdgx_solve apply the same check. */
int hdgx_elemental(const hdgx_master *master, const hdgx_app *app, int ne,
                   const double *dgnodes, const int *bf, const double *UDG, const double *UH,
                   const double *SH, double *AE, double *FE, double *DUDG, double *DUDG_DUH,
                   int *status, hdgx_stream_t stream);

/* Mixed-precision form of hdgx_elemental (same arguments and layouts; replaces the same
 * kernel/hdg_elemental.m call).  The local elimination of the Jacobian columns runs in FP32
 * and the local residual solve is refined against the FP64 local matrix, so FE and DUDG
 * are FP64-accurate residual quantities while AE and DUDG_DUH carry FP32-level error (a
 * Jacobian error: Newton converges to the same FP64 solution).  The Schur product of the Jacobian
 * columns, dlu = SD^-1 (B Mi E - F) (schur_primal.m:118), runs on the tensor cores (tcgen05,
 * kind::tf32, as three TF32 products of the split operands: FP32-level accuracy) for every element
 * shape but 2D p = 4 (no room for its operands next to the shared-memory plan; it keeps the FP32
 * elimination of all columns).  status 4: refinement failed, or a tensor-core wait ran out. */
int hdgx_elemental_mixed(const hdgx_master *master, const hdgx_app *app, int ne,
                         const double *dgnodes, const int *bf, const double *UDG, const double *UH,
                         const double *SH, double *AE, double *FE, double *DUDG, double *DUDG_DUH,
                         int *status, hdgx_stream_t stream);

/* hdgx_elemental (mixed = 0) or hdgx_elemental_mixed (mixed = 1) on HOST arrays, for callers
 * whose element data lives in host memory as the reference's does (kernel/hdg_elemental.m:1 is
 * called with host MATLAB arrays).  master stays a DEVICE table set; dgnodes, bf, UDG, UH, SH,
 * AE, FE, DUDG, DUDG_DUH and status (may be NULL) are HOST pointers in the layouts of
 * hdgx_elemental.  Page-locked (pinned) host memory gives full copy bandwidth and overlap;
 * pageable memory works, with the driver staging its copies.  The elements go through two
 * device staging sets of `chunk` elements (0: ne / 16, at least 1024) taken from the library's
 * device pool, and chunk c's upload, chunk c-1's kernel and chunk c-2's download run at the
 * same time, so the call costs about the largest of the three totals.  The results are
 * bitwise those of the device-array call.  The call returns when the outputs are in host
 * memory (it synchronises `stream`). */
int hdgx_elemental_host(const hdgx_master *master, const hdgx_app *app, int ne,
                        const double *dgnodes, const int *bf, const double *UDG, const double *UH,
                        const double *SH, double *AE, double *FE, double *DUDG, double *DUDG_DUH,
                        int *status, int mixed, int chunk, hdgx_stream_t stream);

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

/* One elemental evaluation over several buckets of elements (e.g. one per polynomial degree
 * of a mixed-degree mesh), each with its own master, app and arrays (layouts as
 * hdgx_elemental).  The buckets' kernels run concurrently on side streams forked from and
 * joined back into `stream`, so the whole call is one node sequence of a CUDA graph when the
 * caller captures it (make one uncaptured call first: it creates the side streams and sets
 * the kernels' shared-memory limits).  grid = CTAs of the bucket's launch (0: one wave of
 * resident CTAs on the whole GPU).  mixed != 0 selects the mixed-precision kernel.  No
 * counterpart in the reference, which has no mixed-degree meshes (kernel/hdg_elemental.m is
 * called per uniform mesh). */
typedef struct {
    const hdgx_master *master;
    const hdgx_app *app;
    int ne;
    const double *dgnodes;
    const int *bf;
    const double *UDG, *UH, *SH;
    double *AE, *FE, *DUDG, *DUDG_DUH;
    int *status;
    int grid;
} hdgx_elem_bucket;

int hdgx_elemental_buckets(int nb, const hdgx_elem_bucket *buckets, int mixed, hdgx_stream_t stream);

/* One FP64 elemental launch over the elements of several buckets of ONE element shape (the same
 * nd and porder, masters of the same table sizes; the master tables are read from buckets[0]) and
 * one kind of physics (all viscous, Re finite, or all inviscid): each bucket keeps its own app
 * (constants, boundary data, getdqdg), arrays and status, and its results are bitwise those of
 * hdgx_elemental on that bucket alone.  For callers that evaluate many small independent meshes
 * at once (a serving loop), where one launch fills the GPU that one bucket alone would not.
 * At most hdgx_elemental_shared_max() buckets (-5 beyond); -2 when the buckets' shapes or physics
 * kinds differ; the buckets' `grid` fields are ignored, `grid` = CTAs of the launch (0: one wave
 * of resident CTAs).  The bucket table travels as the kernel's parameter: nothing is allocated or
 * copied, and the call can be captured in a CUDA graph.  No counterpart in the reference, which
 * assembles one mesh per call (kernel/hdg_assemble.m). */
int hdgx_elemental_shared(int nb, const hdgx_elem_bucket *buckets, int grid, hdgx_stream_t stream);
int hdgx_elemental_shared_max(void);

/* Batched u-only Schur complement (kernel/schur_u.c): BD[npv,ncu,npv,nc,ne] (only the
 * first ncu component columns are read), F, GK[ncu,ndf,npv,nc,ne], H, Ru, Rh ->
 * DUDG[npv,nc,ne], DUDG_DUH[npv,nc,ncu,ndf,ne] (components >= ncu set to 0), AE, FE. */
int hdgx_schur_u(int npv, int ncu, int nc, int ndf, int ne,
                 const double *BD, const double *F, const double *GK, const double *H,
                 const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                 double *AE, double *FE, int *status, hdgx_stream_t stream);

/* getq.m: the gradient unknowns q that zero the local q equation for the given u and trace,
 * QDG = SH_q/fc_q + inv(fc_q M) (C u - E uh) per element (volint.m:57-60 / faceint.m:49-51 with
 * Rq = 0), computed by the first phases of the elemental kernel.  Arguments as hdgx_elemental
 * (UH element-gathered; app supplies nd, ncu, nc, fc_q != 0); SH may be NULL (no source, as
 * getq(...,[],fc_q)); QDG[npv, ncu*nd, ne]; status 1 for a singular mass matrix. */
int hdgx_getq(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
              const int *bf, const double *UDG, const double *UH, const double *SH, double *QDG,
              int *status, hdgx_stream_t stream);

/* cuda_residual.m: the residual-only evaluation used by explicit time stepping.  q is first
 * recovered from u and the trace (as hdgx_getq), then the element u residual Ru[npv,ncu,ne] is
 * evaluated at that q: volume flux and (app->tdep = 1) time source terms plus the face fhat /
 * fbou terms, the Ru of volint.m / faceint.m, with no Jacobian and no local solve.  Arguments as
 * hdgx_getq; status as hdgx_elemental. */
int hdgx_residual(const hdgx_master *master, const hdgx_app *app, int ne, const double *dgnodes,
                  const int *bf, const double *UDG, const double *UH, const double *SH, double *Ru,
                  int *status, hdgx_stream_t stream);

/* Adjoint (transposed) local Schur complements, the reference's schur_uq_adjoint.c and
 * schur_u_adjoint.c on the same layouts and arguments as hdgx_schur_uq / hdgx_schur_u: the
 * local system is solved with D^T (plus, for the (u,q) form, the transposed B Mi C coupling),
 * the trace coupling uses GK^T, F^T and H^T.  The u form writes, as that MEX does, du into the
 * first npv*ncu entries of each element's DUDG slab and dlu (column-major [npv*ncu, ncu*ndf])
 * into the first npv*ncu*ncu*ndf entries of its DUDG_DUH slab, and zeros elsewhere.  Inputs are
 * not modified (the reference MEX overwrites M, Rq and Ru).  status as hdgx_schur_uq. */
int hdgx_schur_uq_adjoint(int nd, int npv, int ncu, int ndf, int ne,
                          const double *M, const double *C, const double *E, const double *BD,
                          const double *F, const double *GK, const double *H, const double *Rq,
                          const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                          double *AE, double *FE, int *status, hdgx_stream_t stream);
int hdgx_schur_u_adjoint(int npv, int ncu, int nc, int ndf, int ne,
                         const double *BD, const double *F, const double *GK, const double *H,
                         const double *Ru, const double *Rh, double *DUDG, double *DUDG_DUH,
                         double *AE, double *FE, int *status, hdgx_stream_t stream);

/* ---------------------------------------------------------------- trace system */

/* Face-row block-CSR pattern of the condensed system (mesh.cbsr_* of block_crs.m) and the
 * elimination order used by BILU(0).  Block size bs = ncu*npf.  Device pointers except
 * color_ptr (host).  Rows are eliminated colour by colour; rows of one colour share no
 * block, pos[row] is the row's position in the elimination order. */
typedef struct {
    int nf, bs;
    long long nnzb;
    const long long *rowpts;   /* [nf+1] block offsets, 0-based */
    const int *colind;         /* [nnzb] 1-based block column, diagonal first in each row */
    int ncolors;
    const int *color_ptr;      /* HOST [ncolors+1] offsets into color_rows */
    const int *color_rows;     /* [nf] 0-based rows grouped by colour */
    const int *pos;            /* [nf] elimination position of each row */
    int *sched;                /* ncolors == 0 only: device workspace of 4 + nf ints, zeroed once by
                                  the caller.  Rows are then eliminated one after another in the
                                  order color_rows (e.g. the MDF order of computeMDFordering.m), with
                                  flag-synchronised (not level-synchronised) parallel sweeps.  Every
                                  wait for a row's flag is bounded: sched[3] is the poll limit (0, as
                                  zeroed: 2^22 polls); a wait that runs out sets sched[2], the row goes
                                  on, and hdgx_gmres_bilu0 returns -14 (and clears sched[2]). */
    const int *sweep_plan;     /* optional (NULL: one launch per colour in hdgx_bilu0_apply): the
                                  colours as levels of a sequential order, for single-launch sweeps.
                                  Device ints: [ncolors+1] colour offsets, then for every slot q of
                                  color_rows a record of 2 + 4*sweep_maxd ints: row i, its diagonal
                                  block rowpts[i], sweep_maxd (block k, column j) pairs of the
                                  neighbours eliminated before i, sweep_maxd pairs of those eliminated
                                  after i (k = -1 pads each list; 0-based). */
    int sweep_maxd;            /* 4 (triangles) or 6 (tetrahedra); other values disable the plan */
} hdgx_bsr;

/* Element -> block gather map for hdgx_globalassembly (device pointers):
 * blk_e[2*nnzb] elements (or -1) contributing to block k, blk_ab[2*nnzb] their local
 * faces (a | b << 8), blk_row[nnzb] 0-based block row; face_e[2*nf], face_a[2*nf] the
 * (element, local face) pairs of every face (element -1 when absent). */
typedef struct {
    const int *blk_e, *blk_ab, *blk_row;
    const int *face_e, *face_a;
} hdgx_assembly_map;

/* UHe[ncu, ndf, ne] = UH[:, elcon] (kernel/hdg_assemble.m:34).  elcon [ndf, ne] 1-based. */
int hdgx_gather_uh(int ncu, int ndf, int ne, const int *elcon, const double *UH, double *UHe,
                   hdgx_stream_t stream);

/* Hg[bs,bs,nnzb], Rg[bs,nf] from AE[ncu,ndf,ncu,ndf,ne], FE[ncu,ndf,ne]
 * (kernel/globalassembly.m:21-37; dofs placed by elcon as kernel/hdg_assemble.m:77-87). */
int hdgx_globalassembly(const hdgx_bsr *A, const hdgx_assembly_map *map, int ncu, int npf, int nfe,
                        const int *elcon, const double *AE, const double *FE, double *Hg, double *Rg,
                        hdgx_stream_t stream);

/* C[k] = || inv(H_ii) H_ik ||_F for every block k of row i (kernel/computeMDFordering.m:14-20). */
int hdgx_block_norms(const hdgx_bsr *A, const double *Hg, double *C, hdgx_stream_t stream);

/* Minimum-discarded-fill order (kernel/computeMDFordering.m:21-161) from the block norms C
 * (HOST arrays rowpts[nf+1], colind[nnzb], C[nnzb]); o2u[l] = row pivoted at step l, u2o its
 * inverse (0-based, HOST).  Ties go to the lowest row, as MATLAB's min does. */
int hdgx_mdf_ordering(int nf, const long long *rowpts, const int *colind, const double *C, int *o2u, int *u2o);

/* Level schedule of the sequential elimination order o2u (u2o its inverse): level(i) = 1 + the
 * largest level of the neighbours eliminated before i, so that eliminating level by level gives
 * the factors of the sequential order (computeBILU0.m in the order of computeMDFordering.m).
 * HOST arrays; rowpts [nf+1] 0-based, colind 1-based with the diagonal first; writes level_ptr
 * [nlev + 1] (room for nf + 1) and rows [nf] (grouped by level, by position inside a level) and
 * returns nlev, or -1 for bad arguments. */
int hdgx_level_schedule(int nf, const long long *rowpts, const int *colind, const int *o2u, const int *u2o,
                        int *level_ptr, int *rows);

/* The single-launch sweep plan of a level schedule (hdgx_bsr.sweep_plan), HOST arrays: *maxd = 4
 * or 6 (0 when a row has more than 6 off-diagonal blocks: no plan, nothing written), and plan
 * [nlev + 1 + nf * (2 + 4 maxd)] = the level offsets, then per slot q of rows the record (row i,
 * its diagonal block rowpts[i], maxd (block, column) pairs of the neighbours with pos < pos[i],
 * maxd pairs of those after it), -1 padded, 0-based, in CSR order.  Call with plan = NULL first
 * to learn maxd.  0, or -1 for bad arguments. */
int hdgx_sweep_plan(int nf, const long long *rowpts, const int *colind, int nlev, const int *level_ptr,
                    const int *rows, const int *pos, int *plan, int *maxd);

/* y = Hg x (kernel/matvec.m). */
int hdgx_matvec(const hdgx_bsr *A, const double *Hg, const double *x, double *y, hdgx_stream_t stream);

/* In-place block ILU(0) of Mg (= Hg on entry) in the colour order of A
 * (kernel/computeBILU0.m); diagonal blocks are stored inverted.  status[nf] (optional) is
 * set to 1 for rows whose pivot block is singular. */
int hdgx_bilu0_factor(const hdgx_bsr *A, double *Mg, int *status, hdgx_stream_t stream);

/* v = (L U)^{-1} x (kernel/applyBILU0.m); work[bs*nf] scratch. */
int hdgx_bilu0_apply(const hdgx_bsr *A, const double *Mg, const double *x, double *v, double *work,
                     hdgx_stream_t stream);

/* Bytes of device workspace hdgx_gmres_bilu0 uses for a given restart length. */
size_t hdgx_gmres_workspace_bytes(const hdgx_bsr *A, int restart);

/* Left-preconditioned restarted GMRES with modified Gram-Schmidt (kernel/gmres_bilu0.m):
 * x (in: initial guess, out: solution) [bs,nf]; stops when |P^{-1}(b - A x)| <= tol |P^{-1} b|
 * or after maxit iterations.  iters, flag (0 converged, 1 maxit, 3 breakdown), relres and
 * history[maxit] (optional) are host outputs.  workspace (device, hdgx_gmres_workspace_bytes)
 * may be NULL, in which case it is taken from the stream-ordered allocator. */
int hdgx_gmres_bilu0(const hdgx_bsr *A, const double *Hg, const double *Mg, const double *b, double *x,
                     int restart, double tol, int maxit, int *iters, int *flag, double *relres,
                     double *history, void *workspace, hdgx_stream_t stream);

/* Mg32[bs,bs,nnzb] = (float) Mg: the BILU(0) factors of hdgx_bilu0_factor stored in FP32 for
 * hdgx_gmres_bilu0_mixed.  No counterpart in the reference (its factors are FP64 MATLAB arrays,
 * kernel/computeBILU0.m); part of the mixed-precision Newton step. */
int hdgx_bilu0_to_f32(const hdgx_bsr *A, const double *Mg, float *Mg32, hdgx_stream_t stream);

/* hdgx_gmres_bilu0 (kernel/gmres_bilu0.m) with the preconditioner's factors read in FP32 (Mg32 of
 * hdgx_bilu0_to_f32); the sweeps accumulate in FP64 and the matvec with Hg, the Arnoldi
 * orthogonalisation, the Givens rotations and the residual stay FP64.  The preconditioner is then
 * a slightly different fixed operator, so the converged solution is that of the FP64 system to
 * the same tolerance (the iteration count may differ by a few).  Offered for the single-launch
 * level sweeps of A->sweep_plan; returns -2 otherwise.  Same arguments as hdgx_gmres_bilu0. */
int hdgx_gmres_bilu0_mixed(const hdgx_bsr *A, const double *Hg, const float *Mg32, const double *b, double *x,
                           int restart, double tol, int maxit, int *iters, int *flag, double *relres, double *history,
                           void *workspace, hdgx_stream_t stream);

/* Allocation-free variant of hdgx_gmres_bilu0 (same arguments minus the workspace; the same
 * solver code and kernels, so the same results bit for bit, for every ordering hdgx_bsr
 * describes: colours, single-launch level sweeps, or flag-scheduled sweeps with the caller's
 * `sched` array).  No counterpart in the reference: it exists for callers that may not
 * allocate device or pinned host memory at solve time (a plugin host whose allocator owns
 * every byte, a latency-critical serving loop, memory already reserved in arenas).  Its
 * scratch is one 16 MiB array compiled into the library, held by every GPU that loads the
 * library until exit; systems needing more (hdgx_gmres_workspace_bytes > 16 MiB, roughly
 * N > 88,000 unknowns at restart 20) are rejected with status -5 before any work is queued.
 * All calls share that array and it keeps the last call's contents (each call clears what
 * it uses first), so calls that overlap on the GPU race.  With CUDA's lazy module loading
 * the first call on a device loads the module and with it the array, and resolves the
 * array's address: make that first call (a warm-up solve) before any latency-critical region
 * and before any stream capture. */
int hdgx_gmres_bilu0_noalloc(const hdgx_bsr *A, const double *Hg, const double *Mg, const double *b,
                             double *x, int restart, double tol, int maxit, int *iters, int *flag,
                             double *relres, double *history, hdgx_stream_t stream);

/* DUDGT[npv,nc,ne] = DUDG + DUDG_DUH * DUH(:, elcon(:,e)) (kernel/hdg_solve.m:119-121);
 * DUH[ncu, nsiz]. */
int hdgx_backsub(int npv, int nc, int ncu, int ndf, int ne, const int *elcon, const double *DUDG,
                 const double *DUDG_DUH, const double *DUH, double *DUDGT, hdgx_stream_t stream);

/* ---------------------------------------------------------------- Newton solve */

#define HDGX_SOLVE_MAXIT 16   /* hdg_solve.m:108: at most 16 Newton steps */

/* The mesh of hdgx_solve: per-element arrays on the DEVICE, connectivity on the HOST. */
typedef struct {
    int ne, nf;
    const double *dgnodes;     /* device [npv, nd, ne] */
    const int *bf;             /* device [nfe, ne] (bf < 0: boundary index -bf) */
    const int *elcon;          /* device [npf*nfe, ne], 1-based trace nodes */
    const int *t2f;            /* HOST [ne, nfe] column-major, 1-based faces */
    const long long *rowpts;   /* HOST [nf+1] block-CSR offsets (mesh.cbsr_rowpts) */
    const int *colind;         /* HOST [nnzb] 1-based, diagonal first (mesh.cbsr_colind) */
} hdgx_mesh;

typedef struct {
    int ordering;              /* 0: minimum-discarded-fill (computeMDFordering.m), 1: greedy multicolour */
    int mixed;                 /* 1: mixed-precision elemental kernel */
    int restart;               /* GMRES restart (20) */
    int maxiter;               /* Newton steps (<= HDGX_SOLVE_MAXIT) */
    double tol;                /* Newton stop: |F| / |F0| <= tol (hdg_solve.m:107 uses 1e-9) */
    double gmres_tol;          /* BILU(0)-GMRES relative tolerance */
    int gmres_maxit;
} hdgx_solve_opts;

typedef struct {
    int iterations, converged, ncolors;
    double residuals[HDGX_SOLVE_MAXIT + 1];   /* |F| before the first and after every Newton step */
    double alphas[HDGX_SOLVE_MAXIT];          /* line-search step lengths */
    int gmres_iters[HDGX_SOLVE_MAXIT];
    double gmres_relres[HDGX_SOLVE_MAXIT];
    int graph_assemblies;     /* assemblies replayed from the CUDA graph of the assembly chain */
} hdgx_solve_report;

/* Newton solve of kernel/hdg_solve.m:84-176 on the device: assembly (hdg_assemble.m), BILU(0)-
 * GMRES with x0 = 0 in place of K\F, back-substitution (hdg_solve.m:119-121) and the halving
 * line search (hdg_solve.m:144-163), until |F| / |F0| <= tol or maxiter steps.  UDG [npv,nc,ne]
 * and UH [ncu, nf*npf] (device) are updated in place; SH [npv,nc,ne] (device) is the source,
 * whose q part is taken as zero (hdg_solve.m:62-63, no wave formulation).  app->getdqdg must be
 * 1 (returns -2 otherwise; the Python composition also runs getdqdg = 0).  Workspace comes from a private stream-ordered memory pool of the library (one per device) and
 * is released into it before returning; the pool keeps up to 8 GiB of freed memory for later
 * calls.  The call synchronises the stream (it reads residual norms on the host).  On a
 * non-blocking stream the assembly chain (trace gather, elemental kernel, block-CSR gather, |F|)
 * is captured into a CUDA graph after the first assembly and replayed for the others. */
int hdgx_solve(const hdgx_master *master, const hdgx_app *app, const hdgx_mesh *mesh, double *UDG, double *UH,
               const double *SH, const hdgx_solve_opts *opts, hdgx_solve_report *report, hdgx_stream_t stream);

/* Shared elemental launches across concurrent solves (serving).  A combiner collects the
 * assemblies of the hdgx_solve_combined calls that run at the same time (each on its own host
 * thread and stream) and evaluates each group of equal master tables and one physics kind
 * (viscous or not) as one hdgx_elemental_shared launch on one of the combiner's streams (a group
 * of one as its own launch on its own stream); every solve's results are bitwise those of
 * hdgx_solve.  The first submission of a batch waits until every attached solve of its group has
 * submitted or window_us microseconds have passed (0: it takes what is queued at once).  One
 * combiner serves one device (the current device at creation; -2 for solves on another).
 * hdgx_solve_combined: arguments of hdgx_solve plus the combiner; FP64 only (opts->mixed = 1
 * returns -2); the call reads the master tables once to key its group; its assembly chain is not
 * replayed from a graph (the batching synchronises on the host).  Destroy only when no solve is
 * attached (-1 otherwise).  No counterpart in the reference (kernel/hdg_solve.m solves one
 * problem per call). */
int hdgx_combiner_create(int window_us, hdgx_combiner **out);
int hdgx_combiner_destroy(hdgx_combiner *combiner);
int hdgx_combiner_stats(const hdgx_combiner *combiner, long long *batches, long long *launches,
                        long long *submissions);
/* Host seconds all solves spent keying their group (reading the master tables) and in submissions
 * (queueing, waiting for a batch, launching). */
int hdgx_combiner_times(const hdgx_combiner *combiner, double *key_s, double *submit_s);
int hdgx_solve_combined(const hdgx_master *master, const hdgx_app *app, const hdgx_mesh *mesh, double *UDG,
                        double *UH, const double *SH, const hdgx_solve_opts *opts, hdgx_solve_report *report,
                        hdgx_combiner *combiner, hdgx_stream_t stream);

/* ------------------------------------------------- dense face-block path (app.denseblock = 1) */

/* Batched product (kernel/arraymul.c:11-96).  A is rowsA x colsA x ndim3 (ndim3 = 1 for a 2-D
 * A).  When B is 2-D (ndimB == 2) with colsB == ndim3: C(:, i) = A(:, :, i) B(:, i), C is
 * rowsA x ndim3 (batched GEMV).  Otherwise C(:, :, i) = A(:, :, i) B(:, :, i) with B holding
 * ndim3 rowsB x colsB matrices and C rowsA x colsB x ndim3.  colsA != rowsB -> -1 (the MEX's
 * "Number of columns of A must be equal to numbers of rows B"). */
int hdgx_arraymul(int rowsA, int colsA, int ndim3, int rowsB, int colsB, int ndimB, const double *A,
                  const double *B, double *C, hdgx_stream_t stream);

/* Block-Jacobi-scaled face blocks (kernel/mkDenseBlockSystem.m:9-95) from the block-CSR
 * condensed system: for face i, K(:, :, k, i) = inv(D_i) H(i, f2f(k+1, i)) (zero block where
 * f2f(k+1, i) == 0) and F(:, i) = inv(D_i) Rg(:, i), D_i the diagonal block.  f2f[nbf, nf]
 * (mesh/mkmesh/mkf2f.m, 1-based, 0 = none; row 0 is the face itself).  K[bs, bs*(nbf-1), nf],
 * F[bs, nf].  status[nf] (optional): k+1 when D_i's pivot k is zero or not finite. */
int hdgx_dense_block_system(const hdgx_bsr *A, const double *Hg, const double *Rg, int nbf, const int *f2f,
                            double *K, double *F, int *status, hdgx_stream_t stream);

/* y = x + K gather(x, f2f) (kernel/gmres.m:40-44): y(:, i) = x(:, i) + sum_k K(:, :, k, i) x(:, f2f(k+1, i)). */
int hdgx_dense_matvec(int nb, int nf, int nbf, const double *K, const int *f2f, const double *x, double *y,
                      hdgx_stream_t stream);

/* Bytes of device workspace hdgx_gmres_dense uses for a given restart length. */
size_t hdgx_gmres_dense_workspace_bytes(int nb, int nf, int restart);

/* Unpreconditioned restarted GMRES on (I + K gather) x = b with classical Gram-Schmidt
 * (kernel/gmres.m:1-111).  x (in: initial guess, out: solution) [nb, nf].  Stops when the
 * least-squares residual |b - A x| <= tol |b| or after maxit iterations, counted as gmres.m
 * counts them (each restart's residual evaluation is one).  iters, flag (0 converged,
 * 1 maxit, 3 breakdown to a non-finite value), relres and history[maxit] (optional, relative
 * residuals) are host outputs.  workspace (device, hdgx_gmres_dense_workspace_bytes) may be
 * NULL, in which case it is taken from the stream-ordered allocator. */
int hdgx_gmres_dense(int nb, int nf, int nbf, const double *K, const int *f2f, const double *b, double *x,
                     int restart, double tol, int maxit, int *iters, int *flag, double *relres, double *history,
                     void *workspace, hdgx_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* HDGX_H */
