/*
 * oracle_elemental.c -- FP64 CPU restatement of the reference's HDG elemental path.
 *
 * TEST INFRASTRUCTURE ONLY: this file is the parity oracle and the CPU baseline.  Only
 * tests/, __graft_entry__.smoke() and bench.py's CPU baseline leg may load it.  The product
 * (hdg_b200/libhdgx.so) never calls it.
 *
 * One element at a time, the same operations as the reference's vectorised MATLAB:
 *   volgeom  kernel/volgeom.m:18-61      pg, Jg = dx/dxi, jac = det Jg, Xx = adj(Jg)
 *   volint   kernel/volint.m:25-60,241-263  M, C, Rq, Ru, BD (flux source = 0); time-dependent
 *            problems (tdep = 1, volint.m:180-221 with dtcoef = 1, no axisymmetry) add the
 *            source s = SH_u - fc_u u and its Jacobian -fc_u on the u components
 *   facegeom kernel/facegeom.m:20-52     pg, nlg, jac at face Gauss points
 *   faceint  kernel/faceint.m:29-61,171-360  E, Rq -= E.UH, fhat, fbou, Ru, BD, F, Rh, GK, H
 *   schur    kernel/schur_primal.m:52-150 (schur_uq2): Mi = inv(M), SD = D + B Mi C,
 *            du = SD\(Ru - B Mi Rq), dlu = SD\(B Mi E - F), dq, dlq, FE = Rh - GK DUDG,
 *            AE = H + GK DUDG_DUH
 *            kernel/schur_primal.m:13-49 (schur_u2) when localsolve == 0.
 * Array layouts are MATLAB column-major with the element index last, exactly as
 * kernel/hdg_elemental.m:29-32 returns them.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>
#include "oracle_physics.h"

typedef struct {
    int nd, npv, npf, nfe, ngv, ngf;
    const double *shapvt;          /* [ngv, npv, nd+1] */
    const double *shapvg;          /* [npv, ngv, nd+1] */
    const double *shapmv;          /* [ngv, npv, nd+1] (geometry) */
    const double *shapft;          /* [ngf, npf, nd] */
    const double *shapfg;          /* [npf, ngf, nd] */
    const double *shapmf;          /* [ngf, npf, nd] (geometry) */
    const int *perm;               /* [npf, nfe], 1-based */
} orc_master;

typedef struct {
    int nd, ncu, nc;
    int localsolve;                /* 1: (u,q) form; 0: u only */
    double fc_q;
    const double *param;           /* 6 entries */
    int nbnd;                      /* number of boundary indices */
    const int *bcm;                /* [nbnd] fbou type per boundary index */
    const double *bcs;             /* [nbnd, ncu] column-major */
    double fc_u;                   /* time-derivative coefficient (tdep = 1) */
    int tdep;                      /* 1: time-dependent source (volint.m:180-221) */
    int fbou_family;               /* 0: application/FM/ns/fbou.m, 1: application/FM/euler/fbou.m */
} orc_app;


/* Minimal element-parallel loop on pthreads (dynamic chunks of 8 elements).  The body is
 * a block executed for each element index with a thread-private counter `nbad`. */
typedef struct { int ne, next, nbad; pthread_mutex_t mu; void (*body)(void *, int, int *); void *ctx; } orc_pool;
static void *orc_worker(void *arg)
{
    orc_pool *p = arg; int local = 0;
    for (;;) {
        pthread_mutex_lock(&p->mu); int s = p->next; p->next += 8; pthread_mutex_unlock(&p->mu);
        if (s >= p->ne) break;
        int t = s + 8 < p->ne ? s + 8 : p->ne;
        for (int e = s; e < t; e++) p->body(p->ctx, e, &local);
    }
    pthread_mutex_lock(&p->mu); p->nbad += local; pthread_mutex_unlock(&p->mu);
    return NULL;
}
static int orc_run(int ne, int nthreads, void (*body)(void *, int, int *), void *ctx)
{
    orc_pool p; p.ne = ne; p.next = 0; p.nbad = 0; p.body = body; p.ctx = ctx;
    pthread_mutex_init(&p.mu, NULL);
    if (nthreads <= 1) { orc_worker(&p); return p.nbad; }
    pthread_t th[256]; if (nthreads > 256) nthreads = 256;
    for (int i = 0; i < nthreads; i++) pthread_create(&th[i], NULL, orc_worker, &p);
    for (int i = 0; i < nthreads; i++) pthread_join(th[i], NULL);
    return p.nbad;
}

#define IX2(i, j, n0) ((i) + (size_t)(n0) * (j))
#define IX3(i, j, k, n0, n1) ((i) + (size_t)(n0) * ((j) + (size_t)(n1) * (k)))

/* ---------------------------------------------------------------- dense LU */
/* In-place LU with partial pivoting of column-major A[n,n]; returns 0 or k+1 on a zero pivot. */
static int lu_factor(double *A, int n, int *piv)
{
    for (int k = 0; k < n; k++) {
        int p = k; double mx = fabs(A[IX2(k, k, n)]);
        for (int i = k + 1; i < n; i++) if (fabs(A[IX2(i, k, n)]) > mx) { mx = fabs(A[IX2(i, k, n)]); p = i; }
        piv[k] = p;
        if (mx == 0.0 || !isfinite(mx)) return k + 1;
        if (p != k) for (int j = 0; j < n; j++) { double t = A[IX2(k, j, n)]; A[IX2(k, j, n)] = A[IX2(p, j, n)]; A[IX2(p, j, n)] = t; }
        double inv = 1.0 / A[IX2(k, k, n)];
        for (int i = k + 1; i < n; i++) A[IX2(i, k, n)] *= inv;
        for (int j = k + 1; j < n; j++) {
            double akj = A[IX2(k, j, n)];
            if (akj != 0.0) for (int i = k + 1; i < n; i++) A[IX2(i, j, n)] -= A[IX2(i, k, n)] * akj;
        }
    }
    return 0;
}

static void lu_solve(const double *LU, int n, const int *piv, double *B, int nrhs)
{
    for (int r = 0; r < nrhs; r++) {
        double *b = B + (size_t)n * r;
        for (int k = 0; k < n; k++) if (piv[k] != k) { double t = b[k]; b[k] = b[piv[k]]; b[piv[k]] = t; }
        for (int k = 0; k < n; k++) { double bk = b[k]; for (int i = k + 1; i < n; i++) b[i] -= LU[IX2(i, k, n)] * bk; }
        for (int k = n - 1; k >= 0; k--) { b[k] /= LU[IX2(k, k, n)]; double bk = b[k]; for (int i = 0; i < k; i++) b[i] -= LU[IX2(i, k, n)] * bk; }
    }
}

/* C[m,n] (+)= A[m,k] B[k,n], all column-major with leading dims m,k,m. */
static void gemm(int m, int n, int k, const double *A, int lda, const double *B, int ldb, double *C, int ldc, double beta)
{
    for (int j = 0; j < n; j++) {
        for (int i = 0; i < m; i++) C[i + (size_t)ldc * j] *= beta;
        for (int l = 0; l < k; l++) {
            double b = B[l + (size_t)ldb * j];
            if (b == 0.0) continue;
            for (int i = 0; i < m; i++) C[i + (size_t)ldc * j] += A[i + (size_t)lda * l] * b;
        }
    }
}

/* ------------------------------------------------------------- one element */
typedef struct {
    /* outputs of volint+faceint for one element, reference layouts without the ne index */
    double *M, *C, *E, *BD, *F, *GK, *H, *Rq, *Ru, *Rh;
} orc_blocks;

static size_t blocks_doubles(const orc_master *ms, const orc_app *ap)
{
    int npv = ms->npv, nd = ms->nd, ndf = ms->npf * ms->nfe, ncu = ap->ncu, nc = ap->nc;
    return (size_t)npv * npv + (size_t)npv * npv * nd + (size_t)npv * ndf * nd
         + (size_t)npv * ncu * npv * nc + (size_t)npv * ncu * ncu * ndf + (size_t)ncu * ndf * npv * nc
         + (size_t)ncu * ndf * ncu * ndf + (size_t)npv * ncu * nd + (size_t)npv * ncu + (size_t)ncu * ndf;
}

static void blocks_carve(const orc_master *ms, const orc_app *ap, double *base, orc_blocks *b)
{
    int npv = ms->npv, nd = ms->nd, ndf = ms->npf * ms->nfe, ncu = ap->ncu, nc = ap->nc;
    double *p = base;
    b->M = p;  p += (size_t)npv * npv;
    b->C = p;  p += (size_t)npv * npv * nd;
    b->E = p;  p += (size_t)npv * ndf * nd;
    b->BD = p; p += (size_t)npv * ncu * npv * nc;
    b->F = p;  p += (size_t)npv * ncu * ncu * ndf;
    b->GK = p; p += (size_t)ncu * ndf * npv * nc;
    b->H = p;  p += (size_t)ncu * ndf * ncu * ndf;
    b->Rq = p; p += (size_t)npv * ncu * nd;
    b->Ru = p; p += (size_t)npv * ncu;
    b->Rh = p;
}

/* volint + faceint for one element.  dg[npv,nd], udg[npv,nc], uh[ncu,ndf], sh[npv,nc]. */
static int element_blocks(const orc_master *ms, const orc_app *ap, const double *dg, const int *bf,
                          const double *udg, const double *uh, const double *sh, orc_blocks *b)
{
    const int nd = ms->nd, npv = ms->npv, npf = ms->npf, nfe = ms->nfe, ngv = ms->ngv, ngf = ms->ngf;
    const int ncu = ap->ncu, nc = ap->nc, ndf = npf * nfe, nd1 = nd + 1;
    const double fc_q = ap->fc_q;
    int rc = 0;
    memset(b->M, 0, sizeof(double) * blocks_doubles(ms, ap));

    /* ---- volgeom (volgeom.m:18-61) */
    double *pg = calloc((size_t)ngv * nd, sizeof(double));
    double *Jg = calloc((size_t)ngv * nd * nd, sizeof(double));   /* Jg[g,k,m] = dx_m/dxi_k */
    double *jac = calloc(ngv, sizeof(double));
    double *Xx = calloc((size_t)ngv * nd * nd, sizeof(double));   /* Xx[g,i,j] */
    for (int g = 0; g < ngv; g++) {
        for (int m = 0; m < nd; m++) {
            double s = 0.0;
            for (int n = 0; n < npv; n++) s += ms->shapmv[IX3(g, n, 0, ngv, npv)] * dg[IX2(n, m, npv)];
            pg[IX2(g, m, ngv)] = s;
            for (int k = 0; k < nd; k++) {
                double t = 0.0;
                for (int n = 0; n < npv; n++) t += ms->shapmv[IX3(g, n, k + 1, ngv, npv)] * dg[IX2(n, m, npv)];
                Jg[IX3(g, k, m, ngv, nd)] = t;
            }
        }
#define J(k, m) Jg[IX3(g, (k) - 1, (m) - 1, ngv, nd)]
#define X(i, j) Xx[IX3(g, (i) - 1, (j) - 1, ngv, nd)]
        if (nd == 2) {
            jac[g] = J(1, 1) * J(2, 2) - J(1, 2) * J(2, 1);
            X(1, 1) = J(2, 2); X(2, 1) = -J(2, 1); X(1, 2) = -J(1, 2); X(2, 2) = J(1, 1);
        } else {
            jac[g] = J(1, 1) * J(2, 2) * J(3, 3) - J(1, 1) * J(3, 2) * J(2, 3) + J(2, 1) * J(3, 2) * J(1, 3)
                   - J(2, 1) * J(1, 2) * J(3, 3) + J(3, 1) * J(1, 2) * J(2, 3) - J(3, 1) * J(2, 2) * J(1, 3);
            X(1, 1) = J(2, 2) * J(3, 3) - J(2, 3) * J(3, 2);
            X(2, 1) = J(2, 3) * J(3, 1) - J(2, 1) * J(3, 3);
            X(3, 1) = J(2, 1) * J(3, 2) - J(2, 2) * J(3, 1);
            X(1, 2) = J(1, 3) * J(3, 2) - J(1, 2) * J(3, 3);
            X(2, 2) = J(1, 1) * J(3, 3) - J(1, 3) * J(3, 1);
            X(3, 2) = J(1, 2) * J(3, 1) - J(1, 1) * J(3, 2);
            X(1, 3) = J(1, 2) * J(2, 3) - J(1, 3) * J(2, 2);
            X(2, 3) = J(1, 3) * J(2, 1) - J(1, 1) * J(2, 3);
            X(3, 3) = J(1, 1) * J(2, 2) - J(1, 2) * J(2, 1);
        }
#undef J
#undef X
    }

    /* ---- solution at volume Gauss points (volint.m:31-33) */
    double *ug = calloc((size_t)ngv * nc, sizeof(double));
    for (int c = 0; c < nc; c++)
        for (int g = 0; g < ngv; g++) {
            double s = 0.0;
            for (int n = 0; n < npv; n++) s += ms->shapvt[IX3(g, n, 0, ngv, npv)] * udg[IX2(n, c, npv)];
            ug[IX2(g, c, ngv)] = s;
        }

    /* ---- M, C, Rq (volint.m:43-60) */
    if (ap->localsolve) {
        for (int s = 0; s < npv; s++)
            for (int r = 0; r < npv; r++) {
                double t = 0.0;
                for (int g = 0; g < ngv; g++)
                    t += ms->shapvg[IX3(r, g, 0, npv, ngv)] * ms->shapvt[IX3(g, s, 0, ngv, npv)] * jac[g];
                b->M[IX2(r, s, npv)] = fc_q * t;
                for (int i = 0; i < nd; i++) {
                    double c = 0.0;
                    for (int g = 0; g < ngv; g++) {
                        double w = 0.0;
                        for (int j = 0; j < nd; j++)
                            w += ms->shapvg[IX3(r, g, j + 1, npv, ngv)] * Xx[IX3(g, i, j, ngv, nd)];
                        c += w * ms->shapvt[IX3(g, s, 0, ngv, npv)];
                    }
                    b->C[IX3(r, s, i, npv, npv)] = c;
                }
            }
        for (int i = 0; i < nd; i++)
            for (int a = 0; a < ncu; a++)
                for (int r = 0; r < npv; r++) {
                    double t = 0.0;
                    for (int s = 0; s < npv; s++) {
                        int cq = ncu + a + ncu * i;
                        t += b->M[IX2(r, s, npv)] * (sh[IX2(s, cq, npv)] / fc_q - udg[IX2(s, cq, npv)]);
                    }
                    for (int s = 0; s < npv; s++) t += b->C[IX3(r, s, i, npv, npv)] * udg[IX2(s, a, npv)];
                    b->Rq[IX3(r, a, i, npv, ncu)] = t;
                }
    }

    /* ---- flux at Gauss points, Ru and BD (volint.m:81-263) */
    double *f = calloc((size_t)ngv * ncu * nd, sizeof(double));
    double *fu = calloc((size_t)ngv * ncu * nd * nc, sizeof(double));
    orc_flux(nd, ap->param, ngv, ug, f, fu);
    /* wrk_i(g,a) = sum_j f(g,a,j) Xx(g,j,i); wrl_i(g,a,c) = -sum_j f_udg(g,a,j,c) Xx(g,j,i) */
    double *wrk = calloc((size_t)ngv * nd * ncu, sizeof(double));
    double *wrl = calloc((size_t)ngv * nd * ncu * nc, sizeof(double));
    for (int i = 0; i < nd; i++)
        for (int a = 0; a < ncu; a++)
            for (int g = 0; g < ngv; g++) {
                double t = 0.0;
                for (int j = 0; j < nd; j++) t += f[IX3(g, a, j, ngv, ncu)] * Xx[IX3(g, j, i, ngv, nd)];
                wrk[IX3(g, i, a, ngv, nd)] = t;
                for (int c = 0; c < nc; c++) {
                    double l = 0.0;
                    for (int j = 0; j < nd; j++)
                        l += fu[g + (size_t)ngv * (a + ncu * (j + nd * c))] * Xx[IX3(g, j, i, ngv, nd)];
                    wrl[g + (size_t)ngv * (i + nd * (a + (size_t)ncu * c))] = -l;
                }
            }
    for (int a = 0; a < ncu; a++)
        for (int r = 0; r < npv; r++) {
            double t = 0.0;
            for (int i = 0; i < nd; i++)
                for (int g = 0; g < ngv; g++)
                    t += ms->shapvg[IX3(r, g, i + 1, npv, ngv)] * wrk[IX3(g, i, a, ngv, nd)];
            b->Ru[IX2(r, a, npv)] = t;
        }
    /* time-dependent source (volint.m:180-221): s(g,a) = Stg(g,a) - fc_u u(g,a) with Stg the
     * u part of SH at the Gauss points; Ru += shapvg(:,:,1) (s jac) (volint.m:241,258) */
    if (ap->tdep) {
        for (int a = 0; a < ncu; a++)
            for (int r = 0; r < npv; r++) {
                double t = 0.0;
                for (int g = 0; g < ngv; g++) {
                    double st = 0.0;
                    for (int s = 0; s < npv; s++) st += ms->shapvt[IX3(g, s, 0, ngv, npv)] * sh[IX2(s, a, npv)];
                    t += ms->shapvg[IX3(r, g, 0, npv, ngv)] * ((st - ug[IX2(g, a, ngv)] * ap->fc_u) * jac[g]);
                }
                b->Ru[IX2(r, a, npv)] += t;
            }
    }
    /* BD[r,a,s,c] = sum_g sum_i shapvg(r,g,i+1) shapvl(s,g) wrl_i(g,a,c) */
    for (int c = 0; c < nc; c++)
        for (int s = 0; s < npv; s++)
            for (int a = 0; a < ncu; a++)
                for (int r = 0; r < npv; r++) {
                    double t = 0.0;
                    for (int g = 0; g < ngv; g++) {
                        double w = 0.0;
                        for (int i = 0; i < nd; i++)
                            w += ms->shapvg[IX3(r, g, i + 1, npv, ngv)] * wrl[g + (size_t)ngv * (i + nd * (a + (size_t)ncu * c))];
                        t += w * ms->shapvt[IX3(g, s, 0, ngv, npv)];
                    }
                    b->BD[r + (size_t)npv * (a + (size_t)ncu * (s + (size_t)npv * c))] = t;
                }
    /* ... and its Jacobian: wrl(1:ngv, a, a) = fc_u jac, so BD[r,a,s,a] += fc_u sum_g phi_r phi_s w_g jac_g */
    if (ap->tdep)
        for (int a = 0; a < ncu; a++)
            for (int s = 0; s < npv; s++)
                for (int r = 0; r < npv; r++) {
                    double t = 0.0;
                    for (int g = 0; g < ngv; g++)
                        t += ms->shapvg[IX3(r, g, 0, npv, ngv)] * ms->shapvt[IX3(g, s, 0, ngv, npv)] * jac[g];
                    b->BD[r + (size_t)npv * (a + (size_t)ncu * (s + (size_t)npv * a))] += ap->fc_u * t;
                }

    /* ---- facegeom (facegeom.m:20-52): per face j, ngf points */
    const int ngt = ngf * nfe;
    double *fpg = calloc((size_t)ngt * nd, sizeof(double));
    double *nl = calloc((size_t)ngt * nd, sizeof(double));
    double *fjac = calloc(ngt, sizeof(double));
    for (int j = 0; j < nfe; j++)
        for (int g = 0; g < ngf; g++) {
            int gg = g + ngf * j;
            double dpg[3][2] = {{0}};
            for (int m = 0; m < nd; m++) {
                double s = 0.0;
                for (int n = 0; n < npf; n++) {
                    int vn = ms->perm[IX2(n, j, npf)] - 1;
                    s += ms->shapmf[IX3(g, n, 0, ngf, npf)] * dg[IX2(vn, m, npv)];
                    for (int k = 0; k < nd - 1; k++)
                        dpg[m][k] += ms->shapmf[IX3(g, n, k + 1, ngf, npf)] * dg[IX2(vn, m, npv)];
                }
                fpg[IX2(gg, m, ngt)] = s;
            }
            if (nd == 2) {
                double jc = sqrt(dpg[0][0] * dpg[0][0] + dpg[1][0] * dpg[1][0]);
                fjac[gg] = jc;
                nl[IX2(gg, 0, ngt)] = dpg[1][0] / jc;
                nl[IX2(gg, 1, ngt)] = -dpg[0][0] / jc;
            } else {
                double n0 = dpg[1][0] * dpg[2][1] - dpg[2][0] * dpg[1][1];
                double n1 = dpg[2][0] * dpg[0][1] - dpg[0][0] * dpg[2][1];
                double n2 = dpg[0][0] * dpg[1][1] - dpg[1][0] * dpg[0][1];
                double jc = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
                fjac[gg] = jc;
                nl[IX2(gg, 0, ngt)] = n0 / jc;
                nl[IX2(gg, 1, ngt)] = n1 / jc;
                nl[IX2(gg, 2, ngt)] = n2 / jc;
            }
        }

    /* ---- E and Rq -= E.UH (faceint.m:37-51) */
    if (ap->localsolve) {
        for (int i = 0; i < nd; i++)
            for (int j = 0; j < nfe; j++)
                for (int n = 0; n < npf; n++)
                    for (int m = 0; m < npf; m++) {
                        double t = 0.0;
                        for (int g = 0; g < ngf; g++) {
                            int gg = g + ngf * j;
                            t += ms->shapfg[IX3(m, g, 0, npf, ngf)] * ms->shapft[IX3(g, n, 0, ngf, npf)]
                               * nl[IX2(gg, i, ngt)] * fjac[gg];
                        }
                        int r = ms->perm[IX2(m, j, npf)] - 1;
                        b->E[IX3(r, n + npf * j, i, npv, ndf)] = t;
                    }
        for (int i = 0; i < nd; i++)
            for (int a = 0; a < ncu; a++)
                for (int r = 0; r < npv; r++) {
                    double t = 0.0;
                    for (int fi = 0; fi < ndf; fi++) t += b->E[IX3(r, fi, i, npv, ndf)] * uh[IX2(a, fi, ncu)];
                    b->Rq[IX3(r, a, i, npv, ncu)] -= t;
                }
    }

    /* ---- traces at face Gauss points, fhat (faceint.m:55-74) */
    double *fug = calloc((size_t)ngt * nc, sizeof(double));
    double *fuh = calloc((size_t)ngt * ncu, sizeof(double));
    for (int j = 0; j < nfe; j++)
        for (int g = 0; g < ngf; g++) {
            int gg = g + ngf * j;
            for (int c = 0; c < nc; c++) {
                double s = 0.0;
                for (int n = 0; n < npf; n++)
                    s += ms->shapft[IX3(g, n, 0, ngf, npf)] * udg[IX2(ms->perm[IX2(n, j, npf)] - 1, c, npv)];
                fug[IX2(gg, c, ngt)] = s;
            }
            for (int a = 0; a < ncu; a++) {
                double s = 0.0;
                for (int n = 0; n < npf; n++) s += ms->shapft[IX3(g, n, 0, ngf, npf)] * uh[IX2(a, n + npf * j, ncu)];
                fuh[IX2(gg, a, ngt)] = s;
            }
        }
    double *FH = calloc((size_t)ngt * ncu, sizeof(double));
    double *FHu = calloc((size_t)ngt * ncu * nc, sizeof(double));
    double *FHh = calloc((size_t)ngt * ncu * ncu, sizeof(double));
    orc_fhat(nd, ap->param, ngt, nl, fug, fuh, FH, FHu, FHh);
    /* boundary values (faceint.m:171-268); computed per face with that face's points */
    double *BH = calloc((size_t)ngt * ncu, sizeof(double));
    double *BHu = calloc((size_t)ngt * ncu * nc, sizeof(double));
    double *BHh = calloc((size_t)ngt * ncu * ncu, sizeof(double));
    {
        double *tn = calloc((size_t)ngf * nd, sizeof(double)), *tu = calloc((size_t)ngf * nc, sizeof(double));
        double *th = calloc((size_t)ngf * ncu, sizeof(double)), *o1 = calloc((size_t)ngf * ncu, sizeof(double));
        double *o2 = calloc((size_t)ngf * ncu * nc, sizeof(double)), *o3 = calloc((size_t)ngf * ncu * ncu, sizeof(double));
        for (int j = 0; j < nfe; j++) {
            if (bf[j] >= 0) continue;
            int ibn = -bf[j] - 1;
            if (ibn >= ap->nbnd) { rc = -2; continue; }
            double ui[5];
            for (int a = 0; a < ncu; a++) ui[a] = ap->bcs[IX2(ibn, a, ap->nbnd)];
            for (int g = 0; g < ngf; g++) {
                int gg = g + ngf * j;
                for (int d = 0; d < nd; d++) tn[IX2(g, d, ngf)] = nl[IX2(gg, d, ngt)];
                for (int c = 0; c < nc; c++) tu[IX2(g, c, ngf)] = fug[IX2(gg, c, ngt)];
                for (int a = 0; a < ncu; a++) th[IX2(g, a, ngf)] = fuh[IX2(gg, a, ngt)];
            }
            if (orc_fbou(ap->fbou_family, nd, ap->bcm[ibn], ui, ap->param, ngf, tn, tu, th, o1, o2, o3)) { rc = -3; continue; }
            for (int g = 0; g < ngf; g++) {
                int gg = g + ngf * j;
                for (int a = 0; a < ncu; a++) {
                    BH[IX2(gg, a, ngt)] = o1[IX2(g, a, ngf)];
                    for (int c = 0; c < nc; c++) BHu[IX3(gg, a, c, ngt, ncu)] = o2[IX3(g, a, c, ngf, ncu)];
                    for (int c = 0; c < ncu; c++) BHh[IX3(gg, a, c, ngt, ncu)] = o3[IX3(g, a, c, ngf, ncu)];
                }
            }
        }
        free(tn); free(tu); free(th); free(o1); free(o2); free(o3);
    }

    /* ---- face residuals / Jacobians and the perm scatter (faceint.m:306-360) */
    for (int j = 0; j < nfe; j++) {
        int isb = bf[j] < 0;
        for (int m = 0; m < npf; m++) {
            int r = ms->perm[IX2(m, j, npf)] - 1;
            for (int a = 0; a < ncu; a++) {
                double t = 0.0, tb = 0.0;
                for (int g = 0; g < ngf; g++) {
                    int gg = g + ngf * j;
                    double w = ms->shapfg[IX3(m, g, 0, npf, ngf)] * fjac[gg];
                    t += w * FH[IX2(gg, a, ngt)];
                    tb += w * BH[IX2(gg, a, ngt)];
                }
                b->Ru[IX2(r, a, npv)] -= t;
                b->Rh[IX2(a, m + npf * j, ncu)] = -(isb ? tb : t);
            }
            for (int n = 0; n < npf; n++) {
                int s = ms->perm[IX2(n, j, npf)] - 1;
                for (int a = 0; a < ncu; a++) {
                    for (int c = 0; c < nc; c++) {
                        double t = 0.0, tb = 0.0;
                        for (int g = 0; g < ngf; g++) {
                            int gg = g + ngf * j;
                            double w = ms->shapfg[IX3(m, g, 0, npf, ngf)] * ms->shapft[IX3(g, n, 0, ngf, npf)] * fjac[gg];
                            t += w * FHu[IX3(gg, a, c, ngt, ncu)];
                            tb += w * BHu[IX3(gg, a, c, ngt, ncu)];
                        }
                        /* BD(perm(m), a, perm(n), c) += BDn(m,n) */
                        b->BD[r + (size_t)npv * (a + (size_t)ncu * (s + (size_t)npv * c))] += t;
                        /* GK(a, (n,j), perm(m), c) = Gt(m, n) */
                        b->GK[a + (size_t)ncu * ((n + npf * j) + (size_t)ndf * (r + (size_t)npv * c))] += isb ? tb : t;
                    }
                    for (int c = 0; c < ncu; c++) {
                        double t = 0.0, tb = 0.0;
                        for (int g = 0; g < ngf; g++) {
                            int gg = g + ngf * j;
                            double w = ms->shapfg[IX3(m, g, 0, npf, ngf)] * ms->shapft[IX3(g, n, 0, ngf, npf)] * fjac[gg];
                            t += w * FHh[IX3(gg, a, c, ngt, ncu)];
                            tb += w * BHh[IX3(gg, a, c, ngt, ncu)];
                        }
                        /* F(perm(m), a, c, (n,j)) += Fn(m,n) */
                        b->F[r + (size_t)npv * (a + (size_t)ncu * (c + (size_t)ncu * (n + npf * j)))] += t;
                        /* H(a, (m,j), c, (n,j)) = Ht(m,n) */
                        b->H[a + (size_t)ncu * ((m + npf * j) + (size_t)ndf * (c + (size_t)ncu * (n + npf * j)))] += isb ? tb : t;
                    }
                }
            }
        }
    }
    free(pg); free(Jg); free(jac); free(Xx); free(ug); free(f); free(fu); free(wrk); free(wrl);
    free(fpg); free(nl); free(fjac); free(fug); free(fuh); free(FH); free(FHu); free(FHh);
    free(BH); free(BHu); free(BHh);
    return rc;
}

/* schur_uq2 (schur_primal.m:52-150) for one element; dudg[npv,nc], dudg_duh[npv,nc,ncu,ndf]. */
static int schur_uq_elem(int nd, int npv, int ncu, int ndf, const orc_blocks *b,
                         double *dudg, double *dudg_duh, double *ae, double *fe)
{
    const int nc = ncu * (nd + 1), nu = npv * ncu, nh = ncu * ndf;
    int rc = 0;
    int *piv = malloc(sizeof(int) * (nu > npv ? nu : npv));
    /* Mi = inv(M) */
    double *Mlu = malloc(sizeof(double) * npv * npv), *Mi = calloc((size_t)npv * npv, sizeof(double));
    memcpy(Mlu, b->M, sizeof(double) * npv * npv);
    if (lu_factor(Mlu, npv, piv)) rc = 1;
    for (int i = 0; i < npv; i++) Mi[IX2(i, i, npv)] = 1.0;
    lu_solve(Mlu, npv, piv, Mi, npv);
    /* MiRq[npv, ncu*nd], MiC[npv,npv,nd], MiE[npv,ndf,nd] */
    double *MiRq = calloc((size_t)npv * ncu * nd, sizeof(double));
    double *MiC = calloc((size_t)npv * npv * nd, sizeof(double));
    double *MiE = calloc((size_t)npv * ndf * nd, sizeof(double));
    gemm(npv, ncu * nd, npv, Mi, npv, b->Rq, npv, MiRq, npv, 0.0);
    for (int d = 0; d < nd; d++) {
        gemm(npv, npv, npv, Mi, npv, b->C + (size_t)npv * npv * d, npv, MiC + (size_t)npv * npv * d, npv, 0.0);
        gemm(npv, ndf, npv, Mi, npv, b->E + (size_t)npv * ndf * d, npv, MiE + (size_t)npv * ndf * d, npv, 0.0);
    }
    /* B(i,a,j,b,d) = BD(i,a,j, ncu + b + ncu*d) */
    const double *D = b->BD, *B = b->BD + (size_t)nu * nu;
    double *SD = malloc(sizeof(double) * nu * nu);
    double *rhs = calloc((size_t)nu * (1 + nh), sizeof(double));
    /* BMiR = B(:, :) * MiRq(:) */
    for (int ia = 0; ia < nu; ia++) {
        double t = 0.0;
        for (int k = 0; k < nu * nd; k++) t += B[ia + (size_t)nu * k] * MiRq[k];
        rhs[ia] = b->Ru[ia] - t;
    }
    /* SD(ia, (k,bb)) = D + sum_{j,d} B(ia, j, bb, d) MiC(j, k, d) */
    memcpy(SD, D, sizeof(double) * nu * nu);
    for (int bb = 0; bb < ncu; bb++)
        for (int d = 0; d < nd; d++) {
            const double *Bbd = B + (size_t)nu * npv * (bb + ncu * d);   /* [nu, npv] */
            gemm(nu, npv, npv, Bbd, nu, MiC + (size_t)npv * npv * d, npv, SD + (size_t)nu * npv * bb, nu, 1.0);
            /* BMiE(ia, bb, f) = sum B(ia,j,bb,d) MiE(j,f,d) -> rhs column 1 + bb + ncu*f */
            for (int fidx = 0; fidx < ndf; fidx++) {
                double *col = rhs + (size_t)nu * (1 + bb + ncu * fidx);
                for (int jn = 0; jn < npv; jn++) {
                    double me = MiE[IX3(jn, fidx, d, npv, ndf)];
                    if (me == 0.0) continue;
                    for (int ia = 0; ia < nu; ia++) col[ia] += Bbd[ia + (size_t)nu * jn] * me;
                }
            }
        }
    for (int k = 0; k < nh; k++)
        for (int ia = 0; ia < nu; ia++) rhs[ia + (size_t)nu * (1 + k)] -= b->F[ia + (size_t)nu * k];
    if (lu_factor(SD, nu, piv)) rc = 2;
    lu_solve(SD, nu, piv, rhs, 1 + nh);
    const double *du = rhs, *dlu = rhs + nu;
    /* DUDG = [du, MiRq + MiC du] */
    for (int i = 0; i < nu; i++) dudg[i] = du[i];
    for (int d = 0; d < nd; d++)
        for (int a = 0; a < ncu; a++)
            for (int r = 0; r < npv; r++) {
                double t = MiRq[r + (size_t)npv * (a + ncu * d)];
                for (int s = 0; s < npv; s++) t += MiC[IX3(r, s, d, npv, npv)] * du[s + (size_t)npv * a];
                dudg[r + (size_t)npv * (ncu + a + ncu * d)] = t;
            }
    /* DUDG_DUH[npv, nc, ncu, ndf]: u part = dlu; q part = MiC dlu - MiE (x) I */
    for (int k = 0; k < nh; k++) {
        int bb = k % ncu, fidx = k / ncu;
        for (int a = 0; a < ncu; a++)
            for (int r = 0; r < npv; r++)
                dudg_duh[r + (size_t)npv * (a + (size_t)nc * k)] = dlu[r + (size_t)npv * a + (size_t)nu * k];
        for (int d = 0; d < nd; d++)
            for (int a = 0; a < ncu; a++)
                for (int r = 0; r < npv; r++) {
                    double t = 0.0;
                    for (int s = 0; s < npv; s++) t += MiC[IX3(r, s, d, npv, npv)] * dlu[s + (size_t)npv * a + (size_t)nu * k];
                    if (a == bb) t -= MiE[IX3(r, fidx, d, npv, ndf)];
                    dudg_duh[r + (size_t)npv * ((ncu + a + ncu * d) + (size_t)nc * k)] = t;
                }
    }
    /* FE = Rh - GK DUDG ; AE = H + GK DUDG_DUH */
    const int nq = npv * nc;
    for (int i = 0; i < nh; i++) {
        double t = 0.0;
        for (int k = 0; k < nq; k++) t += b->GK[i + (size_t)nh * k] * dudg[k];
        fe[i] = b->Rh[i] - t;
    }
    memcpy(ae, b->H, sizeof(double) * nh * nh);
    gemm(nh, nh, nq, b->GK, nh, dudg_duh, nq, ae, nh, 1.0);
    free(piv); free(Mlu); free(Mi); free(MiRq); free(MiC); free(MiE); free(SD); free(rhs);
    return rc;
}

/* schur_u2 (schur_primal.m:13-49) for one element: SD = D, no q. */
static int schur_u_elem(int nd, int npv, int ncu, int ndf, const orc_blocks *b, int nc,
                        double *dudg, double *dudg_duh, double *ae, double *fe)
{
    const int nu = npv * ncu, nh = ncu * ndf;
    int rc = 0;
    int *piv = malloc(sizeof(int) * nu);
    double *SD = malloc(sizeof(double) * nu * nu);
    double *rhs = malloc(sizeof(double) * nu * (1 + nh));
    memcpy(SD, b->BD, sizeof(double) * nu * nu);
    for (int i = 0; i < nu; i++) rhs[i] = b->Ru[i];
    for (int k = 0; k < nu * nh; k++) rhs[nu + k] = -b->F[k];
    if (lu_factor(SD, nu, piv)) rc = 2;
    lu_solve(SD, nu, piv, rhs, 1 + nh);
    /* DUDG[npv, nc] with only the first ncu columns set; DUDG_DUH[npv, nc, ncu, ndf] likewise */
    for (int i = 0; i < npv * nc; i++) dudg[i] = 0.0;
    for (int i = 0; i < nu; i++) dudg[i] = rhs[i];
    for (int k = 0; k < nh; k++) {
        for (int i = 0; i < npv * nc; i++) dudg_duh[i + (size_t)npv * nc * k] = 0.0;
        for (int i = 0; i < nu; i++) dudg_duh[i + (size_t)npv * nc * k] = rhs[nu + (size_t)nu * k + i];
    }
    const int nq = npv * nc;
    for (int i = 0; i < nh; i++) {
        double t = 0.0;
        for (int k = 0; k < nq; k++) t += b->GK[i + (size_t)nh * k] * dudg[k];
        fe[i] = b->Rh[i] - t;
    }
    memcpy(ae, b->H, sizeof(double) * nh * nh);
    gemm(nh, nh, nq, b->GK, nh, dudg_duh, nq, ae, nh, 1.0);
    free(piv); free(SD); free(rhs);
    return rc;
}

/* ------------------------------------------------------------------ exports */
/* hdg_elemental (kernel/hdg_elemental.m:1-203) on ne elements.  Any of the intermediate
 * outputs (M..Rh) may be NULL.  status[ne] (optional) gets per-element codes. */
typedef struct {
    const orc_master *ms; const orc_app *ap; size_t nbd;
    const double *dgnodes, *UDG, *UH, *SH; const int *bf;
    double *AE, *FE, *DUDG, *DUDG_DUH, *Mo, *Co, *Eo, *BDo, *Fo, *GKo, *Ho, *Rqo, *Ruo, *Rho;
    int *status;
} elem_ctx;

static void elem_body(void *vctx, int e, int *nbad)
{
    elem_ctx *x = vctx;
    const orc_master *ms = x->ms; const orc_app *ap = x->ap;
    const int nd = ms->nd, npv = ms->npv, ndf = ms->npf * ms->nfe, ncu = ap->ncu, nc = ap->nc;
    double *buf = malloc(sizeof(double) * x->nbd);
    orc_blocks b;
    blocks_carve(ms, ap, buf, &b);
    int rc = element_blocks(ms, ap, x->dgnodes + (size_t)npv * nd * e, x->bf + (size_t)ms->nfe * e,
                            x->UDG + (size_t)npv * nc * e, x->UH + (size_t)ncu * ndf * e,
                            x->SH + (size_t)npv * nc * e, &b);
    if (x->Mo)  memcpy(x->Mo + (size_t)npv * npv * e, b.M, sizeof(double) * npv * npv);
    if (x->Co)  memcpy(x->Co + (size_t)npv * npv * nd * e, b.C, sizeof(double) * npv * npv * nd);
    if (x->Eo)  memcpy(x->Eo + (size_t)npv * ndf * nd * e, b.E, sizeof(double) * npv * ndf * nd);
    if (x->BDo) memcpy(x->BDo + (size_t)npv * ncu * npv * nc * e, b.BD, sizeof(double) * npv * ncu * npv * nc);
    if (x->Fo)  memcpy(x->Fo + (size_t)npv * ncu * ncu * ndf * e, b.F, sizeof(double) * npv * ncu * ncu * ndf);
    if (x->GKo) memcpy(x->GKo + (size_t)ncu * ndf * npv * nc * e, b.GK, sizeof(double) * ncu * ndf * npv * nc);
    if (x->Ho)  memcpy(x->Ho + (size_t)ncu * ndf * ncu * ndf * e, b.H, sizeof(double) * ncu * ndf * ncu * ndf);
    if (x->Rqo) memcpy(x->Rqo + (size_t)npv * ncu * nd * e, b.Rq, sizeof(double) * npv * ncu * nd);
    if (x->Ruo) memcpy(x->Ruo + (size_t)npv * ncu * e, b.Ru, sizeof(double) * npv * ncu);
    if (x->Rho) memcpy(x->Rho + (size_t)ncu * ndf * e, b.Rh, sizeof(double) * ncu * ndf);
    if (rc == 0 && x->AE) {
        if (ap->localsolve)
            rc = schur_uq_elem(nd, npv, ncu, ndf, &b, x->DUDG + (size_t)npv * nc * e,
                               x->DUDG_DUH + (size_t)npv * nc * ncu * ndf * e,
                               x->AE + (size_t)ncu * ndf * ncu * ndf * e, x->FE + (size_t)ncu * ndf * e);
        else
            rc = schur_u_elem(nd, npv, ncu, ndf, &b, nc, x->DUDG + (size_t)npv * nc * e,
                              x->DUDG_DUH + (size_t)npv * nc * ncu * ndf * e,
                              x->AE + (size_t)ncu * ndf * ncu * ndf * e, x->FE + (size_t)ncu * ndf * e);
    }
    if (x->status) x->status[e] = rc;
    if (rc) (*nbad)++;
    free(buf);
}

int orc_hdg_elemental(const orc_master *ms, const orc_app *ap, int ne,
                      const double *dgnodes, const int *bf, const double *UDG, const double *UH,
                      const double *SH, double *AE, double *FE, double *DUDG, double *DUDG_DUH,
                      double *Mo, double *Co, double *Eo, double *BDo, double *Fo, double *GKo,
                      double *Ho, double *Rqo, double *Ruo, double *Rho, int *status, int nthreads)
{
    elem_ctx x = {ms, ap, blocks_doubles(ms, ap), dgnodes, UDG, UH, SH, bf, AE, FE, DUDG, DUDG_DUH,
                  Mo, Co, Eo, BDo, Fo, GKo, Ho, Rqo, Ruo, Rho, status};
    return orc_run(ne, nthreads, elem_body, &x);
}

/* schur_uq2 on reference-layout inputs (the MEX signature of kernel/schur_uq.c:202-252). */
typedef struct {
    int nd, npv, ncu, ndf;
    const double *M, *C, *E, *BD, *F, *GK, *H, *Rq, *Ru, *Rh;
    double *DUDG, *DUDG_DUH, *AE, *FE;
} schur_ctx;

static void schur_body(void *vctx, int e, int *nbad)
{
    schur_ctx *x = vctx;
    const int nd = x->nd, npv = x->npv, ncu = x->ncu, ndf = x->ndf;
    const int nc = ncu * (nd + 1), nh = ncu * ndf;
    orc_blocks b;
    b.M = (double *)x->M + (size_t)npv * npv * e;
    b.C = (double *)x->C + (size_t)npv * npv * nd * e;
    b.E = (double *)x->E + (size_t)npv * ndf * nd * e;
    b.BD = (double *)x->BD + (size_t)npv * ncu * npv * nc * e;
    b.F = (double *)x->F + (size_t)npv * ncu * nh * e;
    b.GK = (double *)x->GK + (size_t)nh * npv * nc * e;
    b.H = (double *)x->H + (size_t)nh * nh * e;
    b.Rq = (double *)x->Rq + (size_t)npv * ncu * nd * e;
    b.Ru = (double *)x->Ru + (size_t)npv * ncu * e;
    b.Rh = (double *)x->Rh + (size_t)nh * e;
    *nbad += schur_uq_elem(nd, npv, ncu, ndf, &b, x->DUDG + (size_t)npv * nc * e,
                           x->DUDG_DUH + (size_t)npv * nc * nh * e, x->AE + (size_t)nh * nh * e,
                           x->FE + (size_t)nh * e) != 0;
}

int orc_schur_uq(int nd, int npv, int ncu, int ndf, int ne,
                 const double *M, const double *C, const double *E, const double *BD, const double *F,
                 const double *GK, const double *H, const double *Rq, const double *Ru, const double *Rh,
                 double *DUDG, double *DUDG_DUH, double *AE, double *FE, int nthreads)
{
    schur_ctx x = {nd, npv, ncu, ndf, M, C, E, BD, F, GK, H, Rq, Ru, Rh, DUDG, DUDG_DUH, AE, FE};
    return orc_run(ne, nthreads, schur_body, &x);
}

/* Point physics, exported for pinning against the reference's generated C kernels. */
void orc_flux_points(int nd, const double *param, int ng, const double *udg, double *f, double *f_udg)
{ orc_flux(nd, param, ng, udg, f, f_udg); }

void orc_fhat_points(int nd, const double *param, int ng, const double *nl, const double *udg,
                     const double *uh, double *fh, double *fh_udg, double *fh_uh)
{ orc_fhat(nd, param, ng, nl, udg, uh, fh, fh_udg, fh_uh); }

int orc_fbou_points(int fam, int nd, int ib, const double *uinf, const double *param, int ng, const double *nl,
                    const double *udg, const double *uh, double *fh, double *fh_udg, double *fh_uh)
{ return orc_fbou(fam, nd, ib, uinf, param, ng, nl, udg, uh, fh, fh_udg, fh_uh); }

/* An[ng, ncu, ncu] and its derivative Anm[ng, ncu, ncu, ncu] (last index: the uh component) of
 * the Roe matrices at the states uh[ng, ncu] (getan.m absolute 0 or 1), for the fixture pins. */
void orc_getan_points(int nd, const double *param, int absolute, int ng, const double *nl, const double *uh,
                      double *An, double *Anm)
{
    const int ncu = nd + 2;
    for (int g = 0; g < ng; g++) {
        double n1[3];
        odual m[5], A[25];
        for (int d = 0; d < nd; d++) n1[d] = nl[g + ng * d];
        for (int c = 0; c < ncu; c++) m[c] = od_var(uh[g + ng * c], c, ncu);
        orc_getan_roe(nd, param, n1, m, absolute, ncu, A);
        for (int k = 0; k < ncu * ncu; k++) {
            An[g + ng * k] = A[k].v;
            for (int c = 0; c < ncu; c++) Anm[g + ng * (k + ncu * ncu * c)] = A[k].d[c];
        }
    }
}
